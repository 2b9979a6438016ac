// rbk_adjoint.h -- the adjoint sweep on reusable state pairs (used by
// rbk_adjoint_gradient and the batch front end).
#pragma once

#include "rbk.h"

namespace rbk {

struct adjoint_workspace;

// psi and lambda of 2^num_qubits amplitudes on one stream, plus scratch.
int adjoint_workspace_create(int num_qubits, int precision, int device, adjoint_workspace** out);
void adjoint_workspace_destroy(adjoint_workspace* w);
// Tile shape (rbk_state_set_tile_shape) of both states' fused passes.
int adjoint_workspace_set_shape(adjoint_workspace* w, int shape);
// rbk_adjoint_gradient on the workspace's states (same arguments and results).
int adjoint_run(adjoint_workspace* w, const rbk_circuit_gate* gates, int num_gates, const double* theta, int num_params,
                int num_terms, const char* strings, const double* coeffs, double* energy, double* grad);

}  // namespace rbk
