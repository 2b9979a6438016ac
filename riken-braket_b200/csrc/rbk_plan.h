// rbk_plan.h -- host-side fusion planner: queued gates -> fused tile passes.
#pragma once

#include <cstdint>
#include <vector>

#include "rbk_internal.h"

namespace rbk {

// A queued gate in LOGICAL qubits.  kind is an op_kind, or HK_SWAP for an
// uncontrolled SWAP, which only relabels the layout map.
constexpr uint8_t HK_SWAP = 100;

struct hgate {
  uint8_t kind;
  int8_t target;     // MAT/X/Y/DIAG target; SWAP: first qubit; -1 for NEG
  int8_t target2;    // SWAP: second qubit
  uint8_t diag_one;  // DIAG with d0 == 1 exactly
  uint64_t cmask;    // controls (NEG: every qubit of the phase flip)
  double m[8];
};

inline bool is_dense(const hgate& g) { return g.kind == OPK_MAT; }

struct plan_params {
  int n;         // state qubits
  int K;         // tile bits
  int R;         // register bits
  int LOW;       // low physical bits that are always tile bits (coalescing)
  int vbits;     // log2 amplitudes per 16-byte vector
  int dense_budget;  // max dense 2x2 gates per pass
  bool fold_x = true;  // fold CNOT / X gates at the end of a phase into its write layout
  bool merge_1q = true;  // merge consecutive uncontrolled single-qubit gates on one qubit
  bool defer_x = true;   // register phases take CNOT / X gates last (so that they fold)
  bool phase_runs = true;  // runs of phase gates behind one PHASES header
  bool layers = true;      // uncontrolled 2x2 gates on distinct register bits behind one LAYER header
  int factored_min = 3;    // layers of at least this many gates take the factored form (0: never)
};

// Plans `gates` (in order) into passes, updating the layout map
// perm (logical -> physical) and inv (physical -> logical).
void plan_passes(const plan_params& p, const std::vector<hgate>& gates, std::vector<int>& perm,
                 std::vector<int>& inv, std::vector<dev_pass>& out);

// Passes that only move data so that perm becomes `target` (a permutation of
// 0..n-1: logical qubit q on physical bit target[q]); the multi-qubit form of
// ket::mpi's swap_permutated_local_qubits
// (ket/include/ket/mpi/utility/detail/swap_permutated_local_qubits.hpp:26-81).
void plan_layout(const plan_params& p, std::vector<int>& perm, std::vector<int>& inv, const std::vector<int>& target,
                 std::vector<dev_pass>& out);
// plan_layout to the identity.
void plan_canonicalize(const plan_params& p, std::vector<int>& perm, std::vector<int>& inv,
                       std::vector<dev_pass>& out);

// Physical form of a gate for the unfused path (states smaller than a tile).
gate_rec to_physical(const hgate& g, const std::vector<int>& perm);

}  // namespace rbk
