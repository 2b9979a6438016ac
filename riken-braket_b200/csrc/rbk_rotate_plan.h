// rbk_rotate_plan.h -- host planning of the adjoint sweep's pair-rotate
// launches (rbk::launch_pair_rotate): which tile bits each launch takes, its
// register phases, and the per-gate records.  Plain C++ on the host; the C ABI
// launches what it returns, and tests/host/rotate_check.cpp runs it through a
// CPU model of the kernel.
#pragma once

#include <cstdint>
#include <vector>

#include "rbk_kernels.h"

namespace rbk {

// One gate of a run of one-qubit gates, on its physical bit: the 2x2 matrix
// (m00 m01 m10 m11 as (re, im)) applied to both states and, for a rotation,
// its X / Y-type overlap spec and result slot (slot < 0: no overlap).
struct rotate_item {
  int bit;
  int slot;
  overlap_spec spec;
  double m[8];
};

// The launches that apply `items` (distinct bits) to two states of n qubits,
// up to 11 gates a launch (the low 3 physical bits plus 8 more per tile).  With
// `owed`, the first launch also applies that diagonal and takes its Z-type
// overlaps (pre_diag's g, u, adj, full and z entries are used; the per-layout
// fields are filled here).
std::vector<pair_rotate_set> plan_rotations(int n, const std::vector<rotate_item>& items, const pre_diag* owed);

}  // namespace rbk
