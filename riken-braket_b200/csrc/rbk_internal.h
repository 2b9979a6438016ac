// rbk_internal.h -- device-side program format shared by the host planner
// (rbk_plan.cpp) and the CUDA kernels (rbk_kernels.cu).
//
// A "pass" is one read + one write of the whole state vector.  The state is
// cut into tiles of 2^K amplitudes; a tile is the set of amplitudes that share
// the values of the n-K physical bits outside the pass's tile bit set.  Each
// CTA stages one tile in shared memory, moves it into registers in a sequence
// of layouts ("phases"), applies the phase's gates in registers, and writes
// the tile back -- optionally with its tile bits permuted, which is how the
// logical->physical qubit layout map (the single-device use of
// ket::mpi::qubit_permutation, ket/include/ket/mpi/qubit_permutation.hpp:40-302)
// changes without a separate swap pass.
#pragma once

#include <cstdint>

namespace rbk {

// Register tiling per precision.
//   c128 (complex<double>, 16 B): K = 12 tile bits, R = 4 register bits,
//        256 threads, 64 KiB of shared memory per tile.
//   c64  (complex<float>,  8 B):  K = 13 tile bits, R = 5 register bits,
//        256 threads, 64 KiB of shared memory per tile.
template <typename Real> struct tiling;
template <> struct tiling<double> {
  static constexpr int K = 12, R = 4, T = K - R, VEC = 1, LOW = 5, SWZ = 3;
};
template <> struct tiling<float> {
  static constexpr int K = 13, R = 5, T = K - R, VEC = 2, LOW = 6, SWZ = 4;
};

constexpr int kMaxPassOps = 112;
constexpr int kMaxPhases = 16;
constexpr int kMaxQubits = 40;

enum op_kind : uint8_t {
  OPK_MAT = 1,   // 2x2 complex matrix on a register bit (controlled)
  OPK_X = 2,     // swap the two halves of a register bit (controlled)
  OPK_Y = 3,     // (a0, a1) -> (-i a1, i a0) on a register bit (controlled)
  OPK_DIAG = 4,  // amplitude *= (target bit ? d1 : d0) when the controls are all one
  OPK_NEG = 5,   // amplitude *= -1 when the controls are all one (Z, CZ: exact)
};

// One gate inside a pass, in the coordinates of the phase it belongs to.
struct alignas(8) dev_op {
  uint8_t kind;
  uint8_t treg;       // MAT/X/Y: target register bit
  uint8_t diag_one;   // DIAG: d0 == 1 exactly (phase-shift form: only the one-half is touched)
  uint8_t real;       // MAT: all four entries are real (H, exp(i theta Y), ...)
  uint32_t creg;      // controls inside the register bits
  uint32_t cthr;      // controls inside the thread bits
  uint32_t dreg;      // DIAG target bit among the register bits (mask), 0 if elsewhere
  uint32_t dthr;      // DIAG target bit among the thread bits (mask)
  uint32_t pad1;
  uint64_t cout;      // controls on physical bits outside the tile
  uint64_t dout;      // DIAG target on a physical bit outside the tile (mask)
  double m[8];        // MAT: m00 m01 m10 m11 as (re, im); DIAG: d0 d1
};

// One register layout of the tile.  Tile index j of the amplitude held in
// register slot i of thread t:  j = sum_b bit_b(i) << reg_pos[b]  |  sum_b bit_b(t) << thr_pos[b].
// After the phase's gates the registers are written back at positions given by
// wreg_pos / wthr_pos (equal to reg_pos / thr_pos except in the last phase,
// where they carry the pass's relabelling of tile bits).
struct dev_phase {
  uint8_t reg_pos[8];
  uint8_t thr_pos[16];
  uint8_t wreg_pos[8];
  uint8_t wthr_pos[16];
  uint16_t op_begin, op_end;
};

struct dev_pass {
  uint8_t tile_phys[16];      // physical bit of tile bit b
  uint8_t nontile_phys[kMaxQubits];  // physical bits outside the tile, ascending
  uint8_t num_nontile;
  uint8_t num_phases;
  uint8_t direct_load;   // phase 0's layout reads HBM coalesced: load straight into registers
  uint8_t direct_store;  // the last phase's write layout is coalesced: store straight from registers
  uint8_t pad[4];
  dev_phase phases[kMaxPhases];
  dev_op ops[kMaxPassOps];
};

// Per-gate (unfused) program record, used for states smaller than one tile
// and by the unfused execution mode.  Bits are physical.
struct alignas(8) gate_rec {
  uint8_t kind;        // op_kind
  uint8_t target;      // physical target bit (MAT/X/Y/DIAG)
  uint8_t diag_one;
  uint8_t pad;
  uint32_t pad1;
  uint64_t cmask;      // physical control mask
  double m[8];
};

}  // namespace rbk
