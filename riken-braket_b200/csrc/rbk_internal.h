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

// Tile shapes.  A shape fixes the tile bits K (2^K amplitudes per CTA) and
// the register bits R (2^R amplitudes per thread, 2^(K-R) threads); LOW low
// physical bits are always tile bits (512-byte contiguous runs in HBM).
//   shape 0: K = 12 (c128) / 13 (c64), 256 threads, 2 CTAs per SM
//   shape 1: same tile, half the registers per thread, 512 threads (planned
//            on the host only; no kernel is built for it)
//   shape 2: K = 11 (c128) / 12 (c64), 128 threads, 4 CTAs per SM
//   shape 3: the tile of shape 2 in a persistent CTA (3 per SM) that copies
//            its next tile into a second shared-memory buffer with cp.async
//            while it works on the current one
constexpr int kNumShapes = 4;
template <typename Real> struct precision_traits;
template <> struct precision_traits<double> { static constexpr int VEC = 1, VB = 0, LOW = 5; };
template <> struct precision_traits<float> { static constexpr int VEC = 2, VB = 1, LOW = 6; };

template <typename Real, int SHAPE> struct tile_shape;
template <> struct tile_shape<double, 0> { static constexpr int K = 12, R = 4, CTAS = 2; static constexpr bool PIPE = false; };
template <> struct tile_shape<double, 2> { static constexpr int K = 11, R = 4, CTAS = 4; static constexpr bool PIPE = false; };
template <> struct tile_shape<double, 3> { static constexpr int K = 11, R = 4, CTAS = 3; static constexpr bool PIPE = true; };
template <> struct tile_shape<float, 0> { static constexpr int K = 13, R = 5, CTAS = 2; static constexpr bool PIPE = false; };
template <> struct tile_shape<float, 2> { static constexpr int K = 12, R = 5, CTAS = 4; static constexpr bool PIPE = false; };
template <> struct tile_shape<float, 3> { static constexpr int K = 12, R = 5, CTAS = 3; static constexpr bool PIPE = true; };

// Host view of a tile shape: tile bits, register bits (precision 0 = c128, 1 = c64).
inline void shape_bits(int precision, int shape, int* K, int* R)
{
  static const int k128[kNumShapes] = {12, 12, 11, 11}, r128[kNumShapes] = {4, 3, 4, 4};
  static const int k64[kNumShapes] = {13, 13, 12, 12}, r64[kNumShapes] = {5, 4, 5, 5};
  *K = precision == 0 ? k128[shape] : k64[shape];
  *R = precision == 0 ? r128[shape] : r64[shape];
}

constexpr int kMaxPassGates = 112;  // gates the planner puts in one pass
constexpr int kMaxPassOps = 128;    // op records of a pass: the gates plus phase-run and layer headers
constexpr int kMaxPhases = 16;
constexpr int kMaxQubits = 40;

enum op_kind : uint8_t {
  OPK_MAT = 1,   // 2x2 complex matrix on a register bit (controlled)
  OPK_X = 2,     // swap the two halves of a register bit (controlled)
  OPK_Y = 3,     // (a0, a1) -> (-i a1, i a0) on a register bit (controlled)
  OPK_DIAG = 4,  // amplitude *= (target bit ? d1 : d0) when the controls are all one
  OPK_NEG = 5,   // amplitude *= -1 when the controls are all one (Z, CZ: exact)
  OPK_PHASES = 6,  // header of a run of `run` phase ops that follow (DIAG with d0 == 1, NEG)
  OPK_LAYER = 7,   // header of `run` uncontrolled MAT ops that follow, on distinct register bits
                   // (mask dreg) in ascending bit order; applied as one straight-line block
};

// LAYER form 3, the factored layer: each gate M = [[a, b], [c, d]] of the layer is
// written as
//   M = diag(p0, p1) * [[1, t0], [t1, 1]] * diag(1, q),  |q| = 1, t0 and t1 real,
// which exists when a and d are non-zero and b c / (a d) is real (every unitary
// with a != 0).  Register slot i of a thread takes
//   pre(i)  = product over the layer's bits b set in i of q_b        (skipped when every q is 1),
//   post(i) = product over the layer's bits b of (bit b of i ? p1_b : p0_b),
// around the middle factors, which cost four real multiply-adds per amplitude
// pair (fourteen for the general 2x2 form).  Both diagonals are products over
// bits, so each is stored as two factors: lo over register bits 0-1 (4 entries)
// and hi over bits 2..R-1 (2^(R-2) entries), pre(i) = pre_lo[i & 3] pre_hi[i >> 2]
// and the same for post (post_hi[0] = 1: the hi part's constant is moved into
// post_lo).  A full 2^R-entry table took one constant load per amplitude and
// kept the constant-load pipe 70 % busy; a shared-memory copy of it exposed the
// load latency instead.  One table slot per layer holds, in the state's
// precision, pre_lo[4], pre_hi[2^(R-2)], post_lo[4], post_hi[2^(R-2)].  The
// member records hold t0, t1 in m[0], m[1]; the header holds its slot in dthr
// and in diag_one whether the pre factors apply.
constexpr int kLayerFactored = 3;
constexpr int kMaxLayerTabs = 8;
constexpr int kTabDoubles = 32;  // 256 bytes per slot

// Dispatch key of a pass op: MAT ops are keyed by matrix form (0 general,
// 1 real, 2 real m00), by whether register-bit controls exist and by the target
// register bit; X and Y by the target bit; NEG, DIAG and PHASES by kind alone;
// LAYER by the form its matrices are applied in and by whether it covers every
// register bit (passed as `controlled`).
#ifdef __CUDACC__
#define RBK_HOST_DEVICE __host__ __device__
#else
#define RBK_HOST_DEVICE
#endif
// Dense codes 0 .. kNumOpCodes-1 (register bits 0..4), so that the kernel's
// switch over them can be a jump table (LAYER forms 0..3: codes 43..50).
RBK_HOST_DEVICE constexpr uint32_t op_code(int kind, int form, bool controlled, int treg)
{
  return kind == OPK_MAT ? uint32_t((form * 2 + (controlled ? 1 : 0)) * 5 + treg)
       : kind == OPK_X ? 30u + uint32_t(treg)
       : kind == OPK_Y ? 35u + uint32_t(treg)
       : kind == OPK_NEG ? 40u : kind == OPK_DIAG ? 41u : kind == OPK_PHASES ? 42u
       : 43u + uint32_t(form * 2 + (controlled ? 1 : 0));
}
constexpr uint32_t kNumOpCodes = 51;

// One gate inside a pass, in the coordinates of the phase it belongs to.
struct alignas(8) dev_op {
  uint8_t kind;
  uint8_t treg;       // MAT/X/Y: target register bit
  uint8_t diag_one;   // DIAG: d0 == 1 exactly (phase-shift form: only the one-half is touched)
  uint8_t real;       // MAT: 1 = all four entries real (H, exp(i theta Y)); 2 = m00 real (U3, U2); LAYER: the form used
  uint32_t creg;      // controls inside the register bits
  uint32_t cthr;      // controls inside the thread bits
  uint32_t dreg;      // DIAG target bit among the register bits (mask), 0 if elsewhere; LAYER: its register bits
  uint32_t dthr;      // DIAG target bit among the thread bits (mask)
  uint32_t code;      // op_code(kind, form, controlled, treg): the kernel's single dispatch key
  uint32_t run;       // PHASES, LAYER: number of ops that follow and belong to the header
  uint64_t cout;      // controls on physical bits outside the tile
  uint64_t dout;      // DIAG target on a physical bit outside the tile (mask); PHASES: the run's class sizes
  double m[8];        // MAT: m00 m01 m10 m11 as (re, im); DIAG: d0 d1
};

// A CNOT/X folded into the write map of a phase whose control outside the tile
// makes it hold on some tiles only: where (base & cout) == cout the write
// position of register slot i of thread t moves by x when the fold's control
// holds -- always (kind 0), register bit `bit` of i (kind 1), or bit `bit` of t
// (kind 2).  x is a shared-memory slot, or a physical offset when the phase
// stores straight to HBM.  Folds with controls inside the tile only are
// composed into wslot / wtslot (or the store layout) on the host.
constexpr int kMaxFolds = 8;
struct dev_fold {
  uint64_t cout;
  uint64_t x;
  uint8_t kind;
  uint8_t bit;
  uint8_t pad[6];
};

// One register layout of the tile.  Tile index j of the amplitude held in
// register slot i of thread t:  j = sum_b bit_b(i) << reg_pos[b]  |  sum_b bit_b(t) << thr_pos[b].
// After the phase's gates the registers are written back at positions given by
// wreg_pos / wthr_pos (equal to reg_pos / thr_pos except in the last phase,
// where they carry the pass's relabelling of tile bits).  The host also
// precomputes the shared-memory slots of these positions: rslot[b] for
// register bit b, and tslot_lo[t & 15] ^ tslot_hi[t >> 4] for thread t (up to
// 9 thread bits; the slot map is linear, so a thread XORs them together).
// CNOTs and X gates at the end of a phase need not run: the host composes them
// into the write slots (they permute tile indices GF(2)-affinely), and folds[]
// holds those that apply on some tiles only.
struct dev_phase {
  uint16_t rslot[8];
  uint16_t wslot[8];
  uint16_t tslot_lo[16], tslot_hi[32];
  uint16_t wtslot_lo[16], wtslot_hi[32];
  uint8_t reg_pos[8];
  uint8_t thr_pos[16];
  uint8_t wreg_pos[8];
  uint8_t wthr_pos[16];
  uint16_t op_begin, op_end;
  uint8_t num_folds;
  uint8_t pad[3];
  dev_fold folds[kMaxFolds];
};

// Physical offsets of a register layout for direct HBM access: register bit b
// contributes rphys[b], thread t tphys_lo[t & 15] ^ tphys_hi[t >> 4], all
// combined with XOR (folded CNOTs can make contributions share bits).
struct dev_hbm_layout {
  uint64_t rphys[8];
  uint64_t tphys_lo[16], tphys_hi[32];
};

struct dev_pass {
  uint8_t tile_phys[16];      // physical bit of tile bit b
  uint8_t num_runs;           // the block index is deposited into the non-tile bits run by run:
  uint8_t run_src[16];        //   base |= ((block >> run_src) & mask(run_len)) << run_dst
  uint8_t run_len[16];
  uint8_t run_dst[16];
  uint8_t num_phases;
  uint8_t direct_load;   // phase 0's layout reads HBM coalesced: load straight into registers
                         // (1: 16-byte vectors; 2: 8-byte complex<float> amplitudes, lanes on HBM bits 0-4)
  uint8_t direct_store;  // the last phase's write layout is coalesced: store straight from registers (modes as above)
  uint8_t pad[4];
  dev_hbm_layout load, store;
  dev_phase phases[kMaxPhases];
  dev_op ops[kMaxPassOps];
  alignas(16) double tabs[kMaxLayerTabs * kTabDoubles];  // factored layers' diagonal factors (complex<double> or complex<float>)
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
