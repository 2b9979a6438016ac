// rbk_kernels.h -- host-side launchers of the kernels in rbk_kernels.cu.
#pragma once

#include <cuda_runtime.h>
#include <cstddef>
#include <cstdint>

#include "rbk_internal.h"

namespace rbk {

constexpr int kMaxPauliTerms = 64;

// Pauli strings that share one flip mask, as weights of sign patterns:
//   W(i) = sum_t w_t * (-1)^popcount(i & sign_t)     (physical bits)
struct pauli_terms {
  int count;
  int one_sided;  // 1: only the conj(a_i) a_{i^F} side with bit lowbit(F) of i clear (spin sums)
  uint64_t sign[kMaxPauliTerms];
  double w[kMaxPauliTerms][2];
};

// One fused pass with tile shape `shape` (see tile_shape in rbk_internal.h).
template <typename Real> cudaError_t launch_tile_pass(void* state, int n, const dev_pass& pass, int shape, cudaStream_t stream);
template <typename Real> cudaError_t launch_gate(void* state, int n, const gate_rec& g, cudaStream_t stream);
template <typename Real> cudaError_t launch_set_basis(void* state, int n, uint64_t index, cudaStream_t stream);
// ket::shor_box on a zeroed state: 2^nx amplitudes of value coeff (divisor, base < 2^32).
template <typename Real>
cudaError_t launch_shor_box(void* state, int n, int nx, uint64_t divisor, uint64_t base, double coeff, cudaStream_t stream);

int reduction_blocks();

// Records msg as the calling thread's rbk_last_error() and returns code.
int set_last_error(int code, const char* msg);
// Scratch needed by the reductions below, in doubles.
inline size_t reduction_scratch_doubles() { return size_t(1 << 12) * (1 + kMaxQubits) + 64; }

template <typename Real> cudaError_t launch_zsum(const void* state, int n, double* partials, double* out, cudaStream_t stream);
template <typename Real> cudaError_t launch_pauli(const void* state, int n, uint64_t flip, const pauli_terms& terms,
                                                  double* partials, double* out, cudaStream_t stream);
// <b| sum_t w_t P_t |a> for strings sharing the flip mask `flip`.
template <typename Real> cudaError_t launch_pauli2(const void* a, const void* b, int n, uint64_t flip, const pauli_terms& terms,
                                                   double* partials, double* out, cudaStream_t stream);
template <typename Real> cudaError_t launch_inner(const void* a, const void* b, int n, double* partials, double* out,
                                                  cudaStream_t stream);
template <typename Real> cudaError_t launch_probs(const void* state, uint64_t offset, uint64_t count, double* out,
                                                  cudaStream_t stream);

// A sum of Pauli strings grouped by flip mask, for applying H to a state:
// group g holds terms [begin[g], begin[g+1]).
constexpr int kMaxSumGroups = 64;
constexpr int kMaxSumTerms = 128;
struct pauli_sum {
  int num_groups;
  int pad;
  uint64_t flip[kMaxSumGroups];
  int begin[kMaxSumGroups + 1];
  int pad2;
  uint64_t sign[kMaxSumTerms];
  double w[kMaxSumTerms][2];
};

template <typename Real> cudaError_t launch_pauli_apply(const void* src, void* dst, int n, const pauli_sum& P, cudaStream_t stream);
// The same sum in tiled passes: each pass takes the groups whose flip bits lie
// in one tile layout (the low 3 bits plus up to 8 more), reads src once and
// writes (first pass) or adds to dst; the diagonal group rides in the first
// pass.  Falls back to launch_pauli_apply below 11 qubits or when a group's
// flip does not fit one layout.
template <typename Real> cudaError_t launch_pauli_apply_tiled(const void* src, void* dst, int n, const pauli_sum& P,
                                                              cudaStream_t stream);
// out (device, 2 doubles) = <lam| P |psi> with P = w (-1)^popcount(i & sign) X^flip
template <typename Real> cudaError_t launch_overlap(const void* lam, const void* psi, int n, uint64_t flip, uint64_t sign,
                                                    double wr, double wi, double* partials, double* out, cudaStream_t stream);
// Up to kMaxOverlaps overlaps <lam| P_y |psi> in one launch; out[2y], out[2y+1] = (re, im) of overlap y.
constexpr int kMaxOverlaps = 64;
struct overlap_spec { uint64_t flip, sign; double wr, wi; };
struct overlap_set { int count; int pad; overlap_spec spec[kMaxOverlaps]; };
size_t overlaps_partials_doubles();
template <typename Real> cudaError_t launch_overlaps(const void* lam, const void* psi, int n, const overlap_set& set,
                                                     double* partials, double* out, cudaStream_t stream);
// The same for overlaps whose flip bits are all tile bits of one tile layout:
// each state is read once per launch.  flip_local / sign_local are tile-index
// masks; sign bits outside the tile go in sign (physical); the result of spec y
// goes to out[2 out_slot], out[2 out_slot + 1].  K <= 12.
struct tile_overlap_spec { uint32_t flip_local, sign_local; uint64_t sign; double wr, wi; int32_t out_slot, pad; };
struct tile_overlap_set {
  int count, K;
  uint8_t tile_phys[16];
  uint8_t num_runs, run_src[16], run_len[16], run_dst[16];
  tile_overlap_spec spec[kMaxOverlaps];
};
size_t tile_overlaps_partials_doubles(int n, int K);

template <typename Real> cudaError_t launch_tile_overlaps(const void* lam, const void* psi, int n, const tile_overlap_set& set,
                                                          double* partials, double* out, cudaStream_t stream);

// All spins of the flip bits of one tile layout in one read of the state.
// Tile t (its bits outside tile_phys spell t, deposited run by run) of 2^K
// amplitudes, K = 8 + RB (RB = 3 for complex<double>, 4 for complex<float>;
// 256 threads), is staged in shared memory; for each flip f the CTAs sum
//   x_f = sum over j with tile bit b_f clear of conj(a_j) a_{j | b_f}   (complex)
//   z_f = sum over j with tile bit b_f set of |a_j|^2
// and the total of |a|^2.  The flips are read in register phases: in phase p
// a thread holds the 2^RB amplitudes whose tile bits phase_reg[p][0..RB-1]
// vary, at the tile bits phase_thr[p][0..7] that its index gives; flip
// f = p * RB + k is register bit k of phase p (entries past nflips are fillers).
// out[3f], out[3f+1] = x_f; out[3f+2] = z_f; out[3 nflips] = total.
constexpr int kMaxSpinFlips = 12;
constexpr int kSpinPhases = 4;
struct spin_group {
  int K, num_runs, nflips, nphases;
  uint8_t tile_phys[16], run_src[16], run_len[16], run_dst[16];
  uint8_t phase_reg[kSpinPhases][4];
  uint8_t phase_thr[kSpinPhases][8];
};
inline int spin_register_bits(int precision) { return precision == 0 ? 3 : 4; }
template <typename Real> cudaError_t launch_spins(const void* state, int n, const spin_group& g, double* partials, double* out,
                                                  cudaStream_t stream);

// Overlaps of one-qubit Paulis in one read of both states (the adjoint sweep's
// rotation runs).  Z type: S_q = sum_j (-1)^{j_q} conj(lam_j) psi_j for
// physical bit q; out[2 slot] = w * S_q for each entry.
struct zsum2_set {
  int count, pad;
  struct { int32_t bit, out_slot; double wr, wi; } spec[kMaxOverlaps];
};
// X / Y type, for the flips of one tile layout (spin_group with K = 11: three
// register bits and eight thread bits, both states' tiles in shared memory):
//   A_f = sum over j with tile bit b_f clear of conj(lam_j) psi_{j | b_f},
//   B_f = the same with lam and psi exchanged in position (conj(lam_{j | b_f}) psi_j),
// out[2 slot_f] = w_f (A_f + B_f) (X, minus 0) or w_f (A_f - B_f) (Y: minus 1,
// the sign bit is the flip).
constexpr int kMaxPairFlips = 8;
constexpr int kPairRegBits = 3;
struct pair_overlap_set {
  spin_group g;
  struct { int32_t out_slot, minus; double wr, wi; } flip[kMaxPairFlips];
};
size_t pair_overlaps_partials_doubles();
// The one-qubit gates of an adjoint run applied to both states in the same
// read and write, with the X / Y-type overlaps of the run's rotations taken
// from that read.  Same tile layout as pair_overlap_set, up to kMaxRotFlips
// register-phase bits (every tile bit).  Flip f: the overlap (as in
// pair_overlap_set; out_slot < 0 for none) from the amplitudes before its
// gate, then m (m00 m01 m10 m11 as (re, im)) on lam and psi.  The gates act on
// distinct bits and commute, so an overlap is the same whichever of the other
// gates are already applied.  Only the imaginary part of w (A + s B), which the
// gradient takes, is summed: out[2 slot] = 0, out[2 slot + 1] = Im.
// okind picks the arithmetic of the overlap: 1 when wr = 0 (only the real parts
// of A and B enter, as for Y types), 2 when wi = 0 (only the imaginary parts, X
// types), 3 otherwise (0: no overlap); mkind 1 marks a real matrix (EY, H),
// 2 a filler position without a gate.  Phase 0 must be the load layout:
// register bits 8, 9, 10 and thread bits 0..7 of the tile, in order.
// block_sync[p] = 1: the layout after phase p (the next phase's, or the load
// layout for the store) puts other tile bits on the warp index, so the
// exchange waits for the whole CTA; 0: every warp reads back only slots it
// wrote itself, and a warp barrier suffices.
constexpr int kMaxRotFlips = 12;
// Optional first step of a launch: a diagonal that both states still owe,
// applied at load time, and Z-type overlaps taken there (a diagonal with
// |d| = 1 leaves conj(lam_j) psi_j unchanged, so before or after is the same).
//   factor(j) = g * prod over the physical bits b set in j of u[b] * (-1)^Q(j),
//   Q(j) = sum over the bits b set in j of popcount(j & adj[b])   (mod 2),
// adj[b] holding b's controlled-Z partners above b.  For register slot it
// (tile bits 8..10), mr[it] is the XOR of the full partner rows of its set
// bits and bit it of qr the parity of its pairs among themselves.  Z entries:
// out[2 slot + 1] = wr Im(S_q), S_q = sum_j (-1)^{j_q} conj(lam_j) psi_j, out[2 slot] = 0.
struct pre_diag {
  int32_t active, nz;
  double g[2];
  double u[kMaxQubits][2];
  uint64_t adj[kMaxQubits];
  uint64_t full[kMaxQubits];  // all partners of each bit (both directions)
  uint64_t mr[8];
  uint32_t qr, pad;
  struct { int32_t bit, out_slot; double wr; } z[kMaxQubits];
};
struct pair_rotate_set {
  spin_group g;
  struct { int32_t out_slot, minus, okind, mkind; double wr, wi; double m[8]; } flip[kMaxRotFlips];
  uint8_t block_sync[kSpinPhases];
  uint8_t pad[4];
  pre_diag pre;
};
size_t pair_rotate_partials_doubles();  // per block: nflips overlap sums, then 1 + n Z sums when pre.nz > 0
template <typename Real> cudaError_t launch_pair_rotate(void* lam, void* psi, int n, const pair_rotate_set& set,
                                                        double* partials, double* out, cudaStream_t stream);
template <typename Real> cudaError_t launch_zsum2(const void* lam, const void* psi, int n, const zsum2_set& set,
                                                  double* partials, double* out, cudaStream_t stream);
template <typename Real> cudaError_t launch_pair_overlaps(const void* lam, const void* psi, int n, const pair_overlap_set& set,
                                                          double* partials, double* out, cudaStream_t stream);

// Sampling: prefix = inclusive scan of |a_i|^2 (scratch: scan_scratch_doubles(count)
// doubles); events[k] = upper_bound(prefix, r[k]).
size_t scan_scratch_doubles(uint64_t count);
template <typename Real> cudaError_t launch_prob_scan(const void* amps, uint64_t count, double* prefix, double* scratch,
                                                      cudaStream_t stream);
cudaError_t launch_upper_bound(const double* prefix, uint64_t count, const double* r, int num, uint64_t* events,
                               cudaStream_t stream);

// Dense k-qubit unitaries.
// Tensor cores (complex<float>, k = 5 or 6, n >= k + 7): w_split holds W_hi then
// W_lo (tc_w_split_floats(k) floats) in the kernel's operand layout; the kernel
// needs tc_shared_bytes(k) of shared memory and sets *error_flag on a timeout.
// Physical bits of the tensor-core kernel's rows: target_bit[i] is target i, row_bit[j]
// row-index bit j of a 128-row tile, and the tile index is deposited run by run
// into the remaining bits (n >= k + 7).
struct tc_layout {
  uint8_t target_bit[6];
  uint8_t row_bit[7];
  uint8_t num_runs;
  uint8_t run_src[16], run_len[16], run_dst[16];
};
size_t tc_w_split_floats(int k);
size_t tc_shared_bytes(int k);
cudaError_t launch_unitary_tf32x3(void* state, int n, int k, const float* w_split, int* error_flag, int grid,
                                  const tc_layout& layout, cudaStream_t stream);
// CUDA cores, any precision, k <= 10, targets on the low k physical bits: U is 2^k x 2^k
// complex (re, im) in row-major order on the device.
template <typename Real> cudaError_t launch_dense_rows(void* state, int n, int k, const double* U, cudaStream_t stream);

}  // namespace rbk
