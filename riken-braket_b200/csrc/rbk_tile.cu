// rbk_tile.cu -- the fused tile pass, the hot kernel of the engine.
//
// One pass reads and writes every amplitude once.  CTA b owns the tile of 2^K
// amplitudes whose physical bits outside the pass's tile bits spell b.  The
// tile moves through a sequence of register layouts ("phases"): in each phase
// every thread holds 2^R amplitudes of the tile in registers, indexed by R
// tile bits, and applies the phase's gates -- 2x2 matrices on a register bit,
// with controls anywhere (register bits are checked per amplitude pair,
// thread bits per thread, bits outside the tile per CTA).  Between phases the
// tile is exchanged through shared memory.  The first phase loads straight
// from HBM and the last phase stores straight to HBM when their layouts put
// the lanes on the contiguous low tile bits; otherwise the tile is staged
// through shared memory with coalesced 16-byte accesses.
//
// Replaces ket's per-gate sweeps (ket/include/ket/gate/hadamard.hpp:52-71,
// phase_shift.hpp:1235-1253, pauli_x.hpp:120-165, ...) and bra's fused replay
// of a BEGIN/END FUSION block on every 2^k chunk (bra/src/nompi_state.cpp:1285-1357).
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cstdint>

#include "rbk_device.cuh"
#include "rbk_internal.h"
#include "rbk_kernels.h"

namespace rbk {
namespace {

template <typename Real>
struct mat2 { Real m00r, m00i, m01r, m01i, m10r, m10i, m11r, m11i; };

// Fused multiply-add, a * b + c with one rounding.
__device__ __forceinline__ double madd(double a, double b, double c) { return __fma_rn(a, b, c); }
__device__ __forceinline__ float madd(float a, float b, float c) { return __fmaf_rn(a, b, c); }

// The 2x2 updates below are ordered so that every input register is dead when
// its output is written (the products that need the old value of a component
// are formed first): each output can take its input's register, and the
// register array needs no copies where the op cases of the dispatch rejoin.

// Complex 2x2 on register bit B; CTRL: also require the register-bit controls.
template <typename Real, int B, int NR, bool CTRL>
__device__ __forceinline__ void apply_mat(typename ctype<Real>::c* a, uint32_t creg, const mat2<Real>& M)
{
#pragma unroll
  for (int i = 0; i < NR; ++i) {
    if (i & (1 << B)) continue;
    if (CTRL && (uint32_t(i) & creg) != creg) continue;
    auto& a0 = a[i];
    auto& a1 = a[i | (1 << B)];
    // m01 a1 and m10 a0, then the m11 and m00 terms in place.
    Real p = madd(-M.m01i, a1.y, M.m01r * a1.x);
    Real q = madd(M.m01i, a1.x, M.m01r * a1.y);
    Real r = madd(-M.m10i, a0.y, M.m10r * a0.x);
    Real t = madd(M.m10i, a0.x, M.m10r * a0.y);
    r = madd(-M.m11i, a1.y, r);
    t = madd(M.m11i, a1.x, t);
    a1.x = madd(M.m11r, a1.x, r);
    a1.y = madd(M.m11r, a1.y, t);
    p = madd(-M.m00i, a0.y, p);
    q = madd(M.m00i, a0.x, q);
    a0.x = madd(M.m00r, a0.x, p);
    a0.y = madd(M.m00r, a0.y, q);
  }
}

// Complex 2x2 whose m00 is real (U3: cos(theta/2); U2: 1/sqrt 2): 14 multiply-adds per pair instead of 16.
template <typename Real, int B, int NR, bool CTRL>
__device__ __forceinline__ void apply_mat_r00(typename ctype<Real>::c* a, uint32_t creg, const mat2<Real>& M)
{
#pragma unroll
  for (int i = 0; i < NR; ++i) {
    if (i & (1 << B)) continue;
    if (CTRL && (uint32_t(i) & creg) != creg) continue;
    auto& a0 = a[i];
    auto& a1 = a[i | (1 << B)];
    const Real p = madd(-M.m01i, a1.y, M.m01r * a1.x);
    const Real q = madd(M.m01i, a1.x, M.m01r * a1.y);
    Real r = madd(-M.m10i, a0.y, M.m10r * a0.x);
    Real t = madd(M.m10i, a0.x, M.m10r * a0.y);
    r = madd(-M.m11i, a1.y, r);
    t = madd(M.m11i, a1.x, t);
    a1.x = madd(M.m11r, a1.x, r);
    a1.y = madd(M.m11r, a1.y, t);
    a0.x = madd(M.m00r, a0.x, p);
    a0.y = madd(M.m00r, a0.y, q);
  }
}

// Real 2x2 (H, exp(i theta Y), ...): half the multiply-adds.
template <typename Real, int B, int NR, bool CTRL>
__device__ __forceinline__ void apply_real(typename ctype<Real>::c* a, uint32_t creg, Real m00, Real m01, Real m10, Real m11)
{
#pragma unroll
  for (int i = 0; i < NR; ++i) {
    if (i & (1 << B)) continue;
    if (CTRL && (uint32_t(i) & creg) != creg) continue;
    auto& a0 = a[i];
    auto& a1 = a[i | (1 << B)];
    const Real px = m01 * a1.x, py = m01 * a1.y;
    const Real ux = m10 * a0.x, uy = m10 * a0.y;
    a1.x = madd(m11, a1.x, ux);
    a1.y = madd(m11, a1.y, uy);
    a0.x = madd(m00, a0.x, px);
    a0.y = madd(m00, a0.y, py);
  }
}

template <typename Real, int B, int NR>
__device__ __forceinline__ void apply_x(typename ctype<Real>::c* a, uint32_t creg)
{
#pragma unroll
  for (int i = 0; i < NR; ++i) {
    if (i & (1 << B)) continue;
    if ((uint32_t(i) & creg) != creg) continue;
    const auto t = a[i];
    a[i] = a[i | (1 << B)];
    a[i | (1 << B)] = t;
  }
}

template <typename Real, int B, int NR>
__device__ __forceinline__ void apply_y(typename ctype<Real>::c* a, uint32_t creg)
{
  using C = typename ctype<Real>::c;
#pragma unroll
  for (int i = 0; i < NR; ++i) {
    if (i & (1 << B)) continue;
    if ((uint32_t(i) & creg) != creg) continue;
    const auto a0 = a[i], a1 = a[i | (1 << B)];
    a[i] = C{a1.y, -a1.x};          // -i * a1
    a[i | (1 << B)] = C{-a0.y, a0.x}; //  i * a0
  }
}

// Multiplies (xr, xi) by (dr, di) in place.
__device__ __forceinline__ void cmul_acc(double& xr, double& xi, double dr, double di)
{
  const double t = xr * dr - xi * di;
  xi = xr * di + xi * dr;
  xr = t;
}

// A run of phase gates (PHASES header; rbk_plan.cpp group_phase_runs): gate k
// multiplies the amplitudes whose bits creg / cthr / cout are all one by its
// factor (m[2], m[3]).  The members come sorted by accumulator, with the class
// sizes in the header's dout: gates on no register bit multiply the thread's
// accumulator, gates on one register bit b that of b, and every amplitude takes
// the product of its accumulators once at the end; gates on two or more
// register bits (the rest of the run) multiply their amplitudes directly.
// Accumulation in double for both precisions.
template <typename Real, int R>
__device__ __forceinline__ void apply_phase_run(typename ctype<Real>::c* a, const dev_op* run, int count,
                                                uint64_t classes, uint32_t tid, uint64_t base)
{
  constexpr int NR = 1 << R;
  double fr = 1.0, fi = 0.0;
  double lr[R], li[R];
#pragma unroll
  for (int b = 0; b < R; ++b) { lr[b] = 1.0; li[b] = 0.0; }
  int k = 0;
  for (const int e = static_cast<int>(classes & 0xff); k < e; ++k) {
    const dev_op& g = run[k];
    if ((tid & g.cthr) == g.cthr && (base & g.cout) == g.cout) cmul_acc(fr, fi, g.m[2], g.m[3]);
  }
#pragma unroll
  for (int b = 0; b < R; ++b) {
    for (const int e = k + static_cast<int>((classes >> (8 * (b + 1))) & 0xff); k < e; ++k) {
      const dev_op& g = run[k];
      if ((tid & g.cthr) == g.cthr && (base & g.cout) == g.cout) cmul_acc(lr[b], li[b], g.m[2], g.m[3]);
    }
  }
  for (; k < count; ++k) {
    const dev_op& g = run[k];
    if ((tid & g.cthr) != g.cthr || (base & g.cout) != g.cout) continue;
    const uint32_t mr = g.creg;
    const double dr = g.m[2], di = g.m[3];
#pragma unroll
    for (int i = 0; i < NR; ++i) {
      if ((uint32_t(i) & mr) != mr) continue;
      double xr = double(a[i].x), xi = double(a[i].y);
      cmul_acc(xr, xi, dr, di);
      a[i].x = static_cast<Real>(xr);
      a[i].y = static_cast<Real>(xi);
    }
  }
#pragma unroll
  for (int i = 0; i < NR; ++i) {
    double pr = fr, pi = fi;
#pragma unroll
    for (int b = 0; b < R; ++b)
      if ((i >> b) & 1) cmul_acc(pr, pi, lr[b], li[b]);
    const double xr = double(a[i].x), xi = double(a[i].y);
    a[i].x = static_cast<Real>(xr * pr - xi * pi);
    a[i].y = static_cast<Real>(xr * pi + xi * pr);
  }
}

// One gate of a LAYER on register bit B, in the layer's matrix form.
template <typename Real, int R, int FORM, int B>
__device__ __forceinline__ void layer_gate(typename ctype<Real>::c* a, const dev_op& g)
{
  constexpr int NR = 1 << R;
  if constexpr (FORM == 1) {
    apply_real<Real, B, NR, false>(a, 0u, (Real)g.m[0], (Real)g.m[2], (Real)g.m[4], (Real)g.m[6]);
  } else {
    const mat2<Real> M{(Real)g.m[0], FORM == 2 ? (Real)0 : (Real)g.m[1], (Real)g.m[2], (Real)g.m[3],
                       (Real)g.m[4], (Real)g.m[5], (Real)g.m[6], (Real)g.m[7]};
    if constexpr (FORM == 2) apply_mat_r00<Real, B, NR, false>(a, 0u, M);
    else apply_mat<Real, B, NR, false>(a, 0u, M);
  }
}

// A LAYER (rbk_plan.cpp group_layers): the uncontrolled 2x2 gates that follow
// the header, one per register bit of `mask` in ascending bit order, with no
// dispatch between them.  FULL: every register bit has one; for complex<double>
// (4 register bits) the gates then run as one straight-line block.  For
// complex<float> (5 register bits) that block made the kernel spill registers
// and run slower (30-qubit brick: 350 ms against 317 ms with the per-bit form),
// so it takes the per-bit form for every mask.
template <typename Real, int R, int FORM, bool FULL, int B = 0>
__device__ __forceinline__ void apply_layer(typename ctype<Real>::c* a, const dev_op* g, uint32_t mask)
{
  if constexpr (B < R) {
    if constexpr (FULL && sizeof(Real) == 8) {
      layer_gate<Real, R, FORM, B>(a, g[B]);
      apply_layer<Real, R, FORM, FULL, B + 1>(a, g, mask);
    } else {
      if ((mask >> B) & 1u) {
        layer_gate<Real, R, FORM, B>(a, *g);
        ++g;
      }
      apply_layer<Real, R, FORM, FULL, B + 1>(a, g, mask);
    }
  }
}

// The middle factor [[1, t0], [t1, 1]] of a factored layer's gate on register
// bit B (kLayerFactored in rbk_internal.h): four real multiply-adds per pair.
template <typename Real, int B, int NR>
__device__ __forceinline__ void apply_factor(typename ctype<Real>::c* a, Real t0, Real t1)
{
#pragma unroll
  for (int i = 0; i < NR; ++i) {
    if (i & (1 << B)) continue;
    auto& a0 = a[i];
    auto& a1 = a[i | (1 << B)];
    const Real x = madd(t0, a1.x, a0.x), y = madd(t0, a1.y, a0.y);
    a1.x = madd(t1, a0.x, a1.x);
    a1.y = madd(t1, a0.y, a1.y);
    a0.x = x;
    a0.y = y;
  }
}

template <typename Real, int R, bool FULL, int B = 0>
__device__ __forceinline__ void apply_factors(typename ctype<Real>::c* a, const dev_op* g, uint32_t mask)
{
  if constexpr (B < R) {
    if (FULL || ((mask >> B) & 1u)) {
      apply_factor<Real, B, 1 << R>(a, (Real)g->m[0], (Real)g->m[1]);
      ++g;
    }
    apply_factors<Real, R, FULL, B + 1>(a, g, mask);
  }
}

// A factored LAYER: the pre factors (when the header asks for them), the
// middle factor of each member, the post factors.  The header's slot holds
// pre_lo[4], pre_hi[2^(R-2)], post_lo[4], post_hi[2^(R-2)] in the state's
// precision; slot i of the registers takes lo[i & 3] hi[i >> 2] (pre_lo[0],
// pre_hi[0] and post_hi[0] are 1 and are not applied).
template <typename Real, int R, bool FULL>
__device__ __forceinline__ void apply_factored_layer(typename ctype<Real>::c* a, const dev_op& h, const double* tabs)
{
  using C = typename ctype<Real>::c;
  constexpr int NR = 1 << R, H = 1 << (R - 2);
  const C* pre_lo = reinterpret_cast<const C*>(tabs + h.dthr * kTabDoubles);
  const C* pre_hi = pre_lo + 4;
  const C* post_lo = pre_hi + H;
  const C* post_hi = post_lo + 4;
  if (h.diag_one) {
#pragma unroll
    for (int i = 1; i < NR; ++i) {
      if (i & 3) a[i] = cmul(a[i], pre_lo[i & 3]);
      if (i >> 2) a[i] = cmul(a[i], pre_hi[i >> 2]);
    }
  }
  apply_factors<Real, R, FULL>(a, &h + 1, h.dreg);
#pragma unroll
  for (int i = 0; i < NR; ++i) {
    a[i] = cmul(a[i], post_lo[i & 3]);
    if (i >> 2) a[i] = cmul(a[i], post_hi[i >> 2]);
  }
}

// One jump per op: the host encodes (kind, matrix form, controls, target bit)
// into op.code (see op_code in rbk_internal.h).  Returns how many of the
// following op records the op consumed (a phase run's gates).
template <typename Real, int R>
__device__ __forceinline__ int apply_op(typename ctype<Real>::c* a, const dev_op& op, uint32_t tid, uint64_t base,
                                        const double* tabs)
{
  using C = typename ctype<Real>::c;
  constexpr int NR = 1 << R;
  if ((tid & op.cthr) != op.cthr || (base & op.cout) != op.cout) return 0;
  const uint32_t creg = op.creg;
#define RBK_MAT_CASES(FORM, CTRL, B)                                                                    \
  case op_code(OPK_MAT, FORM, CTRL, B):                                                                 \
    if constexpr (B < R) {                                                                              \
      if constexpr (FORM == 1) {                                                                        \
        apply_real<Real, B, NR, CTRL>(a, creg, (Real)op.m[0], (Real)op.m[2], (Real)op.m[4], (Real)op.m[6]); \
      } else {                                                                                          \
        const mat2<Real> M{(Real)op.m[0], FORM == 2 ? (Real)0 : (Real)op.m[1], (Real)op.m[2], (Real)op.m[3], \
                           (Real)op.m[4], (Real)op.m[5], (Real)op.m[6], (Real)op.m[7]};                \
        if constexpr (FORM == 2) apply_mat_r00<Real, B, NR, CTRL>(a, creg, M);                          \
        else apply_mat<Real, B, NR, CTRL>(a, creg, M);                                                  \
      }                                                                                                 \
    }                                                                                                   \
    break;
#define RBK_MAT_BITS(FORM, CTRL) \
  RBK_MAT_CASES(FORM, CTRL, 0) RBK_MAT_CASES(FORM, CTRL, 1) RBK_MAT_CASES(FORM, CTRL, 2) \
  RBK_MAT_CASES(FORM, CTRL, 3) RBK_MAT_CASES(FORM, CTRL, 4)
// Register bits at or above R have no case body: a body would index past a[].
#define RBK_PERM_CASE(KIND, FN, B) \
  case op_code(KIND, 0, true, B): if constexpr (B < R) { FN<Real, (B < R ? B : 0), NR>(a, creg); } break;
#define RBK_PERM_CASES(KIND, FN) \
  RBK_PERM_CASE(KIND, FN, 0) RBK_PERM_CASE(KIND, FN, 1) RBK_PERM_CASE(KIND, FN, 2) \
  RBK_PERM_CASE(KIND, FN, 3) RBK_PERM_CASE(KIND, FN, 4)
  switch (op.code) {
    RBK_MAT_BITS(0, false) RBK_MAT_BITS(0, true)
    RBK_MAT_BITS(1, false) RBK_MAT_BITS(1, true)
    RBK_MAT_BITS(2, false) RBK_MAT_BITS(2, true)
    RBK_PERM_CASES(OPK_X, apply_x)
    RBK_PERM_CASES(OPK_Y, apply_y)
    case op_code(OPK_NEG, 0, true, 0):
#pragma unroll
      for (int i = 0; i < NR; ++i)
        if ((uint32_t(i) & creg) == creg) { a[i].x = -a[i].x; a[i].y = -a[i].y; }
      break;
    case op_code(OPK_DIAG, 0, true, 0): {
      const bool tb = ((tid & op.dthr) != 0) || ((base & op.dout) != 0);
      const C d0{(Real)op.m[0], (Real)op.m[1]}, d1{(Real)op.m[2], (Real)op.m[3]};
      const uint32_t dreg = op.dreg;
      const bool one = op.diag_one;
#pragma unroll
      for (int i = 0; i < NR; ++i) {
        if ((uint32_t(i) & creg) != creg) continue;
        const bool bit = tb || (uint32_t(i) & dreg);
        if (bit) a[i] = cmul(a[i], d1);
        else if (!one) a[i] = cmul(a[i], d0);
      }
      break;
    }
    case op_code(OPK_PHASES, 0, true, 0):
      apply_phase_run<Real, R>(a, &op + 1, static_cast<int>(op.run), op.dout, tid, base);
      return static_cast<int>(op.run);
#define RBK_LAYER_CASE(FORM, FULL) \
    case op_code(OPK_LAYER, FORM, FULL, 0): \
      apply_layer<Real, R, FORM, FULL>(a, &op + 1, op.dreg); \
      return static_cast<int>(op.run);
    RBK_LAYER_CASE(0, false) RBK_LAYER_CASE(0, true)
    RBK_LAYER_CASE(1, false) RBK_LAYER_CASE(1, true)
    RBK_LAYER_CASE(2, false) RBK_LAYER_CASE(2, true)
#undef RBK_LAYER_CASE
    case op_code(OPK_LAYER, kLayerFactored, false, 0):
      apply_factored_layer<Real, R, false>(a, op, tabs);
      return static_cast<int>(op.run);
    case op_code(OPK_LAYER, kLayerFactored, true, 0):
      apply_factored_layer<Real, R, true>(a, op, tabs);
      return static_cast<int>(op.run);
    default: break;
  }
  return 0;
#undef RBK_PERM_CASES
#undef RBK_PERM_CASE
#undef RBK_MAT_BITS
#undef RBK_MAT_CASES
}

}  // namespace

namespace {

// 16-byte vectors <-> register amplitudes (1 amplitude for c128, 2 for c64).
template <typename Real> struct vec_io;
template <> struct vec_io<double> {
  static __device__ __forceinline__ void unpack(double2 v, double2* a) { a[0] = v; }
  static __device__ __forceinline__ double2 pack(const double2* a) { return a[0]; }
};
template <> struct vec_io<float> {
  static __device__ __forceinline__ void unpack(float4 v, float2* a) { a[0] = float2{v.x, v.y}; a[1] = float2{v.z, v.w}; }
  static __device__ __forceinline__ float4 pack(const float2* a) { return float4{a[0].x, a[0].y, a[1].x, a[1].y}; }
};

}  // namespace

// Copies a tile between HBM and shared memory with coalesced 16-byte
// vectors: vector u = it * NT + tid holds tile index u << VB, so consecutive
// threads touch consecutive vectors of a contiguous 512-byte run.
// MODE 0: load, 1: store, 2: asynchronous load (cp.async, completes at the
// caller's cp.async.wait_group).
template <typename Real, int K, int T, int MODE>
__device__ __forceinline__ void tile_copy(typename ctype<Real>::c* __restrict__ state, const dev_pass& P,
                                          typename ctype<Real>::c* tile, uint64_t base, uint32_t tid)
{
  using V = typename ctype<Real>::v16;
  constexpr int VB = precision_traits<Real>::VB, NT = 1 << T;
  constexpr int ITBITS = K - VB - T, ITER = 1 << ITBITS;
  uint64_t thr_phys = base;
#pragma unroll
  for (int b = 0; b < T; ++b) thr_phys |= uint64_t((tid >> b) & 1u) << P.tile_phys[VB + b];
  const uint32_t thr_slot = smem_slot<VB>(tid << VB);
#pragma unroll
  for (int it = 0; it < ITER; ++it) {
    uint64_t phys = thr_phys;
#pragma unroll
    for (int b = 0; b < ITBITS; ++b)
      if (it & (1 << b)) phys |= 1ull << P.tile_phys[VB + T + b];
    V* s = reinterpret_cast<V*>(&tile[thr_slot ^ smem_slot<VB>(uint32_t(it * NT) << VB)]);
    V* g = reinterpret_cast<V*>(state) + (phys >> VB);
    if constexpr (MODE == 0) *s = __ldcs(g);
    else if constexpr (MODE == 1) __stcs(g, *s);
    else {
      const uint32_t saddr = static_cast<uint32_t>(__cvta_generic_to_shared(s));
      asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" :: "r"(saddr), "l"(g) : "memory");
    }
  }
}

__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" :: "n"(N) : "memory"); }

// Tile base: tile index b deposited into the physical bits outside the tile.
__device__ __forceinline__ uint64_t tile_base(const dev_pass& P, uint64_t b)
{
  uint64_t base = 0;
  for (int r = 0; r < P.num_runs; ++r)
    base |= ((b >> P.run_src[r]) & ((1ull << P.run_len[r]) - 1)) << P.run_dst[r];
  return base;
}

// The folded CNOTs of a phase that hold on some tiles only (controls outside
// the tile): move the write positions of this tile's registers (dev_fold).
template <int R, typename W>
__device__ __forceinline__ void apply_folds(const dev_phase& ph, uint64_t base, uint32_t tid, W& thr, W (&reg)[R])
{
  const int nf = ph.num_folds;
  for (int f = 0; f < nf; ++f) {
    const dev_fold& F = ph.folds[f];
    if ((base & F.cout) != F.cout) continue;  // the same for the whole CTA
    const W x = static_cast<W>(F.x);
    if (F.kind == 0) {
      thr ^= x;
    } else if (F.kind == 2) {
      if ((tid >> F.bit) & 1u) thr ^= x;
    } else {
#pragma unroll
      for (int b = 0; b < R; ++b) reg[b] ^= (b == F.bit) ? x : W(0);
    }
  }
}

// One tile through the pass's phases, ending with the tile stored to HBM.
// load_mode: phase 0 loads its registers straight from HBM (the pass's direct
// load: 1 in 16-byte vectors, 2 in 8-byte complex<float> amplitudes); 0: the
// tile is already in `tile` and visible to every thread.  The pass's
// direct_store gives the last phase's store the same way.
// The caller synchronises before `tile` is reused.
template <typename Real, int K, int R>
__device__ __forceinline__ void tile_phases(typename ctype<Real>::c* __restrict__ state, const dev_pass& P,
                                            typename ctype<Real>::c* tile, uint64_t base, uint32_t tid, int load_mode)
{
  const bool from_hbm = load_mode != 0;
  using C = typename ctype<Real>::c;
  using V = typename ctype<Real>::v16;
  using PT = precision_traits<Real>;
  constexpr int NR = 1 << R, T = K - R, VEC = PT::VEC, VB = PT::VB;
  const V* gsrc = reinterpret_cast<const V*>(state);
  V* gdst = reinterpret_cast<V*>(state);

  C a[NR];
  const int nph = P.num_phases;
  for (int p = 0; p < nph; ++p) {
    const dev_phase& ph = P.phases[p];
    if (p == 0 && from_hbm) {
      const uint64_t tphys = base | P.load.tphys_lo[tid & 15] | P.load.tphys_hi[tid >> 4];
      uint64_t rphys[R];
#pragma unroll
      for (int b = 0; b < R; ++b) rphys[b] = P.load.rphys[b];
      if (sizeof(Real) == 4 && load_mode == 2) {
        const C* src = state;
#pragma unroll
        for (int i = 0; i < NR; ++i) {
          uint64_t phys = tphys;
#pragma unroll
          for (int b = 0; b < R; ++b) if (i & (1 << b)) phys |= rphys[b];
          a[i] = __ldcs(src + phys);
        }
      } else {
#pragma unroll
        for (int i = 0; i < NR; i += VEC) {
          uint64_t phys = tphys;
#pragma unroll
          for (int b = VB; b < R; ++b) if (i & (1 << b)) phys |= rphys[b];
          vec_io<Real>::unpack(__ldcs(gsrc + (phys >> VB)), &a[i]);
        }
      }
    } else {
      const uint32_t ts = ph.tslot_lo[tid & 15] ^ ph.tslot_hi[tid >> 4];
      uint32_t rs[R];
#pragma unroll
      for (int b = 0; b < R; ++b) rs[b] = ph.rslot[b];
#pragma unroll
      for (int i = 0; i < NR; ++i) {
        uint32_t sidx = ts;
#pragma unroll
        for (int b = 0; b < R; ++b) if (i & (1 << b)) sidx ^= rs[b];
        a[i] = tile[sidx];
      }
    }

    for (int o = ph.op_begin; o < ph.op_end; ++o) o += apply_op<Real, R>(a, P.ops[o], tid, base, P.tabs);

    if (p + 1 == nph && P.direct_store) {
      // A one-phase pass that also loaded straight from HBM: every warp of the
      // CTA must have read its amplitudes before any warp overwrites the tile
      // in its relabelled order.
      if (p == 0 && from_hbm) __syncthreads();
      // base holds only bits outside the tile, the tables only tile bits;
      // folded CNOTs make table contributions overlap, hence XOR.
      uint64_t tphys = base ^ P.store.tphys_lo[tid & 15] ^ P.store.tphys_hi[tid >> 4];
      uint64_t rphys[R];
#pragma unroll
      for (int b = 0; b < R; ++b) rphys[b] = P.store.rphys[b];
      apply_folds<R>(ph, base, tid, tphys, rphys);
      if (sizeof(Real) == 4 && P.direct_store == 2) {
        C* dst = state;
#pragma unroll
        for (int i = 0; i < NR; ++i) {
          uint64_t phys = tphys;
#pragma unroll
          for (int b = 0; b < R; ++b) if (i & (1 << b)) phys ^= rphys[b];
          __stcs(dst + phys, a[i]);
        }
      } else {
#pragma unroll
        for (int i = 0; i < NR; i += VEC) {
          uint64_t phys = tphys;
#pragma unroll
          for (int b = VB; b < R; ++b) if (i & (1 << b)) phys ^= rphys[b];
          __stcs(gdst + (phys >> VB), vec_io<Real>::pack(&a[i]));
        }
      }
    } else {
      // Every thread has read this phase's layout from `tile` (a phase that
      // loaded straight from HBM has not used it).
      if (!(p == 0 && from_hbm)) __syncthreads();
      uint32_t ts = ph.wtslot_lo[tid & 15] ^ ph.wtslot_hi[tid >> 4];
      uint32_t rs[R];
#pragma unroll
      for (int b = 0; b < R; ++b) rs[b] = ph.wslot[b];
      apply_folds<R>(ph, base, tid, ts, rs);
#pragma unroll
      for (int i = 0; i < NR; ++i) {
        uint32_t sidx = ts;
#pragma unroll
        for (int b = 0; b < R; ++b) if (i & (1 << b)) sidx ^= rs[b];
        tile[sidx] = a[i];
      }
      __syncthreads();
    }
  }

  if (!P.direct_store) tile_copy<Real, K, T, 1>(state, P, tile, base, tid);
}

// One CTA per tile (PIPE false): the tile is loaded (straight into registers
// when the pass allows it), run through the phases and stored.
// Persistent CTAs (PIPE true): CTA c takes tiles c, c + grid, c + 2 grid, ...;
// while it works on one tile in one shared-memory buffer, cp.async copies its
// next tile into the other, so that HBM reads stay in flight during the
// arithmetic.  The barrier at the end of each tile orders the last reads of a
// buffer before the copy into it is issued.
template <typename Real, int SHAPE>
__global__ void __launch_bounds__(1 << (tile_shape<Real, SHAPE>::K - tile_shape<Real, SHAPE>::R), tile_shape<Real, SHAPE>::CTAS)
tile_pass_kernel(typename ctype<Real>::c* __restrict__ state, const __grid_constant__ dev_pass P, uint64_t num_tiles)
{
  using C = typename ctype<Real>::c;
  using SH = tile_shape<Real, SHAPE>;
  constexpr int K = SH::K, R = SH::R, T = K - R;
  static_assert(T >= 5 && T <= 9, "the layout tables split the thread index into 4 + up to 5 bits");

  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* tile = reinterpret_cast<C*>(smem_raw);
  const uint32_t tid = threadIdx.x;

  if constexpr (!SH::PIPE) {
    const uint64_t base = tile_base(P, blockIdx.x);
    if (!P.direct_load) {
      tile_copy<Real, K, T, 0>(state, P, tile, base, tid);
      __syncthreads();
    }
    tile_phases<Real, K, R>(state, P, tile, base, tid, P.direct_load);
  } else {
    uint64_t t = blockIdx.x;
    if (t < num_tiles) tile_copy<Real, K, T, 2>(state, P, tile, tile_base(P, t), tid);
    cp_async_commit();
    uint32_t cur = 0;  // buffer of tile t: elements [cur << K, (cur + 1) << K)
    for (; t < num_tiles; t += gridDim.x) {
      const uint64_t next = t + gridDim.x;
      if (next < num_tiles) tile_copy<Real, K, T, 2>(state, P, tile + ((cur ^ 1u) << K), tile_base(P, next), tid);
      cp_async_commit();
      cp_async_wait<1>();  // this thread's copies of tile t have landed
      __syncthreads();     // ... and every other thread's
      tile_phases<Real, K, R>(state, P, tile + (cur << K), tile_base(P, t), tid, 0);
      __syncthreads();
      cur ^= 1u;
    }
    cp_async_wait<0>();
  }
}

namespace {

template <typename Real, int SHAPE>
cudaError_t launch_shape(void* state, int n, const dev_pass& pass, cudaStream_t stream)
{
  using SH = tile_shape<Real, SHAPE>;
  const size_t smem = (sizeof(typename ctype<Real>::c) << SH::K) * (SH::PIPE ? 2 : 1);
  // Per device; states on several host threads may race here.  resident[dev]:
  // CTAs of the persistent form that fit on the device at once.
  static std::atomic<bool> configured[64] = {};
  static std::atomic<int> resident[64] = {};
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
  if (!configured[dev].load(std::memory_order_acquire)) {
    e = cudaFuncSetAttribute(tile_pass_kernel<Real, SHAPE>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    if constexpr (SH::PIPE) {
      int per_sm = 0, sms = 0;
      e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, tile_pass_kernel<Real, SHAPE>, 1 << (SH::K - SH::R), smem);
      if (e != cudaSuccess) return e;
      e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
      if (e != cudaSuccess) return e;
      if (per_sm < 1 || sms < 1) return cudaErrorInvalidConfiguration;
      resident[dev].store(per_sm * sms, std::memory_order_relaxed);
    }
    configured[dev].store(true, std::memory_order_release);
  }
  if (n < SH::K) return cudaErrorInvalidValue;
  const uint64_t tiles = 1ull << (n - SH::K);
  uint64_t grid = tiles;
  if constexpr (SH::PIPE) grid = std::min<uint64_t>(tiles, static_cast<uint64_t>(resident[dev].load(std::memory_order_relaxed)));
  tile_pass_kernel<Real, SHAPE><<<(unsigned)grid, 1 << (SH::K - SH::R), smem, stream>>>(
    static_cast<typename ctype<Real>::c*>(state), pass, tiles);
  return cudaGetLastError();
}

}  // namespace

template <typename Real>
cudaError_t launch_tile_pass(void* state, int n, const dev_pass& pass, int shape, cudaStream_t stream)
{
  switch (shape) {
    case 0: return launch_shape<Real, 0>(state, n, pass, stream);
    // Shape 1 (2^12-amplitude tile, 8 per thread, 512 threads) is not built:
    // its instantiation raised an illegal memory access whose cause is not found.
    case 2: return launch_shape<Real, 2>(state, n, pass, stream);
    case 3: return launch_shape<Real, 3>(state, n, pass, stream);
    default: return cudaErrorInvalidValue;
  }
}

template cudaError_t launch_tile_pass<double>(void*, int, const dev_pass&, int, cudaStream_t);
template cudaError_t launch_tile_pass<float>(void*, int, const dev_pass&, int, cudaStream_t);

}  // namespace rbk
