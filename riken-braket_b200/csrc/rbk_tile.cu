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

#include <atomic>
#include <cstdint>

#include "rbk_device.cuh"
#include "rbk_internal.h"
#include "rbk_kernels.h"

namespace rbk {
namespace {

template <typename Real>
struct mat2 { Real m00r, m00i, m01r, m01i, m10r, m10i, m11r, m11i; };

// Complex 2x2 on register bit B; CTRL: also require the register-bit controls.
template <typename Real, int B, int NR, bool CTRL>
__device__ __forceinline__ void apply_mat(typename ctype<Real>::c* a, uint32_t creg, const mat2<Real>& M)
{
#pragma unroll
  for (int i = 0; i < NR; ++i) {
    if (i & (1 << B)) continue;
    if (CTRL && (uint32_t(i) & creg) != creg) continue;
    const auto a0 = a[i], a1 = a[i | (1 << B)];
    a[i] = cmac2(a0, a1, M.m00r, M.m00i, M.m01r, M.m01i);
    a[i | (1 << B)] = cmac2(a0, a1, M.m10r, M.m10i, M.m11r, M.m11i);
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
    const auto a0 = a[i], a1 = a[i | (1 << B)];
    a[i].x = M.m00r * a0.x + M.m01r * a1.x - M.m01i * a1.y;
    a[i].y = M.m00r * a0.y + M.m01r * a1.y + M.m01i * a1.x;
    a[i | (1 << B)] = cmac2(a0, a1, M.m10r, M.m10i, M.m11r, M.m11i);
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
    const auto a0 = a[i], a1 = a[i | (1 << B)];
    a[i].x = m00 * a0.x + m01 * a1.x;
    a[i].y = m00 * a0.y + m01 * a1.y;
    a[i | (1 << B)].x = m10 * a0.x + m11 * a1.x;
    a[i | (1 << B)].y = m10 * a0.y + m11 * a1.y;
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

// Runs CALL with the register bit b as the compile-time constant BB, so that
// the register array is only ever indexed with constants.
#define RBK_DISPATCH_BIT(b, CALL)                                       \
  switch (b) {                                                          \
    case 0: { constexpr int BB = 0; CALL; } break;                      \
    case 1: { constexpr int BB = 1; CALL; } break;                      \
    case 2: { constexpr int BB = 2; CALL; } break;                      \
    case 3: { constexpr int BB = 3; CALL; } break;                      \
    case 4: if constexpr (R > 4) { constexpr int BB = 4; CALL; } break; \
    default: break;                                                     \
  }

// One jump per op: the host encodes (kind, matrix form, controls, target bit)
// into op.code (see op_code in rbk_internal.h).
template <typename Real, int R>
__device__ __forceinline__ void apply_op(typename ctype<Real>::c* a, const dev_op& op, uint32_t tid, uint64_t base)
{
  using C = typename ctype<Real>::c;
  constexpr int NR = 1 << R;
  if ((tid & op.cthr) != op.cthr || (base & op.cout) != op.cout) return;
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
#define RBK_PERM_CASES(KIND, FN) \
  case op_code(KIND, 0, true, 0): FN<Real, 0, NR>(a, creg); break; \
  case op_code(KIND, 0, true, 1): FN<Real, 1, NR>(a, creg); break; \
  case op_code(KIND, 0, true, 2): FN<Real, 2, NR>(a, creg); break; \
  case op_code(KIND, 0, true, 3): FN<Real, 3, NR>(a, creg); break; \
  case op_code(KIND, 0, true, 4): if constexpr (R > 4) { FN<Real, (R > 4 ? 4 : 0), NR>(a, creg); } break;
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
    default: break;
  }
#undef RBK_PERM_CASES
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

template <typename Real, int SHAPE>
__global__ void __launch_bounds__(1 << (tile_shape<Real, SHAPE>::K - tile_shape<Real, SHAPE>::R), tile_shape<Real, SHAPE>::CTAS)
tile_pass_kernel(typename ctype<Real>::c* __restrict__ state, const __grid_constant__ dev_pass P)
{
  using C = typename ctype<Real>::c;
  using V = typename ctype<Real>::v16;
  using SH = tile_shape<Real, SHAPE>;
  using PT = precision_traits<Real>;
  constexpr int K = SH::K, R = SH::R, NR = 1 << R, T = K - R, NT = 1 << T, VEC = PT::VEC, VB = PT::VB;
  constexpr int ITER = (1 << K) / VEC / NT;
  constexpr int ITBITS = K - VB - T;
  static_assert((1 << ITBITS) == ITER, "tile copy iterations");
  static_assert(T >= 5 && T <= 9, "the layout tables split the thread index into 4 + up to 5 bits");

  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* tile = reinterpret_cast<C*>(smem_raw);
  const V* gsrc = reinterpret_cast<const V*>(state);
  V* gdst = reinterpret_cast<V*>(state);
  const uint32_t tid = threadIdx.x;

  // Tile base: the block index deposited into the physical bits outside the tile.
  uint64_t base = 0;
  {
    const uint64_t b = blockIdx.x;
    for (int r = 0; r < P.num_runs; ++r)
      base |= ((b >> P.run_src[r]) & ((1ull << P.run_len[r]) - 1)) << P.run_dst[r];
  }

  // Coalesced staging copy: vector u = it * NT + tid holds tile index u << VB;
  // consecutive threads read consecutive 16-byte vectors of a contiguous run.
  auto staged_copy = [&](bool to_smem) {
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
      if (to_smem) *s = __ldcs(gsrc + (phys >> VB));
      else __stcs(gdst + (phys >> VB), *s);
    }
  };

  if (!P.direct_load) {
    staged_copy(true);
    __syncthreads();
  }

  C a[NR];
  const int nph = P.num_phases;
  for (int p = 0; p < nph; ++p) {
    const dev_phase& ph = P.phases[p];
    if (p == 0 && P.direct_load) {
      const uint64_t tphys = base | P.load.tphys_lo[tid & 15] | P.load.tphys_hi[tid >> 4];
      uint64_t rphys[R];
#pragma unroll
      for (int b = 0; b < R; ++b) rphys[b] = P.load.rphys[b];
#pragma unroll
      for (int i = 0; i < NR; i += VEC) {
        uint64_t phys = tphys;
#pragma unroll
        for (int b = VB; b < R; ++b) if (i & (1 << b)) phys |= rphys[b];
        vec_io<Real>::unpack(__ldcs(gsrc + (phys >> VB)), &a[i]);
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

    for (int o = ph.op_begin; o < ph.op_end; ++o) apply_op<Real, R>(a, P.ops[o], tid, base);

    if (p + 1 == nph && P.direct_store) {
      // A one-phase pass that also loaded straight from HBM: every warp of the
      // CTA must have read its amplitudes before any warp overwrites the tile
      // in its relabelled order.
      if (p == 0 && P.direct_load) __syncthreads();
      const uint64_t tphys = base | P.store.tphys_lo[tid & 15] | P.store.tphys_hi[tid >> 4];
      uint64_t rphys[R];
#pragma unroll
      for (int b = 0; b < R; ++b) rphys[b] = P.store.rphys[b];
#pragma unroll
      for (int i = 0; i < NR; i += VEC) {
        uint64_t phys = tphys;
#pragma unroll
        for (int b = VB; b < R; ++b) if (i & (1 << b)) phys |= rphys[b];
        __stcs(gdst + (phys >> VB), vec_io<Real>::pack(&a[i]));
      }
    } else {
      __syncthreads();  // every thread has read this phase's layout
      const uint32_t ts = ph.wtslot_lo[tid & 15] ^ ph.wtslot_hi[tid >> 4];
      uint32_t rs[R];
#pragma unroll
      for (int b = 0; b < R; ++b) rs[b] = ph.wslot[b];
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

  if (!P.direct_store) staged_copy(false);
}

namespace {

template <typename Real, int SHAPE>
cudaError_t launch_shape(void* state, int n, const dev_pass& pass, cudaStream_t stream)
{
  using SH = tile_shape<Real, SHAPE>;
  const size_t smem = sizeof(typename ctype<Real>::c) << SH::K;
  static std::atomic<bool> configured[64] = {};  // per device; states on several host threads may race here
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
  if (!configured[dev].load(std::memory_order_acquire)) {
    e = cudaFuncSetAttribute(tile_pass_kernel<Real, SHAPE>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    configured[dev].store(true, std::memory_order_release);
  }
  if (n < SH::K) return cudaErrorInvalidValue;
  const uint64_t blocks = 1ull << (n - SH::K);
  tile_pass_kernel<Real, SHAPE><<<(unsigned)blocks, 1 << (SH::K - SH::R), smem, stream>>>(
    static_cast<typename ctype<Real>::c*>(state), pass);
  return cudaGetLastError();
}

}  // namespace

template <typename Real>
cudaError_t launch_tile_pass(void* state, int n, const dev_pass& pass, int shape, cudaStream_t stream)
{
  switch (shape) {
    case 0: return launch_shape<Real, 0>(state, n, pass, stream);
    case 1: return launch_shape<Real, 1>(state, n, pass, stream);
    case 2: return launch_shape<Real, 2>(state, n, pass, stream);
    default: return cudaErrorInvalidValue;
  }
}

template cudaError_t launch_tile_pass<double>(void*, int, const dev_pass&, int, cudaStream_t);
template cudaError_t launch_tile_pass<float>(void*, int, const dev_pass&, int, cudaStream_t);

}  // namespace rbk
