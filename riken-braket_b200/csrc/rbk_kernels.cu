// rbk_kernels.cu -- sm_100a kernels of the state-vector engine.
//
//   (the fused tile pass lives in rbk_tile.cu)
//   gate_kernel        one unfused gate straight on HBM (states smaller than a
//                      tile, and the unfused execution mode).
//   reductions         norm, probabilities, Z / pair sums for spins and Pauli
//                      strings, inner product: warp-shuffle + block reduction
//                      with FP64 accumulation, per-block partials reduced in a
//                      fixed order (deterministic).
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cstdint>
#include <vector>

#include "rbk_device.cuh"
#include "rbk_internal.h"
#include "rbk_kernels.h"

namespace rbk {

// ---------------------------------------------------------------------------
// Unfused gate straight on HBM
// ---------------------------------------------------------------------------

template <typename Real>
__global__ void gate_kernel(typename ctype<Real>::c* __restrict__ a, uint64_t size, const gate_rec g)
{
  using C = typename ctype<Real>::c;
  const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
  const uint64_t tmask = 1ull << g.target;
  if (g.kind == OPK_MAT || g.kind == OPK_X || g.kind == OPK_Y) {
    const Real m00r = (Real)g.m[0], m00i = (Real)g.m[1], m01r = (Real)g.m[2], m01i = (Real)g.m[3];
    const Real m10r = (Real)g.m[4], m10i = (Real)g.m[5], m11r = (Real)g.m[6], m11i = (Real)g.m[7];
    for (uint64_t v = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; v < (size >> 1); v += stride) {
      const uint64_t i0 = insert_zero(v, g.target), i1 = i0 | tmask;
      if ((i0 & g.cmask) != g.cmask) continue;
      C a0 = a[i0], a1 = a[i1];
      if (g.kind == OPK_X) { a[i0] = a1; a[i1] = a0; }
      else if (g.kind == OPK_Y) { a[i0] = C{a1.y, -a1.x}; a[i1] = C{-a0.y, a0.x}; }
      else {
        a[i0] = cmac2(a0, a1, m00r, m00i, m01r, m01i);
        a[i1] = cmac2(a0, a1, m10r, m10i, m11r, m11i);
      }
    }
  } else {
    const C d0{(Real)g.m[0], (Real)g.m[1]}, d1{(Real)g.m[2], (Real)g.m[3]};
    for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < size; i += stride) {
      if ((i & g.cmask) != g.cmask) continue;
      if (g.kind == OPK_NEG) { a[i].x = -a[i].x; a[i].y = -a[i].y; }
      else if (i & tmask) a[i] = cmul(a[i], d1);
      else if (!g.diag_one) a[i] = cmul(a[i], d0);
    }
  }
}

static unsigned grid_for(uint64_t work, int threads)
{
  uint64_t b = (work + threads - 1) / threads;
  const uint64_t cap = 148ull * 16;
  if (b > cap) b = cap;
  return (unsigned)(b == 0 ? 1 : b);
}

template <typename Real>
cudaError_t launch_gate(void* state, int n, const gate_rec& g, cudaStream_t stream)
{
  const uint64_t size = 1ull << n;
  gate_kernel<Real><<<grid_for(size >> 1, 256), 256, 0, stream>>>(static_cast<typename ctype<Real>::c*>(state), size, g);
  return cudaGetLastError();
}
template cudaError_t launch_gate<double>(void*, int, const gate_rec&, cudaStream_t);
template cudaError_t launch_gate<float>(void*, int, const gate_rec&, cudaStream_t);

// ---------------------------------------------------------------------------
// Basis-state initialisation
// ---------------------------------------------------------------------------
template <typename Real>
__global__ void set_basis_kernel(typename ctype<Real>::c* a, uint64_t size, uint64_t index)
{
  using C = typename ctype<Real>::c;
  const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
  for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < size; i += stride)
    a[i] = i == index ? C{(Real)1, (Real)0} : C{(Real)0, (Real)0};
}

template <typename Real>
cudaError_t launch_set_basis(void* state, int n, uint64_t index, cudaStream_t stream)
{
  const uint64_t size = 1ull << n;
  set_basis_kernel<Real><<<grid_for(size, 256), 256, 0, stream>>>(static_cast<typename ctype<Real>::c*>(state), size, index);
  return cudaGetLastError();
}
template cudaError_t launch_set_basis<double>(void*, int, uint64_t, cudaStream_t);
template cudaError_t launch_set_basis<float>(void*, int, uint64_t, cudaStream_t);

// ---------------------------------------------------------------------------
// Reductions.  Each block writes `width` doubles of partial sums; one block
// then sums the partials in block order (deterministic for a given grid).
// ---------------------------------------------------------------------------
constexpr int kRedThreads = 256;

__device__ __forceinline__ double warp_sum(double v)
{
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Sums `count` per-thread values over the block; thread 0 writes them to out.
template <int MAXW>
__device__ __forceinline__ void block_sum_store(double* vals, int count, double* out)
{
  __shared__ double red[kRedThreads / 32][MAXW];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int k = 0; k < count; ++k) {
    double v = warp_sum(vals[k]);
    if (lane == 0) red[warp][k] = v;
  }
  __syncthreads();
  if (threadIdx.x < count) {
    double s = 0;
    for (int w = 0; w < kRedThreads / 32; ++w) s += red[w][threadIdx.x];
    out[threadIdx.x] = s;
  }
}

__global__ void finish_partials_kernel(const double* __restrict__ partials, int blocks, int width, double* __restrict__ out)
{
  // One thread per output column; fixed summation order.
  for (int c = threadIdx.x; c < width; c += blockDim.x) {
    double s = 0;
    for (int b = 0; b < blocks; ++b) s += partials[size_t(b) * width + c];
    out[c] = s;
  }
}

// Z sums: out[0] = sum |a|^2, out[1 + q] = sum of |a|^2 over the amplitudes
// whose physical bit q is set.  Launched with exactly 2^kZsumLogThreads
// threads in total, so that bits below kZsumLogThreads of every index a thread
// visits are that thread's global id and only the higher bits vary.
constexpr int kZsumLogThreads = 17;
template <typename Real>
__global__ void __launch_bounds__(kRedThreads) zsum_kernel(const typename ctype<Real>::c* __restrict__ a, int n, double* partials)
{
  constexpr int HI = kMaxQubits - kZsumLogThreads;
  const uint64_t size = 1ull << n;
  const uint64_t gid = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x;
  double total = 0, hi[HI];
#pragma unroll
  for (int k = 0; k < HI; ++k) hi[k] = 0;
  for (uint64_t k = 0; (k << kZsumLogThreads) + gid < size; ++k) {
    const auto v = a[(k << kZsumLogThreads) | gid];
    const double p = double(v.x) * double(v.x) + double(v.y) * double(v.y);
    total += p;
#pragma unroll
    for (int b = 0; b < HI; ++b) if ((k >> b) & 1) hi[b] += p;
  }
  double vals[1 + kMaxQubits];
  vals[0] = total;
  for (int q = 0; q < n; ++q) {
    if (q < kZsumLogThreads) vals[1 + q] = ((gid >> q) & 1) ? total : 0.0;
    else {
      double h = 0;
#pragma unroll
      for (int b = 0; b < HI; ++b) if (b == q - kZsumLogThreads) h = hi[b];
      vals[1 + q] = h;
    }
  }
  block_sum_store<1 + kMaxQubits>(vals, n + 1, partials + size_t(blockIdx.x) * (n + 1));
}

// Pair sums for Pauli strings sharing one flip mask F:
//   out = sum_i conj(a_i) a_{i^F} W(i),  W(i) = sum_t w_t (-1)^popcount(i & s_t)
// with complex weights w_t (terms given in physical bits).  F == 0 is allowed.
template <typename Real>
__global__ void __launch_bounds__(kRedThreads)
pauli_kernel(const typename ctype<Real>::c* __restrict__ a, int n, uint64_t flip,
             const pauli_terms T, double* partials)
{
  const uint64_t size = 1ull << n;
  double re = 0, im = 0;
  const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
  if (flip == 0) {
    for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < size; i += stride) {
      const auto v = a[i];
      const double p = double(v.x) * double(v.x) + double(v.y) * double(v.y);
      double wr = 0, wi = 0;
      for (int t = 0; t < T.count; ++t) {
        const double s = (__popcll(i & T.sign[t]) & 1) ? -1.0 : 1.0;
        wr += s * T.w[t][0]; wi += s * T.w[t][1];
      }
      re += p * wr; im += p * wi;
    }
  } else {
    const int low = __ffsll((long long)flip) - 1;
    for (uint64_t v = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; v < (size >> 1); v += stride) {
      const uint64_t i = insert_zero(v, low), j = i ^ flip;
      const auto ai = a[i], aj = a[j];
      // c = conj(a_i) a_j ;  conj(a_j) a_i = conj(c)
      const double cr = double(ai.x) * double(aj.x) + double(ai.y) * double(aj.y);
      const double ci = double(ai.x) * double(aj.y) - double(ai.y) * double(aj.x);
      for (int t = 0; t < T.count; ++t) {
        const double si = (__popcll(i & T.sign[t]) & 1) ? -1.0 : 1.0;
        const double sj = (__popcll(j & T.sign[t]) & 1) ? -1.0 : 1.0;
        // si * c * w + sj * conj(c) * w   (one-sided: si * c * w)
        const double xr = T.one_sided ? si * cr : si * cr + sj * cr;
        const double xi = T.one_sided ? si * ci : si * ci - sj * ci;
        re += xr * T.w[t][0] - xi * T.w[t][1];
        im += xr * T.w[t][1] + xi * T.w[t][0];
      }
    }
  }
  double vals[2] = {re, im};
  block_sum_store<2>(vals, 2, partials + size_t(blockIdx.x) * 2);
}

// spin_group (rbk_kernels.h): persistent CTAs, one tile at a time, two CTAs
// per SM (one loads while the other sums).  Element j = it * 256 + tid of a
// tile sits at shared-memory slot smem_slot(j) (the fused pass's XOR swizzle,
// linear, so a thread composes slots with XORs and every phase reads without
// bank conflicts).
template <typename Real>
__global__ void __launch_bounds__(kRedThreads, 2)
spins_kernel(const typename ctype<Real>::c* __restrict__ a, const __grid_constant__ spin_group S, uint64_t num_tiles,
             double* partials)
{
  using C = typename ctype<Real>::c;
  constexpr int VB = precision_traits<Real>::VB;
  constexpr int RB = sizeof(Real) == 8 ? 3 : 4, NE = 1 << RB;  // 256 threads x NE = 2^(8 + RB) = the tile
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* tile = reinterpret_cast<C*>(smem_raw);
  const uint32_t tid = threadIdx.x;
  // The thread's parts of addresses, the same for every tile.
  uint64_t tphys = 0;
  for (int b = 0; b < 8; ++b) tphys |= uint64_t((tid >> b) & 1u) << S.tile_phys[b];
  const uint32_t st = smem_slot<VB>(tid);
  uint32_t sbase[kSpinPhases];
#pragma unroll
  for (int p = 0; p < kSpinPhases; ++p) {
    uint32_t j = 0;
    if (p < S.nphases)
      for (int b = 0; b < 8; ++b) j |= ((tid >> b) & 1u) << S.phase_thr[p][b];
    sbase[p] = smem_slot<VB>(j);
  }
  double xr[kMaxSpinFlips], xi[kMaxSpinFlips], z[kMaxSpinFlips];
#pragma unroll
  for (int f = 0; f < kMaxSpinFlips; ++f) xr[f] = xi[f] = z[f] = 0.0;
  double total = 0.0;
  for (uint64_t t = blockIdx.x; t < num_tiles; t += gridDim.x) {
    uint64_t base = tphys;
    for (int r = 0; r < S.num_runs; ++r) base |= ((t >> S.run_src[r]) & ((1ull << S.run_len[r]) - 1)) << S.run_dst[r];
    C v[NE];
#pragma unroll
    for (int it = 0; it < NE; ++it) {
      uint64_t p = base;
#pragma unroll
      for (int b = 0; b < RB; ++b)
        if ((it >> b) & 1) p |= 1ull << S.tile_phys[8 + b];
      v[it] = __ldcs(a + p);
    }
    __syncthreads();  // the previous tile is no longer read
#pragma unroll
    for (int it = 0; it < NE; ++it) {
      tile[st ^ smem_slot<VB>(uint32_t(it) << 8)] = v[it];
      total += double(v[it].x) * double(v[it].x) + double(v[it].y) * double(v[it].y);
    }
    __syncthreads();
#pragma unroll
    for (int p = 0; p < kSpinPhases; ++p) {
      if (p < S.nphases) {
        uint32_t rs[RB];
#pragma unroll
        for (int k = 0; k < RB; ++k) rs[k] = smem_slot<VB>(1u << S.phase_reg[p][k]);
        C e[NE];
#pragma unroll
        for (int i = 0; i < NE; ++i) {
          uint32_t sidx = sbase[p];
#pragma unroll
          for (int k = 0; k < RB; ++k)
            if ((i >> k) & 1) sidx ^= rs[k];
          e[i] = tile[sidx];
        }
#pragma unroll
        for (int k = 0; k < RB; ++k) {
          const int f = p * RB + k;
          if (f < kMaxSpinFlips && f < S.nflips) {
#pragma unroll
            for (int i = 0; i < NE; ++i) {
              if ((i >> k) & 1) continue;
              const C u = e[i], w = e[i | (1 << k)];
              xr[f] += double(u.x) * double(w.x) + double(u.y) * double(w.y);
              xi[f] += double(u.x) * double(w.y) - double(u.y) * double(w.x);
              z[f] += double(w.x) * double(w.x) + double(w.y) * double(w.y);
            }
          }
        }
      }
    }
  }
  // Block sums, in a fixed order, of 3 nflips + 1 values.
  __shared__ double red[kRedThreads / 32][3 * kMaxSpinFlips + 1];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int f = 0; f < kMaxSpinFlips; ++f) {
    if (f < S.nflips) {
      const double a0 = warp_sum(xr[f]), a1 = warp_sum(xi[f]), a2 = warp_sum(z[f]);
      if (lane == 0) { red[warp][3 * f] = a0; red[warp][3 * f + 1] = a1; red[warp][3 * f + 2] = a2; }
    }
  }
  const double tt = warp_sum(total);
  if (lane == 0) red[warp][3 * S.nflips] = tt;
  __syncthreads();
  const int width = 3 * S.nflips + 1;
  for (int k = threadIdx.x; k < width; k += blockDim.x) {
    double acc = 0.0;
    for (int w = 0; w < kRedThreads / 32; ++w) acc += red[w][k];
    partials[size_t(blockIdx.x) * width + k] = acc;
  }
}

// <b| P |a> summed over Pauli strings sharing one flip mask F:
//   out = sum_i conj(b_i) a_{i^F} W(i),  W(i) = sum_t w_t (-1)^popcount(i & s_t)
// ((P a)_i = coeff(i) a_{i^F}, ket/include/ket/gate/utility/pauli_index_coeff.hpp:17-59).
template <typename Real>
__global__ void __launch_bounds__(kRedThreads)
pauli2_kernel(const typename ctype<Real>::c* __restrict__ a, const typename ctype<Real>::c* __restrict__ b, int n,
              uint64_t flip, const pauli_terms T, double* partials)
{
  const uint64_t size = 1ull << n;
  double re = 0, im = 0;
  const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
  for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < size; i += stride) {
    const auto x = a[i ^ flip], y = b[i];
    // c = conj(b_i) a_{i^F}
    const double cr = double(y.x) * double(x.x) + double(y.y) * double(x.y);
    const double ci = double(y.x) * double(x.y) - double(y.y) * double(x.x);
    double wr = 0, wi = 0;
    for (int t = 0; t < T.count; ++t) {
      const double s = (__popcll(i & T.sign[t]) & 1) ? -1.0 : 1.0;
      wr += s * T.w[t][0];
      wi += s * T.w[t][1];
    }
    re += cr * wr - ci * wi;
    im += cr * wi + ci * wr;
  }
  double vals[2] = {re, im};
  block_sum_store<2>(vals, 2, partials + size_t(blockIdx.x) * 2);
}

// <b|a> = sum conj(b_i) a_i
template <typename Real>
__global__ void __launch_bounds__(kRedThreads)
inner_kernel(const typename ctype<Real>::c* __restrict__ a, const typename ctype<Real>::c* __restrict__ b,
             uint64_t size, double* partials)
{
  double re = 0, im = 0;
  const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
  for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < size; i += stride) {
    const auto x = a[i], y = b[i];
    re += double(y.x) * double(x.x) + double(y.y) * double(x.y);
    im += double(y.x) * double(x.y) - double(y.y) * double(x.x);
  }
  double vals[2] = {re, im};
  block_sum_store<2>(vals, 2, partials + size_t(blockIdx.x) * 2);
}

// |a_i|^2 for i in [offset, offset + count) (physical order).
template <typename Real>
__global__ void probs_kernel(const typename ctype<Real>::c* __restrict__ a, uint64_t offset, uint64_t count, double* out)
{
  const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
  for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < count; i += stride) {
    const auto v = a[offset + i];
    out[i] = double(v.x) * double(v.x) + double(v.y) * double(v.y);
  }
}

int reduction_blocks() { return 148 * 4; }

template <typename Real>
cudaError_t launch_zsum(const void* state, int n, double* partials, double* out, cudaStream_t stream)
{
  const int blocks = (1 << kZsumLogThreads) / kRedThreads;
  zsum_kernel<Real><<<blocks, kRedThreads, 0, stream>>>(static_cast<const typename ctype<Real>::c*>(state), n, partials);
  finish_partials_kernel<<<1, 64, 0, stream>>>(partials, blocks, n + 1, out);
  return cudaGetLastError();
}

template <typename Real>
cudaError_t launch_pauli(const void* state, int n, uint64_t flip, const pauli_terms& terms, double* partials, double* out, cudaStream_t stream)
{
  const int blocks = reduction_blocks();
  pauli_kernel<Real><<<blocks, kRedThreads, 0, stream>>>(static_cast<const typename ctype<Real>::c*>(state), n, flip, terms, partials);
  finish_partials_kernel<<<1, 32, 0, stream>>>(partials, blocks, 2, out);
  return cudaGetLastError();
}

template <typename Real>
cudaError_t launch_spins(const void* state, int n, const spin_group& g, double* partials, double* out, cudaStream_t stream)
{
  const int rb = sizeof(Real) == 8 ? 3 : 4;
  if (g.K != 8 + rb || g.K > n || g.nflips < 1 || g.nflips > kMaxSpinFlips || g.nphases < 1 ||
      g.nphases > kSpinPhases || g.nphases * rb < g.nflips)
    return cudaErrorInvalidValue;
  const size_t smem = sizeof(typename ctype<Real>::c) << g.K;
  static std::atomic<bool> configured[64] = {};
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
  if (!configured[dev].load(std::memory_order_acquire)) {
    e = cudaFuncSetAttribute(spins_kernel<Real>, cudaFuncAttributeMaxDynamicSharedMemorySize, 16 << 12);
    if (e != cudaSuccess) return e;
    configured[dev].store(true, std::memory_order_release);
  }
  const uint64_t tiles = 1ull << (n - g.K);
  const int blocks = static_cast<int>(std::min<uint64_t>(tiles, 148 * 2));
  spins_kernel<Real><<<blocks, kRedThreads, smem, stream>>>(static_cast<const typename ctype<Real>::c*>(state), g, tiles, partials);
  finish_partials_kernel<<<1, 64, 0, stream>>>(partials, blocks, 3 * g.nflips + 1, out);
  return cudaGetLastError();
}

template <typename Real>
cudaError_t launch_pauli2(const void* a, const void* b, int n, uint64_t flip, const pauli_terms& terms, double* partials,
                          double* out, cudaStream_t stream)
{
  const int blocks = reduction_blocks();
  pauli2_kernel<Real><<<blocks, kRedThreads, 0, stream>>>(static_cast<const typename ctype<Real>::c*>(a),
                                                          static_cast<const typename ctype<Real>::c*>(b), n, flip, terms, partials);
  finish_partials_kernel<<<1, 32, 0, stream>>>(partials, blocks, 2, out);
  return cudaGetLastError();
}

template <typename Real>
cudaError_t launch_inner(const void* a, const void* b, int n, double* partials, double* out, cudaStream_t stream)
{
  const int blocks = reduction_blocks();
  inner_kernel<Real><<<blocks, kRedThreads, 0, stream>>>(static_cast<const typename ctype<Real>::c*>(a),
                                                         static_cast<const typename ctype<Real>::c*>(b), 1ull << n, partials);
  finish_partials_kernel<<<1, 32, 0, stream>>>(partials, blocks, 2, out);
  return cudaGetLastError();
}

template <typename Real>
cudaError_t launch_probs(const void* state, uint64_t offset, uint64_t count, double* out, cudaStream_t stream)
{
  probs_kernel<Real><<<grid_for(count, 256), 256, 0, stream>>>(static_cast<const typename ctype<Real>::c*>(state), offset, count, out);
  return cudaGetLastError();
}

template cudaError_t launch_zsum<double>(const void*, int, double*, double*, cudaStream_t);
template cudaError_t launch_zsum<float>(const void*, int, double*, double*, cudaStream_t);
template cudaError_t launch_pauli<double>(const void*, int, uint64_t, const pauli_terms&, double*, double*, cudaStream_t);
template cudaError_t launch_pauli<float>(const void*, int, uint64_t, const pauli_terms&, double*, double*, cudaStream_t);
template cudaError_t launch_spins<double>(const void*, int, const spin_group&, double*, double*, cudaStream_t);
template cudaError_t launch_spins<float>(const void*, int, const spin_group&, double*, double*, cudaStream_t);
template cudaError_t launch_pauli2<double>(const void*, const void*, int, uint64_t, const pauli_terms&, double*, double*, cudaStream_t);
template cudaError_t launch_pauli2<float>(const void*, const void*, int, uint64_t, const pauli_terms&, double*, double*, cudaStream_t);
template cudaError_t launch_inner<double>(const void*, const void*, int, double*, double*, cudaStream_t);
template cudaError_t launch_inner<float>(const void*, const void*, int, double*, double*, cudaStream_t);
template cudaError_t launch_probs<double>(const void*, uint64_t, uint64_t, double*, cudaStream_t);
template cudaError_t launch_probs<float>(const void*, uint64_t, uint64_t, double*, cudaStream_t);

}  // namespace rbk

namespace rbk {

// ---------------------------------------------------------------------------
// Adjoint-gradient helpers
// ---------------------------------------------------------------------------

// dst_i = sum_g sum_{t in g} w_t (-1)^popcount(i & sign_t) src_{i ^ flip_g}
// (a Pauli-string sum applied to a state; pauli_index_coeff.hpp:17-59 form).
template <typename Real>
__global__ void pauli_apply_kernel(const typename ctype<Real>::c* __restrict__ src, typename ctype<Real>::c* __restrict__ dst,
                                   uint64_t size, const pauli_sum P)
{
  using C = typename ctype<Real>::c;
  const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
  for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < size; i += stride) {
    double re = 0, im = 0;
    for (int g = 0; g < P.num_groups; ++g) {
      const C v = src[i ^ P.flip[g]];
      double wr = 0, wi = 0;
      for (int t = P.begin[g]; t < P.begin[g + 1]; ++t) {
        const double s = (__popcll(i & P.sign[t]) & 1) ? -1.0 : 1.0;
        wr += s * P.w[t][0];
        wi += s * P.w[t][1];
      }
      re += wr * double(v.x) - wi * double(v.y);
      im += wr * double(v.y) + wi * double(v.x);
    }
    dst[i] = C{(Real)re, (Real)im};
  }
}

// sum_i conj(lam_i) w (-1)^popcount(i & sign) psi_{i ^ flip}: <lam| P |psi> for
// one Pauli string P given as (flip, sign, w) -- the overlap of the adjoint sweep.
template <typename Real>
__global__ void __launch_bounds__(kRedThreads)
overlap_kernel(const typename ctype<Real>::c* __restrict__ lam, const typename ctype<Real>::c* __restrict__ psi,
               uint64_t size, uint64_t flip, uint64_t sign, double wr, double wi, double* partials)
{
  double re = 0, im = 0;
  const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
  for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < size; i += stride) {
    const auto l = lam[i], p = psi[i ^ flip];
    const double s = (__popcll(i & sign) & 1) ? -1.0 : 1.0;
    // conj(l) * p
    const double cr = double(l.x) * double(p.x) + double(l.y) * double(p.y);
    const double ci = double(l.x) * double(p.y) - double(l.y) * double(p.x);
    re += s * (cr * wr - ci * wi);
    im += s * (cr * wi + ci * wr);
  }
  double vals[2] = {re, im};
  block_sum_store<2>(vals, 2, partials + size_t(blockIdx.x) * 2);
}

template <typename Real>
cudaError_t launch_pauli_apply(const void* src, void* dst, int n, const pauli_sum& P, cudaStream_t stream)
{
  const uint64_t size = 1ull << n;
  pauli_apply_kernel<Real><<<grid_for(size, 256), 256, 0, stream>>>(
    static_cast<const typename ctype<Real>::c*>(src), static_cast<typename ctype<Real>::c*>(dst), size, P);
  return cudaGetLastError();
}

// One pass of launch_pauli_apply_tiled: tile bits tile_phys[0..10] (the block
// index deposited run by run into the other bits), the pass's groups as tile
// masks of their flips and their terms.
constexpr int kTileSumTerms = 96;
constexpr int kTileSumBits = 11;
// pair_group >= 0: that group's terms are all two-bit Z-type strings with one
// real weight pw (ZZ couplings), and its weight at j is
//   pw * (count - 2 * (number of pairs with odd parity at j)),
// the pairs on adjacent bits counted at once as popcount((j ^ j >> 1) & madj)
// and the others one by one from other[].
constexpr int kTilePairOthers = 16;
struct pauli_tile_pass {
  int32_t num_groups, first;
  uint8_t tile_phys[16], num_runs, run_src[16], run_len[16], run_dst[16];
  uint8_t begin[kMaxSumGroups + 1];
  uint16_t flip_local[kMaxSumGroups];
  uint64_t sign[kTileSumTerms];
  double w[kTileSumTerms][2];
  int32_t pair_group, pair_count, num_others, pad;
  double pw;
  uint64_t madj;
  uint8_t other[kTilePairOthers][2];
};

// Persistent CTAs, one tile of src at a time in shared memory; thread t holds
// tile indices t + 256 it (it = 0..7), whose partners j ^ flip it reads from
// the tile.  dst is written (first pass) or accumulated, in place.
template <typename Real>
__global__ void __launch_bounds__(kRedThreads)
pauli_apply_tile_kernel(const typename ctype<Real>::c* __restrict__ src, typename ctype<Real>::c* __restrict__ dst,
                        const __grid_constant__ pauli_tile_pass T, uint64_t num_tiles)
{
  using C = typename ctype<Real>::c;
  constexpr int NE = 1 << (kTileSumBits - 8);
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* tile = reinterpret_cast<C*>(smem_raw);
  const uint32_t tid = threadIdx.x;
  uint64_t tphys = 0;
  for (int b = 0; b < 8; ++b) tphys |= uint64_t((tid >> b) & 1u) << T.tile_phys[b];
  for (uint64_t t = blockIdx.x; t < num_tiles; t += gridDim.x) {
    uint64_t base = tphys;
    for (int r = 0; r < T.num_runs; ++r) base |= ((t >> T.run_src[r]) & ((1ull << T.run_len[r]) - 1)) << T.run_dst[r];
    uint64_t phys[NE];
#pragma unroll
    for (int it = 0; it < NE; ++it) {
      phys[it] = base;
#pragma unroll
      for (int b = 0; b < kTileSumBits - 8; ++b)
        if ((it >> b) & 1) phys[it] |= 1ull << T.tile_phys[8 + b];
    }
    // Both loads of the tile issued together: src, and the dst the pass adds to
    // (read here, before any store to dst, so that the loads stay in flight at once).
    C v[NE], d[NE];
#pragma unroll
    for (int it = 0; it < NE; ++it) v[it] = __ldcs(src + phys[it]);
    if (!T.first) {
#pragma unroll
      for (int it = 0; it < NE; ++it) d[it] = __ldcs(dst + phys[it]);
    }
    __syncthreads();  // the previous tile is no longer read
#pragma unroll
    for (int it = 0; it < NE; ++it) tile[tid | (uint32_t(it) << 8)] = v[it];
    __syncthreads();
#pragma unroll
    for (int it = 0; it < NE; ++it) {
      const uint32_t j = tid | (uint32_t(it) << 8);
      double re = 0.0, im = 0.0;
      if (!T.first) {
        re = double(d[it].x);
        im = double(d[it].y);
      }
      for (int g = 0; g < T.num_groups; ++g) {
        const C a = tile[j ^ T.flip_local[g]];
        double wr = 0.0, wi = 0.0;
        if (T.begin[g + 1] == T.begin[g] + 1 && T.sign[T.begin[g]] == 0) {  // one term, no sign bits: a constant weight
          wr = T.w[T.begin[g]][0];
          wi = T.w[T.begin[g]][1];
        } else if (g == T.pair_group) {
          const uint64_t x = phys[it];
          int odd = __popcll((x ^ (x >> 1)) & T.madj);
          for (int k = 0; k < T.num_others; ++k) odd += int(((x >> T.other[k][0]) ^ (x >> T.other[k][1])) & 1);
          wr = T.pw * double(T.pair_count - 2 * odd);
        } else {
          for (int k = T.begin[g]; k < T.begin[g + 1]; ++k) {
            const double sg = (__popcll(phys[it] & T.sign[k]) & 1) ? -1.0 : 1.0;
            wr += sg * T.w[k][0];
            wi += sg * T.w[k][1];
          }
        }
        re += wr * double(a.x) - wi * double(a.y);
        im += wr * double(a.y) + wi * double(a.x);
      }
      v[it] = C{(Real)re, (Real)im};
    }
#pragma unroll
    for (int it = 0; it < NE; ++it) __stcs(dst + phys[it], v[it]);
  }
}

template <typename Real>
cudaError_t launch_pauli_apply_tiled(const void* src, void* dst, int n, const pauli_sum& P, cudaStream_t stream)
{
  constexpr int LOWB = 3, FREE = kTileSumBits - LOWB;
  if (n < kTileSumBits || n > 63) return launch_pauli_apply<Real>(src, dst, n, P, stream);
  // Group the flips into layouts: each layout's high bits (>= LOWB) number at most FREE.
  std::vector<std::vector<int>> passes;
  std::vector<uint64_t> highs;
  int diag = -1;
  for (int g = 0; g < P.num_groups; ++g) {
    const uint64_t f = P.flip[g];
    if (f == 0) { diag = g; continue; }
    const uint64_t hb = f & ~((1ull << LOWB) - 1);
    if (__builtin_popcountll(hb) > FREE) return launch_pauli_apply<Real>(src, dst, n, P, stream);
    bool placed = false;
    for (size_t q = 0; q < passes.size() && !placed; ++q) {
      int terms = 0;
      for (int h : passes[q]) terms += P.begin[h + 1] - P.begin[h];
      if (__builtin_popcountll(highs[q] | hb) <= FREE && terms + (P.begin[g + 1] - P.begin[g]) <= kTileSumTerms &&
          static_cast<int>(passes[q].size()) < kMaxSumGroups) {
        passes[q].push_back(g);
        highs[q] |= hb;
        placed = true;
      }
    }
    if (!placed) { passes.push_back({g}); highs.push_back(hb); }
  }
  if (passes.empty()) { passes.push_back({}); highs.push_back(0); }
  if (diag >= 0) {
    int terms = P.begin[diag + 1] - P.begin[diag];
    for (int h : passes[0]) terms += P.begin[h + 1] - P.begin[h];
    if (terms > kTileSumTerms) return launch_pauli_apply<Real>(src, dst, n, P, stream);
    passes[0].insert(passes[0].begin(), diag);
  }
  static std::atomic<bool> configured[64] = {};
  const size_t smem = sizeof(typename ctype<Real>::c) << kTileSumBits;
  int dev = 0, sms = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
  if (!configured[dev].load(std::memory_order_acquire)) {
    e = cudaFuncSetAttribute(pauli_apply_tile_kernel<Real>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    configured[dev].store(true, std::memory_order_release);
  }
  e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (e != cudaSuccess) return e;
  const uint64_t tiles = 1ull << (n - kTileSumBits);
  const int blocks = static_cast<int>(std::min<uint64_t>(tiles, uint64_t(sms) * 4));
  for (size_t q = 0; q < passes.size(); ++q) {
    pauli_tile_pass T{};
    T.first = q == 0 ? 1 : 0;
    std::vector<int> bits;
    for (int b = 0; b < LOWB; ++b) bits.push_back(b);
    for (int b = LOWB; b < n; ++b)
      if ((highs[q] >> b) & 1) bits.push_back(b);
    for (int b = LOWB; static_cast<int>(bits.size()) < kTileSumBits; ++b)  // fillers
      if (!((highs[q] >> b) & 1)) bits.push_back(b);
    std::sort(bits.begin(), bits.end());
    uint64_t mask = 0;
    for (int b = 0; b < kTileSumBits; ++b) { T.tile_phys[b] = static_cast<uint8_t>(bits[static_cast<size_t>(b)]); mask |= 1ull << bits[static_cast<size_t>(b)]; }
    int runs = 0, srcb = 0;
    for (int b = 0; b < n;) {
      if ((mask >> b) & 1) { ++b; continue; }
      int len = 0;
      while (b + len < n && !((mask >> (b + len)) & 1)) ++len;
      T.run_src[runs] = static_cast<uint8_t>(srcb);
      T.run_len[runs] = static_cast<uint8_t>(len);
      T.run_dst[runs] = static_cast<uint8_t>(b);
      ++runs;
      srcb += len;
      b += len;
    }
    T.num_runs = static_cast<uint8_t>(runs);
    int k = 0;
    T.num_groups = static_cast<int>(passes[q].size());
    for (int gi = 0; gi < T.num_groups; ++gi) {
      const int g = passes[q][static_cast<size_t>(gi)];
      uint32_t fl = 0;
      for (int b = 0; b < kTileSumBits; ++b)
        if ((P.flip[g] >> T.tile_phys[b]) & 1) fl |= 1u << b;
      T.flip_local[gi] = static_cast<uint16_t>(fl);
      T.begin[gi] = static_cast<uint8_t>(k);
      for (int t = P.begin[g]; t < P.begin[g + 1]; ++t, ++k) {
        T.sign[k] = P.sign[t];
        T.w[k][0] = P.w[t][0];
        T.w[k][1] = P.w[t][1];
      }
    }
    T.begin[T.num_groups] = static_cast<uint8_t>(k);
    // The ZZ-coupling form of the diagonal group, where it applies.
    T.pair_group = -1;
    if (q == 0 && diag >= 0 && P.begin[diag + 1] > P.begin[diag]) {
      const int t0 = P.begin[diag], t1 = P.begin[diag + 1];
      bool pairs = true;
      uint64_t madj = 0;
      int others = 0;
      for (int t = t0; t < t1 && pairs; ++t) {
        const uint64_t sg = P.sign[t];
        pairs = __builtin_popcountll(sg) == 2 && P.w[t][1] == 0.0 && P.w[t][0] == P.w[t0][0];
        if (!pairs) break;
        const int a = __builtin_ctzll(sg), b = 63 - __builtin_clzll(sg);
        if (b == a + 1 && !((madj >> a) & 1)) {
          madj |= 1ull << a;
        } else if (others < kTilePairOthers) {
          T.other[others][0] = static_cast<uint8_t>(a);
          T.other[others][1] = static_cast<uint8_t>(b);
          ++others;
        } else {
          pairs = false;
        }
      }
      if (pairs) {
        T.pair_group = 0;  // the diagonal group is the pass's first
        T.pair_count = t1 - t0;
        T.pw = P.w[t0][0];
        T.madj = madj;
        T.num_others = others;
      }
    }
    pauli_apply_tile_kernel<Real><<<blocks, kRedThreads, smem, stream>>>(
      static_cast<const typename ctype<Real>::c*>(src), static_cast<typename ctype<Real>::c*>(dst), T, tiles);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}
template cudaError_t launch_pauli_apply_tiled<double>(const void*, void*, int, const pauli_sum&, cudaStream_t);
template cudaError_t launch_pauli_apply_tiled<float>(const void*, void*, int, const pauli_sum&, cudaStream_t);

template <typename Real>
cudaError_t launch_overlap(const void* lam, const void* psi, int n, uint64_t flip, uint64_t sign, double wr, double wi,
                           double* partials, double* out, cudaStream_t stream)
{
  const int blocks = reduction_blocks();
  overlap_kernel<Real><<<blocks, kRedThreads, 0, stream>>>(static_cast<const typename ctype<Real>::c*>(lam),
                                                           static_cast<const typename ctype<Real>::c*>(psi), 1ull << n,
                                                           flip, sign, wr, wi, partials);
  finish_partials_kernel<<<1, 32, 0, stream>>>(partials, blocks, 2, out);
  return cudaGetLastError();
}

// Several overlaps in one launch: blockIdx.y selects the Pauli of overlap y;
// partials of overlap y sit at partials[(y * gridDim.x + x) * 2].
template <typename Real>
__global__ void __launch_bounds__(kRedThreads)
overlaps_kernel(const typename ctype<Real>::c* __restrict__ lam, const typename ctype<Real>::c* __restrict__ psi,
                uint64_t size, const __grid_constant__ overlap_set S, double* partials)
{
  const overlap_spec P = S.spec[blockIdx.y];
  double re = 0, im = 0;
  const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
  for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < size; i += stride) {
    const auto l = lam[i], p = psi[i ^ P.flip];
    const double s = (__popcll(i & P.sign) & 1) ? -1.0 : 1.0;
    const double cr = double(l.x) * double(p.x) + double(l.y) * double(p.y);
    const double ci = double(l.x) * double(p.y) - double(l.y) * double(p.x);
    re += s * (cr * P.wr - ci * P.wi);
    im += s * (cr * P.wi + ci * P.wr);
  }
  double vals[2] = {re, im};
  block_sum_store<2>(vals, 2, partials + (size_t(blockIdx.y) * gridDim.x + blockIdx.x) * 2);
}

// Sum of the (re, im) partials p[0..blocks) by one warp: lane l takes blocks
// l, l + 32, ... in order, then a fixed butterfly adds the lanes.  The order is
// the same on every run; the loads of a lane are independent, so the sum costs
// a few L2 round trips instead of one per block.
__device__ __forceinline__ double2 warp_sum_partials(const double* __restrict__ p, int blocks)
{
  const int lane = threadIdx.x & 31;
  double re = 0, im = 0;
  for (int b = lane; b < blocks; b += 32) {
    re += p[2 * b];
    im += p[2 * b + 1];
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    re += __shfl_xor_sync(0xffffffffu, re, o);
    im += __shfl_xor_sync(0xffffffffu, im, o);
  }
  return make_double2(re, im);
}

// out[2y], out[2y+1] = sum over the partials of overlap y (one warp per overlap).
__global__ void finish_overlaps_kernel(const double* __restrict__ partials, int blocks, double* __restrict__ out)
{
  const double2 v = warp_sum_partials(partials + size_t(blockIdx.x) * blocks * 2, blocks);
  if (threadIdx.x == 0) {
    out[2 * blockIdx.x] = v.x;
    out[2 * blockIdx.x + 1] = v.y;
  }
}

size_t overlaps_partials_doubles() { return size_t(reduction_blocks()) * 2 * kMaxOverlaps; }

template <typename Real>
cudaError_t launch_overlaps(const void* lam, const void* psi, int n, const overlap_set& set, double* partials, double* out,
                            cudaStream_t stream)
{
  if (set.count < 1 || set.count > kMaxOverlaps) return cudaErrorInvalidValue;
  const int blocks = reduction_blocks();
  overlaps_kernel<Real><<<dim3(blocks, set.count), kRedThreads, 0, stream>>>(
    static_cast<const typename ctype<Real>::c*>(lam), static_cast<const typename ctype<Real>::c*>(psi), 1ull << n, set,
    partials);
  finish_overlaps_kernel<<<set.count, 32, 0, stream>>>(partials, blocks, out);
  return cudaGetLastError();
}
// Tiled form: CTA b stages the tile of psi and lambda whose bits outside
// T.tile_phys spell b (as a fused pass does) and evaluates every overlap of
// the set whose flip bit is a tile bit, reading each state once for the whole
// set instead of once per overlap.
template <typename Real>
__global__ void __launch_bounds__(kRedThreads)
tile_overlaps_kernel(const typename ctype<Real>::c* __restrict__ lam, const typename ctype<Real>::c* __restrict__ psi,
                     const __grid_constant__ tile_overlap_set T, double* partials)
{
  using C = typename ctype<Real>::c;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* ps = reinterpret_cast<C*>(smem_raw);
  C* ls = ps + (1u << T.K);
  __shared__ double red[kMaxOverlaps][kRedThreads / 32][2];
  const uint32_t tile = 1u << T.K;
  uint64_t base = 0;
  {
    const uint64_t b = blockIdx.x;
    for (int r = 0; r < T.num_runs; ++r) base |= ((b >> T.run_src[r]) & ((1ull << T.run_len[r]) - 1)) << T.run_dst[r];
  }
  auto phys_of = [&](uint32_t j) {
    uint64_t p = base;
    for (int b = 0; b < T.K; ++b) p |= uint64_t((j >> b) & 1u) << T.tile_phys[b];
    return p;
  };
  for (uint32_t j = threadIdx.x; j < tile; j += blockDim.x) {
    const uint64_t p = phys_of(j);
    ps[j] = psi[p];
    ls[j] = lam[p];
  }
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int y = 0; y < T.count; ++y) {
    const tile_overlap_spec S = T.spec[y];
    const double base_sign = (__popcll(base & S.sign) & 1) ? -1.0 : 1.0;
    double re = 0, im = 0;
    for (uint32_t j = threadIdx.x; j < tile; j += blockDim.x) {
      const C l = ls[j], p = ps[j ^ S.flip_local];
      const double s = (__popc(j & S.sign_local) & 1) ? -base_sign : base_sign;
      const double cr = double(l.x) * double(p.x) + double(l.y) * double(p.y);
      const double ci = double(l.x) * double(p.y) - double(l.y) * double(p.x);
      re += s * (cr * S.wr - ci * S.wi);
      im += s * (cr * S.wi + ci * S.wr);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      re += __shfl_xor_sync(0xffffffffu, re, o);
      im += __shfl_xor_sync(0xffffffffu, im, o);
    }
    if (lane == 0) { red[y][warp][0] = re; red[y][warp][1] = im; }
  }
  __syncthreads();
  for (int y = threadIdx.x; y < T.count; y += blockDim.x) {
    double re = 0, im = 0;
    for (int w = 0; w < kRedThreads / 32; ++w) { re += red[y][w][0]; im += red[y][w][1]; }
    partials[(size_t(y) * gridDim.x + blockIdx.x) * 2] = re;
    partials[(size_t(y) * gridDim.x + blockIdx.x) * 2 + 1] = im;
  }
}

__global__ void finish_tile_overlaps_kernel(const double* __restrict__ partials, int blocks,
                                            const __grid_constant__ tile_overlap_set T, double* __restrict__ out)
{
  const double2 v = warp_sum_partials(partials + size_t(blockIdx.x) * blocks * 2, blocks);
  if (threadIdx.x == 0) {
    out[2 * T.spec[blockIdx.x].out_slot] = v.x;
    out[2 * T.spec[blockIdx.x].out_slot + 1] = v.y;
  }
}

size_t tile_overlaps_partials_doubles(int n, int K) { return (size_t(1) << (n > K ? n - K : 0)) * 2 * kMaxOverlaps; }

template <typename Real>
cudaError_t launch_tile_overlaps(const void* lam, const void* psi, int n, const tile_overlap_set& set, double* partials,
                                 double* out, cudaStream_t stream)
{
  if (set.count < 1 || set.count > kMaxOverlaps || n < set.K) return cudaErrorInvalidValue;
  const size_t smem = 2 * sizeof(typename ctype<Real>::c) << set.K;
  static std::atomic<bool> configured[64] = {};
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
  if (!configured[dev].load(std::memory_order_acquire)) {
    e = cudaFuncSetAttribute(tile_overlaps_kernel<Real>, cudaFuncAttributeMaxDynamicSharedMemorySize, 2 * (16 << 12));
    if (e != cudaSuccess) return e;
    configured[dev].store(true, std::memory_order_release);
  }
  const unsigned tiles = unsigned(1ull << (n - set.K));
  tile_overlaps_kernel<Real><<<tiles, kRedThreads, smem, stream>>>(static_cast<const typename ctype<Real>::c*>(lam),
                                                                  static_cast<const typename ctype<Real>::c*>(psi), set,
                                                                  partials);
  finish_tile_overlaps_kernel<<<set.count, 32, 0, stream>>>(partials, int(tiles), set, out);
  return cudaGetLastError();
}
// zsum2_set (rbk_kernels.h): exactly 2^kZsumLogThreads threads, thread gid
// visiting indices (k << kZsumLogThreads) | gid as in zsum_kernel.  Per block
// the partial sums of c_j = conj(lam_j) psi_j: the total, then for every bit q
// the sum over j with bit q set.  k runs in groups of 8 where it can: the
// group's three low bits of k are known at compile time, and its higher bits
// add the group's sum once instead of once per amplitude.
template <typename Real>
__global__ void __launch_bounds__(kRedThreads)
zsum2_kernel(const typename ctype<Real>::c* __restrict__ lam, const typename ctype<Real>::c* __restrict__ psi, int n,
             double* partials)
{
  constexpr int HI = kMaxQubits - kZsumLogThreads;
  const uint64_t size = 1ull << n;
  const uint64_t gid = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x;
  double tr = 0, ti = 0, hr[HI], hi[HI];
#pragma unroll
  for (int k = 0; k < HI; ++k) hr[k] = hi[k] = 0;
  const uint64_t ks = size >> kZsumLogThreads;  // k values of every thread (n >= kZsumLogThreads)
  if (ks >= 8) {
    for (uint64_t m = 0; m < ks / 8; ++m) {
      double gr = 0, gi = 0, r0 = 0, i0 = 0, r1 = 0, i1 = 0, r2 = 0, i2 = 0;
#pragma unroll
      for (int r = 0; r < 8; ++r) {
        const uint64_t j = ((m * 8 + r) << kZsumLogThreads) | gid;
        const auto l = __ldcs(lam + j), p = __ldcs(psi + j);
        const double cr = double(l.x) * double(p.x) + double(l.y) * double(p.y);
        const double ci = double(l.x) * double(p.y) - double(l.y) * double(p.x);
        gr += cr;
        gi += ci;
        if (r & 1) { r0 += cr; i0 += ci; }
        if (r & 2) { r1 += cr; i1 += ci; }
        if (r & 4) { r2 += cr; i2 += ci; }
      }
      tr += gr;
      ti += gi;
      hr[0] += r0; hi[0] += i0;
      hr[1] += r1; hi[1] += i1;
      hr[2] += r2; hi[2] += i2;
#pragma unroll
      for (int b = 3; b < HI; ++b)
        if ((m >> (b - 3)) & 1) { hr[b] += gr; hi[b] += gi; }
    }
  } else {
    for (uint64_t k = 0; (k << kZsumLogThreads) + gid < size; ++k) {
      const uint64_t j = (k << kZsumLogThreads) | gid;
      const auto l = __ldcs(lam + j), p = __ldcs(psi + j);
      const double cr = double(l.x) * double(p.x) + double(l.y) * double(p.y);
      const double ci = double(l.x) * double(p.y) - double(l.y) * double(p.x);
      tr += cr;
      ti += ci;
#pragma unroll
      for (int b = 0; b < HI; ++b)
        if ((k >> b) & 1) { hr[b] += cr; hi[b] += ci; }
    }
  }
  double vals[2 * (1 + kMaxQubits)];
  vals[0] = tr;
  vals[1] = ti;
  for (int q = 0; q < n; ++q) {
    double a = 0, c = 0;
    if (q < kZsumLogThreads) {
      if ((gid >> q) & 1) { a = tr; c = ti; }
    } else {
#pragma unroll
      for (int b = 0; b < HI; ++b)
        if (b == q - kZsumLogThreads) { a = hr[b]; c = hi[b]; }
    }
    vals[2 + 2 * q] = a;
    vals[3 + 2 * q] = c;
  }
  block_sum_store<2 * (1 + kMaxQubits)>(vals, 2 * (n + 1), partials + size_t(blockIdx.x) * 2 * (n + 1));
}

// One warp per entry: S_q = total - 2 (sum over bit q set), out = w S_q.
__global__ void finish_zsum2_kernel(const double* __restrict__ partials, int blocks, int n,
                                    const __grid_constant__ zsum2_set set, double* __restrict__ out)
{
  const int lane = threadIdx.x & 31, width = 2 * (n + 1);
  const int q = set.spec[blockIdx.x].bit;
  double tr = 0, ti = 0, or_ = 0, oi = 0;
  for (int b = lane; b < blocks; b += 32) {
    const double* p = partials + size_t(b) * width;
    tr += p[0];
    ti += p[1];
    or_ += p[2 + 2 * q];
    oi += p[3 + 2 * q];
  }
  tr = warp_sum(tr);
  ti = warp_sum(ti);
  or_ = warp_sum(or_);
  oi = warp_sum(oi);
  if (lane == 0) {
    const double sr = tr - 2.0 * or_, si = ti - 2.0 * oi;
    const double wr = set.spec[blockIdx.x].wr, wi = set.spec[blockIdx.x].wi;
    const int slot = set.spec[blockIdx.x].out_slot;
    out[2 * slot] = sr * wr - si * wi;
    out[2 * slot + 1] = sr * wi + si * wr;
  }
}

template <typename Real>
cudaError_t launch_zsum2(const void* lam, const void* psi, int n, const zsum2_set& set, double* partials, double* out,
                         cudaStream_t stream)
{
  if (set.count < 1 || set.count > kMaxOverlaps || n < 1 || n > kMaxQubits) return cudaErrorInvalidValue;
  for (int y = 0; y < set.count; ++y)
    if (set.spec[y].bit < 0 || set.spec[y].bit >= n) return cudaErrorInvalidValue;
  const int blocks = (1 << kZsumLogThreads) / kRedThreads;
  zsum2_kernel<Real><<<blocks, kRedThreads, 0, stream>>>(static_cast<const typename ctype<Real>::c*>(lam),
                                                          static_cast<const typename ctype<Real>::c*>(psi), n, partials);
  finish_zsum2_kernel<<<set.count, 32, 0, stream>>>(partials, blocks, n, set, out);
  return cudaGetLastError();
}

// pair_overlap_set (rbk_kernels.h): persistent CTAs, two per SM, each taking
// tiles blockIdx.x, + gridDim.x, ...; both states' tiles of 2^11 amplitudes
// sit in shared memory at the fused pass's swizzled slots.  In register phase
// p a thread holds the 8 amplitudes of each state whose tile bits
// phase_reg[p][0..2] vary; flip f = 3 p + k is register bit k of phase p.
constexpr int kPairBlocksPerSm = 2;
template <typename Real>
__global__ void __launch_bounds__(kRedThreads, kPairBlocksPerSm)
pair_overlaps_kernel(const typename ctype<Real>::c* __restrict__ lam, const typename ctype<Real>::c* __restrict__ psi,
                     const __grid_constant__ pair_overlap_set PS, uint64_t num_tiles, double* partials)
{
  const spin_group& S = PS.g;
  using C = typename ctype<Real>::c;
  constexpr int VB = precision_traits<Real>::VB;
  constexpr int RB = kPairRegBits, NE = 1 << RB, KT = 8 + RB;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* tl = reinterpret_cast<C*>(smem_raw);
  C* tp = tl + (1u << KT);
  const uint32_t tid = threadIdx.x;
  uint64_t tphys = 0;
  for (int b = 0; b < 8; ++b) tphys |= uint64_t((tid >> b) & 1u) << S.tile_phys[b];
  const uint32_t st = smem_slot<VB>(tid);
  uint32_t sbase[kSpinPhases];
#pragma unroll
  for (int p = 0; p < kSpinPhases; ++p) {
    uint32_t j = 0;
    if (p < S.nphases)
      for (int b = 0; b < 8; ++b) j |= ((tid >> b) & 1u) << S.phase_thr[p][b];
    sbase[p] = smem_slot<VB>(j);
  }
  // A_f + s_f B_f per flip (s_f = -1 for Y type), which is all the result needs.
  double xr[kMaxPairFlips], xi[kMaxPairFlips];
#pragma unroll
  for (int f = 0; f < kMaxPairFlips; ++f) xr[f] = xi[f] = 0.0;
  for (uint64_t t = blockIdx.x; t < num_tiles; t += gridDim.x) {
    uint64_t base = tphys;
    for (int r = 0; r < S.num_runs; ++r) base |= ((t >> S.run_src[r]) & ((1ull << S.run_len[r]) - 1)) << S.run_dst[r];
    C vl[NE], vp[NE];
#pragma unroll
    for (int it = 0; it < NE; ++it) {
      uint64_t p = base;
#pragma unroll
      for (int b = 0; b < RB; ++b)
        if ((it >> b) & 1) p |= 1ull << S.tile_phys[8 + b];
      vl[it] = __ldcs(lam + p);
      vp[it] = __ldcs(psi + p);
    }
    __syncthreads();  // the previous tile is no longer read
#pragma unroll
    for (int it = 0; it < NE; ++it) {
      const uint32_t s = st ^ smem_slot<VB>(uint32_t(it) << 8);
      tl[s] = vl[it];
      tp[s] = vp[it];
    }
    __syncthreads();
#pragma unroll
    for (int p = 0; p < kSpinPhases; ++p) {
      if (p < S.nphases) {
        uint32_t rs[RB];
#pragma unroll
        for (int k = 0; k < RB; ++k) rs[k] = smem_slot<VB>(1u << S.phase_reg[p][k]);
        C el[NE], ep[NE];
#pragma unroll
        for (int i = 0; i < NE; ++i) {
          uint32_t sidx = sbase[p];
#pragma unroll
          for (int k = 0; k < RB; ++k)
            if ((i >> k) & 1) sidx ^= rs[k];
          el[i] = tl[sidx];
          ep[i] = tp[sidx];
        }
#pragma unroll
        for (int k = 0; k < RB; ++k) {
          const int f = p * RB + k;
          if (f < kMaxPairFlips && f < S.nflips) {
            const double s = PS.flip[f].minus ? -1.0 : 1.0;
#pragma unroll
            for (int i = 0; i < NE; ++i) {
              if ((i >> k) & 1) continue;
              const C l0 = el[i], l1 = el[i | (1 << k)], p0 = ep[i], p1 = ep[i | (1 << k)];
              const double ar = double(l0.x) * double(p1.x) + double(l0.y) * double(p1.y);
              const double ai = double(l0.x) * double(p1.y) - double(l0.y) * double(p1.x);
              const double br = double(l1.x) * double(p0.x) + double(l1.y) * double(p0.y);
              const double bi = double(l1.x) * double(p0.y) - double(l1.y) * double(p0.x);
              xr[f] += __fma_rn(s, br, ar);
              xi[f] += __fma_rn(s, bi, ai);
            }
          }
        }
      }
    }
  }
  // Block sums, in a fixed order: A_f + s_f B_f as 2 doubles per flip.
  __shared__ double red[kRedThreads / 32][2 * kMaxPairFlips];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int f = 0; f < kMaxPairFlips; ++f) {
    if (f < S.nflips) {
      const double a0 = warp_sum(xr[f]), a1 = warp_sum(xi[f]);
      if (lane == 0) { red[warp][2 * f] = a0; red[warp][2 * f + 1] = a1; }
    }
  }
  __syncthreads();
  const int width = 2 * S.nflips;
  for (int k = threadIdx.x; k < width; k += blockDim.x) {
    double acc = 0.0;
    for (int w = 0; w < kRedThreads / 32; ++w) acc += red[w][k];
    partials[size_t(blockIdx.x) * width + k] = acc;
  }
}

// One warp per flip: A + s B over the blocks, then out = w (A + s B).
__global__ void finish_pair_overlaps_kernel(const double* __restrict__ partials, int blocks, int nflips,
                                            const __grid_constant__ pair_overlap_set set, double* __restrict__ out)
{
  const int lane = threadIdx.x & 31, f = blockIdx.x, width = 2 * nflips;
  double xr = 0, xi = 0;
  for (int b = lane; b < blocks; b += 32) {
    xr += partials[size_t(b) * width + 2 * f];
    xi += partials[size_t(b) * width + 2 * f + 1];
  }
  xr = warp_sum(xr);
  xi = warp_sum(xi);
  if (lane == 0) {
    const double wr = set.flip[f].wr, wi = set.flip[f].wi;
    const int slot = set.flip[f].out_slot;
    out[2 * slot] = xr * wr - xi * wi;
    out[2 * slot + 1] = xr * wi + xi * wr;
  }
}

size_t pair_overlaps_partials_doubles() { return size_t(148) * kPairBlocksPerSm * 2 * kMaxPairFlips; }

template <typename Real>
cudaError_t launch_pair_overlaps(const void* lam, const void* psi, int n, const pair_overlap_set& set, double* partials,
                                 double* out, cudaStream_t stream)
{
  const spin_group& g = set.g;
  if (g.K != 8 + kPairRegBits || g.K > n || g.nflips < 1 || g.nflips > kMaxPairFlips || g.nphases < 1 ||
      g.nphases > kSpinPhases || g.nphases * kPairRegBits < g.nflips)
    return cudaErrorInvalidValue;
  const size_t smem = 2 * sizeof(typename ctype<Real>::c) << g.K;
  static std::atomic<bool> configured[64] = {};
  int dev = 0, sms = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
  if (!configured[dev].load(std::memory_order_acquire)) {
    e = cudaFuncSetAttribute(pair_overlaps_kernel<Real>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    configured[dev].store(true, std::memory_order_release);
  }
  e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (e != cudaSuccess) return e;
  const uint64_t tiles = 1ull << (n - g.K);
  // Capped at 148 SMs' worth: the partials buffer is sized for that.
  const int blocks = static_cast<int>(std::min<uint64_t>(tiles, uint64_t(std::min(sms, 148)) * kPairBlocksPerSm));
  pair_overlaps_kernel<Real><<<blocks, kRedThreads, smem, stream>>>(static_cast<const typename ctype<Real>::c*>(lam),
                                                                   static_cast<const typename ctype<Real>::c*>(psi), set, tiles,
                                                                   partials);
  finish_pair_overlaps_kernel<<<g.nflips, 32, 0, stream>>>(partials, blocks, g.nflips, set, out);
  return cudaGetLastError();
}
// pair_rotate_set (rbk_kernels.h): the tile traffic of pair_overlaps_kernel
// plus a write-back.  Per tile: both states' tiles into shared memory; in each
// register phase the overlaps of the phase's flips, then their gates on both
// states in registers, written back to the same slots; after the last phase
// the tiles go back to HBM where they came from.
template <typename Real>
__global__ void __launch_bounds__(kRedThreads, kPairBlocksPerSm)
pair_rotate_kernel(typename ctype<Real>::c* __restrict__ lam, typename ctype<Real>::c* __restrict__ psi,
                   const __grid_constant__ pair_rotate_set PS, uint64_t num_tiles, double* partials)
{
  const spin_group& S = PS.g;
  using C = typename ctype<Real>::c;
  constexpr int VB = precision_traits<Real>::VB;
  constexpr int RB = kPairRegBits, NE = 1 << RB, KT = 8 + RB;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* tl = reinterpret_cast<C*>(smem_raw);
  C* tp = tl + (1u << KT);
  // Im(w_f (A_f + s_f B_f)) per flip and thread, kept in shared memory between
  // tiles to spare registers.
  __shared__ double acc[kMaxRotFlips][kRedThreads];
  const uint32_t tid = threadIdx.x;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int f = 0; f < kMaxRotFlips; ++f) acc[f][tid] = 0.0;
  uint64_t tphys = 0;
  for (int b = 0; b < 8; ++b) tphys |= uint64_t((tid >> b) & 1u) << S.tile_phys[b];
  const uint32_t st = smem_slot<VB>(tid);
  // Pre-step state (PS.pre): the diagonal's factor over this thread's tile bits
  // and over each register slot's bits; Z sums per thread (total and register
  // bits) and per warp (bits outside the tile).
  const pre_diag& D = PS.pre;
  __shared__ double2 fthr[kRedThreads], freg[1 << kPairRegBits];
  __shared__ uint64_t mthr[kRedThreads];  // partner row of this thread's tile bits, XORed; bit 63: their pair parity
  __shared__ double zt[4][kRedThreads];
  __shared__ double zh[kMaxQubits][kRedThreads / 32];
  if (D.active) {
    double2 f{1.0, 0.0};
    for (int b = 0; b < 8; ++b)
      if ((tid >> b) & 1) f = cmul(f, double2{D.u[S.tile_phys[b]][0], D.u[S.tile_phys[b]][1]});
    fthr[tid] = f;
    uint64_t m = 0;
    uint32_t qt = 0;
    for (int b = 0; b < 8; ++b)
      if ((tid >> b) & 1) {
        m ^= D.full[S.tile_phys[b]];
        qt ^= __popcll(tphys & D.adj[S.tile_phys[b]]);
      }
    mthr[tid] = (m & ~(1ull << 63)) | (uint64_t(qt & 1u) << 63);
    if (tid < (1u << kPairRegBits)) {
      double2 r{1.0, 0.0};
      for (int b = 0; b < kPairRegBits; ++b)
        if ((tid >> b) & 1) r = cmul(r, double2{D.u[S.tile_phys[8 + b]][0], D.u[S.tile_phys[8 + b]][1]});
      freg[tid] = r;
    }
    for (int k = 0; k < 4; ++k) zt[k][tid] = 0.0;
    for (int q = tid; q < kMaxQubits * (kRedThreads / 32); q += kRedThreads) zh[q / (kRedThreads / 32)][q % (kRedThreads / 32)] = 0.0;
    __syncthreads();
  }
  auto tile_base = [&](uint64_t t) {
    uint64_t b = tphys;
    for (int r = 0; r < S.num_runs; ++r) b |= ((t >> S.run_src[r]) & ((1ull << S.run_len[r]) - 1)) << S.run_dst[r];
    return b;
  };
  // Phase 0 is the load layout (register bits = tile bits 8..10, thread bits
  // 0..7): a tile goes from HBM straight into its registers.  The next tile's
  // loads are issued before this tile's store, so that they are in flight
  // while the store runs.
  C el[NE], ep[NE];
  auto load_tile = [&](uint64_t b) {
#pragma unroll
    for (int it = 0; it < NE; ++it) {
      uint64_t p = b;
#pragma unroll
      for (int k = 0; k < RB; ++k)
        if ((it >> k) & 1) p |= 1ull << S.tile_phys[8 + k];
      el[it] = __ldcs(lam + p);
      ep[it] = __ldcs(psi + p);
    }
  };
  if (blockIdx.x < num_tiles) load_tile(tile_base(blockIdx.x));
  for (uint64_t t = blockIdx.x; t < num_tiles; t += gridDim.x) {
    const uint64_t base = tile_base(t);
    {
      C* vl = el;
      C* vp = ep;
      if (D.active) {
        if (D.nz > 0) {
          // Im conj(lam_j) psi_j: thread total, register-bit sums, and the warp's
          // total for the bits outside the tile that are set in this tile.
          double tot = 0.0, r0 = 0.0, r1 = 0.0, r2 = 0.0;
#pragma unroll
          for (int it = 0; it < NE; ++it) {
            const double c = double(vl[it].x) * double(vp[it].y) - double(vl[it].y) * double(vp[it].x);
            tot += c;
            if (it & 1) r0 += c;
            if (it & 2) r1 += c;
            if (it & 4) r2 += c;
          }
          zt[0][tid] += tot;
          zt[1][tid] += r0;
          zt[2][tid] += r1;
          zt[3][tid] += r2;
          const double wtot = warp_sum(tot);
          if (lane == 0)
            for (uint64_t hb = base ^ tphys; hb; hb &= hb - 1) zh[__ffsll(static_cast<long long>(hb)) - 1][warp] += wtot;
        }
        // The diagonal: g times u over the set bits, times (-1)^Q.
        double2 f{D.g[0], D.g[1]};
        for (uint64_t hb = base ^ tphys; hb; hb &= hb - 1) {
          const int q = __ffsll(static_cast<long long>(hb)) - 1;
          f = cmul(f, double2{D.u[q][0], D.u[q][1]});
        }
        f = cmul(f, fthr[tid]);
        // Q(base) = Q(bits outside the tile) ^ Q(thread bits) ^ their cross
        // pairs; the first is the same for the whole CTA (uniform loop).
        const uint64_t hbase = base ^ tphys;
        uint32_t qb = 0;
        for (uint64_t hb = hbase; hb; hb &= hb - 1) qb ^= __popcll(hbase & D.adj[__ffsll(static_cast<long long>(hb)) - 1]);
        const uint64_t mt = mthr[tid];
        qb ^= uint32_t(mt >> 63) ^ __popcll(hbase & mt & ~(1ull << 63));
#pragma unroll
        for (int it = 0; it < NE; ++it) {
          double2 fi = cmul(f, freg[it]);
          if ((qb ^ (D.qr >> it) ^ __popcll(base & D.mr[it])) & 1) fi = double2{-fi.x, -fi.y};
          const C fc{Real(fi.x), Real(fi.y)};
          vl[it] = cmul(vl[it], fc);
          vp[it] = cmul(vp[it], fc);
        }
      }
      // The previous tile's last shared-memory reads (its store, in the load
      // layout) were made by this warp on the slots phase 0 writes.
      __syncwarp();
    }
#pragma unroll
    for (int p = 0; p < kSpinPhases; ++p) {
      if (p < S.nphases) {
        uint32_t j = 0;
        for (int b = 0; b < 8; ++b) j |= ((tid >> b) & 1u) << S.phase_thr[p][b];
        const uint32_t sbase = smem_slot<VB>(j);
        uint32_t rs[RB];
#pragma unroll
        for (int k = 0; k < RB; ++k) rs[k] = smem_slot<VB>(1u << S.phase_reg[p][k]);
        if (p > 0) {
#pragma unroll
          for (int i = 0; i < NE; ++i) {
            uint32_t sidx = sbase;
#pragma unroll
            for (int k = 0; k < RB; ++k)
              if ((i >> k) & 1) sidx ^= rs[k];
            el[i] = tl[sidx];
            ep[i] = tp[sidx];
          }
        }
#pragma unroll
        for (int k = 0; k < RB; ++k) {
          const int f = p * RB + k;
          const int okind = (f < kMaxRotFlips && f < S.nflips) ? PS.flip[f].okind : 0;
          if (okind != 0) {
            // Im(w (A + s B)) = wi Re(A + s B) + wr Im(A + s B); the sums of
            // A + s B are formed first and weighted once per tile.
            const double s = PS.flip[f].minus ? -1.0 : 1.0;
            double xr = 0.0, xi = 0.0;
#pragma unroll
            for (int i = 0; i < NE; ++i) {
              if ((i >> k) & 1) continue;
              const C l0 = el[i], l1 = el[i | (1 << k)], p0 = ep[i], p1 = ep[i | (1 << k)];
              if (okind & 1) {
                const double ar = double(l0.x) * double(p1.x) + double(l0.y) * double(p1.y);
                const double br = double(l1.x) * double(p0.x) + double(l1.y) * double(p0.y);
                xr += __fma_rn(s, br, ar);
              }
              if (okind & 2) {
                const double ai = double(l0.x) * double(p1.y) - double(l0.y) * double(p1.x);
                const double bi = double(l1.x) * double(p0.y) - double(l1.y) * double(p0.x);
                xi += __fma_rn(s, bi, ai);
              }
            }
            acc[f][tid] += PS.flip[f].wi * xr + PS.flip[f].wr * xi;
          }
        }
        // The gates, lambda's registers first and written back before psi's,
        // so that fewer registers are live at once.
#pragma unroll
        for (int k = 0; k < RB; ++k) {
          const int f = p * RB + k;
          if (f < kMaxRotFlips && f < S.nflips && PS.flip[f].mkind != 2) {
            const double* m = PS.flip[f].m;
            if (PS.flip[f].mkind == 1) {
#pragma unroll
              for (int i = 0; i < NE; ++i) {
                if ((i >> k) & 1) continue;
                const int i1 = i | (1 << k);
                const C l0 = el[i], l1 = el[i1];
                el[i] = rmac2(l0, l1, Real(m[0]), Real(m[2]));
                el[i1] = rmac2(l0, l1, Real(m[4]), Real(m[6]));
              }
            } else {
#pragma unroll
              for (int i = 0; i < NE; ++i) {
                if ((i >> k) & 1) continue;
                const int i1 = i | (1 << k);
                const C l0 = el[i], l1 = el[i1];
                el[i] = cmac2(l0, l1, Real(m[0]), Real(m[1]), Real(m[2]), Real(m[3]));
                el[i1] = cmac2(l0, l1, Real(m[4]), Real(m[5]), Real(m[6]), Real(m[7]));
              }
            }
          }
        }
#pragma unroll
        for (int i = 0; i < NE; ++i) {
          uint32_t sidx = sbase;
#pragma unroll
          for (int k = 0; k < RB; ++k)
            if ((i >> k) & 1) sidx ^= rs[k];
          tl[sidx] = el[i];
        }
#pragma unroll
        for (int k = 0; k < RB; ++k) {
          const int f = p * RB + k;
          if (f < kMaxRotFlips && f < S.nflips && PS.flip[f].mkind != 2) {
            const double* m = PS.flip[f].m;
            if (PS.flip[f].mkind == 1) {
#pragma unroll
              for (int i = 0; i < NE; ++i) {
                if ((i >> k) & 1) continue;
                const int i1 = i | (1 << k);
                const C p0 = ep[i], p1 = ep[i1];
                ep[i] = rmac2(p0, p1, Real(m[0]), Real(m[2]));
                ep[i1] = rmac2(p0, p1, Real(m[4]), Real(m[6]));
              }
            } else {
#pragma unroll
              for (int i = 0; i < NE; ++i) {
                if ((i >> k) & 1) continue;
                const int i1 = i | (1 << k);
                const C p0 = ep[i], p1 = ep[i1];
                ep[i] = cmac2(p0, p1, Real(m[0]), Real(m[1]), Real(m[2]), Real(m[3]));
                ep[i1] = cmac2(p0, p1, Real(m[4]), Real(m[5]), Real(m[6]), Real(m[7]));
              }
            }
          }
        }
#pragma unroll
        for (int i = 0; i < NE; ++i) {
          uint32_t sidx = sbase;
#pragma unroll
          for (int k = 0; k < RB; ++k)
            if ((i >> k) & 1) sidx ^= rs[k];
          tp[sidx] = ep[i];
        }
        // The next phase (or the store) reads other threads' slots: those of
        // other warps too where the warp index moves to other tile bits.
        if (PS.block_sync[p]) __syncthreads();
        else __syncwarp();
      }
    }
    // The store addresses are recomputed from an opaque copy of the tile base:
    // kept from the loads, the eight of them would hold 16 registers through the phases.
    uint64_t sbase_hbm;
    asm volatile("mov.b64 %0, %1;" : "=l"(sbase_hbm) : "l"(base));
    if (t + gridDim.x < num_tiles) load_tile(tile_base(t + gridDim.x));
#pragma unroll
    for (int it = 0; it < NE; ++it) {
      const uint32_t s = st ^ smem_slot<VB>(uint32_t(it) << 8);
      uint64_t p = sbase_hbm;
#pragma unroll
      for (int b = 0; b < RB; ++b)
        if ((it >> b) & 1) p |= 1ull << S.tile_phys[8 + b];
      __stcs(lam + p, tl[s]);
      __stcs(psi + p, tp[s]);
    }
  }
  // Block sums in a fixed order, one double per flip; then, with Z sums, the
  // total and the sum over j with each physical bit set (tile bits from the
  // per-thread sums, the others from the per-warp sums).
  constexpr int NZ = 1 + 8 + kPairRegBits;
  __shared__ double red[kRedThreads / 32][kMaxRotFlips + NZ];
#pragma unroll
  for (int f = 0; f < kMaxRotFlips; ++f) {
    if (f < S.nflips) {
      const double a = warp_sum(acc[f][tid]);
      if (lane == 0) red[warp][f] = a;
    }
  }
  const bool zs = D.active && D.nz > 0;
  if (zs) {
    double v[NZ];
    v[0] = zt[0][tid];
#pragma unroll
    for (int b = 0; b < 8; ++b) v[1 + b] = ((tid >> b) & 1) ? zt[0][tid] : 0.0;
#pragma unroll
    for (int k = 0; k < kPairRegBits; ++k) v[9 + k] = zt[1 + k][tid];
#pragma unroll
    for (int k = 0; k < NZ; ++k) {
      const double a = warp_sum(v[k]);
      if (lane == 0) red[warp][kMaxRotFlips + k] = a;
    }
  }
  __syncthreads();
  const int nzw = zs ? 1 + kMaxQubits : 0;
  const int width = S.nflips + nzw;
  for (int k = threadIdx.x; k < width; k += blockDim.x) {
    double sum = 0.0;
    if (k < S.nflips) {
      for (int w = 0; w < kRedThreads / 32; ++w) sum += red[w][k];
    } else {
      const int q = k - S.nflips - 1;  // -1: the total
      int col = -1;
      if (q < 0) col = 0;
      for (int b = 0; b < 8 + kPairRegBits; ++b)
        if (q >= 0 && S.tile_phys[b] == q) col = 1 + b;
      if (col >= 0) {
        for (int w = 0; w < kRedThreads / 32; ++w) sum += red[w][kMaxRotFlips + col];
      } else {
        for (int w = 0; w < kRedThreads / 32; ++w) sum += zh[q][w];
      }
    }
    partials[size_t(blockIdx.x) * width + k] = sum;
  }
}

// One warp per flip that has an overlap: out[2 slot + 1] = Im(w (A + s B)) summed
// over the blocks; out[2 slot] = 0 (the real part is not formed).
// Blocks past nflips: one per Z entry of the pre-step, out[2 slot + 1] = wr (total - 2 sum over bit q set).
__global__ void finish_pair_rotate_kernel(const double* __restrict__ partials, int blocks, int nflips, int width,
                                          const __grid_constant__ pair_rotate_set set, double* __restrict__ out)
{
  const int lane = threadIdx.x & 31, f = blockIdx.x;
  if (f < nflips) {
    const int slot = set.flip[f].out_slot;
    if (slot < 0) return;
    double x = 0;
    for (int b = lane; b < blocks; b += 32) x += partials[size_t(b) * width + f];
    x = warp_sum(x);
    if (lane == 0) {
      out[2 * slot] = 0.0;
      out[2 * slot + 1] = x;
    }
    return;
  }
  const auto& z = set.pre.z[f - nflips];
  double t = 0, o = 0;
  for (int b = lane; b < blocks; b += 32) {
    t += partials[size_t(b) * width + nflips];
    o += partials[size_t(b) * width + nflips + 1 + z.bit];
  }
  t = warp_sum(t);
  o = warp_sum(o);
  if (lane == 0) {
    out[2 * z.out_slot] = 0.0;
    out[2 * z.out_slot + 1] = z.wr * (t - 2.0 * o);
  }
}

size_t pair_rotate_partials_doubles() { return size_t(148) * kPairBlocksPerSm * (kMaxRotFlips + 1 + kMaxQubits); }

template <typename Real>
cudaError_t launch_pair_rotate(void* lam, void* psi, int n, const pair_rotate_set& set, double* partials, double* out,
                               cudaStream_t stream)
{
  const spin_group& g = set.g;
  if (g.K != 8 + kPairRegBits || g.K > n || n > kMaxQubits || g.nflips < 1 || g.nflips > kMaxRotFlips || g.nphases < 1 ||
      g.nphases > kSpinPhases || g.nphases * kPairRegBits < g.nflips)
    return cudaErrorInvalidValue;
  const int nz = set.pre.active ? set.pre.nz : 0;
  if (nz < 0 || nz > kMaxQubits) return cudaErrorInvalidValue;
  for (int k = 0; k < nz; ++k)
    if (set.pre.z[k].bit < 0 || set.pre.z[k].bit >= n) return cudaErrorInvalidValue;
  const size_t smem = 2 * sizeof(typename ctype<Real>::c) << g.K;
  static std::atomic<bool> configured[64] = {};
  int dev = 0, sms = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
  if (!configured[dev].load(std::memory_order_acquire)) {
    e = cudaFuncSetAttribute(pair_rotate_kernel<Real>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    configured[dev].store(true, std::memory_order_release);
  }
  e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (e != cudaSuccess) return e;
  const uint64_t tiles = 1ull << (n - g.K);
  // Capped at 148 SMs' worth: the partials buffer is sized for that.
  const int blocks = static_cast<int>(std::min<uint64_t>(tiles, uint64_t(std::min(sms, 148)) * kPairBlocksPerSm));
  pair_rotate_kernel<Real><<<blocks, kRedThreads, smem, stream>>>(static_cast<typename ctype<Real>::c*>(lam),
                                                                 static_cast<typename ctype<Real>::c*>(psi), set, tiles,
                                                                 partials);
  const int width = g.nflips + (nz > 0 ? 1 + kMaxQubits : 0);
  finish_pair_rotate_kernel<<<g.nflips + nz, 32, 0, stream>>>(partials, blocks, g.nflips, width, set, out);
  return cudaGetLastError();
}
template cudaError_t launch_pair_rotate<double>(void*, void*, int, const pair_rotate_set&, double*, double*, cudaStream_t);
template cudaError_t launch_pair_rotate<float>(void*, void*, int, const pair_rotate_set&, double*, double*, cudaStream_t);

template cudaError_t launch_zsum2<double>(const void*, const void*, int, const zsum2_set&, double*, double*, cudaStream_t);
template cudaError_t launch_zsum2<float>(const void*, const void*, int, const zsum2_set&, double*, double*, cudaStream_t);
template cudaError_t launch_pair_overlaps<double>(const void*, const void*, int, const pair_overlap_set&, double*, double*, cudaStream_t);
template cudaError_t launch_pair_overlaps<float>(const void*, const void*, int, const pair_overlap_set&, double*, double*, cudaStream_t);

template cudaError_t launch_tile_overlaps<double>(const void*, const void*, int, const tile_overlap_set&, double*, double*, cudaStream_t);
template cudaError_t launch_tile_overlaps<float>(const void*, const void*, int, const tile_overlap_set&, double*, double*, cudaStream_t);

template cudaError_t launch_overlaps<double>(const void*, const void*, int, const overlap_set&, double*, double*, cudaStream_t);
template cudaError_t launch_overlaps<float>(const void*, const void*, int, const overlap_set&, double*, double*, cudaStream_t);

template cudaError_t launch_pauli_apply<double>(const void*, void*, int, const pauli_sum&, cudaStream_t);
template cudaError_t launch_pauli_apply<float>(const void*, void*, int, const pauli_sum&, cudaStream_t);
template cudaError_t launch_overlap<double>(const void*, const void*, int, uint64_t, uint64_t, double, double, double*, double*, cudaStream_t);
template cudaError_t launch_overlap<float>(const void*, const void*, int, uint64_t, uint64_t, double, double, double*, double*, cudaStream_t);

}  // namespace rbk

namespace rbk {

// ---------------------------------------------------------------------------
// Sampling: inclusive prefix sums of |a_i|^2 and upper_bound searches
// (the device form of ket::generate_events, ket/include/ket/generate_events.hpp:18-51)
// ---------------------------------------------------------------------------
constexpr int kScanThreads = 256;
constexpr int kScanPerThread = 16;
constexpr int kScanChunk = kScanThreads * kScanPerThread;  // values per block

// One block scans kScanChunk consecutive values: out[i] = sum_{j<=i in chunk} v[j],
// and writes the chunk total to sums[block].  v = |a_i|^2 when amps != nullptr,
// else v = in[i].
template <typename Real>
__global__ void __launch_bounds__(kScanThreads)
chunk_scan_kernel(const typename ctype<Real>::c* __restrict__ amps, const double* __restrict__ in, uint64_t count,
                  double* __restrict__ out, double* __restrict__ sums)
{
  __shared__ double warp_tot[kScanThreads / 32];
  const uint64_t base = uint64_t(blockIdx.x) * kScanChunk + uint64_t(threadIdx.x) * kScanPerThread;
  double v[kScanPerThread];
  double run = 0;
#pragma unroll
  for (int k = 0; k < kScanPerThread; ++k) {
    const uint64_t i = base + k;
    double x = 0;
    if (i < count) {
      if (amps) { const auto a = amps[i]; x = double(a.x) * double(a.x) + double(a.y) * double(a.y); }
      else x = in[i];
    }
    run += x;
    v[k] = run;
  }
  // exclusive scan of the per-thread totals over the block
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  double incl = run;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const double y = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += y;
  }
  if (lane == 31) warp_tot[warp] = incl;
  __syncthreads();
  double warp_off = 0, block_tot = 0;
  for (int w = 0; w < kScanThreads / 32; ++w) {
    if (w < warp) warp_off += warp_tot[w];
    block_tot += warp_tot[w];
  }
  const double off = warp_off + (incl - run);
#pragma unroll
  for (int k = 0; k < kScanPerThread; ++k) {
    const uint64_t i = base + k;
    if (i < count) out[i] = v[k] + off;
  }
  if (threadIdx.x == 0 && sums) sums[blockIdx.x] = block_tot;
}

// out[i] += offsets[block of i - 1] (offsets = inclusive scan of the chunk totals)
__global__ void add_offsets_kernel(double* __restrict__ out, uint64_t count, const double* __restrict__ offsets)
{
  const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
  for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < count; i += stride) {
    const uint64_t chunk = i / kScanChunk;
    if (chunk > 0) out[i] += offsets[chunk - 1];
  }
}

// events[k] = first index i with prefix[i] > r[k]  (std::upper_bound)
__global__ void upper_bound_kernel(const double* __restrict__ prefix, uint64_t count, const double* __restrict__ r,
                                   int num, uint64_t* __restrict__ events)
{
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= num) return;
  const double x = r[k];
  uint64_t lo = 0, hi = count;
  while (lo < hi) {
    const uint64_t mid = lo + ((hi - lo) >> 1);
    if (prefix[mid] > x) hi = mid;
    else lo = mid + 1;
  }
  events[k] = lo;
}

size_t scan_scratch_doubles(uint64_t count)
{
  size_t total = 0;
  uint64_t m = count;
  while (m > 1) {
    m = (m + kScanChunk - 1) / kScanChunk;
    total += m;
  }
  return total + 1;
}

// Inclusive scan of |a|^2 (level 0) with the chunk totals scanned recursively in `scratch`.
template <typename Real>
cudaError_t launch_prob_scan(const void* amps, uint64_t count, double* prefix, double* scratch, cudaStream_t stream)
{
  // level list: (values, count, out, sums)
  const double* in = nullptr;
  const void* a = amps;
  double* out = prefix;
  uint64_t m = count;
  double* level_out[64];
  uint64_t level_count[64];
  int levels = 0;
  double* s = scratch;
  while (true) {
    const uint64_t blocks = (m + kScanChunk - 1) / kScanChunk;
    double* sums = blocks > 1 ? s : nullptr;
    if (a) chunk_scan_kernel<Real><<<(unsigned)blocks, kScanThreads, 0, stream>>>(static_cast<const typename ctype<Real>::c*>(a), nullptr, m, out, sums);
    else chunk_scan_kernel<double><<<(unsigned)blocks, kScanThreads, 0, stream>>>(nullptr, in, m, out, sums);
    level_out[levels] = out;
    level_count[levels] = m;
    ++levels;
    if (blocks <= 1) break;
    // scan the chunk totals in place: next level reads `sums`, writes into the same array
    in = sums;
    a = nullptr;
    out = sums;
    m = blocks;
    s += blocks;
  }
  for (int l = levels - 2; l >= 0; --l) {
    add_offsets_kernel<<<grid_for(level_count[l], 256), 256, 0, stream>>>(level_out[l], level_count[l], level_out[l + 1]);
  }
  return cudaGetLastError();
}

cudaError_t launch_upper_bound(const double* prefix, uint64_t count, const double* r, int num, uint64_t* events, cudaStream_t stream)
{
  upper_bound_kernel<<<(num + 255) / 256, 256, 0, stream>>>(prefix, count, r, num, events);
  return cudaGetLastError();
}

template cudaError_t launch_prob_scan<double>(const void*, uint64_t, double*, double*, cudaStream_t);
template cudaError_t launch_prob_scan<float>(const void*, uint64_t, double*, double*, cudaStream_t);

}  // namespace rbk

namespace rbk {

// ---------------------------------------------------------------------------
// SHORBOX: ket::shor_box (ket/include/ket/shor_box.hpp) writes, for every
// exponent e < 2^nx, the amplitude 2^(-nx/2) at the index whose top nx qubits
// hold e bit-reversed and whose low n - nx qubits hold (base^e mod divisor)
// truncated to n - nx bits; e = 0 holds 1 (the running value starts at 1 and
// is reduced only after use).  The reference walks e sequentially; here every
// thread computes its own power by squaring.  With divisor, base < 2^32 every
// product stays below 2^64, so the values are the reference's exactly.
// ---------------------------------------------------------------------------
template <typename Real>
__global__ void shor_box_kernel(typename ctype<Real>::c* __restrict__ a, int n, int nx, uint64_t divisor, uint64_t base,
                                Real coeff)
{
  using C = typename ctype<Real>::c;
  const uint64_t count = 1ull << nx;
  const int low = n - nx;
  const uint64_t low_mask = (1ull << low) - 1;
  const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
  for (uint64_t e = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; e < count; e += stride) {
    uint64_t v = 1;
    if (e > 0) {
      uint64_t x = base % divisor, r = 1 % divisor;
      for (uint64_t k = e; k; k >>= 1) {
        if (k & 1) r = r * x % divisor;
        x = x * x % divisor;
      }
      v = r;
    }
    const uint64_t rev = nx > 0 ? (__brevll(e) >> (64 - nx)) : 0;
    a[(rev << low) | (v & low_mask)] = C{coeff, (Real)0};
  }
}

template <typename Real>
cudaError_t launch_shor_box(void* state, int n, int nx, uint64_t divisor, uint64_t base, double coeff, cudaStream_t stream)
{
  const uint64_t count = 1ull << nx;
  shor_box_kernel<Real><<<grid_for(count, 256), 256, 0, stream>>>(static_cast<typename ctype<Real>::c*>(state), n, nx,
                                                                divisor, base, static_cast<Real>(coeff));
  return cudaGetLastError();
}
template cudaError_t launch_shor_box<double>(void*, int, int, uint64_t, uint64_t, double, cudaStream_t);
template cudaError_t launch_shor_box<float>(void*, int, int, uint64_t, uint64_t, double, cudaStream_t);

}  // namespace rbk
