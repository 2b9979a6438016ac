// rbk_kernels.cu -- sm_100a kernels of the state-vector engine.
//
//   tile_pass_kernel   one fused pass: stage a 2^K-amplitude tile in shared
//                      memory, apply a gate program in registers, write back
//                      (optionally with the tile bits relabelled).  Replaces
//                      ket's per-gate loops (ket/include/ket/gate/*.hpp, e.g.
//                      hadamard.hpp:52-71, phase_shift.hpp:1235-1253) and bra's
//                      fused replay (bra/src/nompi_state.cpp:1285-1357).
//   gate_kernel        one unfused gate straight on HBM (states smaller than a
//                      tile, and the unfused execution mode).
//   reductions         norm, probabilities, Z / pair sums for spins and Pauli
//                      strings, inner product: warp-shuffle + block reduction
//                      with FP64 accumulation, per-block partials reduced in a
//                      fixed order (deterministic).
#include <cuda_runtime.h>
#include <cstdint>

#include "rbk_internal.h"
#include "rbk_kernels.h"

namespace rbk {

template <typename Real> struct ctype;
template <> struct ctype<double> { using c = double2; using v16 = double2; };
template <> struct ctype<float> { using c = float2; using v16 = float4; };

template <typename C>
__device__ __forceinline__ C cmul(C a, C b) { return C{a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x}; }
template <typename C, typename Real>
__device__ __forceinline__ C cmac2(C a0, C a1, Real m0r, Real m0i, Real m1r, Real m1i)
{
  // m0 * a0 + m1 * a1
  C r;
  r.x = m0r * a0.x - m0i * a0.y + m1r * a1.x - m1i * a1.y;
  r.y = m0r * a0.y + m0i * a0.x + m1r * a1.y + m1i * a1.x;
  return r;
}

// Shared-memory slot of tile index j: XOR-fold of the 16-byte-vector index so
// that register layouts whose lanes sit on arbitrary tile bits still spread
// over the banks.  Bijective (only bits >= 3 of the vector index feed the fold).
template <int VEC>
__device__ __forceinline__ uint32_t smem_slot(uint32_t j)
{
  constexpr int v = VEC == 2 ? 1 : 0;
  uint32_t u = j >> v;
  uint32_t f = (u >> 3) ^ (u >> 6) ^ (u >> 9) ^ (u >> 12);
  u ^= f & 7u;
  return (u << v) | (j & (VEC - 1));
}

// ---------------------------------------------------------------------------
// Fused tile pass
// ---------------------------------------------------------------------------
template <typename Real>
struct mat2 { Real m00r, m00i, m01r, m01i, m10r, m10i, m11r, m11i; };

template <typename Real, int B, int NR>
__device__ __forceinline__ void apply_mat(typename ctype<Real>::c* a, uint32_t creg, const mat2<Real> M)
{
  const Real m00r = M.m00r, m00i = M.m00i, m01r = M.m01r, m01i = M.m01i;
  const Real m10r = M.m10r, m10i = M.m10i, m11r = M.m11r, m11i = M.m11i;
#pragma unroll
  for (int i = 0; i < NR; ++i) {
    if (i & (1 << B)) continue;
    if ((uint32_t(i) & creg) != creg) continue;
    auto a0 = a[i], a1 = a[i | (1 << B)];
    a[i] = cmac2(a0, a1, m00r, m00i, m01r, m01i);
    a[i | (1 << B)] = cmac2(a0, a1, m10r, m10i, m11r, m11i);
  }
}

template <typename Real, int B, int NR>
__device__ __forceinline__ void apply_x(typename ctype<Real>::c* a, uint32_t creg)
{
#pragma unroll
  for (int i = 0; i < NR; ++i) {
    if (i & (1 << B)) continue;
    if ((uint32_t(i) & creg) != creg) continue;
    auto t = a[i]; a[i] = a[i | (1 << B)]; a[i | (1 << B)] = t;
  }
}

template <typename Real, int B, int NR>
__device__ __forceinline__ void apply_y(typename ctype<Real>::c* a, uint32_t creg)
{
#pragma unroll
  for (int i = 0; i < NR; ++i) {
    if (i & (1 << B)) continue;
    if ((uint32_t(i) & creg) != creg) continue;
    auto a0 = a[i], a1 = a[i | (1 << B)];
    a[i] = typename ctype<Real>::c{a1.y, -a1.x};          // -i * a1
    a[i | (1 << B)] = typename ctype<Real>::c{-a0.y, a0.x}; //  i * a0
  }
}

// Runs F on register bit b (0 <= b < R); the bit must be a compile-time index
// so that the register array stays in registers.
#define RBK_DISPATCH_BIT(b, CALL)                                   \
  switch (b) {                                                      \
    case 0: { constexpr int BB = 0; CALL; } break;                  \
    case 1: { constexpr int BB = 1; CALL; } break;                  \
    case 2: { constexpr int BB = 2; CALL; } break;                  \
    case 3: { constexpr int BB = 3; CALL; } break;                  \
    case 4: if constexpr (R > 4) { constexpr int BB = 4; CALL; } break; \
    default: break;                                                 \
  }

template <typename Real>
__global__ void __launch_bounds__(1 << tiling<Real>::T, 2)
tile_pass_kernel(typename ctype<Real>::c* __restrict__ state, const __grid_constant__ dev_pass P)
{
  using C = typename ctype<Real>::c;
  using V = typename ctype<Real>::v16;
  using TL = tiling<Real>;
  constexpr int K = TL::K, R = TL::R, NR = 1 << R, NT = 1 << TL::T, VEC = TL::VEC;
  constexpr int vbits = VEC == 2 ? 1 : 0;
  constexpr int ITER = (1 << K) / VEC / NT;
  constexpr int ITBITS = K - vbits - TL::T;
  static_assert((1 << ITBITS) == ITER, "tile copy iterations");

  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* tile = reinterpret_cast<C*>(smem_raw);

  const uint32_t tid = threadIdx.x;

  // Tile base: deposit the block index into the physical bits outside the tile.
  uint64_t base = 0;
  {
    uint64_t b = blockIdx.x;
    for (int k = 0; k < P.num_nontile; ++k)
      base |= ((b >> k) & 1ull) << P.nontile_phys[k];
  }
  // Physical offsets for the coalesced copy: tile index j = (it * NT + tid) * VEC.
  uint64_t thr_phys = 0;
#pragma unroll
  for (int b = 0; b < TL::T; ++b) thr_phys |= uint64_t((tid >> b) & 1u) << P.tile_phys[vbits + b];
  uint64_t it_bit_phys[ITBITS];
#pragma unroll
  for (int b = 0; b < ITBITS; ++b) it_bit_phys[b] = 1ull << P.tile_phys[vbits + TL::T + b];

  const V* gsrc = reinterpret_cast<const V*>(state);
#pragma unroll
  for (int it = 0; it < ITER; ++it) {
    uint64_t phys = base | thr_phys;
#pragma unroll
    for (int b = 0; b < ITBITS; ++b) if (it & (1 << b)) phys |= it_bit_phys[b];
    const uint32_t j = uint32_t((it * NT + tid) * VEC);
    V v = __ldcs(gsrc + (phys >> vbits));
    *reinterpret_cast<V*>(&tile[smem_slot<VEC>(j)]) = v;
  }
  __syncthreads();

  C a[NR];
  for (int p = 0; p < P.num_phases; ++p) {
    const dev_phase& ph = P.phases[p];
    uint32_t toff = 0;
#pragma unroll
    for (int b = 0; b < TL::T; ++b) toff |= ((tid >> b) & 1u) << ph.thr_pos[b];
    uint32_t rbit[R];
#pragma unroll
    for (int b = 0; b < R; ++b) rbit[b] = 1u << ph.reg_pos[b];
#pragma unroll
    for (int i = 0; i < NR; ++i) {
      uint32_t j = toff;
#pragma unroll
      for (int b = 0; b < R; ++b) if (i & (1 << b)) j |= rbit[b];
      a[i] = tile[smem_slot<VEC>(j)];
    }

    for (int o = ph.op_begin; o < ph.op_end; ++o) {
      const dev_op& op = P.ops[o];
      if ((tid & op.cthr) != op.cthr || (base & op.cout) != op.cout) continue;
      switch (op.kind) {
        case OPK_MAT: {
          const mat2<Real> M{(Real)op.m[0], (Real)op.m[1], (Real)op.m[2], (Real)op.m[3],
                             (Real)op.m[4], (Real)op.m[5], (Real)op.m[6], (Real)op.m[7]};
          const uint32_t creg = op.creg;
          RBK_DISPATCH_BIT(op.treg, (apply_mat<Real, BB, NR>(a, creg, M)));
          break;
        }
        case OPK_X: { const uint32_t creg = op.creg; RBK_DISPATCH_BIT(op.treg, (apply_x<Real, BB, NR>(a, creg))); break; }
        case OPK_Y: { const uint32_t creg = op.creg; RBK_DISPATCH_BIT(op.treg, (apply_y<Real, BB, NR>(a, creg))); break; }
        case OPK_NEG: {
#pragma unroll
          for (int i = 0; i < NR; ++i)
            if ((uint32_t(i) & op.creg) == op.creg) { a[i].x = -a[i].x; a[i].y = -a[i].y; }
          break;
        }
        case OPK_DIAG: {
          const bool tb = ((tid & op.dthr) != 0) || ((base & op.dout) != 0);
          const C d0{(Real)op.m[0], (Real)op.m[1]}, d1{(Real)op.m[2], (Real)op.m[3]};
#pragma unroll
          for (int i = 0; i < NR; ++i) {
            if ((uint32_t(i) & op.creg) != op.creg) continue;
            const bool bit = tb || (uint32_t(i) & op.dreg);
            if (bit) a[i] = cmul(a[i], d1);
            else if (!op.diag_one) a[i] = cmul(a[i], d0);
          }
          break;
        }
        default: break;
      }
    }
    __syncthreads();
    uint32_t woff = 0;
#pragma unroll
    for (int b = 0; b < TL::T; ++b) woff |= ((tid >> b) & 1u) << ph.wthr_pos[b];
#pragma unroll
    for (int b = 0; b < R; ++b) rbit[b] = 1u << ph.wreg_pos[b];
#pragma unroll
    for (int i = 0; i < NR; ++i) {
      uint32_t j = woff;
#pragma unroll
      for (int b = 0; b < R; ++b) if (i & (1 << b)) j |= rbit[b];
      tile[smem_slot<VEC>(j)] = a[i];
    }
    __syncthreads();
  }

  V* gdst = reinterpret_cast<V*>(state);
#pragma unroll
  for (int it = 0; it < ITER; ++it) {
    uint64_t phys = base | thr_phys;
#pragma unroll
    for (int b = 0; b < ITBITS; ++b) if (it & (1 << b)) phys |= it_bit_phys[b];
    const uint32_t j = uint32_t((it * NT + tid) * VEC);
    V v = *reinterpret_cast<const V*>(&tile[smem_slot<VEC>(j)]);
    __stcs(gdst + (phys >> vbits), v);
  }
}

template <typename Real>
size_t tile_pass_smem_bytes() { return sizeof(typename ctype<Real>::c) << tiling<Real>::K; }

template <typename Real>
cudaError_t launch_tile_pass(void* state, int n, const dev_pass& pass, cudaStream_t stream)
{
  const size_t smem = tile_pass_smem_bytes<Real>();
  static bool configured[64] = {};
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
  if (!configured[dev]) {
    e = cudaFuncSetAttribute(tile_pass_kernel<Real>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    configured[dev] = true;
  }
  const uint64_t blocks = 1ull << (n - tiling<Real>::K);
  tile_pass_kernel<Real><<<(unsigned)blocks, 1 << tiling<Real>::T, smem, stream>>>(
    static_cast<typename ctype<Real>::c*>(state), pass);
  return cudaGetLastError();
}

template cudaError_t launch_tile_pass<double>(void*, int, const dev_pass&, cudaStream_t);
template cudaError_t launch_tile_pass<float>(void*, int, const dev_pass&, cudaStream_t);

// ---------------------------------------------------------------------------
// Unfused gate straight on HBM
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint64_t insert_zero(uint64_t v, int q)
{
  const uint64_t low = (1ull << q) - 1;
  return ((v & ~low) << 1) | (v & low);
}

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
template cudaError_t launch_inner<double>(const void*, const void*, int, double*, double*, cudaStream_t);
template cudaError_t launch_inner<float>(const void*, const void*, int, double*, double*, cudaStream_t);
template cudaError_t launch_probs<double>(const void*, uint64_t, uint64_t, double*, cudaStream_t);
template cudaError_t launch_probs<float>(const void*, uint64_t, uint64_t, double*, cudaStream_t);

}  // namespace rbk
