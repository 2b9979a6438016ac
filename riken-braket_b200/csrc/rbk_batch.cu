// rbk_batch.cu -- energies and adjoint gradients of many parametrised circuits
// of uneven size in one call (rbk_batch_* of include/rbk.h).
//
// Instances small enough for two state vectors to sit in one CTA's shared
// memory (n <= 12 for complex<double>, n <= 13 for complex<float>) run in ONE
// persistent kernel launch: every CTA takes the next instance from a work
// counter and does the whole job there -- forward sweep from |0...0>, lambda =
// H psi, E = <psi|lambda>, and the reverse sweep that un-applies each gate on
// psi and lambda and, at every parametrised rotation exp(i phi P) with
// phi = scale * theta + offset, adds dE/dtheta = -2 scale Im <lambda|P|psi>.
// The launch and its copies are captured in a CUDA graph on first use and
// replayed for every later parameter vector.  The CTA size is picked by an
// autotuner that times the candidates on the batch's own small instances.
// Larger instances run through the engine's adjoint sweep
// (rbk_adjoint_gradient) on worker threads, with the fused passes' tile shape
// (their fusion width) picked per qubit count by a second autotuner.
//
// The reference has no differentiation or batching; the gate arithmetic is
// ket's (exponential_pauli_y.hpp:40-85, exponential_pauli_z.hpp:40-78,
// phase_shift.hpp:660-709 and :1200-1254), the same matrices as the engine's.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <atomic>
#include <exception>
#include <map>
#include <memory>
#include <mutex>
#include <new>
#include <string>
#include <thread>
#include <vector>

#include "rbk.h"
#include "rbk_adjoint.h"
#include "rbk_device.cuh"
#include "rbk_kernels.h"

namespace rbk {
namespace {

// One gate of a small instance.  Bits are logical qubits (< 32).
enum : uint8_t { BOP_MAT = 1, BOP_X = 2, BOP_PHASE = 3, BOP_SWAP = 4, BOP_ROT = 5 };

struct bgate {
  uint8_t op;
  uint8_t pauli;   // BOP_ROT: 1 = X, 2 = Y, 3 = Z
  uint8_t q0, q1;  // target (MAT, X, ROT) / the two qubits (SWAP)
  int32_t param;   // BOP_ROT: parameter index within the instance, -1 = fixed angle
  uint32_t cmask;  // MAT / X: control mask; PHASE: the qubits that must all be one
  uint32_t pad;
  double scale, offset;  // BOP_ROT: phi = scale * theta[param] + offset
  double m[8];           // MAT: m00 m01 m10 m11 (re, im); PHASE: m[0], m[1] = coefficient
};

struct binst {
  int32_t n, num_gates, gate_begin, param_begin, num_terms, term_begin, out_index, pad;
};

struct bterm {  // (P psi)_i = w (-1)^popcount(i & sign) psi_{i ^ flip}
  uint32_t flip, sign;
  double w[2];
};

template <typename C>
__device__ __forceinline__ C cadd(C a, C b) { return C{a.x + b.x, a.y + b.y}; }

template <typename Real>
__device__ __forceinline__ typename ctype<Real>::c cplx_of(double re, double im)
{
  return typename ctype<Real>::c{(Real)re, (Real)im};
}

// Sums (a, b) over the CTA; every thread gets the totals.
__device__ __forceinline__ void block_sum2(double& a, double& b, double (*red)[2])
{
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    a += __shfl_xor_sync(0xffffffffu, a, o);
    b += __shfl_xor_sync(0xffffffffu, b, o);
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, warps = blockDim.x >> 5;
  if (lane == 0) { red[warp][0] = a; red[warp][1] = b; }
  __syncthreads();
  a = 0.0;
  b = 0.0;
  for (int w = 0; w < warps; ++w) { a += red[w][0]; b += red[w][1]; }  // fixed order: deterministic
  __syncthreads();
}

// 2x2 matrix (inverse: conjugate transpose) on target t where the controls are one, on one or two states.
template <typename Real>
__device__ __forceinline__ void smem_mat(typename ctype<Real>::c* s, uint32_t half, int t, uint32_t cmask, const double* m,
                                         bool inverse)
{
  using C = typename ctype<Real>::c;
  const C m00 = inverse ? cplx_of<Real>(m[0], -m[1]) : cplx_of<Real>(m[0], m[1]);
  const C m01 = inverse ? cplx_of<Real>(m[4], -m[5]) : cplx_of<Real>(m[2], m[3]);
  const C m10 = inverse ? cplx_of<Real>(m[2], -m[3]) : cplx_of<Real>(m[4], m[5]);
  const C m11 = inverse ? cplx_of<Real>(m[6], -m[7]) : cplx_of<Real>(m[6], m[7]);
  for (uint32_t p = threadIdx.x; p < half; p += blockDim.x) {
    const uint32_t i0 = uint32_t(insert_zero(p, t));
    if ((i0 & cmask) != cmask) continue;
    const uint32_t i1 = i0 | (1u << t);
    const C a0 = s[i0], a1 = s[i1];
    s[i0] = cadd(cmul(m00, a0), cmul(m01, a1));
    s[i1] = cadd(cmul(m10, a0), cmul(m11, a1));
  }
}

template <typename Real>
__device__ void smem_gate(typename ctype<Real>::c* s, uint32_t N, const bgate& g, const double* theta, bool inverse)
{
  using C = typename ctype<Real>::c;
  switch (g.op) {
    case BOP_MAT: smem_mat<Real>(s, N >> 1, g.q0, g.cmask, g.m, inverse); break;
    case BOP_X:
      for (uint32_t p = threadIdx.x; p < (N >> 1); p += blockDim.x) {
        const uint32_t i0 = uint32_t(insert_zero(p, g.q0));
        if ((i0 & g.cmask) != g.cmask) continue;
        const uint32_t i1 = i0 | (1u << g.q0);
        const C t = s[i0];
        s[i0] = s[i1];
        s[i1] = t;
      }
      break;
    case BOP_PHASE: {
      const C c = cplx_of<Real>(g.m[0], inverse ? -g.m[1] : g.m[1]);
      for (uint32_t i = threadIdx.x; i < N; i += blockDim.x)
        if ((i & g.cmask) == g.cmask) s[i] = cmul(s[i], c);
      break;
    }
    case BOP_SWAP: {
      const uint32_t b0 = 1u << g.q0, b1 = 1u << g.q1;
      for (uint32_t i = threadIdx.x; i < N; i += blockDim.x)
        if ((i & b0) && !(i & b1)) {
          const uint32_t j = i ^ b0 ^ b1;
          const C t = s[i];
          s[i] = s[j];
          s[j] = t;
        }
      break;
    }
    case BOP_ROT: {
      const double phi = (g.param >= 0 ? g.scale * theta[g.param] : 0.0) + g.offset;
      double sn, cs;
      sincos(inverse ? -phi : phi, &sn, &cs);
      double m[8] = {0, 0, 0, 0, 0, 0, 0, 0};
      if (g.pauli == 1) { m[0] = cs; m[3] = sn; m[5] = sn; m[6] = cs; }        // cos I + i sin X
      else if (g.pauli == 2) { m[0] = cs; m[2] = sn; m[4] = -sn; m[6] = cs; }  // cos I + i sin Y
      else { m[0] = cs; m[1] = sn; m[6] = cs; m[7] = -sn; }                   // diag(e^{i phi}, e^{-i phi})
      smem_mat<Real>(s, N >> 1, g.q0, 0u, m, false);
      break;
    }
    default: break;
  }
}

template <typename Real>
__global__ void batch_adjoint_kernel(const binst* __restrict__ inst, int count, const bgate* __restrict__ gates,
                                     const bterm* __restrict__ terms, const double* __restrict__ theta,
                                     double* __restrict__ energy, double* __restrict__ grad, unsigned* next)
{
  using C = typename ctype<Real>::c;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ double red[32][2];
  __shared__ int item;
  C* const base = reinterpret_cast<C*>(smem_raw);
  while (true) {
    if (threadIdx.x == 0) item = int(atomicAdd(next, 1u));
    __syncthreads();
    const int it = item;
    __syncthreads();
    if (it >= count) break;
    const binst I = inst[it];
    const uint32_t N = 1u << I.n;
    C* psi = base;
    C* lam = base + N;
    const double* th = theta + I.param_begin;
    const bgate* G = gates + I.gate_begin;
    for (uint32_t i = threadIdx.x; i < N; i += blockDim.x) psi[i] = cplx_of<Real>(i == 0 ? 1.0 : 0.0, 0.0);
    __syncthreads();
    for (int k = 0; k < I.num_gates; ++k) {
      smem_gate<Real>(psi, N, G[k], th, false);
      __syncthreads();
    }
    // lambda = H psi, E = <psi|lambda>
    double er = 0.0, ei = 0.0;
    for (uint32_t i = threadIdx.x; i < N; i += blockDim.x) {
      double lr = 0.0, li = 0.0;
      for (int t = 0; t < I.num_terms; ++t) {
        const bterm T = terms[I.term_begin + t];
        const C v = psi[i ^ T.flip];
        const double sg = (__popc(i & T.sign) & 1) ? -1.0 : 1.0;
        lr += sg * (T.w[0] * double(v.x) - T.w[1] * double(v.y));
        li += sg * (T.w[0] * double(v.y) + T.w[1] * double(v.x));
      }
      lam[i] = cplx_of<Real>(lr, li);
      const C p = psi[i];
      er += double(p.x) * lr + double(p.y) * li;
      ei += double(p.x) * li - double(p.y) * lr;
    }
    block_sum2(er, ei, red);
    if (threadIdx.x == 0) energy[I.out_index] = er;
    // Reverse sweep.
    for (int k = I.num_gates - 1; k >= 0; --k) {
      const bgate& g = G[k];
      if (g.op == BOP_ROT && g.param >= 0) {
        const uint32_t t = 1u << g.q0;
        const uint32_t flip = g.pauli == 3 ? 0u : t, sign = g.pauli == 1 ? 0u : t;
        const double wr = g.pauli == 2 ? 0.0 : 1.0, wi = g.pauli == 2 ? -1.0 : 0.0;
        double orr = 0.0, oi = 0.0;
        for (uint32_t i = threadIdx.x; i < N; i += blockDim.x) {
          const C v = psi[i ^ flip];
          const double sg = (i & sign) ? -1.0 : 1.0;
          const double pr = sg * (wr * double(v.x) - wi * double(v.y)), pi = sg * (wr * double(v.y) + wi * double(v.x));
          const C l = lam[i];
          orr += double(l.x) * pr + double(l.y) * pi;
          oi += double(l.x) * pi - double(l.y) * pr;
        }
        block_sum2(orr, oi, red);
        if (threadIdx.x == 0) grad[I.param_begin + g.param] += -2.0 * g.scale * oi;
      }
      smem_gate<Real>(psi, N, g, th, true);
      smem_gate<Real>(lam, N, g, th, true);
      __syncthreads();
    }
  }
}

// ---- host side ------------------------------------------------------------

using cplx = std::complex<double>;
constexpr double kOneDivRootTwo = 0.707106781186547524400844362104849039284835937688474036588;
constexpr double kTwoPi = 6.28318530717958647692528676655900576839433879875021164195;

void put(double* m, int k, cplx v) { m[2 * k] = v.real(); m[2 * k + 1] = v.imag(); }

// The engine's matrices for the fixed gates (rbk_capi.cpp rbk_hadamard, rbk_phase_shift2/3, ...).
bool lower_gate(const rbk_circuit_gate& g, bgate& out)
{
  std::memset(&out, 0, sizeof(out));
  out.param = -1;
  out.q0 = static_cast<uint8_t>(g.qubits[0]);
  out.q1 = static_cast<uint8_t>(g.qubits[1]);
  const uint32_t b0 = 1u << g.qubits[0];
  switch (g.kind) {
    case RBK_GATE_H:
      out.op = BOP_MAT;
      put(out.m, 0, {kOneDivRootTwo, 0}); put(out.m, 1, {kOneDivRootTwo, 0});
      put(out.m, 2, {kOneDivRootTwo, 0}); put(out.m, 3, {-kOneDivRootTwo, 0});
      return true;
    case RBK_GATE_X: out.op = BOP_X; return true;
    case RBK_GATE_Y:
      out.op = BOP_MAT;
      put(out.m, 1, {0, -1}); put(out.m, 2, {0, 1});
      return true;
    case RBK_GATE_Z: out.op = BOP_PHASE; out.cmask = b0; put(out.m, 0, {-1, 0}); return true;
    case RBK_GATE_U1: out.op = BOP_PHASE; out.cmask = b0; put(out.m, 0, std::exp(cplx{0, g.angles[0]})); return true;
    case RBK_GATE_U2: {
      const cplx c1 = std::exp(cplx{0, g.angles[0]}), c2 = std::exp(cplx{0, g.angles[1]});
      const cplx mc1 = kOneDivRootTwo * c1;
      out.op = BOP_MAT;
      put(out.m, 0, {kOneDivRootTwo, 0}); put(out.m, 1, -(kOneDivRootTwo * c2));
      put(out.m, 2, mc1); put(out.m, 3, mc1 * c2);
      return true;
    }
    case RBK_GATE_U3: {
      const double sine = std::sin(0.5 * g.angles[0]), cosine = std::cos(0.5 * g.angles[0]);
      const cplx c2 = std::exp(cplx{0, g.angles[1]}), c3 = std::exp(cplx{0, g.angles[2]});
      out.op = BOP_MAT;
      put(out.m, 0, {cosine, 0}); put(out.m, 1, -(sine * c3));
      put(out.m, 2, sine * c2); put(out.m, 3, (cosine * c3) * c2);
      return true;
    }
    case RBK_GATE_CNOT:  // qubits[0] = control, qubits[1] = target
      out.op = BOP_X;
      out.q0 = static_cast<uint8_t>(g.qubits[1]);
      out.cmask = b0;
      return true;
    case RBK_GATE_CZ: out.op = BOP_PHASE; out.cmask = b0 | (1u << g.qubits[1]); put(out.m, 0, {-1, 0}); return true;
    case RBK_GATE_U: {
      const int k = static_cast<int>(g.angles[0]);
      const int ak = k < 0 ? -k : k;
      cplx c = std::exp(cplx{0, kTwoPi / static_cast<double>(1ull << ak)});
      if (k < 0) c = std::conj(c);
      out.op = BOP_PHASE;
      out.cmask = b0 | (1u << g.qubits[1]);
      put(out.m, 0, c);
      return true;
    }
    case RBK_GATE_EX: case RBK_GATE_EY: case RBK_GATE_EZ:
      out.op = BOP_ROT;
      out.pauli = static_cast<uint8_t>(g.kind == RBK_GATE_EX ? 1 : g.kind == RBK_GATE_EY ? 2 : 3);
      out.param = g.param;
      out.scale = g.scale;
      out.offset = g.angles[0];
      return true;
    case RBK_GATE_SWAP: out.op = BOP_SWAP; return true;
    default: return false;
  }
}

}  // namespace
}  // namespace rbk

namespace {

int fail(int code, const std::string& m) { return rbk::set_last_error(code, m.c_str()); }

struct dev_free {
  void operator()(void* p) const { if (p) cudaFree(p); }
};
template <typename T>
using dptr = std::unique_ptr<T, dev_free>;

template <typename T>
T* dalloc(size_t count)
{
  void* p = nullptr;
  if (cudaMalloc(&p, sizeof(T) * (count ? count : 1)) != cudaSuccess) throw std::bad_alloc();
  return static_cast<T*>(p);
}

}  // namespace

struct rbk_batch {
  int precision = RBK_C128;
  int device = 0;
  int num_instances = 0;
  int total_params = 0;
  std::vector<int> param_begin, num_params;
  // small instances: one persistent launch
  int small_count = 0, small_max_n = 0, threads = 256;
  size_t smem = 0;
  std::vector<int> small_out;  // instance index of each small slot (largest first)
  dptr<rbk::binst> d_inst;
  dptr<rbk::bgate> d_gates;
  dptr<rbk::bterm> d_terms;
  dptr<double> d_theta, d_energy, d_grad;
  dptr<unsigned> d_next;
  std::vector<double> h_energy;  // per small slot (pinned below)
  double* h_theta = nullptr;     // pinned staging
  double* h_out = nullptr;       // pinned: energies[small_count] then grads[total_params]
  cudaStream_t stream = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  // large instances: the engine's adjoint sweep
  std::vector<int> large;
  std::vector<std::vector<rbk_circuit_gate>> large_gates;
  std::vector<std::string> large_strings;
  std::vector<std::vector<double>> large_coeffs;
  rbk_batch_stats stats{};
  // Worker threads for the large instances, each with its own workspaces by size.
  int workers = 8;
  std::vector<std::map<int, rbk::adjoint_workspace*>> pools;
  // Tile shape of the fused passes per qubit count of the large instances (the
  // fusion width: 2^11 or 2^12 amplitudes per tile), picked by timing.
  std::map<int, int> shape_of;

  ~rbk_batch()
  {
    cudaSetDevice(device);
    for (auto& pool : pools)
      for (auto& kv : pool) rbk::adjoint_workspace_destroy(kv.second);
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    if (h_theta) cudaFreeHost(h_theta);
    if (h_out) cudaFreeHost(h_out);
    if (stream) cudaStreamDestroy(stream);
  }
};

namespace {

// Records the small-instance job (copies in, the persistent launch, copies out) on b->stream.
int record_small(rbk_batch* b)
{
  const size_t np = static_cast<size_t>(b->total_params);
  if (cudaMemcpyAsync(b->d_theta.get(), b->h_theta, sizeof(double) * np, cudaMemcpyHostToDevice, b->stream) != cudaSuccess ||
      cudaMemsetAsync(b->d_grad.get(), 0, sizeof(double) * np, b->stream) != cudaSuccess ||
      cudaMemsetAsync(b->d_next.get(), 0, sizeof(unsigned), b->stream) != cudaSuccess)
    return fail(RBK_ERR_CUDA, "batch copies");
  int sms = 1;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, b->device);
  int per_sm = 1;
  if (b->precision == RBK_C128)
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, rbk::batch_adjoint_kernel<double>, b->threads, b->smem);
  else
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, rbk::batch_adjoint_kernel<float>, b->threads, b->smem);
  const int grid = std::max(1, std::min(b->small_count, std::max(1, per_sm) * sms));
  if (b->precision == RBK_C128)
    rbk::batch_adjoint_kernel<double><<<grid, b->threads, b->smem, b->stream>>>(
      b->d_inst.get(), b->small_count, b->d_gates.get(), b->d_terms.get(), b->d_theta.get(), b->d_energy.get(),
      b->d_grad.get(), b->d_next.get());
  else
    rbk::batch_adjoint_kernel<float><<<grid, b->threads, b->smem, b->stream>>>(
      b->d_inst.get(), b->small_count, b->d_gates.get(), b->d_terms.get(), b->d_theta.get(), b->d_energy.get(),
      b->d_grad.get(), b->d_next.get());
  if (cudaGetLastError() != cudaSuccess) return fail(RBK_ERR_CUDA, "batch kernel launch");
  if (cudaMemcpyAsync(b->h_out, b->d_energy.get(), sizeof(double) * b->small_count, cudaMemcpyDeviceToHost, b->stream) != cudaSuccess ||
      cudaMemcpyAsync(b->h_out + b->small_count, b->d_grad.get(), sizeof(double) * np, cudaMemcpyDeviceToHost, b->stream) != cudaSuccess)
    return fail(RBK_ERR_CUDA, "batch copies");
  return RBK_OK;
}

int sync_bounded(cudaStream_t s)
{
  const char* env = std::getenv("RBK_TIMEOUT_S");
  const double limit = env ? std::atof(env) : 600.0;
  const auto t0 = std::chrono::steady_clock::now();
  while (true) {
    const cudaError_t e = cudaStreamQuery(s);
    if (e == cudaSuccess) return RBK_OK;
    if (e != cudaErrorNotReady) return fail(RBK_ERR_CUDA, std::string("batch: ") + cudaGetErrorString(e));
    if (std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count() > limit)
      return fail(RBK_ERR_TIMEOUT, "batch: device wait timed out");
    std::this_thread::yield();
  }
}

// Fusion width of the large instances: for every qubit count from
// kTuneMinQubits up, one instance of that size is run through the sweep with
// each tile shape (2^11 amplitudes per tile in 4 CTAs per SM, 2^12 in 2, and
// 2^11 in 3 persistent CTAs that prefetch), and the fastest shape is kept for
// all instances of that size.  Below that size the default shape is kept: the
// sweeps there are bound by launches, not by the passes.
constexpr int kTuneMinQubits = 16;
int tune_shapes(rbk_batch* b)
{
  std::map<int, size_t> rep;  // qubit count -> index into b->large of the first instance of that size
  for (size_t k = 0; k < b->large.size(); ++k) {
    const int nt = static_cast<int>(b->large_coeffs[k].size() / 2);
    const int nq = static_cast<int>(b->large_strings[k].size() / static_cast<size_t>(nt));
    if (nq >= kTuneMinQubits && !rep.count(nq)) rep.emplace(nq, k);
  }
  for (const auto& kv : rep) {
    const int nq = kv.first;
    const size_t k = kv.second;
    const int i = b->large[k];
    const auto& gs = b->large_gates[k];
    const int nt = static_cast<int>(b->large_coeffs[k].size() / 2);
    std::vector<double> theta(static_cast<size_t>(std::max(1, b->num_params[i])), 0.1);
    std::vector<double> grad(theta.size());
    double energy = 0.0;
    rbk::adjoint_workspace* w = nullptr;
    if (int rc = rbk::adjoint_workspace_create(nq, b->precision, b->device, &w)) return rc;
    double best = 1e300;
    int best_shape = 2;
    int rc = RBK_OK;
    for (int shape : {2, 0, 3}) {
      rc = rbk::adjoint_workspace_set_shape(w, shape);
      double ms = 1e300;
      for (int r = 0; rc == RBK_OK && r < 3; ++r) {  // the first run warms up
        const auto t0 = std::chrono::steady_clock::now();
        rc = rbk::adjoint_run(w, gs.data(), static_cast<int>(gs.size()), theta.data(), b->num_params[i], nt,
                              b->large_strings[k].data(), b->large_coeffs[k].data(), &energy, grad.data());
        const double t = 1e3 * std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        if (r > 0) ms = std::min(ms, t);
      }
      if (rc != RBK_OK) break;
      if (ms < best) { best = ms; best_shape = shape; }
    }
    rbk::adjoint_workspace_destroy(w);
    if (rc != RBK_OK) return rc;
    b->shape_of[nq] = best_shape;
  }
  return RBK_OK;
}

}  // namespace

extern "C" int rbk_batch_tuned_shape(const rbk_batch* b, int num_qubits, int* shape)
{
  if (!b || !shape) return fail(RBK_ERR_INVALID, "null argument");
  const auto it = b->shape_of.find(num_qubits);
  *shape = it == b->shape_of.end() ? -1 : it->second;
  return RBK_OK;
}

extern "C" int rbk_batch_create(int precision, int device, int num_instances, const rbk_batch_instance* instances,
                                rbk_batch** out)
{
  try {
    if (!out || num_instances < 0 || (num_instances > 0 && !instances)) return fail(RBK_ERR_INVALID, "bad batch arguments");
    if (precision != RBK_C128 && precision != RBK_C64) return fail(RBK_ERR_INVALID, "unknown precision");
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return fail(RBK_ERR_CUDA, "no CUDA device available");
    if (device < 0 || device >= ndev) return fail(RBK_ERR_INVALID, "device out of range");
    if (cudaSetDevice(device) != cudaSuccess) return fail(RBK_ERR_CUDA, "cudaSetDevice");
    auto b = std::make_unique<rbk_batch>();
    b->precision = precision;
    b->device = device;
    b->num_instances = num_instances;
    const int small_limit = precision == RBK_C128 ? 12 : 13;
    std::vector<int> small;
    for (int i = 0; i < num_instances; ++i) {
      const auto& I = instances[i];
      if (I.num_qubits < 1 || I.num_qubits > 33 || I.num_gates < 0 || (I.num_gates > 0 && !I.gates) || I.num_params < 0 ||
          I.num_terms < 1 || !I.strings || !I.coeffs)
        return fail(RBK_ERR_INVALID, "instance " + std::to_string(i) + ": bad arguments");
      bool lowerable = I.num_qubits <= small_limit;
      for (int k = 0; k < I.num_gates; ++k) {
        const auto& g = I.gates[k];
        const bool two = g.kind == RBK_GATE_CNOT || g.kind == RBK_GATE_CZ || g.kind == RBK_GATE_U || g.kind == RBK_GATE_SWAP;
        if (g.qubits[0] < 0 || g.qubits[0] >= I.num_qubits || (two && (g.qubits[1] < 0 || g.qubits[1] >= I.num_qubits ||
                                                                      g.qubits[1] == g.qubits[0])))
          return fail(RBK_ERR_INVALID, "instance " + std::to_string(i) + ": qubit out of range");
        if (g.param >= I.num_params) return fail(RBK_ERR_INVALID, "instance " + std::to_string(i) + ": parameter out of range");
        if (g.param >= 0 && g.kind != RBK_GATE_EX && g.kind != RBK_GATE_EY && g.kind != RBK_GATE_EZ)
          return fail(RBK_ERR_UNSUPPORTED, "only EX, EY and EZ gates take parameters");
        rbk::bgate tmp;
        if (!rbk::lower_gate(g, tmp)) return fail(RBK_ERR_INVALID, "instance " + std::to_string(i) + ": unknown gate kind");
      }
      b->param_begin.push_back(b->total_params);
      b->num_params.push_back(I.num_params);
      b->total_params += I.num_params;
      (lowerable ? small : b->large).push_back(i);
    }
    // Small instances, largest first: the work counter hands the long jobs out early.
    std::stable_sort(small.begin(), small.end(),
                     [&](int x, int y) { return instances[x].num_qubits > instances[y].num_qubits; });
    std::vector<rbk::binst> inst;
    std::vector<rbk::bgate> gates;
    std::vector<rbk::bterm> terms;
    static const std::complex<double> pow_mi[4] = {{1, 0}, {0, -1}, {-1, 0}, {0, 1}};
    for (int slot = 0; slot < static_cast<int>(small.size()); ++slot) {
      const auto& I = instances[small[slot]];
      rbk::binst d{};
      d.n = I.num_qubits;
      d.num_gates = I.num_gates;
      d.gate_begin = static_cast<int32_t>(gates.size());
      d.param_begin = b->param_begin[small[slot]];
      d.num_terms = I.num_terms;
      d.term_begin = static_cast<int32_t>(terms.size());
      d.out_index = slot;
      for (int k = 0; k < I.num_gates; ++k) {
        rbk::bgate g;
        rbk::lower_gate(I.gates[k], g);
        gates.push_back(g);
      }
      for (int t = 0; t < I.num_terms; ++t) {
        uint32_t x = 0, y = 0, z = 0;
        for (int q = 0; q < I.num_qubits; ++q) {
          const char c = I.strings[static_cast<size_t>(t) * I.num_qubits + q];
          if (c == 'X') x |= 1u << q;
          else if (c == 'Y') y |= 1u << q;
          else if (c == 'Z') z |= 1u << q;
          else if (c != 'I') return fail(RBK_ERR_INVALID, "Pauli strings use the characters I, X, Y, Z");
        }
        const auto w = std::complex<double>{I.coeffs[2 * t], I.coeffs[2 * t + 1]} * pow_mi[__builtin_popcount(y) & 3];
        terms.push_back(rbk::bterm{x | y, y | z, {w.real(), w.imag()}});
      }
      inst.push_back(d);
      b->small_max_n = std::max(b->small_max_n, I.num_qubits);
    }
    b->small_count = static_cast<int>(small.size());
    b->small_out = small;
    std::stable_sort(b->large.begin(), b->large.end(),
                     [&](int x, int y) { return instances[x].num_qubits > instances[y].num_qubits; });
    for (int li : b->large) {
      const auto& I = instances[li];
      b->large_gates.emplace_back(I.gates, I.gates + I.num_gates);
      b->large_strings.emplace_back(I.strings, static_cast<size_t>(I.num_terms) * I.num_qubits);
      b->large_coeffs.emplace_back(I.coeffs, I.coeffs + 2 * I.num_terms);
    }
    if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess) return fail(RBK_ERR_CUDA, "stream");
    const size_t np = static_cast<size_t>(b->total_params);
    if (cudaMallocHost(reinterpret_cast<void**>(&b->h_theta), sizeof(double) * (np ? np : 1)) != cudaSuccess ||
        cudaMallocHost(reinterpret_cast<void**>(&b->h_out), sizeof(double) * (np + b->small_count + 1)) != cudaSuccess)
      return fail(RBK_ERR_OOM, "pinned host memory");
    std::memset(b->h_theta, 0, sizeof(double) * (np ? np : 1));
    b->stats.num_small = b->small_count;
    b->stats.num_large = static_cast<int>(b->large.size());
    if (b->small_count > 0) {
      b->d_inst.reset(dalloc<rbk::binst>(inst.size()));
      b->d_gates.reset(dalloc<rbk::bgate>(gates.size()));
      b->d_terms.reset(dalloc<rbk::bterm>(terms.size()));
      b->d_theta.reset(dalloc<double>(np));
      b->d_grad.reset(dalloc<double>(np));
      b->d_energy.reset(dalloc<double>(b->small_count));
      b->d_next.reset(dalloc<unsigned>(1));
      if (cudaMemcpy(b->d_inst.get(), inst.data(), sizeof(rbk::binst) * inst.size(), cudaMemcpyHostToDevice) != cudaSuccess ||
          (!gates.empty() && cudaMemcpy(b->d_gates.get(), gates.data(), sizeof(rbk::bgate) * gates.size(), cudaMemcpyHostToDevice) != cudaSuccess) ||
          cudaMemcpy(b->d_terms.get(), terms.data(), sizeof(rbk::bterm) * terms.size(), cudaMemcpyHostToDevice) != cudaSuccess)
        return fail(RBK_ERR_CUDA, "batch upload");
      const size_t amp = precision == RBK_C128 ? 16 : 8;
      b->smem = 2 * (size_t(1) << b->small_max_n) * amp;
      cudaError_t e = precision == RBK_C128
                          ? cudaFuncSetAttribute(rbk::batch_adjoint_kernel<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(b->smem))
                          : cudaFuncSetAttribute(rbk::batch_adjoint_kernel<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(b->smem));
      if (e != cudaSuccess) return fail(RBK_ERR_CUDA, std::string("batch shared memory: ") + cudaGetErrorString(e));
      // Autotuner: time each CTA size on the batch's own small instances (theta = 0) and keep the fastest.
      cudaEvent_t e0, e1;
      cudaEventCreate(&e0);
      cudaEventCreate(&e1);
      float best = 1e30f;
      int best_threads = 256;
      for (int threads : {128, 256, 512, 1024}) {
        int per_sm = 0;
        if (precision == RBK_C128)
          cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, rbk::batch_adjoint_kernel<double>, threads, b->smem);
        else
          cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, rbk::batch_adjoint_kernel<float>, threads, b->smem);
        if (per_sm < 1) continue;  // this CTA size does not fit (registers or shared memory)
        b->threads = threads;
        cudaEventRecord(e0, b->stream);
        if (int rc = record_small(b.get())) { cudaEventDestroy(e0); cudaEventDestroy(e1); return rc; }
        cudaEventRecord(e1, b->stream);
        if (int rc = sync_bounded(b->stream)) { cudaEventDestroy(e0); cudaEventDestroy(e1); return rc; }
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, e0, e1);
        if (ms < best) { best = ms; best_threads = threads; }
      }
      cudaEventDestroy(e0);
      cudaEventDestroy(e1);
      b->threads = best_threads;
      b->stats.threads = best_threads;
      b->stats.small_ms = best;
      // The small-instance job as a CUDA graph, replayed by every rbk_batch_run.
      if (cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess)
        return fail(RBK_ERR_CUDA, "graph capture");
      const int rc = record_small(b.get());
      const cudaError_t ce = cudaStreamEndCapture(b->stream, &b->graph);
      if (rc) return rc;
      if (ce != cudaSuccess || cudaGraphInstantiate(&b->exec, b->graph, 0) != cudaSuccess)
        return fail(RBK_ERR_CUDA, "graph instantiate");
    }
    if (int rc = tune_shapes(b.get())) return rc;
    *out = b.release();
    return RBK_OK;
  } catch (std::bad_alloc const&) {
    return fail(RBK_ERR_OOM, "batch: memory exhausted");
  } catch (std::exception const& e) {
    return fail(RBK_ERR_STATE, e.what());
  }
}

extern "C" int rbk_batch_run(rbk_batch* b, const double* theta, double* energies, double* grads)
{
  try {
    if (!b || !energies || (b->total_params > 0 && (!theta || !grads))) return fail(RBK_ERR_INVALID, "bad batch arguments");
    if (cudaSetDevice(b->device) != cudaSuccess) return fail(RBK_ERR_CUDA, "cudaSetDevice");
    const auto t0 = std::chrono::steady_clock::now();
    const size_t np = static_cast<size_t>(b->total_params);
    if (np) std::memcpy(b->h_theta, theta, sizeof(double) * np);
    if (b->small_count > 0 && cudaGraphLaunch(b->exec, b->stream) != cudaSuccess) return fail(RBK_ERR_CUDA, "graph launch");
    // Large instances meanwhile, through the engine's adjoint sweep: worker
    // threads take them largest first, each on its own streams and reusable
    // state pairs, so that host planning overlaps device work.
    if (!b->large.empty()) {
      if (b->pools.empty()) b->pools.resize(static_cast<size_t>(b->workers));
      std::atomic<size_t> next{0};
      std::atomic<int> first_rc{RBK_OK};
      std::mutex err_mu;
      std::string err;
      auto work = [&](int wid) {
        cudaSetDevice(b->device);
        auto& pool = b->pools[static_cast<size_t>(wid)];
        while (first_rc.load() == RBK_OK) {
          const size_t k = next.fetch_add(1);
          if (k >= b->large.size()) break;
          const int i = b->large[k];
          const int pb = b->param_begin[i];
          const auto& gs = b->large_gates[k];
          const int nt = static_cast<int>(b->large_coeffs[k].size() / 2);
          const int nq = static_cast<int>(b->large_strings[k].size() / static_cast<size_t>(nt));
          int rc = RBK_OK;
          auto it = pool.find(nq);
          if (it == pool.end()) {
            rbk::adjoint_workspace* w = nullptr;
            rc = rbk::adjoint_workspace_create(nq, b->precision, b->device, &w);
            const auto sh = b->shape_of.find(nq);
            if (rc == RBK_OK && sh != b->shape_of.end()) rc = rbk::adjoint_workspace_set_shape(w, sh->second);
            if (rc == RBK_OK) it = pool.emplace(nq, w).first;
            else if (w) rbk::adjoint_workspace_destroy(w);
          }
          if (rc == RBK_OK)
            rc = rbk::adjoint_run(it->second, gs.data(), static_cast<int>(gs.size()), theta + pb, b->num_params[i], nt,
                                  b->large_strings[k].data(), b->large_coeffs[k].data(), &energies[i], grads + pb);
          if (rc != RBK_OK) {
            int expected = RBK_OK;
            if (first_rc.compare_exchange_strong(expected, rc)) {
              std::lock_guard<std::mutex> lk(err_mu);
              err = rbk_last_error();
            }
          }
        }
      };
      std::vector<std::thread> threads;
      for (int t = 1; t < b->workers; ++t) threads.emplace_back(work, t);
      work(0);
      for (auto& t : threads) t.join();
      if (first_rc.load() != RBK_OK) return fail(first_rc.load(), "batch: " + err);
    }
    if (b->small_count > 0) {
      if (int rc = sync_bounded(b->stream)) return rc;
      for (int slot = 0; slot < b->small_count; ++slot) {
        const int i = b->small_out[slot];
        energies[i] = b->h_out[slot];
        const int pb = b->param_begin[i];
        for (int p = 0; p < b->num_params[i]; ++p) grads[pb + p] = b->h_out[b->small_count + pb + p];
      }
    }
    b->stats.last_run_ms = 1e3 * std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    return RBK_OK;
  } catch (std::bad_alloc const&) {
    return fail(RBK_ERR_OOM, "batch: memory exhausted");
  } catch (std::exception const& e) {
    return fail(RBK_ERR_STATE, e.what());
  }
}

extern "C" int rbk_batch_set_workers(rbk_batch* b, int workers)
{
  if (!b || workers < 1 || workers > 64) return fail(RBK_ERR_INVALID, "workers must be between 1 and 64");
  cudaSetDevice(b->device);
  for (auto& pool : b->pools)
    for (auto& kv : pool) rbk::adjoint_workspace_destroy(kv.second);
  b->pools.clear();
  b->workers = workers;
  return RBK_OK;
}

extern "C" int rbk_batch_get_stats(const rbk_batch* b, rbk_batch_stats* out)
{
  if (!b || !out) return fail(RBK_ERR_INVALID, "null argument");
  *out = b->stats;
  return RBK_OK;
}

extern "C" int rbk_batch_destroy(rbk_batch* b)
{
  if (b) {
    cudaSetDevice(b->device);
    delete b;
  }
  return RBK_OK;
}
