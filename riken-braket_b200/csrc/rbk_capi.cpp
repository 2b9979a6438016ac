// rbk_capi.cpp -- the C ABI of include/rbk.h: state handles, named gates,
// the deferred gate queue, execution of planned passes, observables.
#include "rbk.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <chrono>
#include <cmath>
#include <complex>
#include <cstdlib>
#include <cstring>
#include <exception>
#include <memory>
#include <random>
#include <string>
#include <thread>
#include <vector>

#include "rbk_adjoint.h"
#include "rbk_rotate_plan.h"
#include "rbk_internal.h"
#include "rbk_kernels.h"
#include "rbk_plan.h"

using rbk::hgate;

struct rbk_state {
  int n = 0;
  int precision = RBK_C128;
  int device = 0;
  void* amps = nullptr;
  cudaStream_t stream = nullptr;
  double* d_partials = nullptr;
  double* d_out = nullptr;
  double* h_out = nullptr;  // pinned
  float* d_tc_w = nullptr;   // W_hi, W_lo of the tensor-core unitaries (largest k), kept between calls
  int* d_tc_flag = nullptr;  // set by a tensor-core unitary whose bounded wait ran out (sticky)
  int* h_tc_flag = nullptr;  // pinned copy, read at every bounded_sync
  std::vector<int> perm, inv;
  std::vector<hgate> queue;
  bool deferred = true;
  bool in_fusion = false;
  int fusion_mode = 0;       // 1: c64 fusion blocks of 5-6 qubits become dense unitaries on tensor cores
  size_t fusion_begin = 0;   // queue index of the current BEGIN FUSION
  int dense_budget = 0;
  int shape = 2;
  rbk_stats stats{};
  cudaEvent_t ev_first = nullptr, ev_last = nullptr, ev_sync = nullptr;
  bool timing_started = false;
  bool owns_stream = true;  // false when the stream is borrowed from another state
  std::mt19937_64 rng{1};   // bra::state's random_number_generator_ (bra/include/bra/state.hpp:459-479)
};

namespace {

thread_local std::string g_error;

int fail(int code, const std::string& msg)
{
  g_error = msg;
  return code;
}

int cuda_fail(cudaError_t e, const char* what)
{
  const int code = (e == cudaErrorMemoryAllocation) ? RBK_ERR_OOM : RBK_ERR_CUDA;
  return fail(code, std::string(what) + ": " + cudaGetErrorString(e));
}

#define RBK_CUDA(call)                                    \
  do {                                                    \
    cudaError_t e_ = (call);                              \
    if (e_ != cudaSuccess) return cuda_fail(e_, #call);   \
  } while (0)

struct device_guard {
  int prev = -1;
  explicit device_guard(int dev)
  {
    if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
    if (prev != dev) cudaSetDevice(dev);
  }
  ~device_guard() { if (prev >= 0) cudaSetDevice(prev); }
};

double wait_timeout_seconds()
{
  const char* v = std::getenv("RBK_TIMEOUT_S");
  if (v) { const double t = std::atof(v); if (t > 0) return t; }
  return 600.0;
}

// Bounded wait for everything issued on the state's stream.
// Waits for the state's stream, polling: the first 200 us without sleeping
// (short device work returns at once), then with sleeps that grow to 200 us,
// so a wait ends at most that long after the device does.  Bounded by the
// RBK_TIMEOUT_S limit.  Also reports a tensor-core unitary that gave up.
int bounded_sync(rbk_state* s)
{
  RBK_CUDA(cudaEventRecord(s->ev_sync, s->stream));
  const auto t0 = std::chrono::steady_clock::now();
  const double limit = wait_timeout_seconds();
  int sleep_us = 5;
  while (true) {
    const cudaError_t e = cudaEventQuery(s->ev_sync);
    if (e == cudaSuccess) break;
    if (e != cudaErrorNotReady) return cuda_fail(e, "device execution");
    const double el = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    if (el > limit) return fail(RBK_ERR_TIMEOUT, "timed out waiting for the device");
    if (el > 2e-4) {
      std::this_thread::sleep_for(std::chrono::microseconds(sleep_us));
      if (sleep_us < 200) sleep_us *= 2;
    }
  }
  if (s->h_tc_flag && *s->h_tc_flag) return fail(RBK_ERR_TIMEOUT, "tensor-core unitary: a wait for the MMAs ran out");
  return RBK_OK;
}

inline size_t amp_bytes(int precision) { return precision == RBK_C128 ? 16 : 8; }

rbk::plan_params params_of(const rbk_state* s)
{
  rbk::plan_params p{};
  p.n = s->n;
  rbk::shape_bits(s->precision, s->shape, &p.K, &p.R);
  p.LOW = s->precision == RBK_C128 ? rbk::precision_traits<double>::LOW : rbk::precision_traits<float>::LOW;
  p.vbits = s->precision == RBK_C128 ? 0 : 1;
  p.dense_budget = s->dense_budget > 0 ? s->dense_budget : (s->precision == RBK_C128 ? 12 : 14);
  return p;
}

int tile_bits(const rbk_state* s)
{
  int K = 0, R = 0;
  rbk::shape_bits(s->precision, s->shape, &K, &R);
  return K;
}

int mark_launch_start(rbk_state* s)
{
  if (!s->timing_started) {
    RBK_CUDA(cudaEventRecord(s->ev_first, s->stream));
    s->timing_started = true;
  }
  return RBK_OK;
}

int run_passes(rbk_state* s, const std::vector<rbk::dev_pass>& passes)
{
  for (const auto& pass : passes) {
    const cudaError_t e = s->precision == RBK_C128
      ? rbk::launch_tile_pass<double>(s->amps, s->n, pass, s->shape, s->stream)
      : rbk::launch_tile_pass<float>(s->amps, s->n, pass, s->shape, s->stream);
    if (e != cudaSuccess) return cuda_fail(e, "tile pass launch");
    ++s->stats.kernel_launches;
  }
  return RBK_OK;
}

int flush(rbk_state* s)
{
  if (s->queue.empty()) return RBK_OK;
  device_guard g(s->device);
  int rc = mark_launch_start(s);
  if (rc) return rc;
  try {
    if (s->n >= tile_bits(s)) {
      std::vector<rbk::dev_pass> passes;
      rbk::plan_passes(params_of(s), s->queue, s->perm, s->inv, passes);
      rc = run_passes(s, passes);
      if (rc) { s->queue.clear(); return rc; }
      s->stats.passes += passes.size();
    } else {
      for (const hgate& h : s->queue) {
        if (h.kind == rbk::HK_SWAP) {
          const int pa = s->perm[h.target], pb = s->perm[h.target2];
          s->perm[h.target] = pb; s->perm[h.target2] = pa;
          s->inv[pa] = h.target2; s->inv[pb] = h.target;
          continue;
        }
        const rbk::gate_rec r = rbk::to_physical(h, s->perm);
        const cudaError_t e = s->precision == RBK_C128 ? rbk::launch_gate<double>(s->amps, s->n, r, s->stream)
                                                      : rbk::launch_gate<float>(s->amps, s->n, r, s->stream);
        if (e != cudaSuccess) { s->queue.clear(); return cuda_fail(e, "gate launch"); }
        ++s->stats.gate_launches;
        ++s->stats.kernel_launches;
      }
    }
  } catch (std::exception const& ex) {
    s->queue.clear();
    return fail(RBK_ERR_STATE, std::string("planner: ") + ex.what());
  }
  s->queue.clear();
  RBK_CUDA(cudaEventRecord(s->ev_last, s->stream));
  return RBK_OK;
}

// Moves the data so that the layout map becomes `target` (logical qubit q on
// physical bit target[q]).
int move_layout(rbk_state* s, const std::vector<int>& target)
{
  int rc = flush(s);
  if (rc) return rc;
  if (s->perm == target) return RBK_OK;
  device_guard g(s->device);
  if (s->n < tile_bits(s)) {
    // Small states: move qubits to their targets one transposition at a time.
    for (int q = 0; q < s->n; ++q) {
      while (s->perm[q] != target[q]) {
        const int home = target[q];
        const int other = s->inv[home];  // logical qubit sitting on q's target bit
        const int pq = s->perm[q];
        // Swap physical bits pq and home with three controlled-X permutations.
        for (int step = 0; step < 3; ++step) {
          rbk::gate_rec r{};
          r.kind = rbk::OPK_X;
          r.target = static_cast<uint8_t>(step == 1 ? pq : home);
          r.cmask = 1ull << (step == 1 ? home : pq);
          const cudaError_t e = s->precision == RBK_C128 ? rbk::launch_gate<double>(s->amps, s->n, r, s->stream)
                                                        : rbk::launch_gate<float>(s->amps, s->n, r, s->stream);
          if (e != cudaSuccess) return cuda_fail(e, "swap launch");
          ++s->stats.kernel_launches;
        }
        s->perm[q] = home; s->inv[home] = q;
        s->perm[other] = pq; s->inv[pq] = other;
      }
    }
    return RBK_OK;
  }
  std::vector<rbk::dev_pass> passes;
  try {
    rbk::plan_layout(params_of(s), s->perm, s->inv, target, passes);
  } catch (std::exception const& ex) {
    return fail(RBK_ERR_STATE, std::string("planner: ") + ex.what());
  }
  rc = mark_launch_start(s);
  if (rc) return rc;
  rc = run_passes(s, passes);
  if (rc) return rc;
  s->stats.relabel_passes += passes.size();
  RBK_CUDA(cudaEventRecord(s->ev_last, s->stream));
  return RBK_OK;
}

int canonicalize(rbk_state* s)
{
  std::vector<int> identity(static_cast<size_t>(s->n));
  for (int q = 0; q < s->n; ++q) identity[static_cast<size_t>(q)] = q;
  return move_layout(s, identity);
}

// A layout map from the caller: a permutation of 0..n-1.
int read_layout(const rbk_state* s, const uint32_t* perm, std::vector<int>& out)
{
  if (!perm) return fail(RBK_ERR_INVALID, "null permutation");
  out.assign(static_cast<size_t>(s->n), -1);
  std::vector<char> seen(static_cast<size_t>(s->n), 0);
  for (int q = 0; q < s->n; ++q) {
    if (perm[q] >= static_cast<uint32_t>(s->n) || seen[perm[q]])
      return fail(RBK_ERR_INVALID, "not a permutation of the state's qubits");
    seen[perm[q]] = 1;
    out[static_cast<size_t>(q)] = static_cast<int>(perm[q]);
  }
  return RBK_OK;
}

int check_state(const rbk_state* s)
{
  if (!s) return fail(RBK_ERR_INVALID, "null state");
  return RBK_OK;
}

// Validates target/control qubits: in range and pairwise distinct.
int check_qubits(const rbk_state* s, const uint32_t* qs, int count, uint64_t* mask_out)
{
  if (count < 0) return fail(RBK_ERR_INVALID, "negative qubit count");
  if (count > 0 && !qs) return fail(RBK_ERR_INVALID, "null qubit array");
  uint64_t m = 0;
  for (int i = 0; i < count; ++i) {
    if (qs[i] >= static_cast<uint32_t>(s->n)) return fail(RBK_ERR_INVALID, "qubit index out of range");
    const uint64_t b = 1ull << qs[i];
    if (m & b) return fail(RBK_ERR_INVALID, "repeated qubit");
    m |= b;
  }
  *mask_out = m;
  return RBK_OK;
}

int enqueue(rbk_state* s, const hgate& g)
{
  s->queue.push_back(g);
  ++s->stats.gates_issued;
  if (!s->deferred && !s->in_fusion) return flush(s);
  return RBK_OK;
}

int enqueue_target(rbk_state* s, uint8_t kind, uint32_t target, const uint32_t* controls, int nc,
                   const double* m, uint8_t diag_one = 0)
{
  int rc = check_state(s);
  if (rc) return rc;
  uint64_t cm = 0;
  rc = check_qubits(s, controls, nc, &cm);
  if (rc) return rc;
  if (target >= static_cast<uint32_t>(s->n)) return fail(RBK_ERR_INVALID, "target qubit out of range");
  if (cm & (1ull << target)) return fail(RBK_ERR_INVALID, "target qubit is also a control qubit");
  hgate g{};
  g.kind = kind;
  g.target = static_cast<int8_t>(target);
  g.target2 = -1;
  g.diag_one = diag_one;
  g.cmask = cm;
  if (m) std::memcpy(g.m, m, sizeof(g.m));
  return enqueue(s, g);
}

using cplx = std::complex<double>;

// ket::utility::exp_i (ket/include/ket/utility/exp_i.hpp:21-36)
cplx exp_i(double theta) { return std::exp(cplx{0.0, theta}); }

constexpr double kOneDivRootTwo = 0.707106781186547524400844362104849039284835937688474036588;
constexpr double kTwoPi = 6.28318530717958647692528676655900576839433879875021164195;

void put(double* m, int k, cplx v) { m[2 * k] = v.real(); m[2 * k + 1] = v.imag(); }

// Phase on the all-ones subspace of `qubits` (phase_shift_coeff form).
int enqueue_phase(rbk_state* s, cplx coeff, const uint32_t* qubits, int nq)
{
  int rc = check_state(s);
  if (rc) return rc;
  if (nq < 1) return fail(RBK_ERR_INVALID, "phase shift needs at least one qubit");
  uint64_t mask = 0;
  rc = check_qubits(s, qubits, nq, &mask);
  if (rc) return rc;
  hgate g{};
  g.target2 = -1;
  if (coeff == cplx{-1.0, 0.0}) {
    g.kind = rbk::OPK_NEG;
    g.target = -1;
    g.cmask = mask;
  } else {
    g.kind = rbk::OPK_DIAG;
    g.target = static_cast<int8_t>(qubits[nq - 1]);
    g.cmask = mask & ~(1ull << qubits[nq - 1]);
    g.diag_one = 1;
    put(g.m, 0, cplx{1.0, 0.0});
    put(g.m, 1, coeff);
  }
  return enqueue(s, g);
}

template <typename F>
int guarded(F&& f)
{
  try { return f(); }
  catch (std::bad_alloc const&) { return fail(RBK_ERR_OOM, "host memory exhausted"); }
  catch (std::exception const& e) { return fail(RBK_ERR_STATE, e.what()); }
}

// Reductions need an identity-free view: the kernels work on physical bits.
template <typename Fn>
int launch_reduction(rbk_state* s, Fn&& fn)
{
  int rc = flush(s);
  if (rc) return rc;
  device_guard g(s->device);
  rc = mark_launch_start(s);
  if (rc) return rc;
  const cudaError_t e = fn();
  if (e != cudaSuccess) return cuda_fail(e, "reduction launch");
  s->stats.kernel_launches += 2;
  ++s->stats.reduction_passes;
  RBK_CUDA(cudaEventRecord(s->ev_last, s->stream));
  return RBK_OK;
}

int read_out(rbk_state* s, int count)
{
  RBK_CUDA(cudaMemcpyAsync(s->h_out, s->d_out, sizeof(double) * count, cudaMemcpyDeviceToHost, s->stream));
  return bounded_sync(s);
}

// Pauli strings (one character per logical qubit) as physical flip/sign masks,
// grouped by flip mask:  (P psi)(i) = (-i)^{#Y} (-1)^{popcount(i & (Y|Z))} psi(i ^ (X|Y))
// (ket/include/ket/gate/utility/pauli_index_coeff.hpp:17-59).  Uses s->perm:
// call after the queued gates have run.
struct pauli_group_terms { uint64_t flip; rbk::pauli_terms terms; };

int group_pauli_terms(const rbk_state* s, int num_terms, const char* strings, const double* coeffs,
                      std::vector<pauli_group_terms>& groups)
{
  struct term { uint64_t flip, sign; cplx w; };
  std::vector<term> terms;
  for (int t = 0; t < num_terms; ++t) {
    uint64_t x = 0, y = 0, z = 0;
    for (int k = 0; k < s->n; ++k) {
      const char c = strings[static_cast<size_t>(t) * s->n + k];
      const uint64_t b = 1ull << s->perm[k];
      if (c == 'X') x |= b;
      else if (c == 'Y') y |= b;
      else if (c == 'Z') z |= b;
      else if (c != 'I') return fail(RBK_ERR_INVALID, "Pauli strings use the characters I, X, Y, Z");
    }
    static const cplx pow_mi[4] = {{1, 0}, {0, -1}, {-1, 0}, {0, 1}};
    const cplx w = cplx{coeffs[2 * t], coeffs[2 * t + 1]} * pow_mi[__builtin_popcountll(y) & 3];
    terms.push_back({x | y, y | z, w});
  }
  std::vector<char> done(terms.size(), 0);
  for (size_t i = 0; i < terms.size(); ++i) {
    if (done[i]) continue;
    pauli_group_terms g{};
    g.flip = terms[i].flip;
    for (size_t j = i; j < terms.size() && g.terms.count < rbk::kMaxPauliTerms; ++j) {
      if (done[j] || terms[j].flip != terms[i].flip) continue;
      g.terms.sign[g.terms.count] = terms[j].sign;
      g.terms.w[g.terms.count][0] = terms[j].w.real();
      g.terms.w[g.terms.count][1] = terms[j].w.imag();
      ++g.terms.count;
      done[j] = 1;
    }
    groups.push_back(g);
  }
  return RBK_OK;
}

// sum over one flip-mask group of Pauli terms (physical masks).
int pauli_group(rbk_state* s, uint64_t flip, const rbk::pauli_terms& t, double* out2)
{
  int rc = launch_reduction(s, [&] {
    return s->precision == RBK_C128 ? rbk::launch_pauli<double>(s->amps, s->n, flip, t, s->d_partials, s->d_out, s->stream)
                                    : rbk::launch_pauli<float>(s->amps, s->n, flip, t, s->d_partials, s->d_out, s->stream);
  });
  if (rc) return rc;
  rc = read_out(s, 2);
  if (rc) return rc;
  out2[0] = s->h_out[0];
  out2[1] = s->h_out[1];
  return RBK_OK;
}

}  // namespace

int rbk::set_last_error(int code, const char* msg) { return fail(code, msg); }

extern "C" {

const char* rbk_last_error(void) { return g_error.c_str(); }
int rbk_version(void) { return 1; }

int rbk_pass_descriptor_bytes(uint64_t* out)
{
  if (!out) return rbk::set_last_error(RBK_ERR_INVALID, "null pointer");
  *out = sizeof(rbk::dev_pass);
  return RBK_OK;
}

int rbk_state_create(int num_qubits, int precision, uint64_t initial_index, int device, rbk_state** out)
{
  return guarded([&]() -> int {
    if (!out) return fail(RBK_ERR_INVALID, "null output pointer");
    *out = nullptr;
    if (precision != RBK_C128 && precision != RBK_C64) return fail(RBK_ERR_INVALID, "unknown precision");
    const int max_q = precision == RBK_C128 ? 33 : 34;
    if (num_qubits < 1 || num_qubits > max_q) return fail(RBK_ERR_INVALID, "number of qubits out of range");
    if (initial_index >= (1ull << num_qubits)) return fail(RBK_ERR_INVALID, "initial index out of range");
    int ndev = 0;
    cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess || ndev == 0) return fail(RBK_ERR_CUDA, "no CUDA device available");
    if (device < 0 || device >= ndev) return fail(RBK_ERR_INVALID, "device index out of range");
    device_guard g(device);
    auto* s = new rbk_state();
    s->n = num_qubits;
    s->precision = precision;
    s->device = device;
    s->perm.resize(num_qubits);
    s->inv.resize(num_qubits);
    for (int q = 0; q < num_qubits; ++q) s->perm[q] = s->inv[q] = q;
    auto cleanup = [&](int rc) { rbk_state_destroy(s); return rc; };
    const size_t bytes = amp_bytes(precision) << num_qubits;
    e = cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) return cleanup(cuda_fail(e, "cudaStreamCreate"));
    e = cudaMalloc(&s->amps, bytes);
    if (e != cudaSuccess) return cleanup(cuda_fail(e, "cudaMalloc(state)"));
    e = cudaMalloc(reinterpret_cast<void**>(&s->d_partials), sizeof(double) * rbk::reduction_scratch_doubles());
    if (e != cudaSuccess) return cleanup(cuda_fail(e, "cudaMalloc(scratch)"));
    e = cudaMalloc(reinterpret_cast<void**>(&s->d_out), sizeof(double) * 4 * (rbk::kMaxQubits + 8));
    if (e != cudaSuccess) return cleanup(cuda_fail(e, "cudaMalloc(results)"));
    e = cudaMallocHost(reinterpret_cast<void**>(&s->h_out), sizeof(double) * 4 * (rbk::kMaxQubits + 8));
    if (e != cudaSuccess) return cleanup(cuda_fail(e, "cudaMallocHost"));
    for (cudaEvent_t* ev : {&s->ev_first, &s->ev_last, &s->ev_sync}) {
      e = cudaEventCreate(ev);
      if (e != cudaSuccess) return cleanup(cuda_fail(e, "cudaEventCreate"));
    }
    e = precision == RBK_C128 ? rbk::launch_set_basis<double>(s->amps, num_qubits, initial_index, s->stream)
                              : rbk::launch_set_basis<float>(s->amps, num_qubits, initial_index, s->stream);
    if (e != cudaSuccess) return cleanup(cuda_fail(e, "set basis"));
    ++s->stats.kernel_launches;
    const int rc = bounded_sync(s);
    if (rc) return cleanup(rc);
    *out = s;
    return RBK_OK;
  });
}

int rbk_state_destroy(rbk_state* s)
{
  if (!s) return RBK_OK;
  device_guard g(s->device);
  if (s->stream) cudaStreamSynchronize(s->stream);
  if (s->amps) cudaFree(s->amps);
  if (s->d_partials) cudaFree(s->d_partials);
  if (s->d_out) cudaFree(s->d_out);
  if (s->h_out) cudaFreeHost(s->h_out);
  if (s->d_tc_w) cudaFree(s->d_tc_w);
  if (s->d_tc_flag) cudaFree(s->d_tc_flag);
  if (s->h_tc_flag) cudaFreeHost(s->h_tc_flag);
  for (cudaEvent_t ev : {s->ev_first, s->ev_last, s->ev_sync}) if (ev) cudaEventDestroy(ev);
  if (s->stream && s->owns_stream) cudaStreamDestroy(s->stream);
  delete s;
  return RBK_OK;
}

int rbk_state_num_qubits(const rbk_state* s, int* out)
{
  if (int rc = check_state(s)) return rc;
  if (!out) return fail(RBK_ERR_INVALID, "null output pointer");
  *out = s->n;
  return RBK_OK;
}

int rbk_state_precision(const rbk_state* s, int* out)
{
  if (int rc = check_state(s)) return rc;
  if (!out) return fail(RBK_ERR_INVALID, "null output pointer");
  *out = s->precision;
  return RBK_OK;
}

int rbk_state_reset(rbk_state* s, uint64_t index)
{
  if (int rc = check_state(s)) return rc;
  if (index >= (1ull << s->n)) return fail(RBK_ERR_INVALID, "index out of range");
  s->queue.clear();
  s->in_fusion = false;
  for (int q = 0; q < s->n; ++q) s->perm[q] = s->inv[q] = q;
  device_guard g(s->device);
  if (int rc = mark_launch_start(s)) return rc;
  const cudaError_t e = s->precision == RBK_C128 ? rbk::launch_set_basis<double>(s->amps, s->n, index, s->stream)
                                                : rbk::launch_set_basis<float>(s->amps, s->n, index, s->stream);
  if (e != cudaSuccess) return cuda_fail(e, "set basis");
  ++s->stats.kernel_launches;
  RBK_CUDA(cudaEventRecord(s->ev_last, s->stream));
  return RBK_OK;
}

int rbk_state_upload(rbk_state* s, const void* host, uint64_t offset, uint64_t count)
{
  return guarded([&]() -> int {
    if (int rc = check_state(s)) return rc;
    const uint64_t size = 1ull << s->n;
    if (!host && count) return fail(RBK_ERR_INVALID, "null host pointer");
    if (offset > size || count > size - offset) return fail(RBK_ERR_INVALID, "range out of bounds");
    if (offset == 0 && count == size) {
      s->queue.clear();
      for (int q = 0; q < s->n; ++q) s->perm[q] = s->inv[q] = q;
    } else if (int rc = canonicalize(s)) {
      return rc;
    }
    device_guard g(s->device);
    const size_t ab = amp_bytes(s->precision);
    RBK_CUDA(cudaMemcpyAsync(static_cast<char*>(s->amps) + offset * ab, host, count * ab, cudaMemcpyHostToDevice, s->stream));
    return bounded_sync(s);
  });
}

int rbk_state_download(rbk_state* s, void* host, uint64_t offset, uint64_t count)
{
  return guarded([&]() -> int {
    if (int rc = check_state(s)) return rc;
    const uint64_t size = 1ull << s->n;
    if (!host && count) return fail(RBK_ERR_INVALID, "null host pointer");
    if (offset > size || count > size - offset) return fail(RBK_ERR_INVALID, "range out of bounds");
    if (int rc = canonicalize(s)) return rc;
    device_guard g(s->device);
    const size_t ab = amp_bytes(s->precision);
    RBK_CUDA(cudaMemcpyAsync(host, static_cast<const char*>(s->amps) + offset * ab, count * ab, cudaMemcpyDeviceToHost, s->stream));
    return bounded_sync(s);
  });
}

int rbk_state_synchronize(rbk_state* s)
{
  return guarded([&]() -> int {
    if (int rc = check_state(s)) return rc;
    if (int rc = flush(s)) return rc;
    device_guard g(s->device);
    return bounded_sync(s);
  });
}

int rbk_flush(rbk_state* s)
{
  return guarded([&]() -> int {
    if (int rc = check_state(s)) return rc;
    return flush(s);
  });
}

int rbk_state_set_deferred(rbk_state* s, int deferred)
{
  if (int rc = check_state(s)) return rc;
  s->deferred = deferred != 0;
  if (!s->deferred && !s->in_fusion) return guarded([&] { return flush(s); });
  return RBK_OK;
}

int rbk_state_set_pass_budget(rbk_state* s, int max_dense)
{
  if (int rc = check_state(s)) return rc;
  if (max_dense < 0) return fail(RBK_ERR_INVALID, "negative budget");
  s->dense_budget = max_dense;
  return RBK_OK;
}

int rbk_state_set_tile_shape(rbk_state* s, int shape)
{
  if (int rc = check_state(s)) return rc;
  if (shape < 0 || shape >= rbk::kNumShapes) return fail(RBK_ERR_INVALID, "unknown tile shape");
  if (shape == 1) return fail(RBK_ERR_INVALID, "tile shape 1 is not built");
  if (int rc = guarded([&] { return canonicalize(s); })) return rc;
  s->shape = shape;
  return RBK_OK;
}

int rbk_state_get_stats(const rbk_state* s, rbk_stats* out)
{
  if (int rc = check_state(s)) return rc;
  if (!out) return fail(RBK_ERR_INVALID, "null output pointer");
  *out = s->stats;
  return RBK_OK;
}

int rbk_state_reset_stats(rbk_state* s)
{
  if (int rc = check_state(s)) return rc;
  s->stats = rbk_stats{};
  s->timing_started = false;
  return RBK_OK;
}

int rbk_state_device_ms(rbk_state* s, double* out)
{
  return guarded([&]() -> int {
    if (int rc = check_state(s)) return rc;
    if (!out) return fail(RBK_ERR_INVALID, "null output pointer");
    if (int rc = flush(s)) return rc;
    device_guard g(s->device);
    if (int rc = bounded_sync(s)) return rc;
    if (!s->timing_started) { *out = 0.0; return RBK_OK; }
    float ms = 0.f;
    RBK_CUDA(cudaEventElapsedTime(&ms, s->ev_first, s->ev_last));
    *out = ms;
    return RBK_OK;
  });
}

int rbk_state_get_permutation(rbk_state* s, uint32_t* perm)
{
  return guarded([&]() -> int {
    if (int rc = check_state(s)) return rc;
    if (!perm) return fail(RBK_ERR_INVALID, "null output pointer");
    if (int rc = flush(s)) return rc;
    for (int q = 0; q < s->n; ++q) perm[q] = static_cast<uint32_t>(s->perm[q]);
    return RBK_OK;
  });
}

int rbk_state_canonicalize(rbk_state* s)
{
  return guarded([&]() -> int {
    if (int rc = check_state(s)) return rc;
    return canonicalize(s);
  });
}

int rbk_state_set_permutation(rbk_state* s, const uint32_t* perm)
{
  return guarded([&]() -> int {
    if (int rc = check_state(s)) return rc;
    std::vector<int> map;
    if (int rc = read_layout(s, perm, map)) return rc;
    if (int rc = flush(s)) return rc;  // queued gates name logical qubits of the old map
    s->perm = map;
    for (int q = 0; q < s->n; ++q) s->inv[static_cast<size_t>(map[static_cast<size_t>(q)])] = q;
    return RBK_OK;
  });
}

int rbk_state_set_layout(rbk_state* s, const uint32_t* perm)
{
  return guarded([&]() -> int {
    if (int rc = check_state(s)) return rc;
    std::vector<int> map;
    if (int rc = read_layout(s, perm, map)) return rc;
    return move_layout(s, map);
  });
}

int rbk_state_device_pointer(rbk_state* s, void** out)
{
  return guarded([&]() -> int {
    if (int rc = check_state(s)) return rc;
    if (!out) return fail(RBK_ERR_INVALID, "null output pointer");
    if (int rc = flush(s)) return rc;
    *out = s->amps;
    return RBK_OK;
  });
}

namespace {
constexpr int RBK_NOT_FUSED = -1;
int fuse_block_to_unitary(rbk_state* s);
}  // namespace

int rbk_begin_fusion(rbk_state* s)
{
  if (int rc = check_state(s)) return rc;
  if (s->in_fusion) return fail(RBK_ERR_STATE, "BEGIN FUSION inside a fusion block");
  s->in_fusion = true;
  s->fusion_begin = s->queue.size();
  return RBK_OK;
}

int rbk_end_fusion(rbk_state* s)
{
  if (int rc = check_state(s)) return rc;
  if (!s->in_fusion) return fail(RBK_ERR_STATE, "END FUSION without BEGIN FUSION");
  s->in_fusion = false;
  if (s->fusion_mode == 1 && s->precision == RBK_C64) {
    const int rc = guarded([&] { return fuse_block_to_unitary(s); });
    if (rc != RBK_NOT_FUSED) return rc;
  }
  if (!s->deferred) return guarded([&] { return flush(s); });
  return RBK_OK;
}

// ---- gates ------------------------------------------------------------------

int rbk_hadamard(rbk_state* s, uint32_t target, const uint32_t* controls, int nc)
{
  return guarded([&]() -> int {
    double m[8];
    put(m, 0, {kOneDivRootTwo, 0.0}); put(m, 1, {kOneDivRootTwo, 0.0});
    put(m, 2, {kOneDivRootTwo, 0.0}); put(m, 3, {-kOneDivRootTwo, 0.0});
    return enqueue_target(s, rbk::OPK_MAT, target, controls, nc, m);
  });
}

int rbk_pauli_x(rbk_state* s, uint32_t target, const uint32_t* controls, int nc)
{
  return guarded([&] { return enqueue_target(s, rbk::OPK_X, target, controls, nc, nullptr); });
}

int rbk_pauli_y(rbk_state* s, uint32_t target, const uint32_t* controls, int nc)
{
  return guarded([&] { return enqueue_target(s, rbk::OPK_Y, target, controls, nc, nullptr); });
}

int rbk_pauli_z(rbk_state* s, const uint32_t* qubits, int nq)
{
  return guarded([&] { return enqueue_phase(s, cplx{-1.0, 0.0}, qubits, nq); });
}

int rbk_phase_shift_coeff(rbk_state* s, double re, double im, const uint32_t* qubits, int nq)
{
  return guarded([&] { return enqueue_phase(s, cplx{re, im}, qubits, nq); });
}

int rbk_phase_shift(rbk_state* s, double phase, const uint32_t* qubits, int nq)
{
  return guarded([&] { return enqueue_phase(s, exp_i(phase), qubits, nq); });
}

int rbk_controlled_phase_shift_k(rbk_state* s, int k, const uint32_t* qubits, int nq)
{
  return guarded([&]() -> int {
    if (int rc = check_state(s)) return rc;
    const int ak = k < 0 ? -k : k;
    if (ak > s->n) return fail(RBK_ERR_INVALID, "phase exponent larger than the number of qubits");
    // bra's table entry: exp_i(2 pi / 2^k) (generate_phase_coefficients.hpp:20-39)
    cplx c = exp_i(kTwoPi / static_cast<double>(1ull << ak));
    if (k < 0) c = std::conj(c);
    return enqueue_phase(s, c, qubits, nq);
  });
}

int rbk_phase_shift2(rbk_state* s, double phase1, double phase2, uint32_t target, const uint32_t* controls, int nc)
{
  return guarded([&]() -> int {
    // phase_shift.hpp:660-709: a0' = (a0 - c2 a1)/sqrt2, a1' = r c1 (c2 a1 + a0)
    const cplx c1 = exp_i(phase1), c2 = exp_i(phase2);
    const cplx mc1 = kOneDivRootTwo * c1;
    double m[8];
    put(m, 0, {kOneDivRootTwo, 0.0});
    put(m, 1, -(kOneDivRootTwo * c2));
    put(m, 2, mc1);
    put(m, 3, mc1 * c2);
    return enqueue_target(s, rbk::OPK_MAT, target, controls, nc, m);
  });
}

int rbk_phase_shift3(rbk_state* s, double phase1, double phase2, double phase3, uint32_t target,
                     const uint32_t* controls, int nc)
{
  return guarded([&]() -> int {
    // phase_shift.hpp:1200-1254: a0' = cos a0 - (sin c3) a1, a1' = ((cos c3) a1 + sin a0) c2
    const double sine = std::sin(0.5 * phase1), cosine = std::cos(0.5 * phase1);
    const cplx c2 = exp_i(phase2), c3 = exp_i(phase3);
    double m[8];
    put(m, 0, {cosine, 0.0});
    put(m, 1, -(sine * c3));
    put(m, 2, sine * c2);
    put(m, 3, (cosine * c3) * c2);
    return enqueue_target(s, rbk::OPK_MAT, target, controls, nc, m);
  });
}

int rbk_exponential_pauli_x(rbk_state* s, double phase, uint32_t target, const uint32_t* controls, int nc)
{
  return guarded([&]() -> int {
    // exp(i theta X) = cos I + i sin X
    const cplx c = exp_i(phase);
    double m[8];
    put(m, 0, {c.real(), 0.0}); put(m, 1, {0.0, c.imag()});
    put(m, 2, {0.0, c.imag()}); put(m, 3, {c.real(), 0.0});
    return enqueue_target(s, rbk::OPK_MAT, target, controls, nc, m);
  });
}

int rbk_exponential_pauli_y(rbk_state* s, double phase, uint32_t target, const uint32_t* controls, int nc)
{
  return guarded([&]() -> int {
    // exponential_pauli_y.hpp:40-85: a0' = cos a0 + sin a1, a1' = cos a1 - sin a0
    const cplx c = exp_i(phase);
    double m[8];
    put(m, 0, {c.real(), 0.0}); put(m, 1, {c.imag(), 0.0});
    put(m, 2, {-c.imag(), 0.0}); put(m, 3, {c.real(), 0.0});
    return enqueue_target(s, rbk::OPK_MAT, target, controls, nc, m);
  });
}

int rbk_exponential_pauli_z(rbk_state* s, double phase, uint32_t target, const uint32_t* controls, int nc)
{
  return guarded([&]() -> int {
    // exponential_pauli_z.hpp:40-78: a0 *= e^{i theta}, a1 *= e^{-i theta}
    const cplx c = exp_i(phase);
    double d[8] = {};
    put(d, 0, c);
    put(d, 1, std::conj(c));
    return enqueue_target(s, rbk::OPK_DIAG, target, controls, nc, d, 0);
  });
}

int rbk_swap(rbk_state* s, uint32_t q1, uint32_t q2, const uint32_t* controls, int nc)
{
  return guarded([&]() -> int {
    if (int rc = check_state(s)) return rc;
    uint64_t cm = 0;
    if (int rc = check_qubits(s, controls, nc, &cm)) return rc;
    if (q1 >= static_cast<uint32_t>(s->n) || q2 >= static_cast<uint32_t>(s->n))
      return fail(RBK_ERR_INVALID, "qubit index out of range");
    if (q1 == q2) return fail(RBK_ERR_INVALID, "repeated qubit");
    if (cm & ((1ull << q1) | (1ull << q2))) return fail(RBK_ERR_INVALID, "swap qubit is also a control qubit");
    if (nc == 0) {
      hgate g{};
      g.kind = rbk::HK_SWAP;
      g.target = static_cast<int8_t>(q1);
      g.target2 = static_cast<int8_t>(q2);
      return enqueue(s, g);
    }
    // Controlled swap = X(q1 <- q2) . C..C X(q2 <- q1) . X(q1 <- q2), all exact permutations.
    const uint32_t c2[1] = {q2};
    if (int rc = enqueue_target(s, rbk::OPK_X, q1, c2, 1, nullptr)) return rc;
    std::vector<uint32_t> cc(controls, controls + nc);
    cc.push_back(q1);
    if (int rc = enqueue_target(s, rbk::OPK_X, q2, cc.data(), static_cast<int>(cc.size()), nullptr)) return rc;
    return enqueue_target(s, rbk::OPK_X, q1, c2, 1, nullptr);
  });
}

int rbk_apply_matrix2(rbk_state* s, const double* m, uint32_t target, const uint32_t* controls, int nc)
{
  return guarded([&]() -> int {
    if (!m) return fail(RBK_ERR_INVALID, "null matrix");
    return enqueue_target(s, rbk::OPK_MAT, target, controls, nc, m);
  });
}

int rbk_apply_diagonal2(rbk_state* s, const double* d, uint32_t target, const uint32_t* controls, int nc)
{
  return guarded([&]() -> int {
    if (!d) return fail(RBK_ERR_INVALID, "null diagonal");
    double m[8] = {d[0], d[1], d[2], d[3], 0, 0, 0, 0};
    const uint8_t one = (d[0] == 1.0 && d[1] == 0.0) ? 1 : 0;
    return enqueue_target(s, rbk::OPK_DIAG, target, controls, nc, m, one);
  });
}

// ---- observables -------------------------------------------------------------

int rbk_norm2(rbk_state* s, double* out)
{
  return guarded([&]() -> int {
    if (int rc = check_state(s)) return rc;
    if (!out) return fail(RBK_ERR_INVALID, "null output pointer");
    rbk::pauli_terms t{};
    t.count = 1;
    t.w[0][0] = 1.0;
    double r[2];
    if (int rc = pauli_group(s, 0, t, r)) return rc;
    *out = r[0];
    return RBK_OK;
  });
}

int rbk_probabilities(rbk_state* s, double* host_out, uint64_t offset, uint64_t count)
{
  return guarded([&]() -> int {
    if (int rc = check_state(s)) return rc;
    const uint64_t size = 1ull << s->n;
    if (!host_out && count) return fail(RBK_ERR_INVALID, "null output pointer");
    if (offset > size || count > size - offset) return fail(RBK_ERR_INVALID, "range out of bounds");
    if (int rc = canonicalize(s)) return rc;
    device_guard g(s->device);
    const uint64_t chunk = std::min<uint64_t>(count, 1ull << 24);
    double* dbuf = nullptr;
    if (chunk) RBK_CUDA(cudaMalloc(reinterpret_cast<void**>(&dbuf), chunk * sizeof(double)));
    int rc = RBK_OK;
    for (uint64_t done = 0; done < count && rc == RBK_OK; done += chunk) {
      const uint64_t c = std::min(chunk, count - done);
      const cudaError_t e = s->precision == RBK_C128 ? rbk::launch_probs<double>(s->amps, offset + done, c, dbuf, s->stream)
                                                    : rbk::launch_probs<float>(s->amps, offset + done, c, dbuf, s->stream);
      if (e != cudaSuccess) { rc = cuda_fail(e, "probabilities"); break; }
      ++s->stats.kernel_launches;
      const cudaError_t e2 = cudaMemcpyAsync(host_out + done, dbuf, c * sizeof(double), cudaMemcpyDeviceToHost, s->stream);
      if (e2 != cudaSuccess) { rc = cuda_fail(e2, "probabilities copy"); break; }
      rc = bounded_sync(s);
    }
    if (dbuf) cudaFree(dbuf);
    return rc;
  });
}

int rbk_spin_expectation_values(rbk_state* s, double* out)
{
  return guarded([&]() -> int {
    if (int rc = check_state(s)) return rc;
    if (!out) return fail(RBK_ERR_INVALID, "null output pointer");
    if (int rc = flush(s)) return rc;  // the layout map is final only after the queued gates ran
    const bool c128 = s->precision == RBK_C128;
    const int n = s->n, RB = rbk::spin_register_bits(c128 ? 0 : 1), KT = 8 + RB;
    if (n < KT) {
      // Small states: one Z-sum pass and one pair-sum pass per qubit.
      int rc = launch_reduction(s, [&] {
        return c128 ? rbk::launch_zsum<double>(s->amps, n, s->d_partials, s->d_out, s->stream)
                    : rbk::launch_zsum<float>(s->amps, n, s->d_partials, s->d_out, s->stream);
      });
      if (rc) return rc;
      if ((rc = read_out(s, n + 1))) return rc;
      const double total = s->h_out[0];
      std::vector<double> ones(static_cast<size_t>(n));
      for (int p = 0; p < n; ++p) ones[static_cast<size_t>(p)] = s->h_out[1 + p];
      for (int q = 0; q < n; ++q) {
        const double one = ones[static_cast<size_t>(s->perm[q])];
        out[3 * q + 2] = 0.5 * ((total - one) - one);
        rbk::pauli_terms t{};
        t.count = 1;
        t.w[0][0] = 1.0;
        t.one_sided = 1;  // <S_x> + i <S_y> = sum over pairs with the qubit clear of conj(a0) a1
        double r[2];
        if ((rc = pauli_group(s, 1ull << s->perm[q], t, r))) return rc;
        out[3 * q + 0] = r[0];
        out[3 * q + 1] = r[1];
      }
      return RBK_OK;
    }
    // Tile layouts of KT bits whose flips cover every physical bit once: the
    // low KT bits, then the coalescing bits 0..LOW-1 with up to KT - LOW
    // further bits (filled up with other bits when fewer remain).  Each layout
    // is one read of the state (spins_kernel) for all its flips.
    const int LOW = c128 ? rbk::precision_traits<double>::LOW : rbk::precision_traits<float>::LOW;
    std::vector<rbk::spin_group> groups;
    std::vector<std::vector<int>> group_flips;  // physical bits flipped by each group, in flip order
    auto add_group = [&](const std::vector<int>& tile_bits, const std::vector<int>& flips_local) {
      rbk::spin_group g{};
      g.K = KT;
      uint64_t mask = 0;
      for (int b = 0; b < KT; ++b) { g.tile_phys[b] = static_cast<uint8_t>(tile_bits[b]); mask |= 1ull << tile_bits[b]; }
      g.nflips = static_cast<int>(flips_local.size());
      g.nphases = (g.nflips + RB - 1) / RB;
      std::vector<int> phys;
      for (int p = 0; p < g.nphases; ++p) {
        std::vector<int> regs;
        for (int k = 0; k < RB; ++k) {
          const int f = p * RB + k;
          if (f < g.nflips) regs.push_back(flips_local[static_cast<size_t>(f)]);
        }
        for (int b = 0; static_cast<int>(regs.size()) < RB; ++b)  // fillers: other tile bits
          if (std::find(regs.begin(), regs.end(), b) == regs.end()) regs.push_back(b);
        int nt = 0;
        for (int b = 0; b < KT; ++b)
          if (std::find(regs.begin(), regs.end(), b) == regs.end()) g.phase_thr[p][nt++] = static_cast<uint8_t>(b);
        for (int k = 0; k < RB; ++k) g.phase_reg[p][k] = static_cast<uint8_t>(regs[static_cast<size_t>(k)]);
      }
      for (int f : flips_local) phys.push_back(tile_bits[static_cast<size_t>(f)]);
      int runs = 0, src = 0;
      for (int q = 0; q < n;) {
        if ((mask >> q) & 1) { ++q; continue; }
        int len = 0;
        while (q + len < n && !((mask >> (q + len)) & 1)) ++len;
        g.run_src[runs] = static_cast<uint8_t>(src);
        g.run_len[runs] = static_cast<uint8_t>(len);
        g.run_dst[runs] = static_cast<uint8_t>(q);
        ++runs;
        src += len;
        q += len;
      }
      g.num_runs = runs;
      groups.push_back(g);
      group_flips.push_back(phys);
    };
    {
      std::vector<int> bits, flips;
      for (int b = 0; b < KT; ++b) { bits.push_back(b); flips.push_back(b); }
      add_group(bits, flips);
      for (int b = KT; b < n; b += KT - LOW) {
        std::vector<int> tile_bits, local;
        for (int l = 0; l < LOW; ++l) tile_bits.push_back(l);
        for (int c = b; c < std::min(n, b + KT - LOW); ++c) {
          local.push_back(static_cast<int>(tile_bits.size()));
          tile_bits.push_back(c);
        }
        for (int c = KT - 1; static_cast<int>(tile_bits.size()) < KT; --c) tile_bits.push_back(c);  // fillers
        std::vector<int> order(tile_bits);  // tile bits ascending keeps the 512-byte runs of the low bits
        std::sort(order.begin(), order.end());
        std::vector<int> flips;
        for (int f : local) flips.push_back(static_cast<int>(std::find(order.begin(), order.end(), tile_bits[static_cast<size_t>(f)]) - order.begin()));
        add_group(order, flips);
      }
    }
    std::vector<int> slot_of_bit(static_cast<size_t>(n), -1);  // d_out offset of a physical bit's (x, y, z)
    int width = 0;
    for (size_t gi = 0; gi < groups.size(); ++gi) {
      for (int f = 0; f < groups[gi].nflips; ++f) slot_of_bit[static_cast<size_t>(group_flips[gi][static_cast<size_t>(f)])] = width + 3 * f;
      width += 3 * groups[gi].nflips + 1;
    }
    if (width > 4 * (rbk::kMaxQubits + 8)) return fail(RBK_ERR_INVALID, "too many qubits for the spin layouts");
    for (int q = 0; q < n; ++q)
      if (slot_of_bit[static_cast<size_t>(q)] < 0) return fail(RBK_ERR_STATE, "spin layouts miss a qubit");
    int offset = 0;
    for (const auto& g : groups) {
      int rc = launch_reduction(s, [&] {
        return c128 ? rbk::launch_spins<double>(s->amps, n, g, s->d_partials, s->d_out + offset, s->stream)
                    : rbk::launch_spins<float>(s->amps, n, g, s->d_partials, s->d_out + offset, s->stream);
      });
      if (rc) return rc;
      offset += 3 * g.nflips + 1;
    }
    if (int rc = read_out(s, width)) return rc;
    const double total = s->h_out[3 * groups.front().nflips];  // sum |a|^2 of the first layout
    for (int q = 0; q < n; ++q) {
      const int k = slot_of_bit[static_cast<size_t>(s->perm[q])];
      const double one = s->h_out[k + 2];
      out[3 * q + 0] = s->h_out[k];      // <S_x> = Re sum conj(a0) a1
      out[3 * q + 1] = s->h_out[k + 1];  // <S_y> = Im sum conj(a0) a1
      out[3 * q + 2] = 0.5 * ((total - one) - one);
    }
    return RBK_OK;
  });
}

int rbk_expectation_pauli(rbk_state* s, int num_terms, const char* strings, const double* coeffs, double* out)
{
  return guarded([&]() -> int {
    if (int rc = check_state(s)) return rc;
    if (num_terms < 0 || (num_terms > 0 && (!strings || !coeffs)) || !out)
      return fail(RBK_ERR_INVALID, "bad Pauli term arguments");
    // The queued gates may move qubits (SWAPs, relabelling): map logical
    // qubits to physical bits only after they have run.
    if (int rc = flush(s)) return rc;
    std::vector<pauli_group_terms> groups;
    if (int rc = group_pauli_terms(s, num_terms, strings, coeffs, groups)) return rc;
    double acc_re = 0, acc_im = 0;
    for (const auto& g : groups) {
      double r[2];
      if (int rc = pauli_group(s, g.flip, g.terms, r)) return rc;
      acc_re += r[0];
      acc_im += r[1];
    }
    out[0] = acc_re;
    out[1] = acc_im;
    return RBK_OK;
  });
}

int rbk_inner_product(rbk_state* a, rbk_state* b, double* out)
{
  return guarded([&]() -> int {
    if (int rc = check_state(a)) return rc;
    if (int rc = check_state(b)) return rc;
    if (!out) return fail(RBK_ERR_INVALID, "null output pointer");
    if (a->n != b->n || a->precision != b->precision) return fail(RBK_ERR_INVALID, "states differ in size or precision");
    if (a->device != b->device) return fail(RBK_ERR_UNSUPPORTED, "states live on different devices");
    if (int rc = flush(a)) return rc;  // layouts are final only after the queued gates ran
    if (int rc = flush(b)) return rc;
    if (a->perm != b->perm) {
      if (int rc = canonicalize(a)) return rc;
      if (int rc = canonicalize(b)) return rc;
    }
    if (int rc = flush(b)) return rc;
    {
      device_guard g(b->device);
      if (int rc = bounded_sync(b)) return rc;
    }
    int rc = launch_reduction(a, [&] {
      return a->precision == RBK_C128 ? rbk::launch_inner<double>(a->amps, b->amps, a->n, a->d_partials, a->d_out, a->stream)
                                      : rbk::launch_inner<float>(a->amps, b->amps, a->n, a->d_partials, a->d_out, a->stream);
    });
    if (rc) return rc;
    if ((rc = read_out(a, 2))) return rc;
    out[0] = a->h_out[0];
    out[1] = a->h_out[1];
    return RBK_OK;
  });
}

int rbk_fidelity(rbk_state* a, rbk_state* b, double* out)
{
  if (!out) return fail(RBK_ERR_INVALID, "null output pointer");
  double ip[2];
  if (int rc = rbk_inner_product(a, b, ip)) return rc;
  *out = ip[0] * ip[0] + ip[1] * ip[1];
  return RBK_OK;
}

int rbk_inner_product_pauli(rbk_state* a, rbk_state* b, int num_terms, const char* strings, const double* coeffs, double* out)
{
  return guarded([&]() -> int {
    if (int rc = check_state(a)) return rc;
    if (int rc = check_state(b)) return rc;
    if (num_terms < 0 || (num_terms > 0 && (!strings || !coeffs)) || !out)
      return fail(RBK_ERR_INVALID, "bad Pauli term arguments");
    if (a->n != b->n || a->precision != b->precision) return fail(RBK_ERR_INVALID, "states differ in size or precision");
    if (a->device != b->device) return fail(RBK_ERR_UNSUPPORTED, "states live on different devices");
    if (int rc = flush(a)) return rc;
    if (int rc = flush(b)) return rc;
    if (a->perm != b->perm) {
      if (int rc = canonicalize(a)) return rc;
      if (int rc = canonicalize(b)) return rc;
    }
    if (int rc = flush(b)) return rc;
    {
      device_guard g(b->device);
      if (int rc = bounded_sync(b)) return rc;
    }
    std::vector<pauli_group_terms> groups;
    if (int rc = group_pauli_terms(a, num_terms, strings, coeffs, groups)) return rc;
    double acc_re = 0, acc_im = 0;
    for (const auto& g : groups) {
      int rc = launch_reduction(a, [&] {
        return a->precision == RBK_C128
          ? rbk::launch_pauli2<double>(a->amps, b->amps, a->n, g.flip, g.terms, a->d_partials, a->d_out, a->stream)
          : rbk::launch_pauli2<float>(a->amps, b->amps, a->n, g.flip, g.terms, a->d_partials, a->d_out, a->stream);
      });
      if (rc) return rc;
      if ((rc = read_out(a, 2))) return rc;
      acc_re += a->h_out[0];
      acc_im += a->h_out[1];
    }
    out[0] = acc_re;
    out[1] = acc_im;
    return RBK_OK;
  });
}

int rbk_fidelity_pauli(rbk_state* a, rbk_state* b, int num_terms, const char* strings, const double* coeffs, double* out)
{
  if (!out) return fail(RBK_ERR_INVALID, "null output pointer");
  double ip[2];
  if (int rc = rbk_inner_product_pauli(a, b, num_terms, strings, coeffs, ip)) return rc;
  *out = ip[0] * ip[0] + ip[1] * ip[1];
  return RBK_OK;
}

}  // extern "C"

// ---- adjoint gradient ---------------------------------------------------------
//
// No counterpart in the reference (which has no differentiation support).
// Forward: psi = U(theta)|0...0> through the fused passes.  Then lambda = H psi
// and E = <psi|lambda>.  Reverse: for g = last..first, a rotation
// exp(i phi P) with phi = scale * theta[k] + offset contributes
//   dE/dtheta_k += 2 Re(i scale <lambda|P|psi>) = -2 scale Im <lambda|P|psi>
// (psi, lambda taken after gate g), then U_g^dagger is applied to both states.
// The gate inverses are exact (rotation angle negated, U3(t,p,l)^dagger =
// U3(-t,-l,-p), self-inverse Paulis), so no intermediate state is stored.

namespace {

int apply_circuit_gate(rbk_state* s, const rbk_circuit_gate& g, const double* theta, bool inverse)
{
  const uint32_t q0 = static_cast<uint32_t>(g.qubits[0]), q1 = static_cast<uint32_t>(g.qubits[1]);
  const double sign = inverse ? -1.0 : 1.0;
  const double phase = (g.param >= 0 ? g.scale * theta[g.param] : 0.0) + g.angles[0];
  switch (g.kind) {
    case RBK_GATE_H: return rbk_hadamard(s, q0, nullptr, 0);
    case RBK_GATE_X: return rbk_pauli_x(s, q0, nullptr, 0);
    case RBK_GATE_Y: return rbk_pauli_y(s, q0, nullptr, 0);
    case RBK_GATE_Z: return rbk_pauli_z(s, &q0, 1);
    case RBK_GATE_U1: return rbk_phase_shift(s, sign * phase, &q0, 1);
    case RBK_GATE_U2:
      return inverse ? rbk_phase_shift3(s, -1.5707963267948966192, -g.angles[1], -g.angles[0], q0, nullptr, 0)
                     : rbk_phase_shift2(s, g.angles[0], g.angles[1], q0, nullptr, 0);
    case RBK_GATE_U3:
      return inverse ? rbk_phase_shift3(s, -g.angles[0], -g.angles[2], -g.angles[1], q0, nullptr, 0)
                     : rbk_phase_shift3(s, g.angles[0], g.angles[1], g.angles[2], q0, nullptr, 0);
    case RBK_GATE_CNOT: return rbk_pauli_x(s, q1, &q0, 1);
    case RBK_GATE_CZ: { const uint32_t qs[2] = {q0, q1}; return rbk_pauli_z(s, qs, 2); }
    case RBK_GATE_U: {
      const uint32_t qs[2] = {q0, q1};
      const int k = static_cast<int>(g.angles[0]);
      return rbk_controlled_phase_shift_k(s, inverse ? -k : k, qs, 2);
    }
    case RBK_GATE_EX: return rbk_exponential_pauli_x(s, sign * phase, q0, nullptr, 0);
    case RBK_GATE_EY: return rbk_exponential_pauli_y(s, sign * phase, q0, nullptr, 0);
    case RBK_GATE_EZ: return rbk_exponential_pauli_z(s, sign * phase, q0, nullptr, 0);
    case RBK_GATE_SWAP: return rbk_swap(s, q0, q1, nullptr, 0);
    default: return fail(RBK_ERR_INVALID, "unknown circuit gate kind");
  }
}

struct state_guard {
  rbk_state* s = nullptr;
  ~state_guard() { if (s) rbk_state_destroy(s); }
};

struct device_buffer {
  double* p = nullptr;
  ~device_buffer() { if (p) cudaFree(p); }
};

}  // namespace

// Tile bits of the tiled overlap launches (both states of a tile in shared memory).
constexpr int kOverlapTileBits128 = 11, kOverlapTileBits64 = 12;

// Overlaps of one group on the device, with as few reads of the states as
// possible.  One-qubit Paulis (the rotation runs' EX, EY, EZ): every Z type in
// one two-state Z-sum launch, X and Y types as pair sums, up to eight flip bits
// per launch (rbk::launch_zsum2, rbk::launch_pair_overlaps).  Anything else:
// one tiled launch covers every overlap whose flip bit is among the launch's
// tile bits (the low coalescing bits plus up to K - LOW chosen ones), Z-type
// overlaps (no flip) riding along in the first launch.
int launch_group_overlaps(const rbk::adjoint_workspace& w, rbk_state* lam, rbk_state* psi,
                          const std::vector<rbk::overlap_spec>& specs, int first_slot, double* ov, double* mpart,
                          double* tpart);

// Two states of one size on one stream plus the sweep's device buffers, kept
// between calls so that repeated gradients (batches, optimiser loops)
// allocate nothing.
struct rbk::adjoint_workspace {
  int n = 0, precision = RBK_C128, device = 0;
  rbk_state* psi = nullptr;
  rbk_state* lam = nullptr;
  double* ov = nullptr;  // (re, im) of <lambda|P|psi> per parametrised gate, then E
  int ov_cap = 0;
  double* mpart = nullptr;
  double* tpart = nullptr;  // tiled overlaps (n >= tile bits)
  double* ppart = nullptr;  // Z sums and pair sums (n >= 8 + kPairRegBits)
  ~adjoint_workspace()
  {
    if (ov) cudaFree(ov);
    if (mpart) cudaFree(mpart);
    if (tpart) cudaFree(tpart);
    if (ppart) cudaFree(ppart);
    if (lam) rbk_state_destroy(lam);
    if (psi) rbk_state_destroy(psi);
  }
};

constexpr int kPairTileBits = 8 + rbk::kPairRegBits;
constexpr int kPairLowBits = 3;  // tile bits always on the lowest physical bits: 128-byte runs

size_t zsum2_partials_doubles() { return size_t(1 << 17) / 256 * 2 * (rbk::kMaxQubits + 1); }

// The one-qubit-Pauli overlaps of `specs` (see launch_group_overlaps); marks
// those it schedules in `done`.
int launch_paired_overlaps(const rbk::adjoint_workspace& w, rbk_state* lam, rbk_state* psi,
                           const std::vector<rbk::overlap_spec>& specs, int first_slot, double* ov,
                           std::vector<char>& done)
{
  const bool c128 = w.precision == RBK_C128;
  const int n = w.n;
  cudaError_t e = cudaSuccess;
  std::vector<size_t> zs, xs;  // Z type; X / Y type
  for (size_t y = 0; y < specs.size(); ++y) {
    const auto& sp = specs[y];
    if (sp.flip == 0 && __builtin_popcountll(sp.sign) == 1) zs.push_back(y);
    else if (__builtin_popcountll(sp.flip) == 1 && (sp.sign == 0 || sp.sign == sp.flip)) xs.push_back(y);
  }
  for (size_t c0 = 0; c0 < zs.size(); c0 += rbk::kMaxOverlaps) {
    rbk::zsum2_set set{};
    set.count = static_cast<int>(std::min<size_t>(rbk::kMaxOverlaps, zs.size() - c0));
    for (int k = 0; k < set.count; ++k) {
      const auto& sp = specs[zs[c0 + k]];
      set.spec[k].bit = __builtin_ctzll(sp.sign);
      set.spec[k].out_slot = first_slot + static_cast<int>(zs[c0 + k]);
      set.spec[k].wr = sp.wr;
      set.spec[k].wi = sp.wi;
    }
    e = c128 ? rbk::launch_zsum2<double>(lam->amps, psi->amps, n, set, w.ppart, ov, psi->stream)
             : rbk::launch_zsum2<float>(lam->amps, psi->amps, n, set, w.ppart, ov, psi->stream);
    if (e != cudaSuccess) return cuda_fail(e, "Z-sum overlaps");
    for (int k = 0; k < set.count; ++k) done[zs[c0 + k]] = 1;
  }
  // Pair groups: the low kPairLowBits bits plus up to 8 more tile bits; the
  // flips of a group are up to kMaxPairFlips of the remaining X / Y types.
  constexpr int RB = rbk::kPairRegBits, KT = kPairTileBits;
  size_t next = 0;
  while (next < xs.size()) {
    std::vector<int> tile_bits;
    for (int b = 0; b < kPairLowBits; ++b) tile_bits.push_back(b);
    std::vector<size_t> mine;
    uint64_t flips = 0;
    while (next < xs.size() && static_cast<int>(mine.size()) < rbk::kMaxPairFlips) {
      const int b = __builtin_ctzll(specs[xs[next]].flip);
      const bool in = std::find(tile_bits.begin(), tile_bits.end(), b) != tile_bits.end();
      if ((flips >> b) & 1) break;  // one register bit per flip in a group
      if (!in && static_cast<int>(tile_bits.size()) >= KT) break;
      flips |= 1ull << b;
      if (!in) tile_bits.push_back(b);
      mine.push_back(xs[next++]);
    }
    for (int b = 0; static_cast<int>(tile_bits.size()) < KT; ++b)  // fillers
      if (std::find(tile_bits.begin(), tile_bits.end(), b) == tile_bits.end()) tile_bits.push_back(b);
    std::sort(tile_bits.begin(), tile_bits.end());
    rbk::pair_overlap_set set{};
    rbk::spin_group& g = set.g;
    g.K = KT;
    uint64_t mask = 0;
    for (int b = 0; b < KT; ++b) { g.tile_phys[b] = static_cast<uint8_t>(tile_bits[static_cast<size_t>(b)]); mask |= 1ull << tile_bits[static_cast<size_t>(b)]; }
    std::vector<int> local;
    for (size_t y : mine) {
      const int b = __builtin_ctzll(specs[y].flip);
      local.push_back(static_cast<int>(std::find(tile_bits.begin(), tile_bits.end(), b) - tile_bits.begin()));
    }
    g.nflips = static_cast<int>(mine.size());
    g.nphases = (g.nflips + RB - 1) / RB;
    for (int p = 0; p < g.nphases; ++p) {
      std::vector<int> regs;
      for (int k = 0; k < RB; ++k) {
        const int f = p * RB + k;
        if (f < g.nflips) regs.push_back(local[static_cast<size_t>(f)]);
      }
      for (int b = 0; static_cast<int>(regs.size()) < RB; ++b)  // fillers: other tile bits
        if (std::find(regs.begin(), regs.end(), b) == regs.end()) regs.push_back(b);
      int nt = 0;
      for (int b = 0; b < KT; ++b)
        if (std::find(regs.begin(), regs.end(), b) == regs.end()) g.phase_thr[p][nt++] = static_cast<uint8_t>(b);
      for (int k = 0; k < RB; ++k) g.phase_reg[p][k] = static_cast<uint8_t>(regs[static_cast<size_t>(k)]);
    }
    int runs = 0, src = 0;
    for (int q = 0; q < n;) {
      if ((mask >> q) & 1) { ++q; continue; }
      int len = 0;
      while (q + len < n && !((mask >> (q + len)) & 1)) ++len;
      g.run_src[runs] = static_cast<uint8_t>(src);
      g.run_len[runs] = static_cast<uint8_t>(len);
      g.run_dst[runs] = static_cast<uint8_t>(q);
      ++runs;
      src += len;
      q += len;
    }
    g.num_runs = runs;
    for (size_t f = 0; f < mine.size(); ++f) {
      const auto& sp = specs[mine[f]];
      set.flip[f].out_slot = first_slot + static_cast<int>(mine[f]);
      set.flip[f].minus = sp.sign != 0 ? 1 : 0;
      set.flip[f].wr = sp.wr;
      set.flip[f].wi = sp.wi;
    }
    e = c128 ? rbk::launch_pair_overlaps<double>(lam->amps, psi->amps, n, set, w.ppart, ov, psi->stream)
             : rbk::launch_pair_overlaps<float>(lam->amps, psi->amps, n, set, w.ppart, ov, psi->stream);
    if (e != cudaSuccess) return cuda_fail(e, "pair overlaps");
    for (size_t y : mine) done[y] = 1;
  }
  return RBK_OK;
}

// The queued records of s as the diagonal both states owe (rbk::pre_diag in
// physical bits: g, u, adj, full).  false when one of them is not a one-bit
// diagonal or a controlled Z (a multi-controlled phase, for instance).
bool owed_from_queue(const rbk_state* s, rbk::pre_diag& o)
{
  using cplx_t = std::complex<double>;
  cplx_t g{1.0, 0.0};
  std::vector<cplx_t> u(rbk::kMaxQubits, cplx_t{1.0, 0.0});
  for (const hgate& h : s->queue) {
    if (h.kind == rbk::OPK_NEG) {
      const int c = __builtin_popcountll(h.cmask);
      if (c == 1) {
        u[static_cast<size_t>(s->perm[__builtin_ctzll(h.cmask)])] *= -1.0;
      } else if (c == 2) {
        const int a = s->perm[__builtin_ctzll(h.cmask)], b = s->perm[63 - __builtin_clzll(h.cmask)];
        o.adj[std::min(a, b)] ^= 1ull << std::max(a, b);
        o.full[a] ^= 1ull << b;
        o.full[b] ^= 1ull << a;
      } else {
        return false;
      }
    } else if (h.kind == rbk::OPK_DIAG && h.cmask == 0) {
      const size_t t = static_cast<size_t>(s->perm[h.target]);
      const cplx_t d0{h.m[0], h.m[1]}, d1{h.m[2], h.m[3]};
      if (h.diag_one) {
        u[t] *= d1;
      } else {
        g *= d0;
        u[t] *= d1 / d0;
      }
    } else {
      return false;
    }
  }
  o.g[0] = g.real();
  o.g[1] = g.imag();
  for (int b = 0; b < rbk::kMaxQubits; ++b) {
    o.u[b][0] = u[static_cast<size_t>(b)].real();
    o.u[b][1] = u[static_cast<size_t>(b)].imag();
  }
  return true;
}

// Pair-rotate launches over `items` (rbk::plan_rotations), the owed diagonal,
// if any, in the first.
int launch_rotations(const rbk::adjoint_workspace& w, rbk_state* lam, rbk_state* psi,
                     const std::vector<rbk::rotate_item>& items, double* ov, const rbk::pre_diag* owed)
{
  const bool c128 = w.precision == RBK_C128;
  for (const rbk::pair_rotate_set& set : rbk::plan_rotations(w.n, items, owed)) {
    const cudaError_t e = c128 ? rbk::launch_pair_rotate<double>(lam->amps, psi->amps, w.n, set, w.ppart, ov, psi->stream)
                               : rbk::launch_pair_rotate<float>(lam->amps, psi->amps, w.n, set, w.ppart, ov, psi->stream);
    if (e != cudaSuccess) return cuda_fail(e, "pair rotations");
  }
  return RBK_OK;
}

bool queue_is_diagonal(const rbk_state* s)
{
  for (const hgate& h : s->queue)
    if (h.kind != rbk::OPK_DIAG && h.kind != rbk::OPK_NEG) return false;
  return true;
}

// The engine's record of U_g^dagger for a one-qubit circuit gate: what
// apply_circuit_gate(s, g, theta, true) queues, taken back off s's queue.
int inverse_record(rbk_state* s, const rbk_circuit_gate& g, const double* theta, hgate* out)
{
  const size_t mark = s->queue.size();
  const auto issued = s->stats.gates_issued;
  if (int rc = apply_circuit_gate(s, g, theta, true)) return rc;
  if (s->queue.size() != mark + 1) return fail(RBK_ERR_STATE, "adjoint sweep: a one-qubit gate queued other than one record");
  *out = s->queue.back();
  s->queue.pop_back();
  s->stats.gates_issued = issued;
  return RBK_OK;
}

int launch_group_overlaps(const rbk::adjoint_workspace& w, rbk_state* lam, rbk_state* psi,
                          const std::vector<rbk::overlap_spec>& specs, int first_slot, double* ov, double* mpart,
                          double* tpart)
{
  const bool c128 = w.precision == RBK_C128;
  const int n = w.n;
  const int K = c128 ? kOverlapTileBits128 : kOverlapTileBits64;
  const int LOW = c128 ? rbk::precision_traits<double>::LOW : rbk::precision_traits<float>::LOW;
  cudaError_t e = cudaSuccess;
  std::vector<char> done(specs.size(), 0);
  if (n >= kPairTileBits && w.ppart) {
    if (int rc = launch_paired_overlaps(w, lam, psi, specs, first_slot, ov, done)) return rc;
    bool all = true;
    for (char d : done) all = all && d;
    if (all) return RBK_OK;
  }
  if (n < K || !tpart) {
    for (size_t c0 = 0; c0 < specs.size(); c0 += rbk::kMaxOverlaps) {
      rbk::overlap_set set{};
      set.count = static_cast<int>(std::min<size_t>(rbk::kMaxOverlaps, specs.size() - c0));
      for (int y = 0; y < set.count; ++y) set.spec[y] = specs[c0 + y];
      double* out = ov + 2 * (first_slot + c0);
      e = c128 ? rbk::launch_overlaps<double>(lam->amps, psi->amps, n, set, mpart, out, psi->stream)
               : rbk::launch_overlaps<float>(lam->amps, psi->amps, n, set, mpart, out, psi->stream);
      if (e != cudaSuccess) return cuda_fail(e, "overlaps");
    }
    return RBK_OK;
  }
  std::vector<int> high;
  for (size_t y = 0; y < specs.size(); ++y) {
    const auto& sp = specs[y];
    if (sp.flip && !done[y]) {
      const int b = __builtin_ctzll(sp.flip);
      if (b >= LOW && std::find(high.begin(), high.end(), b) == high.end()) high.push_back(b);
    }
  }
  std::sort(high.begin(), high.end());
  const int per = K - LOW;
  const int chunks = std::max<int>(1, static_cast<int>((high.size() + per - 1) / per));
  for (int c = 0; c < chunks; ++c) {
    uint64_t tmask = (1ull << LOW) - 1;
    int tile_phys[16];
    int k = 0;
    for (int b = 0; b < LOW; ++b) tile_phys[k++] = b;
    for (size_t h = static_cast<size_t>(c) * per; h < high.size() && h < static_cast<size_t>(c + 1) * per; ++h) {
      tile_phys[k++] = high[h];
      tmask |= 1ull << high[h];
    }
    for (int b = LOW; b < n && k < K; ++b)
      if (!(tmask & (1ull << b))) { tile_phys[k++] = b; tmask |= 1ull << b; }
    rbk::tile_overlap_set base{};
    base.K = K;
    for (int b = 0; b < K; ++b) base.tile_phys[b] = static_cast<uint8_t>(tile_phys[b]);
    int src = 0;
    for (int b = 0; b < n;) {
      if (tmask & (1ull << b)) { ++b; continue; }
      int len = 0;
      while (b + len < n && !(tmask & (1ull << (b + len)))) ++len;
      base.run_src[base.num_runs] = static_cast<uint8_t>(src);
      base.run_len[base.num_runs] = static_cast<uint8_t>(len);
      base.run_dst[base.num_runs] = static_cast<uint8_t>(b);
      ++base.num_runs;
      src += len;
      b += len;
    }
    auto local = [&](uint64_t mask) {
      uint32_t m = 0;
      for (int t = 0; t < K; ++t)
        if (mask & (1ull << tile_phys[t])) m |= 1u << t;
      return m;
    };
    std::vector<size_t> mine;
    for (size_t y = 0; y < specs.size(); ++y) {
      if (done[y]) continue;
      const uint64_t f = specs[y].flip;
      if ((f == 0 && c == 0) || (f != 0 && (f & tmask) == f)) { mine.push_back(y); done[y] = 1; }
    }
    for (size_t c0 = 0; c0 < mine.size(); c0 += rbk::kMaxOverlaps) {
      rbk::tile_overlap_set set = base;
      set.count = static_cast<int>(std::min<size_t>(rbk::kMaxOverlaps, mine.size() - c0));
      for (int y = 0; y < set.count; ++y) {
        const auto& sp = specs[mine[c0 + y]];
        auto& t = set.spec[y];
        t.flip_local = local(sp.flip);
        t.sign_local = local(sp.sign);
        t.sign = sp.sign & ~tmask;
        t.wr = sp.wr;
        t.wi = sp.wi;
        t.out_slot = first_slot + static_cast<int>(mine[c0 + y]);
      }
      e = c128 ? rbk::launch_tile_overlaps<double>(lam->amps, psi->amps, n, set, tpart, ov, psi->stream)
               : rbk::launch_tile_overlaps<float>(lam->amps, psi->amps, n, set, tpart, ov, psi->stream);
      if (e != cudaSuccess) return cuda_fail(e, "tiled overlaps");
    }
  }
  for (size_t y = 0; y < specs.size(); ++y)
    if (!done[y]) return fail(RBK_ERR_STATE, "adjoint sweep: an overlap was not scheduled");
  return RBK_OK;
}

int rbk::adjoint_workspace_create(int num_qubits, int precision, int device, adjoint_workspace** out)
{
  return guarded([&]() -> int {
    if (!out) return fail(RBK_ERR_INVALID, "null output pointer");
    *out = nullptr;
    auto w = std::make_unique<adjoint_workspace>();
    w->n = num_qubits;
    w->precision = precision;
    w->device = device;
    if (int rc = rbk_state_create(num_qubits, precision, 0, device, &w->psi)) return rc;
    if (int rc = rbk_state_create(num_qubits, precision, 0, device, &w->lam)) return rc;
    device_guard dg(device);
    // One stream for both states: every kernel of the sweep is ordered without host waits.
    cudaStreamSynchronize(w->lam->stream);
    cudaStreamDestroy(w->lam->stream);
    w->lam->stream = w->psi->stream;
    w->lam->owns_stream = false;
    RBK_CUDA(cudaMalloc(reinterpret_cast<void**>(&w->mpart), sizeof(double) * rbk::overlaps_partials_doubles()));
    const int K = precision == RBK_C128 ? kOverlapTileBits128 : kOverlapTileBits64;
    if (num_qubits >= K)
      RBK_CUDA(cudaMalloc(reinterpret_cast<void**>(&w->tpart), sizeof(double) * rbk::tile_overlaps_partials_doubles(num_qubits, K)));
    if (num_qubits >= kPairTileBits)
      RBK_CUDA(cudaMalloc(reinterpret_cast<void**>(&w->ppart),
                          sizeof(double) * std::max({rbk::pair_overlaps_partials_doubles(), rbk::pair_rotate_partials_doubles(),
                                                     zsum2_partials_doubles()})));
    *out = w.release();
    return RBK_OK;
  });
}

int rbk::adjoint_workspace_set_shape(adjoint_workspace* w, int shape)
{
  if (!w) return fail(RBK_ERR_INVALID, "null workspace");
  device_guard dg(w->device);
  if (int rc = rbk_state_set_tile_shape(w->psi, shape)) return rc;
  return rbk_state_set_tile_shape(w->lam, shape);
}

void rbk::adjoint_workspace_destroy(adjoint_workspace* w)
{
  if (!w) return;
  device_guard dg(w->device);
  delete w;
}

int rbk::adjoint_run(adjoint_workspace* w, const rbk_circuit_gate* gates, int num_gates, const double* theta,
                     int num_params, int num_terms, const char* strings, const double* coeffs, double* energy,
                     double* grad)
{
  return guarded([&]() -> int {
    if (!w) return fail(RBK_ERR_INVALID, "null workspace");
    const int num_qubits = w->n, precision = w->precision;
    if (num_gates < 0 || (num_gates > 0 && !gates) || num_params < 0 || (num_params > 0 && (!theta || !grad)) ||
        num_terms < 1 || !strings || !coeffs || !energy)
      return fail(RBK_ERR_INVALID, "bad adjoint-gradient arguments");
    for (int i = 0; i < num_gates; ++i) {
      const auto& g = gates[i];
      if (g.param >= num_params) return fail(RBK_ERR_INVALID, "gate parameter index out of range");
      if (g.param >= 0 && g.kind != RBK_GATE_EX && g.kind != RBK_GATE_EY && g.kind != RBK_GATE_EZ)
        return fail(RBK_ERR_UNSUPPORTED, "only EX, EY and EZ gates take parameters");
    }
    // Observable as grouped Pauli sums (logical bits: both states are kept canonical).
    rbk::pauli_sum H{};
    {
      struct term { uint64_t flip, sign; cplx w; };
      std::vector<term> terms;
      static const cplx pow_mi[4] = {{1, 0}, {0, -1}, {-1, 0}, {0, 1}};
      for (int t = 0; t < num_terms; ++t) {
        uint64_t x = 0, y = 0, z = 0;
        for (int k = 0; k < num_qubits; ++k) {
          const char c = strings[static_cast<size_t>(t) * num_qubits + k];
          if (c == 'X') x |= 1ull << k;
          else if (c == 'Y') y |= 1ull << k;
          else if (c == 'Z') z |= 1ull << k;
          else if (c != 'I') return fail(RBK_ERR_INVALID, "Pauli strings use the characters I, X, Y, Z");
        }
        terms.push_back({x | y, y | z, cplx{coeffs[2 * t], coeffs[2 * t + 1]} * pow_mi[__builtin_popcountll(y) & 3]});
      }
      std::vector<char> done(terms.size(), 0);
      int nt = 0;
      for (size_t i = 0; i < terms.size(); ++i) {
        if (done[i]) continue;
        if (H.num_groups >= rbk::kMaxSumGroups) return fail(RBK_ERR_INVALID, "more than 64 distinct X/Y patterns in the observable");
        H.flip[H.num_groups] = terms[i].flip;
        H.begin[H.num_groups] = nt;
        for (size_t j = i; j < terms.size(); ++j) {
          if (done[j] || terms[j].flip != terms[i].flip) continue;
          if (nt >= rbk::kMaxSumTerms) return fail(RBK_ERR_INVALID, "more than 128 Pauli strings in the observable");
          H.sign[nt] = terms[j].sign;
          H.w[nt][0] = terms[j].w.real();
          H.w[nt][1] = terms[j].w.imag();
          ++nt;
          done[j] = 1;
        }
        ++H.num_groups;
      }
      H.begin[H.num_groups] = nt;
    }

    struct { rbk_state* s; } psi{w->psi}, lam{w->lam};
    device_guard dg(w->device);
    if (int rc = rbk_state_reset(psi.s, 0)) return rc;
    if (int rc = rbk_state_reset(lam.s, 0)) return rc;

    int num_pg = 0;
    for (int i = 0; i < num_gates; ++i) num_pg += gates[i].param >= 0 ? 1 : 0;
    if (w->ov_cap < num_pg + 1) {
      if (w->ov) cudaFree(w->ov);
      w->ov = nullptr;
      w->ov_cap = 0;
      RBK_CUDA(cudaMalloc(reinterpret_cast<void**>(&w->ov), sizeof(double) * 2 * (num_pg + 1)));
      w->ov_cap = num_pg + 1;
    }
    struct { double* p; } ov{w->ov};

    for (int i = 0; i < num_gates; ++i)
      if (int rc = apply_circuit_gate(psi.s, gates[i], theta, false)) return rc;
    if (int rc = canonicalize(psi.s)) return rc;
    const bool c128 = precision == RBK_C128;
    cudaError_t e = c128 ? rbk::launch_pauli_apply_tiled<double>(psi.s->amps, lam.s->amps, num_qubits, H, psi.s->stream)
                         : rbk::launch_pauli_apply_tiled<float>(psi.s->amps, lam.s->amps, num_qubits, H, psi.s->stream);
    if (e != cudaSuccess) return cuda_fail(e, "H psi");
    // E = <psi|lambda>
    e = c128 ? rbk::launch_inner<double>(lam.s->amps, psi.s->amps, num_qubits, psi.s->d_partials, ov.p + 2 * num_pg, psi.s->stream)
             : rbk::launch_inner<float>(lam.s->amps, psi.s->amps, num_qubits, psi.s->d_partials, ov.p + 2 * num_pg, psi.s->stream);
    if (e != cudaSuccess) return cuda_fail(e, "energy");

    std::vector<int> slot_param(num_pg);
    std::vector<double> slot_scale(num_pg);
    int slot = num_pg;
    struct { double* p; } mpart{w->mpart};  // partial sums of the grouped overlaps
    auto single_qubit = [](const rbk_circuit_gate& g) {
      return g.kind == RBK_GATE_H || g.kind == RBK_GATE_X || g.kind == RBK_GATE_Y || g.kind == RBK_GATE_Z ||
             g.kind == RBK_GATE_U1 || g.kind == RBK_GATE_U2 || g.kind == RBK_GATE_U3 || g.kind == RBK_GATE_EX ||
             g.kind == RBK_GATE_EY || g.kind == RBK_GATE_EZ;
    };
    // Runs of one-qubit gates take the pair-rotate path where its tile fits
    // (RBK_ADJOINT_PAIR_ROTATE=0 selects the overlap-then-queue path instead).
    // RBK_ADJOINT_PAIR_ROTATE=1 keeps the pair-rotate launches but flushes the
    // owed diagonals and reads the Z-type overlaps separately.
    const char* pr_env = std::getenv("RBK_ADJOINT_PAIR_ROTATE");
    const bool fused_runs = num_qubits >= kPairTileBits && w->ppart && !(pr_env && pr_env[0] == '0');
    const bool fused_pre = fused_runs && !(pr_env && pr_env[0] == '1');
    // Z-type overlaps not taken yet: (physical bit, slot).  Valid while both
    // states owe only diagonal records, which leave conj(lam_j) psi_j unchanged;
    // settled (one Z-sum read) before any flush.
    std::vector<std::pair<int, int>> zpend;
    auto settle_z = [&]() -> int {
      for (size_t c0 = 0; c0 < zpend.size(); c0 += rbk::kMaxOverlaps) {
        rbk::zsum2_set set{};
        set.count = static_cast<int>(std::min<size_t>(rbk::kMaxOverlaps, zpend.size() - c0));
        for (int k = 0; k < set.count; ++k) {
          set.spec[k].bit = zpend[c0 + k].first;
          set.spec[k].out_slot = zpend[c0 + k].second;
          set.spec[k].wr = 1.0;
          set.spec[k].wi = 0.0;
        }
        const cudaError_t e = precision == RBK_C128
          ? rbk::launch_zsum2<double>(lam.s->amps, psi.s->amps, num_qubits, set, w->ppart, ov.p, psi.s->stream)
          : rbk::launch_zsum2<float>(lam.s->amps, psi.s->amps, num_qubits, set, w->ppart, ov.p, psi.s->stream);
        if (e != cudaSuccess) return cuda_fail(e, "Z-sum overlaps");
      }
      zpend.clear();
      return RBK_OK;
    };
    int i = num_gates - 1;
    while (i >= 0) {
      // A run of single-qubit gates on distinct qubits commutes gate by gate, so
      // every rotation in it sees the same (psi, lambda) pair -- the one after the
      // run -- and all its overlaps come from one launch: for rotation k,
      // <lambda_k|P_k|psi_k> = <lambda|G P_k G^dagger|psi> with G the later gates
      // of the run, which act on other qubits.
      int j = i;
      uint64_t used = 0;
      while (j >= 0 && single_qubit(gates[j]) && !(used & (1ull << gates[j].qubits[0]))) {
        used |= 1ull << gates[j].qubits[0];
        --j;
      }
      const bool run1q = single_qubit(gates[i]);
      if (j == i) j = i - 1;  // a gate on two qubits: no rotation, un-applied below
      std::vector<rbk::overlap_spec> specs;
      int first = slot;
      for (int k = i; k > j; --k)
        if (gates[k].param >= 0) --first;
      if (run1q && fused_runs) {
        // The run in as few reads of both states as possible: Z-type overlaps from
        // one two-state Z sum (no flush needed while only diagonal gates are queued:
        // those commute with Z), the run's diagonal gates queued on both states,
        // and every other gate of the run applied by pair-rotate launches that also
        // take the X / Y-type overlaps.
        std::vector<hgate> recs;
        for (int k = i; k > j; --k) {
          hgate h{};
          if (int rc = inverse_record(psi.s, gates[k], theta, &h)) return rc;
          recs.push_back(h);
        }
        auto is_diag = [](const hgate& h) { return h.kind == rbk::OPK_DIAG || h.kind == rbk::OPK_NEG; };
        std::vector<size_t> zidx;
        specs.assign(static_cast<size_t>(slot - first), rbk::overlap_spec{0, 0, 1.0, 0.0});
        std::vector<int> slot_of(static_cast<size_t>(i - j), -1);
        {
          int y = slot - first;
          for (int k = i; k > j; --k) {
            const auto& g = gates[k];
            if (g.param < 0) continue;
            --y;
            slot_param[first + y] = g.param;
            slot_scale[first + y] = g.scale;
            slot_of[static_cast<size_t>(i - k)] = first + y;
            if (g.kind == RBK_GATE_EZ) zidx.push_back(static_cast<size_t>(y));
            else if (is_diag(recs[static_cast<size_t>(i - k)])) return fail(RBK_ERR_STATE, "adjoint sweep: diagonal rotation of X / Y type");
          }
        }
        if (!zidx.empty()) {
          if (!queue_is_diagonal(psi.s) || !queue_is_diagonal(lam.s)) {
            if (int rc = settle_z()) return rc;
            if (int rc = flush(psi.s)) return rc;
            if (int rc = flush(lam.s)) return rc;
          }
          if (psi.s->perm != lam.s->perm) return fail(RBK_ERR_STATE, "adjoint sweep: layouts diverged");
          if (zpend.size() + zidx.size() > static_cast<size_t>(rbk::kMaxQubits))
            if (int rc = settle_z()) return rc;
          for (int k = i; k > j; --k) {
            const int sl = slot_of[static_cast<size_t>(i - k)];
            if (sl >= 0 && gates[k].kind == RBK_GATE_EZ) zpend.emplace_back(psi.s->perm[gates[k].qubits[0]], sl);
          }
          if (!fused_pre)
            if (int rc = settle_z()) return rc;
        }
        bool any_rotation = false;
        for (int k = i; k > j; --k) {
          const hgate& h = recs[static_cast<size_t>(i - k)];
          if (is_diag(h)) {
            if (int rc = enqueue(psi.s, h)) return rc;
            if (int rc = enqueue(lam.s, h)) return rc;
          } else {
            any_rotation = true;
          }
        }
        if (any_rotation) {
          // What both states owe, applied and summed in the first launch when it
          // is a product of one-bit diagonals and controlled Zs; else flushed.
          rbk::pre_diag owed{};
          bool use_owed = fused_pre && (!zpend.empty() || !psi.s->queue.empty()) &&
                          psi.s->queue.size() == lam.s->queue.size() && owed_from_queue(psi.s, owed);
          if (use_owed) {
            owed.nz = static_cast<int>(zpend.size());
            for (size_t k = 0; k < zpend.size(); ++k) {
              owed.z[k].bit = zpend[k].first;
              owed.z[k].out_slot = zpend[k].second;
              owed.z[k].wr = 1.0;
            }
            zpend.clear();
            psi.s->queue.clear();
            lam.s->queue.clear();
          } else {
            if (int rc = settle_z()) return rc;
            if (int rc = flush(psi.s)) return rc;
            if (int rc = flush(lam.s)) return rc;
          }
          if (psi.s->perm != lam.s->perm) return fail(RBK_ERR_STATE, "adjoint sweep: layouts diverged");
          std::vector<rbk::rotate_item> items;
          for (int k = i; k > j; --k) {
            const hgate& h = recs[static_cast<size_t>(i - k)];
            if (is_diag(h)) continue;
            if (h.cmask != 0) return fail(RBK_ERR_STATE, "adjoint sweep: controlled gate in a one-qubit run");
            rbk::rotate_item it{};
            it.bit = psi.s->perm[gates[k].qubits[0]];
            it.slot = slot_of[static_cast<size_t>(i - k)];
            it.spec = rbk::overlap_spec{0, 0, 1.0, 0.0};
            if (it.slot >= 0) {
              const uint64_t t = 1ull << it.bit;
              it.spec.flip = t;
              if (gates[k].kind == RBK_GATE_EY) { it.spec.sign = t; it.spec.wr = 0.0; it.spec.wi = -1.0; }
            }
            if (h.kind == rbk::OPK_MAT) {
              std::memcpy(it.m, h.m, sizeof(it.m));
            } else if (h.kind == rbk::OPK_X) {
              const double m[8] = {0, 0, 1, 0, 1, 0, 0, 0};
              std::memcpy(it.m, m, sizeof(it.m));
            } else if (h.kind == rbk::OPK_Y) {  // (a0, a1) -> (-i a1, i a0)
              const double m[8] = {0, 0, 0, -1, 0, 1, 0, 0};
              std::memcpy(it.m, m, sizeof(it.m));
            } else {
              return fail(RBK_ERR_STATE, "adjoint sweep: unexpected gate record");
            }
            items.push_back(it);
          }
          if (int rc = launch_rotations(*w, lam.s, psi.s, items, ov.p, use_owed ? &owed : nullptr)) return rc;
        }
        slot = first;
        i = j;
        continue;
      }
      if (first < slot) {
        if (int rc = settle_z()) return rc;
        if (int rc = flush(psi.s)) return rc;
        if (int rc = flush(lam.s)) return rc;
        if (psi.s->perm != lam.s->perm) return fail(RBK_ERR_STATE, "adjoint sweep: layouts diverged");
        specs.resize(static_cast<size_t>(slot - first));
        int y = slot - first;
        for (int k = i; k > j; --k) {
          const auto& g = gates[k];
          if (g.param < 0) continue;
          --y;
          slot_param[first + y] = g.param;
          slot_scale[first + y] = g.scale;
          const uint64_t t = 1ull << psi.s->perm[g.qubits[0]];
          rbk::overlap_spec& sp = specs[static_cast<size_t>(y)];
          sp = rbk::overlap_spec{0, 0, 1.0, 0.0};
          if (g.kind == RBK_GATE_EX) sp.flip = t;
          else if (g.kind == RBK_GATE_EY) { sp.flip = t; sp.sign = t; sp.wr = 0.0; sp.wi = -1.0; }
          else sp.sign = t;  // EZ
        }
        if (int rc = launch_group_overlaps(*w, lam.s, psi.s, specs, first, ov.p, mpart.p, w->tpart)) return rc;
        slot = first;
      }
      for (int k = i; k > j; --k) {
        if (int rc = apply_circuit_gate(psi.s, gates[k], theta, true)) return rc;
        if (int rc = apply_circuit_gate(lam.s, gates[k], theta, true)) return rc;
      }
      i = j;
    }
    if (int rc = settle_z()) return rc;
    std::vector<double> host(2 * (num_pg + 1));
    RBK_CUDA(cudaMemcpyAsync(host.data(), ov.p, sizeof(double) * host.size(), cudaMemcpyDeviceToHost, psi.s->stream));
    if (int rc = bounded_sync(psi.s)) return rc;
    *energy = host[2 * num_pg];
    for (int k = 0; k < num_params; ++k) grad[k] = 0.0;
    for (int j = 0; j < num_pg; ++j) grad[slot_param[j]] += -2.0 * slot_scale[j] * host[2 * j + 1];
    return RBK_OK;
  });
}

extern "C" int rbk_adjoint_create(int num_qubits, int precision, int device, rbk_adjoint_ctx** out)
{
  if (!out) return fail(RBK_ERR_INVALID, "null output pointer");
  rbk::adjoint_workspace* w = nullptr;
  const int rc = rbk::adjoint_workspace_create(num_qubits, precision, device, &w);
  *out = reinterpret_cast<rbk_adjoint_ctx*>(w);
  return rc;
}

extern "C" int rbk_adjoint_run(rbk_adjoint_ctx* ctx, const rbk_circuit_gate* gates, int num_gates, const double* theta,
                               int num_params, int num_terms, const char* strings, const double* coeffs, double* energy,
                               double* grad)
{
  return rbk::adjoint_run(reinterpret_cast<rbk::adjoint_workspace*>(ctx), gates, num_gates, theta, num_params, num_terms,
                          strings, coeffs, energy, grad);
}

extern "C" int rbk_adjoint_destroy(rbk_adjoint_ctx* ctx)
{
  rbk::adjoint_workspace_destroy(reinterpret_cast<rbk::adjoint_workspace*>(ctx));
  return RBK_OK;
}

extern "C" int rbk_adjoint_gradient(int num_qubits, int precision, int device, const rbk_circuit_gate* gates,
                                    int num_gates, const double* theta, int num_params, int num_terms,
                                    const char* strings, const double* coeffs, double* energy, double* grad)
{
  rbk::adjoint_workspace* w = nullptr;
  if (int rc = rbk::adjoint_workspace_create(num_qubits, precision, device, &w)) return rc;
  const int rc = rbk::adjoint_run(w, gates, num_gates, theta, num_params, num_terms, strings, coeffs, energy, grad);
  rbk::adjoint_workspace_destroy(w);
  return rc;
}

// ---- sampling and measurement ------------------------------------------------

namespace {

// ket::utility::positive_random_value_upto (ket/include/ket/utility/positive_random_value_upto.hpp):
// a uniform_real_distribution on [0, maximum).
double random_upto(std::mt19937_64& g, double maximum)
{
  std::uniform_real_distribution<double> d{0.0, maximum};
  return d(g);
}

// Inclusive prefix sums of |a_i|^2 in logical order, plus the total.
int prob_prefix(rbk_state* s, device_buffer& prefix, device_buffer& scratch, double* total)
{
  if (int rc = canonicalize(s)) return rc;
  device_guard g(s->device);
  const uint64_t size = 1ull << s->n;
  RBK_CUDA(cudaMalloc(reinterpret_cast<void**>(&prefix.p), sizeof(double) * size));
  RBK_CUDA(cudaMalloc(reinterpret_cast<void**>(&scratch.p), sizeof(double) * rbk::scan_scratch_doubles(size)));
  const cudaError_t e = s->precision == RBK_C128 ? rbk::launch_prob_scan<double>(s->amps, size, prefix.p, scratch.p, s->stream)
                                                : rbk::launch_prob_scan<float>(s->amps, size, prefix.p, scratch.p, s->stream);
  if (e != cudaSuccess) return cuda_fail(e, "probability scan");
  s->stats.kernel_launches += 2;
  RBK_CUDA(cudaMemcpyAsync(s->h_out, prefix.p + (size - 1), sizeof(double), cudaMemcpyDeviceToHost, s->stream));
  if (int rc = bounded_sync(s)) return rc;
  *total = s->h_out[0];
  return RBK_OK;
}

// draw(upper): one uniform value on [0, upper), taken in event order.
template <typename Draw>
int sample_indices(rbk_state* s, Draw&& draw, int num, uint64_t* out)
{
  device_buffer prefix, scratch, rbuf;
  double total = 0;
  if (int rc = prob_prefix(s, prefix, scratch, &total)) return rc;
  std::vector<double> r(num);
  for (auto& x : r) x = draw(total);
  RBK_CUDA(cudaMalloc(reinterpret_cast<void**>(&rbuf.p), sizeof(double) * 2 * num));
  uint64_t* ev = reinterpret_cast<uint64_t*>(rbuf.p + num);
  RBK_CUDA(cudaMemcpyAsync(rbuf.p, r.data(), sizeof(double) * num, cudaMemcpyHostToDevice, s->stream));
  RBK_CUDA(rbk::launch_upper_bound(prefix.p, 1ull << s->n, rbuf.p, num, ev, s->stream));
  ++s->stats.kernel_launches;
  RBK_CUDA(cudaMemcpyAsync(out, ev, sizeof(uint64_t) * num, cudaMemcpyDeviceToHost, s->stream));
  if (int rc = bounded_sync(s)) return rc;
  // upper_bound can land past the end only when r reaches the total (rounding); clamp like the last bin.
  const uint64_t last = (1ull << s->n) - 1;
  for (int k = 0; k < num; ++k) if (out[k] > last) out[k] = last;
  return RBK_OK;
}

}  // namespace

extern "C" int rbk_state_seed(rbk_state* s, uint64_t seed)
{
  if (int rc = check_state(s)) return rc;
  s->rng.seed(seed);
  return RBK_OK;
}

extern "C" int rbk_generate_events(rbk_state* s, int num_events, int64_t seed, uint64_t* events)
{
  return guarded([&]() -> int {
    if (int rc = check_state(s)) return rc;
    if (num_events < 0 || (num_events > 0 && !events)) return fail(RBK_ERR_INVALID, "bad event arguments");
    if (num_events == 0) return RBK_OK;
    if (seed < 0) return sample_indices(s, [&](double upper) { return random_upto(s->rng, upper); }, num_events, events);
    std::mt19937_64 fresh(static_cast<uint64_t>(seed));  // generate_events.hpp: a generator built from the seed
    return sample_indices(s, [&](double upper) { return random_upto(fresh, upper); }, num_events, events);
  });
}

extern "C" int rbk_measure(rbk_state* s, uint64_t* outcome)
{
  return guarded([&]() -> int {
    if (int rc = check_state(s)) return rc;
    if (!outcome) return fail(RBK_ERR_INVALID, "null output pointer");
    uint64_t idx = 0;
    if (int rc = sample_indices(s, [&](double upper) { return random_upto(s->rng, upper); }, 1, &idx)) return rc;
    *outcome = idx;
    return rbk_state_reset(s, idx);  // measure.hpp: the state becomes |outcome>
  });
}

extern "C" int rbk_generate_events_with(rbk_state* s, int num_events, rbk_uniform_fn draw, void* context, uint64_t* events)
{
  return guarded([&]() -> int {
    if (int rc = check_state(s)) return rc;
    if (num_events < 0 || (num_events > 0 && !events) || !draw) return fail(RBK_ERR_INVALID, "bad event arguments");
    if (num_events == 0) return RBK_OK;
    return sample_indices(s, [&](double upper) { return draw(context, upper); }, num_events, events);
  });
}

extern "C" int rbk_measure_with(rbk_state* s, rbk_uniform_fn draw, void* context, uint64_t* outcome)
{
  return guarded([&]() -> int {
    if (int rc = check_state(s)) return rc;
    if (!outcome || !draw) return fail(RBK_ERR_INVALID, "null output pointer or random source");
    uint64_t idx = 0;
    if (int rc = sample_indices(s, [&](double upper) { return draw(context, upper); }, 1, &idx)) return rc;
    *outcome = idx;
    return rbk_state_reset(s, idx);
  });
}

extern "C" int rbk_projective_measurement(rbk_state* s, uint32_t qubit, int* outcome)
{
  return guarded([&]() -> int {
    if (int rc = check_state(s)) return rc;
    if (!outcome) return fail(RBK_ERR_INVALID, "null output pointer");
    if (qubit >= static_cast<uint32_t>(s->n)) return fail(RBK_ERR_INVALID, "qubit index out of range");
    int rc = launch_reduction(s, [&] {
      return s->precision == RBK_C128 ? rbk::launch_zsum<double>(s->amps, s->n, s->d_partials, s->d_out, s->stream)
                                      : rbk::launch_zsum<float>(s->amps, s->n, s->d_partials, s->d_out, s->stream);
    });
    if (rc) return rc;
    if ((rc = read_out(s, s->n + 1))) return rc;
    const double p1 = s->h_out[1 + s->perm[qubit]];
    const double p0 = s->h_out[0] - p1;
    const int one = random_upto(s->rng, p0 + p1) < p0 ? 0 : 1;
    // projective_measurement.hpp: keep the measured half scaled by p^(-1/2), zero the other half.
    double d[4] = {0, 0, 0, 0};
    if (one) d[2] = std::pow(p1, -0.5);
    else d[0] = std::pow(p0, -0.5);
    *outcome = one;
    if ((rc = rbk_apply_diagonal2(s, d, qubit, nullptr, 0))) return rc;
    return flush(s);
  });
}

// ---- further ket gate families ---------------------------------------------
// Gates outside the brick/QFT hot path that bra's instruction set reaches.
// Each is written as a short sequence of the queued primitives above, so it
// joins the same fused passes; only CLEAR/SET and SHORBOX run kernels of their
// own.

namespace {

int enqueue_matrix(rbk_state* s, const std::array<cplx, 4>& u, uint32_t target, const uint32_t* controls, int nc)
{
  double m[8];
  for (int k = 0; k < 4; ++k) put(m, k, u[k]);
  return enqueue_target(s, rbk::OPK_MAT, target, controls, nc, m);
}

// controls + extra, as one qubit list.
std::vector<uint32_t> with_qubit(const uint32_t* controls, int nc, uint32_t extra)
{
  std::vector<uint32_t> v(controls, controls + nc);
  v.push_back(extra);
  return v;
}

// Targets and controls all valid and pairwise distinct.
int check_targets_controls(rbk_state* s, const uint32_t* targets, int nt, const uint32_t* controls, int nc)
{
  if (int rc = check_state(s)) return rc;
  if (nt < 1) return fail(RBK_ERR_INVALID, "at least one target qubit is needed");
  if (nc < 0) return fail(RBK_ERR_INVALID, "negative control count");
  std::vector<uint32_t> all(targets, targets + nt);
  if (nc > 0) {
    if (!controls) return fail(RBK_ERR_INVALID, "null control array");
    all.insert(all.end(), controls, controls + nc);
  }
  uint64_t mask = 0;
  return check_qubits(s, all.data(), static_cast<int>(all.size()), &mask);
}

// Probabilities of qubit q being 0 and 1 (logical qubit; one reduction pass).
int qubit_probabilities(rbk_state* s, uint32_t q, double* p0, double* p1)
{
  int rc = launch_reduction(s, [&] {
    return s->precision == RBK_C128 ? rbk::launch_zsum<double>(s->amps, s->n, s->d_partials, s->d_out, s->stream)
                                    : rbk::launch_zsum<float>(s->amps, s->n, s->d_partials, s->d_out, s->stream);
  });
  if (rc) return rc;
  if ((rc = read_out(s, s->n + 1))) return rc;
  *p1 = s->h_out[1 + s->perm[q]];
  *p0 = s->h_out[0] - *p1;
  return RBK_OK;
}

// Keeps the half of qubit q equal to `one`, scaled by p^(-1/2); zeroes the other.
int collapse(rbk_state* s, uint32_t q, int one, double p)
{
  double d[4] = {0, 0, 0, 0};
  d[one ? 2 : 0] = std::pow(p, -0.5);
  if (int rc = rbk_apply_diagonal2(s, d, q, nullptr, 0)) return rc;
  return flush(s);
}

}  // namespace

extern "C" int rbk_projective_measurement_with(rbk_state* s, uint32_t qubit, rbk_uniform_fn draw, void* context,
                                               int* outcome)
{
  return guarded([&]() -> int {
    if (int rc = check_state(s)) return rc;
    if (!outcome || !draw) return fail(RBK_ERR_INVALID, "null output pointer or random source");
    if (qubit >= static_cast<uint32_t>(s->n)) return fail(RBK_ERR_INVALID, "qubit index out of range");
    double p0 = 0, p1 = 0;
    if (int rc = qubit_probabilities(s, qubit, &p0, &p1)) return rc;
    const int one = draw(context, p0 + p1) < p0 ? 0 : 1;
    *outcome = one;
    return collapse(s, qubit, one, one ? p1 : p0);
  });
}

extern "C" int rbk_x_rotation_half_pi(rbk_state* s, int adjoint, uint32_t target, const uint32_t* controls, int nc)
{
  // +X: ((a0 + i a1), (i a0 + a1)) / sqrt2; -X conjugates i (x_rotation_half_pi.hpp:34, :254)
  return guarded([&]() -> int {
    const double si = adjoint ? -kOneDivRootTwo : kOneDivRootTwo;
    const std::array<cplx, 4> u{cplx{kOneDivRootTwo, 0}, cplx{0, si}, cplx{0, si}, cplx{kOneDivRootTwo, 0}};
    return enqueue_matrix(s, u, target, controls, nc);
  });
}

extern "C" int rbk_y_rotation_half_pi(rbk_state* s, int adjoint, uint32_t target, const uint32_t* controls, int nc)
{
  // +Y: ((a0 + a1), (-a0 + a1)) / sqrt2; -Y: ((a0 - a1), (a0 + a1)) / sqrt2 (y_rotation_half_pi.hpp:33, :251)
  return guarded([&]() -> int {
    const double r = kOneDivRootTwo, off = adjoint ? -r : r;
    const std::array<cplx, 4> u{cplx{r, 0}, cplx{off, 0}, cplx{-off, 0}, cplx{r, 0}};
    return enqueue_matrix(s, u, target, controls, nc);
  });
}

extern "C" int rbk_sqrt_pauli_x(rbk_state* s, int adjoint, uint32_t target, const uint32_t* controls, int nc)
{
  // sX = [[1+i, 1-i], [1-i, 1+i]] / 2, sX+ its conjugate (sqrt_pauli_x.hpp:32, :259)
  return guarded([&]() -> int {
    const double sg = adjoint ? -0.5 : 0.5;
    const cplx p{0.5, sg}, m{0.5, -sg};
    const std::array<cplx, 4> u{p, m, m, p};
    return enqueue_matrix(s, u, target, controls, nc);
  });
}

extern "C" int rbk_sqrt_pauli_y(rbk_state* s, int adjoint, uint32_t target, const uint32_t* controls, int nc)
{
  // sY = (1+i)/2 [[1, -1], [1, 1]]; sY+ = (1-i)/2 [[1, 1], [-1, 1]] (sqrt_pauli_y.hpp:33, :256)
  return guarded([&]() -> int {
    const cplx c = adjoint ? cplx{0.5, -0.5} : cplx{0.5, 0.5};
    const std::array<cplx, 4> u = adjoint ? std::array<cplx, 4>{c, c, -c, c} : std::array<cplx, 4>{c, -c, c, c};
    return enqueue_matrix(s, u, target, controls, nc);
  });
}

extern "C" int rbk_sqrt_pauli_z(rbk_state* s, int adjoint, const uint32_t* targets, int nt, const uint32_t* controls, int nc)
{
  // C...C(sZ_t1 ... sZ_tm): each target's |1> times i (or -i) where all controls are one
  // (sqrt_pauli_z.hpp:55-57, :459-461; runtime form :137-205)
  return guarded([&]() -> int {
    if (int rc = check_targets_controls(s, targets, nt, controls, nc)) return rc;
    const cplx c{0.0, adjoint ? -1.0 : 1.0};
    for (int k = 0; k < nt; ++k) {
      auto qs = with_qubit(controls, nc, targets[k]);
      if (int rc = enqueue_phase(s, c, qs.data(), static_cast<int>(qs.size()))) return rc;
    }
    return RBK_OK;
  });
}

extern "C" int rbk_pauli_string(rbk_state* s, const char* paulis, const uint32_t* targets, int nt, const uint32_t* controls,
                                int nc)
{
  // C...C(P_t1 ... P_tm), P in {X, Y, Z}: the single-qubit Paulis commute, so the
  // product is applied factor by factor under the same controls (pauli_x.hpp runtime
  // form :288-572; pauli_y.hpp, pauli_z.hpp likewise).  Exact: every factor only
  // moves amplitudes and multiplies them by +-1 or +-i.
  return guarded([&]() -> int {
    if (!paulis) return fail(RBK_ERR_INVALID, "null Pauli string");
    if (int rc = check_targets_controls(s, targets, nt, controls, nc)) return rc;
    for (int k = 0; k < nt; ++k) {
      const char p = paulis[k];
      int rc;
      if (p == 'X') rc = enqueue_target(s, rbk::OPK_X, targets[k], controls, nc, nullptr);
      else if (p == 'Y') rc = enqueue_target(s, rbk::OPK_Y, targets[k], controls, nc, nullptr);
      else if (p == 'Z') {
        auto qs = with_qubit(controls, nc, targets[k]);
        rc = enqueue_phase(s, cplx{-1.0, 0.0}, qs.data(), static_cast<int>(qs.size()));
      } else if (p == 'I') rc = RBK_OK;
      else return fail(RBK_ERR_INVALID, "Pauli string characters must be I, X, Y or Z");
      if (rc) return rc;
    }
    return RBK_OK;
  });
}

extern "C" int rbk_exponential_pauli_string(rbk_state* s, double phase, const char* paulis, const uint32_t* targets, int nt,
                                            const uint32_t* controls, int nc)
{
  // C...C exp(i phase P_t1 ... P_tm) (exponential_pauli_x.hpp, _y.hpp, _z.hpp runtime forms).
  // One target: the single-qubit kernels.  Several: rotate each X/Y factor into Z
  // (H for X; S+ then H for Y), gather the parity of the targets into the last one
  // with CNOTs, apply C...C exp(i phase Z) there, and undo the ladder and the basis
  // change.  The outer steps need no controls: they cancel where a control is zero.
  return guarded([&]() -> int {
    if (!paulis) return fail(RBK_ERR_INVALID, "null Pauli string");
    if (int rc = check_targets_controls(s, targets, nt, controls, nc)) return rc;
    std::vector<uint32_t> act;
    std::vector<char> kind;
    for (int k = 0; k < nt; ++k) {
      const char p = paulis[k];
      if (p == 'I') continue;
      if (p != 'X' && p != 'Y' && p != 'Z') return fail(RBK_ERR_INVALID, "Pauli string characters must be I, X, Y or Z");
      act.push_back(targets[k]);
      kind.push_back(p);
    }
    if (act.empty()) {  // exp(i phase I) under the controls: a phase on the all-ones subspace
      if (nc == 0) {
        const cplx c = exp_i(phase);
        double d[4] = {c.real(), c.imag(), c.real(), c.imag()};
        return rbk_apply_diagonal2(s, d, targets[0], nullptr, 0);
      }
      return enqueue_phase(s, exp_i(phase), controls, nc);
    }
    const int m = static_cast<int>(act.size());
    if (m == 1) {
      if (kind[0] == 'X') return rbk_exponential_pauli_x(s, phase, act[0], controls, nc);
      if (kind[0] == 'Y') return rbk_exponential_pauli_y(s, phase, act[0], controls, nc);
      return rbk_exponential_pauli_z(s, phase, act[0], controls, nc);
    }
    const cplx sdag[2] = {{1.0, 0.0}, {0.0, -1.0}};
    for (int k = 0; k < m; ++k) {
      if (kind[k] == 'Y') {
        double d[4] = {sdag[0].real(), sdag[0].imag(), sdag[1].real(), sdag[1].imag()};
        if (int rc = rbk_apply_diagonal2(s, d, act[k], nullptr, 0)) return rc;
      }
      if (kind[k] != 'Z')
        if (int rc = rbk_hadamard(s, act[k], nullptr, 0)) return rc;
    }
    for (int k = 0; k + 1 < m; ++k) {
      const uint32_t c1[1] = {act[k]};
      if (int rc = enqueue_target(s, rbk::OPK_X, act[k + 1], c1, 1, nullptr)) return rc;
    }
    if (int rc = rbk_exponential_pauli_z(s, phase, act[m - 1], controls, nc)) return rc;
    for (int k = m - 2; k >= 0; --k) {
      const uint32_t c1[1] = {act[k]};
      if (int rc = enqueue_target(s, rbk::OPK_X, act[k + 1], c1, 1, nullptr)) return rc;
    }
    for (int k = 0; k < m; ++k) {
      if (kind[k] != 'Z')
        if (int rc = rbk_hadamard(s, act[k], nullptr, 0)) return rc;
      if (kind[k] == 'Y') {
        double d[4] = {1.0, 0.0, 0.0, 1.0};  // S
        if (int rc = rbk_apply_diagonal2(s, d, act[k], nullptr, 0)) return rc;
      }
    }
    return RBK_OK;
  });
}

extern "C" int rbk_exponential_swap(rbk_state* s, double phase, uint32_t q1, uint32_t q2, const uint32_t* controls, int nc)
{
  // C...C exp(i phase SWAP) = e^{i phase} on |00>, |11>; [[cos, i sin], [i sin, cos]] on
  // |01>, |10> (exponential_swap.hpp:37-40, :103).  After CNOT(q1 -> q2) the swapped
  // pair differs only in q1 with q2 = 1, and |00>, |11> sit at q2 = 0: so
  // CNOT . [C...C exp(i phase X_q1) controlled by q2 too] . [C...C diag(e^{i phase}, 1) on q2] . CNOT.
  return guarded([&]() -> int {
    const uint32_t t[2] = {q1, q2};
    if (int rc = check_targets_controls(s, t, 2, controls, nc)) return rc;
    const uint32_t c1[1] = {q1};
    if (int rc = enqueue_target(s, rbk::OPK_X, q2, c1, 1, nullptr)) return rc;
    auto cq2 = with_qubit(controls, nc, q2);
    if (int rc = rbk_exponential_pauli_x(s, phase, q1, cq2.data(), static_cast<int>(cq2.size()))) return rc;
    const cplx e = exp_i(phase);
    double d[4] = {e.real(), e.imag(), 1.0, 0.0};
    if (int rc = rbk_apply_diagonal2(s, d, q2, controls, nc)) return rc;
    return enqueue_target(s, rbk::OPK_X, q2, c1, 1, nullptr);
  });
}

extern "C" int rbk_clear(rbk_state* s, uint32_t qubit)
{
  // CLEAR i: ket::gate::clear (ket/include/ket/gate/clear.hpp): qubit i projected onto |0>,
  // renormalised by p0^(-1/2).
  return guarded([&]() -> int {
    if (int rc = check_state(s)) return rc;
    if (qubit >= static_cast<uint32_t>(s->n)) return fail(RBK_ERR_INVALID, "qubit index out of range");
    if (s->in_fusion) return fail(RBK_ERR_STATE, "CLEAR inside a fusion block");
    double p0 = 0, p1 = 0;
    if (int rc = qubit_probabilities(s, qubit, &p0, &p1)) return rc;
    return collapse(s, qubit, 0, p0);
  });
}

extern "C" int rbk_set(rbk_state* s, uint32_t qubit)
{
  // SET i: ket::gate::set (ket/include/ket/gate/set.hpp): projected onto |1>, renormalised by p1^(-1/2).
  return guarded([&]() -> int {
    if (int rc = check_state(s)) return rc;
    if (qubit >= static_cast<uint32_t>(s->n)) return fail(RBK_ERR_INVALID, "qubit index out of range");
    if (s->in_fusion) return fail(RBK_ERR_STATE, "SET inside a fusion block");
    double p0 = 0, p1 = 0;
    if (int rc = qubit_probabilities(s, qubit, &p0, &p1)) return rc;
    return collapse(s, qubit, 1, p1);
  });
}

extern "C" int rbk_shor_box(rbk_state* s, uint32_t num_exponent_qubits, uint64_t divisor, uint64_t base)
{
  // SHORBOX nx N a: ket::ranges::shor_box (ket/include/ket/shor_box.hpp) with the exponent on
  // the top nx qubits and the modular register on the rest (bra/src/state.cpp, shor_box).
  // The previous contents are discarded.
  return guarded([&]() -> int {
    if (int rc = check_state(s)) return rc;
    if (s->in_fusion) return fail(RBK_ERR_STATE, "SHORBOX inside a fusion block");
    if (num_exponent_qubits > static_cast<uint32_t>(s->n)) return fail(RBK_ERR_INVALID, "more exponent qubits than qubits");
    if (divisor == 0 || divisor > (1ull << 32) || base >= (1ull << 32))
      return fail(RBK_ERR_INVALID, "SHORBOX needs 0 < divisor <= 2^32 and base < 2^32");
    s->queue.clear();
    for (int q = 0; q < s->n; ++q) s->perm[q] = s->inv[q] = q;
    device_guard g(s->device);
    if (int rc = mark_launch_start(s)) return rc;
    const uint64_t size = 1ull << s->n;
    RBK_CUDA(cudaMemsetAsync(s->amps, 0, size * amp_bytes(s->precision), s->stream));
    const int nx = static_cast<int>(num_exponent_qubits);
    const double coeff = std::pow(static_cast<double>(1ull << nx), -0.5);
    const cudaError_t e = s->precision == RBK_C128
                              ? rbk::launch_shor_box<double>(s->amps, s->n, nx, divisor, base, coeff, s->stream)
                              : rbk::launch_shor_box<float>(s->amps, s->n, nx, divisor, base, coeff, s->stream);
    if (e != cudaSuccess) return cuda_fail(e, "shor box");
    ++s->stats.kernel_launches;
    RBK_CUDA(cudaEventRecord(s->ev_last, s->stream));
    return RBK_OK;
  });
}

// ---- dense k-qubit unitaries and the tensor-core fusion mode ---------------

namespace {

// Moves logical qubits q[0..k-1] onto physical bits 0..k-1 (in that order) with
// the canonicalising passes: the planner moves logical j to physical j, so the
// map is first renamed so that q[i] is "logical i", then restored.
int move_to_low(rbk_state* s, const uint32_t* q, int k)
{
  if (int rc = flush(s)) return rc;
  const int n = s->n;
  // Virtual names chosen so that canonicalising moves as little as possible:
  // target i is named i; every other qubit keeps the name of its physical bit,
  // except those sitting on bits 0..k-1, which take the bits the targets leave.
  std::vector<int> sigma(n, -1);  // real logical -> virtual logical
  std::vector<char> is_target(n, 0);
  for (int i = 0; i < k; ++i) { sigma[q[i]] = i; is_target[q[i]] = 1; }
  std::vector<int> freed;
  for (int i = 0; i < k; ++i)
    if (s->perm[q[i]] >= k) freed.push_back(s->perm[q[i]]);
  size_t f = 0;
  for (int l = 0; l < n; ++l) {
    if (is_target[l]) continue;
    sigma[l] = s->perm[l] >= k ? s->perm[l] : freed.at(f++);
  }
  bool in_place = true;
  for (int i = 0; i < k; ++i) in_place = in_place && s->perm[q[i]] == i;
  if (in_place) return RBK_OK;
  std::vector<int> perm_v(n), inv_v(n);
  for (int l = 0; l < n; ++l) perm_v[sigma[l]] = s->perm[l];
  for (int v = 0; v < n; ++v) inv_v[perm_v[v]] = v;
  std::vector<int> unsigma(n);
  for (int l = 0; l < n; ++l) unsigma[sigma[l]] = l;
  s->perm = perm_v;
  s->inv = inv_v;
  const int rc = canonicalize(s);
  // canonicalize leaves virtual v on physical v, i.e. real l on physical sigma[l]
  for (int l = 0; l < n; ++l) s->perm[l] = sigma[l];
  for (int v = 0; v < n; ++v) s->inv[v] = unsigma[v];
  return rc;
}

// W_hi, W_lo of the 3xTF32 kernel (see rbk_tc.cu) in its operand layout:
// operand row = output column j of W, 4-float chunks along K.
float tf32_round_host(float x)
{
  uint32_t b;
  std::memcpy(&b, &x, 4);
  if ((b & 0x7F800000u) != 0x7F800000u) b = (b + 0x1000u) & ~0x1FFFu;  // round to nearest, ties away (cvt.rna)
  float r;
  std::memcpy(&r, &b, 4);
  return r;
}

std::vector<float> build_w_split(const std::vector<cplx>& U, int k)
{
  const int dim = 1 << k, K = 2 * dim;
  std::vector<float> W(static_cast<size_t>(K) * K);  // W[kk * K + j]
  for (int a = 0; a < dim; ++a)
    for (int b = 0; b < dim; ++b) {
      const cplx u = U[static_cast<size_t>(b) * dim + a];
      W[(2 * a) * K + 2 * b] = static_cast<float>(u.real());
      W[(2 * a + 1) * K + 2 * b] = static_cast<float>(-u.imag());
      W[(2 * a) * K + 2 * b + 1] = static_cast<float>(u.imag());
      W[(2 * a + 1) * K + 2 * b + 1] = static_cast<float>(u.real());
    }
  std::vector<float> out(rbk::tc_w_split_floats(k), 0.0f);
  const size_t half = out.size() / 2;
  for (int j = 0; j < K; ++j)        // operand row (N index)
    for (int kk = 0; kk < K; ++kk) {  // K index
      const size_t off = static_cast<size_t>(j >> 3) * (K / 4) * 32 + static_cast<size_t>(kk >> 2) * 32 + (j & 7) * 4 + (kk & 3);
      const float w = W[static_cast<size_t>(kk) * K + j];
      const float hi = tf32_round_host(w);
      out[off] = hi;
      out[half + off] = tf32_round_host(w - hi);
    }
  return out;
}

int apply_unitary(rbk_state* s, const std::vector<cplx>& U, const uint32_t* q, int k)
{
  device_guard g(s->device);
  const bool tensor = s->precision == RBK_C64 && (k == 5 || k == 6) && s->n >= k + 7;
  if (tensor) {
    if (int rc = flush(s)) return rc;
  } else if (int rc = move_to_low(s, q, k)) {
    return rc;
  }
  if (int rc = mark_launch_start(s)) return rc;
  ++s->stats.gates_issued;
  if (tensor) {
    // The kernel gathers rows at the targets' current physical bits: no relabelling pass.
    rbk::tc_layout lay{};
    uint64_t used = 0;
    for (int i = 0; i < k; ++i) {
      lay.target_bit[i] = static_cast<uint8_t>(s->perm[q[i]]);
      used |= 1ull << s->perm[q[i]];
    }
    int j = 0;
    for (int b = 0; b < s->n && j < 7; ++b)
      if (!(used & (1ull << b))) { lay.row_bit[j++] = static_cast<uint8_t>(b); used |= 1ull << b; }
    int src = 0;
    for (int b = 0; b < s->n;) {
      if (used & (1ull << b)) { ++b; continue; }
      int len = 0;
      while (b + len < s->n && !(used & (1ull << (b + len)))) ++len;
      lay.run_src[lay.num_runs] = static_cast<uint8_t>(src);
      lay.run_len[lay.num_runs] = static_cast<uint8_t>(len);
      lay.run_dst[lay.num_runs] = static_cast<uint8_t>(b);
      ++lay.num_runs;
      src += len;
      b += len;
    }
    const std::vector<float> w = build_w_split(U, k);
    if (!s->d_tc_w) {  // once per state: W of the largest k, and the sticky error flag
      RBK_CUDA(cudaMalloc(reinterpret_cast<void**>(&s->d_tc_w), sizeof(float) * rbk::tc_w_split_floats(6)));
      RBK_CUDA(cudaMalloc(reinterpret_cast<void**>(&s->d_tc_flag), sizeof(int)));
      RBK_CUDA(cudaMallocHost(reinterpret_cast<void**>(&s->h_tc_flag), sizeof(int)));
      *s->h_tc_flag = 0;
      RBK_CUDA(cudaMemsetAsync(s->d_tc_flag, 0, sizeof(int), s->stream));
    }
    // Stream order keeps this copy behind the previous unitary's reads of the buffer; the
    // pageable source is staged by the copy call, so w may go when it returns.
    RBK_CUDA(cudaMemcpyAsync(s->d_tc_w, w.data(), sizeof(float) * w.size(), cudaMemcpyHostToDevice, s->stream));
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, s->device);
    const uint64_t tiles = (1ull << (s->n - k)) / 128;
    const int grid = static_cast<int>(std::min<uint64_t>(tiles, static_cast<uint64_t>(sms)));
    const cudaError_t e = rbk::launch_unitary_tf32x3(s->amps, s->n, k, s->d_tc_w, s->d_tc_flag, grid, lay, s->stream);
    if (e != cudaSuccess) return cuda_fail(e, "tensor-core unitary");
    ++s->stats.kernel_launches;
    ++s->stats.passes;
    // No wait here: the flag reaches the pinned copy in stream order and the next
    // bounded_sync (every read of the state) reports a wait that ran out.
    RBK_CUDA(cudaMemcpyAsync(s->h_tc_flag, s->d_tc_flag, sizeof(int), cudaMemcpyDeviceToHost, s->stream));
  } else {
    device_buffer du;
    const size_t count = 2 * U.size();
    RBK_CUDA(cudaMalloc(reinterpret_cast<void**>(&du.p), sizeof(double) * count));
    RBK_CUDA(cudaMemcpyAsync(du.p, reinterpret_cast<const double*>(U.data()), sizeof(double) * count,
                             cudaMemcpyHostToDevice, s->stream));
    const cudaError_t e = s->precision == RBK_C128 ? rbk::launch_dense_rows<double>(s->amps, s->n, k, du.p, s->stream)
                                                  : rbk::launch_dense_rows<float>(s->amps, s->n, k, du.p, s->stream);
    if (e != cudaSuccess) return cuda_fail(e, "dense unitary");
    ++s->stats.kernel_launches;
    ++s->stats.passes;
    if (int rc = bounded_sync(s)) return rc;  // the matrix buffer is freed on return
  }
  RBK_CUDA(cudaEventRecord(s->ev_last, s->stream));
  return RBK_OK;
}

// One queued gate on a vector over the local basis of the block's qubits.
void host_apply(std::vector<cplx>& v, const hgate& g, const std::vector<int>& local)
{
  const int dim = static_cast<int>(v.size());
  uint32_t cm = 0;
  for (int l = 0; l < 64; ++l)
    if (g.cmask & (1ull << l)) cm |= 1u << local[l];
  auto m = [&](int i) { return cplx{g.m[2 * i], g.m[2 * i + 1]}; };
  if (g.kind == rbk::OPK_NEG) {
    for (int i = 0; i < dim; ++i)
      if ((static_cast<uint32_t>(i) & cm) == cm) v[i] = -v[i];
    return;
  }
  if (g.kind == rbk::HK_SWAP) {
    const int a = local[g.target], b = local[g.target2];
    for (int i = 0; i < dim; ++i)
      if (((i >> a) & 1) && !((i >> b) & 1)) std::swap(v[i], v[i ^ (1 << a) ^ (1 << b)]);
    return;
  }
  const int t = local[g.target];
  for (int i = 0; i < dim; ++i) {
    if ((static_cast<uint32_t>(i) & cm) != cm) continue;
    if (g.kind == rbk::OPK_DIAG) {
      if (g.diag_one && !((i >> t) & 1)) continue;
      v[i] *= ((i >> t) & 1) ? m(1) : m(0);
      continue;
    }
    if ((i >> t) & 1) continue;
    const int j = i | (1 << t);
    const cplx a0 = v[i], a1 = v[j];
    if (g.kind == rbk::OPK_X) { v[i] = a1; v[j] = a0; }
    else if (g.kind == rbk::OPK_Y) { v[i] = cplx{a1.imag(), -a1.real()}; v[j] = cplx{-a0.imag(), a0.real()}; }
    else { v[i] = m(0) * a0 + m(1) * a1; v[j] = m(2) * a0 + m(3) * a1; }
  }
}

// END FUSION in the tensor-core mode: the block's gates (queue[fusion_begin..])
// become one dense unitary when they touch 5 or 6 qubits; otherwise the block
// stays in the queue for the fused passes (RBK_NOT_FUSED).
int fuse_block_to_unitary(rbk_state* s)
{
  const size_t b = s->fusion_begin, e = s->queue.size();
  if (b >= e) return RBK_NOT_FUSED;
  uint64_t touched = 0;
  for (size_t i = b; i < e; ++i) {
    const auto& g = s->queue[i];
    touched |= g.cmask;
    if (g.target >= 0) touched |= 1ull << g.target;
    if (g.kind == rbk::HK_SWAP) touched |= 1ull << g.target2;
  }
  const int k = __builtin_popcountll(touched);
  if (k < 5 || k > 6 || s->n < k + 7) return RBK_NOT_FUSED;
  std::vector<uint32_t> q;
  std::vector<int> local(64, -1);
  for (int l = 0; l < s->n; ++l)
    if (touched & (1ull << l)) { local[l] = static_cast<int>(q.size()); q.push_back(static_cast<uint32_t>(l)); }
  const int dim = 1 << k;
  std::vector<cplx> U(static_cast<size_t>(dim) * dim);
  for (int c = 0; c < dim; ++c) {
    std::vector<cplx> v(dim, cplx{0.0, 0.0});
    v[c] = 1.0;
    for (size_t i = b; i < e; ++i) host_apply(v, s->queue[i], local);
    for (int r = 0; r < dim; ++r) U[static_cast<size_t>(r) * dim + c] = v[r];
  }
  s->queue.resize(b);
  return apply_unitary(s, U, q.data(), k);
}

}  // namespace

extern "C" int rbk_apply_unitary(rbk_state* s, const double* u, const uint32_t* qubits, int k)
{
  return guarded([&]() -> int {
    if (int rc = check_state(s)) return rc;
    if (!u) return fail(RBK_ERR_INVALID, "null matrix");
    if (k < 1 || k > 10 || k > s->n) return fail(RBK_ERR_INVALID, "a dense unitary acts on 1 to 10 qubits");
    uint64_t mask = 0;
    if (int rc = check_qubits(s, qubits, k, &mask)) return rc;
    if (s->in_fusion) return fail(RBK_ERR_STATE, "a dense unitary inside a fusion block");
    const int dim = 1 << k;
    std::vector<cplx> U(static_cast<size_t>(dim) * dim);
    for (size_t i = 0; i < U.size(); ++i) U[i] = cplx{u[2 * i], u[2 * i + 1]};
    return apply_unitary(s, U, qubits, k);
  });
}

extern "C" int rbk_state_set_fusion_mode(rbk_state* s, int mode)
{
  if (int rc = check_state(s)) return rc;
  if (mode < 0 || mode > 1) return fail(RBK_ERR_INVALID, "fusion mode must be 0 or 1");
  s->fusion_mode = mode;
  return RBK_OK;
}
