// rbk_noalloc.cu -- rbk_expectation_pauli_noalloc: the Pauli-string
// expectation value of a caller-owned device state, allocating no memory.
//
// Some callers cannot allocate device memory at the time they need an
// observable: a process whose HBM is already reserved in full by another
// allocator (a 33-qubit complex<double> state alone is 128 GiB), or a loop
// that must not hit the implicit device synchronisation of cudaMalloc /
// cudaFree.  This entry point takes the amplitudes and the output from the
// caller and keeps its scratch -- the per-block partial sums of the reduction
// -- in a fixed file-scope device array, so it never allocates.  It does make
// CUDA runtime calls, so a stream callback or host function cannot use it.
#include <cuda_runtime.h>

#include <chrono>
#include <cstdlib>
#include <complex>
#include <cstdint>
#include <string>
#include <thread>
#include <vector>

#include "rbk.h"
#include "rbk_internal.h"
#include "rbk_kernels.h"

namespace {

// Scratch for one call: kNoAllocPartials doubles of per-block partial sums
// (rbk::reduction_blocks() blocks x 2) and kNoAllocGroups (re, im) results,
// one per group of Pauli strings that share their X/Y positions.  About 10 KB
// on every device where this library's device code has been loaded (at the
// first launch or symbol lookup on that device under lazy loading), until the
// process exits.
constexpr int kNoAllocPartials = 2 * 148 * 4;
constexpr int kNoAllocGroups = 64;
__device__ __align__(256) double g_noalloc_scratch[kNoAllocPartials + 2 * kNoAllocGroups];

// Device address of g_noalloc_scratch for each device, looked up once per
// device by the first call made with that device current.  A cudaDeviceReset
// unloads the module, so the address is not valid after one.
double* g_scratch_ptr[64] = {};

int noalloc_fail(int code, const std::string& msg) { return rbk::set_last_error(code, msg.c_str()); }

// Bounded wait on the caller's stream (RBK_TIMEOUT_S seconds, default 600),
// polling so that nothing has to be created.
int bounded_stream_wait(cudaStream_t st)
{
  const char* v = std::getenv("RBK_TIMEOUT_S");
  const double limit = (v && std::atof(v) > 0) ? std::atof(v) : 600.0;
  const auto t0 = std::chrono::steady_clock::now();
  int sleep_us = 20;
  while (true) {
    const cudaError_t e = cudaStreamQuery(st);
    if (e == cudaSuccess) return RBK_OK;
    if (e != cudaErrorNotReady) return noalloc_fail(RBK_ERR_CUDA, std::string("device execution: ") + cudaGetErrorString(e));
    if (std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count() > limit)
      return noalloc_fail(RBK_ERR_TIMEOUT, "timed out waiting for the device");
    std::this_thread::sleep_for(std::chrono::microseconds(sleep_us));
    if (sleep_us < 2000) sleep_us *= 2;
  }
}

}  // namespace

extern "C" int rbk_expectation_pauli_noalloc(const void* device_amps, int num_qubits, int precision, int num_terms,
                                             const char* strings, const double* coeffs, double* out, void* stream)
{
  if (!device_amps || !out || num_terms < 0 || (num_terms > 0 && (!strings || !coeffs)))
    return noalloc_fail(RBK_ERR_INVALID, "null pointer or negative term count");
  if (precision != RBK_C128 && precision != RBK_C64) return noalloc_fail(RBK_ERR_INVALID, "unknown precision");
  const int max_q = precision == RBK_C128 ? 33 : 34;
  if (num_qubits < 1 || num_qubits > max_q) return noalloc_fail(RBK_ERR_INVALID, "number of qubits out of range");
  if (rbk::reduction_blocks() * 2 > kNoAllocPartials)
    return noalloc_fail(RBK_ERR_UNSUPPORTED, "reduction grid larger than the fixed scratch");

  // Group the terms by flip mask: (P psi)(i) = (-i)^{#Y} (-1)^{popcount(i & (Y|Z))} psi(i ^ (X|Y))
  // (ket/include/ket/gate/utility/pauli_index_coeff.hpp:17-59).
  struct term { uint64_t flip, sign; std::complex<double> w; };
  std::vector<term> terms;
  static const std::complex<double> pow_mi[4] = {{1, 0}, {0, -1}, {-1, 0}, {0, 1}};
  for (int t = 0; t < num_terms; ++t) {
    uint64_t x = 0, y = 0, z = 0;
    for (int k = 0; k < num_qubits; ++k) {
      const char c = strings[static_cast<size_t>(t) * num_qubits + k];
      if (c == 'X') x |= 1ull << k;
      else if (c == 'Y') y |= 1ull << k;
      else if (c == 'Z') z |= 1ull << k;
      else if (c != 'I') return noalloc_fail(RBK_ERR_INVALID, "Pauli strings use the characters I, X, Y, Z");
    }
    terms.push_back({x | y, y | z, std::complex<double>{coeffs[2 * t], coeffs[2 * t + 1]} * pow_mi[__builtin_popcountll(y) & 3]});
  }
  std::vector<rbk::pauli_terms> groups;
  std::vector<uint64_t> flips;
  std::vector<char> done(terms.size(), 0);
  for (size_t i = 0; i < terms.size(); ++i) {
    if (done[i]) continue;
    rbk::pauli_terms pt{};
    for (size_t j = i; j < terms.size() && pt.count < rbk::kMaxPauliTerms; ++j) {
      if (done[j] || terms[j].flip != terms[i].flip) continue;
      pt.sign[pt.count] = terms[j].sign;
      pt.w[pt.count][0] = terms[j].w.real();
      pt.w[pt.count][1] = terms[j].w.imag();
      ++pt.count;
      done[j] = 1;
    }
    groups.push_back(pt);
    flips.push_back(terms[i].flip);
  }
  if (static_cast<int>(groups.size()) > kNoAllocGroups)
    return noalloc_fail(RBK_ERR_INVALID, "more than 64 groups of Pauli strings with distinct X/Y positions");

  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return noalloc_fail(RBK_ERR_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
  if (dev < 0 || dev >= 64) return noalloc_fail(RBK_ERR_UNSUPPORTED, "device index above 63");
  // Set-up, once per device: the host name g_noalloc_scratch is only a host-side
  // stand-in; the kernels need the device address of the array.
  if (!g_scratch_ptr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess)
      return noalloc_fail(RBK_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
    g_scratch_ptr[dev] = static_cast<double*>(p);
  }
  double* partials = g_scratch_ptr[dev];
  double* results = partials + kNoAllocPartials;
  cudaStream_t st = static_cast<cudaStream_t>(stream);

  for (size_t g = 0; g < groups.size(); ++g) {
    e = precision == RBK_C128
      ? rbk::launch_pauli<double>(device_amps, num_qubits, flips[g], groups[g], partials, results + 2 * g, st)
      : rbk::launch_pauli<float>(device_amps, num_qubits, flips[g], groups[g], partials, results + 2 * g, st);
    if (e != cudaSuccess) return noalloc_fail(RBK_ERR_CUDA, std::string("reduction launch: ") + cudaGetErrorString(e));
  }
  double host[2 * kNoAllocGroups] = {};
  if (!groups.empty()) {
    // Pageable destination: the copy returns once the data is in host memory.
    e = cudaMemcpyAsync(host, results, sizeof(double) * 2 * groups.size(), cudaMemcpyDeviceToHost, st);
    if (e != cudaSuccess) return noalloc_fail(RBK_ERR_CUDA, std::string("result copy: ") + cudaGetErrorString(e));
    if (int rc = bounded_stream_wait(st)) return rc;
  }
  double re = 0, im = 0;
  for (size_t g = 0; g < groups.size(); ++g) { re += host[2 * g]; im += host[2 * g + 1]; }
  out[0] = re;
  out[1] = im;
  return RBK_OK;
}
