// rbk_device.cuh -- device helpers shared by the kernels.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>

namespace rbk {

template <typename Real> struct ctype;
template <> struct ctype<double> { using c = double2; using v16 = double2; };
template <> struct ctype<float> { using c = float2; using v16 = float4; };

template <typename C>
__device__ __forceinline__ C cmul(C a, C b) { return C{a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x}; }

// m0 * a0 + m1 * a1
template <typename C, typename Real>
__device__ __forceinline__ C cmac2(C a0, C a1, Real m0r, Real m0i, Real m1r, Real m1i)
{
  C r;
  r.x = m0r * a0.x - m0i * a0.y + m1r * a1.x - m1i * a1.y;
  r.y = m0r * a0.y + m0i * a0.x + m1r * a1.y + m1i * a1.x;
  return r;
}

// m0 * a0 + m1 * a1 with real m0, m1
template <typename C, typename Real>
__device__ __forceinline__ C rmac2(C a0, C a1, Real m0, Real m1)
{
  C r;
  r.x = m0 * a0.x + m1 * a1.x;
  r.y = m0 * a0.y + m1 * a1.y;
  return r;
}

// Inserts a zero bit at position q of v (the index arithmetic of ket's pair
// loops, e.g. ket/include/ket/gate/hadamard.hpp:57-59).
__device__ __forceinline__ uint64_t insert_zero(uint64_t v, int q)
{
  const uint64_t low = (1ull << q) - 1;
  return ((v & ~low) << 1) | (v & low);
}

// Shared-memory slot of tile index j.  The 16-byte vector index u = j >> vbits
// gets its low 3 bits XORed with the XOR-fold of its higher 3-bit groups, so
// that layouts whose lanes sit on any tile bits spread over the 8 bank groups
// of a 128-byte row.  The map is linear over GF(2): slot(x ^ y) = slot(x) ^ slot(y),
// which lets a thread compose addresses from per-bit slots with XORs.
template <int VBITS>
__device__ __forceinline__ uint32_t smem_slot(uint32_t j)
{
  uint32_t u = j >> VBITS;
  const uint32_t f = (u >> 3) ^ (u >> 6) ^ (u >> 9) ^ (u >> 12);
  u ^= f & 7u;
  return (u << VBITS) | (j & ((1u << VBITS) - 1));
}

}  // namespace rbk
