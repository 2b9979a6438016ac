// rbk_tc.cu -- dense k-qubit unitaries (k = 5, 6) on a complex<float> state as
// tensor-core GEMMs with 3xTF32 split products (tcgen05, accumulator in TMEM).
//
// Rows are the 2^(n-k) groups of 2^k amplitudes that differ only in the k
// target bits; a row, read as 2K = 2^(k+1) interleaved floats, is one GEMM row.
// The loads and stores gather rows through offset tables, so the targets may sit
// on any physical bits; a CTA tile is 128 rows spread over the 7 lowest
// non-target bits (contiguous 64-byte or longer runs in HBM).  Applying U is out_row = in_row . W with the real
// 2K x 2K matrix
//   W[2a][2b] = Re U[b][a],  W[2a+1][2b] = -Im U[b][a],
//   W[2a][2b+1] = Im U[b][a], W[2a+1][2b+1] = Re U[b][a],
// a plain real GEMM of M = R rows, N = K = 2^(k+1).  Each product is split as
// x = hi + lo with hi = tf32(x) and lo = tf32(x - hi), and
//   A.W ~ A_hi.W_hi + A_hi.W_lo + A_lo.W_hi   (FP32 accumulation in TMEM),
// which carries about 21 mantissa bits per product -- the FP32 result, on the
// tensor cores.  This is the bra-fused 2^k x 2^k unitary of a fusion block
// (bra/src/nompi_state.cpp:1285-1357 replays the gates instead).
//
// One CTA per SM (persistent), 288 threads in three roles that meet at
// mbarriers (see the kernel): producer warps stream K quarters of 128-row
// tiles from HBM, kTcDepth quarters ahead in registers, and split them into
// A_hi / A_lo operand slots; one thread issues the tcgen05.mma of each quarter;
// epilogue warps read finished accumulators with tcgen05.ld and write the rows
// back in place.  W_hi and W_lo stay in shared memory for the whole launch in
// the canonical K-major layout without swizzle (8-row x 16-byte core
// matrices).  Every mbarrier wait is bounded: on expiry the kernel raises an
// error flag, every role stops, the MMA thread waits (bounded) for its own
// MMAs, and the CTA frees its TMEM and returns.
#include <cuda_runtime.h>

#include <cstdint>

#include "rbk_device.cuh"
#include "rbk_kernels.h"

namespace rbk {
namespace {

constexpr int kTcThreads = 288;  // 4 producer, 4 epilogue and 1 MMA warp
constexpr int kTcDepth = 3;       // K quarters whose loads are in flight
constexpr int kTcM = 128;
constexpr uint32_t kWaitLimit = 1u << 22;

__device__ __forceinline__ uint32_t smem_addr(const void* p) { return static_cast<uint32_t>(__cvta_generic_to_shared(p)); }

// Shared-memory matrix descriptor, K-major, no swizzle (SWIZZLE_NONE = 0 in bits 61-63),
// version 1 in bits 46-47.  lbo: byte step between the two 16-byte K chunks of one
// MMA; sbo: byte step between 8-row groups.
__device__ __forceinline__ uint64_t kmajor_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo)
{
  return uint64_t((saddr >> 4) & 0x3FFFu) | (uint64_t((lbo >> 4) & 0x3FFFu) << 16) |
         (uint64_t((sbo >> 4) & 0x3FFFu) << 32) | (uint64_t(1) << 46);
}

// Instruction descriptor of kind::tf32: D in F32, A and B TF32, both K-major.
__host__ __device__ constexpr uint32_t tf32_idesc(int M, int N)
{
  return (1u << 4) | (2u << 7) | (2u << 10) | (uint32_t(N >> 3) << 17) | (uint32_t(M >> 4) << 24);
}

// Round to TF32 (10 mantissa bits), nearest with ties away from zero, with the
// 13 dropped bits cleared so that x - tf32(x) is the exact remainder.
__device__ __forceinline__ float tf32_rna(float x)
{
  uint32_t b = __float_as_uint(x);
  if ((b & 0x7F800000u) != 0x7F800000u) b = (b + 0x1000u) & 0xFFFFE000u;
  return __uint_as_float(b);
}

__device__ __forceinline__ void umma_tf32(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc, uint32_t acc)
{
  asm volatile(
    "{\n\t"
    ".reg .pred p;\n\t"
    "setp.ne.b32 p, %4, 0;\n\t"
    "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t"
    "}\n" ::"r"(tmem_d),
    "l"(adesc), "l"(bdesc), "r"(idesc), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void async_proxy_fence() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ bool mbar_try_wait(uint32_t addr, uint32_t parity)
{
  uint32_t ok;
  asm volatile(
    "{\n\t"
    ".reg .pred P1;\n\t"
    "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
    "selp.b32 %0, 1, 0, P1;\n\t"
    "}\n"
    : "=r"(ok)
    : "r"(addr), "r"(parity)
    : "memory");
  return ok != 0;
}

__device__ __forceinline__ uint64_t global_ns()
{
  uint64_t t;
  asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
  return t;
}

// Gives up after kWaitLimit polls or 2 s of wall time, whichever comes first.
__device__ __forceinline__ bool mbar_wait_bounded(uint32_t addr, uint32_t parity)
{
  const uint64_t t0 = global_ns();
  for (uint32_t it = 0; it < kWaitLimit; ++it) {
    if (mbar_try_wait(addr, parity)) return true;
    if ((it & 255u) == 255u && global_ns() - t0 > 2000000000ull) return false;
  }
  return false;
}

// Byte offset of element (row, kk) in a K-major operand buffer with kc K-elements per row.
__device__ __forceinline__ uint32_t kmajor_offset(uint32_t row, uint32_t kk, uint32_t kc)
{
  return (row >> 3) * (kc / 4) * 128u + (kk >> 2) * 128u + (row & 7u) * 16u + (kk & 3u) * 4u;
}

// Warp-collective load of 32 consecutive TMEM columns of the warp's lane quarter (one per thread).
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&v)[32])
{
  asm volatile(
    "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
    "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
    "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
    : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
      "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]),
      "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]),
      "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
    : "r"(taddr)
    : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint32_t addr)
{
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(addr) : "memory");
}

template <int KB>  // KB = k + 1: K = N = 2^KB floats per row
__global__ void __launch_bounds__(kTcThreads, 1)
unitary_tf32x3_kernel(float2* __restrict__ state, uint64_t rows, const float4* __restrict__ w_split, int* error_flag,
                      const __grid_constant__ tc_layout L)
{
  // Warp roles, all running at once and meeting at mbarriers:
  //   warps 0-3 (producers): load a K quarter ("stage") of the CTA's next
  //     128-row tile from HBM into registers, kTcDepth stages ahead, split it
  //     into TF32 hi / lo and store both into A slot (stage % 2), then arrive
  //     on full[slot];
  //   warp 8 (MMA issuer, one thread): for each stage wait full[slot], issue
  //     the 3 x K/32 tcgen05.mma into accumulator (tile % 2) and commit to
  //     empty[slot]; after a tile's fourth stage also commit to acc_full[acc];
  //   warps 4-7 (epilogue): wait acc_full[acc], read the accumulator rows
  //     (warp 4 + q owns TMEM lanes 32q..32q+31), write them back to HBM and
  //     arrive on acc_empty[acc] for the MMA issuer.
  // The producers stream the next tile while the tensor cores multiply and
  // the epilogue stores the previous one.
  constexpr uint32_t K = 1u << KB, N = K, KQ = K / 4;
  constexpr uint32_t B_BYTES = N * K * 4, AQ_BYTES = kTcM * KQ * 4;
  constexpr uint32_t SBO_A = (KQ / 4) * 128u, SBO_B = (K / 4) * 128u;
  constexpr uint32_t NCOLS = 2 * N;  // two FP32 accumulators of 128 lanes x N columns
  constexpr uint32_t CG = KQ / 16;   // groups of 4 float4 per row quarter
  constexpr uint32_t PROD_WARPS = 4, PROD_THREADS = PROD_WARPS * 32, EPI_THREADS = 128, MMA_WARP = 8;
  constexpr uint32_t PER_THREAD = (kTcM / 8) * CG / PROD_WARPS;  // float4 per producer thread per stage
  static_assert(PER_THREAD * PROD_WARPS == (kTcM / 8) * CG, "stage split over the producer warps");
  static_assert(kTcThreads == 9 * 32, "4 producer warps, 4 epilogue warps, 1 MMA warp");
  extern __shared__ __align__(1024) unsigned char smem[];
  unsigned char* b_hi = smem;
  unsigned char* b_lo = smem + B_BYTES;
  unsigned char* a_base = smem + 2 * B_BYTES;  // slot b: hi at a_base + 2b AQ, lo at + (2b + 1) AQ
  __shared__ __align__(8) uint64_t full[2], empty[2], acc_full[2], acc_empty[2], done;
  __shared__ uint32_t tmem_slot;
  __shared__ int abort_flag;
  __shared__ uint64_t row_off[kTcM], elem_off[N / 2];  // physical offsets of row bits / target bits
  const uint32_t tid = threadIdx.x, warp = tid >> 5, lane = tid & 31u;
  for (uint32_t i = tid; i < kTcM; i += kTcThreads) {
    uint64_t o = 0;
    for (int b = 0; b < 7; ++b) o |= uint64_t((i >> b) & 1u) << L.row_bit[b];
    row_off[i] = o;
  }
  for (uint32_t i = tid; i < N / 2; i += kTcThreads) {
    uint64_t o = 0;
    for (int b = 0; b < KB - 1; ++b) o |= uint64_t((i >> b) & 1u) << L.target_bit[b];
    elem_off[i] = o;
  }
  const bool pair = L.target_bit[0] == 0;  // then element pairs (2m, 2m+1) are 16-byte aligned neighbours

  if (warp == 0)
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(&tmem_slot)),
                 "r"(NCOLS));
  if (tid == 0) {
    for (int i = 0; i < 2; ++i) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(&full[i])), "r"(PROD_THREADS));
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(&empty[i])), "r"(1u));
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(&acc_full[i])), "r"(1u));
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(&acc_empty[i])), "r"(EPI_THREADS));
    }
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(&done)), "r"(1u));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    abort_flag = 0;
  }
  {
    float4* dst = reinterpret_cast<float4*>(smem);
    for (uint32_t i = tid; i < 2 * B_BYTES / 16; i += kTcThreads) dst[i] = w_split[i];
  }
  async_proxy_fence();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tmem_slot;
  if (warp == 0) asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  const uint32_t idesc = tf32_idesc(kTcM, N);
  const uint64_t tiles = rows / kTcM;
  const uint64_t my_tiles = blockIdx.x < tiles ? (tiles - 1 - blockIdx.x) / gridDim.x + 1 : 0;
  const uint64_t stages = my_tiles * 4;
  // Tile of stage st: its 2^(n-k-7) index deposited into the bits that are neither row nor target bits.
  auto tile_base = [&](uint64_t st) {
    const uint64_t t = blockIdx.x + (st >> 2) * gridDim.x;
    uint64_t v = 0;
    for (int r = 0; r < L.num_runs; ++r) v |= ((t >> L.run_src[r]) & ((1ull << L.run_len[r]) - 1)) << L.run_dst[r];
    return v;
  };
  volatile int* const aborted = &abort_flag;  // written by the role that gives up, read by all
  auto wait = [&](uint64_t* bar, uint32_t parity) {
    if (*aborted) return false;
    if (mbar_wait_bounded(smem_addr(bar), parity)) return true;
    atomicExch(error_flag, 1);
    *aborted = 1;
    return false;
  };

  if (warp < PROD_WARPS) {
    // Where producer thread tid's float4 number i of a stage lives: row r, float column c (within the quarter).
    auto slot_of = [&](uint32_t i, uint32_t& r, uint32_t& c) {
      const uint32_t blk = warp + i * PROD_WARPS;
      const uint32_t rg = blk / CG, cg = blk % CG;
      r = rg * 8 + (lane & 7u);
      c = (cg * 4 + (lane >> 3)) * 4;
    };
    float4 regs[kTcDepth][PER_THREAD];  // a ring of stages in flight, indexed statically
    auto fetch = [&](uint64_t st, float4 (&out)[PER_THREAD]) {
      const uint64_t base = tile_base(st);
      const uint32_t e0 = (uint32_t(st & 3u) * KQ) >> 1;  // first complex element of the quarter
#pragma unroll
      for (uint32_t i = 0; i < PER_THREAD; ++i) {
        uint32_t r, c;
        slot_of(i, r, c);
        const uint64_t rb = base | row_off[r];
        if (pair) {  // elements 2m and 2m+1 are neighbours in memory: one 16-byte load
          out[i] = *reinterpret_cast<const float4*>(state + (rb | elem_off[e0 + (c >> 1)]));
        } else {
          const float2 x0 = state[rb | elem_off[e0 + (c >> 1)]], x1 = state[rb | elem_off[e0 + (c >> 1) + 1]];
          out[i] = make_float4(x0.x, x0.y, x1.x, x1.y);
        }
      }
    };
#pragma unroll
    for (uint32_t d = 0; d < kTcDepth; ++d)
      if (d < stages) fetch(d, regs[d]);
    bool stop = false;
    for (uint64_t s0 = 0; s0 < stages && !stop; s0 += kTcDepth) {
#pragma unroll
      for (uint32_t d = 0; d < kTcDepth; ++d) {
        const uint64_t st = s0 + d;
        if (st >= stages) break;
        const uint32_t buf = uint32_t(st & 1u);
        if (st >= 2 && !wait(&empty[buf], uint32_t((st - 2) >> 1) & 1u)) { stop = true; break; }
        unsigned char* a_hi = a_base + (2 * buf) * AQ_BYTES;
        unsigned char* a_lo = a_hi + AQ_BYTES;
#pragma unroll
        for (uint32_t i = 0; i < PER_THREAD; ++i) {
          uint32_t r, c;
          slot_of(i, r, c);
          const float4 v = regs[d][i];
          float4 hi, lo;
          hi.x = tf32_rna(v.x); lo.x = tf32_rna(v.x - hi.x);
          hi.y = tf32_rna(v.y); lo.y = tf32_rna(v.y - hi.y);
          hi.z = tf32_rna(v.z); lo.z = tf32_rna(v.z - hi.z);
          hi.w = tf32_rna(v.w); lo.w = tf32_rna(v.w - hi.w);
          const uint32_t off = kmajor_offset(r, c, KQ);
          *reinterpret_cast<float4*>(a_hi + off) = hi;
          *reinterpret_cast<float4*>(a_lo + off) = lo;
        }
        async_proxy_fence();  // these generic-proxy stores become visible to the tensor cores
        mbar_arrive(smem_addr(&full[buf]));
        if (st + kTcDepth < stages) fetch(st + kTcDepth, regs[d]);  // in flight while the tensor cores work
      }
    }
  } else if (warp == MMA_WARP) {
    if (lane == 0) {
      for (uint64_t st = 0; st < stages; ++st) {
        const uint32_t buf = uint32_t(st & 1u), q = uint32_t(st & 3u);
        const uint64_t tl = st >> 2;  // tile number within this CTA
        const uint32_t accn = uint32_t(tl & 1u);
        if (q == 0 && tl >= 2 && !wait(&acc_empty[accn], uint32_t((tl - 2) >> 1) & 1u)) break;
        if (!wait(&full[buf], uint32_t(st >> 1) & 1u)) break;
        tc_fence_after();
        const uint32_t acc = tmem + accn * N;
        unsigned char* a_hi = a_base + (2 * buf) * AQ_BYTES;
        unsigned char* a_lo = a_hi + AQ_BYTES;
        const uint32_t ah = smem_addr(a_hi), al = smem_addr(a_lo), bh = smem_addr(b_hi), bl = smem_addr(b_lo);
#pragma unroll
        for (uint32_t j = 0; j < KQ / 8; ++j) {
          const uint32_t g = q * (KQ / 8) + j;
          const uint64_t da_hi = kmajor_desc(ah + j * 256u, 128u, SBO_A), da_lo = kmajor_desc(al + j * 256u, 128u, SBO_A);
          const uint64_t db_hi = kmajor_desc(bh + g * 256u, 128u, SBO_B), db_lo = kmajor_desc(bl + g * 256u, 128u, SBO_B);
          umma_tf32(acc, da_hi, db_hi, idesc, (q | j) != 0 ? 1u : 0u);
          umma_tf32(acc, da_hi, db_lo, idesc, 1u);
          umma_tf32(acc, da_lo, db_hi, idesc, 1u);
        }
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                       smem_addr(&empty[buf]))
                     : "memory");
        if (q == 3)
          asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                         smem_addr(&acc_full[accn]))
                       : "memory");
      }
      // Every MMA issued above has completed once this commit arrives (bounded).
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_addr(&done))
                   : "memory");
      if (!mbar_wait_bounded(smem_addr(&done), 0u)) atomicExch(error_flag, 1);
    }
  } else {
    // Epilogue: warp 4 + q reads TMEM lanes 32q .. 32q + 31 (its rows), 32 columns at a time, and
    // turns them around in its 4 KB of shared memory so that 8 lanes write one row's 128 bytes
    // (lane = row would put the 32 lanes of a store 512 bytes apart).  The float4 slots of a
    // staged row are XOR-swizzled by the row, which keeps both sides free of bank conflicts.
    const uint32_t quad = warp & 3u;
    float4* stage = reinterpret_cast<float4*>(a_base + 4 * AQ_BYTES) + quad * (32 * 8);  // 32 rows x 8 float4
    for (uint64_t tl = 0; tl < my_tiles; ++tl) {
      const uint32_t accn = uint32_t(tl & 1u);
      if (!wait(&acc_full[accn], uint32_t(tl >> 1) & 1u)) break;
      tc_fence_after();
      const uint32_t acc = tmem + accn * N;
      const uint64_t base = tile_base(tl << 2);
#pragma unroll 1
      for (uint32_t c = 0; c < N / 32; ++c) {
        uint32_t v[32];
        tmem_ld32(acc + ((quad * 32u) << 16) + c * 32u, v);
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
        for (uint32_t j = 0; j < 8; ++j)
          stage[lane * 8 + (j ^ (lane & 7u))] = make_float4(__uint_as_float(v[4 * j]), __uint_as_float(v[4 * j + 1]),
                                                            __uint_as_float(v[4 * j + 2]), __uint_as_float(v[4 * j + 3]));
        __syncwarp();
        const uint32_t j = lane & 7u;  // float4 j of the chunk: complex elements c * 16 + 2j, + 1
#pragma unroll
        for (uint32_t i = 0; i < 8; ++i) {
          const uint32_t r = (lane >> 3) + 4 * i;
          const float4 x = stage[r * 8 + (j ^ (r & 7u))];
          const uint64_t row = base | row_off[quad * 32 + r];
          const uint32_t e = c * 16 + 2 * j;
          if (pair) {
            *reinterpret_cast<float4*>(state + (row | elem_off[e])) = x;
          } else {
            state[row | elem_off[e]] = make_float2(x.x, x.y);
            state[row | elem_off[e + 1]] = make_float2(x.z, x.w);
          }
        }
        __syncwarp();
      }
      tc_fence_before();  // the accumulator is written again two tiles later
      mbar_arrive(smem_addr(&acc_empty[accn]));
    }
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(NCOLS));
}

// Dense k-qubit unitary on CUDA cores (any precision; the targets on the low k
// physical bits): one CTA per row of 2^k amplitudes, thread b computes output b.
template <typename Real>
__global__ void dense_rows_kernel(typename ctype<Real>::c* __restrict__ state, uint64_t rows, int k,
                                  const double* __restrict__ U)
{
  using C = typename ctype<Real>::c;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* in = reinterpret_cast<C*>(smem_raw);
  const uint32_t dim = 1u << k;
  for (uint64_t r = blockIdx.x; r < rows; r += gridDim.x) {
    C* row = state + r * dim;
    for (uint32_t i = threadIdx.x; i < dim; i += blockDim.x) in[i] = row[i];
    __syncthreads();
    for (uint32_t b = threadIdx.x; b < dim; b += blockDim.x) {
      double re = 0, im = 0;
      for (uint32_t a = 0; a < dim; ++a) {
        const double ur = U[2 * (size_t(b) * dim + a)], ui = U[2 * (size_t(b) * dim + a) + 1];
        const double xr = double(in[a].x), xi = double(in[a].y);
        re += ur * xr - ui * xi;
        im += ur * xi + ui * xr;
      }
      row[b] = C{(Real)re, (Real)im};
    }
    __syncthreads();
  }
}

}  // namespace

size_t tc_w_split_floats(int k) { return size_t(2) << (2 * (k + 1)); }

size_t tc_shared_bytes(int k)
{
  const size_t K = size_t(1) << (k + 1);
  // W hi/lo + two A stages (hi/lo) of K/4 columns + the epilogue's 4 x 4 KB turn-around
  return 2 * K * K * 4 + 4 * size_t(kTcM) * (K / 4) * 4 + 4 * 32 * 32 * 4;
}

cudaError_t launch_unitary_tf32x3(void* state, int n, int k, const float* w_split, int* error_flag, int grid,
                                  const tc_layout& layout, cudaStream_t stream)
{
  if ((k != 5 && k != 6) || n < k + 7) return cudaErrorInvalidValue;
  const uint64_t rows = 1ull << (n - k);
  const size_t smem = tc_shared_bytes(k);
  cudaError_t e;
  if (k == 6) {
    e = cudaFuncSetAttribute(unitary_tf32x3_kernel<7>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
    if (e != cudaSuccess) return e;
    unitary_tf32x3_kernel<7><<<grid, kTcThreads, smem, stream>>>(static_cast<float2*>(state), rows,
                                                                  reinterpret_cast<const float4*>(w_split), error_flag, layout);
  } else {
    e = cudaFuncSetAttribute(unitary_tf32x3_kernel<6>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
    if (e != cudaSuccess) return e;
    unitary_tf32x3_kernel<6><<<grid, kTcThreads, smem, stream>>>(static_cast<float2*>(state), rows,
                                                                  reinterpret_cast<const float4*>(w_split), error_flag, layout);
  }
  return cudaGetLastError();
}

template <typename Real>
cudaError_t launch_dense_rows(void* state, int n, int k, const double* U, cudaStream_t stream)
{
  const uint64_t rows = 1ull << (n - k);
  const int threads = (1 << k) < 256 ? (1 << k) < 32 ? 32 : (1 << k) : 256;
  const unsigned grid = unsigned(rows < 148 * 16 ? rows : 148 * 16);
  dense_rows_kernel<Real><<<grid, threads, sizeof(typename ctype<Real>::c) << k, stream>>>(
    static_cast<typename ctype<Real>::c*>(state), rows, k, U);
  return cudaGetLastError();
}
template cudaError_t launch_dense_rows<double>(void*, int, int, const double*, cudaStream_t);
template cudaError_t launch_dense_rows<float>(void*, int, int, const double*, cudaStream_t);

}  // namespace rbk
