// The mixed form's P^-1 apply (z = P^-1 p per 8x8 block, FP32 operands,
// split-TF32 accuracy) on the 5th-generation tensor cores: tcgen05.mma with
// operands in shared memory and the accumulator in tensor memory (TMEM).
// The role of the reference's cublasDgemm(T, N, 64, Nblocks, 64) with P_inv
// (source/Poisson/BiCGSTAB.cu:520,545), in the precision of the mixed form.
//
// One CTA of 128 threads (one warpgroup, the 128 TMEM lanes) walks tiles of
// kN = 32 blocks.  Per tile, D (128 x kN, FP32, in TMEM) = A x B with
//   A = [P_hi ; P_lo]   128 x 64, the TF32 split of P (rows 0-63 hi, 64-127 lo)
//   B = x_hi, then x_lo  kN x 64, the TF32 split of the tile's p
// accumulated over K = 64 in steps of 8 (16 MMAs of M=128, N=32, K=8), so
// D[i] = P_hi (x_hi + x_lo) and D[64+i] = P_lo (x_hi + x_lo); z = D[i] +
// D[64+i] is P x to FP32 accuracy (the P_lo x_lo term is kept).  One thread
// issues the MMAs and commits them to an mbarrier; after the (bounded) wait
// every warp reads its 32 TMEM lanes with tcgen05.ld.
//
// Shared-memory operands use the no-swizzle K-major canonical layout: 8-row
// x 16-byte core matrices, rows 16 bytes apart inside a core matrix, the two
// K-halves of an 8-wide K step LBO = 128 bytes apart, 8-row groups SBO =
// 2048 bytes apart (all 16 K-chunks of a row group are contiguous).
//
// The plain form of this apply is k_precond32 (mma.sync m16n8k8 TF32, the
// one the solver's passes use); both are exported so that they can be timed
// side by side.  A wait that outlives 2 s of globaltimer raises *err, and
// the CTA still frees its tensor memory before leaving.
#include <cuda_runtime.h>

#include <algorithm>

#include "kernels.hpp"

namespace cup2d {

namespace {

constexpr int kTcThreads = 128;
constexpr int kN = 32;                     // blocks per tile (MMA N)
constexpr uint32_t kTmemCols = 32;         // accumulator columns (power of 2, >= 32)
constexpr unsigned long long kTcWaitNs = 2000000000ull;

struct TcSmem {
  alignas(1024) uint32_t a[128 * 64];      // [P_hi; P_lo], canonical K-major
  alignas(1024) uint32_t bhi[kN * 64];     // x_hi, canonical K-major
  alignas(1024) uint32_t blo[kN * 64];     // x_lo
  alignas(16) float lo_rows[64][kN + 1];   // D rows 64..127 handed to the warps of rows 0..63
  alignas(8) unsigned long long bar;
  uint32_t tmem_base;
};

__device__ __forceinline__ uint32_t smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ uint32_t tf32_bits(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return r;
}

// word offset of element (row r, k) in the canonical K-major layout
__device__ __forceinline__ int canon(int r, int k) { return (r >> 3) * 512 + (k >> 2) * 32 + (r & 7) * 4 + (k & 3); }

// shared-memory matrix descriptor: no swizzle, LBO = 128 B, SBO = 2048 B,
// descriptor version 1 (sm_100)
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr) {
  uint64_t d = 0;
  d |= (uint64_t)((addr >> 4) & 0x3FFFu);
  d |= (uint64_t)(128u >> 4) << 16;
  d |= (uint64_t)(2048u >> 4) << 32;
  d |= (uint64_t)1 << 46;
  return d;
}

// instruction descriptor: D FP32, A and B TF32, both K-major, N = kN, M = 128
constexpr uint32_t kIdesc = (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(kN >> 3) << 17) | ((128u >> 4) << 24);

__device__ __forceinline__ void mma_tf32(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem_d),
      "l"(da), "l"(db), "r"(kIdesc), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}

__device__ __forceinline__ void mbar_wait_bounded(unsigned long long* bar, unsigned parity, int* ok) {
  const unsigned long long t0 = globaltimer_ns();
  for (;;) {
    unsigned done;
    asm volatile(
        "{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3; selp.u32 %0, 1, 0, p; }"
        : "=r"(done)
        : "r"(smem_addr(bar)), "r"(parity), "r"(10000u)
        : "memory");
    if (done) return;
    if (globaltimer_ns() - t0 > kTcWaitNs) {
      *ok = 0;
      return;
    }
  }
}

extern __shared__ __align__(1024) unsigned char g_tc_smem[];

__global__ void __launch_bounds__(kTcThreads) k_precond32_tc(const float* __restrict__ P32, int nb,
                                                             const float* __restrict__ p, float* __restrict__ z,
                                                             int* __restrict__ err) {
  TcSmem& sm = *reinterpret_cast<TcSmem*>((reinterpret_cast<uintptr_t>(g_tc_smem) + 1023) & ~uintptr_t(1023));
  const int tid = threadIdx.x, w = tid >> 5, lane = tid & 31;
  // A = [P_hi ; P_lo]
  for (int q = tid; q < 64 * 64; q += kTcThreads) {
    const int r = q >> 6, k = q & 63;
    const float v = __ldg(P32 + q);
    const uint32_t hi = tf32_bits(v);
    sm.a[canon(r, k)] = hi;
    sm.a[canon(r + 64, k)] = tf32_bits(v - __uint_as_float(hi));
  }
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(&sm.bar)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (w == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(&sm.tmem_base)),
                 "r"(kTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = sm.tmem_base;
  const uint64_t da0 = smem_desc(smem_addr(sm.a));
  const uint64_t dh0 = smem_desc(smem_addr(sm.bhi));
  const uint64_t dl0 = smem_desc(smem_addr(sm.blo));
  unsigned phase = 0;
  bool failed = false;
  for (int tb = blockIdx.x * kN; tb < nb; tb += gridDim.x * kN) {
    const int nvalid = min(kN, nb - tb);
    // B: the tile's p split into TF32 hi / lo (zero past the last block)
    for (int q = tid; q < kN * 64; q += kTcThreads) {
      const int n = q >> 6, k = q & 63;
      const float v = n < nvalid ? p[(size_t)(tb + n) * kBLEN + k] : 0.f;
      const uint32_t hi = tf32_bits(v);
      sm.bhi[canon(n, k)] = hi;
      sm.blo[canon(n, k)] = tf32_bits(v - __uint_as_float(hi));
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // generic-proxy writes -> tensor core
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (tid == 0) {
      // an 8-wide K step advances the start address by two 128-byte K-chunks
#pragma unroll
      for (int kk = 0; kk < 8; ++kk) mma_tf32(tmem, da0 + (uint64_t)(kk * 16), dh0 + (uint64_t)(kk * 16), kk > 0);
#pragma unroll
      for (int kk = 0; kk < 8; ++kk) mma_tf32(tmem, da0 + (uint64_t)(kk * 16), dl0 + (uint64_t)(kk * 16), 1u);
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                       smem_addr(&sm.bar))
                   : "memory");
    }
    int ok = 1;
    mbar_wait_bounded(&sm.bar, phase, &ok);
    phase ^= 1u;
    if (!__syncthreads_and(ok)) {  // the MMAs did not complete in time: leave the loop together
      failed = true;
      break;
    }
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    // warp w reads TMEM lanes 32w..32w+31 (rows of D), kN columns (blocks)
    uint32_t v[kN];
    const uint32_t taddr = tmem + ((uint32_t)(32 * w) << 16);
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
        : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
          "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]),
          "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]),
          "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
    // rows 64..127 (the P_lo part) to shared memory, then rows 0..63 add them
    if (w >= 2) {
#pragma unroll
      for (int n = 0; n < kN; ++n) sm.lo_rows[32 * (w - 2) + lane][n] = __uint_as_float(v[n]);
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (w < 2) {
      const int i = 32 * w + lane;
#pragma unroll
      for (int n = 0; n < kN; ++n)
        if (n < nvalid) z[(size_t)(tb + n) * kBLEN + i] = __uint_as_float(v[n]) + sm.lo_rows[i][n];
    }
    __syncthreads();  // lo_rows and B are rewritten by the next tile
  }
  if (failed) {
    // report, give the MMAs in flight one more bounded wait, then free TMEM
    if (tid == 0) atomicExch(err, 1);
    int ok = 1;
    mbar_wait_bounded(&sm.bar, phase ^ 1u, &ok);
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (w == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols) : "memory");
}

}  // namespace

cudaError_t launch_precond32_tc(const float* P32, int64_t nb, const float* p, float* z, int* err, cudaStream_t s) {
  if (nb <= 0) return cudaSuccess;
  const int bytes = (int)sizeof(TcSmem) + 1024;  // + alignment slack
  cudaError_t e = cudaFuncSetAttribute(k_precond32_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  if (e != cudaSuccess) return e;
  int dev = 0, sms = 0, per_sm = 0;
  if ((e = cudaGetDevice(&dev)) != cudaSuccess ||
      (e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess ||
      (e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_precond32_tc, kTcThreads, bytes)) != cudaSuccess)
    return e;
  const int64_t tiles = (nb + kN - 1) / kN;
  const int grid = (int)std::min<int64_t>(tiles, (int64_t)sms * std::max(1, per_sm));
  k_precond32_tc<<<grid, kTcThreads, bytes, s>>>(P32, (int)nb, p, z, err);
  return cudaGetLastError();
}

}  // namespace cup2d
