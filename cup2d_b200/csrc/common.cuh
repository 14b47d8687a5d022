// Device-side building blocks shared by the Poisson kernels (sm_100a).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/cup2d_poisson.h"

namespace cup2d {

constexpr int kBS = 8;          // cells per block side (CUP2D _BS_)
constexpr int kBLEN = 64;       // cells per block
constexpr unsigned kFull = 0xffffffffu;

// Face codes stored per block and face in the mesh's neighbour table.
constexpr int32_t kWall = -1;      // non-periodic domain edge: no flux
constexpr int32_t kExplicit = -2;  // coarse/fine face: rows stored explicitly

// Device image of an assembled AMR Laplacian (block-structured).
//   nbr[4*b+f]  : same-level neighbour block across face f (0 Xm,1 Xp,2 Ym,3 Yp),
//                 or kWall / kExplicit
//   xmask[b]    : bit c set <=> row of cell c is stored explicitly
//   xbase[b]    : index of block b's first explicit row
//   xptr[R+1], xcol[nnz], xval[nnz] (+ xval32): explicit rows, CSR, columns
//                 ascending, values as the reference's row accumulation
struct MeshView {
  int64_t nb;
  const int32_t* __restrict__ nbr;
  const unsigned long long* __restrict__ xmask;
  const int32_t* __restrict__ xbase;
  const int32_t* __restrict__ xptr;
  const int32_t* __restrict__ xcol;
  const double* __restrict__ xval;
  const float* __restrict__ xval32;
  const double* __restrict__ hblk;     // cell size per block
  const int32_t* __restrict__ rowcell; // [R] cell index of each explicit row
  int64_t R;                           // explicit rows
};

__device__ __forceinline__ unsigned long long globaltimer_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ int ld_volatile_s32(const int* p) {
  int v;
  asm volatile("ld.volatile.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ void red_release_add_u32(unsigned* p, unsigned v) {
  asm volatile("red.release.gpu.global.add.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Barrier over `nparties` CTAs built on a monotonically increasing arrival
// counter: the k-th barrier of a launch waits until the counter reaches
// k*nparties.  The wait is bounded: past `deadline_ns` (globaltimer) or when
// another CTA raised `abort_flag`, the CTA raises the flag itself and the
// barrier returns false; callers then leave the kernel.  Every thread of the
// CTA must call it (it contains __syncthreads).
//
// Profiling (the device-side counterpart of CUP2D's DeviceProfiler regions,
// source/Utils/DeviceProfiler.cuh): when `prof` is set, thread 0 adds to
// prof[(cta*kProfPhases + phase)*2 + {0,1}] the ns spent computing the phase
// that ends at this barrier and the ns spent waiting in it.
constexpr int kProfPhases = 10;

struct GridBarrier {
  unsigned* counter;
  int* abort_flag;
  unsigned nparties;
  unsigned long long deadline_ns;
  unsigned epoch;  // barriers passed so far by this CTA
  unsigned long long* prof;
  unsigned long long last;  // thread 0: when it left the previous barrier

  // Called by all threads of the CTA; only thread 0 reads or updates the
  // fields.
  __device__ __forceinline__ bool sync(int* smem_flag, int phase = 0) {
    __syncthreads();
    if (threadIdx.x == 0) {
      ++epoch;
      int ok = 1;
      unsigned long long t_arrive = 0;
      if (prof) t_arrive = globaltimer_ns();
      __threadfence();
      red_release_add_u32(counter, 1u);
      const unsigned target = epoch * nparties;
      unsigned spins = 0;
      // the deadline bounds the whole launch: checked at every barrier (a
      // register read), the abort flag only while spinning
      if (globaltimer_ns() > deadline_ns) {
        atomicExch(abort_flag, 1);
        ok = 0;
      }
      while (ok && ld_acquire_u32(counter) < target) {
        if ((++spins & 63u) == 0) {
          if (ld_volatile_s32(abort_flag) != 0 || globaltimer_ns() > deadline_ns) {
            atomicExch(abort_flag, 1);
            ok = 0;
            break;
          }
        }
        if (spins > 256) __nanosleep(64);
      }
      __threadfence();
      if (prof) {
        const unsigned long long t_depart = globaltimer_ns();
        unsigned long long* p = prof + ((size_t)blockIdx.x * kProfPhases + phase) * 2;
        p[0] += t_arrive - last;
        p[1] += t_depart - t_arrive;
        last = t_depart;
      }
      *smem_flag = ok;
    }
    __syncthreads();
    return *smem_flag != 0;
  }
};

__host__ __device__ __forceinline__ int64_t imin64(int64_t a, int64_t b) { return a < b ? a : b; }

// Start of part k of n equal parts of [0, total): 64-bit product, 32-bit
// result (cell and block indices of one problem fit in 31 bits).
__device__ __forceinline__ int share(long long total, unsigned k, unsigned n) {
  return (int)(total * (long long)k / (long long)n);
}

template <class T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
  return v;
}

template <class T>
__device__ __forceinline__ T warp_max(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(kFull, v, o));
  return v;
}

// FP64 tensor-core MMA, D(8x8) += A(8x4, row) * B(4x8, col).
// Lane l holds A[l/4][l%4], B[l%4][l/4], and C[l/4][2*(l%4) + {0,1}].
__device__ __forceinline__ void dmma_884(double& d0, double& d1, double a, double b) {
  asm volatile(
      "mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
      : "+d"(d0), "+d"(d1)
      : "d"(a), "d"(b));
}

}  // namespace cup2d
