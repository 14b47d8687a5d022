// Operator apply y = A x with tiles staged in shared memory by the copy
// engines: the standalone SpMV of the library (the role of the reference's
// hd_cusparseSpMV on the assembled CSR, source/Poisson/BiCGSTAB.cu), built on
// the block structure instead of a CSR of the whole matrix.
//
// A persistent CTA walks its contiguous range of blocks in tiles of 8 KB
// (16 FP64 or 32 FP32 blocks) through a pipeline of kStages tiles:
//   tile i+D  (D = kStages - 1) the cells (one bulk copy, cp.async.bulk,
//             completing on an mbarrier) and the neighbour table and
//             explicit-row masks of its blocks (cp.async);
//   tile i+2  the halos: the edge row or column of every same-level
//             neighbour outside the tile across each face (cp.async,
//             addresses from the table staged earlier);
//   tile i    the 5-point rows from shared memory in the solver's 16-byte
//             lane layout (spmv.cuh): a lane's cells and the rows above and
//             below are 16-byte shared loads, the neighbours across a face
//             come from the same tile or the halo (address chosen without a
//             branch); summed left, right, below, above and minus n z as the
//             solver's SpMV does, so both give the same bits.
// The explicit (coarse/fine) rows follow, CSR, as in the solver's passes.
//
// Every wait on a bulk copy is bounded (2 s of globaltimer): past it the CTA
// raises *err, waits (bounded) for its copies still in flight and returns.
#include <cuda_runtime.h>

#include <algorithm>

#include "kernels.hpp"
#include "spmv.cuh"

namespace cup2d {

namespace {

#ifndef CUP2D_STAGED_TILE_BYTES
#define CUP2D_STAGED_TILE_BYTES 8192
#endif
#ifndef CUP2D_STAGED_STAGES
#define CUP2D_STAGED_STAGES 4
#endif
constexpr int kTileBytes = CUP2D_STAGED_TILE_BYTES;  // cells per tile (8 KB: 16 FP64 or 32 FP32 blocks)
constexpr int kStages = CUP2D_STAGED_STAGES;         // cell tiles staged: i .. i+kStages-1
constexpr int kHaloSlots = 3;                        // halos staged: i, i+1, i+2
static_assert(kStages >= 4, "the halos of tile i+2 need the table of tile i+2 one step ahead");
constexpr int kThreads = 256;
constexpr unsigned kSuspendNs = 20000;                // try_wait suspend hint
constexpr unsigned long long kWaitLimitNs = 2000000000ull;  // bound of one wait

template <class T>
struct StagedSmem {
  static constexpr int kTB = kTileBytes / (kBLEN * (int)sizeof(T));  // blocks per tile
  alignas(128) T x[kStages][kTB * kBLEN];
  alignas(16) T halo[kHaloSlots][kTB][4][kBS];  // faces: 0 Xm (col 7 of the left block), 1 Xp (col 0), 2 Ym (row 7), 3 Yp (row 0)
  alignas(16) int4 nbr[kStages][kTB];
  alignas(16) unsigned long long mask[kStages][kTB];
  alignas(8) unsigned long long bar[kStages];
};

__device__ __forceinline__ uint32_t saddr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(unsigned long long* bar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(saddr(bar)) : "memory");
}

__device__ __forceinline__ void fence_barrier_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// One thread: a bulk copy of `bytes` (a multiple of 16, both ends 16-byte
// aligned) completing on `bar`.
__device__ __forceinline__ void bulk_load(void* dst, const void* src, unsigned bytes, unsigned long long* bar) {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(saddr(bar)), "r"(bytes) : "memory");
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   saddr(dst)),
               "l"(src), "r"(bytes), "r"(saddr(bar))
               : "memory");
}

// Wait for the phase of `bar` with this parity: try_wait suspends the thread
// until the phase completes or the hint (ns) runs out, so the wait costs a few
// instructions per microsecond.  Gives up after 2 s (globaltimer).
__device__ __forceinline__ bool mbar_wait(unsigned long long* bar, unsigned parity) {
  unsigned long long deadline = 0;
  for (;;) {
    unsigned ok;
    asm volatile(
        "{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3; selp.u32 %0, 1, 0, p; }"
        : "=r"(ok)
        : "r"(saddr(bar)), "r"(parity), "r"(kSuspendNs)
        : "memory");
    if (ok) return true;
    __nanosleep(64);
    const unsigned long long now = globaltimer_ns();
    if (deadline == 0) deadline = now + kWaitLimitNs;
    else if (now > deadline) return false;
  }
}

// N consecutive values from shared memory as one 16-byte vector.
template <int N, class T>
__device__ __forceinline__ void lds(const T* p, T (&v)[N]) {
  static_assert(N * sizeof(T) == 16, "one 16-byte vector");
  if constexpr (sizeof(T) == 4) {
    const float4 a = *reinterpret_cast<const float4*>(p);
    v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w;
  } else {
    const double2 a = *reinterpret_cast<const double2*>(p);
    v[0] = a.x; v[1] = a.y;
  }
}

template <int B>
__device__ __forceinline__ void cp_async(void* dst, const void* src) {
  if constexpr (B == 16)
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(saddr(dst)), "l"(src) : "memory");
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], %2;" ::"r"(saddr(dst)), "l"(src), "n"(B) : "memory");
}

__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait_group() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

extern __shared__ __align__(128) unsigned char smem_raw[];

template <class T>
__global__ void __launch_bounds__(kThreads) k_apply_staged(MeshView M, const T* __restrict__ x,
                                                           T* __restrict__ y, int* __restrict__ err) {
  constexpr int ROWC = kBS * (int)sizeof(T) / 16;  // 16-byte pieces of a row
  constexpr int V = Lane<T>::V, CB = Lane<T>::CB;  // cells per lane, blocks per warp chunk
  constexpr int kTB = StagedSmem<T>::kTB;
  constexpr int D = kStages - 1;
  StagedSmem<T>& sm = *reinterpret_cast<StagedSmem<T>*>(smem_raw);
  const int tid = threadIdx.x, w = tid >> 5;
  const Lane<T> L(tid & 31);
  const int b0 = share(M.nb, blockIdx.x, gridDim.x), b1 = share(M.nb, blockIdx.x + 1, gridDim.x);
  const int ntiles = (b1 - b0 + kTB - 1) / kTB;
  auto tile_start = [&](int i) { return b0 + i * kTB; };
  auto tile_len = [&](int i) { return min(kTB, b1 - tile_start(i)); };

  if (tid == 0) {
    for (int s = 0; s < kStages; ++s) mbar_init(&sm.bar[s]);
    fence_barrier_init();
  }
  __syncthreads();

  auto issue_cells = [&](int i) {  // thread 0
    if (i < ntiles)
      bulk_load(sm.x[i % kStages], x + (size_t)tile_start(i) * kBLEN,
                (unsigned)(tile_len(i) * kBLEN * sizeof(T)), &sm.bar[i % kStages]);
  };
  auto issue_tables = [&](int i) {
    if (i < ntiles && tid < tile_len(i)) {
      const int blk = tile_start(i) + tid;
      cp_async<16>(&sm.nbr[i % kStages][tid], M.nbr + 4 * (size_t)blk);
      cp_async<8>(&sm.mask[i % kStages][tid], M.xmask + blk);
    }
  };
  // halos of tile i from its staged table, one thread per (block, face)
  // whose neighbour is outside the tile: 8 column values for an x face, the
  // 16-byte pieces of a row for a y face
  auto issue_halos = [&](int i) {
    if (i >= ntiles) return;
    const int t0 = tile_start(i), tn = tile_len(i);
    for (int q = tid; q < tn * 4; q += kThreads) {
      const int bl = q >> 2, f = q & 3;
      const int4 nb = sm.nbr[i % kStages][bl];
      const int nbid = f == 0 ? nb.x : f == 1 ? nb.y : f == 2 ? nb.z : nb.w;
      if (nbid < 0 || (unsigned)(nbid - t0) < (unsigned)tn) continue;
      T* h = sm.halo[i % kHaloSlots][bl][f];
      const T* src = x + (size_t)nbid * kBLEN;
      if (f < 2) {
        src += f == 0 ? kBS - 1 : 0;
#pragma unroll
        for (int r = 0; r < kBS; ++r) cp_async<sizeof(T)>(h + r, src + r * kBS);
      } else {
        src += f == 2 ? (kBS - 1) * kBS : 0;
#pragma unroll
        for (int piece = 0; piece < ROWC; ++piece)
          cp_async<16>(h + piece * (16 / (int)sizeof(T)), src + piece * (16 / (int)sizeof(T)));
      }
    }
  };

  // prologue: cells and tables of tiles 0 .. D-1, halos of tiles 0 and 1
  for (int j = 0; j < D; ++j) issue_tables(j);
  cp_async_commit();
  if (tid == 0)
    for (int j = 0; j < D; ++j) issue_cells(j);
  cp_async_wait_all();
  __syncthreads();
  issue_halos(0);
  cp_async_commit();
  issue_halos(1);
  cp_async_commit();

  int i = 0;
  bool ok = true;
  for (; i < ntiles; ++i) {
    // every copy group but the newest (the halos of tile i+1) has landed:
    // the halos of tile i and the tables up to tile i+D-1
    cp_async_wait_group<1>();
    __syncthreads();
    issue_tables(i + D);
    cp_async_commit();
    issue_halos(i + 2);
    cp_async_commit();
    // one thread issues the next cells and waits for this tile's; the CTA
    // barrier then hands the tile to every thread
    if (tid == 0) {
      issue_cells(i + D);
      ok = mbar_wait(&sm.bar[i % kStages], (unsigned)(i / kStages) & 1u);
    }
    if (!__syncthreads_and(ok)) break;
    const T* xs = sm.x[i % kStages];
    const int n = tile_len(i), blk0 = tile_start(i);
    T* yt = y + (size_t)blk0 * kBLEN;
    for (int c = w; c < (n + CB - 1) / CB; c += kThreads / 32) {
      const int bl = c * CB + L.bl;
      if (bl >= n) continue;
      const int4 nb = sm.nbr[i % kStages][bl];
      const T(*h)[kBS] = sm.halo[i % kHaloSlots][bl];
      const T* xb = xs + bl * kBLEN;
      auto in_tile = [&](int nbid) { return (unsigned)(nbid - blk0) < (unsigned)n; };
      T z[V], dn[V], up[V];
      lds<V>(xb + L.cell0, z);
      // neighbours: inside the block from shared memory, across a face from
      // the same tile or the halo (address chosen, no branch), absent -> 0
      const bool has_l = L.ix0 > 0 || nb.x >= 0, has_r = L.ix0 + V < kBS || nb.y >= 0;
      const bool has_d = L.iy > 0 || nb.z >= 0, has_u = L.iy < kBS - 1 || nb.w >= 0;
      const T* pl = L.ix0 > 0 ? xb + L.cell0 - 1
                              : (in_tile(nb.x) ? xs + (nb.x - blk0) * kBLEN + L.iy * kBS + kBS - 1 : &h[0][L.iy]);
      const T* pr = L.ix0 + V < kBS ? xb + L.cell0 + V
                                    : (in_tile(nb.y) ? xs + (nb.y - blk0) * kBLEN + L.iy * kBS : &h[1][L.iy]);
      const T* pd = L.iy > 0 ? xb + L.cell0 - kBS
                             : (in_tile(nb.z) ? xs + (nb.z - blk0) * kBLEN + (kBS - 1) * kBS + L.ix0 : &h[2][L.ix0]);
      const T* pu = L.iy < kBS - 1 ? xb + L.cell0 + kBS
                                   : (in_tile(nb.w) ? xs + (nb.w - blk0) * kBLEN + L.ix0 : &h[3][L.ix0]);
      const T vl = has_l ? *pl : T(0), vr = has_r ? *pr : T(0);
      lds<V>(pd, dn);
      lds<V>(pu, up);
      T out[V];
#pragma unroll
      for (int j = 0; j < V; ++j) {
        T a = T(0);
        int cnt = 0;
        if (j > 0) { a += z[j - 1]; cnt++; } else if (has_l) { a += vl; cnt++; }
        if (j < V - 1) { a += z[j + 1]; cnt++; } else if (has_r) { a += vr; cnt++; }
        if (has_d) { a += dn[j]; cnt++; }
        if (has_u) { a += up[j]; cnt++; }
        out[j] = a - T(cnt) * z[j];
      }
      const unsigned mk = (unsigned)(sm.mask[i % kStages][bl] >> L.cell0) & ((1u << V) - 1u);
      T* yo = yt + bl * kBLEN + L.cell0;
      if (mk == 0u) {
        stv<V>(yo, out);
      } else {
#pragma unroll
        for (int j = 0; j < V; ++j)
          if (!((mk >> j) & 1u)) yo[j] = out[j];
      }
    }
    // no barrier here: the next step's first barrier orders every read of
    // tile i before its buffers are refilled
  }
  if (i < ntiles) {
    // a bulk copy did not complete in time: report, let the copies still in
    // flight land (bounded) and leave
    if (tid == 0) {
      atomicExch(err, 1);
      for (int j = i; j < ntiles && j <= i + D; ++j)
        (void)mbar_wait(&sm.bar[j % kStages], (unsigned)(j / kStages) & 1u);
    }
    cp_async_wait_all();
    __syncthreads();
    return;
  }
  cp_async_wait_all();

  // explicit rows
  const int r0 = share(M.R, blockIdx.x, gridDim.x), r1 = share(M.R, blockIdx.x + 1, gridDim.x);
  const T* __restrict__ vals = row_vals<T>(M);
  for (int r = r0 + tid; r < r1; r += kThreads) {
    const int k0 = __ldg(M.xptr + r), k1 = __ldg(M.xptr + r + 1);
    T acc = T(0);
#pragma unroll 4
    for (int k = k0; k < k1; ++k) acc += __ldg(vals + k) * ldcg(x + __ldg(M.xcol + k));
    y[__ldg(M.rowcell + r)] = acc;
  }
}

template <class T>
int staged_grid(int dev) {
  static int cap[2][64] = {};
  int& c = cap[sizeof(T) == 8][dev & 63];
  if (c == 0) {
    int sms = 0, per_sm = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaFuncSetAttribute(k_apply_staged<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)sizeof(StagedSmem<T>));
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_apply_staged<T>, kThreads, sizeof(StagedSmem<T>));
    c = std::max(1, sms * std::max(1, per_sm));
  }
  return c;
}

template <class T>
cudaError_t launch_staged(const MeshView& M, const T* x, T* y, int* err, cudaStream_t s) {
  if (M.nb <= 0) return cudaSuccess;
  int dev = 0;
  cudaGetDevice(&dev);
  // at least two tiles per CTA, so that the pipeline has something to overlap
  constexpr int kTB = StagedSmem<T>::kTB;
  const int64_t ctas = std::min<int64_t>((M.nb + 2 * kTB - 1) / (2 * kTB), staged_grid<T>(dev));
  k_apply_staged<T><<<(unsigned)ctas, kThreads, sizeof(StagedSmem<T>), s>>>(M, x, y, err);
  return cudaGetLastError();
}

}  // namespace

cudaError_t launch_spmv64(const MeshView& M, const double* x, double* y, int* err, cudaStream_t s) {
  return launch_staged<double>(M, x, y, err, s);
}

cudaError_t launch_spmv32(const MeshView& M, const float* x, float* y, int* err, cudaStream_t s) {
  return launch_staged<float>(M, x, y, err, s);
}

}  // namespace cup2d
