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
//   tile i    the 5-point rows from shared memory with the solver's lane
//             layout and register stencil (spmv.cuh), so both SpMVs give
//             the same bits; a face whose neighbour is in the same tile
//             reads it there.
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
  // halos of tile i from its staged table: per block 16 column values (x
  // faces) and the 16-byte pieces of two rows (y faces), for neighbours
  // outside the tile
  auto issue_halos = [&](int i) {
    if (i >= ntiles) return;
    const int t0 = tile_start(i), tn = tile_len(i);
    auto outside = [&](int nbid) { return nbid >= 0 && (unsigned)(nbid - t0) >= (unsigned)tn; };
    for (int q = tid; q < tn * 16; q += kThreads) {
      const int bl = q >> 4, k = q & 15;
      const int4 nb = sm.nbr[i % kStages][bl];
      T(*h)[kBS] = sm.halo[i % kHaloSlots][bl];
      const int f = k >> 3, r = k & 7;  // x face f, row r
      const int nx = f == 0 ? nb.x : nb.y;
      if (outside(nx)) cp_async<sizeof(T)>(&h[f][r], x + (size_t)nx * kBLEN + r * kBS + (f == 0 ? kBS - 1 : 0));
      if (k < 2 * ROWC) {
        const int g = k / ROWC, piece = k % ROWC;  // y face 2 + g
        const int ny = g == 0 ? nb.z : nb.w;
        if (outside(ny))
          cp_async<16>(&h[2 + g][piece * (16 / (int)sizeof(T))],
                       x + (size_t)ny * kBLEN + (g == 0 ? (kBS - 1) * kBS : 0) + piece * (16 / (int)sizeof(T)));
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
      const bool valid = bl < n;
      ChunkGather<T> g;
      g.nb = valid ? sm.nbr[i % kStages][bl] : make_int4(kWall, kWall, kWall, kWall);
      g.xm = g.xp = T(0);
#pragma unroll
      for (int j = 0; j < V; ++j) g.z[j] = g.ym[j] = g.yp[j] = T(0);
      if (valid) {
        const T(*h)[kBS] = sm.halo[i % kHaloSlots][bl];
        auto in_tile = [&](int nbid) { return (unsigned)(nbid - blk0) < (unsigned)n; };
        lds<V>(xs + bl * kBLEN + L.cell0, g.z);
        if (L.ix0 == 0 && g.nb.x >= 0)
          g.xm = in_tile(g.nb.x) ? xs[(g.nb.x - blk0) * kBLEN + L.iy * kBS + kBS - 1] : h[0][L.iy];
        if (L.ix0 + V == kBS && g.nb.y >= 0)
          g.xp = in_tile(g.nb.y) ? xs[(g.nb.y - blk0) * kBLEN + L.iy * kBS] : h[1][L.iy];
        if (L.iy == 0 && g.nb.z >= 0)
          lds<V>(in_tile(g.nb.z) ? xs + (g.nb.z - blk0) * kBLEN + (kBS - 1) * kBS + L.ix0 : &h[2][L.ix0], g.ym);
        if (L.iy == kBS - 1 && g.nb.w >= 0)
          lds<V>(in_tile(g.nb.w) ? xs + (g.nb.w - blk0) * kBLEN + L.ix0 : &h[3][L.ix0], g.yp);
      }
      T out[V];
      stencil_chunk<T>(g, L, out);
      if (!valid) continue;
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
    __syncthreads();  // the buffers of tile i are refilled from the next step on
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
