// Forest adaptation on the device: the remesh step of a time-stepping run
// without a host forest.
//
// CUP2D adapts its forest every few steps (source/Operators/AdaptTheMesh.cpp:
// 80-110): it tags blocks by a refinement criterion, Cubism's MeshAdaptation
// refines/compresses them and restores the 2:1 balance, and the pressure
// solver re-assembles its operator (ExpAMRSolver.cpp:370-376).  Here the
// criterion is the benchmark's geometry (blocks meeting the band
// { p : | |p - c| - r | <= band } of a disk are refined to the finest level),
// and the whole forest is rebuilt on the device from it:
//
//   tag      level by level from the roots: a position exists when its parent
//            was refined; it is refined when it is above the finest level and
//            meets a band, else it is a leaf (one thread per position);
//   balance  every leaf at level l >= 2 looks at its 8 face and corner
//            neighbours; a covering leaf more than one level coarser is marked
//            and split into its 4 children; rounds of descending levels run
//            until a round marks nothing (the balanced refinement of a leaf
//            set is unique, so the order of the splits does not matter);
//   order    every leaf's Morton key (its finest-level corner, bits of i and j
//            interleaved) marks a dense key array, an exclusive scan of which
//            gives each leaf its position: the leaves in Morton order.
//
// The result is the forest the host generator builds for the same geometry
// (forest.cpp build_disk_forest: same geometric test with the same rounded
// operations, same balance rule, same order); the device assembly and the
// pressure transfer then take it from there.  States live in dense per-level
// byte arrays laid out like the assembly's leaf tables.
#include <cuda_runtime.h>

#include <algorithm>

#include "kernels.hpp"

namespace cup2d {

namespace {

constexpr uint8_t kAbsent = 0, kLeaf = 1, kRefined = 2, kSplit = 3;  // kSplit: a leaf marked for splitting

__device__ __forceinline__ int64_t nx_at(const AdaptGeom& g, int l) { return (int64_t)g.bpdx << l; }
__device__ __forceinline__ int64_t ny_at(const AdaptGeom& g, int l) { return (int64_t)g.bpdy << l; }

// forest.cpp rect_meets_band with the host's rounding: separately rounded
// products and sums (no contraction into FMAs), correctly rounded sqrt.
__device__ __forceinline__ bool meets_band(double x0, double y0, double x1, double y1, double cx, double cy,
                                           double r, double band) {
  const double dx = fmax(fmax(__dadd_rn(x0, -cx), 0.0), __dadd_rn(cx, -x1));
  const double dy = fmax(fmax(__dadd_rn(y0, -cy), 0.0), __dadd_rn(cy, -y1));
  const double dmin = __dsqrt_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)));
  const double fx = fmax(fabs(__dadd_rn(x0, -cx)), fabs(__dadd_rn(x1, -cx)));
  const double fy = fmax(fabs(__dadd_rn(y0, -cy)), fabs(__dadd_rn(y1, -cy)));
  const double dmax = __dsqrt_rn(__dadd_rn(__dmul_rn(fx, fx), __dmul_rn(fy, fy)));
  return dmin <= __dadd_rn(r, band) && dmax >= __dadd_rn(r, -band);
}

__global__ void k_adapt_tag(const __grid_constant__ AdaptGeom g, const __grid_constant__ AdaptDisks D, int l,
                            uint8_t* __restrict__ state) {
  const int64_t nx = nx_at(g, l), n = nx * ny_at(g, l);
  // block size at this level: 8 * extent / (max(bpdx, bpdy) * 8 * 2^l), as forest.cpp cell_h
  const double h = __ddiv_rn(g.extent, __dmul_rn(__dmul_rn((double)max(g.bpdx, g.bpdy), 8.0), (double)(1ll << l)));
  const double bs = __dmul_rn(8.0, h);
  for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < n; p += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = p % nx, j = p / nx;
    bool exists = l == 0;
    if (!exists) exists = state[g.off[l - 1] + (j >> 1) * nx_at(g, l - 1) + (i >> 1)] == kRefined;
    uint8_t st = kAbsent;
    if (exists) {
      bool refine = false;
      if (l < g.L - 1) {
        const double x0 = __dmul_rn((double)i, bs), y0 = __dmul_rn((double)j, bs);
        const double x1 = __dadd_rn(x0, bs), y1 = __dadd_rn(y0, bs);
        for (int k = 0; k < D.n && !refine; ++k)
          refine = meets_band(x0, y0, x1, y1, D.d[k][0], D.d[k][1], D.d[k][2], D.band);
      }
      st = refine ? kRefined : kLeaf;
    }
    state[g.off[l] + p] = st;
  }
}

// Level of the leaf covering position (l, i, j), or -1 when the position is
// refined (covered by finer leaves); a leaf marked for splitting still counts.
__device__ __forceinline__ int covering_level(const AdaptGeom& g, const uint8_t* state, int l, int64_t i, int64_t j) {
  for (int q = l; q >= 0; --q) {
    const int sh = l - q;
    const uint8_t s = state[g.off[q] + (j >> sh) * nx_at(g, q) + (i >> sh)];
    if (s == kLeaf || s == kSplit) return q;
    if (s == kRefined) return -1;
  }
  return -1;
}

__global__ void k_adapt_mark(const __grid_constant__ AdaptGeom g, int l, uint8_t* __restrict__ state,
                             int* __restrict__ changed) {
  const int64_t nx = nx_at(g, l), ny = ny_at(g, l), n = nx * ny;
  for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < n; p += (int64_t)gridDim.x * blockDim.x) {
    const uint8_t s = state[g.off[l] + p];
    if (s != kLeaf && s != kSplit) continue;
    const int64_t i = p % nx, j = p / nx;
    for (int dj = -1; dj <= 1; ++dj)
      for (int di = -1; di <= 1; ++di) {
        if (!di && !dj) continue;
        int64_t ni = i + di, nj = j + dj;
        if (ni < 0 || ni >= nx) {
          if (!g.px) continue;
          ni = (ni + nx) % nx;
        }
        if (nj < 0 || nj >= ny) {
          if (!g.py) continue;
          nj = (nj + ny) % ny;
        }
        const int q = covering_level(g, state, l, ni, nj);
        if (q >= 0 && q < l - 1) {
          const int sh = l - q;
          state[g.off[q] + (nj >> sh) * nx_at(g, q) + (ni >> sh)] = kSplit;
          *changed = 1;
        }
      }
  }
}

// Splits the marked leaves of level l into their four children.
__global__ void k_adapt_split(const __grid_constant__ AdaptGeom g, int l, uint8_t* __restrict__ state) {
  const int64_t nx = nx_at(g, l), n = nx * ny_at(g, l);
  for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < n; p += (int64_t)gridDim.x * blockDim.x) {
    if (state[g.off[l] + p] != kSplit) continue;
    state[g.off[l] + p] = kRefined;
    const int64_t i = p % nx, j = p / nx, cnx = nx_at(g, l + 1);
    for (int c = 0; c < 4; ++c)
      state[g.off[l + 1] + (2 * j + (c >> 1)) * cnx + 2 * i + (c & 1)] = kLeaf;
  }
}

__device__ __forceinline__ uint64_t spread_bits(uint64_t v) {
  v &= 0xffffffffull;
  v = (v | (v << 16)) & 0x0000ffff0000ffffull;
  v = (v | (v << 8)) & 0x00ff00ff00ff00ffull;
  v = (v | (v << 4)) & 0x0f0f0f0f0f0f0f0full;
  v = (v | (v << 2)) & 0x3333333333333333ull;
  v = (v | (v << 1)) & 0x5555555555555555ull;
  return v;
}

__device__ __forceinline__ uint64_t leaf_key(const AdaptGeom& g, int l, int64_t i, int64_t j) {
  const int sh = g.L - 1 - l;
  return spread_bits((uint64_t)i << sh) | (spread_bits((uint64_t)j << sh) << 1);
}

// mark[key] = 1 for every leaf (the array is cleared before)
__global__ void k_adapt_keys(const __grid_constant__ AdaptGeom g, int l, const uint8_t* __restrict__ state,
                             int32_t* __restrict__ mark) {
  const int64_t nx = nx_at(g, l), n = nx * ny_at(g, l);
  for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < n; p += (int64_t)gridDim.x * blockDim.x)
    if (state[g.off[l] + p] == kLeaf) mark[leaf_key(g, l, p % nx, p / nx)] = 1;
}

__global__ void k_adapt_scatter(const __grid_constant__ AdaptGeom g, int l, const uint8_t* __restrict__ state,
                                const int32_t* __restrict__ rank, int64_t nb, int32_t* __restrict__ level,
                                int32_t* __restrict__ bx, int32_t* __restrict__ by, int* __restrict__ err) {
  const int64_t nx = nx_at(g, l), n = nx * ny_at(g, l);
  for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < n; p += (int64_t)gridDim.x * blockDim.x)
    if (state[g.off[l] + p] == kLeaf) {
      const int64_t i = p % nx, j = p / nx;
      const int32_t b = rank[leaf_key(g, l, i, j)];
      if (b < 0 || b >= nb) {  // cannot happen for a consistent scan; never write outside the arrays
        atomicExch(err, 1);
        continue;
      }
      level[b] = l;
      bx[b] = (int32_t)i;
      by[b] = (int32_t)j;
    }
}

unsigned grid_for(int64_t n) {
  const int64_t b = (n + 255) / 256;
  return (unsigned)(b < 4096 ? (b > 0 ? b : 1) : 4096);
}

}  // namespace

int64_t adapt_key_space(int bpdx, int bpdy, int level_max) {
  const int64_t finest = (int64_t)std::max(bpdx, bpdy) << (level_max - 1);
  int b = 0;
  while (((int64_t)1 << b) < finest) ++b;
  return (int64_t)1 << (2 * b);
}

int adapt_build(const AdaptGeom& g, const AdaptDisks& D, const AdaptScratch& sc, int64_t* nleaves,
                cudaStream_t s) {
  for (int l = 0; l < g.L; ++l)
    k_adapt_tag<<<grid_for(((int64_t)g.bpdx << l) * ((int64_t)g.bpdy << l)), 256, 0, s>>>(g, D, l, sc.state);
  // balance: rounds of descending levels until one marks nothing.  A round
  // carries the splits it causes down to the coarse levels, so two rounds
  // settle it in practice; the bound only guards the loop.
  bool settled = false;
  for (int round = 0; round < 4 * g.L + 4 && !settled; ++round) {
    if (cudaMemsetAsync(sc.changed, 0, sizeof(int), s) != cudaSuccess) return CUP2D_CUDA_ERROR;
    for (int l = g.L - 1; l >= 2; --l) {
      const int64_t n = ((int64_t)g.bpdx << l) * ((int64_t)g.bpdy << l);
      k_adapt_mark<<<grid_for(n), 256, 0, s>>>(g, l, sc.state, sc.changed);
      for (int q = l - 2; q >= 0; --q)
        k_adapt_split<<<grid_for(((int64_t)g.bpdx << q) * ((int64_t)g.bpdy << q)), 256, 0, s>>>(g, q, sc.state);
    }
    int changed = 0;
    if (cudaMemcpyAsync(&changed, sc.changed, sizeof(int), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess)
      return CUP2D_CUDA_ERROR;
    settled = changed == 0;
  }
  if (!settled) return CUP2D_BAD_MESH;
  const int64_t K = adapt_key_space(g.bpdx, g.bpdy, g.L);
  if (cudaMemsetAsync(sc.mark, 0, sizeof(int32_t) * K, s) != cudaSuccess) return CUP2D_CUDA_ERROR;
  for (int l = 0; l < g.L; ++l)
    k_adapt_keys<<<grid_for(((int64_t)g.bpdx << l) * ((int64_t)g.bpdy << l)), 256, 0, s>>>(g, l, sc.state, sc.mark);
  // rank[0..K) exclusive prefix of the marks, rank[K] their total: the leaf count
  if (launch_exclusive_scan(sc.mark, K, sc.rank, sc.scan_tmp, s) != cudaSuccess) return CUP2D_CUDA_ERROR;
  int32_t count = 0;
  if (cudaMemcpyAsync(&count, sc.rank + K, sizeof(int32_t), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
      cudaStreamSynchronize(s) != cudaSuccess)
    return CUP2D_CUDA_ERROR;
  *nleaves = count;
  return cudaGetLastError() == cudaSuccess ? CUP2D_OK : CUP2D_CUDA_ERROR;
}

int adapt_scatter(const AdaptGeom& g, const AdaptScratch& sc, int64_t nb, int32_t* level, int32_t* bx, int32_t* by,
                  cudaStream_t s) {
  if (cudaMemsetAsync(sc.changed, 0, sizeof(int), s) != cudaSuccess) return CUP2D_CUDA_ERROR;
  for (int l = 0; l < g.L; ++l)
    k_adapt_scatter<<<grid_for(((int64_t)g.bpdx << l) * ((int64_t)g.bpdy << l)), 256, 0, s>>>(
        g, l, sc.state, sc.rank, nb, level, bx, by, sc.changed);
  int err = 0;
  if (cudaGetLastError() != cudaSuccess ||
      cudaMemcpyAsync(&err, sc.changed, sizeof(int), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
      cudaStreamSynchronize(s) != cudaSuccess)
    return CUP2D_CUDA_ERROR;
  return err ? CUP2D_BAD_MESH : CUP2D_OK;
}

}  // namespace cup2d
