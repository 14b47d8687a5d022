// Device-side steps around the solve in a time-stepping loop:
//   * the right-hand side of the synthetic pressure problem, evaluated on the
//     device from its Fourier coefficients (the role of CUP2D's
//     updatePressureRHS, source/Operators/PressureSingle.cpp:324-456: the
//     divergence of a velocity field by central differences, 0.5 h (du + dv)
//     with the reference's dt = 1 scaling), made zero-sum for the Neumann
//     walls as ExpAMRSolver::solve expects (source/Poisson/ExpAMRSolver.cpp);
//   * the transfer of a cell field (the pressure, the warm start of the next
//     solve) from one forest to the next after the mesh adapts, the role of
//     Cubism's refinement/compression of blocks in MeshAdaptation.
//
// Both are plain streaming kernels: one thread per cell.
#include <cuda_runtime.h>

#include "kernels.hpp"

namespace cup2d {

namespace {

constexpr int kRhsThreads = 256;  // 4 blocks of 64 cells per CTA

// Velocity component `comp` of the Fourier field at (x, y): the modes in the
// order of the host generator (ky outer, kx inner, kx = 0 only for ky > 0,
// |k|^2 <= kmax^2), amplitude |k|^-2, coefficients coef[4q + 2 comp + {0,1}]
// for the cosine and sine of k.(x, y).
__device__ double fourier_velocity(double x, double y, int comp, int kmax, double wx, double wy,
                                   const double* __restrict__ coef) {
  double cx[kMaxFourierK + 1], sx[kMaxFourierK + 1];
  for (int k = 0; k <= kmax; ++k) sincos(wx * (double)k * x, &sx[k], &cx[k]);
  double acc = 0.0;
  int q = 0;
  for (int ky = -kmax; ky <= kmax; ++ky) {
    double sy, cy;
    sincos(wy * (double)ky * y, &sy, &cy);
    for (int kx = 0; kx <= kmax; ++kx) {
      if (kx == 0 && ky <= 0) continue;
      const int k2 = kx * kx + ky * ky;
      if (k2 > kmax * kmax) continue;
      const double c = cx[kx] * cy - sx[kx] * sy;
      const double s = sx[kx] * cy + cx[kx] * sy;
      const double a = coef[4 * q + 2 * comp], b = coef[4 * q + 2 * comp + 1];
      acc += (1.0 / (double)k2) * (a * c + b * s);
      ++q;
    }
  }
  return acc;
}

__global__ void __launch_bounds__(kRhsThreads) k_rhs_fourier(ForestView F, int kmax, int nm,
                                                             const double* __restrict__ coef_g,
                                                             double* __restrict__ b, double* __restrict__ partial) {
  extern __shared__ double coef[];  // [4 nm]
  for (int i = threadIdx.x; i < 4 * nm; i += blockDim.x) coef[i] = coef_g[i];
  __syncthreads();
  const int64_t cell = (int64_t)blockIdx.x * kRhsThreads + threadIdx.x;
  double v = 0.0;
  if (cell < F.nb * kBLEN) {
    const int64_t blk = cell >> 6;
    const int c = (int)(cell & 63), ix = c & 7, iy = c >> 3;
    const double h = F.h0 / (double)(1ll << F.level[blk]);
    const double Lx = F.bpdx * 8.0 * F.h0, Ly = F.bpdy * 8.0 * F.h0;
    const double wx = 2.0 * M_PI / Lx, wy = 2.0 * M_PI / Ly;
    const double x = ((double)F.bx[blk] * 8 + ix + 0.5) * h;
    const double y = ((double)F.by[blk] * 8 + iy + 0.5) * h;
    const double du = fourier_velocity(x + h, y, 0, kmax, wx, wy, coef) -
                      fourier_velocity(x - h, y, 0, kmax, wx, wy, coef);
    const double dv = fourier_velocity(x, y + h, 1, kmax, wx, wy, coef) -
                      fourier_velocity(x, y - h, 1, kmax, wx, wy, coef);
    v = 0.5 * h * (du + dv);
    b[cell] = v;
  }
  // per-CTA partial sum, fixed order
  __shared__ double ws[kRhsThreads / 32];
  v = warp_sum(v);
  if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int w = 0; w < kRhsThreads / 32; ++w) s += ws[w];
    partial[blockIdx.x] = s;
  }
}

// One CTA: the mean of the entries from the partial sums (fixed order).
__global__ void __launch_bounds__(256) k_mean_from_partials(const double* __restrict__ partial, int64_t nparts,
                                                            int64_t n, double* __restrict__ mean) {
  __shared__ double ws[8];
  double s = 0.0;
  for (int64_t i = threadIdx.x; i < nparts; i += blockDim.x) s += partial[i];
  s = warp_sum(s);
  if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < 8; ++w) t += ws[w];
    *mean = t / (double)n;
  }
}

__global__ void k_subtract(double* __restrict__ b, int64_t n, const double* __restrict__ mean) {
  const double m = *mean;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    b[i] -= m;
}

// Integer point location: positions in units of the cell size at level G
// (a level finer than both forests), so cell centres and quadrant centres
// are exact.  Returns the leaf block of F containing the point and the cell
// inside it, or -1 (outside the forest: never for a valid forest).
__device__ __forceinline__ int64_t locate(const ForestView& F, int G, int64_t px, int64_t py, int& cell) {
  for (int l = 0; l < F.L; ++l) {
    const int64_t ci = px >> (G - l), cj = py >> (G - l);  // cell at level l
    const int64_t bi = ci >> 3, bj = cj >> 3;
    if (bi < 0 || bj < 0 || bi >= ((int64_t)F.bpdx << l) || bj >= ((int64_t)F.bpdy << l)) return -1;
    const int32_t b = F.table[F.off[l] + bj * ((int64_t)F.bpdx << l) + bi];
    if (b >= 0) {
      cell = (int)((cj & 7) * 8 + (ci & 7));
      return b;
    }
  }
  return -1;
}

// dst cell value: the src cell holding its centre when the src leaf there is
// as coarse or coarser (injection, exact copy on the same level); else the
// mean of the src cells at the centres of its four quadrants (the average
// of the four children for a one-level coarsening).
__global__ void k_transfer(ForestView S, const double* __restrict__ xs, ForestView D, double* __restrict__ xd,
                           int G) {
  const int64_t cell = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (cell >= D.nb * kBLEN) return;
  const int64_t blk = cell >> 6;
  const int c = (int)(cell & 63), ix = c & 7, iy = c >> 3;
  const int l = D.level[blk];
  const int sh = G - l;  // >= 2
  const int64_t px = (((int64_t)D.bx[blk] * 8 + ix) << sh) + (1ll << (sh - 1));
  const int64_t py = (((int64_t)D.by[blk] * 8 + iy) << sh) + (1ll << (sh - 1));
  int sc = 0;
  const int64_t sb = locate(S, G, px, py, sc);
  if (sb < 0) {
    xd[cell] = 0.0;
    return;
  }
  if (S.level[sb] <= l) {
    xd[cell] = xs[sb * kBLEN + sc];
    return;
  }
  const int64_t q = 1ll << (sh - 2);
  double acc = 0.0;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const int64_t qx = px + ((k & 1) ? q : -q), qy = py + ((k & 2) ? q : -q);
    int qc = 0;
    const int64_t qb = locate(S, G, qx, qy, qc);
    acc += qb >= 0 ? xs[qb * kBLEN + qc] : 0.0;
  }
  xd[cell] = 0.25 * acc;
}

// ------------------------------------------------ pressure step helpers --

// Per-CTA partial sums of h^2 p and of h^2 over the cells (the volume
// weights of PressureSingle.cpp:853-868), in a fixed order.
__global__ void __launch_bounds__(kRhsThreads) k_wsum_partials(const double* __restrict__ p,
                                                               const double* __restrict__ hblk, int64_t n,
                                                               double* __restrict__ partial) {
  const int64_t cell = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  double v = 0.0, w = 0.0;
  if (cell < n) {
    const double h = hblk[cell >> 6];
    w = h * h;
    v = p[cell] * w;
  }
  __shared__ double ws[2][kRhsThreads / 32];
  v = warp_sum(v);
  w = warp_sum(w);
  if ((threadIdx.x & 31) == 0) {
    ws[0][threadIdx.x >> 5] = v;
    ws[1][threadIdx.x >> 5] = w;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double a = 0.0, b = 0.0;
    for (int k = 0; k < kRhsThreads / 32; ++k) {
      a += ws[0][k];
      b += ws[1][k];
    }
    partial[2 * blockIdx.x] = a;
    partial[2 * blockIdx.x + 1] = b;
  }
}

// One CTA: avg = sum(h^2 p) / sum(h^2) from the partials (fixed order).
__global__ void __launch_bounds__(256) k_wmean(const double* __restrict__ partial, int64_t nparts,
                                               double* __restrict__ avg) {
  __shared__ double ws[2][8];
  double a = 0.0, b = 0.0;
  for (int64_t i = threadIdx.x; i < nparts; i += blockDim.x) {
    a += partial[2 * i];
    b += partial[2 * i + 1];
  }
  a = warp_sum(a);
  b = warp_sum(b);
  if ((threadIdx.x & 31) == 0) {
    ws[0][threadIdx.x >> 5] = a;
    ws[1][threadIdx.x >> 5] = b;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double sa = 0.0, sb = 0.0;
    for (int k = 0; k < 8; ++k) {
      sa += ws[0][k];
      sb += ws[1][k];
    }
    *avg = sa / sb;
  }
}

// pres += pold - avg (PressureSingle.cpp:869-879)
__global__ void k_add_pold(double* __restrict__ pres, const double* __restrict__ pold, int64_t n,
                           const double* __restrict__ avg) {
  const double a = *avg;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    pres[i] += pold[i] - a;
}

}  // namespace


int64_t wmean_partials(int64_t nb) { return 2 * ((nb * kBLEN + kRhsThreads - 1) / kRhsThreads) + 1; }

cudaError_t launch_add_pold(double* pres, const double* pold, const double* hblk, int64_t nb, double* partial,
                            cudaStream_t s) {
  const int64_t n = nb * kBLEN;
  if (n <= 0) return cudaSuccess;
  const int64_t parts = (n + kRhsThreads - 1) / kRhsThreads;
  double* avg = partial + 2 * parts;
  k_wsum_partials<<<(unsigned)parts, kRhsThreads, 0, s>>>(pres, hblk, n, partial);
  k_wmean<<<1, 256, 0, s>>>(partial, parts, avg);
  k_add_pold<<<(unsigned)std::min<int64_t>((n + 255) / 256, 148 * 16), 256, 0, s>>>(pres, pold, n, avg);
  return cudaGetLastError();
}

int fourier_mode_count(int kmax) {
  int n = 0;
  for (int ky = -kmax; ky <= kmax; ++ky)
    for (int kx = 0; kx <= kmax; ++kx)
      if (!(kx == 0 && ky <= 0) && kx * kx + ky * ky <= kmax * kmax) ++n;
  return n;
}

int64_t rhs_partials(int64_t nb) { return (nb * kBLEN + kRhsThreads - 1) / kRhsThreads; }

cudaError_t launch_rhs_fourier(const ForestView& F, int kmax, const double* coef, double* b, double* partial,
                               double* mean, cudaStream_t s) {
  const int64_t n = F.nb * kBLEN;
  if (n <= 0) return cudaSuccess;
  const int nm = fourier_mode_count(kmax);
  const int64_t parts = rhs_partials(F.nb);
  const size_t smem = sizeof(double) * 4 * nm;
  k_rhs_fourier<<<(unsigned)parts, kRhsThreads, smem, s>>>(F, kmax, nm, coef, b, partial);
  k_mean_from_partials<<<1, 256, 0, s>>>(partial, parts, n, mean);
  k_subtract<<<(unsigned)std::min<int64_t>((n + 255) / 256, 148 * 16), 256, 0, s>>>(b, n, mean);
  return cudaGetLastError();
}

cudaError_t launch_transfer(const ForestView& S, const double* xs, const ForestView& D, double* xd,
                            cudaStream_t s) {
  const int64_t n = D.nb * kBLEN;
  if (n <= 0) return cudaSuccess;
  const int G = (S.L > D.L ? S.L : D.L) + 1;
  k_transfer<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(S, xs, D, xd, G);
  return cudaGetLastError();
}

}  // namespace cup2d
