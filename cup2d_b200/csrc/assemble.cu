// Device-side construction of P^-1 and of the AMR 5-point operator.
//
// P^-1: ExpAMRSolver's constructor (source/Poisson/ExpAMRSolver.cpp:25-99)
// factors the 64x64 block Laplacian K (4 on the diagonal, -1 between grid
// neighbours of one 8x8 block) by Cholesky-Crout, inverts L by Gauss-Jordan
// and forms P^-1 = -(L^T)^-1 L^-1.  The kernel below runs the same
// recurrences in the same order with explicitly rounded FP64 operations
// (no FMA contraction), so the result is bit-identical to a plain IEEE CPU
// evaluation.
//
// Operator: ExpAMRSolver::getMat (ExpAMRSolver.cpp:180-313) on the host
// walks every cell and accumulates a std::map per edge row.  Here the
// operator is stored block-structured instead:
//   * interior cells and edge cells whose out-of-block faces are walls or
//     same-level neighbours are not stored at all; the SpMV evaluates them
//     from a 4-entry neighbour table per block;
//   * rows of cells on a coarse/fine face are stored explicitly (CSR) with
//     exactly the coefficients getMat produces: the same makeFlux /
//     interpolate / D1 / D2 contributions (ExpAMRSolver.cpp:100-178,
//     ExpAMRSolver.h:268-300) summed per column in call order, columns
//     ascending.
// The forest is indexed by dense per-level leaf tables (block id or -1),
// which answer Cubism's Exists / CheckCoarser / CheckFiner.
#include <cuda_runtime.h>

#include "common.cuh"
#include "kernels.hpp"

namespace cup2d {

// ---------------------------------------------------------------- P^-1 ----

__device__ __forceinline__ double blockK(int I1, int I2) {
  const int j1 = I1 / kBS, i1 = I1 % kBS, j2 = I2 / kBS, i2 = I2 % kBS;
  if (i1 == i2 && j1 == j2) return 4.0;
  if (abs(i1 - i2) + abs(j1 - j2) == 1) return -1.0;
  return 0.0;
}

// One CTA of 64 threads; L and Linv (lower triangles, 64x64) in shared memory.
__global__ void __launch_bounds__(64) k_build_pinv(double* __restrict__ P) {
  extern __shared__ double sm[];
  double* L = sm;              // L[i*64+k]
  double* Li = sm + 64 * 64;   // Linv[i*64+c]
  const int t = threadIdx.x;
  for (int q = t; q < 64 * 64; q += 64) {
    L[q] = 0.0;
    Li[q] = ((q / 64) == (q % 64)) ? 1.0 : 0.0;
  }
  __syncthreads();
  for (int i = 0; i < 64; ++i) {
    if (t == 0) {
      double s1 = 0.0;
      for (int k = 0; k <= i - 1; ++k) s1 = __dadd_rn(s1, __dmul_rn(L[i * 64 + k], L[i * 64 + k]));
      L[i * 64 + i] = __dsqrt_rn(__dadd_rn(blockK(i, i), -s1));
    }
    __syncthreads();
    const int j = t;
    if (j > i) {
      double s2 = 0.0;
      for (int k = 0; k <= i - 1; ++k) s2 = __dadd_rn(s2, __dmul_rn(L[i * 64 + k], L[j * 64 + k]));
      L[j * 64 + i] = __ddiv_rn(__dadd_rn(blockK(j, i), -s2), L[i * 64 + i]);
    }
    __syncthreads();
  }
  for (int br = 0; br < 64; ++br) {
    const double bsf = __ddiv_rn(1.0, L[br * 64 + br]);
    if (t <= br) Li[br * 64 + t] = __dmul_rn(Li[br * 64 + t], bsf);
    __syncthreads();
    const int wr = t;
    if (wr > br) {
      const double wsf = L[wr * 64 + br];
      for (int c = 0; c <= br; ++c)
        Li[wr * 64 + c] = __dadd_rn(Li[wr * 64 + c], -__dmul_rn(wsf, Li[br * 64 + c]));
    }
    __syncthreads();
  }
  // P[i][j] = -sum_{k >= max(i,j)} Li[k][i] Li[k][j]; the reference adds
  // 0.0 for k < max(i,j), which leaves the sum unchanged.
  for (int q = t; q < 64 * 64; q += 64) {
    const int i = q / 64, j = q % 64;
    double aux = 0.0;
    for (int k = 0; k < 64; ++k)
      aux = __dadd_rn(aux, (i <= k && j <= k) ? __dmul_rn(Li[k * 64 + i], Li[k * 64 + j]) : 0.0);
    P[q] = -aux;
  }
}

cudaError_t launch_build_pinv(double* d_P, cudaStream_t s) {
  const int smem = 2 * 64 * 64 * (int)sizeof(double);
  cudaError_t e = cudaFuncSetAttribute(k_build_pinv, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  if (e != cudaSuccess) return e;
  k_build_pinv<<<1, 64, smem, s>>>(d_P);
  return cudaGetLastError();
}

__global__ void k_convert_f64_f32(const double* __restrict__ a, float* __restrict__ b, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    b[i] = (float)a[i];
}

cudaError_t launch_convert_f64_f32(const double* a, float* b, int64_t n, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  const int threads = 256;
  const int64_t blocks = (n + threads - 1) / threads;
  k_convert_f64_f32<<<(unsigned)(blocks < 4096 ? blocks : 4096), threads, 0, s>>>(a, b, n);
  return cudaGetLastError();
}

// -------------------------------------------------------------- forest ----

struct ForestDev {
  int32_t bpdx, bpdy, L, px, py;
  int64_t nb;
  const int32_t* level;
  const int32_t* bx;
  const int32_t* by;
  const int32_t* table;  // per-level dense leaf tables
  int64_t off[kMaxLevels + 1];

  __device__ __forceinline__ int64_t nx(int l) const { return (int64_t)bpdx << l; }
  __device__ __forceinline__ int64_t ny(int l) const { return (int64_t)bpdy << l; }
  __device__ __forceinline__ int32_t leaf(int l, int64_t i, int64_t j) const {
    if (l < 0 || l >= L) return -1;
    return table[off[l] + j * nx(l) + i];
  }
};

__global__ void k_fill_tables(ForestDev F, int32_t* __restrict__ table, int* __restrict__ err) {
  const int64_t b = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (b >= F.nb) return;
  const int l = F.level[b];
  if (l < 0 || l >= F.L) { atomicExch(err, 1); return; }
  const int64_t i = F.bx[b], j = F.by[b];
  if (i < 0 || j < 0 || i >= F.nx(l) || j >= F.ny(l)) { atomicExch(err, 1); return; }
  const int prev = atomicCAS(&table[F.off[l] + j * F.nx(l) + i], -1, (int)b);
  if (prev != -1) atomicExch(err, 2);  // duplicate leaf
}

// Neighbour position across face f at the block's level; false for a wall.
__device__ __forceinline__ bool face_pos(const ForestDev& F, int l, int64_t i, int64_t j, int f,
                                         int64_t& ni, int64_t& nj) {
  ni = i + (f == 0 ? -1 : f == 1 ? 1 : 0);
  nj = j + (f == 2 ? -1 : f == 3 ? 1 : 0);
  const int64_t nx = F.nx(l), ny = F.ny(l);
  if (ni < 0 || ni >= nx) {
    if (!F.px) return false;
    ni = (ni + nx) % nx;
  }
  if (nj < 0 || nj >= ny) {
    if (!F.py) return false;
    nj = (nj + ny) % ny;
  }
  return true;
}

// Children of the same-level position (ni,nj) that touch face f of the block.
__device__ __forceinline__ void touching_children(int f, int64_t ni, int64_t nj, int64_t ci[2], int64_t cj[2]) {
  for (int h = 0; h < 2; ++h) {
    switch (f) {
      case 0: ci[h] = 2 * ni + 1; cj[h] = 2 * nj + h; break;
      case 1: ci[h] = 2 * ni + 0; cj[h] = 2 * nj + h; break;
      case 2: ci[h] = 2 * ni + h; cj[h] = 2 * nj + 1; break;
      default: ci[h] = 2 * ni + h; cj[h] = 2 * nj + 0; break;
    }
  }
}

__global__ void k_classify(ForestDev F, int32_t* __restrict__ nbr, unsigned long long* __restrict__ xmask,
                           int32_t* __restrict__ xcount, double* __restrict__ hblk, double h0,
                           int* __restrict__ err) {
  const int64_t b = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (b >= F.nb) return;
  const int l = F.level[b];
  const int64_t i = F.bx[b], j = F.by[b];
  if (l < 0 || l >= F.L || i < 0 || j < 0 || i >= F.nx(l) || j >= F.ny(l)) {
    atomicExch(err, 1);  // reported by k_fill_tables too; never index with it
    for (int f = 0; f < 4; ++f) nbr[4 * b + f] = kWall;
    xmask[b] = 0ull;     // no explicit rows: the row pass skips the block
    xcount[b] = 0;
    hblk[b] = 0.0;
    return;
  }
  // a leaf must not have a leaf ancestor
  for (int q = l - 1; q >= 0; --q)
    if (F.leaf(q, i >> (l - q), j >> (l - q)) >= 0) { atomicExch(err, 3); }
  unsigned long long mask = 0ull;
  for (int f = 0; f < 4; ++f) {
    int64_t ni, nj;
    int32_t code;
    if (!face_pos(F, l, i, j, f, ni, nj)) {
      code = kWall;
    } else {
      const int32_t s = F.leaf(l, ni, nj);
      if (s >= 0) {
        code = s;
      } else if (F.leaf(l - 1, ni >> 1, nj >> 1) >= 0) {
        code = kExplicit;
      } else {
        int64_t ci[2], cj[2];
        touching_children(f, ni, nj, ci, cj);
        if (F.leaf(l + 1, ci[0], cj[0]) >= 0 && F.leaf(l + 1, ci[1], cj[1]) >= 0) {
          code = kExplicit;
        } else {
          atomicExch(err, 4);  // hole or 2:1 violation
          code = kWall;
        }
      }
    }
    nbr[4 * b + f] = code;
    if (code == kExplicit) {
      for (int c = 0; c < 8; ++c) {
        const int ix = f == 0 ? 0 : f == 1 ? 7 : c;
        const int iy = f == 2 ? 0 : f == 3 ? 7 : c;
        mask |= 1ull << (iy * 8 + ix);
      }
    }
  }
  xmask[b] = mask;
  xcount[b] = __popcll(mask);
  hblk[b] = h0 / (double)(1ll << l);
}

// The leaf at the domain's (0, 0) corner: the block whose index is (0, 0) at
// its level (ExpAMRSolver.cpp:251-256 places bMeanConstraint's row there).
__global__ void k_origin(ForestDev F, int* __restrict__ out) {
  int32_t b = -1;
  for (int l = 0; l < F.L && b < 0; ++l) b = F.leaf(l, 0, 0);
  *out = b;
}

// ------------------------------------------------------------- scans ------

// Exclusive scan of int32 counts into int32 offsets (out[n] = total), in
// three passes: per-CTA sums, a single-CTA scan of the sums, a fix-up.
constexpr int kScanThreads = 512;
constexpr int kScanItems = 4;
constexpr int kScanTile = kScanThreads * kScanItems;

__device__ __forceinline__ int cta_exclusive_scan(int v, int* sh, int& total) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  int inc = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int n = __shfl_up_sync(kFull, inc, o);
    if (lane >= o) inc += n;
  }
  if (lane == 31) sh[w] = inc;
  __syncthreads();
  if (w == 0) {
    const int nw = blockDim.x >> 5;
    int s = lane < nw ? sh[lane] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int n = __shfl_up_sync(kFull, s, o);
      if (lane >= o) s += n;
    }
    if (lane < nw) sh[lane] = s;  // inclusive warp sums
  }
  __syncthreads();
  const int before = (w > 0 ? sh[w - 1] : 0) + inc - v;
  total = sh[(blockDim.x >> 5) - 1];
  __syncthreads();
  return before;
}

__global__ void __launch_bounds__(kScanThreads) k_scan_tiles(const int32_t* __restrict__ in, int64_t n,
                                                             int32_t* __restrict__ out, int32_t* __restrict__ tile_sums) {
  __shared__ int sh[32];
  const int64_t base = (int64_t)blockIdx.x * kScanTile + threadIdx.x * kScanItems;
  int v[kScanItems], s = 0;
#pragma unroll
  for (int q = 0; q < kScanItems; ++q) {
    v[q] = (base + q < n) ? in[base + q] : 0;
    s += v[q];
  }
  int total;
  int run = cta_exclusive_scan(s, sh, total);
#pragma unroll
  for (int q = 0; q < kScanItems; ++q) {
    if (base + q < n) out[base + q] = run;
    run += v[q];
  }
  if (threadIdx.x == 0) tile_sums[blockIdx.x] = total;
}

__global__ void __launch_bounds__(kScanThreads) k_scan_sums(int32_t* __restrict__ sums, int64_t ntiles,
                                                            int32_t* __restrict__ total_out) {
  __shared__ int sh[32];
  int carry = 0;
  for (int64_t b0 = 0; b0 < ntiles; b0 += kScanThreads) {
    const int64_t q = b0 + threadIdx.x;
    const int v = q < ntiles ? sums[q] : 0;
    int total;
    const int ex = cta_exclusive_scan(v, sh, total);
    if (q < ntiles) sums[q] = carry + ex;
    carry += total;
  }
  if (threadIdx.x == 0) *total_out = carry;
}

__global__ void k_scan_fix(int32_t* __restrict__ out, int64_t n, const int32_t* __restrict__ sums,
                           const int32_t* __restrict__ total) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < n) out[i] += sums[i / kScanTile];
  if (i == n) out[n] = *total;
}

int64_t scan_temp_ints(int64_t n) { return (n + kScanTile - 1) / kScanTile + 1; }

cudaError_t launch_exclusive_scan(const int32_t* in, int64_t n, int32_t* out, int32_t* tmp, cudaStream_t s) {
  const int64_t ntiles = (n + kScanTile - 1) / kScanTile;
  if (ntiles > 0) k_scan_tiles<<<(unsigned)ntiles, kScanThreads, 0, s>>>(in, n, out, tmp);
  k_scan_sums<<<1, kScanThreads, 0, s>>>(tmp, ntiles, tmp + ntiles);
  k_scan_fix<<<(unsigned)((n + 1 + 255) / 256), 256, 0, s>>>(out, n, tmp, tmp + ntiles);
  return cudaGetLastError();
}

// --------------------------------------------------------- explicit rows ---

constexpr int kMaxRowNnz = 32;

struct RowAcc {  // SpRowInfo::mapColVal: columns ascending, values summed in call order
  int n;
  int32_t c[kMaxRowNnz];
  double v[kMaxRowNnz];
  bool overflow;
  __device__ __forceinline__ void add(int64_t col, double val) {
    int k = 0;
    while (k < n && c[k] < col) ++k;
    if (k < n && c[k] == col) {
      v[k] = __dadd_rn(v[k], val);
      return;
    }
    if (n == kMaxRowNnz) { overflow = true; return; }
    for (int q = n; q > k; --q) { c[q] = c[q - 1]; v[q] = v[q - 1]; }
    c[k] = (int32_t)col;
    v[k] = __dadd_rn(0.0, val);
    ++n;
  }
};

__device__ __forceinline__ int64_t cell(int64_t blk, int ix, int iy) { return blk * kBLEN + iy * kBS + ix; }

// Index maps of the four face indexers (ExpAMRSolver.h:150-258).
struct Face {
  int f;  // 0 Xm, 1 Xp, 2 Ym, 3 Yp
  __device__ __forceinline__ bool xb() const { return f < 2; }
  __device__ __forceinline__ double taylorSign(int ix, int iy) const {
    return xb() ? (iy % 2 == 0 ? -1. : 1.) : (ix % 2 == 0 ? -1. : 1.);
  }
  __device__ __forceinline__ bool isBD(int ix, int iy) const {
    return xb() ? (iy == 7 || iy == 3) : (ix == 7 || ix == 3);
  }
  __device__ __forceinline__ bool isFD(int ix, int iy) const {
    return xb() ? (iy == 0 || iy == 4) : (ix == 0 || ix == 4);
  }
  __device__ __forceinline__ int64_t nei(int64_t blk, int ix, int iy, int d) const {
    return xb() ? cell(blk, ix, iy + d) : cell(blk, ix + d, iy);
  }
  // cell of a neighbour block that sits across the face, `off` cells deep
  __device__ __forceinline__ int64_t across(int64_t nblk, int ix, int iy, int off) const {
    switch (f) {
      case 0: return cell(nblk, 7 - off, iy);
      case 1: return cell(nblk, off, iy);
      case 2: return cell(nblk, ix, 7 - off);
      default: return cell(nblk, ix, off);
    }
  }
  __device__ __forceinline__ int64_t inward(int64_t blk, int ix, int iy) const {
    switch (f) {
      case 0: return cell(blk, ix + 1, iy);
      case 1: return cell(blk, ix - 1, iy);
      case 2: return cell(blk, ix, iy + 1);
      default: return cell(blk, ix, iy - 1);
    }
  }
};

__device__ void taylor_terms(const Face& F, int64_t blk_c, int ixc, int iyc, double sT, double tf, RowAcc& row) {
  int64_t c0, c1, c2;
  double w0, w1, w2;
  // D1, scaled by h/4 (ExpAMRSolver.h:268-283)
  if (F.isBD(ixc, iyc)) {
    c0 = F.nei(blk_c, ixc, iyc, -2); w0 = 1. / 8.;
    c1 = F.nei(blk_c, ixc, iyc, -1); w1 = -1. / 2.;
    c2 = cell(blk_c, ixc, iyc);      w2 = 3. / 8.;
  } else if (F.isFD(ixc, iyc)) {
    c0 = F.nei(blk_c, ixc, iyc, 2);  w0 = -1. / 8.;
    c1 = F.nei(blk_c, ixc, iyc, 1);  w1 = 1. / 2.;
    c2 = cell(blk_c, ixc, iyc);      w2 = -3. / 8.;
  } else {
    c0 = F.nei(blk_c, ixc, iyc, -1); w0 = -1. / 8.;
    c1 = F.nei(blk_c, ixc, iyc, 1);  w1 = 1. / 8.;
    c2 = cell(blk_c, ixc, iyc);      w2 = 0.;
  }
  const double st = __dmul_rn(sT, tf);
  row.add(c0, __dmul_rn(st, w0));
  row.add(c1, __dmul_rn(st, w1));
  row.add(c2, __dmul_rn(st, w2));
  // D2, scaled by (h/4)^2/2 (ExpAMRSolver.h:285-300)
  if (F.isBD(ixc, iyc)) {
    c0 = F.nei(blk_c, ixc, iyc, -2); w0 = 1. / 32.;
    c1 = F.nei(blk_c, ixc, iyc, -1); w1 = -1. / 16.;
    c2 = cell(blk_c, ixc, iyc);      w2 = 1. / 32.;
  } else if (F.isFD(ixc, iyc)) {
    c0 = F.nei(blk_c, ixc, iyc, 2);  w0 = 1. / 32.;
    c1 = F.nei(blk_c, ixc, iyc, 1);  w1 = -1. / 16.;
    c2 = cell(blk_c, ixc, iyc);      w2 = 1. / 32.;
  } else {
    c0 = F.nei(blk_c, ixc, iyc, -1); w0 = 1. / 32.;
    c1 = F.nei(blk_c, ixc, iyc, 1);  w1 = 1. / 32.;
    c2 = cell(blk_c, ixc, iyc);      w2 = -1. / 16.;
  }
  row.add(c0, __dmul_rn(tf, w0));
  row.add(c1, __dmul_rn(tf, w1));
  row.add(c2, __dmul_rn(tf, w2));
}

// interpolate(): ghost value of a fine cell from (close, far) fine cells and
// a quadratic Taylor expansion around coarse cell (ixc, iyc).
__device__ void interp(const Face& F, int64_t blk_c, int ixc, int iyc, int64_t close, int64_t far,
                       double sI, double sT, RowAcc& row) {
  row.add(close, __ddiv_rn(__dmul_rn(sI, 2.), 3.));
  row.add(far, __ddiv_rn(__dmul_rn(-sI, 1.), 5.));
  const double tf = __ddiv_rn(__dmul_rn(sI, 8.), 15.);
  row.add(cell(blk_c, ixc, iyc), tf);
  taylor_terms(F, blk_c, ixc, iyc, sT, tf, row);
}

// Row of edge cell (ix,iy) of block b, in getMat's order of contributions.
__device__ void build_row(const ForestDev& Fd, int64_t b, int ix, int iy, RowAcc& row, int* err) {
  row.n = 0;
  row.overflow = false;
  const int l = Fd.level[b];
  const int64_t bi = Fd.bx[b], bj = Fd.by[b];
  const int64_t self = cell(b, ix, iy);
  const bool valid[4] = {ix > 0, ix < 7, iy > 0, iy < 7};
  const int64_t inb[4] = {cell(b, ix - 1, iy), cell(b, ix + 1, iy), cell(b, ix, iy - 1), cell(b, ix, iy + 1)};
  for (int f = 0; f < 4; ++f) {
    if (valid[f]) {
      row.add(inb[f], 1.);
      row.add(self, -1.);
      continue;
    }
    int64_t ni, nj;
    if (!face_pos(Fd, l, bi, bj, f, ni, nj)) continue;  // wall: no flux
    const Face F{f};
    const int32_t same = Fd.leaf(l, ni, nj);
    if (same >= 0) {
      row.add(F.across(same, ix, iy, 0), 1.);
      row.add(self, -1.);
      continue;
    }
    const int32_t coarse = Fd.leaf(l - 1, ni >> 1, nj >> 1);
    if (coarse >= 0) {
      const int ixc = f == 0 ? 7 : f == 1 ? 0 : (bi % 2 == 0 ? ix / 2 : ix / 2 + 4);
      const int iyc = f == 2 ? 7 : f == 3 ? 0 : (bj % 2 == 0 ? iy / 2 : iy / 2 + 4);
      interp(F, coarse, ixc, iyc, self, F.inward(b, ix, iy), 1., F.taylorSign(ix, iy), row);
      row.add(self, -1.);
      continue;
    }
    // finer neighbour: child touching this cell (Zchild), fine cells of
    // rows/columns 2*(i%4) and 2*(i%4)+1
    const int half = F.xb() ? (iy >= 4) : (ix >= 4);
    int64_t ci, cj;
    switch (f) {
      case 0: ci = 2 * ni + 1; cj = 2 * nj + half; break;
      case 1: ci = 2 * ni + 0; cj = 2 * nj + half; break;
      case 2: ci = 2 * ni + half; cj = 2 * nj + 1; break;
      default: ci = 2 * ni + half; cj = 2 * nj + 0; break;
    }
    const int32_t fine = Fd.leaf(l + 1, ci, cj);
    if (fine < 0) { atomicExch(err, 4); return; }
    const int fx = (ix % 4) * 2, fy = (iy % 4) * 2;
    for (int q = 0; q < 2; ++q) {
      const int gx = F.xb() ? fx : fx + q;  // neiFine1 (q=0) / neiFine2 (q=1)
      const int gy = F.xb() ? fy + q : fy;
      const int64_t close = F.across(fine, gx, gy, 0);
      const int64_t far = F.across(fine, gx, gy, 1);
      row.add(close, 1.);
      interp(F, b, ix, iy, close, far, -1., q == 0 ? -1. : 1., row);
    }
  }
  if (row.overflow) atomicExch(err, 5);
}

// One CTA of 64 threads per block; thread = cell.  Pass 0 writes the row
// length, pass 1 the row.
__global__ void __launch_bounds__(64) k_rows(ForestDev Fd, const unsigned long long* __restrict__ xmask,
                                             const int32_t* __restrict__ xbase, int32_t* __restrict__ rowlen,
                                             int32_t* __restrict__ rowcell, const int32_t* __restrict__ xptr,
                                             int32_t* __restrict__ xcol, double* __restrict__ xval, int pass,
                                             int64_t cap, int* __restrict__ err) {
  const int64_t b = blockIdx.x;
  const int c = threadIdx.x;
  const unsigned long long m = xmask[b];  // 0 for a block k_classify rejected
  if (!((m >> c) & 1ull)) return;
  const int64_t r = xbase[b] + __popcll(m & ((1ull << c) - 1ull));
  if (r < 0 || r >= cap) {  // never for masks k_classify wrote; keep every index valid
    atomicExch(err, 6);
    return;
  }
  RowAcc row;
  build_row(Fd, b, c & 7, c >> 3, row, err);
  if (pass == 0) {
    rowlen[r] = row.n;
    rowcell[r] = (int32_t)(b * kBLEN + c);
  } else {
    const int32_t o = xptr[r];
    for (int k = 0; k < row.n; ++k) {
      xcol[o + k] = row.c[k];
      xval[o + k] = row.v[k];
    }
  }
}

// ------------------------------------------------------------ driver ------

int assemble_on_device(const AssembleIn& in, DeviceMesh& out, cudaStream_t s) {
  // All device buffers in `out` are owned by the caller (allocated through
  // the callbacks); this routine only fills them.
  ForestDev F{};
  F.bpdx = in.bpdx;
  F.bpdy = in.bpdy;
  F.L = in.level_max;
  F.px = in.periodic_x;
  F.py = in.periodic_y;
  F.nb = in.nblocks;
  F.level = out.level;
  F.bx = out.bx;
  F.by = out.by;
  F.table = out.table;
  int64_t off = 0;
  for (int l = 0; l < in.level_max; ++l) {
    F.off[l] = off;
    off += ((int64_t)in.bpdx << l) * ((int64_t)in.bpdy << l);
  }
  F.off[in.level_max] = off;
  const int64_t nb = in.nblocks;
  const unsigned g = (unsigned)((nb + 255) / 256);
  if (cudaMemsetAsync(out.table, 0xff, sizeof(int32_t) * off, s) != cudaSuccess) return CUP2D_CUDA_ERROR;
  if (cudaMemsetAsync(out.err, 0, sizeof(int), s) != cudaSuccess) return CUP2D_CUDA_ERROR;
  k_fill_tables<<<g, 256, 0, s>>>(F, out.table, out.err);
  k_classify<<<g, 256, 0, s>>>(F, out.nbr, out.xmask, out.xcount, out.hblk, in.h0, out.err);
  k_origin<<<1, 1, 0, s>>>(F, out.err + 1);
  launch_exclusive_scan(out.xcount, nb, out.xbase, out.scan_tmp, s);
  // Row arrays at their bound (a block's explicit rows are cells of its four
  // faces: at most 28), so that the row lengths are built and scanned before
  // the host knows the row count: one host round trip reads the row count,
  // the non-zero count and the error flags together.
  const int64_t cap = kMaxExplicitRowsPerBlock * nb;
  int st = out.alloc_rows(out.ctx, cap);
  if (st != CUP2D_OK) return st;
  if (cudaMemsetAsync(out.rowlen, 0, sizeof(int32_t) * cap, s) != cudaSuccess) return CUP2D_CUDA_ERROR;
  k_rows<<<(unsigned)nb, 64, 0, s>>>(F, out.xmask, out.xbase, out.rowlen, out.rowcell, nullptr, nullptr, nullptr, 0,
                                     cap, out.err);
  launch_exclusive_scan(out.rowlen, cap, out.xptr, out.scan_tmp, s);
  if (cudaGetLastError() != cudaSuccess) return CUP2D_CUDA_ERROR;
  int32_t hR = 0, hnnz = 0;
  int herr[2] = {0, -1};
  if (cudaMemcpyAsync(&hR, out.xbase + nb, sizeof(int32_t), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
      cudaMemcpyAsync(&hnnz, out.xptr + cap, sizeof(int32_t), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
      cudaMemcpyAsync(herr, out.err, 2 * sizeof(int), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
      cudaStreamSynchronize(s) != cudaSuccess)
    return CUP2D_CUDA_ERROR;
  if (herr[0] != 0 || herr[1] < 0 || hR > cap) return CUP2D_BAD_MESH;
  out.origin = herr[1];
  out.R = hR;
  out.nnz = hnnz;
  st = out.alloc_nnz(out.ctx, hnnz);
  if (st != CUP2D_OK) return st;
  if (hR > 0) {
    // the same rows as the length pass (build_row is deterministic): any
    // malformed face was flagged there already
    k_rows<<<(unsigned)nb, 64, 0, s>>>(F, out.xmask, out.xbase, out.rowlen, out.rowcell, out.xptr, out.xcol,
                                       out.xval, 1, cap, out.err);
    launch_convert_f64_f32(out.xval, out.xval32, hnnz, s);
  }
  // the operator is complete when this returns: solves on other streams use it
  if (cudaGetLastError() != cudaSuccess || cudaStreamSynchronize(s) != cudaSuccess) return CUP2D_CUDA_ERROR;
  return CUP2D_OK;
}

int64_t leaf_table_entries(int bpdx, int bpdy, int level_max) {
  int64_t off = 0;
  for (int l = 0; l < level_max; ++l) off += ((int64_t)bpdx << l) * ((int64_t)bpdy << l);
  return off;
}

}  // namespace cup2d
