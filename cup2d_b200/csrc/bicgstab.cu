// BiCGSTAB with the 64x64 block-Jacobi preconditioner, one persistent launch
// per solve.
//
//   k_bicgstab64     plain FP64: the drop-in form of BiCGSTABSolver::main
//                    (source/Poisson/BiCGSTAB.cu:412-620)
//   k_bicgstab_mixed FP32 Krylov vectors and split-TF32 tensor-core P^-1;
//                    FP64 solution update, FP64 true-residual replacement
//                    ("reliable updates") and FP64 convergence test
//
// The reference runs each iteration as ~25 library launches (cuSPARSE COO
// SpMV, cuBLAS dot/nrm2/axpy/scal/Idamax/Dgemm), 8 one-thread scalar kernels
// and 4 host round-trips.  Here one cooperative kernel runs the whole solve.
// Each CTA owns an equal contiguous range of blocks, and an equal share of
// the explicit (coarse/fine) rows for the SpMVs; an iteration is five fused
// passes over them, separated by bounded grid barriers:
//
//   A  p = r + beta (p - omega nu);  z = P^-1 p          (R r,p,nu  W p,z)
//   B  nu = A z;  (rhat, nu)                             (R z,rhat  W nu)
//   C  s = r - alpha nu;  z2 = P^-1 s                    (R r,nu    W s,z2)
//   D  t = A z2;  (t,s), (t,t)                           (R z2,s    W t)
//   E  x += alpha z, x += omega z2;  r = s - omega t;
//      |r|_inf, (rhat,r), |r|^2, |rhat|^2                (R x,z,z2,s,t,rhat W x,r)
//
// The two x updates of the reference (alpha z after the first half step,
// omega z2 after the second) are applied in that order in pass E, which
// gives the same values while touching x once per iteration.
//
// Scalar recurrences, the breakdown/restart rule (rho^2 < 1e-16|r|^2|rhat|^2),
// best-iterate tracking and the L-inf stopping test follow the reference.
// Every CTA reduces the per-CTA partials in the same fixed order (FP64), so
// all CTAs take identical decisions and results are bitwise reproducible for
// a given grid.  The best iterate is copied lazily: pass E of the next
// iteration stores the old x when the previous iterate was the best so far.
//
// Mixed form.  A correction accumulated in FP32 loses eps32*kappa of the
// residual (kappa ~ 1e5..1e7 on these meshes), so restarted FP32 inner
// solves cannot refine.  Instead x stays FP64 and is updated in pass E from
// the FP32 z and z2; only the Krylov vectors (r, rhat, p, nu, t, z, z2) are
// FP32.  When the FP32 residual has dropped by `reliable_delta` since its
// last replacement, claims convergence, or a sweep stalls, it is replaced by
// the true residual b - A x computed in FP64 (with b projected to zero sum,
// the Neumann compatibility condition); by default the recurrences restart
// from it (rhat = r, p = nu = 0), which FP32 needs here: on the large
// meshes the unrestarted FP32 recurrences diverge.  Convergence is declared
// only on the true FP64 residual, and the best iterate (returned when the
// solve stops unconverged) is the refreshed x with the lowest true residual.
#include <cuda_runtime.h>

#include <atomic>

#include <algorithm>
#include <type_traits>

#include "common.cuh"
#include "kernels.hpp"
#include "spmv.cuh"

namespace cup2d {

namespace {

constexpr int kWarps = kSolveThreads / 32;
constexpr int kPad = 68;  // staged block row (conflict-free fragment loads)
constexpr int kMaxSweep = 64;  // mixed: longest FP32 sweep between true residuals

enum : int {
  Q_INIT = 0,   // 3: |A x0|_inf, |r0|_inf, |r0|^2
  Q_RHNU = 3,   // pass B
  Q_TS = 4,     // pass D: (t,s), (t,t)
  Q_RMAX = 6,   // pass E: |r|_inf, (rhat,r), |r|^2, |rhat|^2
  Q_HX = 10,    // mean removal: sum h^2 x, sum h^2
  Q_RU = 12,    // true residual: |r64|_inf, (rhat,r), |r|^2, |rhat|^2, |r32|_inf
  Q_SUMB = 17,  // sum b
  // single solves with the mean constraint (kRedQMean slots)
  Q_MB = 20,    // pass B: (rhat,nu), sum h^2 z, rhat_m nu_m, rhat_m
  Q_MD = 24,    // pass D: (t,s), (t,t), sum h^2 z2, t_m s_m, t_m t_m, s_m
  Q_MX = 30     // sum h^2 x0
};
static_assert(Q_SUMB + 1 <= kRedQ, "reduction slots");
static_assert(Q_MX + 1 <= kRedQMean, "reduction slots (mean constraint)");

// Shared memory of the solve kernels, per precision T of the Krylov vectors:
// P^-1, the P^-1 staging tiles, the staged SpMV rings and the reduction
// scratch.  Both layouts stay below 54 KB so that the kernels run at 3 CTAs
// per SM (the FP64 batch and the server's instances) within the 164 KB
// shared carve-out and leave 92 KB of the unified L1/shared array as L1
// (their spill reloads and table reads live there: the same kernel with the
// whole array given to shared memory ran 11 % slower).  The kernels at 2
// CTAs per SM take a smaller carve-out and keep more L1.
template <class T>
union TileSmem;
template <>
union TileSmem<double> {
  double d[2][8][kPad];             // P^-1 staging tiles, FP64 SpMV scratch
  SpmvStage<double> s64[kWarps];    // staged SpMV rings (passes B, D), one per warp
};
template <>
union TileSmem<float> {
  double d[2][8][kPad];             // FP64 SpMV scratch (true residual)
  float f[2][16][kPad];             // P^-1 staging tiles
  SpmvStage<float> s32[kWarps];     // staged SpMV rings (passes B, D), one per warp
};

// P^-1 operand: FP64 rows, or the TF32 split of the FP32 P^-1 (hi, lo),
// in rows of 64 values with the columns XOR-swizzled by the row (see the
// Pinv specialisations): conflict-free fragment loads without padding.
template <class T>
struct PinvSmem;
template <>
struct PinvSmem<double> {
  double v[kBLEN][kBLEN];
};
template <>
struct PinvSmem<float> {
  uint32_t hi[kBLEN][kBLEN];
  uint32_t lo[kBLEN][kBLEN];
};

template <class T>
struct Smem {
  PinvSmem<T> P;
  TileSmem<T> tile;
  double wred[kWarps][6];
  double gres[6];
  int flag;
  // the CTAs solving one problem together: this CTA's rank among them and
  // their number (the whole grid for a single solve, a group in a batch)
  int team_rank, team_size;
  int slot;           // batch: the problem the team works on
};

// the warp's ring of the staged SpMV
__device__ __forceinline__ SpmvStage<float>& spmv_stage(Smem<float>& sm) { return sm.tile.s32[threadIdx.x >> 5]; }
__device__ __forceinline__ SpmvStage<double>& spmv_stage(Smem<double>& sm) { return sm.tile.s64[threadIdx.x >> 5]; }

// the warp's block row of the FP64 staging tile, as SpMV scratch
template <class SM>
__device__ __forceinline__ double* spmv_row(SM& sm) {
  return sm.tile.d[0][threadIdx.x >> 5];
}

// max that propagates NaN (fmax drops it, which would let a blown-up
// residual read as converged)
__device__ __forceinline__ double nanmax(double a, double b) { return (a > b || a != a) ? a : b; }

template <int NV, class SM>
__device__ __forceinline__ void cta_partials(SM& sm, const double (&v)[NV], unsigned is_max,
                                             double* __restrict__ red, int q0) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
  for (int q = 0; q < NV; ++q) {
    double r = v[q];
    if ((is_max >> q) & 1u) {
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) r = nanmax(r, __shfl_xor_sync(kFull, r, o));
    } else {
      r = warp_sum(r);
    }
    if (lane == 0) sm.wred[w][q] = r;
  }
  __syncthreads();
  if (threadIdx.x < NV) {
    const int q = threadIdx.x;
    double acc = sm.wred[0][q];
    for (int k = 1; k < kWarps; ++k)
      acc = ((is_max >> q) & 1u) ? nanmax(acc, sm.wred[k][q]) : acc + sm.wred[k][q];
    red[(q0 + q) * sm.team_size + sm.team_rank] = acc;
  }
}

template <int NV, class SM>
__device__ __forceinline__ void grid_reduce(SM& sm, unsigned is_max, const double* __restrict__ red, int q0) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (w < NV) {
    const bool mx = (is_max >> w) & 1u;
    const double* src = red + (q0 + w) * sm.team_size;
    double acc = 0.0;
    for (int j = lane; j < sm.team_size; j += 32) {
      const double v = __ldcg(src + j);
      acc = mx ? nanmax(acc, v) : acc + v;
    }
    if (mx) {
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) acc = nanmax(acc, __shfl_xor_sync(kFull, acc, o));
    } else {
      acc = warp_sum(acc);
    }
    if (lane == 0) sm.gres[w] = acc;
  }
  __syncthreads();
}

// ------------------------------------------------ P^-1 tile application ----

template <class T>
struct Pinv;

// FP64: tiles of 8 blocks; warp w computes rows 8w..8w+7 with DMMA m8n8k4.
// P^-1 stays in shared memory in rows of 64 doubles whose column c is stored
// at c ^ 4*(r mod 8): the A-fragment loads (lane g,t reads row 8w+g, column
// 4kk+t) hit every bank pair once per 16 lanes, the minimum two wavefronts
// for 32 doubles.
template <>
struct Pinv<double> {
  static constexpr int kTile = 8;
  const double (*P)[kBLEN];
  __device__ __forceinline__ static int swz(int r, int c) { return c ^ ((r & 7) << 2); }
  // all threads; the caller synchronises before the first apply
  __device__ __forceinline__ void load(PinvSmem<double>& s, const double* __restrict__ Pg, const float*) {
    for (int q = threadIdx.x; q < kBLEN * kBLEN; q += blockDim.x) {
      const int r = q / kBLEN, c = q % kBLEN;
      s.v[r][swz(r, c)] = __ldg(Pg + q);
    }
    P = s.v;
  }
  template <class SM>
  __device__ __forceinline__ static double (*rows(SM& sm, int buf))[kPad] { return sm.tile.d[buf]; }
  __device__ __forceinline__ void apply(const double (*tile)[kPad], int w, int lane, int tb, int nvalid,
                                        double* __restrict__ z) const {
    const int g = lane >> 2, t = lane & 3;
    const int r = 8 * w + g;  // r mod 8 == g
    const double* arow = P[r];
    double c0 = 0.0, c1 = 0.0, e0 = 0.0, e1 = 0.0;
#pragma unroll
    for (int kk = 0; kk < 16; kk += 2) {
      dmma_884(c0, c1, arow[swz(r, 4 * kk + t)], tile[g][4 * kk + t]);
      dmma_884(e0, e1, arow[swz(r, 4 * (kk + 1) + t)], tile[g][4 * (kk + 1) + t]);
    }
    c0 += e0;
    c1 += e1;
    if (2 * t < nvalid) z[(tb + 2 * t) * kBLEN + 8 * w + g] = c0;
    if (2 * t + 1 < nvalid) z[(tb + 2 * t + 1) * kBLEN + 8 * w + g] = c1;
  }
};

__device__ __forceinline__ uint32_t to_tf32(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return r;
}

__device__ __forceinline__ void mma_tf32(float (&d)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// FP32: tiles of 16 blocks; warp w computes rows 16*(w&3).. of blocks
// 8*(w>>2).. with m16n8k8 TF32 MMA.  Operands are split x = hi + lo (both
// TF32) and z = Phi*hi + Phi*lo + Plo*hi, accumulated in FP32, which keeps
// the preconditioner apply at FP32 accuracy.  The split P = Phi + Plo (TF32
// bit patterns) is formed once, in rows of 64 words whose column c is
// stored at c ^ 4*(r mod 8): the A-fragment loads (lane g, t reads row
// 16m+g, column 8kk+t) then fall in 32 distinct banks.
template <>
struct Pinv<float> {
  static constexpr int kTile = 16;
  const uint32_t (*Ph)[kBLEN];
  const uint32_t (*Pl)[kBLEN];
  __device__ __forceinline__ static int swz(int r, int c) { return c ^ ((r & 7) << 2); }
  // all threads; the caller synchronises before the first apply
  __device__ __forceinline__ void load(PinvSmem<float>& s, const double*, const float* __restrict__ P32) {
    for (int q = threadIdx.x; q < kBLEN * kBLEN; q += blockDim.x) {
      const int r = q / kBLEN, c = q % kBLEN;
      const float v = __ldg(P32 + q);
      const uint32_t hi = to_tf32(v);
      s.hi[r][swz(r, c)] = hi;
      s.lo[r][swz(r, c)] = to_tf32(v - __uint_as_float(hi));
    }
    Ph = s.hi;
    Pl = s.lo;
  }
  template <class SM>
  __device__ __forceinline__ static float (*rows(SM& sm, int buf))[kPad] { return sm.tile.f[buf]; }
  __device__ __forceinline__ void apply(const float (*tile)[kPad], int w, int lane, int tb, int nvalid,
                                        float* __restrict__ z) const {
    const int g = lane >> 2, t = lane & 3, m = w & 3, nt = w >> 2;
    float acc[4] = {0.f, 0.f, 0.f, 0.f};
    const float* brow = tile[8 * nt + g];
    const int ra = 16 * m + g, rb = ra + 8;  // ra mod 8 == rb mod 8: one swizzle for both
#pragma unroll
    for (int kk = 0; kk < 8; ++kk) {
      const int c = 8 * kk + t;
      const int c0 = swz(ra, c), c1 = swz(ra, c + 4);
      const uint32_t ahi[4] = {Ph[ra][c0], Ph[rb][c0], Ph[ra][c1], Ph[rb][c1]};
      const uint32_t alo[4] = {Pl[ra][c0], Pl[rb][c0], Pl[ra][c1], Pl[rb][c1]};
      const float x0 = brow[c], x1 = brow[c + 4];
      const uint32_t h0 = to_tf32(x0), h1 = to_tf32(x1);
      const uint32_t l0 = to_tf32(x0 - __uint_as_float(h0)), l1 = to_tf32(x1 - __uint_as_float(h1));
      mma_tf32(acc, alo, h0, h1);
      mma_tf32(acc, ahi, l0, l1);
      mma_tf32(acc, ahi, h0, h1);
    }
    const int n0 = 8 * nt + 2 * t, n1 = n0 + 1;
    const int r0 = 16 * m + g, r1 = r0 + 8;
    if (n0 < nvalid) {
      z[(tb + n0) * kBLEN + r0] = acc[0];
      z[(tb + n0) * kBLEN + r1] = acc[2];
    }
    if (n1 < nvalid) {
      z[(tb + n1) * kBLEN + r0] = acc[1];
      z[(tb + n1) * kBLEN + r1] = acc[3];
    }
  }
};

// ----------------------------------------------------- iteration core -----

// bMeanConstraint (BiCGSTAB.cu:393-410, ExpAMRSolver.cpp:251-256, 340-346):
// the SpMV's row `mean_row` is replaced by sum_i h_i^2 v_i over the operand v
// and the right-hand side reads 0 there.  Each CTA adds the h^2-weighted sum
// of its own blocks of v (this thread's share).
template <class T>
__device__ __forceinline__ double hsum_part(const MeshView& M, const T* __restrict__ v, int b0, int b1) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  double a = 0.0;
  for (int blk = b0 + w; blk < b1; blk += kWarps) {
    const double hb = __ldg(M.hblk + blk);
    const int o = blk * kBLEN;
    a += ((double)__ldcg(v + o + lane) + (double)__ldcg(v + o + lane + 32)) * (hb * hb);
  }
  return a;
}

__device__ __forceinline__ bool owns_row(int row, int b0, int b1) { return row >= b0 * kBLEN && row < b1 * kBLEN; }

// Whether this CTA's SpMV computes row `row`: a cell on a coarse/fine face
// (its block's explicit mask bit set; possible for the corner cell across a
// periodic edge) is an explicit row, computed by the CTA whose row range
// [r0, r1) holds it; any other cell by the owner of its block.
__device__ __forceinline__ bool computes_row(const MeshView& M, int row, int b0, int b1, int r0, int r1) {
  const int blk = row / kBLEN, c = row % kBLEN;
  const unsigned long long m = __ldg(M.xmask + blk);
  if ((m >> c) & 1ull) {
    const int xr = __ldg(M.xbase + blk) + __popcll(m & ((1ull << c) - 1ull));
    return xr >= r0 && xr < r1;
  }
  return owns_row(row, b0, b1);
}

struct IterState {
  double rho, nr, nrh;  // (rhat,r), |r|^2, |rhat|^2 of the current residual
  double err_init;      // L-inf norm the relative test divides by
  double err_opt;       // best residual norm seen (FP64: recursive; mixed: true)
  double err_true;      // mixed: last true residual |b - A x|_inf
  int restarts;
  int iters;
  int updates;          // mixed: true-residual replacements
  int status;
  bool best_is_x;
};

__device__ __forceinline__ double dprod(double a, double b) { return a * b; }
__device__ __forceinline__ double dprod(float a, float b) { return (double)a * (double)b; }

// SpMV epilogue of pass B: nu = y, (rhat, nu).
template <class T>
struct EpiRhNu {
  static constexpr int LV = Lane<T>::V;
  const T* rh;
  T* nu;
  double acc;
  struct Pre {
    T v[LV];  // rhat
  };
  __device__ __forceinline__ Pre load(int i0) const {
    Pre p;
    ldv<LV>(rh + i0, p.v);
    return p;
  }
  __device__ __forceinline__ Pre load1(int i) const {
    Pre p{};
    p.v[0] = __ldcg(rh + i);
    return p;
  }
  __device__ __forceinline__ void vec(int i0, const T (&y)[LV], const Pre& p) {
    stv<LV>(nu + i0, y);
#pragma unroll
    for (int j = 0; j < LV; ++j) acc += dprod(p.v[j], y[j]);
  }
  __device__ __forceinline__ void one(int i, T y, const Pre& p, int j) {
    nu[i] = y;
    acc += dprod(p.v[j], y);
  }
};

// SpMV epilogue of pass D: t = y, (t, s), (t, t).
template <class T>
struct EpiTS {
  static constexpr int LV = Lane<T>::V;
  const T* s;
  T* t;
  double ts, tt;
  struct Pre {
    T v[LV];  // s
  };
  __device__ __forceinline__ Pre load(int i0) const {
    Pre p;
    ldv<LV>(s + i0, p.v);
    return p;
  }
  __device__ __forceinline__ Pre load1(int i) const {
    Pre p{};
    p.v[0] = __ldcg(s + i);
    return p;
  }
  __device__ __forceinline__ void vec(int i0, const T (&y)[LV], const Pre& p) {
    stv<LV>(t + i0, y);
#pragma unroll
    for (int j = 0; j < LV; ++j) {
      ts += dprod(y[j], p.v[j]);
      tt += dprod(y[j], y[j]);
    }
  }
  __device__ __forceinline__ void one(int i, T y, const Pre& p, int j) {
    t[i] = y;
    ts += dprod(y, p.v[j]);
    tt += dprod(y, y);
  }
};

// Mixed form: r = (b - mean_b) - A x in FP64, stored as FP32 (and as rhat
// when set_rh); partials |r64|_inf, (rhat,r), |r|^2, |rhat|^2, |r32|_inf.
template <class SM>
__device__ __forceinline__ void true_residual(SM& sm, const MeshView& M, const double* __restrict__ b,
                                              double mean_b, const double* __restrict__ x, float* __restrict__ r,
                                              float* __restrict__ rh, bool set_rh, double* __restrict__ red,
                                              int b0, int b1, int r0, int r1) {
  struct Epi {
    const double* b;
    double mean_b;
    float* r;
    float* rh;
    bool set_rh;
    double v[5];
    struct Pre {
      double b[2];
      float rh[2];
    };
    __device__ __forceinline__ Pre load(int i0) const {
      Pre p;
      ldv<2>(b + i0, p.b);
      if (set_rh) p.rh[0] = p.rh[1] = 0.f;
      else ldv<2>(rh + i0, p.rh);
      return p;
    }
    __device__ __forceinline__ Pre load1(int i) const {
      Pre p{};
      p.b[0] = __ldg(b + i);
      if (!set_rh) p.rh[0] = __ldcg(rh + i);
      return p;
    }
    __device__ __forceinline__ float acc(double y, double bi, float rhi) {
      const double r64 = (bi - mean_b) - y;
      const float r32 = (float)r64;
      const float rhv = set_rh ? r32 : rhi;
      v[0] = nanmax(v[0], fabs(r64));
      v[1] += dprod(rhv, r32);
      v[2] += dprod(r32, r32);
      v[3] += dprod(rhv, rhv);
      v[4] = nanmax(v[4], fabs((double)r32));
      return r32;
    }
    __device__ __forceinline__ void vec(int i0, const double (&y)[2], const Pre& p) {
      float rr[2];
      rr[0] = acc(y[0], p.b[0], p.rh[0]);
      rr[1] = acc(y[1], p.b[1], p.rh[1]);
      stv<2>(r + i0, rr);
      if (set_rh) stv<2>(rh + i0, rr);
    }
    __device__ __forceinline__ void one(int i, double y, const Pre& p, int j) {
      const float r32 = acc(y, p.b[j], p.rh[j]);
      r[i] = r32;
      if (set_rh) rh[i] = r32;
    }
  } epi{b, mean_b, r, rh, set_rh, {0.0, 0.0, 0.0, 0.0, 0.0}};
  spmv_range<double>(M, x, b0, b1, r0, r1, epi, spmv_row(sm));
  cta_partials<5>(sm, epi.v, 0x11u, red, Q_RU);
}

struct MixedCtx {  // what the reliable update needs
  const double* b;
  double mean_b;
  double delta;
  double tol_abs, tol_rel;
  bool restart;  // restart the recurrences at each replacement
};

// Runs BiCGSTABSolver::main's loop from a prepared state (r, rhat = r,
// st.rho/nr/nrh/err_init set, p = nu = 0 implied).  T is the Krylov type,
// X the solution type; RU enables the mixed form's true-residual
// replacement; MC the mean constraint (FP64 only).  Returns false if a
// barrier gave up.
template <class T, bool RU, bool MC>
__device__ bool bicgstab_loop(Smem<T>& sm, GridBarrier& B, const Pinv<T>& pin, const Problem<T>& V,
                              double* __restrict__ red, int b0, int b1, int r0, int r1, const SolveParams& sp,
                              const MixedCtx& mx, IterState& st) {
  static_assert(!(MC && RU), "the mean constraint runs in the FP64 form only");
  using X = double;
  const MeshView& M = V.M;
  constexpr int TB = Pinv<T>::kTile;
  constexpr int LV = Lane<T>::V, CB = Lane<T>::CB;  // 16-byte lane layout
  static_assert(TB == CB * kWarps, "one chunk of each tile per warp");
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const Lane<T> L(lane);
  const double eps = 1e-21;
  // MC: the CTA whose SpMV computes the mean row records that row's own
  // product (its partials subtract it and add the sum h^2 v in its place)
  const bool rec_mean = MC && computes_row(M, sp.mean_row, b0, b1, r0, r1);
  double rho_prev = 1.0, alpha = 1.0, omega = 1.0, beta;
  bool zero_pnu = true;
  double rho = st.rho, nr = st.nr, nrh = st.nrh;
  double rmax_since = sqrt(nr);  // largest |r|_2 since the last true residual
  int since = 0;                 // iterations since the last true residual
  int k;
  st.status = CUP2D_NOT_CONVERGED;
  for (k = 0; k < sp.max_iter; ++k) {
    // scalar step (BiCGSTAB.cu:471-509)
    const bool serious_breakdown = rho * rho < 1e-16 * nr * nrh;
    beta = (rho / (rho_prev + eps)) * (alpha / (omega + eps));
    bool restart_now = false;
    if (serious_breakdown && sp.max_restarts > 0) {
      ++st.restarts;
      if (st.restarts >= sp.max_restarts) { st.status = CUP2D_BREAKDOWN_LIMIT; break; }
      restart_now = true;
      rho = nr;  // |rhat|^2 after rhat = r
      nrh = nr;
      zero_pnu = true;
      rho_prev = 1.0; alpha = 1.0; omega = 1.0;
      beta = (rho / (rho_prev + eps)) * (alpha / (omega + eps));
    }
    const T tb_beta = (T)beta, tb_omega = (T)omega;
    // pass A: p = r + beta (p - omega nu); z = P^-1 p.  Warp w stages chunk w
    // of each tile and loads its operands of the next tile before the
    // tensor-core apply of the current one, so the loads overlap the apply.
    {
      T rr[LV], pp[LV], nn[LV];
      auto load = [&](int tb) {
        const int blk = tb + w * CB + L.bl;
        if (blk < b1) {
          const int i0 = blk * kBLEN + L.cell0;
          ldv<LV>(V.r + i0, rr);
          if (!zero_pnu) {
            ldv<LV>(V.p + i0, pp);
            ldv<LV>(V.nu + i0, nn);
          }
        }
      };
      int buf = 0;
      if (b0 < b1) load(b0);
      for (int tb = b0; tb < b1; tb += TB) {
        const int nvalid = (int)imin64(TB, b1 - tb);
        auto tile = Pinv<T>::rows(sm, buf);
        const int j = w * CB + L.bl;
        T pv[LV];
        if (j < nvalid) {
          const int i0 = (tb + j) * kBLEN + L.cell0;
#pragma unroll
          for (int k = 0; k < LV; ++k) pv[k] = zero_pnu ? rr[k] : rr[k] + tb_beta * (pp[k] - tb_omega * nn[k]);
          if (restart_now) stv<LV>(V.rh + i0, rr);
          stv<LV>(V.p + i0, pv);
        } else {
#pragma unroll
          for (int k = 0; k < LV; ++k) pv[k] = T(0);
        }
        stv<LV>(&tile[j][L.cell0], pv);
        if (tb + TB < b1) load(tb + TB);
        __syncthreads();
        pin.apply(tile, w, lane, tb, nvalid, V.z);
        buf ^= 1;
      }
      zero_pnu = false;
    }
    if (!B.sync(&sm.flag, 1)) return false;
    // pass B: nu = A z; (rhat, nu)
    {
      EpiRhNu<T> epi{V.rh, V.nu, 0.0};
      spmv_range_staged<T>(M, V.z, V.rh, b0, b1, r0, r1, epi, spmv_stage(sm));
      if constexpr (MC) {
        // the mean row's own product and rhat, to swap in sum h^2 z below
        double v[4] = {epi.acc, hsum_part(M, V.z, b0, b1), 0.0, 0.0};
        __syncthreads();
        if (threadIdx.x == 0 && rec_mean) {
          const T y = __ldcg(V.nu + sp.mean_row), rv = __ldcg(V.rh + sp.mean_row);
          v[2] = dprod(rv, y);
          v[3] = (double)rv;
        }
        cta_partials<4>(sm, v, 0u, red, Q_MB);
      } else {
        const double v[1] = {epi.acc};
        cta_partials<1>(sm, v, 0u, red, Q_RHNU);
      }
    }
    if (!B.sync(&sm.flag, 2)) return false;
    double rhnu;
    if constexpr (MC) {
      grid_reduce<4>(sm, 0u, red, Q_MB);
      const T m = (T)sm.gres[1];
      rhnu = (sm.gres[0] - sm.gres[2]) + sm.gres[3] * (double)m;
      if (threadIdx.x == 0 && owns_row(sp.mean_row, b0, b1)) V.nu[sp.mean_row] = m;
      __syncthreads();
    } else {
      grid_reduce<1>(sm, 0u, red, Q_RHNU);
      rhnu = sm.gres[0];
    }
    alpha = rho / (rhnu + eps);
    const T ta = (T)alpha;
    // pass C: s = r - alpha nu (in place of r); z2 = P^-1 s
    {
      T rr[LV], nn[LV];
      auto load = [&](int tb) {
        const int blk = tb + w * CB + L.bl;
        if (blk < b1) {
          const int i0 = blk * kBLEN + L.cell0;
          ldv<LV>(V.r + i0, rr);
          ldv<LV>(V.nu + i0, nn);
        }
      };
      int buf = 0;
      if (b0 < b1) load(b0);
      for (int tb = b0; tb < b1; tb += TB) {
        const int nvalid = (int)imin64(TB, b1 - tb);
        auto tile = Pinv<T>::rows(sm, buf);
        const int j = w * CB + L.bl;
        T sv[LV];
        if (j < nvalid) {
          const int i0 = (tb + j) * kBLEN + L.cell0;
#pragma unroll
          for (int k = 0; k < LV; ++k) sv[k] = rr[k] - ta * nn[k];
          stv<LV>(V.r + i0, sv);
        } else {
#pragma unroll
          for (int k = 0; k < LV; ++k) sv[k] = T(0);
        }
        stv<LV>(&tile[j][L.cell0], sv);
        if (tb + TB < b1) load(tb + TB);
        __syncthreads();
        pin.apply(tile, w, lane, tb, nvalid, V.z2);
        buf ^= 1;
      }
    }
    if (!B.sync(&sm.flag, 3)) return false;
    // pass D: t = A z2; (t,s), (t,t)
    {
      EpiTS<T> epi{V.r, V.t, 0.0, 0.0};
      spmv_range_staged<T>(M, V.z2, V.r, b0, b1, r0, r1, epi, spmv_stage(sm));
      if constexpr (MC) {
        double v[6] = {epi.ts, epi.tt, hsum_part(M, V.z2, b0, b1), 0.0, 0.0, 0.0};
        __syncthreads();
        if (threadIdx.x == 0 && rec_mean) {
          const T y = __ldcg(V.t + sp.mean_row), sv = __ldcg(V.r + sp.mean_row);
          v[3] = dprod(y, sv);
          v[4] = dprod(y, y);
          v[5] = (double)sv;
        }
        cta_partials<6>(sm, v, 0u, red, Q_MD);
      } else {
        const double v[2] = {epi.ts, epi.tt};
        cta_partials<2>(sm, v, 0u, red, Q_TS);
      }
    }
    if (!B.sync(&sm.flag, 4)) return false;
    if constexpr (MC) {
      grid_reduce<6>(sm, 0u, red, Q_MD);
      const T m = (T)sm.gres[2];
      const double ts = (sm.gres[0] - sm.gres[3]) + sm.gres[5] * (double)m;
      const double tt = (sm.gres[1] - sm.gres[4]) + dprod(m, m);
      omega = ts / (tt + eps);
      if (threadIdx.x == 0 && owns_row(sp.mean_row, b0, b1)) V.t[sp.mean_row] = m;
      __syncthreads();
    } else {
      grid_reduce<2>(sm, 0u, red, Q_TS);
      omega = sm.gres[0] / (sm.gres[1] + eps);
    }
    const T to = (T)omega;
    // pass E: x += alpha z, then x += omega z2 (the reference's two axpys,
    // fused into one pass); r = s - omega t; norms.  The best iterate is
    // saved lazily here: x still holds the previous iterate.  One chunk per
    // warp step: two chunks in flight kept twice the vectors live across the
    // loads, and the spills this forced slowed every pass of the kernel
    // (measured: 12 % on the mixed batch, 20 % on a large FP64 solve).
    {
      double v[4] = {0.0, 0.0, 0.0, 0.0};
      const int nch = (b1 - b0 + CB - 1) / CB;
      for (int c = w; c < nch; c += kWarps) {
        const int blk = b0 + c * CB + L.bl;
        if (blk >= b1) continue;
        const int i0 = blk * kBLEN + L.cell0;
        X xv[LV];
        T zv[LV], z2v[LV], sv[LV], tv[LV], rhv[LV];
        ldv<LV>(V.x + i0, xv);
        ldv<LV>(V.z + i0, zv);
        ldv<LV>(V.z2 + i0, z2v);
        ldv<LV>(V.r + i0, sv);
        ldv<LV>(V.t + i0, tv);
        ldv<LV>(V.rh + i0, rhv);
        if (st.best_is_x) stv<LV>(V.xo + i0, xv);
        X xn[LV];
        T rn[LV];
#pragma unroll
        for (int k = 0; k < LV; ++k) {
          const X x1 = xv[k] + (X)alpha * (X)zv[k];
          xn[k] = x1 + (X)omega * (X)z2v[k];
          rn[k] = sv[k] - to * tv[k];
          v[0] = nanmax(v[0], fabs((double)rn[k]));
          v[1] += dprod(rhv[k], rn[k]);
          v[2] += dprod(rn[k], rn[k]);
          v[3] += dprod(rhv[k], rhv[k]);
        }
        stv<LV>(V.x + i0, xn);
        stv<LV>(V.r + i0, rn);
      }
      cta_partials<4>(sm, v, 0x1u, red, Q_RMAX);
    }
    if (!B.sync(&sm.flag, 5)) return false;
    grid_reduce<4>(sm, 0x1u, red, Q_RMAX);
    double error = sm.gres[0];
    double rho_new = sm.gres[1];
    nr = sm.gres[2];
    nrh = sm.gres[3];
    if (!(error == error) || !(rho_new == rho_new)) {  // non-finite: stop, keep the best iterate
      st.best_is_x = false;
      ++k;
      break;
    }
    bool refreshed = false;
    if constexpr (RU) {
      rmax_since = fmax(rmax_since, sqrt(nr));
      ++since;
      const bool claims = (error <= sp.tol_abs) || (error / st.err_init <= sp.tol_rel);
      // refresh when the FP32 residual dropped by delta, claims convergence,
      // or a sweep stalls for kMaxSweep iterations
      if (claims || sqrt(nr) < mx.delta * rmax_since || since >= kMaxSweep) {
        since = 0;
        // pass E's barrier already ordered every CTA's x update before this
        true_residual(sm, M, mx.b, mx.mean_b, V.x, V.r, V.rh, mx.restart, red, b0, b1, r0, r1);
        if (!B.sync(&sm.flag, 6)) return false;
        grid_reduce<5>(sm, 0x11u, red, Q_RU);
        ++st.updates;
        refreshed = true;
        st.err_true = sm.gres[0];
        rho_new = sm.gres[1];
        nr = sm.gres[2];
        nrh = sm.gres[3];
        error = sm.gres[4];
        rmax_since = sqrt(nr);
        if ((st.err_true <= mx.tol_abs) || (st.err_true / st.err_init <= mx.tol_rel)) {
          st.err_opt = fmin(st.err_opt, st.err_true);
          st.best_is_x = true;
          st.status = CUP2D_OK;
          ++k;
          break;
        }
      }
    }
    // convergence (BiCGSTAB.cu:571-600)
    if constexpr (RU) {
      // mixed: an iterate is judged by its true residual, which only a
      // refresh computes (err_opt is the best true residual so far).  x
      // moves in every pass E, so between refreshes the best iterate is the
      // copy in xo, written by the pass E after the refresh that found it:
      // one copy per refresh, not one per iteration
      st.best_is_x = refreshed && st.err_true < st.err_opt;
      if (st.best_is_x) st.err_opt = st.err_true;
    } else if (error < st.err_opt) {
      st.err_opt = error;
      st.best_is_x = true;
      if ((error <= sp.tol_abs) || (error / st.err_init <= sp.tol_rel)) {
        st.status = CUP2D_OK;
        ++k;
        break;
      }
    } else {
      st.best_is_x = false;
    }
    if (RU && refreshed && mx.restart) {
      // rhat = r was written with the true residual: fresh recurrences
      rho_prev = 1.0; alpha = 1.0; omega = 1.0;
      rho = rho_new;
      zero_pnu = true;
    } else {
      rho_prev = rho;
      rho = rho_new;
    }
  }
  st.iters += k;
  return true;
}

// x -= sum(h^2 x)/sum(h^2) over the CTA's blocks (ExpAMRSolver.cpp:383-415);
// x already holds the final iterate.
template <class SM>
__device__ bool subtract_mean(SM& sm, GridBarrier& B, const MeshView& M, double* __restrict__ x,
                              double* __restrict__ red, int b0, int b1) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  double v[2] = {0.0, 0.0};
  for (int blk = b0 + w; blk < b1; blk += kWarps) {
    const int o = blk * kBLEN;
    const double hb = __ldg(M.hblk + blk);
    v[0] += (__ldcg(x + o + lane) + __ldcg(x + o + lane + 32)) * (hb * hb);
    v[1] += 2.0 * (hb * hb);
  }
  cta_partials<2>(sm, v, 0u, red, Q_HX);
  if (!B.sync(&sm.flag, 7)) return false;
  grid_reduce<2>(sm, 0u, red, Q_HX);
  const double avg = sm.gres[0] / sm.gres[1];
  for (int blk = b0 + w; blk < b1; blk += kWarps) {
    const int o = blk * kBLEN;
    x[o + lane] = __ldcg(x + o + lane) - avg;
    x[o + lane + 32] = __ldcg(x + o + lane + 32) - avg;
  }
  return true;
}

// x <- x_opt when the last iterate was not the best
__device__ __forceinline__ void take_best(bool best_is_x, double* __restrict__ x, const double* __restrict__ xo,
                                          int b0, int b1) {
  if (best_is_x) return;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  for (int blk = b0 + w; blk < b1; blk += kWarps) {
    const int o = blk * kBLEN;
    x[o + lane] = __ldcg(xo + o + lane);
    x[o + lane + 32] = __ldcg(xo + o + lane + 32);
  }
}

// ============================================ one problem, one team ========

template <class SM>
__device__ __forceinline__ void write_stats(const SM& sm, DevStats* stats, const IterState& st, int refinements,
                                            double err_final, double norm_ax0) {
  if (sm.team_rank == 0 && threadIdx.x == 0) {
    stats->status = st.status;
    stats->iterations = st.iters;
    stats->restarts = st.restarts;
    stats->refinements = refinements;
    stats->err_init = st.err_init;
    stats->err_opt = err_final;
    stats->norm_ax0 = norm_ax0;
  }
}

// Plain FP64 solve of one problem by the team: BiCGSTABSolver::main
// (BiCGSTAB.cu:412-620) and the mean removal (ExpAMRSolver.cpp:383-415).
// [b0,b1) is this CTA's block range, [r0,r1) its explicit rows.
// MC: the mean constraint (sp.mean_row).
template <bool MC>
__device__ bool solve_fp64(Smem<double>& sm, GridBarrier& B, const Pinv<double>& pin, const Problem64& pr,
                           const SolveParams& sp, double* __restrict__ red, int b0, int b1, int r0,
                           int r1) {
  const MeshView& M = pr.M;
  double x0sum = 0.0;  // MC: sum h^2 x0, the mean row of A x0
  if constexpr (MC) {
    const double v[1] = {hsum_part(M, pr.x, b0, b1)};
    cta_partials<1>(sm, v, 0u, red, Q_MX);
    if (!B.sync(&sm.flag, 9)) return false;
    grid_reduce<1>(sm, 0u, red, Q_MX);
    x0sum = sm.gres[0];
  }
  // r = b - A x0, rhat = r, |A x0|_inf, |r0|_inf (BiCGSTAB.cu:430-465)
  {
    struct Epi {
      const double* b;
      double* r;
      double* rh;
      int mrow;
      double msum;
      double v[3];
      struct Pre {
        double b[2];
      };
      __device__ __forceinline__ Pre load(int i0) const {
        Pre p;
        ldv<2>(b + i0, p.b);
        return p;
      }
      __device__ __forceinline__ Pre load1(int i) const {
        Pre p{};
        p.b[0] = __ldg(b + i);
        return p;
      }
      __device__ __forceinline__ double acc(double y, double bi) {
        const double rv = bi - y;
        v[0] = nanmax(v[0], fabs(y));
        v[1] = nanmax(v[1], fabs(rv));
        v[2] += rv * rv;
        return rv;
      }
      // the mean row: (A x0) reads sum h^2 x0, b reads 0 (getVec, ExpAMRSolver.cpp:340-346)
      __device__ __forceinline__ double accm(int i, double y, double bi) {
        return (MC && i == mrow) ? acc(msum, 0.0) : acc(y, bi);
      }
      __device__ __forceinline__ void vec(int i0, const double (&y)[2], const Pre& p) {
        double rr[2];
        rr[0] = accm(i0, y[0], p.b[0]);
        rr[1] = accm(i0 + 1, y[1], p.b[1]);
        stv<2>(r + i0, rr);
        stv<2>(rh + i0, rr);
      }
      __device__ __forceinline__ void one(int i, double y, const Pre& p, int j) {
        const double rv = accm(i, y, p.b[j]);
        r[i] = rv;
        rh[i] = rv;
      }
    } epi{pr.b, pr.r, pr.rh, sp.mean_row, x0sum, {0.0, 0.0, 0.0}};
    spmv_range<double>(M, pr.x, b0, b1, r0, r1, epi, spmv_row(sm));
    cta_partials<3>(sm, epi.v, 0x3u, red, Q_INIT);
  }
  if (!B.sync(&sm.flag, 0)) return false;
  grid_reduce<3>(sm, 0x3u, red, Q_INIT);
  IterState st;
  const double norm_ax0 = sm.gres[0];
  st.err_init = sm.gres[1];
  st.err_opt = st.err_init;
  st.err_true = st.err_init;
  st.rho = st.nr = st.nrh = sm.gres[2];
  st.restarts = 0;
  st.iters = 0;
  st.updates = 0;
  st.best_is_x = true;
  st.status = CUP2D_NOT_CONVERGED;
  const MixedCtx none{};
  if (!bicgstab_loop<double, false, MC>(sm, B, pin, pr, red, b0, b1, r0, r1, sp, none, st))
    return false;
  take_best(st.best_is_x, pr.x, pr.xo, b0, b1);
  if (sp.subtract_mean && !subtract_mean(sm, B, M, pr.x, red, b0, b1)) return false;
  write_stats(sm, pr.stats, st, 0, st.err_opt, norm_ax0);
  return true;
}

// Mixed-precision solve of one problem by the team.
__device__ bool solve_mixed(Smem<float>& sm, GridBarrier& B, const Pinv<float>& pin, const ProblemMixed& pr,
                            const SolveParams& sp, double* __restrict__ red, int b0, int b1, int r0,
                            int r1) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  // Neumann compatibility: project b to zero sum (sum b / n)
  {
    double v[1] = {0.0};
    for (int blk = b0 + w; blk < b1; blk += kWarps) {
      const int o = blk * kBLEN;
      v[0] += __ldg(pr.b + o + lane) + __ldg(pr.b + o + lane + 32);
    }
    cta_partials<1>(sm, v, 0u, red, Q_SUMB);
  }
  if (!B.sync(&sm.flag, 8)) return false;
  grid_reduce<1>(sm, 0u, red, Q_SUMB);
  MixedCtx mx;
  mx.b = pr.b;
  mx.mean_b = sm.gres[0] / (double)(pr.M.nb * kBLEN);
  mx.delta = sp.reliable_delta;
  mx.tol_abs = sp.tol_abs;
  mx.tol_rel = sp.tol_rel;
  mx.restart = sp.reliable_restart != 0;
  true_residual(sm, pr.M, pr.b, mx.mean_b, pr.x, pr.r, pr.rh, true, red, b0, b1, r0, r1);
  if (!B.sync(&sm.flag, 0)) return false;
  grid_reduce<5>(sm, 0x11u, red, Q_RU);
  IterState st;
  st.err_init = sm.gres[0];
  st.err_true = sm.gres[0];
  st.err_opt = sm.gres[0];  // best true residual: x0's
  st.rho = sm.gres[1];
  st.nr = sm.gres[2];
  st.nrh = sm.gres[3];
  st.restarts = 0;
  st.iters = 0;
  st.updates = 0;
  st.best_is_x = true;
  st.status = CUP2D_NOT_CONVERGED;
  const bool done0 = st.err_true <= sp.tol_abs || st.err_true == 0.0;
  if (done0) {
    st.status = CUP2D_OK;
  } else if (!bicgstab_loop<float, true, false>(sm, B, pin, pr, red, b0, b1, r0, r1, sp, mx, st)) {
    return false;
  }
  take_best(st.best_is_x, pr.x, pr.xo, b0, b1);
  if (sp.subtract_mean && !subtract_mean(sm, B, pr.M, pr.x, red, b0, b1)) return false;
  write_stats(sm, pr.stats, st, st.updates, st.status == CUP2D_OK ? st.err_true : st.err_opt, 0.0);
  return true;
}

}  // namespace

// The kernels' shared memory (P^-1, staging tiles and SpMV rings, reduction
// scratch) is above the 48 KB of a static allocation: dynamic, sized
// sizeof(Smem<T>) at every launch.
extern __shared__ __align__(16) unsigned char g_solve_smem[];
template <class T>
__device__ __forceinline__ Smem<T>& solve_smem() {
  return *reinterpret_cast<Smem<T>*>(g_solve_smem);
}

// ====================================================== single solves =====

// kSolveCtasPerSm CTAs per SM (2: up to 128 registers, no spills).  With the
// SpMV operands staged in shared memory the spill-free build gained 6-7 % per
// iteration on the large workload and ~10 % on time stepping over 3 CTAs at
// 80 registers (an earlier kernel, gathering its operands into registers,
// had measured 97/95/104 us per iteration at 2/3/4).
__global__ void __launch_bounds__(kSolveThreads, kSolveCtasPerSm) k_bicgstab64(const __grid_constant__ SolveArgs64 S) {
  Smem<double>& sm = solve_smem<double>();
  const int b0 = share(S.prob.M.nb, blockIdx.x, gridDim.x), b1 = share(S.prob.M.nb, blockIdx.x + 1, gridDim.x);
  const int r0 = share(S.prob.M.R, blockIdx.x, gridDim.x), r1 = share(S.prob.M.R, blockIdx.x + 1, gridDim.x);
  GridBarrier B{S.bar, S.abort_flag, gridDim.x, globaltimer_ns() + S.timeout_ns, 0u, S.prof, globaltimer_ns()};
  if (threadIdx.x == 0) {
    sm.team_rank = blockIdx.x;
    sm.team_size = gridDim.x;
  }
  Pinv<double> pin;
  pin.load(sm.P, S.P, nullptr);
  __syncthreads();
  solve_fp64<false>(sm, B, pin, S.prob, S.sp, S.red, b0, b1, r0, r1);
}

// With bMeanConstraint: the same solve on the system whose row S.sp.mean_row
// is sum h^2 x = 0.
__global__ void __launch_bounds__(kSolveThreads, kSolveCtasPerSm)
    k_bicgstab64_mean(const __grid_constant__ SolveArgs64 S) {
  Smem<double>& sm = solve_smem<double>();
  const int b0 = share(S.prob.M.nb, blockIdx.x, gridDim.x), b1 = share(S.prob.M.nb, blockIdx.x + 1, gridDim.x);
  const int r0 = share(S.prob.M.R, blockIdx.x, gridDim.x), r1 = share(S.prob.M.R, blockIdx.x + 1, gridDim.x);
  GridBarrier B{S.bar, S.abort_flag, gridDim.x, globaltimer_ns() + S.timeout_ns, 0u, S.prof, globaltimer_ns()};
  if (threadIdx.x == 0) {
    sm.team_rank = blockIdx.x;
    sm.team_size = gridDim.x;
  }
  Pinv<double> pin;
  pin.load(sm.P, S.P, nullptr);
  __syncthreads();
  solve_fp64<true>(sm, B, pin, S.prob, S.sp, S.red, b0, b1, r0, r1);
}

__global__ void __launch_bounds__(kSolveThreads, kSolveCtasPerSm) k_bicgstab_mixed(const __grid_constant__ SolveArgsMixed S) {
  Smem<float>& sm = solve_smem<float>();
  const int b0 = share(S.prob.M.nb, blockIdx.x, gridDim.x), b1 = share(S.prob.M.nb, blockIdx.x + 1, gridDim.x);
  const int r0 = share(S.prob.M.R, blockIdx.x, gridDim.x), r1 = share(S.prob.M.R, blockIdx.x + 1, gridDim.x);
  GridBarrier B{S.bar, S.abort_flag, gridDim.x, globaltimer_ns() + S.timeout_ns, 0u, S.prof, globaltimer_ns()};
  if (threadIdx.x == 0) {
    sm.team_rank = blockIdx.x;
    sm.team_size = gridDim.x;
  }
  Pinv<float> pin;
  pin.load(sm.P, nullptr, S.P32);
  __syncthreads();
  solve_mixed(sm, B, pin, S.prob, S.sp, S.red, b0, b1, r0, r1);
}


// The server's instances of the two single solves: the same bodies at
// kServedCtasPerSm CTAs per SM.
__global__ void __launch_bounds__(kSolveThreads, kServedCtasPerSm)
    k_bicgstab64_served(const __grid_constant__ SolveArgs64 S) {
  Smem<double>& sm = solve_smem<double>();
  const int b0 = share(S.prob.M.nb, blockIdx.x, gridDim.x), b1 = share(S.prob.M.nb, blockIdx.x + 1, gridDim.x);
  const int r0 = share(S.prob.M.R, blockIdx.x, gridDim.x), r1 = share(S.prob.M.R, blockIdx.x + 1, gridDim.x);
  GridBarrier B{S.bar, S.abort_flag, gridDim.x, globaltimer_ns() + S.timeout_ns, 0u, S.prof, globaltimer_ns()};
  if (threadIdx.x == 0) {
    sm.team_rank = blockIdx.x;
    sm.team_size = gridDim.x;
  }
  Pinv<double> pin;
  pin.load(sm.P, S.P, nullptr);
  __syncthreads();
  solve_fp64<false>(sm, B, pin, S.prob, S.sp, S.red, b0, b1, r0, r1);
}

__global__ void __launch_bounds__(kSolveThreads, kServedCtasPerSm)
    k_bicgstab_mixed_served(const __grid_constant__ SolveArgsMixed S) {
  Smem<float>& sm = solve_smem<float>();
  const int b0 = share(S.prob.M.nb, blockIdx.x, gridDim.x), b1 = share(S.prob.M.nb, blockIdx.x + 1, gridDim.x);
  const int r0 = share(S.prob.M.R, blockIdx.x, gridDim.x), r1 = share(S.prob.M.R, blockIdx.x + 1, gridDim.x);
  GridBarrier B{S.bar, S.abort_flag, gridDim.x, globaltimer_ns() + S.timeout_ns, 0u, S.prof, globaltimer_ns()};
  if (threadIdx.x == 0) {
    sm.team_rank = blockIdx.x;
    sm.team_size = gridDim.x;
  }
  Pinv<float> pin;
  pin.load(sm.P, nullptr, S.P32);
  __syncthreads();
  solve_mixed(sm, B, pin, S.prob, S.sp, S.red, b0, b1, r0, r1);
}

// ========================================================= batches ========
//
// Many independent problems in one cooperative launch.  The grid is split
// into groups of `team` consecutive CTAs; each group takes problems from a
// shared queue (largest first, so the tail is short) and solves each one
// with the same code as a single solve, synchronising on its own bounded
// barrier.  All groups share the abort flag: a timeout anywhere ends the
// launch.

template <bool MIXED>
__device__ __forceinline__ void batch_body(const BatchArgs& A) {
  using KT = typename std::conditional<MIXED, float, double>::type;
  Smem<KT>& sm = solve_smem<KT>();
  const int team = A.team;
  const int g = blockIdx.x / team, rank = blockIdx.x % team;
  GridBarrier B{A.bars + g, A.abort_flag, (unsigned)team, globaltimer_ns() + A.timeout_ns, 0u, A.prof,
                globaltimer_ns()};
  if (threadIdx.x == 0) {
    sm.team_rank = rank;
    sm.team_size = team;
  }
  typename std::conditional<MIXED, Pinv<float>, Pinv<double>>::type pin;
  pin.load(sm.P, A.P, A.P32);
  __syncthreads();
  double* red = A.red + (size_t)g * kRedQ * team;
  while (true) {
    if (rank == 0 && threadIdx.x == 0) A.slots[g] = atomicAdd(A.queue, 1);
    if (!B.sync(&sm.flag, 9)) return;
    unsigned long long t_begin = 0;
    if (threadIdx.x == 0) {
      t_begin = globaltimer_ns();
      sm.slot = __ldcg(A.slots + g);
    }
    __syncthreads();
    const int q = sm.slot;
    if (q >= A.nprob) return;
    const int p = __ldg(A.order + q);
    bool ok;
    if constexpr (MIXED) {
      const ProblemMixed& pr = A.pmx[p];
      const int b0 = share(pr.M.nb, rank, team), b1 = share(pr.M.nb, rank + 1, team);
      const int r0 = share(pr.M.R, rank, team), r1 = share(pr.M.R, rank + 1, team);
      ok = solve_mixed(sm, B, pin, pr, A.sp, red, b0, b1, r0, r1);
    } else {
      const Problem64& pr = A.p64[p];
      const int b0 = share(pr.M.nb, rank, team), b1 = share(pr.M.nb, rank + 1, team);
      const int r0 = share(pr.M.R, rank, team), r1 = share(pr.M.R, rank + 1, team);
      ok = solve_fp64<false>(sm, B, pin, pr, A.sp, red, b0, b1, r0, r1);
    }
    if (!ok) return;
    if (rank == 0 && threadIdx.x == 0) {
      DevStats* ds = MIXED ? A.pmx[p].stats : A.p64[p].stats;
      ds->t_begin = t_begin;
      ds->t_end = globaltimer_ns();
    }
  }
}

__global__ void __launch_bounds__(kSolveThreads, kBatch64CtasPerSm) k_bicgstab_batch64(const __grid_constant__ BatchArgs A) {
  batch_body<false>(A);
}

__global__ void __launch_bounds__(kSolveThreads, kBatchMixedCtasPerSm) k_bicgstab_batch_mixed(const __grid_constant__ BatchArgs A) {
  batch_body<true>(A);
}

// ------------------------------------------------------------ launch -----

namespace {
constexpr int kNumSolveFns = 7;
const void* const kSolveFns[kNumSolveFns] = {(const void*)k_bicgstab64,        (const void*)k_bicgstab_mixed,
                                             (const void*)k_bicgstab_batch64,  (const void*)k_bicgstab_batch_mixed,
                                             (const void*)k_bicgstab64_mean,   (const void*)k_bicgstab64_served,
                                             (const void*)k_bicgstab_mixed_served};
// CTAs per SM each kernel is built for
const int kSolveFnCtas[kNumSolveFns] = {kSolveCtasPerSm,  kSolveCtasPerSm,  kBatch64CtasPerSm, kBatchMixedCtasPerSm,
                                        kSolveCtasPerSm,  kServedCtasPerSm, kServedCtasPerSm};

size_t smem_bytes(const void* fn) {
  return (fn == kSolveFns[1] || fn == kSolveFns[3] || fn == kSolveFns[6]) ? sizeof(Smem<float>)
                                                                           : sizeof(Smem<double>);
}

// Allows the dynamic shared memory of a solve kernel on the current device
// (once per device and kernel) and asks for the smallest shared-memory
// carve-out that holds the CTAs per SM it is built for (kSolveFnCtas), so
// that the rest of the
// unified array stays L1.
cudaError_t allow_smem(const void* fn) {
  static unsigned done[64] = {};
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  int k = 0;
  while (k < kNumSolveFns && kSolveFns[k] != fn) ++k;
  const unsigned bit = 1u << k;
  if (dev >= 0 && dev < 64 && (__atomic_load_n(&done[dev], __ATOMIC_ACQUIRE) & bit)) return cudaSuccess;
  const size_t bytes = smem_bytes(fn);
  e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
  int per_sm = 0, reserved = 0;
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&per_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&reserved, cudaDevAttrReservedSharedMemoryPerBlock, dev);
  if (e == cudaSuccess && per_sm > 0) {
    const int ctas = k < kNumSolveFns ? kSolveFnCtas[k] : kSolveCtasPerSm;
    const size_t need = (size_t)ctas * (bytes + (size_t)reserved);
    const int pct = (int)std::min<size_t>(100, (need * 100 + per_sm - 1) / (size_t)per_sm);
    e = cudaFuncSetAttribute(fn, cudaFuncAttributePreferredSharedMemoryCarveout, pct);
  }
  if (e == cudaSuccess && dev >= 0 && dev < 64) __atomic_fetch_or(&done[dev], bit, __ATOMIC_ACQ_REL);
  return e;
}

// The largest co-resident grid of a solve kernel on a device: queried once
// per device and kernel (handles are created often, e.g. by a server).
int coop_grid_query(const void* fn, int device) {
  int sms = 0, per_sm = 0, cur = 0;
  if (cudaGetDevice(&cur) != cudaSuccess) return 0;
  if (cur != device && cudaSetDevice(device) != cudaSuccess) return 0;
  const bool ok = allow_smem(fn) == cudaSuccess &&
                  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) == cudaSuccess &&
                  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, kSolveThreads, smem_bytes(fn)) ==
                      cudaSuccess;
  if (cur != device) cudaSetDevice(cur);
  return ok ? sms * per_sm : 0;
}

int coop_grid(const void* fn, int device) {
  static std::atomic<int> cache[64][kNumSolveFns];
  int k = 0;
  while (k < kNumSolveFns && kSolveFns[k] != fn) ++k;
  if (device < 0 || device >= 64 || k == kNumSolveFns) return coop_grid_query(fn, device);
  int g = cache[device][k].load(std::memory_order_acquire);
  if (g > 0) return g;
  g = coop_grid_query(fn, device);
  if (g > 0) cache[device][k].store(g, std::memory_order_release);
  return g;
}
}  // namespace

int max_coop_grid_fp64(int device, bool served) {
  return coop_grid(served ? (const void*)k_bicgstab64_served : (const void*)k_bicgstab64, device);
}
int max_coop_grid_mixed(int device, bool served) {
  return coop_grid(served ? (const void*)k_bicgstab_mixed_served : (const void*)k_bicgstab_mixed, device);
}

int max_coop_grid_mean(int device) { return coop_grid((const void*)k_bicgstab64_mean, device); }

cudaError_t launch_bicgstab64(const SolveArgs64& a, int grid, cudaStream_t s, bool served) {
  void* args[] = {const_cast<SolveArgs64*>(&a)};
  const void* fn = a.sp.mean_row >= 0 ? (const void*)k_bicgstab64_mean
                   : served           ? (const void*)k_bicgstab64_served
                                      : (const void*)k_bicgstab64;
  if (cudaError_t e = allow_smem(fn)) return e;
  return cudaLaunchCooperativeKernel(fn, dim3(grid), dim3(kSolveThreads), args, sizeof(Smem<double>), s);
}

cudaError_t launch_bicgstab_mixed(const SolveArgsMixed& a, int grid, cudaStream_t s, bool served) {
  void* args[] = {const_cast<SolveArgsMixed*>(&a)};
  if (a.sp.mean_row >= 0) return cudaErrorInvalidValue;  // FP64 only
  const void* fn = served ? (const void*)k_bicgstab_mixed_served : (const void*)k_bicgstab_mixed;
  if (cudaError_t e = allow_smem(fn)) return e;
  return cudaLaunchCooperativeKernel(fn, dim3(grid), dim3(kSolveThreads), args, sizeof(Smem<float>), s);
}

int max_coop_grid_batch(int device, bool mixed) {
  return coop_grid(mixed ? (const void*)k_bicgstab_batch_mixed : (const void*)k_bicgstab_batch64, device);
}

// Cooperative launch through the extensible launch API, so that a stream
// capture records the cooperative attribute in the graph's kernel node.
cudaError_t launch_bicgstab_batch(const BatchArgs& a, int grid, bool mixed, cudaStream_t s) {
  void* args[] = {const_cast<BatchArgs*>(&a)};
  const void* fn = mixed ? (const void*)k_bicgstab_batch_mixed : (const void*)k_bicgstab_batch64;
  if (cudaError_t e = allow_smem(fn)) return e;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(kSolveThreads);
  cfg.dynamicSmemBytes = smem_bytes(fn);
  cfg.stream = s;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelExC(&cfg, fn, args);
}

// ------------------------------------------------------- single ops -------

__global__ void __launch_bounds__(kSolveThreads) k_precond64(const double* __restrict__ P, int nb,
                                                             const double* __restrict__ p, double* __restrict__ z) {
  __shared__ double tile[8][kPad];
  __shared__ PinvSmem<double> Ps;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  Pinv<double> pin;
  pin.load(Ps, P, nullptr);
  __syncthreads();
  for (int tb = (int)blockIdx.x * 8; tb < nb; tb += (int)gridDim.x * 8) {
    const int nvalid = (int)imin64(8, nb - tb);
    if (w < nvalid) {
      tile[w][lane] = p[(tb + w) * kBLEN + lane];
      tile[w][lane + 32] = p[(tb + w) * kBLEN + lane + 32];
    } else {
      tile[w][lane] = 0.0;
      tile[w][lane + 32] = 0.0;
    }
    __syncthreads();
    pin.apply(tile, w, lane, tb, nvalid, z);
    __syncthreads();
  }
}

cudaError_t launch_precond64(const double* P, int64_t nb, const double* p, double* z, cudaStream_t s) {
  if (nb <= 0) return cudaSuccess;
  const int ctas = (nb + 7) / 8;
  k_precond64<<<(unsigned)(ctas < 65535 ? ctas : 65535), kSolveThreads, 0, s>>>(P, nb, p, z);
  return cudaGetLastError();
}

__global__ void __launch_bounds__(kSolveThreads) k_precond32(const float* __restrict__ P32, int nb,
                                                             const float* __restrict__ p, float* __restrict__ z) {
  __shared__ float tile[16][kPad];
  __shared__ PinvSmem<float> Ps;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  Pinv<float> pin;
  pin.load(Ps, nullptr, P32);
  __syncthreads();
  for (int tb = (int)blockIdx.x * 16; tb < nb; tb += (int)gridDim.x * 16) {
    const int nvalid = (int)imin64(16, nb - tb);
    for (int j = w; j < 16; j += kWarps) {
      tile[j][lane] = j < nvalid ? p[(tb + j) * kBLEN + lane] : 0.f;
      tile[j][lane + 32] = j < nvalid ? p[(tb + j) * kBLEN + lane + 32] : 0.f;
    }
    __syncthreads();
    pin.apply(tile, w, lane, tb, nvalid, z);
    __syncthreads();
  }
}

cudaError_t launch_precond32(const float* P32, int64_t nb, const float* p, float* z, cudaStream_t s) {
  if (nb <= 0) return cudaSuccess;
  const int ctas = (nb + 15) / 16;
  k_precond32<<<(unsigned)(ctas < 65535 ? ctas : 65535), kSolveThreads, 0, s>>>(P32, nb, p, z);
  return cudaGetLastError();
}

}  // namespace cup2d
