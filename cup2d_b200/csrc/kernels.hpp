// Host-side launch interface of the device kernels (internal to the library).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "common.cuh"

namespace cup2d {

constexpr int kMaxLevels = 24;

// The solve kernels access vectors 16 bytes per lane: caller buffers must be
// 16-byte aligned (cudaMalloc gives 256).
inline bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

struct AssembleIn {
  int32_t bpdx, bpdy, level_max, periodic_x, periodic_y;
  int64_t nblocks;
  double h0;  // cell size at level 0
};

// Device buffers of one assembled operator.  Buffers sized by the block
// count are allocated by the owner before assembly; the explicit-row
// buffers are allocated through the callbacks once their sizes are known.
struct DeviceMesh {
  int64_t nb = 0;
  int32_t* level = nullptr;
  int32_t* bx = nullptr;
  int32_t* by = nullptr;
  int32_t* table = nullptr;       // per-level dense leaf tables
  int32_t* nbr = nullptr;         // [4*nb]
  unsigned long long* xmask = nullptr;  // [nb]
  int32_t* xcount = nullptr;      // [nb]
  int32_t* xbase = nullptr;       // [nb+1]
  double* hblk = nullptr;         // [nb]
  int32_t* scan_tmp = nullptr;
  int* err = nullptr;             // [2]: error flag, then the origin block
  int32_t origin = -1;            // leaf at the domain's (0, 0) corner (read back)
  int64_t R = 0, nnz = 0;
  int32_t* rowlen = nullptr;      // [R]
  int32_t* rowcell = nullptr;     // [R]
  int32_t* xptr = nullptr;        // [R+1]
  int32_t* xcol = nullptr;        // [nnz]
  double* xval = nullptr;         // [nnz]
  float* xval32 = nullptr;        // [nnz]
  void* ctx = nullptr;
  int (*alloc_rows)(void* ctx, int64_t R) = nullptr;
  int (*alloc_nnz)(void* ctx, int64_t nnz) = nullptr;

  MeshView view() const {
    MeshView v;
    v.nb = nb;
    v.nbr = nbr;
    v.xmask = xmask;
    v.xbase = xbase;
    v.xptr = xptr;
    v.xcol = xcol;
    v.xval = xval;
    v.xval32 = xval32;
    v.rowcell = rowcell;
    v.R = R;
    v.hblk = hblk;
    return v;
  }
};

// Explicit (coarse/fine) rows of one block at most: the cells on its four faces.
constexpr int64_t kMaxExplicitRowsPerBlock = 28;

int64_t leaf_table_entries(int bpdx, int bpdy, int level_max);
int64_t scan_temp_ints(int64_t n);
int assemble_on_device(const AssembleIn& in, DeviceMesh& out, cudaStream_t s);
cudaError_t launch_build_pinv(double* d_P, cudaStream_t s);
cudaError_t launch_convert_f64_f32(const double* a, float* b, int64_t n, cudaStream_t s);
cudaError_t launch_exclusive_scan(const int32_t* in, int64_t n, int32_t* out, int32_t* tmp, cudaStream_t s);

// ------------------------------------------------------------ solver ----

// Per-solve results written by the persistent kernel (one struct per solve).
struct DevStats {
  int status;        // cup2d_status
  int iterations;
  int restarts;
  int refinements;
  double err_init;
  double err_opt;
  double norm_ax0;
  unsigned long long t_begin, t_end;  // batch: globaltimer ns when the team took / finished the problem
};

constexpr int kRedQ = 20;      // reduction quantities per CTA
constexpr int kRedQMean = 31;  // ... of the FP64 single solve with the mean constraint

// One problem of a solve: its operator, right-hand side, FP64 solution and
// best iterate, and the Krylov vectors (type T: FP64, or FP32 for the mixed
// form) it uses.
template <class T>
struct Problem {
  MeshView M;
  const double* b;
  double* x;
  double* xo;
  T* r;   // residual; s in place between passes C and E
  T* rh;
  T* p;
  T* nu;
  T* t;
  T* z;   // P^-1 p
  T* z2;  // P^-1 s
  DevStats* stats;
};
using Problem64 = Problem<double>;
using ProblemMixed = Problem<float>;

struct SolveParams {
  double tol_abs, tol_rel, reliable_delta;
  int max_restarts, max_iter, subtract_mean, reliable_restart;
  // bMeanConstraint: the cell whose equation is replaced by sum(h^2 x) = 0
  // (its right-hand side read as 0); -1 when off.  Read only by
  // k_bicgstab64_mean.
  int mean_row = -1;
};

// A single solve.  The kernels take these as __grid_constant__ parameters
// and refer to the problem and parameters in place (no per-thread copies).
struct SolveArgs64 {
  Problem64 prob;       // operator, b, x (x0 in, solution out), Krylov vectors
  const double* P;      // 64x64 row-major P^-1
  double* red;          // [kRedQ][grid]
  unsigned* bar;        // arrival counter, zeroed before launch
  int* abort_flag;      // zeroed before launch
  SolveParams sp;
  unsigned long long timeout_ns;
  unsigned long long* prof;  // per-CTA phase timers, or null
};

// Mixed precision: FP32 Krylov vectors, FP64 solution and true residual.
struct SolveArgsMixed {
  ProblemMixed prob;
  const float* P32;     // 64x64 row-major FP32 P^-1 (rounded from the FP64 build)
  double* red;
  unsigned* bar;
  int* abort_flag;
  SolveParams sp;
  unsigned long long timeout_ns;
  unsigned long long* prof;  // per-CTA phase timers, or null
};

// Many problems in one launch: groups of `team` CTAs take problems from a
// queue in `order` (largest first).
struct BatchArgs {
  const Problem64* p64;     // [nprob] (FP64 batches)
  const ProblemMixed* pmx;  // [nprob] (mixed batches)
  const int32_t* order;     // [nprob] queue order
  int nprob;
  int team;                 // CTAs per problem; the grid is a multiple of it
  const double* P;          // FP64 P^-1
  const float* P32;         // FP32 P^-1
  double* red;              // [groups][kRedQ][team]
  unsigned* bars;           // [groups] barrier counters, zeroed
  int* slots;               // [groups]
  int* queue;               // queue head, zeroed
  int* abort_flag;          // zeroed
  SolveParams sp;
  unsigned long long timeout_ns;
  unsigned long long* prof;  // per-CTA phase timers, or null
};

constexpr int kSolveThreads = 256;
// CTAs per SM of the persistent kernels (launch bounds and shared-memory
// carve-out).  Single solves run 2 (128 registers): against 3 (80 registers,
// spilling), on one box, time stepping 16.3 -> 18.3 solves/s (mixed) and
// 19.0 -> 21.0 (FP64), the plain FP64 loop +9 %.  The server's solves run
// their own instances at 3: many small teams in flight need the CTA slots
// (at 2 the server saturated at 95-113 solves/s against 127).
#ifndef CUP2D_CTAS_PER_SM
#define CUP2D_CTAS_PER_SM 2
#endif
constexpr int kSolveCtasPerSm = CUP2D_CTAS_PER_SM;
#ifndef CUP2D_SERVED_CTAS_PER_SM
#define CUP2D_SERVED_CTAS_PER_SM 3
#endif
constexpr int kServedCtasPerSm = CUP2D_SERVED_CTAS_PER_SM;
// The mixed batch kernel: 2 CTAs per SM (128 registers, no spills).  Measured
// on the 512-problem batch, same box, one build against the other: 806-808
// solves/s against 781 at 3 CTAs per SM (team 6 against 8); the FP64 batch
// lost 8.5 % the same way, so it stays at 3.
#ifndef CUP2D_BATCH_MIXED_CTAS_PER_SM
#define CUP2D_BATCH_MIXED_CTAS_PER_SM 2
#endif
constexpr int kBatchMixedCtasPerSm = CUP2D_BATCH_MIXED_CTAS_PER_SM;
#ifndef CUP2D_BATCH64_CTAS_PER_SM
#define CUP2D_BATCH64_CTAS_PER_SM 3
#endif
constexpr int kBatch64CtasPerSm = CUP2D_BATCH64_CTAS_PER_SM;

// Largest co-resident grid of the persistent kernels on this device.
// `served`: the server's instances (kServedCtasPerSm).
int max_coop_grid_fp64(int device, bool served = false);
int max_coop_grid_mixed(int device, bool served = false);
// With a.sp.mean_row >= 0 the FP64 launch runs the mean-constraint variant
// (its red holds kRedQMean quantities per CTA); the mixed form has none.
cudaError_t launch_bicgstab64(const SolveArgs64& a, int grid, cudaStream_t s, bool served = false);
cudaError_t launch_bicgstab_mixed(const SolveArgsMixed& a, int grid, cudaStream_t s, bool served = false);
int max_coop_grid_mean(int device);
int max_coop_grid_batch(int device, bool mixed);
cudaError_t launch_bicgstab_batch(const BatchArgs& a, int grid, bool mixed, cudaStream_t s);

// Single operations (tests, residual checks).
// y = A x (spmv_staged.cu); *err raised if a staged copy did not complete.
cudaError_t launch_spmv64(const MeshView& M, const double* x, double* y, int* err, cudaStream_t s);
cudaError_t launch_spmv32(const MeshView& M, const float* x, float* y, int* err, cudaStream_t s);
cudaError_t launch_precond64(const double* P, int64_t nb, const double* p, double* z, cudaStream_t s);
cudaError_t launch_precond32(const float* P32, int64_t nb, const float* p, float* z, cudaStream_t s);
// The same apply on tcgen05 tensor cores with TMEM accumulators (precond_tc.cu).
cudaError_t launch_precond32_tc(const float* P32, int64_t nb, const float* p, float* z, int* err, cudaStream_t s);

// Forest of a handle on the device: per-block level and coordinates, and the
// per-level dense leaf tables (block id or -1, level l at off[l], row-major
// with (bpdx << l) columns).
struct ForestView {
  int32_t bpdx, bpdy, L;
  int32_t px, py;  // periodic in x / y
  int64_t nb;
  double h0;  // cell size at level 0
  const int32_t* level;
  const int32_t* bx;
  const int32_t* by;
  const int32_t* table;
  int64_t off[kMaxLevels + 1];
};

// Forest adaptation on the device (adapt.cu).  States are dense per-level
// byte arrays at the offsets of the leaf tables.
constexpr int kMaxAdaptDisks = 64;
struct AdaptGeom {
  int32_t bpdx, bpdy, L, px, py;
  double extent;
  int64_t off[kMaxLevels + 1];
};
struct AdaptDisks {
  int32_t n;
  double band;
  double d[kMaxAdaptDisks][3];  // cx, cy, r
};
struct AdaptScratch {
  uint8_t* state;    // [leaf_table_entries]
  int32_t* mark;     // [adapt_key_space]
  int32_t* rank;     // [adapt_key_space + 1]: exclusive prefix sums, then the total
  int32_t* scan_tmp; // [scan_temp_ints(adapt_key_space)]
  int* changed;      // [1]: balance round flag, scatter error flag
};
// Size of the dense Morton key space of a forest's leaves (a power of 4).
int64_t adapt_key_space(int bpdx, int bpdy, int level_max);
// Tags, balances and orders the leaves; returns their number in *nleaves
// (read back: the caller sizes the block arrays with it).  CUP2D_OK,
// CUP2D_CUDA_ERROR, or CUP2D_BAD_MESH if the balance did not settle.
int adapt_build(const AdaptGeom& g, const AdaptDisks& D, const AdaptScratch& sc, int64_t* nleaves,
                cudaStream_t s);
// Writes the nb leaves (level, bx, by) in Morton order (CUP2D_OK, or an error
// status; synchronises the stream).
int adapt_scatter(const AdaptGeom& g, const AdaptScratch& sc, int64_t nb, int32_t* level, int32_t* bx, int32_t* by,
                  cudaStream_t s);

// Time-stepping steps around the solve (timestep.cu).
constexpr int kMaxFourierK = 24;
int fourier_mode_count(int kmax);
int64_t rhs_partials(int64_t nb);  // scratch doubles of launch_rhs_fourier
// b = zero-sum RHS of the Fourier velocity field with coefficients coef
// (device, 4 per mode); partial [rhs_partials(nb)] and mean [1] scratch.
cudaError_t launch_rhs_fourier(const ForestView& F, int kmax, const double* coef, double* b, double* partial,
                               double* mean, cudaStream_t s);
// After the solve of the pressure step (PressureSingle.cpp:853-879):
// pres += pold - (volume-weighted mean of pres), with `partial` scratch of
// wmean_partials(nb) doubles.
int64_t wmean_partials(int64_t nb);
cudaError_t launch_add_pold(double* pres, const double* pold, const double* hblk, int64_t nb, double* partial,
                            cudaStream_t s);
// Pressure projection around the solve (projection.cu), one thread per cell.
// Velocity-like fields hold (u, v) per cell, interleaved, in block-major
// cell order; scalars one double per cell.
//   rhs:  tmp = h/(2dt) (central div vel - chi central div udef)  (vel set)
//         tmp -= 5-point L(pres), pold = pres                       (pres set)
//   correction: vel += -(dt h/2)(central difference of pres) / h^2
// Coarse/fine faces take the fine side's ghosts from the coarse block by
// the quadratic rule of the operator and correct the coarse side's fluxes.
struct ProjFields {
  const double* vel;
  const double* udef;
  const double* chi;
  const double* pres;
  double* tmp;
  double* pold;
};
cudaError_t launch_pressure_rhs(const ForestView& F, const int32_t* nbr, double dt, const ProjFields& f,
                                cudaStream_t s);
cudaError_t launch_pressure_correction(const ForestView& F, const int32_t* nbr, double dt, const double* pres,
                                       double* vel, cudaStream_t s);
// xd (on D) = xs (on S) carried across a change of forest.
cudaError_t launch_transfer(const ForestView& S, const double* xs, const ForestView& D, double* xd,
                            cudaStream_t s);

}  // namespace cup2d
