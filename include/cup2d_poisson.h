/*
 * cup2d_poisson.h — C ABI of the B200 pressure-Poisson solver.
 *
 * Drop-in for CUP2D's GPU Poisson path ("-poissonSolver cuda_iterative"):
 * BiCGSTAB with the shared 64x64 block-Jacobi preconditioner on the 8x8-cell
 * block-AMR forest.  Reference interfaces replaced (paths in the CUP2D tree):
 *
 *   PoissonSolver::solve(const ScalarGrid*, ScalarGrid*)   source/Poisson/Base.h:12
 *   makePoissonSolver(SimulationData&)                      source/Poisson/Base.cpp:8-30
 *   ExpAMRSolver::ExpAMRSolver (P^-1 build)                 source/Poisson/ExpAMRSolver.cpp:25-99
 *   ExpAMRSolver::getMat (assembly, on flux-correction update)
 *                                                           source/Poisson/ExpAMRSolver.cpp:180-313,370-376
 *   ExpAMRSolver::getVec + solve (b, x0, mean removal)      source/Poisson/ExpAMRSolver.cpp:315-416
 *   LocalSpMatDnVec::solveWithUpdate / solveNoUpdate        source/Poisson/LocalSpMatDnVec.cpp:318-332
 *   BiCGSTABSolver::main                                    source/Poisson/BiCGSTAB.cu:412-620
 *
 * Conventions
 *   - Cell vectors are FP64, block-major: v[block*64 + iy*8 + ix], blocks in
 *     the order of the forest passed at creation (CUP2D's blockID order).
 *   - Every entry point returns a cup2d_status; none exits or aborts.
 *   - A handle is not thread-safe; it runs its work on one CUDA stream.
 *   - Pointers named d_* are device pointers on the handle's device, 16-byte
 *     aligned for the solves (cudaMalloc gives 256); the others are host
 *     pointers.  `stream` is a cudaStream_t used as given
 *     (NULL is the legacy default stream, as in the CUDA runtime).  The
 *     host-buffer solve runs on the handle's own stream.
 */
#ifndef CUP2D_POISSON_H
#define CUP2D_POISSON_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum cup2d_status {
  CUP2D_OK = 0,
  CUP2D_NOT_CONVERGED = 1,     /* iteration cap reached; best iterate returned */
  CUP2D_BREAKDOWN_LIMIT = 2,   /* restart cap reached; best iterate returned */
  CUP2D_BAD_MESH = 3,          /* forest not a valid 2:1-balanced leaf set */
  CUP2D_OOM = 4,               /* device allocation failed */
  CUP2D_TIMEOUT = 5,           /* a bounded device-side wait expired */
  CUP2D_CUDA_ERROR = 6,        /* any other CUDA runtime error */
  CUP2D_INVALID_ARGUMENT = 7,
  CUP2D_NO_DEVICE = 8,
  CUP2D_QUEUE_FULL = 9,        /* serving: no slot / memory for the request now */
  CUP2D_PENDING = 10           /* serving: request not finished yet */
} cup2d_status;

typedef enum cup2d_precision {
  CUP2D_PREC_FP64 = 0,   /* plain FP64 BiCGSTAB: the reference's solve */
  CUP2D_PREC_MIXED = 1   /* FP32 Krylov vectors and split-TF32 P^-1; FP64 solution
                            update, true-residual refresh and convergence test */
} cup2d_precision;

/* The block list Cubism hands to ExpAMRSolver::getMat. */
typedef struct cup2d_forest {
  int32_t bpdx, bpdy;            /* root blocks per direction (-bpdx, -bpdy) */
  int32_t level_max;             /* number of levels (-levelMax) */
  int32_t periodic_x, periodic_y;/* 1 periodic, 0 wall (homogeneous Neumann) */
  double extent;                 /* longer domain side (-extent) */
  int64_t nblocks;
  const int32_t* level;          /* [nblocks] refinement level of each block */
  const int32_t* bx;             /* [nblocks] block index at its level, x */
  const int32_t* by;             /* [nblocks] block index at its level, y */
} cup2d_forest;

/* Solver options: SimulationData's Poisson fields plus the additions. */
typedef struct cup2d_solve_opts {
  double tol_abs;          /* sim.PoissonTol (max_error) */
  double tol_rel;          /* sim.PoissonTolRel (max_rel_error) */
  int32_t max_restarts;    /* sim.maxPoissonRestarts */
  int32_t max_iter;        /* BiCGSTAB.cu:468 fixes 1000 */
  int32_t precision;       /* cup2d_precision */
  int32_t subtract_mean;   /* 1: x -= sum(h^2 x)/sum(h^2) after the solve */
  double reliable_delta;   /* mixed: once the FP32 residual has dropped by this factor
                              since the last replacement, replace it by the true FP64
                              residual b - A x */
  int32_t timeout_ms;      /* bound on the device time of a launch, checked at every
                              barrier; a wait for another CTA also ends there */
  int32_t reliable_restart;/* mixed: 1 restarts the BiCGSTAB recurrences (rhat = r,
                              p = nu = 0) at each replacement: FP64 iterative
                              refinement of restarted FP32 BiCGSTAB sweeps whose
                              solution update is accumulated in FP64; 0 keeps the
                              recurrences running (reliable updates) */
  int32_t mean_constraint; /* sim.bMeanConstraint (0 by default): nonzero replaces the
                              equation of cell (0,0) of the leaf at the domain's (0,0)
                              corner by sum(h^2 x) = 0 with right-hand side 0
                              (ExpAMRSolver.cpp:251-256, 340-346; BiCGSTAB.cu:393-410).
                              FP64 single solves and the server only: the mixed
                              precision (whose FP32 sweeps derail on the constrained
                              system), a batch and cup2d_poisson_solve_device_noalloc
                              reject it with CUP2D_INVALID_ARGUMENT. */
} cup2d_solve_opts;

typedef struct cup2d_solve_stats {
  int32_t status;          /* cup2d_status of this solve */
  int32_t iterations;      /* BiCGSTAB iterations (summed over inner solves) */
  int32_t restarts;
  int32_t refinements;     /* mixed: FP64 true-residual replacements taken */
  double err_init;         /* |b - A x0|_inf */
  double err_final;        /* fp64: best recursive |r|_inf (the reference's test);
                              mixed: true |b - A x|_inf in FP64 of the returned
                              x (converged: the final iterate; otherwise the
                              refreshed iterate with the lowest one) */
  double rel_res_inf;      /* err_final / err_init */
  double solve_ms;         /* device time of the solve (CUDA events) */
} cup2d_solve_stats;

typedef struct cup2d_poisson cup2d_poisson;

/* ------------------------------------------------------------ library ---- */
const char* cup2d_version(void);
const char* cup2d_status_string(int status);
void cup2d_default_opts(cup2d_solve_opts* opts);
/* Copies the 64x64 row-major P^-1 = -K^-1 built on the device (FP64). */
int cup2d_pinv(double* P_out);

/* ------------------------------------------------------------ solver ----- */
/* makePoissonSolver + ExpAMRSolver ctor + first getMat: builds P^-1 and the
 * operator on the device. */
int cup2d_poisson_create(const cup2d_forest* forest, const cup2d_solve_opts* opts,
                         cup2d_poisson** out);
/* Re-assembly after mesh adaptation (the UpdateFluxCorrection branch). */
int cup2d_poisson_update_mesh(cup2d_poisson* h, const cup2d_forest* forest);
/* Mesh adaptation on the device, then re-assembly: the role of
 * AdaptTheMesh::adapt (source/Operators/AdaptTheMesh.cpp:80-110: tag, then
 * Cubism's refinement/compression and 2:1 balance) followed by the
 * UpdateFluxCorrection branch of ExpAMRSolver::solve
 * (source/Poisson/ExpAMRSolver.cpp:370-376), for the benchmark's geometric
 * criterion.  The handle's forest is replaced by the one cup2d_mesh_disks
 * builds for the handle's bpdx, bpdy, level_max, extent and periodicity:
 * blocks meeting the band | |p - c| - r | <= band of a disk refined to
 * level_max - 1, 2:1 balanced across faces and corners, Morton-ordered --
 * built on the device (no host forest, one read-back of the block count)
 * and assembled as update_mesh does.  disks: host array of ndisks
 * (cx, cy, r) triples, ndisks <= 64.  *nblocks receives the new block count
 * (NULL to ignore).  Like update_mesh, it waits for the device first. */
int cup2d_poisson_adapt_disks(cup2d_poisson* h, int32_t ndisks, const double* disks, double band,
                              int64_t* nblocks);
/* The handle's current forest, in the block order of its vectors: level and
 * (i, j) index of each of its cup2d_poisson_num_cells/64 blocks (host
 * arrays). */
int cup2d_poisson_get_forest(const cup2d_poisson* h, int32_t* level, int32_t* bx, int32_t* by);
int cup2d_poisson_set_opts(cup2d_poisson* h, const cup2d_solve_opts* opts);
int64_t cup2d_poisson_num_cells(const cup2d_poisson* h);
/* Number of CTAs of the persistent solve kernels (0 = size heuristic).  The
 * launch is clamped to what fits co-resident on the device. */
int cup2d_poisson_set_grid(cup2d_poisson* h, int32_t grid);
int cup2d_poisson_destroy(cup2d_poisson* h);

/* PoissonSolver::solve: b is the RHS (sim.tmp), x holds x0 on entry and the
 * solution on exit (sim.pres).  Host buffers: copies are part of the call. */
int cup2d_poisson_solve(cup2d_poisson* h, const double* b, double* x,
                        cup2d_solve_stats* stats);
/* Same on device buffers, asynchronous on `stream` unless stats != NULL
 * (stats are read back after the solve, which synchronises the stream). */
int cup2d_poisson_solve_device(cup2d_poisson* h, const double* d_b, double* d_x,
                               cup2d_solve_stats* stats, void* stream);

/* The FP64 device solve without any device allocation.  This entry point has
 * no counterpart in the reference.  It is for callers that must not allocate
 * device memory when they solve: an application whose device memory belongs
 * to its own pool allocator, or a time-step loop that cannot afford the
 * device-wide synchronisation cudaMalloc/cudaFree can cause.  The handle's
 * operator (built at create/update time) and the caller's b and x are the
 * inputs and outputs; every scratch buffer of the solve lives in one static
 * device array of 16.2 MiB.  The array is committed on a GPU when the first
 * handle is created there (cup2d_poisson_create looks up its address, which
 * under CUDA's lazy module loading loads and allocates it) and held until
 * exit, so the solve itself loads and allocates nothing.  Limits: at most
 * CUP2D_NOALLOC_MAX_BLOCKS blocks (larger problems return
 * CUP2D_INVALID_ARGUMENT) and always the plain FP64 form.  All calls share
 * the array, which keeps the last call's contents: calls whose GPU work
 * overlaps race, so serialise them.  The handle's device must be current.
 * Otherwise behaves as cup2d_poisson_solve_device. */
#define CUP2D_NOALLOC_MAX_BLOCKS 4096
int cup2d_poisson_solve_device_noalloc(cup2d_poisson* h, const double* d_b, double* d_x,
                                       cup2d_solve_stats* stats, void* stream);

/* Building blocks (device buffers), exposed for parity tests.  The operator
 * apply is the solver's own SpMV, in FP64 and in the FP32 of the mixed form. */
int cup2d_poisson_apply(cup2d_poisson* h, const double* d_x, double* d_y, void* stream);
int cup2d_poisson_apply32(cup2d_poisson* h, const float* d_x, float* d_y, void* stream);
/* Time-stepping steps around the solve, on the device.
 * rhs_fourier_device: d_b = the zero-sum RHS of the synthetic pressure
 * problem on the handle's forest, 0.5 h (u(x+h)-u(x-h) + v(y+h)-v(y-h)) of
 * the Fourier velocity with host coefficients `coef` (cup2d_fourier_coefs /
 * cup2d_fourier_advance layout, kmax 1..24) -- the device counterpart of
 * cup2d_rhs_from_coefs, equal to it to rounding (CUP2D computes the RHS
 * from the velocity field in updatePressureRHS,
 * source/Operators/PressureSingle.cpp:324-456).
 * transfer: d_xdst (on dst's forest) = d_xsrc (on src's forest), for a warm
 * start across a mesh adaptation: same-level cells copied, a finer dst cell
 * takes the coarse src cell holding its centre, a coarser dst cell the mean
 * of the src cells at its four quadrant centres.  Both forests must share
 * bpdx, bpdy and extent.  Asynchronous on `stream`. */
int cup2d_poisson_rhs_fourier_device(cup2d_poisson* h, int32_t kmax, const double* coef, double* d_b,
                                     void* stream);
int cup2d_poisson_transfer(const cup2d_poisson* src, const double* d_xsrc, const cup2d_poisson* dst,
                           double* d_xdst, void* stream);
/* The pressure step around the solve, as PressureSingle::operator() runs it
 * (source/Operators/PressureSingle.cpp:831-879), on device buffers:
 *   pold = pres; tmp -= L(pold); pres = 0            (:836-848, 411-418)
 *   solve L pres = tmp (cup2d_poisson_solve_device)  (:850)
 *   pres += pold - mean(pres), volume-weighted       (:853-879)
 * L(pold) is updatePressureRHS1's 5-point stencil on block labs with the
 * coarse/fine flux correction (the kernel of cup2d_poisson_pressure_rhs; in
 * exact arithmetic the assembled operator).  On entry d_tmp holds the
 * divergence part of the right-hand side (updatePressureRHS) and d_pres the
 * previous pressure; on return d_pres holds the new pressure, d_pold the
 * previous one and d_tmp the right-hand side that was solved.  The three
 * buffers must be distinct.  Asynchronous on `stream` unless stats != NULL,
 * when the solve's statistics are read back (the final update stays
 * queued on the stream). */
int cup2d_poisson_pressure_step(cup2d_poisson* h, double* d_tmp, double* d_pres, double* d_pold,
                                cup2d_solve_stats* stats, void* stream);

/* The field kernels of the pressure projection (source/Operators/
 * PressureSingle.cpp), on device buffers in block-major cell order.
 * Velocity-like fields hold (u, v) per cell, interleaved (Cubism's
 * VectorBlock layout), scalars one double per cell; each buffer holds the
 * handle's ncells cells; velocity-like buffers 16-byte aligned (cudaMalloc
 * gives 256).  Ghost cells follow CUP2D's labs: same-level
 * neighbours, domain edges (velocities: normal component sign-flipped;
 * scalars: copied), coarser neighbours by the operator's quadratic
 * interpolation (ExpAMRSolver.cpp:100-128), and coarse cells next to finer
 * blocks take the fine side's fluxes (Cubism's flux correction).
 *
 * cup2d_poisson_pressure_rhs: everything operator() does before the solve
 * (:826-849).  With d_vel set (then d_udef and d_chi too):
 *   tmp = 0.5 h/dt ((u_E - u_W) + (v_N - v_S))
 *         - 0.5 h/dt chi ((ud_E - ud_W) + (vd_N - vd_S))   (updatePressureRHS)
 * else d_tmp is read as it is.  With d_pres set (then d_pold too):
 *   pold = pres; tmp -= (p_W + p_E + p_S + p_N - 4 p)[pold]; pres = 0
 *                                                       (updatePressureRHS1)
 * At least one of d_vel, d_pres must be set; tmp, pres, pold, vel, udef and
 * chi must not overlap.  Asynchronous on `stream`. */
int cup2d_poisson_pressure_rhs(cup2d_poisson* h, double dt, const double* d_vel, const double* d_udef,
                               const double* d_chi, double* d_pres, double* d_pold, double* d_tmp, void* stream);
/* PressureSingle::pressureCorrection (:123-210): with pFac = -0.5 dt h,
 *   vel += pFac (P_E - P_W, P_N - P_S) / h^2   (flux-corrected at coarse/fine faces).
 * d_pres and d_vel must not overlap.  Asynchronous on `stream`. */
int cup2d_poisson_pressure_correction(cup2d_poisson* h, double dt, const double* d_pres, double* d_vel,
                                      void* stream);
/* The whole pressure projection of PressureSingle::operator() (:826-882)
 * without the obstacle terms: cup2d_poisson_pressure_rhs (velocities and
 * pres), the solve, pres += pold - mean(pres), cup2d_poisson_pressure_correction.
 * On return d_vel holds the projected velocity, d_pres the new pressure,
 * d_pold the previous one, d_tmp the right-hand side that was solved.
 * Statistics as cup2d_poisson_pressure_step. */
int cup2d_poisson_pressure_projection(cup2d_poisson* h, double dt, double* d_vel, const double* d_udef,
                                      const double* d_chi, double* d_pres, double* d_pold, double* d_tmp,
                                      cup2d_solve_stats* stats, void* stream);
int cup2d_poisson_precond(cup2d_poisson* h, const double* d_p, double* d_z, void* stream);
/* FP32 P^-1 apply of the mixed form (split-TF32 tensor-core MMA). */
int cup2d_poisson_precond32(cup2d_poisson* h, const float* d_p, float* d_z, void* stream);
/* The same FP32 P^-1 apply on the 5th-generation tensor cores (tcgen05.mma,
 * accumulators in tensor memory): the cublasDgemm of P_inv
 * (source/Poisson/BiCGSTAB.cu:520,545) in the mixed form's precision,
 * measured beside cup2d_poisson_precond32.  Synchronises the stream;
 * CUP2D_TIMEOUT if the tensor-core work did not complete within 2 s. */
int cup2d_poisson_precond32_tc(cup2d_poisson* h, const float* d_p, float* d_z, void* stream);
/* The assembled operator as CSR (host buffers).  Call with NULL arrays to
 * get n and nnz. */
int cup2d_poisson_export_csr(cup2d_poisson* h, int64_t* n, int64_t* nnz,
                             int64_t* row_ptr, int32_t* col, double* val);
/* Per-phase device timers (the counterpart of DeviceProfiler,
 * source/Utils/DeviceProfiler.cuh:26-108, compiled in with -DBICGSTAB_PROFILER
 * in the reference; here switched at run time).  While enabled, every solve
 * adds, per CTA, the time spent computing each phase and waiting at the grid
 * barrier that ends it.  cup2d_poisson_profile returns the per-CTA averages
 * in ms accumulated since enabling, for phases 0 residual / mean, 1 pass A
 * (p, P^-1), 2 pass B (SpMV), 3 pass C (x, s, P^-1), 4 pass D (SpMV),
 * 5 pass E (x, r, norms), 6 true-residual refresh, 7 mean removal, 8 sum b;
 * nphases >= 10. */
int cup2d_poisson_set_profiling(cup2d_poisson* h, int32_t enable);
int cup2d_poisson_profile(cup2d_poisson* h, double* compute_ms, double* wait_ms, int32_t nphases);
/* Explicit (coarse/fine) rows only: number of rows and non-zeros. */
int cup2d_poisson_explicit_info(cup2d_poisson* h, int64_t* rows, int64_t* nnz);

/* ------------------------------------------------------------- batches ---- */
/* Many independent problems solved in one persistent launch.  No counterpart
 * in the reference, which solves one problem per PoissonSolver::solve call
 * (source/Poisson/Base.h:12); each problem of a batch gets exactly that solve
 * (same operator, same BiCGSTAB, same mean removal).  The grid is split into
 * groups of `team` CTAs that take problems largest first from a device
 * queue, so uneven sizes balance by work, not by count. */
typedef struct cup2d_batch cup2d_batch;
/* Assembles the n operators (one per forest) on the device. */
int cup2d_batch_create(int32_t n, const cup2d_forest* forests, const cup2d_solve_opts* opts,
                       cup2d_batch** out);
int cup2d_batch_set_opts(cup2d_batch* B, const cup2d_solve_opts* opts);
/* CTAs per problem (1..256); 8 by default or $CUP2D_BATCH_TEAM. */
int cup2d_batch_set_team(cup2d_batch* B, int32_t team);
int32_t cup2d_batch_size(const cup2d_batch* B);
int64_t cup2d_batch_num_cells(const cup2d_batch* B, int32_t i);
/* Solves problem i with RHS d_b[i] and initial guess / solution d_x[i]
 * (device pointers, arrays of n host-side entries).  Asynchronous on
 * `stream` unless stats != NULL, in which case stats[0..n-1] are filled
 * after the launch ends (solve_ms: the problem's own span inside the
 * launch, from its team taking it to its solution written). */
int cup2d_batch_solve_device(cup2d_batch* B, const double* const* d_b, double* const* d_x,
                             cup2d_solve_stats* stats, void* stream);
/* CTAs per SM of batched launches (the occupancy cap, 0..32; 0 = as many
 * as fit, the default): smaller caps trade latency hiding for fewer
 * barrier parties and less L2 pressure. */
int cup2d_batch_set_occupancy(cup2d_batch* B, int32_t ctas_per_sm);
/* Autotuner for the launch shape: times a batched launch of every pair
 * (teams[k], ctas_per_sm[c]) -- each problem capped at `iters` iterations,
 * so every candidate does the same work, or with iters = 0 full solves to
 * the batch's tolerance, each from the caller's x; one warm-up launch each
 * -- writes the rates in cell-iterations/s to rates[k*max(ncps,1) + c] (0
 * where the pair does not fit the device), keeps the fastest pair for later
 * solves and returns it.  ncps = 0 tunes the team alone at the current
 * occupancy cap.  x is overwritten. */
int cup2d_batch_tune(cup2d_batch* B, const double* const* d_b, double* const* d_x, const int32_t* teams,
                     int32_t nteams, const int32_t* ctas_per_sm, int32_t ncps, int32_t iters, double* rates,
                     int32_t* best_team, int32_t* best_ctas_per_sm);
/* CUDA-graph form of a batched solve, for repeated solves on the same
 * device buffers (time stepping: new b in place, x warm from the last step).
 * cup2d_batch_capture records one whole solve of d_b/d_x -- state resets,
 * with CUP2D_GRAPH_ZERO_X zeroing every x first, the persistent launch, the
 * read-back of the statistics -- with the options, team and occupancy cap
 * in force at capture time; a new capture replaces the old graph.
 * cup2d_batch_replay enqueues one replay on `stream` (asynchronous);
 * cup2d_batch_replay_stats waits for the last replay and fills stats[0..n-1]
 * as cup2d_batch_solve_device does.  One solve or replay of a batch may be
 * in flight at a time. */
#define CUP2D_GRAPH_ZERO_X 1
int cup2d_batch_capture(cup2d_batch* B, const double* const* d_b, double* const* d_x, int32_t flags);
int cup2d_batch_replay(cup2d_batch* B, void* stream);
int cup2d_batch_replay_stats(cup2d_batch* B, cup2d_solve_stats* stats);
/* Same on host buffers (b[i] the RHS, x[i] initial guess in, solution out);
 * the copies are part of the call, on the batch's own stream. */
int cup2d_batch_solve(cup2d_batch* B, const double* const* b, double* const* x,
                      cup2d_solve_stats* stats);
/* Schedule of the last solve that returned stats: when each problem's team
 * took it and finished it, in ms from the first start, and the launch's
 * duration (CUDA events); for tuning the team size. */
int cup2d_batch_timeline(const cup2d_batch* B, double* begin_ms, double* end_ms, double* launch_ms);
/* Per-phase device timers of batched launches, as cup2d_poisson_profile
 * (per-CTA averages in ms since enabling); phase 9 is the wait for the next
 * problem of the queue. */
int cup2d_batch_set_profiling(cup2d_batch* B, int32_t enable);
int cup2d_batch_profile(cup2d_batch* B, double* compute_ms, double* wait_ms, int32_t nphases);
int cup2d_batch_destroy(cup2d_batch* B);

/* ------------------------------------------------------------- serving ---- */
/* A request server (no counterpart in the reference, which solves one
 * simulation's step per PoissonSolver::solve call, source/Poisson/Base.h:12).
 * Callers register meshes once and submit solves against them from any
 * thread; a worker thread admits requests in submission order as solve slots
 * and device memory free up, keeps each mesh's operator and vectors resident
 * while the memory budget allows (least-recently-used idle meshes are
 * evicted first; one request per mesh runs at a time), and runs every
 * admitted request as its own persistent solve of `team` CTAs on a stream of
 * its own, overlapping with the requests already running.  A request's
 * result is bit-identical to the same solve alone (cup2d_poisson_solve with
 * grid = team).  b is read when the request is admitted and x (x0 in,
 * solution out) is written when it completes: both host buffers must stay
 * valid until then (pinned memory makes the copies asynchronous). */
typedef struct cup2d_server cup2d_server;
typedef struct cup2d_server_opts {
  int32_t max_inflight;      /* solves on the device at once (one stream each); default 24 */
  int32_t team;              /* CTAs per solve; default 16; 0: by mesh size (one CTA per
                                blocks_per_cta blocks, 2..128) */
  int32_t blocks_per_cta;    /* with team 0; default 320 (measured best of 160/256/320/400/640 at saturation) */
  double solve_share;        /* share of the device's co-resident solve CTAs that solves
                                may hold at once (the rest stays free for assembly
                                kernels and copies); default 0.9 */
  int64_t hbm_budget_bytes;  /* device memory for resident meshes; 0: 80% of the free memory */
  cup2d_solve_opts solve;    /* tolerances and precision of every solve */
} cup2d_server_opts;
typedef struct cup2d_server_counters {
  int64_t submitted, admitted, completed, failed, queued, inflight;
  int64_t resident_meshes, evictions, assemblies;
  int64_t resident_bytes, budget_bytes;
  int64_t assembly_us;  /* wall time spent making meshes resident (handle creation + assembly), summed */
} cup2d_server_counters;
/* x0 = this mesh's last solution when it is still resident (else 0); the
 * request's x is then only written. */
#define CUP2D_SUBMIT_WARM_START 1
void cup2d_server_default_opts(cup2d_server_opts* opts);
int cup2d_server_create(const cup2d_server_opts* opts, cup2d_server** out);
/* Copies the forest; the operator is assembled when a request first needs it. */
int cup2d_server_add_mesh(cup2d_server* S, const cup2d_forest* forest, int64_t* mesh_id);
int cup2d_server_submit(cup2d_server* S, int64_t mesh_id, const double* b, double* x, int32_t flags,
                        int64_t* request_id);
/* CUP2D_PENDING while the request runs or waits; afterwards its status, its
 * statistics and the time from submission to completion (ms), once. */
int cup2d_server_poll(cup2d_server* S, int64_t request_id, cup2d_solve_stats* stats, double* latency_ms);
int cup2d_server_wait(cup2d_server* S, int64_t request_id, int32_t timeout_ms, cup2d_solve_stats* stats,
                      double* latency_ms);
/* Ids of finished requests (up to max_ids, oldest first), each reported
 * once; waits up to timeout_ms for the first.  Then poll them for results. */
int cup2d_server_take_completed(cup2d_server* S, int64_t* ids, int32_t max_ids, int32_t timeout_ms,
                                int32_t* n);
int cup2d_server_get_counters(cup2d_server* S, cup2d_server_counters* out);
int cup2d_server_destroy(cup2d_server* S);

/* ------------------------------------------------- synthetic problems ---- */
typedef struct cup2d_mesh cup2d_mesh;
/* Forest refined to the finest level where a block meets the band
 * | |p - c| - r | <= band of any disk (cx, cy, r triples), 2:1 balanced,
 * Morton ordered.  The mesh owns the arrays that cup2d_mesh_forest exposes. */
int cup2d_mesh_disks(int32_t bpdx, int32_t bpdy, int32_t level_max, double extent,
                     int32_t periodic_x, int32_t periodic_y, int32_t ndisks,
                     const double* disks, double band, cup2d_mesh** out);
int cup2d_mesh_uniform(int32_t bpdx, int32_t bpdy, int32_t level_max, int32_t level,
                       double extent, int32_t periodic_x, int32_t periodic_y,
                       cup2d_mesh** out);
int cup2d_mesh_forest(const cup2d_mesh* m, cup2d_forest* out);
int cup2d_mesh_destroy(cup2d_mesh* m);
/* 0 if the forest is a valid 2:1-balanced leaf set, else CUP2D_BAD_MESH. */
int cup2d_forest_validate(const cup2d_forest* f);
/* Cell size of each block: h = extent / (max(bpdx,bpdy) * 8 * 2^level). */
int cup2d_forest_cell_h(const cup2d_forest* f, double* h_out);
/* Seeded Fourier-velocity divergence RHS, zero entry-sum (n = 64*nblocks). */
int cup2d_rhs_fourier(const cup2d_forest* f, uint64_t seed, int32_t kmax, double* b);
int32_t cup2d_fourier_num_modes(int32_t kmax);
int cup2d_fourier_coefs(uint64_t seed, int32_t kmax, double* coef);
int cup2d_fourier_advance(uint64_t seed, int32_t kmax, double rho, int64_t step, double* coef);
int cup2d_rhs_from_coefs(const cup2d_forest* f, int32_t kmax, const double* coef, double* b);

#ifdef __cplusplus
}
#endif
#endif /* CUP2D_POISSON_H */
