// C ABI of the B200 Poisson solver (include/cup2d_poisson.h).
//
// A handle plays the roles of ExpAMRSolver + LocalSpMatDnVec + BiCGSTABSolver
// in CUP2D (source/Poisson/ExpAMRSolver.cpp, LocalSpMatDnVec.cpp, BiCGSTAB.cu):
// it owns P^-1, the assembled operator and the Krylov vectors on the device.
// Unlike BiCGSTABSolver::updateAll (BiCGSTAB.cu:142-244), a mesh update
// reuses its buffers when the new mesh fits and assembles on the device; a
// solve is one persistent kernel launch and one 64-byte status read.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <new>
#include <vector>

#include "../../include/cup2d_poisson.h"
#include "forest.hpp"
#include "handle_view.hpp"
#include "kernels.hpp"

using namespace cup2d;

namespace {

// Device memory comes from the stream-ordered allocator on a library
// stream per device and host thread: unlike cudaMalloc/cudaFree this does not
// serialise the work other streams have on the device, so handles can be
// created and destroyed while other solves run (the request server relies
// on it).  An allocation is complete (usable from any stream) when ensure()
// returns; a buffer is released only when nothing uses it any more.  The
// device's default pool keeps freed memory for reuse.
constexpr int kMaxAllocDevices = 64;
std::mutex g_alloc_mu;
bool g_pool_set[kMaxAllocDevices] = {};
thread_local cudaStream_t t_alloc_stream[kMaxAllocDevices] = {};

// The calling thread's allocation stream on the current device (threads do
// not wait for each other's allocations).
cudaStream_t alloc_stream() {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxAllocDevices) return nullptr;
  if (!t_alloc_stream[dev]) {
    {
      std::lock_guard<std::mutex> g(g_alloc_mu);
      if (!g_pool_set[dev]) {
        cudaMemPool_t pool;
        if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
          uint64_t keep = ~0ull;
          cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
        }
        g_pool_set[dev] = true;
      }
    }
    if (cudaStreamCreateWithFlags(&t_alloc_stream[dev], cudaStreamNonBlocking) != cudaSuccess) {
      t_alloc_stream[dev] = nullptr;
      return nullptr;
    }
  }
  return t_alloc_stream[dev];
}

// P^-1 depends on nothing but the 8x8 block Laplacian: built once per
// device (FP64, and rounded to FP32) and shared by every handle and batch.
struct SharedPinv {
  double* P = nullptr;
  float* P32 = nullptr;
};
SharedPinv g_pinv[kMaxAllocDevices];

int shared_pinv(const double** P, const float** P32) {
  cudaStream_t s = alloc_stream();
  int dev = 0;
  if (!s || cudaGetDevice(&dev) != cudaSuccess) return CUP2D_CUDA_ERROR;
  std::lock_guard<std::mutex> g(g_alloc_mu);
  SharedPinv& sp = g_pinv[dev];
  if (!sp.P) {
    double* p = nullptr;
    float* p32 = nullptr;
    if (cudaMallocAsync(reinterpret_cast<void**>(&p), sizeof(double) * 4096, s) != cudaSuccess ||
        cudaMallocAsync(reinterpret_cast<void**>(&p32), sizeof(float) * 4096, s) != cudaSuccess ||
        launch_build_pinv(p, s) != cudaSuccess || launch_convert_f64_f32(p, p32, 4096, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess) {
      cudaGetLastError();
      return CUP2D_CUDA_ERROR;
    }
    sp.P = p;
    sp.P32 = p32;
  }
  *P = sp.P;
  *P32 = sp.P32;
  return CUP2D_OK;
}

template <class T>
struct DevBuf {
  T* p = nullptr;
  int64_t cap = 0;  // elements
  // Grows the buffer to n elements.  The old buffer is freed in stream order
  // on `last_user` when given (the stream whose queued work may still read
  // or write it), else on the allocation stream, where it must be idle.
  int ensure(int64_t n, cudaStream_t last_user = nullptr) {
    if (n <= cap && p) return CUP2D_OK;
    if (p && last_user) {
      cudaFreeAsync(p, last_user);
      p = nullptr;
      cap = 0;
    }
    release();
    const int64_t m = std::max<int64_t>(n, 1);
    cudaStream_t s = alloc_stream();
    if (!s) return CUP2D_CUDA_ERROR;
    if (cudaMallocAsync(reinterpret_cast<void**>(&p), sizeof(T) * m, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess) {
      cudaGetLastError();
      p = nullptr;
      return CUP2D_OOM;
    }
    cap = m;
    return CUP2D_OK;
  }
  void release() {
    if (p) {
      if (cudaStream_t s = alloc_stream()) cudaFreeAsync(p, s);
    }
    p = nullptr;
    cap = 0;
  }
};

int validate_opts(const cup2d_solve_opts& o) {
  if (!(o.tol_abs >= 0.0) || !(o.tol_rel >= 0.0)) return CUP2D_INVALID_ARGUMENT;
  if (o.max_iter < 0 || o.max_restarts < 0) return CUP2D_INVALID_ARGUMENT;
  if (!(o.reliable_delta > 0.0 && o.reliable_delta < 1.0)) return CUP2D_INVALID_ARGUMENT;
  if (o.reliable_restart != 0 && o.reliable_restart != 1) return CUP2D_INVALID_ARGUMENT;
  if (o.precision != CUP2D_PREC_FP64 && o.precision != CUP2D_PREC_MIXED) return CUP2D_INVALID_ARGUMENT;
  if (o.timeout_ms <= 0) return CUP2D_INVALID_ARGUMENT;
  // the mean constraint is the FP64 drop-in's (the mixed form's FP32 sweeps
  // derail on the constrained system)
  if (o.mean_constraint && o.precision != CUP2D_PREC_FP64) return CUP2D_INVALID_ARGUMENT;
  return CUP2D_OK;
}

int from_cuda(cudaError_t e) {
  if (e == cudaSuccess) return CUP2D_OK;
  if (e == cudaErrorMemoryAllocation) return CUP2D_OOM;
  if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver) return CUP2D_NO_DEVICE;
  return CUP2D_CUDA_ERROR;
}

}  // namespace

struct cup2d_poisson {
  int device = 0;
  cudaStream_t stream = nullptr;
  bool owns_stream = true;  // false for the problems of a batch (batch stream)
  bool served = false;      // a server's handle: its solves run the served kernel instances
  cup2d_solve_opts opts{};
  // forest
  int32_t bpdx = 0, bpdy = 0, level_max = 0, px = 0, py = 0;
  double extent = 1.0;
  int64_t nb = 0;
  // operator
  DevBuf<int32_t> level, bx, by, table, nbr, xcount, xbase, scan_tmp, rowlen, xptr, xcol, rowcell;
  DevBuf<unsigned long long> xmask;
  DevBuf<double> hblk, xval;
  DevBuf<float> xval32;
  const double* P = nullptr;  // shared per device
  const float* P32 = nullptr;
  DevBuf<int> err;
  DeviceMesh mesh;
  // Krylov vectors (FP64)
  DevBuf<double> xo, r, rh, p, nu, t, z, z2, bstage, xstage;
  // mixed-precision vectors
  DevBuf<float> f_r, f_rh, f_p, f_nu, f_t, f_z, f_z2;
  // persistent-kernel scratch
  DevBuf<double> red;
  DevBuf<unsigned> bar;
  DevBuf<int> abort_flag;
  DevBuf<DevStats> dstats;
  DevBuf<unsigned long long> prof;  // phase timers (profiling on)
  DevBuf<double> rhs_coef, rhs_part;  // device RHS: coefficients, partial sums + mean
  // device forest adaptation: per-level states, Morton key marks and ranks,
  // scan scratch, flag
  DevBuf<uint8_t> ad_state;
  DevBuf<int32_t> ad_mark, ad_rank, ad_scan, ad_flags;
  DevBuf<double> ps_part;  // pressure step: weighted-mean partials
  uint64_t mesh_version = 0;
  bool profiling = false;
  int prof_grid = 0;                // grid of the profiled solves
  DevStats* hstats = nullptr;  // pinned
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  int grid64 = 0, gridmx = 0;      // max co-resident grids
  int grid64m = 0;                 // ... of the mean-constraint kernel
  int grid_override = 0;           // tuner / user choice (0 = heuristic)
  int blocks_per_cta = 8;          // heuristic target

  int grid_for(int maxg) const {
    if (grid_override > 0) return std::min(grid_override, maxg);
    const int64_t want = (nb + blocks_per_cta - 1) / blocks_per_cta;
    return (int)std::max<int64_t>(1, std::min<int64_t>(want, maxg));
  }
};

namespace {

int alloc_rows_cb(void* ctx, int64_t R) {
  auto* h = static_cast<cup2d_poisson*>(ctx);
  int st = h->rowlen.ensure(R);
  if (st) return st;
  st = h->xptr.ensure(R + 1);
  if (st) return st;
  st = h->rowcell.ensure(R);
  if (st) return st;
  h->mesh.rowlen = h->rowlen.p;
  h->mesh.xptr = h->xptr.p;
  h->mesh.rowcell = h->rowcell.p;
  return CUP2D_OK;
}

int alloc_nnz_cb(void* ctx, int64_t nnz) {
  auto* h = static_cast<cup2d_poisson*>(ctx);
  int st = h->xcol.ensure(nnz);
  if (st) return st;
  st = h->xval.ensure(nnz);
  if (st) return st;
  st = h->xval32.ensure(nnz);
  if (st) return st;
  h->mesh.xcol = h->xcol.p;
  h->mesh.xval = h->xval.p;
  h->mesh.xval32 = h->xval32.p;
  return CUP2D_OK;
}

int check_forest(const cup2d_forest* f) {
  if (!f || f->nblocks <= 0 || !f->level || !f->bx || !f->by) return CUP2D_INVALID_ARGUMENT;
  if (f->bpdx < 1 || f->bpdy < 1 || f->level_max < 1 || f->level_max > kMaxLevels || !(f->extent > 0.0))
    return CUP2D_INVALID_ARGUMENT;
  if (f->nblocks > (int64_t)(INT32_MAX / kBLEN)) return CUP2D_INVALID_ARGUMENT;
  const int64_t entries = leaf_table_entries(f->bpdx, f->bpdy, f->level_max);
  if (entries > ((int64_t)1 << 30)) return CUP2D_BAD_MESH;  // dense tables would exceed 4 GB
  return CUP2D_OK;
}

// Assembles the operator of the forest whose blocks are already in the
// handle's level/bx/by buffers (nb of them), for the geometry of f (its
// block arrays are not read).
int assemble_blocks(cup2d_poisson* h, const cup2d_forest* f, int64_t nb) {
  int st;
  const int64_t n = nb * kBLEN;
  const int64_t entries = leaf_table_entries(f->bpdx, f->bpdy, f->level_max);
  if ((st = h->table.ensure(entries)) || (st = h->nbr.ensure(4 * nb)) || (st = h->xmask.ensure(nb)) ||
      (st = h->xcount.ensure(nb)) || (st = h->xbase.ensure(nb + 1)) || (st = h->hblk.ensure(nb)) ||
      (st = h->scan_tmp.ensure(scan_temp_ints(n) + 2)) || (st = h->err.ensure(2)))
    return st;
  // the best-iterate copy; the Krylov vectors of a precision are allocated
  // by its first solve
  if ((st = h->xo.ensure(n))) return st;
  cudaStream_t s = h->stream;
  DeviceMesh& m = h->mesh;
  m.nb = nb;
  m.level = h->level.p;
  m.bx = h->bx.p;
  m.by = h->by.p;
  m.table = h->table.p;
  m.nbr = h->nbr.p;
  m.xmask = h->xmask.p;
  m.xcount = h->xcount.p;
  m.xbase = h->xbase.p;
  m.hblk = h->hblk.p;
  m.scan_tmp = h->scan_tmp.p;
  m.err = h->err.p;
  m.ctx = h;
  m.alloc_rows = alloc_rows_cb;
  m.alloc_nnz = alloc_nnz_cb;
  // a mesh without explicit rows still needs valid (empty) row arrays
  if ((st = alloc_rows_cb(h, 0)) || (st = alloc_nnz_cb(h, 0))) return st;
  AssembleIn in{f->bpdx, f->bpdy, f->level_max, f->periodic_x, f->periodic_y, nb,
                f->extent / ((double)std::max(f->bpdx, f->bpdy) * 8.0)};
  st = assemble_on_device(in, m, s);
  if (st) return st;
  ++h->mesh_version;
  h->bpdx = f->bpdx;
  h->bpdy = f->bpdy;
  h->level_max = f->level_max;
  h->px = f->periodic_x;
  h->py = f->periodic_y;
  h->extent = f->extent;
  h->nb = nb;
  return CUP2D_OK;
}

int do_assemble(cup2d_poisson* h, const cup2d_forest* f) {
  int st = check_forest(f);
  if (st) return st;
  const int64_t nb = f->nblocks;
  if ((st = h->level.ensure(nb)) || (st = h->bx.ensure(nb)) || (st = h->by.ensure(nb))) return st;
  cudaStream_t s = h->stream;
  if (cudaMemcpyAsync(h->level.p, f->level, sizeof(int32_t) * nb, cudaMemcpyHostToDevice, s) != cudaSuccess ||
      cudaMemcpyAsync(h->bx.p, f->bx, sizeof(int32_t) * nb, cudaMemcpyHostToDevice, s) != cudaSuccess ||
      cudaMemcpyAsync(h->by.p, f->by, sizeof(int32_t) * nb, cudaMemcpyHostToDevice, s) != cudaSuccess)
    return CUP2D_CUDA_ERROR;
  return assemble_blocks(h, f, nb);
}

// The timing events of a handle (made on first use for handles that were
// created on a caller's stream).
int ensure_events(cup2d_poisson* h) {
  if (h->ev0 && h->ev1) return CUP2D_OK;
  if ((!h->ev0 && cudaEventCreate(&h->ev0) != cudaSuccess) || (!h->ev1 && cudaEventCreate(&h->ev1) != cudaSuccess))
    return CUP2D_CUDA_ERROR;
  return CUP2D_OK;
}

int ensure_scratch(cup2d_poisson* h) {
  int st;
  const int g = std::max(h->grid64, h->gridmx);
  if ((st = h->red.ensure((int64_t)kRedQMean * std::max(g, 1))) || (st = h->bar.ensure(1)) ||
      (st = h->abort_flag.ensure(1)) || (st = h->dstats.ensure(1)))
    return st;
  return CUP2D_OK;
}

int ensure_fp64(cup2d_poisson* h) {
  const int64_t n = h->nb * kBLEN;
  int st;
  if ((st = h->r.ensure(n)) || (st = h->rh.ensure(n)) || (st = h->p.ensure(n)) || (st = h->nu.ensure(n)) ||
      (st = h->t.ensure(n)) || (st = h->z.ensure(n)) || (st = h->z2.ensure(n)))
    return st;
  return CUP2D_OK;
}

int ensure_mixed(cup2d_poisson* h) {
  const int64_t n = h->nb * kBLEN;
  int st;
  if ((st = h->f_r.ensure(n)) || (st = h->f_rh.ensure(n)) || (st = h->f_p.ensure(n)) ||
      (st = h->f_nu.ensure(n)) || (st = h->f_t.ensure(n)) || (st = h->f_z.ensure(n)) ||
      (st = h->f_z2.ensure(n)))
    return st;
  return CUP2D_OK;
}

void fill_stats(const cup2d_poisson* h, int launch_status, float ms, cup2d_solve_stats* out) {
  const DevStats& d = *h->hstats;
  out->status = launch_status != CUP2D_OK ? launch_status : d.status;
  out->iterations = d.iterations;
  out->restarts = d.restarts;
  out->refinements = d.refinements;
  out->err_init = d.err_init;
  out->err_final = d.err_opt;
  out->rel_res_inf = d.err_init > 0 ? d.err_opt / d.err_init : 0.0;
  out->solve_ms = ms;
}

}  // namespace

extern "C" {

const char* cup2d_version(void) { return "cup2d_b200 0.1.0 (sm_100a)"; }

const char* cup2d_status_string(int s) {
  switch (s) {
    case CUP2D_OK: return "ok";
    case CUP2D_NOT_CONVERGED: return "not converged (iteration cap)";
    case CUP2D_BREAKDOWN_LIMIT: return "restart cap reached after breakdowns";
    case CUP2D_BAD_MESH: return "invalid forest (overlap, hole or 2:1 violation)";
    case CUP2D_OOM: return "device allocation failed";
    case CUP2D_TIMEOUT: return "device-side wait timed out";
    case CUP2D_CUDA_ERROR: return "CUDA error";
    case CUP2D_INVALID_ARGUMENT: return "invalid argument";
    case CUP2D_NO_DEVICE: return "no CUDA device";
    case CUP2D_QUEUE_FULL: return "queue full";
    case CUP2D_PENDING: return "pending";
    default: return "unknown status";
  }
}

void cup2d_default_opts(cup2d_solve_opts* o) {
  if (!o) return;
  o->tol_abs = 0.0;
  o->tol_rel = 1e-8;
  o->max_restarts = 100;
  o->max_iter = 1000;
  o->precision = CUP2D_PREC_FP64;
  o->subtract_mean = 1;
  o->reliable_delta = 0.5;
  o->reliable_restart = 1;
  o->timeout_ms = 20000;
  o->mean_constraint = 0;
}

int cup2d_pinv(double* P_out) {
  if (!P_out) return CUP2D_INVALID_ARGUMENT;
  double* d = nullptr;
  if (cudaMalloc(&d, sizeof(double) * 4096) != cudaSuccess) return CUP2D_OOM;
  cudaError_t e = launch_build_pinv(d, 0);
  if (e == cudaSuccess) e = cudaMemcpy(P_out, d, sizeof(double) * 4096, cudaMemcpyDeviceToHost);
  cudaFree(d);
  return from_cuda(e);
}

int cup2d_poisson_create(const cup2d_forest* forest, const cup2d_solve_opts* opts, cup2d_poisson** out) {
  return handle_create(forest, opts, nullptr, false, out);
}

}  // extern "C"

namespace cup2d {

int handle_create(const cup2d_forest* forest, const cup2d_solve_opts* opts, cudaStream_t stream, bool served,
                  cup2d_poisson** out) {
  if (!out) return CUP2D_INVALID_ARGUMENT;
  *out = nullptr;
  cup2d_solve_opts o;
  cup2d_default_opts(&o);
  if (opts) o = *opts;
  int st = validate_opts(o);
  if (st) return st;
  if ((st = check_forest(forest))) return st;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return CUP2D_NO_DEVICE;
  }
  auto* h = new (std::nothrow) cup2d_poisson();
  if (!h) return CUP2D_OOM;
  h->opts = o;
  cudaGetDevice(&h->device);
  // the handle's own stream (assembly, host-buffer solves) at the highest
  // priority: when a server assembles a new mesh while persistent solves
  // hold most of the device, its short assembly kernels take the CTA slots
  // that free up before queued solve work does
  if (stream) {  // the caller's (a server's assembly stream): no stream or events of its own
    h->stream = stream;
    h->owns_stream = false;
  } else {
    int prio_lo = 0, prio_hi = 0;
    cudaDeviceGetStreamPriorityRange(&prio_lo, &prio_hi);
    if (cudaStreamCreateWithPriority(&h->stream, cudaStreamNonBlocking, prio_hi) != cudaSuccess ||
        ensure_events(h) != CUP2D_OK) {
      cup2d_poisson_destroy(h);
      return CUP2D_CUDA_ERROR;
    }
  }
  h->served = served;
  h->grid64 = max_coop_grid_fp64(h->device, served);
  h->gridmx = max_coop_grid_mixed(h->device, served);
  h->grid64m = std::min(h->grid64, max_coop_grid_mean(h->device));
  if (h->grid64 <= 0 || h->gridmx <= 0) {
    cup2d_poisson_destroy(h);
    return CUP2D_CUDA_ERROR;
  }
  if (const char* e = std::getenv("CUP2D_GRID")) h->grid_override = std::atoi(e);
  // the no-allocation solve's static scratch is committed here, with the
  // rest of the handle's memory, so that those solves never load or allocate
  if ((st = shared_pinv(&h->P, &h->P32)) || (st = ensure_scratch(h)) || (st = noalloc_prepare(h->device))) {
    cup2d_poisson_destroy(h);
    return st;
  }
  if ((st = do_assemble(h, forest))) {
    cup2d_poisson_destroy(h);
    return st;
  }
  *out = h;
  return CUP2D_OK;
}

}  // namespace cup2d

extern "C" {

int cup2d_poisson_update_mesh(cup2d_poisson* h, const cup2d_forest* forest) {
  if (!h) return CUP2D_INVALID_ARGUMENT;
  // buffers may be reallocated: let solves queued on any stream finish first
  if (cudaDeviceSynchronize() != cudaSuccess) return CUP2D_CUDA_ERROR;
  return do_assemble(h, forest);
}

int cup2d_poisson_adapt_disks(cup2d_poisson* h, int32_t ndisks, const double* disks, double band,
                              int64_t* nblocks) {
  if (!h || h->nb <= 0 || ndisks < 0 || ndisks > kMaxAdaptDisks || (ndisks > 0 && !disks) || !(band >= 0.0))
    return CUP2D_INVALID_ARGUMENT;
  AdaptGeom g{};
  g.bpdx = h->bpdx;
  g.bpdy = h->bpdy;
  g.L = h->level_max;
  g.px = h->px;
  g.py = h->py;
  g.extent = h->extent;
  int64_t off = 0;
  for (int l = 0; l < h->level_max; ++l) {
    g.off[l] = off;
    off += ((int64_t)h->bpdx << l) * ((int64_t)h->bpdy << l);
  }
  g.off[h->level_max] = off;
  AdaptDisks D{};
  D.n = ndisks;
  D.band = band;
  for (int k = 0; k < ndisks; ++k)
    for (int c = 0; c < 3; ++c) D.d[k][c] = disks[3 * k + c];
  const int64_t K = adapt_key_space(h->bpdx, h->bpdy, h->level_max);
  if (K > ((int64_t)1 << 30)) return CUP2D_BAD_MESH;  // key space beyond 4 GB
  // buffers may be reallocated: let solves queued on any stream finish first
  if (cudaDeviceSynchronize() != cudaSuccess) return CUP2D_CUDA_ERROR;
  int st;
  if ((st = h->ad_state.ensure(off)) || (st = h->ad_mark.ensure(K)) || (st = h->ad_rank.ensure(K + 1)) ||
      (st = h->ad_scan.ensure(scan_temp_ints(K) + 2)) || (st = h->ad_flags.ensure(1)))
    return st;
  const AdaptScratch sc{h->ad_state.p, h->ad_mark.p, h->ad_rank.p, h->ad_scan.p, h->ad_flags.p};
  int64_t nb = 0;
  if ((st = adapt_build(g, D, sc, &nb, h->stream))) return st;
  if (nb <= 0 || nb > (int64_t)(INT32_MAX / kBLEN)) return CUP2D_BAD_MESH;
  if ((st = h->level.ensure(nb)) || (st = h->bx.ensure(nb)) || (st = h->by.ensure(nb))) return st;
  if ((st = adapt_scatter(g, sc, nb, h->level.p, h->bx.p, h->by.p, h->stream))) return st;
  cup2d_forest f{};
  f.bpdx = h->bpdx;
  f.bpdy = h->bpdy;
  f.level_max = h->level_max;
  f.periodic_x = h->px;
  f.periodic_y = h->py;
  f.extent = h->extent;
  f.nblocks = nb;
  if ((st = assemble_blocks(h, &f, nb))) return st;
  if (nblocks) *nblocks = nb;
  return CUP2D_OK;
}

int cup2d_poisson_get_forest(const cup2d_poisson* h, int32_t* level, int32_t* bx, int32_t* by) {
  if (!h || h->nb <= 0 || !level || !bx || !by) return CUP2D_INVALID_ARGUMENT;
  const size_t bytes = sizeof(int32_t) * (size_t)h->nb;
  if (cudaMemcpyAsync(level, h->level.p, bytes, cudaMemcpyDeviceToHost, h->stream) != cudaSuccess ||
      cudaMemcpyAsync(bx, h->bx.p, bytes, cudaMemcpyDeviceToHost, h->stream) != cudaSuccess ||
      cudaMemcpyAsync(by, h->by.p, bytes, cudaMemcpyDeviceToHost, h->stream) != cudaSuccess ||
      cudaStreamSynchronize(h->stream) != cudaSuccess)
    return CUP2D_CUDA_ERROR;
  return CUP2D_OK;
}

int cup2d_poisson_set_opts(cup2d_poisson* h, const cup2d_solve_opts* opts) {
  if (!h || !opts) return CUP2D_INVALID_ARGUMENT;
  int st = validate_opts(*opts);
  if (st) return st;
  h->opts = *opts;
  return CUP2D_OK;
}

int64_t cup2d_poisson_num_cells(const cup2d_poisson* h) { return h ? h->nb * kBLEN : 0; }

int cup2d_poisson_set_grid(cup2d_poisson* h, int32_t grid) {
  if (!h || grid < 0) return CUP2D_INVALID_ARGUMENT;
  h->grid_override = grid;
  return CUP2D_OK;
}

int cup2d_poisson_destroy(cup2d_poisson* h) {
  if (!h) return CUP2D_OK;
  // solves may have been queued on any stream: let them finish before the
  // buffers go back to the allocator
  cudaDeviceSynchronize();
  return cup2d::handle_destroy_idle(h);
}

}  // extern "C"

namespace cup2d {

int handle_destroy_idle(cup2d_poisson* h) {
  if (!h) return CUP2D_OK;
  if (h->stream) cudaStreamSynchronize(h->stream);
  DevBuf<int32_t>* i32[] = {&h->level, &h->bx, &h->by, &h->table, &h->nbr, &h->xcount, &h->xbase,
                            &h->scan_tmp, &h->rowlen, &h->xptr, &h->xcol,
                            &h->rowcell};
  for (auto* b : i32) b->release();
  h->xmask.release();
  DevBuf<double>* f64[] = {&h->hblk, &h->xval, &h->xo, &h->r, &h->rh, &h->p, &h->nu, &h->t,
                           &h->z, &h->z2, &h->bstage, &h->xstage, &h->red, &h->rhs_coef, &h->rhs_part};
  for (auto* b : f64) b->release();
  DevBuf<float>* f32[] = {&h->xval32, &h->f_r, &h->f_rh, &h->f_p,
                          &h->f_nu, &h->f_t, &h->f_z, &h->f_z2};
  for (auto* b : f32) b->release();
  h->err.release();
  h->bar.release();
  h->abort_flag.release();
  h->dstats.release();
  h->prof.release();
  if (h->hstats) cudaFreeHost(h->hstats);
  if (h->ev0) cudaEventDestroy(h->ev0);
  if (h->ev1) cudaEventDestroy(h->ev1);
  if (h->stream && h->owns_stream) cudaStreamDestroy(h->stream);
  delete h;
  return CUP2D_OK;
}

}  // namespace cup2d

extern "C" {

int cup2d_poisson_solve_device(cup2d_poisson* h, const double* d_b, double* d_x, cup2d_solve_stats* stats,
                               void* stream) {
  if (!h || !d_b || !d_x) return CUP2D_INVALID_ARGUMENT;
  if (!aligned16(d_b) || !aligned16(d_x)) return CUP2D_INVALID_ARGUMENT;  // 16-byte vector accesses
  cudaStream_t s = static_cast<cudaStream_t>(stream);  // NULL: the legacy default stream
  const cup2d_solve_opts& o = h->opts;
  int st;
  if ((st = ensure_scratch(h))) return st;
  if (cudaMemsetAsync(h->bar.p, 0, sizeof(unsigned), s) != cudaSuccess ||
      cudaMemsetAsync(h->abort_flag.p, 0, sizeof(int), s) != cudaSuccess)
    return CUP2D_CUDA_ERROR;
  const unsigned long long tns = (unsigned long long)o.timeout_ms * 1000000ull;
  // the barrier counter counts arrivals of the whole solve in 32 bits
  // bMeanConstraint: row of cell (0,0) of the leaf at the domain's corner
  const int mean_row = o.mean_constraint ? (int)h->mesh.origin * kBLEN : -1;
  const bool mixed = o.precision == CUP2D_PREC_MIXED;
  const int grid = h->grid_for(mixed ? h->gridmx : mean_row >= 0 ? h->grid64m : h->grid64);
  if (grid <= 0) return CUP2D_CUDA_ERROR;
  const uint64_t arrivals = ((uint64_t)o.max_iter * 7 + 16) * (uint64_t)grid;
  if (arrivals >= (1ull << 32)) return CUP2D_INVALID_ARGUMENT;
  unsigned long long* prof = nullptr;
  if (h->profiling) {
    const int64_t words = (int64_t)grid * kProfPhases * 2;
    // sized once for the handle's largest grid, so it never grows under
    // solves still queued on a stream
    if ((st = h->prof.ensure((int64_t)std::max(h->grid64, h->gridmx) * kProfPhases * 2))) return st;
    if (h->prof_grid != grid) {  // timers accumulate over solves of one grid size
      if (cudaMemsetAsync(h->prof.p, 0, sizeof(unsigned long long) * words, s) != cudaSuccess)
        return CUP2D_CUDA_ERROR;
      h->prof_grid = grid;
    }
    prof = h->prof.p;
  }
  // the pinned statistics record is allocated when statistics are first
  // asked for (a page-locked allocation serialises the device's streams)
  if (stats && !h->hstats && cudaMallocHost(&h->hstats, sizeof(DevStats)) != cudaSuccess) {
    h->hstats = nullptr;
    return CUP2D_OOM;
  }
  if (stats && (st = ensure_events(h))) return st;
  if (stats) cudaEventRecord(h->ev0, s);
  cudaError_t e;
  if (o.precision == CUP2D_PREC_MIXED) {
    if ((st = ensure_mixed(h))) return st;
    SolveArgsMixed a{};
    a.prob = ProblemMixed{h->mesh.view(), d_b, d_x, h->xo.p, h->f_r.p, h->f_rh.p, h->f_p.p, h->f_nu.p,
                          h->f_t.p, h->f_z.p, h->f_z2.p, h->dstats.p};
    a.P32 = h->P32;
    a.red = h->red.p;
    a.bar = h->bar.p;
    a.abort_flag = h->abort_flag.p;
    a.sp = SolveParams{o.tol_abs, o.tol_rel, o.reliable_delta, o.max_restarts, o.max_iter, o.subtract_mean,
                       o.reliable_restart, mean_row};
    a.timeout_ns = tns;
    a.prof = prof;
    e = launch_bicgstab_mixed(a, grid, s, h->served);
  } else {
    if ((st = ensure_fp64(h))) return st;
    SolveArgs64 a{};
    a.prob = Problem64{h->mesh.view(), d_b, d_x, h->xo.p, h->r.p, h->rh.p, h->p.p, h->nu.p, h->t.p, h->z.p,
                       h->z2.p, h->dstats.p};
    a.P = h->P;
    a.red = h->red.p;
    a.bar = h->bar.p;
    a.abort_flag = h->abort_flag.p;
    a.sp = SolveParams{o.tol_abs, o.tol_rel, 0.0, o.max_restarts, o.max_iter, o.subtract_mean, 0, mean_row};
    a.timeout_ns = tns;
    a.prof = prof;
    e = launch_bicgstab64(a, grid, s, h->served);
  }
  if (e != cudaSuccess) return from_cuda(e);
  if (!stats) return CUP2D_OK;
  int habort = 0;
  cudaEventRecord(h->ev1, s);
  if (cudaMemcpyAsync(h->hstats, h->dstats.p, sizeof(DevStats), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
      cudaMemcpyAsync(&habort, h->abort_flag.p, sizeof(int), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
      cudaStreamSynchronize(s) != cudaSuccess)
    return CUP2D_CUDA_ERROR;
  float ms = 0.f;
  cudaEventElapsedTime(&ms, h->ev0, h->ev1);
  fill_stats(h, habort ? CUP2D_TIMEOUT : CUP2D_OK, ms, stats);
  return stats->status == CUP2D_TIMEOUT ? CUP2D_TIMEOUT : CUP2D_OK;
}

int cup2d_poisson_solve(cup2d_poisson* h, const double* b, double* x, cup2d_solve_stats* stats) {
  if (!h || !b || !x) return CUP2D_INVALID_ARGUMENT;
  const int64_t n = h->nb * kBLEN;
  int st;
  if ((st = h->bstage.ensure(n)) || (st = h->xstage.ensure(n))) return st;
  cudaStream_t s = h->stream;
  if (cudaMemcpyAsync(h->bstage.p, b, sizeof(double) * n, cudaMemcpyHostToDevice, s) != cudaSuccess ||
      cudaMemcpyAsync(h->xstage.p, x, sizeof(double) * n, cudaMemcpyHostToDevice, s) != cudaSuccess)
    return CUP2D_CUDA_ERROR;
  cup2d_solve_stats local;
  st = cup2d_poisson_solve_device(h, h->bstage.p, h->xstage.p, stats ? stats : &local, s);
  if (st != CUP2D_OK && st != CUP2D_NOT_CONVERGED && st != CUP2D_BREAKDOWN_LIMIT) return st;
  if (cudaMemcpyAsync(x, h->xstage.p, sizeof(double) * n, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
      cudaStreamSynchronize(s) != cudaSuccess)
    return CUP2D_CUDA_ERROR;
  return CUP2D_OK;
}

int cup2d_poisson_apply(cup2d_poisson* h, const double* d_x, double* d_y, void* stream) {
  if (!h || !d_x || !d_y || !aligned16(d_x) || !aligned16(d_y)) return CUP2D_INVALID_ARGUMENT;
  cudaStream_t s = static_cast<cudaStream_t>(stream);  // NULL: the legacy default stream
  return from_cuda(launch_spmv64(h->mesh.view(), d_x, d_y, h->err.p, s));
}

int cup2d_poisson_apply32(cup2d_poisson* h, const float* d_x, float* d_y, void* stream) {
  if (!h || !d_x || !d_y || !aligned16(d_x) || !aligned16(d_y)) return CUP2D_INVALID_ARGUMENT;
  cudaStream_t s = static_cast<cudaStream_t>(stream);  // NULL: the legacy default stream
  return from_cuda(launch_spmv32(h->mesh.view(), d_x, d_y, h->err.p, s));
}

}  // extern "C"

namespace {

ForestView forest_view(const cup2d_poisson* h) {
  ForestView F{};
  F.bpdx = h->bpdx;
  F.bpdy = h->bpdy;
  F.L = h->level_max;
  F.px = h->px;
  F.py = h->py;
  F.nb = h->nb;
  F.h0 = h->extent / ((double)std::max(h->bpdx, h->bpdy) * 8.0);
  F.level = h->level.p;
  F.bx = h->bx.p;
  F.by = h->by.p;
  F.table = h->table.p;
  int64_t off = 0;
  for (int l = 0; l < h->level_max; ++l) {
    F.off[l] = off;
    off += ((int64_t)h->bpdx << l) * ((int64_t)h->bpdy << l);
  }
  F.off[h->level_max] = off;
  return F;
}

}  // namespace

extern "C" {

namespace {

bool overlaps(const void* a, size_t na, const void* b, size_t nb) {
  if (!a || !b) return false;
  const char* pa = static_cast<const char*>(a);
  const char* pb = static_cast<const char*>(b);
  return pa < pb + nb && pb < pa + na;
}

}  // namespace

int cup2d_poisson_pressure_rhs(cup2d_poisson* h, double dt, const double* d_vel, const double* d_udef,
                               const double* d_chi, double* d_pres, double* d_pold, double* d_tmp, void* stream) {
  if (!h || !d_tmp || h->nb <= 0) return CUP2D_INVALID_ARGUMENT;
  if (!d_vel && !d_pres) return CUP2D_INVALID_ARGUMENT;
  if (d_vel && (!d_udef || !d_chi || !(dt > 0.0) || !std::isfinite(dt))) return CUP2D_INVALID_ARGUMENT;
  if (d_vel && (!aligned16(d_vel) || !aligned16(d_udef))) return CUP2D_INVALID_ARGUMENT;  // 16-byte (u, v) pairs
  if (d_pres && !d_pold) return CUP2D_INVALID_ARGUMENT;
  const size_t n = (size_t)h->nb * kBLEN * sizeof(double);
  const void* bufs[6] = {d_tmp, d_pres, d_pold, d_vel, d_udef, d_chi};
  const size_t size[6] = {n, n, n, 2 * n, 2 * n, n};
  for (int a = 0; a < 6; ++a)
    for (int b = a + 1; b < 6; ++b)
      if (overlaps(bufs[a], size[a], bufs[b], size[b])) return CUP2D_INVALID_ARGUMENT;
  cudaStream_t s = static_cast<cudaStream_t>(stream);  // NULL: the legacy default stream
  const ProjFields f{d_vel, d_vel ? d_udef : nullptr, d_vel ? d_chi : nullptr, d_pres, d_tmp, d_pold};
  if (launch_pressure_rhs(forest_view(h), h->nbr.p, d_vel ? dt : 1.0, f, s) != cudaSuccess) return CUP2D_CUDA_ERROR;
  // PRES = 0 (PressureSingle.cpp:845): the solve's initial guess
  if (d_pres && cudaMemsetAsync(d_pres, 0, n, s) != cudaSuccess) return CUP2D_CUDA_ERROR;
  return CUP2D_OK;
}

int cup2d_poisson_pressure_correction(cup2d_poisson* h, double dt, const double* d_pres, double* d_vel,
                                      void* stream) {
  if (!h || !d_pres || !d_vel || h->nb <= 0 || !(dt > 0.0) || !std::isfinite(dt)) return CUP2D_INVALID_ARGUMENT;
  if (!aligned16(d_vel)) return CUP2D_INVALID_ARGUMENT;  // 16-byte (u, v) pairs
  const size_t n = (size_t)h->nb * kBLEN * sizeof(double);
  if (overlaps(d_pres, n, d_vel, 2 * n)) return CUP2D_INVALID_ARGUMENT;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  return from_cuda(launch_pressure_correction(forest_view(h), h->nbr.p, dt, d_pres, d_vel, s));
}

int cup2d_poisson_pressure_step(cup2d_poisson* h, double* d_tmp, double* d_pres, double* d_pold,
                                cup2d_solve_stats* stats, void* stream) {
  if (!h || !d_tmp || !d_pres || !d_pold || h->nb <= 0) return CUP2D_INVALID_ARGUMENT;
  if (!aligned16(d_tmp) || !aligned16(d_pres) || !aligned16(d_pold)) return CUP2D_INVALID_ARGUMENT;
  cudaStream_t s = static_cast<cudaStream_t>(stream);  // NULL: the legacy default stream
  int st;
  if ((st = h->ps_part.ensure(wmean_partials(h->nb), s))) return st;
  // POLD = PRES; TMP -= L(POLD); PRES = 0 (PressureSingle.cpp:836-848, 399-456)
  if ((st = cup2d_poisson_pressure_rhs(h, 0.0, nullptr, nullptr, nullptr, d_pres, d_pold, d_tmp, stream))) return st;
  // pressureSolver->solve(sim.tmp, sim.pres) (:850)
  if ((st = cup2d_poisson_solve_device(h, d_tmp, d_pres, stats, stream))) return st;
  // PRES += POLD - mean(PRES), volume-weighted (:853-879)
  return from_cuda(launch_add_pold(d_pres, d_pold, h->hblk.p, h->nb, h->ps_part.p, s));
}

int cup2d_poisson_pressure_projection(cup2d_poisson* h, double dt, double* d_vel, const double* d_udef,
                                      const double* d_chi, double* d_pres, double* d_pold, double* d_tmp,
                                      cup2d_solve_stats* stats, void* stream) {
  if (!h || !d_vel || !d_udef || !d_chi || !d_pres || !d_pold || !d_tmp || h->nb <= 0) return CUP2D_INVALID_ARGUMENT;
  if (!aligned16(d_tmp) || !aligned16(d_pres) || !aligned16(d_pold)) return CUP2D_INVALID_ARGUMENT;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  int st;
  if ((st = h->ps_part.ensure(wmean_partials(h->nb), s))) return st;
  // updatePressureRHS; POLD = PRES, PRES = 0; updatePressureRHS1 (:826-849)
  if ((st = cup2d_poisson_pressure_rhs(h, dt, d_vel, d_udef, d_chi, d_pres, d_pold, d_tmp, stream))) return st;
  // solve (:850); PRES += POLD - mean(PRES) (:853-879)
  if ((st = cup2d_poisson_solve_device(h, d_tmp, d_pres, stats, stream))) return st;
  if ((st = from_cuda(launch_add_pold(d_pres, d_pold, h->hblk.p, h->nb, h->ps_part.p, s)))) return st;
  // pressureCorrection(dt) (:881)
  return cup2d_poisson_pressure_correction(h, dt, d_pres, d_vel, stream);
}

int cup2d_poisson_rhs_fourier_device(cup2d_poisson* h, int32_t kmax, const double* coef, double* d_b,
                                     void* stream) {
  if (!h || !coef || !d_b || kmax < 1 || kmax > kMaxFourierK || h->nb <= 0) return CUP2D_INVALID_ARGUMENT;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const int nm = fourier_mode_count(kmax);
  int st;
  // coefficients: sized for the largest kmax once; partials: grow with the
  // mesh, the old buffer freed behind the work already queued on s
  if ((st = h->rhs_coef.ensure(4 * (int64_t)fourier_mode_count(kMaxFourierK))) ||
      (st = h->rhs_part.ensure(rhs_partials(h->nb) + 1, s)))
    return st;
  if (cudaMemcpyAsync(h->rhs_coef.p, coef, sizeof(double) * 4 * nm, cudaMemcpyHostToDevice, s) != cudaSuccess)
    return CUP2D_CUDA_ERROR;
  const int64_t parts = rhs_partials(h->nb);
  return from_cuda(launch_rhs_fourier(forest_view(h), kmax, h->rhs_coef.p, d_b, h->rhs_part.p,
                                      h->rhs_part.p + parts, s));
}

int cup2d_poisson_transfer(const cup2d_poisson* src, const double* d_xsrc, const cup2d_poisson* dst, double* d_xdst,
                           void* stream) {
  if (!src || !dst || !d_xsrc || !d_xdst || d_xsrc == d_xdst || src->nb <= 0 || dst->nb <= 0)
    return CUP2D_INVALID_ARGUMENT;
  if (src->bpdx != dst->bpdx || src->bpdy != dst->bpdy || src->extent != dst->extent)
    return CUP2D_INVALID_ARGUMENT;  // not the same domain and root grid
  if (std::max(src->level_max, dst->level_max) + 1 + 3 + 7 > 62) return CUP2D_INVALID_ARGUMENT;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  return from_cuda(launch_transfer(forest_view(src), d_xsrc, forest_view(dst), d_xdst, s));
}

int cup2d_poisson_precond(cup2d_poisson* h, const double* d_p, double* d_z, void* stream) {
  if (!h || !d_p || !d_z) return CUP2D_INVALID_ARGUMENT;
  cudaStream_t s = static_cast<cudaStream_t>(stream);  // NULL: the legacy default stream
  return from_cuda(launch_precond64(h->P, h->nb, d_p, d_z, s));
}

int cup2d_poisson_precond32(cup2d_poisson* h, const float* d_p, float* d_z, void* stream) {
  if (!h || !d_p || !d_z) return CUP2D_INVALID_ARGUMENT;
  cudaStream_t s = static_cast<cudaStream_t>(stream);  // NULL: the legacy default stream
  return from_cuda(launch_precond32(h->P32, h->nb, d_p, d_z, s));
}

int cup2d_poisson_precond32_tc(cup2d_poisson* h, const float* d_p, float* d_z, void* stream) {
  if (!h || !d_p || !d_z || h->nb <= 0) return CUP2D_INVALID_ARGUMENT;
  cudaStream_t s = static_cast<cudaStream_t>(stream);  // NULL: the legacy default stream
  if (cudaMemsetAsync(h->err.p, 0, sizeof(int), s) != cudaSuccess) return CUP2D_CUDA_ERROR;
  if (launch_precond32_tc(h->P32, h->nb, d_p, d_z, h->err.p, s) != cudaSuccess) return CUP2D_CUDA_ERROR;
  int err = 0;
  if (cudaMemcpyAsync(&err, h->err.p, sizeof(int), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
      cudaStreamSynchronize(s) != cudaSuccess)
    return CUP2D_CUDA_ERROR;
  return err ? CUP2D_TIMEOUT : CUP2D_OK;
}

int cup2d_poisson_set_profiling(cup2d_poisson* h, int32_t enable) {
  if (!h) return CUP2D_INVALID_ARGUMENT;
  h->profiling = enable != 0;
  h->prof_grid = 0;  // next profiled solve starts from zero
  return CUP2D_OK;
}

int cup2d_poisson_profile(cup2d_poisson* h, double* compute_ms, double* wait_ms, int32_t nphases) {
  if (!h || !compute_ms || !wait_ms || nphases < kProfPhases) return CUP2D_INVALID_ARGUMENT;
  for (int q = 0; q < kProfPhases; ++q) compute_ms[q] = wait_ms[q] = 0.0;
  if (!h->profiling || h->prof_grid <= 0) return CUP2D_OK;
  const int g = h->prof_grid;
  std::vector<unsigned long long> t((size_t)g * kProfPhases * 2);
  if (cudaStreamSynchronize(h->stream) != cudaSuccess ||
      cudaMemcpy(t.data(), h->prof.p, t.size() * sizeof(unsigned long long), cudaMemcpyDeviceToHost) != cudaSuccess)
    return CUP2D_CUDA_ERROR;
  for (int c = 0; c < g; ++c)
    for (int q = 0; q < kProfPhases; ++q) {
      compute_ms[q] += 1e-6 * (double)t[((size_t)c * kProfPhases + q) * 2] / g;
      wait_ms[q] += 1e-6 * (double)t[((size_t)c * kProfPhases + q) * 2 + 1] / g;
    }
  return CUP2D_OK;
}

int cup2d_poisson_explicit_info(cup2d_poisson* h, int64_t* rows, int64_t* nnz) {
  if (!h) return CUP2D_INVALID_ARGUMENT;
  if (rows) *rows = h->mesh.R;
  if (nnz) *nnz = h->mesh.nnz;
  return CUP2D_OK;
}

// Expands the block-structured operator into the CSR that getMat would
// produce: interior rows as (iy-1, ix-1, self, ix+1, iy+1) with (1,1,-4,1,1);
// implicit edge rows in getMat's face order through an ordered map; explicit
// rows verbatim.
int cup2d_poisson_export_csr(cup2d_poisson* h, int64_t* n_out, int64_t* nnz_out, int64_t* row_ptr,
                             int32_t* col, double* val) {
  if (!h) return CUP2D_INVALID_ARGUMENT;
  const int64_t nb = h->nb, n = nb * kBLEN;
  std::vector<int32_t> nbr(4 * nb), xbase(nb + 1), xptr(h->mesh.R + 1), xcol(h->mesh.nnz);
  std::vector<unsigned long long> xmask(nb);
  std::vector<double> xval(h->mesh.nnz);
  if (cudaStreamSynchronize(h->stream) != cudaSuccess) return CUP2D_CUDA_ERROR;
  if (cudaMemcpy(nbr.data(), h->nbr.p, 4 * nb * sizeof(int32_t), cudaMemcpyDeviceToHost) != cudaSuccess ||
      cudaMemcpy(xbase.data(), h->xbase.p, (nb + 1) * sizeof(int32_t), cudaMemcpyDeviceToHost) != cudaSuccess ||
      cudaMemcpy(xmask.data(), h->xmask.p, nb * sizeof(unsigned long long), cudaMemcpyDeviceToHost) != cudaSuccess ||
      cudaMemcpy(xptr.data(), h->xptr.p, (h->mesh.R + 1) * sizeof(int32_t), cudaMemcpyDeviceToHost) != cudaSuccess)
    return CUP2D_CUDA_ERROR;
  if (h->mesh.nnz > 0 &&
      (cudaMemcpy(xcol.data(), h->xcol.p, h->mesh.nnz * sizeof(int32_t), cudaMemcpyDeviceToHost) != cudaSuccess ||
       cudaMemcpy(xval.data(), h->xval.p, h->mesh.nnz * sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess))
    return CUP2D_CUDA_ERROR;
  int64_t nnz = 0;
  const bool fill = row_ptr && col && val;
  if (fill) row_ptr[0] = 0;
  for (int64_t b = 0; b < nb; ++b)
    for (int c = 0; c < kBLEN; ++c) {
      const int ix = c & 7, iy = c >> 3;
      const int64_t self = b * kBLEN + c;
      auto push = [&](int64_t cc, double v) {
        if (fill) {
          col[nnz] = (int32_t)cc;
          val[nnz] = v;
        }
        ++nnz;
      };
      if (ix > 0 && ix < 7 && iy > 0 && iy < 7) {
        push(self - 8, 1);
        push(self - 1, 1);
        push(self, -4);
        push(self + 1, 1);
        push(self + 8, 1);
      } else if ((xmask[b] >> c) & 1ull) {
        const int r = xbase[b] + __builtin_popcountll(xmask[b] & ((1ull << c) - 1ull));
        for (int k = xptr[r]; k < xptr[r + 1]; ++k) push(xcol[k], xval[k]);
      } else {
        std::map<int64_t, double> row;
        const bool valid[4] = {ix > 0, ix < 7, iy > 0, iy < 7};
        const int64_t inb[4] = {self - 1, self + 1, self - 8, self + 8};
        for (int f = 0; f < 4; ++f) {
          int64_t nc = -1;
          if (valid[f]) {
            nc = inb[f];
          } else if (nbr[4 * b + f] >= 0) {
            const int64_t o = (int64_t)nbr[4 * b + f] * kBLEN;
            nc = f == 0 ? o + iy * 8 + 7 : f == 1 ? o + iy * 8 : f == 2 ? o + 56 + ix : o + ix;
          } else {
            continue;  // wall
          }
          row[nc] += 1.0;
          row[self] += -1.0;
        }
        for (auto& kv : row) push(kv.first, kv.second);
      }
      if (fill) row_ptr[self + 1] = nnz;
    }
  if (n_out) *n_out = n;
  if (nnz_out) *nnz_out = nnz;
  return CUP2D_OK;
}

}  // extern "C"

// ================================================================ batches ==
//
// A batch is a set of independent problems solved in one cooperative
// launch (k_bicgstab_batch64 / k_bicgstab_batch_mixed): groups of `team`
// CTAs take problems largest first from a device queue.  Each problem keeps
// its own assembled operator and Krylov vectors (a handle without a stream
// of its own); the per-problem descriptors are rebuilt on the host for each
// solve because the right-hand sides and solutions are call arguments.

// One whole batched solve recorded as a CUDA graph: state resets, the
// persistent launch, the read-back of the statistics into pinned memory.
struct BatchGraph {
  cudaGraphExec_t exec = nullptr;
  cudaEvent_t done = nullptr;   // recorded after each replay
  DevBuf<Problem64> p64;        // the graph's own problem descriptors
  DevBuf<ProblemMixed> pmx;
  DevStats* hstats = nullptr;   // pinned, n entries followed by the abort flag
  int* habort = nullptr;
  int n = 0;
  bool replayed = false;
  void reset() {  // the graph only; buffers stay for the next capture
    if (exec) cudaGraphExecDestroy(exec);
    exec = nullptr;
    replayed = false;
  }
  void release() {
    reset();
    p64.release();
    pmx.release();
    if (hstats) cudaFreeHost(hstats);
    hstats = nullptr;
    habort = nullptr;
    if (done) cudaEventDestroy(done);
    done = nullptr;
  }
};

struct cup2d_batch {
  int device = 0;
  cudaStream_t stream = nullptr;
  cup2d_solve_opts opts{};
  std::vector<cup2d_poisson*> probs;
  std::vector<int32_t> order;  // largest first
  int team = 8;
  int grid64 = 0, gridmx = 0;
  int sms = 0, ctas_per_sm = 0;  // occupancy cap, 0 = every co-resident CTA
  DevBuf<Problem64> d_p64;
  DevBuf<ProblemMixed> d_pmx;
  DevBuf<int32_t> d_order;
  DevBuf<double> red;
  DevBuf<unsigned> bars;
  DevBuf<int> slots, queue, abort_flag;
  DevBuf<DevStats> dstats;
  const double* P = nullptr;  // the device's shared P^-1
  const float* P32 = nullptr;
  std::vector<Problem64> h_p64;
  std::vector<ProblemMixed> h_pmx;
  std::vector<DevStats> hstats;
  std::vector<const double*> stage_b;  // host-buffer solves: per-problem device copies
  std::vector<double*> stage_x;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  float last_ms = 0.f;
  bool have_timeline = false;
  DevBuf<unsigned long long> prof;  // phase timers (profiling on)
  bool profiling = false;
  int prof_grid = 0;
  BatchGraph graph;
};

extern "C" {

int cup2d_batch_destroy(cup2d_batch* B) {
  if (!B) return CUP2D_OK;
  cudaDeviceSynchronize();  // launches may have been queued on any stream
  for (auto* h : B->probs) cup2d::handle_destroy_idle(h);
  B->d_p64.release();
  B->d_pmx.release();
  B->d_order.release();
  B->red.release();
  B->bars.release();
  B->slots.release();
  B->queue.release();
  B->abort_flag.release();
  B->dstats.release();
  B->prof.release();
  B->graph.release();
  if (B->ev0) cudaEventDestroy(B->ev0);
  if (B->ev1) cudaEventDestroy(B->ev1);
  if (B->stream) cudaStreamDestroy(B->stream);
  delete B;
  return CUP2D_OK;
}

int cup2d_batch_create(int32_t n, const cup2d_forest* forests, const cup2d_solve_opts* opts, cup2d_batch** out) {
  if (!out || n <= 0 || !forests) return CUP2D_INVALID_ARGUMENT;
  *out = nullptr;
  cup2d_solve_opts o;
  cup2d_default_opts(&o);
  if (opts) o = *opts;
  int st = validate_opts(o);
  if (st) return st;
  if (o.mean_constraint) return CUP2D_INVALID_ARGUMENT;  // single solves only
  for (int32_t i = 0; i < n; ++i)
    if ((st = check_forest(&forests[i]))) return st;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return CUP2D_NO_DEVICE;
  }
  auto* B = new (std::nothrow) cup2d_batch();
  if (!B) return CUP2D_OOM;
  B->opts = o;
  cudaGetDevice(&B->device);
  if (cudaStreamCreateWithFlags(&B->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreate(&B->ev0) != cudaSuccess || cudaEventCreate(&B->ev1) != cudaSuccess ||
      cudaEventCreateWithFlags(&B->graph.done, cudaEventDisableTiming) != cudaSuccess) {
    cup2d_batch_destroy(B);
    return CUP2D_CUDA_ERROR;
  }
  B->grid64 = max_coop_grid_batch(B->device, false);
  B->gridmx = max_coop_grid_batch(B->device, true);
  cudaDeviceGetAttribute(&B->sms, cudaDevAttrMultiProcessorCount, B->device);
  if (B->grid64 <= 0 || B->gridmx <= 0 || B->sms <= 0) {
    cup2d_batch_destroy(B);
    return CUP2D_CUDA_ERROR;
  }
  B->probs.reserve(n);
  for (int32_t i = 0; i < n; ++i) {
    auto* h = new (std::nothrow) cup2d_poisson();
    if (!h) {
      cup2d_batch_destroy(B);
      return CUP2D_OOM;
    }
    h->device = B->device;
    h->stream = B->stream;
    h->owns_stream = false;
    h->opts = o;
    B->probs.push_back(h);
    if ((st = do_assemble(h, &forests[i]))) {
      cup2d_batch_destroy(B);
      return st;
    }
  }
  B->order.resize(n);
  for (int32_t i = 0; i < n; ++i) B->order[i] = i;
  std::stable_sort(B->order.begin(), B->order.end(),
                   [&](int32_t a, int32_t b) { return B->probs[a]->nb > B->probs[b]->nb; });
  const int gmax = std::max(B->grid64, B->gridmx);
  if ((st = B->d_p64.ensure(n)) || (st = B->d_pmx.ensure(n)) || (st = B->d_order.ensure(n)) ||
      (st = B->red.ensure((int64_t)kRedQ * gmax)) || (st = B->bars.ensure(gmax)) || (st = B->slots.ensure(gmax)) ||
      (st = B->queue.ensure(1)) || (st = B->abort_flag.ensure(1)) || (st = B->dstats.ensure(n)) ||
      (st = shared_pinv(&B->P, &B->P32))) {
    cup2d_batch_destroy(B);
    return st;
  }
  if (cudaMemcpyAsync(B->d_order.p, B->order.data(), sizeof(int32_t) * n, cudaMemcpyHostToDevice, B->stream) !=
          cudaSuccess ||
      cudaStreamSynchronize(B->stream) != cudaSuccess) {
    cup2d_batch_destroy(B);
    return CUP2D_CUDA_ERROR;
  }
  B->h_p64.resize(n);
  B->h_pmx.resize(n);
  B->hstats.resize(n);
  B->stage_b.resize(n);
  B->stage_x.resize(n);
  if (const char* e = std::getenv("CUP2D_BATCH_TEAM")) B->team = std::max(1, std::atoi(e));
  *out = B;
  return CUP2D_OK;
}

int cup2d_batch_set_opts(cup2d_batch* B, const cup2d_solve_opts* opts) {
  if (!B || !opts) return CUP2D_INVALID_ARGUMENT;
  int st = validate_opts(*opts);
  if (st) return st;
  if (opts->mean_constraint) return CUP2D_INVALID_ARGUMENT;  // single solves only
  B->opts = *opts;
  return CUP2D_OK;
}

int cup2d_batch_set_team(cup2d_batch* B, int32_t team) {
  if (!B || team < 1 || team > 256) return CUP2D_INVALID_ARGUMENT;
  B->team = team;
  return CUP2D_OK;
}

int cup2d_batch_set_occupancy(cup2d_batch* B, int32_t ctas_per_sm) {
  if (!B || ctas_per_sm < 0 || ctas_per_sm > 32) return CUP2D_INVALID_ARGUMENT;
  B->ctas_per_sm = ctas_per_sm;
  return CUP2D_OK;
}

int32_t cup2d_batch_size(const cup2d_batch* B) { return B ? (int32_t)B->probs.size() : 0; }

int64_t cup2d_batch_num_cells(const cup2d_batch* B, int32_t i) {
  if (!B || i < 0 || i >= (int32_t)B->probs.size()) return 0;
  return B->probs[i]->nb * kBLEN;
}

}  // extern "C"

namespace {

// Validates the batch's inputs, fills the host-side problem descriptors and
// the launch arguments (descriptor arrays at the given device addresses)
// and picks the grid: groups of `team` CTAs, as many as fit the occupancy
// cap, never more groups than problems.
int batch_prepare(cup2d_batch* B, const double* const* d_b, double* const* d_x, Problem64* dp64,
                  ProblemMixed* dpmx, BatchArgs& a, int& grid) {
  if (!B || !d_b || !d_x) return CUP2D_INVALID_ARGUMENT;
  const int n = (int)B->probs.size();
  for (int i = 0; i < n; ++i)
    if (!d_b[i] || !d_x[i] || !aligned16(d_b[i]) || !aligned16(d_x[i])) return CUP2D_INVALID_ARGUMENT;
  const cup2d_solve_opts& o = B->opts;
  const bool mixed = o.precision == CUP2D_PREC_MIXED;
  int st;
  for (int i = 0; i < n; ++i) {
    cup2d_poisson* h = B->probs[i];
    if ((st = mixed ? ensure_mixed(h) : ensure_fp64(h))) return st;
    const MeshView M = h->mesh.view();
    if (mixed)
      B->h_pmx[i] = ProblemMixed{M, d_b[i], d_x[i], h->xo.p, h->f_r.p, h->f_rh.p, h->f_p.p, h->f_nu.p,
                                 h->f_t.p, h->f_z.p, h->f_z2.p, B->dstats.p + i};
    else
      B->h_p64[i] = Problem64{M, d_b[i], d_x[i], h->xo.p, h->r.p, h->rh.p, h->p.p, h->nu.p, h->t.p, h->z.p, h->z2.p,
                              B->dstats.p + i};
  }
  const int team = B->team;
  int gmax = mixed ? B->gridmx : B->grid64;
  if (B->ctas_per_sm > 0) gmax = std::min(gmax, B->ctas_per_sm * B->sms);
  const int groups = std::max(1, std::min(gmax / team, n));
  if (groups * team > gmax) return CUP2D_INVALID_ARGUMENT;  // team larger than the device
  grid = groups * team;
  // per group: barriers of every problem it may take, in 32 bits
  const uint64_t arrivals = ((uint64_t)o.max_iter * 7 + 16) * (uint64_t)n * (uint64_t)team;
  if (arrivals >= (1ull << 32)) return CUP2D_INVALID_ARGUMENT;
  a = BatchArgs{};
  a.p64 = dp64;
  a.pmx = dpmx;
  a.order = B->d_order.p;
  a.nprob = n;
  a.team = team;
  a.P = B->P;
  a.P32 = B->P32;
  a.red = B->red.p;
  a.bars = B->bars.p;
  a.slots = B->slots.p;
  a.queue = B->queue.p;
  a.abort_flag = B->abort_flag.p;
  a.sp = SolveParams{o.tol_abs, o.tol_rel, o.reliable_delta, o.max_restarts, o.max_iter, o.subtract_mean,
                     o.reliable_restart};
  a.timeout_ns = (unsigned long long)o.timeout_ms * 1000000ull;
  a.prof = nullptr;
  return CUP2D_OK;
}

// The per-launch state resets and the launch itself, in stream order.
cudaError_t batch_enqueue(cup2d_batch* B, const BatchArgs& a, int grid, int groups, cudaStream_t s) {
  cudaError_t e;
  if ((e = cudaMemsetAsync(B->bars.p, 0, sizeof(unsigned) * groups, s)) != cudaSuccess ||
      (e = cudaMemsetAsync(B->queue.p, 0, sizeof(int), s)) != cudaSuccess ||
      (e = cudaMemsetAsync(B->abort_flag.p, 0, sizeof(int), s)) != cudaSuccess)
    return e;
  return launch_bicgstab_batch(a, grid, B->opts.precision == CUP2D_PREC_MIXED, s);
}

void batch_fill_stats(const DevStats* hs, int n, int aborted, float ms, cup2d_solve_stats* stats) {
  for (int i = 0; i < n; ++i) {
    const DevStats& d = hs[i];
    stats[i].status = aborted ? CUP2D_TIMEOUT : d.status;
    stats[i].iterations = d.iterations;
    stats[i].restarts = d.restarts;
    stats[i].refinements = d.refinements;
    stats[i].err_init = d.err_init;
    stats[i].err_final = d.err_opt;
    stats[i].rel_res_inf = d.err_init > 0 ? d.err_opt / d.err_init : 0.0;
    stats[i].solve_ms = aborted ? ms : (double)(d.t_end - d.t_begin) * 1e-6;  // this problem's own span
  }
}

}  // namespace

extern "C" {

int cup2d_batch_solve_device(cup2d_batch* B, const double* const* d_b, double* const* d_x,
                             cup2d_solve_stats* stats, void* stream) {
  if (!B) return CUP2D_INVALID_ARGUMENT;
  BatchArgs a;
  int grid = 0, st;
  if ((st = batch_prepare(B, d_b, d_x, B->d_p64.p, B->d_pmx.p, a, grid))) return st;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const int n = (int)B->probs.size();
  const bool mixed = B->opts.precision == CUP2D_PREC_MIXED;
  if ((mixed ? cudaMemcpyAsync(B->d_pmx.p, B->h_pmx.data(), sizeof(ProblemMixed) * n, cudaMemcpyHostToDevice, s)
             : cudaMemcpyAsync(B->d_p64.p, B->h_p64.data(), sizeof(Problem64) * n, cudaMemcpyHostToDevice, s)) !=
      cudaSuccess)
    return CUP2D_CUDA_ERROR;
  if (B->profiling) {
    const int64_t words = (int64_t)grid * kProfPhases * 2;
    // sized once for the batch's largest grid (see the single-solve timers)
    if ((st = B->prof.ensure((int64_t)std::max(B->grid64, B->gridmx) * kProfPhases * 2))) return st;
    if (B->prof_grid != grid) {  // timers accumulate over launches of one grid size
      if (cudaMemsetAsync(B->prof.p, 0, sizeof(unsigned long long) * words, s) != cudaSuccess)
        return CUP2D_CUDA_ERROR;
      B->prof_grid = grid;
    }
    a.prof = B->prof.p;
  }
  if (stats) cudaEventRecord(B->ev0, s);
  const cudaError_t e = batch_enqueue(B, a, grid, grid / a.team, s);
  if (e != cudaSuccess) return from_cuda(e);
  if (!stats) return CUP2D_OK;
  cudaEventRecord(B->ev1, s);
  int aborted = 0;
  if (cudaMemcpyAsync(B->hstats.data(), B->dstats.p, sizeof(DevStats) * n, cudaMemcpyDeviceToHost, s) !=
          cudaSuccess ||
      cudaMemcpyAsync(&aborted, B->abort_flag.p, sizeof(int), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
      cudaStreamSynchronize(s) != cudaSuccess)
    return CUP2D_CUDA_ERROR;
  float ms = 0.f;
  cudaEventElapsedTime(&ms, B->ev0, B->ev1);
  B->last_ms = ms;
  B->have_timeline = !aborted;
  batch_fill_stats(B->hstats.data(), n, aborted, ms, stats);
  return aborted ? CUP2D_TIMEOUT : CUP2D_OK;
}

int cup2d_batch_capture(cup2d_batch* B, const double* const* d_b, double* const* d_x, int32_t flags) {
  if (!B || (flags & ~CUP2D_GRAPH_ZERO_X)) return CUP2D_INVALID_ARGUMENT;
  BatchGraph& g = B->graph;
  if (g.replayed && cudaEventSynchronize(g.done) != cudaSuccess) return CUP2D_CUDA_ERROR;
  g.reset();
  const int n = (int)B->probs.size();
  const bool mixed = B->opts.precision == CUP2D_PREC_MIXED;
  int st;
  if ((st = mixed ? g.pmx.ensure(n) : g.p64.ensure(n))) return st;
  BatchArgs a;
  int grid = 0;
  if ((st = batch_prepare(B, d_b, d_x, g.p64.p, g.pmx.p, a, grid))) return st;
  if (!g.hstats && cudaMallocHost(&g.hstats, sizeof(DevStats) * n + sizeof(int)) != cudaSuccess) {
    g.hstats = nullptr;
    return CUP2D_OOM;
  }
  g.habort = reinterpret_cast<int*>(g.hstats + n);
  // the graph's own descriptors: solves outside the graph keep theirs
  cudaStream_t s = B->stream;
  if ((mixed ? cudaMemcpyAsync(g.pmx.p, B->h_pmx.data(), sizeof(ProblemMixed) * n, cudaMemcpyHostToDevice, s)
             : cudaMemcpyAsync(g.p64.p, B->h_p64.data(), sizeof(Problem64) * n, cudaMemcpyHostToDevice, s)) !=
          cudaSuccess ||
      cudaStreamSynchronize(s) != cudaSuccess)
    return CUP2D_CUDA_ERROR;
  if (cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal) != cudaSuccess) return CUP2D_CUDA_ERROR;
  cudaError_t e = cudaSuccess;
  if (flags & CUP2D_GRAPH_ZERO_X)
    for (int i = 0; i < n && e == cudaSuccess; ++i)
      e = cudaMemsetAsync(d_x[i], 0, sizeof(double) * B->probs[i]->nb * kBLEN, s);
  if (e == cudaSuccess) e = cudaEventRecordWithFlags(B->ev0, s, cudaEventRecordExternal);
  if (e == cudaSuccess) e = batch_enqueue(B, a, grid, grid / a.team, s);
  if (e == cudaSuccess) e = cudaEventRecordWithFlags(B->ev1, s, cudaEventRecordExternal);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(g.hstats, B->dstats.p, sizeof(DevStats) * n, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(g.habort, B->abort_flag.p, sizeof(int), cudaMemcpyDeviceToHost, s);
  cudaGraph_t graph = nullptr;
  const cudaError_t e2 = cudaStreamEndCapture(s, &graph);
  if (e == cudaSuccess) e = e2;
  if (e == cudaSuccess) e = cudaGraphInstantiate(&g.exec, graph, 0);
  if (graph) cudaGraphDestroy(graph);
  if (e != cudaSuccess) {
    cudaGetLastError();
    g.exec = nullptr;
    return from_cuda(e);
  }
  g.n = n;
  return CUP2D_OK;
}

int cup2d_batch_replay(cup2d_batch* B, void* stream) {
  if (!B || !B->graph.exec) return CUP2D_INVALID_ARGUMENT;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (cudaGraphLaunch(B->graph.exec, s) != cudaSuccess || cudaEventRecord(B->graph.done, s) != cudaSuccess)
    return CUP2D_CUDA_ERROR;
  B->graph.replayed = true;
  return CUP2D_OK;
}

int cup2d_batch_replay_stats(cup2d_batch* B, cup2d_solve_stats* stats) {
  if (!B || !B->graph.exec || !B->graph.replayed || !stats) return CUP2D_INVALID_ARGUMENT;
  BatchGraph& g = B->graph;
  if (cudaEventSynchronize(g.done) != cudaSuccess) return CUP2D_CUDA_ERROR;
  float ms = 0.f;
  cudaEventElapsedTime(&ms, B->ev0, B->ev1);
  B->last_ms = ms;
  const int aborted = *g.habort;
  B->have_timeline = !aborted;
  std::memcpy(B->hstats.data(), g.hstats, sizeof(DevStats) * g.n);
  batch_fill_stats(g.hstats, g.n, aborted, ms, stats);
  return aborted ? CUP2D_TIMEOUT : CUP2D_OK;
}

int cup2d_batch_tune(cup2d_batch* B, const double* const* d_b, double* const* d_x, const int32_t* teams,
                     int32_t nteams, const int32_t* ctas_per_sm, int32_t ncps, int32_t iters, double* rates,
                     int32_t* best_team, int32_t* best_ctas_per_sm) {
  if (!B || !d_b || !d_x || !teams || nteams < 1 || iters < 0 || !best_team) return CUP2D_INVALID_ARGUMENT;
  if (ncps < 0 || (ncps > 0 && !ctas_per_sm)) return CUP2D_INVALID_ARGUMENT;
  const cup2d_solve_opts saved = B->opts;
  const int saved_team = B->team, saved_cps = B->ctas_per_sm;
  const int n = (int)B->probs.size();
  std::vector<double*> x0;  // full solves: every candidate starts from the caller's x
  if (iters > 0) {          // fixed work: every problem runs exactly `iters` iterations
    cup2d_solve_opts o = saved;
    o.tol_abs = 0.0;
    o.tol_rel = 0.0;
    o.max_iter = iters;
    o.max_restarts = std::max(o.max_restarts, iters + 1);
    B->opts = o;
  } else {
    for (int i = 0; i < n; ++i) {
      double* c = nullptr;
      const size_t bytes = sizeof(double) * B->probs[i]->nb * kBLEN;
      if (!d_x[i] || cudaMallocAsync(reinterpret_cast<void**>(&c), bytes, B->stream) != cudaSuccess ||
          cudaMemcpyAsync(c, d_x[i], bytes, cudaMemcpyDeviceToDevice, B->stream) != cudaSuccess) {
        cudaGetLastError();
        for (double* q : x0) cudaFreeAsync(q, B->stream);
        if (c) cudaFreeAsync(c, B->stream);
        cudaStreamSynchronize(B->stream);
        return d_x[i] ? CUP2D_OOM : CUP2D_INVALID_ARGUMENT;
      }
      x0.push_back(c);
    }
  }
  auto restart_x = [&]() {
    for (int i = 0; i < (int)x0.size(); ++i)
      cudaMemcpyAsync(d_x[i], x0[i], sizeof(double) * B->probs[i]->nb * kBLEN, cudaMemcpyDeviceToDevice,
                      B->stream);
  };
  std::vector<cup2d_solve_stats> st(n);
  double best_rate = -1.0;
  int best = saved_team, best_cps = saved_cps, status = CUP2D_OK;
  const int nc = std::max(ncps, 1);
  for (int k = 0; k < nteams && status == CUP2D_OK; ++k) {
    for (int c = 0; c < nc; ++c) {
      const int cps = ncps > 0 ? ctas_per_sm[c] : saved_cps;
      if (teams[k] < 1 || teams[k] > 256 || cps < 0 || cps > 32) {
        status = CUP2D_INVALID_ARGUMENT;
        break;
      }
      B->team = teams[k];
      B->ctas_per_sm = cps;
      double rate = 0.0;
      restart_x();
      int s = cup2d_batch_solve_device(B, d_b, d_x, st.data(), B->stream);  // warm-up
      restart_x();
      if (s == CUP2D_OK) s = cup2d_batch_solve_device(B, d_b, d_x, st.data(), B->stream);
      if (s == CUP2D_OK && B->last_ms > 0.f) {
        double work = 0.0;
        for (int i = 0; i < n; ++i) work += (double)st[i].iterations * (double)B->probs[i]->nb * kBLEN;
        rate = work / (1e-3 * B->last_ms);
      } else if (s != CUP2D_OK && s != CUP2D_INVALID_ARGUMENT) {
        status = s;
        break;
      }
      if (rates) rates[k * nc + c] = rate;
      if (rate > best_rate) {
        best_rate = rate;
        best = teams[k];
        best_cps = cps;
      }
    }
  }
  for (double* q : x0) cudaFreeAsync(q, B->stream);
  cudaStreamSynchronize(B->stream);
  B->opts = saved;
  B->team = status == CUP2D_OK ? best : saved_team;
  B->ctas_per_sm = status == CUP2D_OK ? best_cps : saved_cps;
  *best_team = B->team;
  if (best_ctas_per_sm) *best_ctas_per_sm = B->ctas_per_sm;
  return status;
}

int cup2d_batch_solve(cup2d_batch* B, const double* const* b, double* const* x, cup2d_solve_stats* stats) {
  if (!B || !b || !x) return CUP2D_INVALID_ARGUMENT;
  const int n = (int)B->probs.size();
  cudaStream_t s = B->stream;
  int st;
  for (int i = 0; i < n; ++i) {
    if (!b[i] || !x[i]) return CUP2D_INVALID_ARGUMENT;
    cup2d_poisson* h = B->probs[i];
    const int64_t m = h->nb * kBLEN;
    if ((st = h->bstage.ensure(m)) || (st = h->xstage.ensure(m))) return st;
    B->stage_b[i] = h->bstage.p;
    B->stage_x[i] = h->xstage.p;
    if (cudaMemcpyAsync(h->bstage.p, b[i], sizeof(double) * m, cudaMemcpyHostToDevice, s) != cudaSuccess ||
        cudaMemcpyAsync(h->xstage.p, x[i], sizeof(double) * m, cudaMemcpyHostToDevice, s) != cudaSuccess)
      return CUP2D_CUDA_ERROR;
  }
  std::vector<cup2d_solve_stats> local;
  if (!stats) {
    local.resize(n);
    stats = local.data();
  }
  st = cup2d_batch_solve_device(B, B->stage_b.data(), B->stage_x.data(), stats, s);
  if (st != CUP2D_OK) return st;
  for (int i = 0; i < n; ++i)
    if (cudaMemcpyAsync(x[i], B->stage_x[i], sizeof(double) * B->probs[i]->nb * kBLEN, cudaMemcpyDeviceToHost,
                        s) != cudaSuccess)
      return CUP2D_CUDA_ERROR;
  return cudaStreamSynchronize(s) == cudaSuccess ? CUP2D_OK : CUP2D_CUDA_ERROR;
}

int cup2d_batch_set_profiling(cup2d_batch* B, int32_t enable) {
  if (!B) return CUP2D_INVALID_ARGUMENT;
  B->profiling = enable != 0;
  B->prof_grid = 0;
  return CUP2D_OK;
}

int cup2d_batch_profile(cup2d_batch* B, double* compute_ms, double* wait_ms, int32_t nphases) {
  if (!B || !compute_ms || !wait_ms || nphases < kProfPhases) return CUP2D_INVALID_ARGUMENT;
  for (int q = 0; q < kProfPhases; ++q) compute_ms[q] = wait_ms[q] = 0.0;
  if (!B->profiling || B->prof_grid <= 0) return CUP2D_OK;
  const int g = B->prof_grid;
  std::vector<unsigned long long> t((size_t)g * kProfPhases * 2);
  if (cudaDeviceSynchronize() != cudaSuccess ||
      cudaMemcpy(t.data(), B->prof.p, t.size() * sizeof(unsigned long long), cudaMemcpyDeviceToHost) != cudaSuccess)
    return CUP2D_CUDA_ERROR;
  for (int c = 0; c < g; ++c)
    for (int q = 0; q < kProfPhases; ++q) {
      compute_ms[q] += 1e-6 * (double)t[((size_t)c * kProfPhases + q) * 2] / g;
      wait_ms[q] += 1e-6 * (double)t[((size_t)c * kProfPhases + q) * 2 + 1] / g;
    }
  return CUP2D_OK;
}

int cup2d_batch_timeline(const cup2d_batch* B, double* begin_ms, double* end_ms, double* launch_ms) {
  if (!B || !begin_ms || !end_ms || !B->have_timeline) return CUP2D_INVALID_ARGUMENT;
  const int n = (int)B->probs.size();
  unsigned long long t0 = ~0ull;
  for (int i = 0; i < n; ++i) t0 = std::min(t0, B->hstats[i].t_begin);
  for (int i = 0; i < n; ++i) {
    begin_ms[i] = (double)(B->hstats[i].t_begin - t0) * 1e-6;
    end_ms[i] = (double)(B->hstats[i].t_end - t0) * 1e-6;
  }
  if (launch_ms) *launch_ms = B->last_ms;
  return CUP2D_OK;
}

}  // extern "C"

namespace cup2d {

int64_t handle_bytes(const cup2d_poisson* h) {
  if (!h) return 0;
  int64_t n = 0;
  const DevBuf<int32_t>* i32[] = {&h->level, &h->bx, &h->by, &h->table, &h->nbr, &h->xcount, &h->xbase,
                                  &h->scan_tmp, &h->rowlen, &h->xptr, &h->xcol, &h->rowcell};
  for (auto* b : i32) n += b->cap * (int64_t)sizeof(int32_t);
  n += h->xmask.cap * (int64_t)sizeof(unsigned long long);
  const DevBuf<double>* f64[] = {&h->hblk, &h->xval, &h->xo, &h->r, &h->rh, &h->p, &h->nu,
                                 &h->t, &h->z, &h->z2, &h->bstage, &h->xstage, &h->red, &h->rhs_coef,
                                 &h->rhs_part};
  for (auto* b : f64) n += b->cap * (int64_t)sizeof(double);
  const DevBuf<float>* f32[] = {&h->xval32, &h->f_r, &h->f_rh, &h->f_p, &h->f_nu, &h->f_t, &h->f_z, &h->f_z2};
  for (auto* b : f32) n += b->cap * (int64_t)sizeof(float);
  return n;
}

int handle_stage(cup2d_poisson* h, double** d_b, double** d_x) {
  if (!h || !d_b || !d_x) return CUP2D_INVALID_ARGUMENT;
  const int64_t n = h->nb * kBLEN;
  int st;
  if ((st = h->bstage.ensure(n)) || (st = h->xstage.ensure(n))) return st;
  *d_b = h->bstage.p;
  *d_x = h->xstage.p;
  return CUP2D_OK;
}

namespace {
struct RawStats {
  DevStats d;
  int aborted;
};
}  // namespace

size_t handle_stats_bytes() { return sizeof(RawStats); }

int handle_solve_async(cup2d_poisson* h, const double* d_b, double* d_x, cudaStream_t stream, void* raw) {
  if (!raw) return CUP2D_INVALID_ARGUMENT;
  if (h->opts.precision == CUP2D_PREC_MIXED) {
    const int st = ensure_mixed(h);
    if (st) return st;
  }
  const int st = cup2d_poisson_solve_device(h, d_b, d_x, nullptr, stream);
  if (st) return st;
  auto* rs = static_cast<RawStats*>(raw);
  if (cudaMemcpyAsync(&rs->d, h->dstats.p, sizeof(DevStats), cudaMemcpyDeviceToHost, stream) != cudaSuccess ||
      cudaMemcpyAsync(&rs->aborted, h->abort_flag.p, sizeof(int), cudaMemcpyDeviceToHost, stream) != cudaSuccess)
    return CUP2D_CUDA_ERROR;
  return CUP2D_OK;
}

void handle_stats_from_raw(const void* raw, double solve_ms, cup2d_solve_stats* out) {
  const auto* rs = static_cast<const RawStats*>(raw);
  const DevStats& d = rs->d;
  out->status = rs->aborted ? CUP2D_TIMEOUT : d.status;
  out->iterations = d.iterations;
  out->restarts = d.restarts;
  out->refinements = d.refinements;
  out->err_init = d.err_init;
  out->err_final = d.err_opt;
  out->rel_res_inf = d.err_init > 0 ? d.err_opt / d.err_init : 0.0;
  out->solve_ms = solve_ms;
}

int handle_view(const cup2d_poisson* h, HandleView* out) {
  if (!h || !out || h->nb <= 0) return CUP2D_INVALID_ARGUMENT;
  out->device = h->device;
  out->M = h->mesh.view();
  out->P = h->P;
  out->nb = h->nb;
  out->grid = h->grid_for(h->grid64);
  out->opts = h->opts;
  out->ev0 = h->ev0;
  out->ev1 = h->ev1;
  return CUP2D_OK;
}

}  // namespace cup2d
