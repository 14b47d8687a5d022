// FP64 solve that allocates no device memory.
//
// cup2d_poisson_solve_device allocates its Krylov vectors and reduction
// scratch through the handle the first time they are needed.  Some callers
// must not allocate device memory at solve time: an application whose device
// memory is owned by its own pool allocator (the rest of the GPU is already
// claimed), or a time-step loop that cannot afford the device-wide
// synchronisation cudaMalloc/cudaFree can cause.  This entry point runs the
// same FP64 persistent kernel (k_bicgstab64) with all of its scratch (eight
// Krylov vectors, per-CTA reduction partials, the grid-barrier counter, the
// abort flag and the statistics) in one file-scope
// static device array, so the call itself allocates nothing: no cudaMalloc,
// no cudaFree, no allocating library routine.
//
// Limits and rules (also in include/cup2d_poisson.h):
//  * at most kNoAllocMaxBlocks = 4096 blocks (262,144 cells) and 1024 CTAs;
//    larger problems are rejected with CUP2D_INVALID_ARGUMENT;
//  * the array is 16.2 MiB of static device memory, committed on a GPU when
//    the first handle is created there and held until the process exits;
//  * all calls share the array, which keeps the last call's contents; calls
//    whose work overlaps on the GPU (other streams, other threads) race, so
//    callers serialise them;
//  * the array's device address is looked up with cudaGetSymbolAddress, once
//    per device, when the first handle is created on that device
//    (cup2d_poisson_create calls noalloc_prepare with the device current).
//    Under CUDA's lazy module loading (the default) that lookup is what
//    loads this file's module and commits the array, so the memory is taken
//    at handle creation, where allocating is expected, and never inside a
//    no-allocation solve.  A solve on a device without a prepared address
//    (not expected) looks it up itself; that path may allocate, so it is
//    not meant to run inside a stream capture.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <mutex>
#include <vector>

#include "../../include/cup2d_poisson.h"
#include "handle_view.hpp"
#include "kernels.hpp"

namespace cup2d {
namespace {

constexpr int64_t kNoAllocMaxBlocks = CUP2D_NOALLOC_MAX_BLOCKS;
constexpr int64_t kNoAllocMaxCells = kNoAllocMaxBlocks * kBLEN;
constexpr int kNoAllocMaxGrid = 1024;
constexpr int kMaxDevices = 64;

constexpr size_t align256(size_t v) { return (v + 255) & ~size_t(255); }

// Scratch layout (byte offsets, 256-byte aligned)
constexpr size_t kVecBytes = align256(sizeof(double) * kNoAllocMaxCells);
constexpr size_t kOffVec = 0;  // xo, r, rh, p, nu, t, z, z2
constexpr size_t kOffRed = kOffVec + 8 * kVecBytes;
constexpr size_t kOffBar = kOffRed + align256(sizeof(double) * kRedQ * kNoAllocMaxGrid);
constexpr size_t kOffAbort = kOffBar + 256;
constexpr size_t kOffStats = kOffAbort + 256;
constexpr size_t kScratchBytes = kOffStats + align256(sizeof(DevStats));

}  // namespace
}  // namespace cup2d

// The scratch of every call of cup2d_poisson_solve_device_noalloc.
static __device__ __align__(256) unsigned char g_noalloc_scratch[cup2d::kScratchBytes];

namespace cup2d {
namespace {

std::mutex g_scratch_mu;
char* g_scratch_base[kMaxDevices] = {};

}  // namespace

// Device address of the scratch on the current device (looked up once).
int noalloc_scratch_base(int device, char** out) {
  if (device < 0 || device >= kMaxDevices) return CUP2D_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lock(g_scratch_mu);
  if (!g_scratch_base[device]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) {
      cudaGetLastError();
      return CUP2D_CUDA_ERROR;
    }
    g_scratch_base[device] = static_cast<char*>(p);
  }
  *out = g_scratch_base[device];
  return CUP2D_OK;
}

int noalloc_prepare(int device) {
  char* base = nullptr;
  return noalloc_scratch_base(device, &base);
}

}  // namespace cup2d

extern "C" int cup2d_poisson_solve_device_noalloc(cup2d_poisson* h, const double* d_b, double* d_x,
                                                  cup2d_solve_stats* stats, void* stream) {
  using namespace cup2d;
  if (!h || !d_b || !d_x) return CUP2D_INVALID_ARGUMENT;
  if (!aligned16(d_b) || !aligned16(d_x)) return CUP2D_INVALID_ARGUMENT;  // 16-byte vector accesses
  HandleView v;
  if (handle_view(h, &v) != CUP2D_OK) return CUP2D_INVALID_ARGUMENT;
  if (v.nb > kNoAllocMaxBlocks) return CUP2D_INVALID_ARGUMENT;  // beyond the static scratch
  int current = -1;
  if (cudaGetDevice(&current) != cudaSuccess || current != v.device) return CUP2D_INVALID_ARGUMENT;
  char* base = nullptr;
  int st = noalloc_scratch_base(current, &base);
  if (st != CUP2D_OK) return st;
  const cup2d_solve_opts& o = v.opts;
  if (o.mean_constraint) return CUP2D_INVALID_ARGUMENT;  // the plain FP64 kernel only
  const int grid = std::max(1, std::min(v.grid, kNoAllocMaxGrid));
  const uint64_t arrivals = ((uint64_t)o.max_iter * 7 + 16) * (uint64_t)grid;
  if (arrivals >= (1ull << 32)) return CUP2D_INVALID_ARGUMENT;
  cudaStream_t s = static_cast<cudaStream_t>(stream);

  if (cudaMemsetAsync(base + kOffBar, 0, 256, s) != cudaSuccess ||       // barrier counter starts at 0
      cudaMemsetAsync(base + kOffAbort, 0, 256, s) != cudaSuccess)       // abort flag starts clear
    return CUP2D_CUDA_ERROR;

  double* vec = reinterpret_cast<double*>(base + kOffVec);
  const size_t stride = kVecBytes / sizeof(double);
  SolveArgs64 a{};
  a.prob = Problem64{v.M,
                     d_b,
                     d_x,
                     vec + 0 * stride,  // xo
                     vec + 1 * stride,  // r
                     vec + 2 * stride,  // rh
                     vec + 3 * stride,  // p
                     vec + 4 * stride,  // nu
                     vec + 5 * stride,  // t
                     vec + 6 * stride,  // z
                     vec + 7 * stride,  // z2
                     reinterpret_cast<DevStats*>(base + kOffStats)};
  a.P = v.P;
  a.red = reinterpret_cast<double*>(base + kOffRed);
  a.bar = reinterpret_cast<unsigned*>(base + kOffBar);
  a.abort_flag = reinterpret_cast<int*>(base + kOffAbort);
  a.sp = SolveParams{o.tol_abs, o.tol_rel, 0.0, o.max_restarts, o.max_iter, o.subtract_mean, 0};
  a.timeout_ns = (unsigned long long)o.timeout_ms * 1000000ull;
  a.prof = nullptr;

  if (stats) cudaEventRecord(v.ev0, s);
  const cudaError_t e = launch_bicgstab64(a, grid, s);
  if (e != cudaSuccess) return e == cudaErrorNoDevice ? CUP2D_NO_DEVICE : CUP2D_CUDA_ERROR;
  if (!stats) return CUP2D_OK;
  cudaEventRecord(v.ev1, s);
  DevStats ds;
  int aborted = 0;
  if (cudaMemcpyAsync(&ds, base + kOffStats, sizeof(DevStats), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
      cudaMemcpyAsync(&aborted, base + kOffAbort, sizeof(int), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
      cudaStreamSynchronize(s) != cudaSuccess)
    return CUP2D_CUDA_ERROR;
  float ms = 0.f;
  cudaEventElapsedTime(&ms, v.ev0, v.ev1);
  stats->status = aborted ? CUP2D_TIMEOUT : ds.status;
  stats->iterations = ds.iterations;
  stats->restarts = ds.restarts;
  stats->refinements = 0;
  stats->err_init = ds.err_init;
  stats->err_final = ds.err_opt;
  stats->rel_res_inf = ds.err_init > 0 ? ds.err_opt / ds.err_init : 0.0;
  stats->solve_ms = ms;
  return aborted ? CUP2D_TIMEOUT : CUP2D_OK;
}
