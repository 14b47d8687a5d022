// Read-only view of a solver handle's device operator, for entry points
// that live outside capi.cu.
#pragma once
#include <cuda_runtime.h>

#include <vector>

#include "../../include/cup2d_poisson.h"
#include "kernels.hpp"

namespace cup2d {

struct HandleView {
  int device;                              // the handle's CUDA device
  MeshView M;                              // assembled operator (device)
  const double* P;                         // FP64 P^-1 (device)
  int64_t nb;                              // blocks
  int grid;                                // CTAs the FP64 solve would use
  cup2d_solve_opts opts;
  cudaEvent_t ev0, ev1;                    // the handle's timing events
};

int handle_view(const cup2d_poisson* h, HandleView* out);

// cup2d_poisson_create on the caller's stream: the handle assembles and runs
// its host-buffer work there and owns no stream (the stream must outlive the
// handle); its timing events are made on first use.  `served`: its solves
// run the server's kernel instances (kServedCtasPerSm).
int handle_create(const cup2d_forest* forest, const cup2d_solve_opts* opts, cudaStream_t stream, bool served,
                  cup2d_poisson** out);

// For the request server (server.cpp).
// Device bytes a handle holds (operator, vectors, scratch).
int64_t handle_bytes(const cup2d_poisson* h);
// Device copies of the right-hand side and solution owned by the handle
// (the host-buffer solve stages through them; they persist between solves).
int handle_stage(cup2d_poisson* h, double** d_b, double** d_x);
// Launches the handle's solve on `stream` without waiting and queues the
// copy of its device statistics and abort flag to the pinned `raw` (at
// least handle_stats_bytes() bytes).
int handle_solve_async(cup2d_poisson* h, const double* d_b, double* d_x, cudaStream_t stream, void* raw);
size_t handle_stats_bytes();
// Destroys a handle none of whose work is pending on any stream (the
// public cup2d_poisson_destroy first waits for the whole device).
int handle_destroy_idle(cup2d_poisson* h);
// Statistics from a `raw` record filled by handle_solve_async.
void handle_stats_from_raw(const void* raw, double solve_ms, cup2d_solve_stats* out);
// Looks up (once per device, with that device current) the address of the
// static scratch array of cup2d_poisson_solve_device_noalloc, which commits
// the array on that device (noalloc.cu).
int noalloc_prepare(int device);

}  // namespace cup2d
