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

}  // namespace cup2d
