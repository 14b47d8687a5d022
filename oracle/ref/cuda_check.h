// ORACLE — test infrastructure only.  Force-included (-include) into the
// reference's Poisson sources when oracle/ref/build.py compiles them.  CUP2D's
// sources take their CUDA error check from source/include/helper_cuda.h
// (through source/Utils/DeviceProfiler.cuh:12); that header is not used here.
// Defining its include guard first makes the #include a no-op, and this file
// supplies the one name the Poisson path uses from it, checkCudaErrors, as an
// error check of our own: a failed CUDA, cuBLAS or cuSPARSE call throws
// std::runtime_error naming the call, which the checker's C entry points turn
// into an error code (the reference prints and exits instead).
#pragma once
#define COMMON_HELPER_CUDA_H_

#include <cublas_v2.h>
#include <cuda_runtime.h>
#include <cusparse.h>

#include <stdexcept>
#include <string>

namespace cup2d_ref_check {

inline void fail(const char* what, const char* file, int line, int code) {
  throw std::runtime_error(std::string(file) + ":" + std::to_string(line) + ": " + what + " failed (" +
                           std::to_string(code) + ")");
}
inline void check(cudaError_t e, const char* what, const char* file, int line) {
  if (e != cudaSuccess) fail(what, file, line, (int)e);
}
inline void check(cublasStatus_t e, const char* what, const char* file, int line) {
  if (e != CUBLAS_STATUS_SUCCESS) fail(what, file, line, (int)e);
}
inline void check(cusparseStatus_t e, const char* what, const char* file, int line) {
  if (e != CUSPARSE_STATUS_SUCCESS) fail(what, file, line, (int)e);
}

}  // namespace cup2d_ref_check

#define checkCudaErrors(call) cup2d_ref_check::check((call), #call, __FILE__, __LINE__)
