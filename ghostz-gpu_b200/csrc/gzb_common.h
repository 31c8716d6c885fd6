// gzb_common.h -- host-side error reporting shared by the C-ABI units.
#pragma once

#include <cuda_runtime.h>

#include <cstdarg>
#include <cstdio>
#include <string>

#include "ghostz_b200.h"

namespace gzb {

// Records the message of the latest failure on this thread and returns code.
int set_error(int code, const char *fmt, ...);

inline int cuda_error(cudaError_t e, const char *what, const char *file,
                      int line) {
  return set_error(e == cudaErrorMemoryAllocation ? GZB_ERR_NOMEM : GZB_ERR_CUDA,
                   "%s failed at %s:%d: %s", what, file, line,
                   cudaGetErrorString(e));
}

}  // namespace gzb

// Returns from the enclosing function with an error code when a CUDA call
// fails (no exit(), unlike the reference's CUDA_CHECK_RETURN,
// src/cuda_common.h:13-19).
#define GZB_CUDA(call)                                                   \
  do {                                                                   \
    cudaError_t e_ = (call);                                             \
    if (e_ != cudaSuccess) return gzb::cuda_error(e_, #call, __FILE__, __LINE__); \
  } while (0)

#define GZB_CHECK(cond, code, ...)                                       \
  do {                                                                   \
    if (!(cond)) return gzb::set_error((code), __VA_ARGS__);             \
  } while (0)

#define GZB_TRY(call)                                                    \
  do {                                                                   \
    int r_ = (call);                                                     \
    if (r_ != GZB_OK) return r_;                                         \
  } while (0)
