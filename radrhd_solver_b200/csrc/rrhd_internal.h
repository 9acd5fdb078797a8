// Internal helpers shared by the library's translation units.
#pragma once
#include <stdarg.h>
#include <stdint.h>
#include <stdio.h>

#include "rrhd.h"

// Records a message for rrhd_last_error() (thread-local) and returns `st`.
rrhd_status rrhd_fail(rrhd_status st, const char *fmt, ...);

#define RRHD_CHECK_ARG(cond, ...)                        \
  do {                                                   \
    if (!(cond)) return rrhd_fail(RRHD_ERR_INVALID, __VA_ARGS__); \
  } while (0)

#ifdef __CUDACC__
#include <cuda_runtime.h>
// Returns RRHD_ERR_CUDA (or RRHD_ERR_OOM) from the enclosing function when a
// CUDA call fails; the context stays usable for the caller to inspect.
#define RRHD_CUDA(call)                                                              \
  do {                                                                               \
    cudaError_t e_ = (call);                                                         \
    if (e_ != cudaSuccess) {                                                         \
      return rrhd_fail(e_ == cudaErrorMemoryAllocation ? RRHD_ERR_OOM : RRHD_ERR_CUDA, \
                       "%s:%d %s: %s", __FILE__, __LINE__, #call, cudaGetErrorString(e_)); \
    }                                                                                \
  } while (0)
#endif
