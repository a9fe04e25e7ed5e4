// Status codes, thread-local error text and launch checks shared by every
// translation unit of libopenludwig_b200.so.
#pragma once
#include <cuda_runtime.h>
#include <stdarg.h>
#include <stdio.h>
#include "../../include/openludwig_b200.h"

namespace ol {

int set_error(int code, const char *fmt, ...);
int cuda_status(cudaError_t e, const char *what);

#define OL_CHECK_ARG(cond, ...)                            \
  do {                                                     \
    if (!(cond)) return ::ol::set_error(OL_ERR_ARG, __VA_ARGS__); \
  } while (0)

#define OL_CUDA(call)                                          \
  do {                                                         \
    cudaError_t e_ = (call);                                   \
    if (e_ != cudaSuccess) return ::ol::cuda_status(e_, #call); \
  } while (0)

// After a launch: configuration errors surface here (asynchronous faults
// surface at the next synchronising call).
#define OL_LAUNCHED(name)                                           \
  do {                                                              \
    cudaError_t e_ = cudaGetLastError();                            \
    if (e_ != cudaSuccess) return ::ol::cuda_status(e_, name);      \
  } while (0)

}  // namespace ol
