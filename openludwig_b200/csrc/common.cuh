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

// Programmatic dependent launch.  A kernel launched with launch_pdl has its
// launch processed while the previous kernel on its stream is still running,
// so it starts as soon as that one completes.  Every CTA of it calls
// pdl_wait() (griddepcontrol.wait: the previous grid has completed and its
// memory is visible) before it reads or writes memory that an earlier launch
// writes, and before it can exit, so that its own completion still implies
// the completion of everything before it.  (Letting the next launch start
// even earlier, with griddepcontrol.launch_dependents at the top of each
// kernel, measured 0.9 % slower per coarse step.)
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

template <class... KArgs, class... Args>
inline cudaError_t launch_pdl(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem,
                              cudaStream_t s, Args... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kernel, static_cast<KArgs>(args)...);
}

}  // namespace ol
