// Thread-local error reporting and version of the C ABI.
#include <string.h>
#include "common.cuh"

namespace ol {

static thread_local char g_err[512] = "";

int set_error(int code, const char *fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
  return code;
}

int cuda_status(cudaError_t e, const char *what) {
  return set_error(OL_ERR_CUDA, "%s: %s (%s)", what, cudaGetErrorString(e),
                   cudaGetErrorName(e));
}

}  // namespace ol

extern "C" const char *ol_last_error(void) { return ol::g_err; }
extern "C" const char *ol_version(void) { return "openludwig_b200 0.1 (sm_100a)"; }
