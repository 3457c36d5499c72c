// Error reporting of the C ABI: a per-thread last-error message.
#include <cstdarg>
#include <cstdio>

#include "common.cuh"

namespace {
thread_local char g_last_error[512] = "";
}

namespace atb {

int fail(int code, const char *fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_last_error, sizeof(g_last_error), fmt, ap);
  va_end(ap);
  return code;
}

int check_launch(const char *what) {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return fail(ATB_ECUDA, "%s: %s", what, cudaGetErrorString(e));
  return ATB_OK;
}

}  // namespace atb

extern "C" {

int atb_version(void) { return 100; }

const char *atb_last_error(void) { return g_last_error; }

}  // extern "C"
