// Error reporting of the C ABI: a per-thread last-error message.
#include <cstdarg>
#include <cstdio>
#include <mutex>

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

int ensure_smem_raw(const void *fn, size_t bytes, const char *what) {
  struct Entry {
    const void *fn;
    int dev;
    size_t bytes;
  };
  static Entry table[256];
  static int used = 0;
  static std::mutex mu;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) dev = -1;
  std::lock_guard<std::mutex> lock(mu);
  for (int i = 0; i < used; ++i)
    if (table[i].fn == fn && table[i].dev == dev && table[i].bytes >= bytes) return ATB_OK;
  cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
  if (e != cudaSuccess) return fail(ATB_ECUDA, "%s: %s", what, cudaGetErrorString(e));
  for (int i = 0; i < used; ++i)
    if (table[i].fn == fn && table[i].dev == dev) {
      table[i].bytes = bytes;
      return ATB_OK;
    }
  if (used < 256) table[used++] = Entry{fn, dev, bytes};
  return ATB_OK;
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
