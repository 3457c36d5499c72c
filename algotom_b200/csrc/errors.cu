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

int ensure_smem_raw(const void *fn, size_t bytes, const char *what, int threads, int tmem_cols) {
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
  if (tmem_cols > 0) {
    // every CTA that can be resident on an SM must find its TMEM columns
    // free, so that no allocation ever waits
    int per_sm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, threads, bytes);
    if (e != cudaSuccess) return fail(ATB_ECUDA, "%s: %s", what, cudaGetErrorString(e));
    if ((long long)per_sm * tmem_cols > 512)
      return fail(ATB_ECUDA, "%s: %d resident CTAs x %d TMEM columns exceed 512", what, per_sm, tmem_cols);
  }
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

int atb_copy_2d(void *dst, int64_t dst_pitch, const void *src, int64_t src_pitch, int64_t width, int64_t height,
                int kind, void *stream) {
  if (!dst || !src) return atb::fail(ATB_EINVAL, "atb_copy_2d: null pointer");
  if (width < 0 || height < 0 || dst_pitch < width || src_pitch < width)
    return atb::fail(ATB_EINVAL, "atb_copy_2d: bad extent");
  if (width == 0 || height == 0) return ATB_OK;
  cudaMemcpyKind k;
  switch (kind) {
    case 0: k = cudaMemcpyHostToDevice; break;
    case 1: k = cudaMemcpyDeviceToHost; break;
    case 2: k = cudaMemcpyDeviceToDevice; break;
    default: return atb::fail(ATB_EINVAL, "atb_copy_2d: unknown kind %d", kind);
  }
  cudaError_t e = cudaMemcpy2DAsync(dst, (size_t)dst_pitch, src, (size_t)src_pitch, (size_t)width, (size_t)height,
                                    k, atb::as_stream(stream));
  if (e != cudaSuccess) return atb::fail(ATB_ECUDA, "atb_copy_2d: %s", cudaGetErrorString(e));
  return ATB_OK;
}

const char *atb_last_error(void) { return g_last_error; }

}  // extern "C"
