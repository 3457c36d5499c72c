// Shared helpers of the algotom_b200 CUDA library (sm_100a only).
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/algotom_b200.h"

namespace atb {

// Records a printf-style message as the calling thread's last error and
// returns `code`.
int fail(int code, const char *fmt, ...);

// Checks the launch that just happened on this thread; ATB_ECUDA on error.
int check_launch(const char *what);

inline cudaStream_t as_stream(void *s) { return reinterpret_cast<cudaStream_t>(s); }

// Raises a kernel's dynamic shared-memory limit once per (kernel, device),
// so that launches made while a stream is being captured into a CUDA graph
// issue no configuration calls.  For a kernel whose CTAs of `threads`
// threads each allocate `tmem_cols` TMEM columns, it also checks once that
// all CTAs an SM can hold fit in its 512 columns.  Thread-safe.  Returns 0
// or ATB_ECUDA.
int ensure_smem_raw(const void *fn, size_t bytes, const char *what, int threads = 0, int tmem_cols = 0);
template <typename F>
int ensure_smem(F *fn, size_t bytes, const char *what, int threads = 0, int tmem_cols = 0) {
  return ensure_smem_raw(reinterpret_cast<const void *>(fn), bytes, what, threads, tmem_cols);
}

__device__ __forceinline__ float load_as_float(const float *p) { return __ldg(p); }
__device__ __forceinline__ float load_as_float(const __half *p) { return __half2float(__ldg(p)); }
__device__ __forceinline__ float load_as_float(const __nv_bfloat16 *p) {
  return __bfloat162float(__ldg(p));
}

__device__ __forceinline__ float to_float(float v) { return v; }
__device__ __forceinline__ float to_float(__half v) { return __half2float(v); }
__device__ __forceinline__ float to_float(__nv_bfloat16 v) { return __bfloat162float(v); }
__device__ __forceinline__ float to_float(unsigned short v) { return (float)v; }

// two floats as one 32-bit word of two 16-bit values (first in the low half)
template <typename T> __device__ __forceinline__ unsigned pack_pair(float lo, float hi);
template <> __device__ __forceinline__ unsigned pack_pair<__half>(float lo, float hi) {
  const __half2 h = __floats2half2_rn(lo, hi);
  return *reinterpret_cast<const unsigned *>(&h);
}
template <> __device__ __forceinline__ unsigned pack_pair<__nv_bfloat16>(float lo, float hi) {
  const __nv_bfloat162 h = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<const unsigned *>(&h);
}
// and back: bfloat16 widens by a shift, float16 by conversion
template <typename T> __device__ __forceinline__ void unpack_pair(unsigned w, float &lo, float &hi);
template <> __device__ __forceinline__ void unpack_pair<__half>(unsigned w, float &lo, float &hi) {
  const float2 f = __half22float2(*reinterpret_cast<const __half2 *>(&w));
  lo = f.x;
  hi = f.y;
}
template <> __device__ __forceinline__ void unpack_pair<__nv_bfloat16>(unsigned w, float &lo, float &hi) {
  lo = __uint_as_float(w << 16);
  hi = __uint_as_float(w & 0xffff0000u);
}

__device__ __forceinline__ void store_from_float(float *p, float v) { *p = v; }
__device__ __forceinline__ void store_from_float(__half *p, float v) { *p = __float2half_rn(v); }
__device__ __forceinline__ void store_from_float(__nv_bfloat16 *p, float v) {
  *p = __float2bfloat16_rn(v);
}

// -log of a transmission value; values <= 0 read as 1 (give 0), as the
// reference replaces them before taking the logarithm
// (algotom/rec/reconstruction.py:431-436).  NaN stays NaN.
__device__ __forceinline__ float neg_log(float v) { return v <= 0.0f ? 0.0f : -logf(v); }

}  // namespace atb
