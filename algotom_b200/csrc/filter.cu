// Fused padded ramp-and-window filter of sinogram rows.
//
// Replaces apply_ramp_filter (algotom/rec/reconstruction.py:118-153), whose
// FFT / shift / window / inverse-FFT / real / crop chain is a real circular
// convolution of the padded row of length N = ncol + 2 pad with a periodic
// kernel kappa, cropped to [pad, pad + ncol).  Those ncol outputs only see
// kernel lags in [pad - N + 1, pad + ncol - 1], so the same numbers come out
// of a circular convolution of any length M >= N + ncol - 1 whose kernel b
// holds kappa at those lags (b[u mod M] = kappa[u mod N]) and zero elsewhere.
// The host builds b's spectrum in FP64 for a power-of-two M; this kernel
// then needs nothing but radix-4/2 FFTs of one length.
//
// One CTA filters two rows at once: real rows x1, x2 travel as the complex
// row x1 + i x2 through one forward FFT, a product with the (real-kernel)
// spectrum and one inverse FFT (done as conj(FFT(conj(.))) with 1/M folded
// into the spectrum); the real and imaginary parts of the result are the
// two filtered rows.  Each row is read from HBM once (with the -log folded
// in) and written once; padding, both transforms and the spectral product
// stay in shared memory.
#include <cfloat>

#include "common.cuh"

namespace {

constexpr int kThreads = 512;
constexpr int kMinLog2M = 4;
constexpr int kMaxLog2M = 14;  // 16384 complex = 128 KiB of shared memory
constexpr int kMaxB4 = (1 << kMaxLog2M) / 4 / kThreads;  // radix-4 butterflies per thread
constexpr int kMaxB2 = (1 << kMaxLog2M) / 2 / kThreads;  // radix-2 butterflies per thread

struct FilterArgs {
  const float *src;
  long long srs, sss;  // src row / slice strides (elements)
  int nrow, nslice, ncol, pad, mode, apply_log;
  const float2 *spec;
  int spec_rows;
  const float2 *tw;
  int log2m;
  void *dst;
  long long drs, dss;
  int pair_within_angle;  // 1: a CTA takes slices 2q, 2q+1 of one angle
  int pairs_per_angle;
};

__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }

// In-place forward FFT of length M = 2^log2m in shared memory, Stockham
// ordering (self-sorting: natural order in, natural order out).  Stage with
// sub-transform length Ns and radix R: element j of the M/R butterflies
// reads x[j + r M/R], twiddles input r by w^(r k) (k = j mod Ns,
// w = exp(-2 pi i / (Ns R))), does an R-point DFT and writes output r to
// x[(j - k) R + k + r Ns].  Every thread reads all of its inputs before the
// barrier and writes after it, so one buffer suffices.
__device__ void fft_forward(float2 *x, int log2m, const float2 *__restrict__ tw) {
  const int M = 1 << log2m;
  const int tid = threadIdx.x;
  int logNs = 0;
  if (log2m & 1) {  // one radix-2 stage first (Ns = 1, no twiddles)
    const int H = M >> 1;
    float2 v0[kMaxB2], v1[kMaxB2];
#pragma unroll
    for (int b = 0; b < kMaxB2; ++b) {
      const int j = tid + b * kThreads;
      if (j < H) { v0[b] = x[j]; v1[b] = x[j + H]; }
    }
    __syncthreads();
#pragma unroll
    for (int b = 0; b < kMaxB2; ++b) {
      const int j = tid + b * kThreads;
      if (j < H) { x[2 * j] = cadd(v0[b], v1[b]); x[2 * j + 1] = csub(v0[b], v1[b]); }
    }
    __syncthreads();
    logNs = 1;
  }
  const int Q = M >> 2;
  for (; logNs < log2m; logNs += 2) {
    const int Ns = 1 << logNs;
    const int tshift = log2m - logNs - 2;  // table step M / (4 Ns)
    float2 v[kMaxB4][4];
#pragma unroll
    for (int b = 0; b < kMaxB4; ++b) {
      const int j = tid + b * kThreads;
      if (j < Q) {
#pragma unroll
        for (int r = 0; r < 4; ++r) v[b][r] = x[j + r * Q];
      }
    }
    __syncthreads();
#pragma unroll
    for (int b = 0; b < kMaxB4; ++b) {
      const int j = tid + b * kThreads;
      if (j < Q) {
        const int k = j & (Ns - 1);
        if (k) {
          v[b][1] = cmul(v[b][1], __ldg(&tw[(k) << tshift]));
          v[b][2] = cmul(v[b][2], __ldg(&tw[(2 * k) << tshift]));
          v[b][3] = cmul(v[b][3], __ldg(&tw[(3 * k) << tshift]));
        }
        const float2 a = cadd(v[b][0], v[b][2]), bb = csub(v[b][0], v[b][2]);
        const float2 c = cadd(v[b][1], v[b][3]), d = csub(v[b][1], v[b][3]);
        const int o = ((j - k) << 2) + k;
        x[o] = cadd(a, c);
        x[o + Ns] = make_float2(bb.x + d.y, bb.y - d.x);      // b - i d
        x[o + 2 * Ns] = csub(a, c);
        x[o + 3 * Ns] = make_float2(bb.x - d.y, bb.y + d.x);  // b + i d
      }
    }
    __syncthreads();
  }
}

// Block-wide reduction over kThreads threads (op: 0 sum, 1 max, 2 min).
__device__ float2 block_reduce2(float2 v, int op, float2 *scratch) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    float2 u = make_float2(__shfl_xor_sync(0xffffffffu, v.x, o), __shfl_xor_sync(0xffffffffu, v.y, o));
    if (op == 0) { v.x += u.x; v.y += u.y; }
    else if (op == 1) { v.x = fmaxf(v.x, u.x); v.y = fmaxf(v.y, u.y); }
    else { v.x = fminf(v.x, u.x); v.y = fminf(v.y, u.y); }
  }
  __syncthreads();
  if (lane == 0) scratch[warp] = v;
  __syncthreads();
  if (warp == 0) {
    v = lane < kThreads / 32 ? scratch[lane]
                             : (op == 0 ? make_float2(0.f, 0.f)
                                        : (op == 1 ? make_float2(-FLT_MAX, -FLT_MAX)
                                                   : make_float2(FLT_MAX, FLT_MAX)));
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      float2 u = make_float2(__shfl_xor_sync(0xffffffffu, v.x, o), __shfl_xor_sync(0xffffffffu, v.y, o));
      if (op == 0) { v.x += u.x; v.y += u.y; }
      else if (op == 1) { v.x = fmaxf(v.x, u.x); v.y = fmaxf(v.y, u.y); }
      else { v.x = fminf(v.x, u.x); v.y = fminf(v.y, u.y); }
    }
    if (lane == 0) scratch[0] = v;
  }
  __syncthreads();
  float2 r = scratch[0];
  __syncthreads();
  return r;
}

// Order-preserving map of a float to an unsigned key.
__device__ __forceinline__ unsigned fkey(float f) {
  unsigned u = __float_as_uint(f);
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float fkey_inv(unsigned k) {
  return __uint_as_float((k & 0x80000000u) ? (k & 0x7fffffffu) : ~k);
}

// Order statistic `rank` (0-based) of each of the two rows held in
// x[pad .. pad+ncol) (.x and .y), by bisection on the float keys.
__device__ float2 block_select2(const float2 *x, int pad, int ncol, int rank, float2 *scratch) {
  unsigned lo1 = 0u, hi1 = 0xffffffffu, lo2 = 0u, hi2 = 0xffffffffu;
  for (int it = 0; it < 32; ++it) {
    const unsigned m1 = lo1 + ((hi1 - lo1) >> 1), m2 = lo2 + ((hi2 - lo2) >> 1);
    float c1 = 0.f, c2 = 0.f;
    for (int j = threadIdx.x; j < ncol; j += kThreads) {
      const float2 v = x[pad + j];
      c1 += fkey(v.x) <= m1 ? 1.f : 0.f;
      c2 += fkey(v.y) <= m2 ? 1.f : 0.f;
    }
    const float2 c = block_reduce2(make_float2(c1, c2), 0, scratch);
    if (c.x >= (float)(rank + 1)) hi1 = m1; else lo1 = m1 + 1;
    if (c.y >= (float)(rank + 1)) hi2 = m2; else lo2 = m2 + 1;
  }
  return make_float2(fkey_inv(lo1), fkey_inv(lo2));
}

template <typename OutT>
__global__ void __launch_bounds__(kThreads) filter_rows_kernel(FilterArgs a) {
  extern __shared__ float2 sm[];
  __shared__ float2 scratch[kThreads / 32];
  const int M = 1 << a.log2m;
  const int ncol = a.ncol, pad = a.pad, N = ncol + 2 * pad;
  const int tid = threadIdx.x;

  // the two rows (angle, slice) of this CTA
  int i1, k1, i2, k2;
  bool ok2;
  if (a.pair_within_angle) {
    i1 = blockIdx.x / a.pairs_per_angle;
    k1 = 2 * (blockIdx.x % a.pairs_per_angle);
    i2 = i1;
    k2 = k1 + 1;
    ok2 = k2 < a.nslice;
  } else {
    const long long r1 = 2LL * blockIdx.x, r2 = r1 + 1;
    i1 = (int)(r1 / a.nslice);
    k1 = (int)(r1 % a.nslice);
    i2 = (int)(r2 / a.nslice);
    k2 = (int)(r2 % a.nslice);
    ok2 = r2 < (long long)a.nrow * a.nslice;
  }
  const float *s1 = a.src + i1 * a.srs + k1 * a.sss;
  const float *s2 = a.src + (ok2 ? i2 * a.srs + k2 * a.sss : 0);

  // 1. the two logged rows into the middle of the complex buffer
  for (int j = tid; j < ncol; j += kThreads) {
    float v1 = __ldg(s1 + j);
    float v2 = ok2 ? __ldg(s2 + j) : 0.0f;
    if (a.apply_log) { v1 = atb::neg_log(v1); v2 = ok2 ? atb::neg_log(v2) : 0.0f; }
    sm[pad + j] = make_float2(v1, v2);
  }
  for (int m = N + tid; m < M; m += kThreads) sm[m] = make_float2(0.f, 0.f);
  __syncthreads();

  // 2. padding (numpy.pad semantics along the row)
  if (pad > 0) {
    float2 stat = make_float2(0.f, 0.f);
    if (a.mode == ATB_PAD_MEAN || a.mode == ATB_PAD_MAXIMUM || a.mode == ATB_PAD_MINIMUM) {
      const int op = a.mode == ATB_PAD_MEAN ? 0 : (a.mode == ATB_PAD_MAXIMUM ? 1 : 2);
      float2 acc = op == 0 ? make_float2(0.f, 0.f)
                           : (op == 1 ? make_float2(-FLT_MAX, -FLT_MAX) : make_float2(FLT_MAX, FLT_MAX));
      for (int j = tid; j < ncol; j += kThreads) {
        const float2 v = sm[pad + j];
        if (op == 0) { acc.x += v.x; acc.y += v.y; }
        else if (op == 1) { acc.x = fmaxf(acc.x, v.x); acc.y = fmaxf(acc.y, v.y); }
        else { acc.x = fminf(acc.x, v.x); acc.y = fminf(acc.y, v.y); }
      }
      stat = block_reduce2(acc, op, scratch);
      if (op == 0) { stat.x /= (float)ncol; stat.y /= (float)ncol; }
    } else if (a.mode == ATB_PAD_MEDIAN) {
      const float2 lo = block_select2(sm, pad, ncol, (ncol - 1) / 2, scratch);
      if (ncol & 1) {
        stat = lo;
      } else {
        const float2 hi = block_select2(sm, pad, ncol, ncol / 2, scratch);
        stat = make_float2(0.5f * (lo.x + hi.x), 0.5f * (lo.y + hi.y));
      }
    }
    for (int t = tid; t < 2 * pad; t += kThreads) {
      const bool left = t < pad;
      const int m = left ? t : ncol + t;   // position in the padded row
      const int q = m - pad;               // position relative to the row
      float2 v;
      switch (a.mode) {
        case ATB_PAD_EDGE: v = sm[pad + (left ? 0 : ncol - 1)]; break;
        case ATB_PAD_CONSTANT: v = make_float2(0.f, 0.f); break;
        case ATB_PAD_WRAP: v = sm[pad + ((q % ncol) + ncol) % ncol]; break;
        case ATB_PAD_REFLECT: {
          int r = 0;
          if (ncol > 1) {
            const int P = 2 * (ncol - 1);
            r = ((q % P) + P) % P;
            if (r >= ncol) r = P - r;
          }
          v = sm[pad + r];
          break;
        }
        case ATB_PAD_SYMMETRIC: {
          const int P = 2 * ncol;
          int r = ((q % P) + P) % P;
          if (r >= ncol) r = P - 1 - r;
          v = sm[pad + r];
          break;
        }
        case ATB_PAD_LINEAR_RAMP: {
          // numpy: linspace(end=0, edge, pad, endpoint=False) on each side
          const float2 e = sm[pad + (left ? 0 : ncol - 1)];
          const float f = left ? (float)m / (float)pad : (float)(pad - 1 - (q - ncol)) / (float)pad;
          v = make_float2(e.x * f, e.y * f);
          break;
        }
        default: v = stat; break;  // mean / maximum / minimum / median
      }
      sm[m] = v;
    }
  }
  __syncthreads();

  // 3. forward transform, spectral product (conjugated), second forward
  //    transform = conjugated inverse
  fft_forward(sm, a.log2m, a.tw);
  const float2 *spec = a.spec + (a.spec_rows > 1 ? (long long)i1 * M : 0LL);
  for (int k = tid; k < M; k += kThreads) {
    const float2 y = cmul(sm[k], __ldg(spec + k));
    sm[k] = make_float2(y.x, -y.y);
  }
  __syncthreads();
  fft_forward(sm, a.log2m, a.tw);

  // 4. crop: real part -> row 1, -imag part -> row 2
  OutT *d1 = reinterpret_cast<OutT *>(a.dst) + i1 * a.drs + k1 * a.dss;
  OutT *d2 = reinterpret_cast<OutT *>(a.dst) + (ok2 ? i2 * a.drs + k2 * a.dss : 0);
  for (int j = tid; j < ncol; j += kThreads) {
    const float2 w = sm[pad + j];
    atb::store_from_float(d1 + j, w.x);
    if (ok2) atb::store_from_float(d2 + j, -w.y);
  }
}

__global__ void neg_log_kernel(const float *__restrict__ src, long long srs, long long sss, int nrow,
                               int nslice, int ncol, float *dst, long long drs, long long dss) {
  const long long total = (long long)nrow * nslice * ncol;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    const int j = (int)(t % ncol);
    const long long rk = t / ncol;
    const int k = (int)(rk % nslice), i = (int)(rk / nslice);
    dst[i * drs + k * dss + j] = atb::neg_log(__ldg(src + i * srs + k * sss + j));
  }
}

template <typename OutT>
int launch_filter(const FilterArgs &a, long long npairs, cudaStream_t st) {
  const size_t smem = sizeof(float2) << a.log2m;
  cudaError_t e = cudaFuncSetAttribute(filter_rows_kernel<OutT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)smem);
  if (e != cudaSuccess) return atb::fail(ATB_ECUDA, "atb_filter_rows: %s", cudaGetErrorString(e));
  filter_rows_kernel<OutT><<<(unsigned)npairs, kThreads, smem, st>>>(a);
  return atb::check_launch("atb_filter_rows");
}

}  // namespace

extern "C" {

int atb_filter_log2m(int ncol, int pad) {
  if (ncol < 1 || pad < 0) return atb::fail(ATB_EINVAL, "atb_filter_log2m: ncol=%d pad=%d", ncol, pad);
  const long long need = (long long)ncol + 2LL * pad + ncol - 1;
  int l = kMinLog2M;
  while ((1LL << l) < need) ++l;
  if (l > kMaxLog2M)
    return atb::fail(ATB_ERANGE, "atb_filter_log2m: ncol=%d pad=%d needs FFT length 2^%d > 2^%d", ncol, pad, l,
                     kMaxLog2M);
  return l;
}

int atb_filter_rows(const float *src, int64_t src_row_stride, int64_t src_slice_stride, int nrow, int nslice,
                    int ncol, int pad, int pad_mode, int apply_log, const void *spec, int spec_rows,
                    const void *twiddle, int log2m, void *dst, int dst_dtype, int64_t dst_row_stride,
                    int64_t dst_slice_stride, void *stream) {
  if (!src || !dst || !spec || !twiddle) return atb::fail(ATB_EINVAL, "atb_filter_rows: null pointer");
  if (nrow < 1 || nslice < 1 || ncol < 1 || pad < 0)
    return atb::fail(ATB_EINVAL, "atb_filter_rows: bad shape nrow=%d nslice=%d ncol=%d pad=%d", nrow, nslice,
                     ncol, pad);
  if (pad_mode < ATB_PAD_EDGE || pad_mode > ATB_PAD_MEDIAN)
    return atb::fail(ATB_EINVAL, "atb_filter_rows: unknown pad_mode %d", pad_mode);
  if (log2m < kMinLog2M || log2m > kMaxLog2M)
    return atb::fail(ATB_ERANGE, "atb_filter_rows: log2m=%d outside [%d, %d]", log2m, kMinLog2M, kMaxLog2M);
  if ((1LL << log2m) < (long long)ncol + 2LL * pad + ncol - 1)
    return atb::fail(ATB_EINVAL, "atb_filter_rows: 2^%d < ncol + 2 pad + ncol - 1", log2m);
  if (spec_rows != 1 && spec_rows != nrow)
    return atb::fail(ATB_EINVAL, "atb_filter_rows: spec_rows=%d must be 1 or nrow=%d", spec_rows, nrow);
  FilterArgs a;
  a.src = src; a.srs = src_row_stride; a.sss = src_slice_stride;
  a.nrow = nrow; a.nslice = nslice; a.ncol = ncol; a.pad = pad; a.mode = pad_mode; a.apply_log = apply_log;
  a.spec = reinterpret_cast<const float2 *>(spec); a.spec_rows = spec_rows;
  a.tw = reinterpret_cast<const float2 *>(twiddle); a.log2m = log2m;
  a.dst = dst; a.drs = dst_row_stride; a.dss = dst_slice_stride;
  long long npairs;
  if (spec_rows > 1) {
    a.pair_within_angle = 1;
    a.pairs_per_angle = (nslice + 1) / 2;
    npairs = (long long)nrow * a.pairs_per_angle;
  } else {
    a.pair_within_angle = 0;
    a.pairs_per_angle = 0;
    npairs = ((long long)nrow * nslice + 1) / 2;
  }
  if (npairs > 0x7fffffffLL) return atb::fail(ATB_ERANGE, "atb_filter_rows: too many rows");
  cudaStream_t st = atb::as_stream(stream);
  switch (dst_dtype) {
    case ATB_F32: return launch_filter<float>(a, npairs, st);
    case ATB_F16: return launch_filter<__half>(a, npairs, st);
    case ATB_BF16: return launch_filter<__nv_bfloat16>(a, npairs, st);
    default: return atb::fail(ATB_EINVAL, "atb_filter_rows: unknown dst_dtype %d", dst_dtype);
  }
}

int atb_neg_log(const float *src, int64_t src_row_stride, int64_t src_slice_stride, int nrow, int nslice, int ncol,
                float *dst, int64_t dst_row_stride, int64_t dst_slice_stride, void *stream) {
  if (!src || !dst) return atb::fail(ATB_EINVAL, "atb_neg_log: null pointer");
  if (nrow < 1 || nslice < 1 || ncol < 1) return atb::fail(ATB_EINVAL, "atb_neg_log: bad shape");
  const long long total = (long long)nrow * nslice * ncol;
  long long blocks = (total + 255) / 256;
  if (blocks > 148LL * 32) blocks = 148LL * 32;
  neg_log_kernel<<<(unsigned)blocks, 256, 0, atb::as_stream(stream)>>>(
      src, src_row_stride, src_slice_stride, nrow, nslice, ncol, dst, dst_row_stride, dst_slice_stride);
  return atb::check_launch("atb_neg_log");
}

}  // extern "C"
