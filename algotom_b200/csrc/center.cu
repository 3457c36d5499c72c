// Centre search by slice metrics, sm_100a: the sinogram pre-steps and the
// per-image metrics of algotom's find_center_based_slice_metric
// (algotom/rec/reconstruction.py:1212-1458).  The reconstructions at the
// candidate centres are one persistent batched back-projection
// (backproject.cu); this file holds what surrounds it.
//
// - atb_gaussian_rows: scipy.ndimage.gaussian_filter1d(x, sigma, axis=1)
//   (reconstruction.py:1318).  The symmetric correlation is evaluated as
//   x[i] w0 + sum_j (x[i+j] + x[i-j]) w_j, left to right in FP64 with
//   explicitly rounded operations (no contraction), half-sample symmetric
//   extension, then rounded to float32: the same operations in the same
//   order as scipy's correlate1d, hence the same float32 results.  For an
//   integer input array scipy stores each pass truncated toward zero; the
//   to_int flag does the same, on the same FP64 sums.
// - atb_gaussian_cols: the same filter down the columns of a batch of
//   images (gaussian_filter1d along axis 1 of a [n, rows, cols] stack; the
//   first pass of gaussian_filter(projections, (0, sigma, sigma)) in
//   vertrec.py:1349), each CTA staging a 32-column strip of rows plus the
//   halo in shared memory.
// - atb_zoom_linear: scipy.ndimage.zoom(x, z, order=1, mode="nearest")
//   (reconstruction.py:1427): sample k of an axis sits at input coordinate
//   k (n-1)/(m-1), clamped to [0, n-1]; the four bilinear taps are summed in
//   scipy's order, ((x w_r) w_c), in FP64, then rounded to float32.
// - atb_image_range: min and max of an image (the entropy normalisation
//   range, reconstruction.py:1327-1330); NaN anywhere gives NaN, as NumPy.
// - atb_slice_metric: per image of a batch, the histogram entropy
//   (reconstruction.py:1212-1221 after the normalisation of :1243-1245) or
//   the edge sharpness (:1224-1229).  Both reductions are deterministic:
//   integer histogram counts, and FP64 partial sums reduced in a fixed order.
//   atb_slice_entropy64 is the entropy of float64 images, normalised in FP64
//   (the vertical-slice search, vertrec.py:1389-1392).
#include <cmath>

#include "common.cuh"

namespace {

constexpr int kRowTile = 256;        // output samples per CTA (Gaussian)
constexpr int kColTile = 32;         // columns per CTA (Gaussian, columns)
constexpr int kColRows = 64;         // output rows per CTA (Gaussian, columns)
constexpr int kColThreads = 256;
constexpr int kMaxColRadius = 700;   // strip + halo: <= 190 KB of shared memory
constexpr int kColRadius64 = 300;    // FP64 strip + halo: <= 172 KB
constexpr int kMaxGaussRadius = 8192;
constexpr int kMetricThreads = 256;
constexpr int kMetricBlocks = 256;   // partial sums per image (sharpness)
static_assert(kMetricThreads == 256, "one thread per histogram bin");

// a filtered sample as stored: float32, or (to_int) truncated toward zero
// as scipy stores a filter's output for an integer input array
__device__ __forceinline__ float gauss_out(double v, int to_int) {
  return to_int ? (float)trunc(v) : __double2float_rn(v);
}

__device__ __forceinline__ int reflect_index(long long i, int n) {
  if (i >= 0 && i < n) return (int)i;  // inside: no 64-bit remainder
  const long long period = 2LL * n;
  long long r = i % period;
  if (r < 0) r += period;
  return (int)(r >= n ? period - 1 - r : r);
}

// Row pass: CTA (row, tile) filters 256 samples of one row.  The strip and
// its halo are staged once as FP64 (the conversion is exact), so the taps
// read doubles from shared memory.
__global__ void __launch_bounds__(kRowTile) gaussian_rows_kernel(const float *__restrict__ src, long long srs,
                                                                 int ncol, const double *__restrict__ w, int radius,
                                                                 float *__restrict__ dst, long long drs,
                                                                 int to_int) {
  extern __shared__ __align__(16) unsigned char smem[];
  double *ws = reinterpret_cast<double *>(smem);  // [radius + 1]
  double *xs = ws + radius + 1;                   // [kRowTile + 2 radius]
  const long long row = blockIdx.x;
  const int c0 = blockIdx.y * kRowTile;
  const float *x = src + row * srs;
  for (int j = threadIdx.x; j <= radius; j += kRowTile) ws[j] = w[j];
  const int span = kRowTile + 2 * radius;
  for (int j = threadIdx.x; j < span; j += kRowTile)
    xs[j] = (double)x[reflect_index((long long)c0 - radius + j, ncol)];
  __syncthreads();
  const int c = c0 + threadIdx.x;
  if (c >= ncol) return;
  const double *xc = xs + radius + threadIdx.x;
  double acc = __dmul_rn(xc[0], ws[0]);
  for (int j = 1; j <= radius; ++j) acc = __dadd_rn(acc, __dmul_rn(__dadd_rn(xc[j], xc[-j]), ws[j]));
  dst[row * drs + c] = gauss_out(acc, to_int);
}

// Column pass: CTA (x, y, z) filters columns [32 x, 32 x + 32) of rows
// [64 y, 64 y + 64) of image z; threads (lane = column, warp = row phase)
// read the strip with its halo row by row (coalesced) into shared memory
// as S (FP64 for radii up to kColRadius64: converted once, not per tap),
// then each output takes the symmetric sum down its column.
template <typename S>
__global__ void __launch_bounds__(kColThreads)
    gaussian_cols_kernel(const float *__restrict__ src, long long sis, long long srs, int nrow, int ncol,
                         const double *__restrict__ w, int radius, float *__restrict__ dst, long long dis,
                         long long drs, int to_int) {
  extern __shared__ __align__(16) unsigned char smem[];
  double *ws = reinterpret_cast<double *>(smem);   // [radius + 1]
  S *xs = reinterpret_cast<S *>(ws + radius + 1);  // [kColRows + 2 radius][kColTile]
  const int lane = threadIdx.x & 31, wy = threadIdx.x >> 5;
  const int c = blockIdx.x * kColTile + lane;
  const int r0 = blockIdx.y * kColRows;
  const float *img = src + blockIdx.z * sis;
  for (int j = threadIdx.x; j <= radius; j += kColThreads) ws[j] = w[j];
  const int span = kColRows + 2 * radius;
  for (int j = wy; j < span; j += kColThreads / 32)
    xs[j * kColTile + lane] = c < ncol ? (S)img[reflect_index((long long)r0 - radius + j, nrow) * srs + c] : (S)0;
  __syncthreads();
  if (c >= ncol) return;
  float *out = dst + blockIdx.z * dis;
  for (int k = wy; k < kColRows; k += kColThreads / 32) {
    const int r = r0 + k;
    if (r >= nrow) break;
    const S *xc = xs + (radius + k) * kColTile + lane;
    double acc = __dmul_rn((double)xc[0], ws[0]);
    for (int j = 1; j <= radius; ++j)
      acc = __dadd_rn(acc, __dmul_rn(__dadd_rn((double)xc[j * kColTile], (double)xc[-j * kColTile]), ws[j]));
    out[r * drs + c] = gauss_out(acc, to_int);
  }
}

// Register-window forms for radii up to KR (4, 8, 12 or 16; sigma <= 3.9):
// the strip is staged as float32 by asynchronous copies (all in flight at
// once), and each thread computes kWinOut consecutive outputs of one line
// from a window of kWinOut + 2 radius samples widened to FP64 in registers,
// so a sample is read from shared memory once per thread instead of once
// per tap (the forms above read 2 radius + 1 samples per output and are
// bound by shared memory).  Same operations in the same order as above:
// bit-identical.
constexpr int kWinOut = 8;     // outputs per thread
constexpr int kLineTile = 32;  // lines per CTA (one per lane)
constexpr int kSegs = 8;       // warps per CTA, each kWinOut outputs per line

__device__ __forceinline__ void cp_async4(void *smem, const void *gmem) {
  const unsigned a = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(a), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.commit_group;\n\tcp.async.wait_all;" ::: "memory");
}

template <int KR>
__device__ __forceinline__ void window_filter(const float *xs, int stride, const double *ws, int radius,
                                              double (&acc)[kWinOut]) {
  // xs points at the staged sample of this thread's first output minus
  // `radius` (window element m sits at xs[(m - KR + radius) * stride]);
  // each sample is widened to FP64 once (exact)
  double win[kWinOut + 2 * KR];
#pragma unroll
  for (int m = 0; m < kWinOut + 2 * KR; ++m)
    win[m] = (m >= KR - radius && m < kWinOut + KR + radius) ? (double)xs[(m - KR + radius) * stride] : 0.0;
#pragma unroll
  for (int i = 0; i < kWinOut; ++i) acc[i] = __dmul_rn(win[KR + i], ws[0]);
#pragma unroll
  for (int j = 1; j <= KR; ++j) {
    if (j <= radius) {
      const double wj = ws[j];
#pragma unroll
      for (int i = 0; i < kWinOut; ++i)
        acc[i] = __dadd_rn(acc[i], __dmul_rn(__dadd_rn(win[KR + i + j], win[KR + i - j]), wj));
    }
  }
}

// rows: CTA = 32 rows (lane) x 64 columns (8 warps x 8); the tile plus halo
// is staged row-major with an odd pitch (conflict-free per-lane rows), the
// results go through shared memory for coalesced stores
template <int KR>
__global__ void __launch_bounds__(kLineTile * kSegs, KR <= 4 ? 4 : (KR <= 12 ? 3 : 2)) gaussian_rows_win_kernel(
    const float *__restrict__ src, long long srs, long long nrow, int ncol, const double *__restrict__ w,
    int radius, float *__restrict__ dst, long long drs, int to_int) {
  constexpr int kCols = kSegs * kWinOut;  // 64
  extern __shared__ __align__(16) unsigned char smem[];
  double *ws = reinterpret_cast<double *>(smem);  // [radius + 1]
  const int span = kCols + 2 * radius, pitch = span | 1;
  float *xs = reinterpret_cast<float *>(ws + radius + 1);  // [32][pitch]
  float *ot = xs + kLineTile * pitch;                       // [32][kCols + 1]
  const int tid = threadIdx.x, lane = tid & 31, seg = tid >> 5;
  const long long row0 = (long long)blockIdx.x * kLineTile;
  const int c0 = blockIdx.y * kCols;
  for (int j = tid; j <= radius; j += kLineTile * kSegs) ws[j] = w[j];
  // the whole strip in flight at once: one asynchronous copy per sample
  for (int e = tid; e < kLineTile * span; e += kLineTile * kSegs) {
    const int rr = e / span, cc = e - rr * span;
    const long long row = row0 + rr;
    if (row < nrow)
      cp_async4(xs + rr * pitch + cc, src + row * srs + reflect_index((long long)c0 - radius + cc, ncol));
    else
      xs[rr * pitch + cc] = 0.0f;
  }
  cp_async_wait_all();
  __syncthreads();
  double acc[kWinOut];
  window_filter<KR>(xs + lane * pitch + seg * kWinOut, 1, ws, radius, acc);
#pragma unroll
  for (int i = 0; i < kWinOut; ++i) ot[lane * (kCols + 1) + seg * kWinOut + i] = gauss_out(acc[i], to_int);
  __syncthreads();
  for (int e = tid; e < kLineTile * kCols; e += kLineTile * kSegs) {
    const int rr = e / kCols, cc = e - rr * kCols;
    const long long row = row0 + rr;
    if (row < nrow && c0 + cc < ncol) dst[row * drs + c0 + cc] = ot[rr * (kCols + 1) + cc];
  }
}

// columns: CTA = 32 columns (lane) x 64 rows (8 warps x 8) of one image;
// the strip plus halo is staged as in gaussian_cols_kernel
template <int KR>
__global__ void __launch_bounds__(kLineTile * kSegs, KR <= 4 ? 4 : (KR <= 12 ? 3 : 2)) gaussian_cols_win_kernel(
    const float *__restrict__ src, long long sis, long long srs, int nrow, int ncol, const double *__restrict__ w,
    int radius, float *__restrict__ dst, long long dis, long long drs, int to_int) {
  constexpr int kRowsT = kSegs * kWinOut;  // 64
  extern __shared__ __align__(16) unsigned char smem[];
  double *ws = reinterpret_cast<double *>(smem);  // [radius + 1]
  float *xs = reinterpret_cast<float *>(ws + radius + 1);  // [kRowsT + 2 radius][32]
  const int tid = threadIdx.x, lane = tid & 31, seg = tid >> 5;
  const int c = blockIdx.x * kLineTile + lane;
  const int r0 = blockIdx.y * kRowsT;
  const float *img = src + blockIdx.z * sis;
  for (int j = tid; j <= radius; j += kLineTile * kSegs) ws[j] = w[j];
  const int span = kRowsT + 2 * radius;
  for (int j = seg; j < span; j += kSegs) {
    if (c < ncol)
      cp_async4(xs + j * kLineTile + lane, img + reflect_index((long long)r0 - radius + j, nrow) * srs + c);
    else
      xs[j * kLineTile + lane] = 0.0f;
  }
  cp_async_wait_all();
  __syncthreads();
  const int k0 = seg * kWinOut;
  if (c >= ncol || r0 + k0 >= nrow) return;
  double acc[kWinOut];
  window_filter<KR>(xs + k0 * kLineTile + lane, kLineTile, ws, radius, acc);
  float *out = dst + blockIdx.z * dis;
#pragma unroll
  for (int i = 0; i < kWinOut; ++i)
    if (r0 + k0 + i < nrow) out[(long long)(r0 + k0 + i) * drs + c] = gauss_out(acc[i], to_int);
}

struct ZoomAxis {
  int i0, i1;
  double w0, w1;
};

__device__ __forceinline__ ZoomAxis zoom_axis(int k, int n_in, int n_out) {
  const double step = n_out > 1 ? __ddiv_rn((double)(n_in - 1), (double)(n_out - 1)) : 1.0;
  double c = __dmul_rn((double)k, step);
  if (c < 0.0) c = 0.0;
  if (c > (double)(n_in - 1)) c = (double)(n_in - 1);
  ZoomAxis a;
  a.i0 = (int)floor(c);
  const double t = __dsub_rn(c, (double)a.i0);
  a.i1 = min(a.i0 + 1, n_in - 1);
  a.w0 = __dsub_rn(1.0, t);
  a.w1 = t;
  return a;
}

__global__ void zoom_linear_kernel(const float *__restrict__ src, long long srs, int in_rows, int in_cols,
                                   float *__restrict__ dst, long long drs, int out_rows, int out_cols) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  const int r = blockIdx.y;
  if (c >= out_cols || r >= out_rows) return;
  const ZoomAxis ar = zoom_axis(r, in_rows, out_rows);
  const ZoomAxis ac = zoom_axis(c, in_cols, out_cols);
  const float *p0 = src + (long long)ar.i0 * srs, *p1 = src + (long long)ar.i1 * srs;
  double t = __dmul_rn(__dmul_rn((double)p0[ac.i0], ar.w0), ac.w0);
  t = __dadd_rn(t, __dmul_rn(__dmul_rn((double)p0[ac.i1], ar.w0), ac.w1));
  t = __dadd_rn(t, __dmul_rn(__dmul_rn((double)p1[ac.i0], ar.w1), ac.w0));
  t = __dadd_rn(t, __dmul_rn(__dmul_rn((double)p1[ac.i1], ar.w1), ac.w1));
  dst[(long long)r * drs + c] = __double2float_rn(t);
}

// order-preserving 32-bit keys of floats (NaN is flagged separately)
__device__ __forceinline__ unsigned float_key(float f) {
  const unsigned u = __float_as_uint(f);
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float key_float(unsigned k) {
  return __uint_as_float((k & 0x80000000u) ? (k & 0x7fffffffu) : ~k);
}

// work[0] = min key, work[1] = max key, work[2] = NaN seen
__global__ void __launch_bounds__(kMetricThreads) image_range_kernel(const float *__restrict__ img, long long rs,
                                                                     int rows, int cols, unsigned *work) {
  __shared__ unsigned smin[kMetricThreads / 32], smax[kMetricThreads / 32], snan[kMetricThreads / 32];
  unsigned kmin = 0xffffffffu, kmax = 0u, nan = 0u;
  const long long n = (long long)rows * cols;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const int r = (int)(i / cols), c = (int)(i - (long long)r * cols);
    const float v = img[r * rs + c];
    if (v != v) {
      nan = 1u;
    } else {
      const unsigned k = float_key(v);
      kmin = min(kmin, k);
      kmax = max(kmax, k);
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    kmin = min(kmin, __shfl_xor_sync(0xffffffffu, kmin, o));
    kmax = max(kmax, __shfl_xor_sync(0xffffffffu, kmax, o));
    nan |= __shfl_xor_sync(0xffffffffu, nan, o);
  }
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0) { smin[warp] = kmin; smax[warp] = kmax; snan[warp] = nan; }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int k = 1; k < kMetricThreads / 32; ++k) {
      kmin = min(kmin, smin[k]);
      kmax = max(kmax, smax[k]);
      nan |= snan[k];
    }
    atomicMin(work, kmin);
    atomicMax(work + 1, kmax);
    if (nan) atomicOr(work + 2, 1u);
  }
}

__global__ void image_range_finish(const unsigned *work, float *out2) {
  if (work[2] || work[0] == 0xffffffffu) {
    out2[0] = out2[1] = __int_as_float(0x7fc00000);
  } else {
    out2[0] = key_float(work[0]);
    out2[1] = key_float(work[1]);
  }
}

// uint8 level of clip((v - nmin) / (nmax - nmin), 0, 1) * 255 in float32
__device__ __forceinline__ int level_u8(float v, float nmin, float range) {
  float r = __fdiv_rn(__fsub_rn(v, nmin), range);
  r = fminf(fmaxf(r, 0.0f), 1.0f);
  return (int)__fmul_rn(r, 255.0f);
}

// counts[img][256] += histogram of this CTA's share of image blockIdx.y
// the same in FP64 (float64 images normalised by float64 bounds)
__device__ __forceinline__ int level_u8(double v, double nmin, double range) {
  double r = __ddiv_rn(__dsub_rn(v, nmin), range);
  r = fmin(fmax(r, 0.0), 1.0);
  return (int)__dmul_rn(r, 255.0);
}

template <typename T>
__global__ void __launch_bounds__(kMetricThreads) histogram_kernel(const T *__restrict__ imgs, long long is,
                                                                   long long rs, int rows, int cols, T nmin,
                                                                   T nmax, int *counts) {
  __shared__ int h[256];
  h[threadIdx.x] = 0;
  __syncthreads();
  const T *img = imgs + blockIdx.y * is;
  const T range = nmax - nmin;  // one rounded subtraction in T
  const long long n = (long long)rows * cols;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const int r = (int)(i / cols), c = (int)(i - (long long)r * cols);
    atomicAdd(&h[level_u8(img[r * rs + c], nmin, range)], 1);
  }
  __syncthreads();
  if (h[threadIdx.x]) atomicAdd(&counts[blockIdx.y * 256 + threadIdx.x], h[threadIdx.x]);
}

// fixed-order tree sum of kMetricThreads doubles
__device__ __forceinline__ double block_sum(double v, double *s) {
  s[threadIdx.x] = v;
  __syncthreads();
  for (int o = kMetricThreads / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) s[threadIdx.x] = __dadd_rn(s[threadIdx.x], s[threadIdx.x + o]);
    __syncthreads();
  }
  return s[0];
}

// -sum(b log2 b) over the 250 seven-wide box sums b of 1 + counts
__global__ void __launch_bounds__(kMetricThreads) entropy_kernel(const int *counts, double *out) {
  __shared__ double h[256];
  __shared__ double s[kMetricThreads];
  h[threadIdx.x] = 1.0 + (double)counts[blockIdx.x * 256 + threadIdx.x];
  __syncthreads();
  double term = 0.0;
  if (threadIdx.x < 256 - 6) {
    double b = 0.0;
    for (int k = 0; k < 7; ++k) b += h[threadIdx.x + k];  // integers: exact
    term = __dmul_rn(b, log2(b));
  }
  const double total = block_sum(term, s);
  if (threadIdx.x == 0) out[blockIdx.x] = -total;
}

// float32 gradient magnitude at (r, c) with np.gradient's stencils
__device__ __forceinline__ float grad_mag(const float *img, long long rs, int rows, int cols, int r, int c) {
  float gr, gc;
  if (r == 0) gr = __fsub_rn(img[rs + c], img[c]);
  else if (r == rows - 1) gr = __fsub_rn(img[r * rs + c], img[(r - 1) * rs + c]);
  else gr = __fdiv_rn(__fsub_rn(img[(r + 1) * rs + c], img[(r - 1) * rs + c]), 2.0f);
  const float *row = img + r * rs;
  if (c == 0) gc = __fsub_rn(row[1], row[0]);
  else if (c == cols - 1) gc = __fsub_rn(row[c], row[c - 1]);
  else gc = __fdiv_rn(__fsub_rn(row[c + 1], row[c - 1]), 2.0f);
  return __fsqrt_rn(__fadd_rn(__fmul_rn(gr, gr), __fmul_rn(gc, gc)));
}

// partial[img][blockIdx.x] = FP64 sum of this CTA's gradient magnitudes
__global__ void __launch_bounds__(kMetricThreads) sharpness_kernel(const float *__restrict__ imgs, long long is,
                                                                   long long rs, int rows, int cols,
                                                                   double *partial) {
  __shared__ double s[kMetricThreads];
  const float *img = imgs + blockIdx.y * is;
  const long long n = (long long)rows * cols;
  double acc = 0.0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const int r = (int)(i / cols), c = (int)(i - (long long)r * cols);
    acc += (double)grad_mag(img, rs, rows, cols, r, c);
  }
  const double total = block_sum(acc, s);
  if (threadIdx.x == 0) partial[blockIdx.y * kMetricBlocks + blockIdx.x] = total;
}

__global__ void __launch_bounds__(kMetricThreads) sharpness_finish(const double *partial, int nblk, double npix,
                                                                   double *out) {
  __shared__ double s[kMetricThreads];
  const double v = threadIdx.x < nblk ? partial[blockIdx.x * kMetricBlocks + threadIdx.x] : 0.0;
  const double total = block_sum(v, s);
  if (threadIdx.x == 0) out[blockIdx.x] = total / npix;
}

int metric_blocks(long long npix) {
  long long b = (npix + 4095) / 4096;
  return (int)(b < 1 ? 1 : (b > kMetricBlocks ? kMetricBlocks : b));
}

}  // namespace

extern "C" int atb_gaussian_rows(const float *src, int64_t src_row_stride, int nrow, int ncol, const double *weights,
                                 int radius, float *dst, int64_t dst_row_stride, int to_int, void *stream) {
  if (!src || !dst || !weights) return atb::fail(ATB_EINVAL, "atb_gaussian_rows: null pointer");
  if (nrow < 1 || ncol < 1 || radius < 0)
    return atb::fail(ATB_EINVAL, "atb_gaussian_rows: bad shape nrow=%d ncol=%d radius=%d", nrow, ncol, radius);
  if (ncol > 65535 * kRowTile || radius > kMaxGaussRadius)
    return atb::fail(ATB_ERANGE, "atb_gaussian_rows: ncol=%d or radius=%d too large", ncol, radius);
  if (src == dst) return atb::fail(ATB_EINVAL, "atb_gaussian_rows: in-place filtering is not supported");
  cudaStream_t st = atb::as_stream(stream);
  if (radius <= 16) {
    const int span = kSegs * kWinOut + 2 * radius;
    const size_t wsmem = sizeof(double) * (radius + 1) + sizeof(float) * kLineTile * (span | 1) +
                         sizeof(float) * kLineTile * (kSegs * kWinOut + 1);
    const dim3 wgrid((nrow + kLineTile - 1) / kLineTile, (ncol + kSegs * kWinOut - 1) / (kSegs * kWinOut));
    if (wgrid.y > 65535) return atb::fail(ATB_ERANGE, "atb_gaussian_rows: ncol=%d too large", ncol);
    auto launch = [&](auto kern) {
      int rc = atb::ensure_smem(kern, wsmem, "atb_gaussian_rows");
      if (rc != ATB_OK) return rc;
      kern<<<wgrid, kLineTile * kSegs, wsmem, st>>>(src, src_row_stride, nrow, ncol, weights, radius, dst,
                                                    dst_row_stride, to_int);
      return atb::check_launch("atb_gaussian_rows");
    };
    if (radius <= 4) return launch(gaussian_rows_win_kernel<4>);
    if (radius <= 8) return launch(gaussian_rows_win_kernel<8>);
    if (radius <= 12) return launch(gaussian_rows_win_kernel<12>);
    return launch(gaussian_rows_win_kernel<16>);
  }
  const size_t smem = sizeof(double) * (radius + 1) + sizeof(double) * (kRowTile + 2 * (size_t)radius);
  int rc = atb::ensure_smem(gaussian_rows_kernel, smem, "atb_gaussian_rows");
  if (rc != ATB_OK) return rc;
  dim3 grid(nrow, (ncol + kRowTile - 1) / kRowTile);
  gaussian_rows_kernel<<<grid, kRowTile, smem, st>>>(src, src_row_stride, ncol, weights, radius, dst,
                                                      dst_row_stride, to_int);
  return atb::check_launch("atb_gaussian_rows");
}

extern "C" int atb_gaussian_cols(const float *src, int64_t src_img_stride, int64_t src_row_stride, int nimg,
                                 int nrow, int ncol, const double *weights, int radius, float *dst,
                                 int64_t dst_img_stride, int64_t dst_row_stride, int to_int, void *stream) {
  if (!src || !dst || !weights) return atb::fail(ATB_EINVAL, "atb_gaussian_cols: null pointer");
  if (nimg < 1 || nrow < 1 || ncol < 1 || radius < 0)
    return atb::fail(ATB_EINVAL, "atb_gaussian_cols: bad shape nimg=%d nrow=%d ncol=%d radius=%d", nimg, nrow,
                     ncol, radius);
  if (src == dst) return atb::fail(ATB_EINVAL, "atb_gaussian_cols: in-place filtering is not supported");
  if ((int64_t)nrow * src_row_stride > 2147483647LL || (int64_t)nrow * dst_row_stride > 2147483647LL)
    return atb::fail(ATB_ERANGE, "atb_gaussian_cols: image of %d rows too large", nrow);
  if (radius > kMaxColRadius) return atb::fail(ATB_ERANGE, "atb_gaussian_cols: radius=%d too large", radius);
  if (radius <= 16) {
    const size_t wsmem = sizeof(double) * (radius + 1) + sizeof(float) * kLineTile * (kSegs * kWinOut + 2 * radius);
    auto kern = radius <= 4 ? gaussian_cols_win_kernel<4>
                : radius <= 8 ? gaussian_cols_win_kernel<8>
                : radius <= 12 ? gaussian_cols_win_kernel<12> : gaussian_cols_win_kernel<16>;
    int rc = atb::ensure_smem(kern, wsmem, "atb_gaussian_cols");
    if (rc != ATB_OK) return rc;
    const int gx = (ncol + kLineTile - 1) / kLineTile, gy = (nrow + kSegs * kWinOut - 1) / (kSegs * kWinOut);
    if (gy > 65535) return atb::fail(ATB_ERANGE, "atb_gaussian_cols: nrow=%d too large", nrow);
    cudaStream_t st = atb::as_stream(stream);
    for (int z0 = 0; z0 < nimg; z0 += 65535) {
      const int nz = nimg - z0 < 65535 ? nimg - z0 : 65535;
      const dim3 grid(gx, gy, nz);
      const float *s0 = src + z0 * src_img_stride;
      float *d0 = dst + z0 * dst_img_stride;
      kern<<<grid, kLineTile * kSegs, wsmem, st>>>(s0, src_img_stride, src_row_stride, nrow, ncol, weights, radius,
                                                   d0, dst_img_stride, dst_row_stride, to_int);
      rc = atb::check_launch("atb_gaussian_cols");
      if (rc != ATB_OK) return rc;
    }
    return ATB_OK;
  }
  const bool s64 = radius <= kColRadius64;
  const size_t smem = sizeof(double) * (radius + 1) +
                      (s64 ? sizeof(double) : sizeof(float)) * kColTile * (kColRows + 2 * (size_t)radius);
  int rc = s64 ? atb::ensure_smem(gaussian_cols_kernel<double>, smem, "atb_gaussian_cols")
               : atb::ensure_smem(gaussian_cols_kernel<float>, smem, "atb_gaussian_cols");
  if (rc != ATB_OK) return rc;
  const int gx = (ncol + kColTile - 1) / kColTile, gy = (nrow + kColRows - 1) / kColRows;
  if (gy > 65535) return atb::fail(ATB_ERANGE, "atb_gaussian_cols: nrow=%d too large", nrow);
  cudaStream_t st = atb::as_stream(stream);
  for (int z0 = 0; z0 < nimg; z0 += 65535) {
    const int nz = nimg - z0 < 65535 ? nimg - z0 : 65535;
    const dim3 grid(gx, gy, nz);
    const float *s0 = src + z0 * src_img_stride;
    float *d0 = dst + z0 * dst_img_stride;
    if (s64)
      gaussian_cols_kernel<double><<<grid, kColThreads, smem, st>>>(s0, src_img_stride, src_row_stride, nrow, ncol,
                                                                    weights, radius, d0, dst_img_stride,
                                                                    dst_row_stride, to_int);
    else
      gaussian_cols_kernel<float><<<grid, kColThreads, smem, st>>>(s0, src_img_stride, src_row_stride, nrow, ncol,
                                                                   weights, radius, d0, dst_img_stride,
                                                                   dst_row_stride, to_int);
    rc = atb::check_launch("atb_gaussian_cols");
    if (rc != ATB_OK) return rc;
  }
  return ATB_OK;
}

extern "C" int atb_zoom_linear(const float *src, int64_t src_row_stride, int in_rows, int in_cols, float *dst,
                               int64_t dst_row_stride, int out_rows, int out_cols, void *stream) {
  if (!src || !dst) return atb::fail(ATB_EINVAL, "atb_zoom_linear: null pointer");
  if (in_rows < 1 || in_cols < 1 || out_rows < 1 || out_cols < 1)
    return atb::fail(ATB_EINVAL, "atb_zoom_linear: bad shape %dx%d -> %dx%d", in_rows, in_cols, out_rows, out_cols);
  if (out_rows > 65535) return atb::fail(ATB_ERANGE, "atb_zoom_linear: out_rows=%d too large", out_rows);
  dim3 grid((out_cols + 255) / 256, out_rows);
  zoom_linear_kernel<<<grid, 256, 0, atb::as_stream(stream)>>>(src, src_row_stride, in_rows, in_cols, dst,
                                                               dst_row_stride, out_rows, out_cols);
  return atb::check_launch("atb_zoom_linear");
}

extern "C" int atb_image_range(const float *img, int64_t row_stride, int rows, int cols, void *work, float *out2,
                               void *stream) {
  if (!img || !work || !out2) return atb::fail(ATB_EINVAL, "atb_image_range: null pointer");
  if (rows < 1 || cols < 1) return atb::fail(ATB_EINVAL, "atb_image_range: bad shape %dx%d", rows, cols);
  cudaStream_t st = atb::as_stream(stream);
  unsigned *w = static_cast<unsigned *>(work);
  cudaError_t e;
  if ((e = cudaMemsetAsync(w, 0xff, sizeof(unsigned), st)) != cudaSuccess ||
      (e = cudaMemsetAsync(w + 1, 0, 2 * sizeof(unsigned), st)) != cudaSuccess)
    return atb::fail(ATB_ECUDA, "atb_image_range: %s", cudaGetErrorString(e));
  image_range_kernel<<<metric_blocks((long long)rows * cols), kMetricThreads, 0, st>>>(img, row_stride, rows, cols,
                                                                                      w);
  int rc = atb::check_launch("atb_image_range");
  if (rc != ATB_OK) return rc;
  image_range_finish<<<1, 1, 0, st>>>(w, out2);
  return atb::check_launch("atb_image_range");
}

extern "C" int64_t atb_slice_metric_workspace(int nimg, int rows, int cols, int metric) {
  (void)rows;
  (void)cols;
  if (nimg < 1 || (metric != ATB_METRIC_ENTROPY && metric != ATB_METRIC_SHARPNESS)) return 0;
  return (int64_t)nimg * kMetricBlocks * (int64_t)sizeof(double);
}

extern "C" int atb_slice_metric(const float *imgs, int64_t img_stride, int64_t row_stride, int nimg, int rows,
                                int cols, int metric, float nmin, float nmax, void *work, int64_t work_bytes,
                                double *out, void *stream) {
  if (!imgs || !work || !out) return atb::fail(ATB_EINVAL, "atb_slice_metric: null pointer");
  if (nimg < 1 || rows < 1 || cols < 1)
    return atb::fail(ATB_EINVAL, "atb_slice_metric: bad shape nimg=%d rows=%d cols=%d", nimg, rows, cols);
  if (nimg > 65535) return atb::fail(ATB_ERANGE, "atb_slice_metric: nimg=%d too large", nimg);
  if (work_bytes < atb_slice_metric_workspace(nimg, rows, cols, metric))
    return atb::fail(ATB_EINVAL, "atb_slice_metric: workspace of %lld bytes is too small", (long long)work_bytes);
  cudaStream_t st = atb::as_stream(stream);
  const int nblk = metric_blocks((long long)rows * cols);
  if (metric == ATB_METRIC_ENTROPY) {
    int *counts = static_cast<int *>(work);
    cudaError_t e = cudaMemsetAsync(counts, 0, sizeof(int) * 256 * (size_t)nimg, st);
    if (e != cudaSuccess) return atb::fail(ATB_ECUDA, "atb_slice_metric: %s", cudaGetErrorString(e));
    histogram_kernel<float><<<dim3(nblk, nimg), kMetricThreads, 0, st>>>(imgs, img_stride, row_stride, rows, cols,
                                                                         nmin, nmax, counts);
    int rc = atb::check_launch("atb_slice_metric");
    if (rc != ATB_OK) return rc;
    entropy_kernel<<<nimg, kMetricThreads, 0, st>>>(counts, out);
    return atb::check_launch("atb_slice_metric");
  }
  if (metric == ATB_METRIC_SHARPNESS) {
    if (rows < 2 || cols < 2)
      return atb::fail(ATB_EINVAL, "atb_slice_metric: the gradient needs at least 2 x 2 pixels");
    double *partial = static_cast<double *>(work);
    sharpness_kernel<<<dim3(nblk, nimg), kMetricThreads, 0, st>>>(imgs, img_stride, row_stride, rows, cols,
                                                                  partial);
    int rc = atb::check_launch("atb_slice_metric");
    if (rc != ATB_OK) return rc;
    sharpness_finish<<<nimg, kMetricThreads, 0, st>>>(partial, nblk, (double)rows * (double)cols, out);
    return atb::check_launch("atb_slice_metric");
  }
  return atb::fail(ATB_EINVAL, "atb_slice_metric: unknown metric %d", metric);
}

extern "C" int atb_slice_entropy64(const double *imgs, int64_t img_stride, int64_t row_stride, int nimg, int rows,
                                   int cols, double nmin, double nmax, void *work, int64_t work_bytes, double *out,
                                   void *stream) {
  if (!imgs || !work || !out) return atb::fail(ATB_EINVAL, "atb_slice_entropy64: null pointer");
  if (nimg < 1 || rows < 1 || cols < 1)
    return atb::fail(ATB_EINVAL, "atb_slice_entropy64: bad shape nimg=%d rows=%d cols=%d", nimg, rows, cols);
  if (nimg > 65535) return atb::fail(ATB_ERANGE, "atb_slice_entropy64: nimg=%d too large", nimg);
  if (work_bytes < atb_slice_metric_workspace(nimg, rows, cols, ATB_METRIC_ENTROPY))
    return atb::fail(ATB_EINVAL, "atb_slice_entropy64: workspace of %lld bytes is too small", (long long)work_bytes);
  cudaStream_t st = atb::as_stream(stream);
  const int nblk = metric_blocks((long long)rows * cols);
  int *counts = static_cast<int *>(work);
  cudaError_t e = cudaMemsetAsync(counts, 0, sizeof(int) * 256 * (size_t)nimg, st);
  if (e != cudaSuccess) return atb::fail(ATB_ECUDA, "atb_slice_entropy64: %s", cudaGetErrorString(e));
  histogram_kernel<double><<<dim3(nblk, nimg), kMetricThreads, 0, st>>>(imgs, img_stride, row_stride, rows, cols,
                                                                        nmin, nmax, counts);
  int rc = atb::check_launch("atb_slice_entropy64");
  if (rc != ATB_OK) return rc;
  entropy_kernel<<<nimg, kMetricThreads, 0, st>>>(counts, out);
  return atb::check_launch("atb_slice_entropy64");
}
