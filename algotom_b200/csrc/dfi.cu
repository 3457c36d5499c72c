// Direct Fourier inversion (DFI), sm_100a: the B-spline prefilter and the
// polar-to-Cartesian regridding of algotom's dfi_reconstruction
// (algotom/rec/reconstruction.py:687-907).  The row transform of the
// sinogram and the inverse 2-D transform of the regridded spectrum are
// library FFTs; these two kernels are the rest.
//
// - atb_spline_prefilter: B-spline coefficients (order 3 or 5) of many
//   strided lines, real or interleaved complex, as the FIR of the
//   prefilter's impulse response (spline_fir.cuh), one thread per output
//   sample, each tile staged in shared memory with its halo.  Extension:
//   half-sample symmetric ("reflect": scipy's "reflect" and, after 12 edge
//   samples of padding, "nearest") or whole-sample symmetric ("mirror":
//   scipy's "mirror" and "wrap").
// - atb_dfi_regrid: for every pixel of the W x W Cartesian frequency grid,
//   the polar coordinates of generate_mapping_coordinate
//   (reconstruction.py:687-728: radius clipped to floor((W-1)/2), the half
//   plane folded by the Hermitian symmetry of a real image's spectrum, angle
//   scaled to the sinogram's rows), then the quintic B-spline interpolation
//   of the complex row spectra at that point with half-sample symmetric
//   taps (map_coordinates(order=5, mode="reflect")), times the unit circle
//   mask of make_circle_mask(W, 1.0), written in ifftshift order (ready for
//   the inverse transform).  FP64 throughout.
#include <cmath>

#include "common.cuh"
#include "dfi_grid.cuh"
#include "spline_fir.cuh"

namespace {

constexpr int kFirThreads = 256;
constexpr int kGridThreads = 256;
using atb::spline::fir_block;
using atb::spline::fir_pad;
using atb::spline::sym_index;
using atb::spline::Taps;
using atb::spline::make_taps;

__global__ void __launch_bounds__(kFirThreads)
    prefilter_kernel(const double *__restrict__ src, double *__restrict__ dst, long long line_stride, long long es,
                     int nlines, int ncomp, int n, int boundary, Taps taps) {
  const long long e = blockIdx.x * (long long)kFirThreads + threadIdx.x;
  if (e >= (long long)nlines * ncomp * n) return;
  // element i of line (outer, comp); consecutive threads walk the
  // contiguous direction of the data
  int i, outer, comp;
  if (es == ncomp) {  // elements contiguous: i fastest
    i = (int)(e % n);
    const long long l = e / n;
    comp = (int)(l % ncomp);
    outer = (int)(l / ncomp);
  } else {  // lines contiguous: (outer, comp) fastest
    const long long l = e % ((long long)nlines * ncomp);
    i = (int)(e / ((long long)nlines * ncomp));
    comp = (int)(l % ncomp);
    outer = (int)(l / ncomp);
  }
  const double *line = src + outer * line_stride + comp;
  double acc = taps.h[0] * line[(long long)i * es];
  for (int k = 1; k <= taps.ntaps; ++k) {
    const double a = line[(long long)sym_index(i - k, n, boundary) * es];
    const double b = line[(long long)sym_index(i + k, n, boundary) * es];
    acc += taps.h[k] * (a + b);
  }
  dst[outer * line_stride + comp + (long long)i * es] = acc;
}

// Tiled forms: the strip a CTA filters, plus its 2 x ntaps halo (symmetric
// extension resolved while staging), is staged in shared memory once, and
// every thread computes kFirBlk consecutive outputs of one line from one
// sliding window of kFirBlk + 2 ntaps staged values held in turn in a
// register: each value is read from shared memory once and feeds up to
// kFirBlk outputs, against 2 ntaps + 1 reads per output (the untiled
// kernel above, and a first tiled form, read every tap per output: shared-
// memory bandwidth bound them).  The tap count is a template parameter, so
// the window loop unrolls with its taps as constants.
constexpr int kFirBlk = 8;      // consecutive outputs per thread
constexpr int kFirLines = 32;   // lines per CTA (filter axis strided)
constexpr int kFirRows = kFirBlk * (kFirThreads / 32);  // 64 outputs per line per CTA
constexpr int kFirSeg = kFirBlk * kFirThreads;          // outputs per CTA (filter axis contiguous)

// filter axis strided, lines contiguous: element (i, l) at src[i * es + l],
// l < nl; CTA = 32 consecutive l x 64 consecutive i, warp w computing
// positions [8 w, 8 w + 8) of its lane's line
template <int NT>
__global__ void __launch_bounds__(kFirThreads)
    prefilter_cols_kernel(const double *__restrict__ src, double *__restrict__ dst, long long es, int nl, int n,
                          int boundary, Taps taps) {
  extern __shared__ double xs[];  // [kFirRows + 2 NT][kFirLines]
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int l = blockIdx.x * kFirLines + lane;
  const int i0 = blockIdx.y * kFirRows;
  constexpr int span = kFirRows + 2 * NT;
  for (int q = warp; q < span; q += kFirThreads / 32)
    xs[q * kFirLines + lane] = l < nl ? src[(long long)sym_index(i0 - NT + q, n, boundary) * es + l] : 0.0;
  __syncthreads();
  const int r0 = warp * kFirBlk;
  if (l >= nl || i0 + r0 >= n) return;
  double acc[kFirBlk];
  const double *c = xs + r0 * kFirLines + lane;
  fir_block<NT, kFirBlk>(taps, [&](int t) { return c[t * kFirLines]; }, acc);
#pragma unroll
  for (int r = 0; r < kFirBlk; ++r)
    if (i0 + r0 + r < n) dst[(long long)(i0 + r0 + r) * es + l] = acc[r];
}

// filter axis contiguous: element (line, i, comp) at
// src[line * ls + i * ncomp + comp]; CTA = one line x kFirSeg / ncomp
// positions, thread = one component x kFirBlk consecutive positions
template <int NT>
__global__ void __launch_bounds__(kFirThreads)
    prefilter_rows_kernel(const double *__restrict__ src, double *__restrict__ dst, long long ls, int ncomp, int n,
                          int boundary, Taps taps) {
  extern __shared__ double xs[];  // per component: fir_pad(kSeg / ncomp + 2 NT) values
  const long long line = blockIdx.y;
  const int seg = kFirSeg / ncomp, i0 = blockIdx.x * seg;
  const int span = seg + 2 * NT, stride = fir_pad(span) + 1;
  const double *in = src + line * ls;
  for (int e = threadIdx.x; e < span * ncomp; e += kFirThreads) {
    const int q = e / ncomp, comp = e - q * ncomp;
    xs[comp * stride + fir_pad(q)] = in[(long long)sym_index(i0 - NT + q, n, boundary) * ncomp + comp];
  }
  __syncthreads();
  const int per = kFirThreads / ncomp, comp = threadIdx.x / per;
  const int q0 = (threadIdx.x - comp * per) * kFirBlk;
  if (i0 + q0 >= n) return;
  double acc[kFirBlk];
  const double *c = xs + comp * stride;
  fir_block<NT, kFirBlk>(taps, [&](int t) { return c[fir_pad(q0 + t)]; }, acc);
#pragma unroll
  for (int r = 0; r < kFirBlk; ++r)
    if (i0 + q0 + r < n) dst[line * ls + (long long)(i0 + q0 + r) * ncomp + comp] = acc[r];
}

__global__ void __launch_bounds__(kGridThreads)
    regrid_kernel(const double2 *__restrict__ coef, int nrow, int w, double2 *__restrict__ out) {
  const long long e = blockIdx.x * (long long)kGridThreads + threadIdx.x;
  if (e >= (long long)w * w) return;
  const int i = (int)(e / w), j = (int)(e - (long long)i * w);
  // written where ifftshift puts it: (i - w // 2, j - w // 2) mod w
  const long long oi = (i + w - w / 2) % w, oj = (j + w - w / 2) % w;
  out[oi * w + oj] = atb::dfi::regrid_point(coef, w, nrow, w, i, j);
}

// __dfi_handle_angles (reconstruction.py:731-749), first half: the fold of
// a 360-degree scan (n = nrow_in / 2 + 1 rows, row r = (row r + row
// nrow_in - n + r mirrored) / 2 in float32, as NumPy's float32 arithmetic)
// and the stack the angle shift runs on, rows 0 .. n - 2 followed by all n
// rows mirrored left-right, widened to float64 for the spline prefilter.
// One thread per output sample.
struct StackArgs {
  const float *src;
  long long srs, sss;
  int nrow_in, n, ncol, fold;
  double *dst;
  long long drs, dss;
};

__global__ void __launch_bounds__(kGridThreads) angle_stack_kernel(StackArgs a) {
  const int j = blockIdx.x * kGridThreads + threadIdx.x;
  if (j >= a.ncol) return;
  const int i = blockIdx.y, k = blockIdx.z;
  int r = i, col = j;
  if (i >= a.n - 1) {
    r = i - (a.n - 1);
    col = a.ncol - 1 - j;
  }
  const float *s = a.src + k * a.sss;
  float v = __ldg(s + r * a.srs + col);
  if (a.fold) v = (v + __ldg(s + (long long)(a.nrow_in - a.n + r) * a.srs + (a.ncol - 1 - col))) * 0.5f;
  a.dst[i * a.drs + k * a.dss + j] = (double)v;
}

// second half: scipy.ndimage.shift(stack, (shift, 0), order=3,
// mode="wrap")[:nout] from the stack's cubic B-spline coefficients along
// the rows (whole-sample symmetric prefilter): the sample coordinate
// i - shift wrapped into [0, m - 1] with period m - 1, four taps with
// mirrored indices, rounded to float32; flip reverses rows and columns
// (the flipud(fliplr(.)) of descending angles).
struct WrapArgs {
  const double *coef;
  long long crs, css;
  int m, ncol, nout, flip;
  double shift;
  float *dst;
  long long drs, dss;
};

__device__ __forceinline__ double bspline3(double u) {
  const double a = fabs(u);
  if (a < 1.0) return 2.0 / 3.0 - a * a + a * a * a / 2.0;
  if (a < 2.0) {
    const double b = 2.0 - a;
    return b * b * b / 6.0;
  }
  return 0.0;
}

__global__ void __launch_bounds__(kGridThreads) wrap_shift_kernel(WrapArgs a) {
  const int j = blockIdx.x * kGridThreads + threadIdx.x;
  if (j >= a.ncol) return;
  const int i = blockIdx.y, k = blockIdx.z, m = a.m;
  double cc = (double)i - a.shift;
  const double sz = (double)(m - 1);
  if (m > 1) {
    if (cc < 0.0) cc += sz * (floor(-cc / sz) + 1.0);
    if (cc > sz) cc -= sz * floor(cc / sz);
  }
  const double f = floor(cc);
  const int fi = (int)f;
  const double *c = a.coef + k * a.css + j;
  double v = 0.0;
#pragma unroll
  for (int t = -1; t <= 2; ++t) {
    int idx = 0;
    if (m > 1) {
      const int p = 2 * (m - 1);
      int r = (fi + t) % p;
      if (r < 0) r += p;
      idx = r >= m ? p - r : r;
    }
    v += bspline3(cc - (double)(fi + t)) * __ldg(c + idx * a.crs);
  }
  const int oi = a.flip ? a.nout - 1 - i : i, oj = a.flip ? a.ncol - 1 - j : j;
  a.dst[oi * a.drs + k * a.dss + oj] = (float)v;
}

}  // namespace

extern "C" int atb_spline_prefilter(const double *src, double *dst, int64_t line_stride, int64_t elem_stride,
                                    int nlines, int ncomp, int n, int order, int boundary, void *stream) {
  if (!src || !dst) return atb::fail(ATB_EINVAL, "atb_spline_prefilter: null pointer");
  if (src == dst) return atb::fail(ATB_EINVAL, "atb_spline_prefilter: src and dst must not overlap");
  if (nlines < 1 || n < 1 || (ncomp != 1 && ncomp != 2))
    return atb::fail(ATB_EINVAL, "atb_spline_prefilter: bad shape nlines=%d n=%d ncomp=%d", nlines, n, ncomp);
  if ((order != 3 && order != 5) || (boundary != 0 && boundary != 1))
    return atb::fail(ATB_EINVAL, "atb_spline_prefilter: order %d / boundary %d unsupported", order, boundary);
  if (elem_stride != ncomp && line_stride != ncomp)
    return atb::fail(ATB_EINVAL, "atb_spline_prefilter: lines or elements must be contiguous");
  static const Taps taps3 = make_taps(3), taps5 = make_taps(5);
  const Taps &taps = order == 5 ? taps5 : taps3;
  cudaStream_t st = atb::as_stream(stream);
  const int nt = taps.ntaps;
  if (line_stride == ncomp && (long long)nlines * ncomp <= 2147483647LL && (n + kFirRows - 1) / kFirRows <= 65535) {
    // lines contiguous: tiles of 32 lines x 64 positions
    const int nl = nlines * ncomp;
    const size_t smem = sizeof(double) * kFirLines * (kFirRows + 2 * nt);
    const dim3 grid((nl + kFirLines - 1) / kFirLines, (n + kFirRows - 1) / kFirRows);
    int rc;
    if (nt == 48) {
      rc = atb::ensure_smem(prefilter_cols_kernel<48>, smem, "atb_spline_prefilter");
      if (rc == ATB_OK) prefilter_cols_kernel<48><<<grid, kFirThreads, smem, st>>>(src, dst, elem_stride, nl, n, boundary, taps);
    } else {
      rc = atb::ensure_smem(prefilter_cols_kernel<32>, smem, "atb_spline_prefilter");
      if (rc == ATB_OK) prefilter_cols_kernel<32><<<grid, kFirThreads, smem, st>>>(src, dst, elem_stride, nl, n, boundary, taps);
    }
    return rc != ATB_OK ? rc : atb::check_launch("atb_spline_prefilter");
  }
  if (elem_stride == ncomp && nlines <= 65535) {
    // elements contiguous: one line segment of kFirSeg / ncomp positions per CTA
    const int seg = kFirSeg / ncomp;
    const size_t smem = sizeof(double) * ncomp * (size_t)((seg + 2 * nt) + ((seg + 2 * nt) >> 3) + 1);
    const dim3 grid((n + seg - 1) / seg, nlines);
    int rc;
    if (nt == 48) {
      rc = atb::ensure_smem(prefilter_rows_kernel<48>, smem, "atb_spline_prefilter");
      if (rc == ATB_OK) prefilter_rows_kernel<48><<<grid, kFirThreads, smem, st>>>(src, dst, line_stride, ncomp, n, boundary, taps);
    } else {
      rc = atb::ensure_smem(prefilter_rows_kernel<32>, smem, "atb_spline_prefilter");
      if (rc == ATB_OK) prefilter_rows_kernel<32><<<grid, kFirThreads, smem, st>>>(src, dst, line_stride, ncomp, n, boundary, taps);
    }
    return rc != ATB_OK ? rc : atb::check_launch("atb_spline_prefilter");
  }
  const long long total = (long long)nlines * ncomp * n;
  const long long blocks = (total + kFirThreads - 1) / kFirThreads;
  if (blocks > 2147483647LL) return atb::fail(ATB_ERANGE, "atb_spline_prefilter: too many samples");
  prefilter_kernel<<<(int)blocks, kFirThreads, 0, st>>>(src, dst, line_stride, elem_stride, nlines, ncomp, n,
                                                         boundary, taps);
  return atb::check_launch("atb_spline_prefilter");
}

extern "C" int atb_dfi_regrid(const double *coef, int nrow, int width, double *out, void *stream) {
  if (!coef || !out) return atb::fail(ATB_EINVAL, "atb_dfi_regrid: null pointer");
  if (nrow < 1 || width < 1) return atb::fail(ATB_EINVAL, "atb_dfi_regrid: bad shape %dx%d", nrow, width);
  if (width > 46340) return atb::fail(ATB_ERANGE, "atb_dfi_regrid: width=%d too large", width);
  const long long total = (long long)width * width;
  regrid_kernel<<<(int)((total + kGridThreads - 1) / kGridThreads), kGridThreads, 0, atb::as_stream(stream)>>>(
      reinterpret_cast<const double2 *>(coef), nrow, width, reinterpret_cast<double2 *>(out));
  return atb::check_launch("atb_dfi_regrid");
}

extern "C" int atb_dfi_angle_stack(const float *src, int64_t src_row_stride, int64_t src_slice_stride, int nrow_in,
                                   int nslice, int ncol, int fold, double *dst, int64_t dst_row_stride,
                                   int64_t dst_slice_stride, void *stream) {
  if (!src || !dst) return atb::fail(ATB_EINVAL, "atb_dfi_angle_stack: null pointer");
  if (nrow_in < 1 || nslice < 1 || ncol < 1 || nslice > 65535)
    return atb::fail(ATB_EINVAL, "atb_dfi_angle_stack: bad shape %dx%dx%d", nrow_in, nslice, ncol);
  StackArgs a;
  a.src = src; a.srs = src_row_stride; a.sss = src_slice_stride;
  a.nrow_in = nrow_in; a.n = fold ? nrow_in / 2 + 1 : nrow_in; a.ncol = ncol; a.fold = fold ? 1 : 0;
  a.dst = dst; a.drs = dst_row_stride; a.dss = dst_slice_stride;
  const int m = 2 * a.n - 1;
  if (m > 65535) return atb::fail(ATB_ERANGE, "atb_dfi_angle_stack: %d rows > 65535", m);
  const dim3 grid((ncol + kGridThreads - 1) / kGridThreads, m, nslice);
  angle_stack_kernel<<<grid, kGridThreads, 0, atb::as_stream(stream)>>>(a);
  return atb::check_launch("atb_dfi_angle_stack");
}

extern "C" int atb_wrap_shift_rows(const double *coef, int64_t coef_row_stride, int64_t coef_slice_stride, int m,
                                   int nslice, int ncol, double shift, int nout, int flip, float *dst,
                                   int64_t dst_row_stride, int64_t dst_slice_stride, void *stream) {
  if (!coef || !dst) return atb::fail(ATB_EINVAL, "atb_wrap_shift_rows: null pointer");
  if (m < 1 || nslice < 1 || ncol < 1 || nout < 1 || nout > m || nslice > 65535)
    return atb::fail(ATB_EINVAL, "atb_wrap_shift_rows: bad shape m=%d nslice=%d ncol=%d nout=%d", m, nslice, ncol,
                     nout);
  if (!std::isfinite(shift) || std::fabs(shift) > 1e9)
    return atb::fail(ATB_EINVAL, "atb_wrap_shift_rows: shift %g out of range", shift);
  WrapArgs a;
  a.coef = coef; a.crs = coef_row_stride; a.css = coef_slice_stride;
  a.m = m; a.ncol = ncol; a.nout = nout; a.flip = flip ? 1 : 0; a.shift = shift;
  a.dst = dst; a.drs = dst_row_stride; a.dss = dst_slice_stride;
  const dim3 grid((ncol + kGridThreads - 1) / kGridThreads, nout, nslice);
  wrap_shift_kernel<<<grid, kGridThreads, 0, atb::as_stream(stream)>>>(a);
  return atb::check_launch("atb_wrap_shift_rows");
}
