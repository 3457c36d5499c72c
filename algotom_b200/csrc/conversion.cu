// 360-degree sinograms with an offset rotation axis, sm_100a: the row
// operations of algotom's extend_sinogram, convert_sinogram_360_to_180 and
// convert_sinogram_180_to_360 (algotom/prep/conversion.py:76-454).
//
// One CTA per sinogram row.  The row (optionally mirrored left-right and
// -log'ed in float32, as the reference's NumPy float32 arithmetic does) is
// staged in shared memory with 12 copies of each end sample on either side;
// a sub-pixel shift then follows scipy.ndimage.shift(x, (0, s),
// order 3, mode "nearest"), the published cubic B-spline method: the padded
// row becomes spline coefficients through the prefilter of pole
// z = sqrt(3) - 2 on its half-sample symmetric extension, applied as the
// 65-tap FIR of its impulse response (spline_fir.cuh; every thread one
// coefficient, exact to 1e-17 relative where the recursion is a serial chain
// through the row), and every thread samples the spline at x - s with the
// cubic B-spline weights, coefficient indices clamped to the padded row.  (Along the angle
// axis the shift is zero and a cubic spline sampled at its knots returns its
// samples, so rows are independent.)  The shifted row is rounded to float32
// as scipy's output is.  extend_sinogram then scales the overlap columns by
// a linear ramp, pads with the edge sample and doubles
// (conversion.py:425-454), all in the same pass.
#include <cmath>

#include "common.cuh"
#include "spline_fir.cuh"

namespace {

using atb::spline::fir_block;
using atb::spline::fir_pad;
using atb::spline::make_taps;
using atb::spline::sym_index;
using atb::spline::Taps;

constexpr int kPad = 12;       // end samples replicated on each side
constexpr int kThreads = 256;
constexpr int kMaxCols = 16384;
constexpr int kTaps = 32;      // the cubic prefilter's taps (make_taps(3).ntaps)
constexpr int kBlk = 8;        // coefficients per thread and window

struct RowArgs {
  const float *src;
  long long srs;
  int nrow, ncol;
  int ncol_src;  // source columns (<= ncol); the rest repeat the last one
  int flip, apply_log;
  double shift;  // 0: no shift
  int ov, side;  // extend: overlap columns and side; ov == 0: plain shift
  float *dst;
  long long drs;
};

__global__ void __launch_bounds__(kThreads) row_kernel(RowArgs a, Taps taps) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int n = a.ncol, big = n + 2 * kPad;
  double *c = reinterpret_cast<double *>(smem);  // [big] spline coefficients
  float *x = reinterpret_cast<float *>(c + big);  // [fir_pad(big)] the padded row, padded layout
  float *y;                                       // [n] the (shifted) row
  const int row = blockIdx.x;
  const float *src = a.src + row * a.srs;
  for (int k = threadIdx.x; k < big; k += kThreads) {
    const int col = min(max(k - kPad, 0), n - 1);
    float v = src[min(a.flip ? n - 1 - col : col, a.ncol_src - 1)];
    if (a.apply_log) v = -logf(v);
    x[fir_pad(k)] = v;
  }
  __syncthreads();
  if (a.shift != 0.0) {
    // kBlk consecutive coefficients per thread from one sliding window
    // (each staged value read once per window, not once per tap)
    for (int k0 = threadIdx.x * kBlk; k0 < big; k0 += kThreads * kBlk) {
      double acc[kBlk];
      fir_block<kTaps, kBlk>(
          taps, [&](int t) { return (double)x[fir_pad(sym_index(k0 + t - kTaps, big, 0))]; }, acc);
#pragma unroll
      for (int r = 0; r < kBlk; ++r)
        if (k0 + r < big) c[k0 + r] = acc[r];
    }
    __syncthreads();
    y = x;  // the padded row is no longer read
    for (int k = threadIdx.x; k < n; k += kThreads) {
      const double cc = __dadd_rn(__dsub_rn((double)k, a.shift), (double)kPad);
      const double f = floor(cc), t = __dsub_rn(cc, f), u = __dsub_rn(1.0, t);
      const double t2 = __dmul_rn(t, t), t3 = pow(t, 3.0);
      const int i0 = (int)f;
      // cubic B-spline weights of the taps floor - 1 .. floor + 2
      const double w0 = pow(u, 3.0) / 6.0;
      const double w1 = __dadd_rn(__dsub_rn(4.0, __dmul_rn(6.0, t2)), __dmul_rn(3.0, t3)) / 6.0;
      const double w2 =
          __dsub_rn(__dadd_rn(__dadd_rn(1.0, __dmul_rn(3.0, t)), __dmul_rn(3.0, t2)), __dmul_rn(3.0, t3)) / 6.0;
      const double w3 = t3 / 6.0;
      double v = __dmul_rn(w0, c[min(max(i0 - 1, 0), big - 1)]);
      v = __dadd_rn(v, __dmul_rn(w1, c[min(max(i0, 0), big - 1)]));
      v = __dadd_rn(v, __dmul_rn(w2, c[min(max(i0 + 1, 0), big - 1)]));
      v = __dadd_rn(v, __dmul_rn(w3, c[min(max(i0 + 2, 0), big - 1)]));
      y[k] = __double2float_rn(v);
    }
  } else {
    y = reinterpret_cast<float *>(c);  // no coefficients needed
    for (int k = threadIdx.x; k < n; k += kThreads) y[k] = x[fir_pad(k + kPad)];
  }
  __syncthreads();
  float *dst = a.dst + row * a.drs;
  if (a.ov == 0) {
    for (int k = threadIdx.x; k < n; k += kThreads) dst[k] = y[k];
    return;
  }
  // extend: ramp over the overlap, edge padding to 2 n - ov columns, x 2
  const int ov = a.ov, pad = n - ov;
  const double step = ov > 1 ? 1.0 / (double)(ov - 1) : 0.0;
  // NumPy's linspace(start, stop, ov): m * step + start, the last value
  // exactly stop (a single value is start)
  auto weighted = [&](int k) -> float {  // column k of the ramped row
    if (a.side == 1) {
      if (k < n - ov) return y[k];
      const int m = k - (n - ov);  // linspace(1, 0, ov)[m]
      const double w = ov == 1 ? 1.0 : (m == ov - 1 ? 0.0 : __dadd_rn(__dmul_rn((double)m, -step), 1.0));
      return __double2float_rn(__dmul_rn((double)y[k], w));
    }
    if (k >= ov) return y[k];
    const double w = ov == 1 ? 0.0 : (k == ov - 1 ? 1.0 : __dmul_rn((double)k, step));  // linspace(0, 1, ov)[k]
    return __double2float_rn(__dmul_rn((double)y[k], w));
  };
  for (int k = threadIdx.x; k < n + pad; k += kThreads) {
    float v;
    if (a.side == 1) v = weighted(min(k, n - 1));
    else v = weighted(max(k - pad, 0));
    dst[k] = 2.0f * v;
  }
}

int launch_rows(const RowArgs &a, const char *what, void *stream) {
  static const Taps taps = make_taps(3);
  const int big = a.ncol + 2 * kPad;
  const size_t smem = sizeof(double) * big + sizeof(float) * (big + (big >> 3) + 1);
  int rc = atb::ensure_smem(row_kernel, smem, what);
  if (rc != ATB_OK) return rc;
  row_kernel<<<a.nrow, kThreads, smem, atb::as_stream(stream)>>>(a, taps);
  return atb::check_launch(what);
}

}  // namespace

extern "C" int atb_shift_rows(const float *src, int64_t src_row_stride, int nrow, int ncol, double shift, int flip,
                              float *dst, int64_t dst_row_stride, void *stream) {
  if (!src || !dst) return atb::fail(ATB_EINVAL, "atb_shift_rows: null pointer");
  if (nrow < 1 || ncol < 1) return atb::fail(ATB_EINVAL, "atb_shift_rows: bad shape %dx%d", nrow, ncol);
  if (ncol > kMaxCols) return atb::fail(ATB_ERANGE, "atb_shift_rows: ncol=%d > %d", ncol, kMaxCols);
  if (!std::isfinite(shift)) return atb::fail(ATB_EINVAL, "atb_shift_rows: shift is not finite");
  RowArgs a;
  a.src = src; a.srs = src_row_stride; a.nrow = nrow; a.ncol = ncol; a.ncol_src = ncol;
  a.flip = flip ? 1 : 0; a.apply_log = 0; a.shift = shift; a.ov = 0; a.side = 0;
  a.dst = dst; a.drs = dst_row_stride;
  return launch_rows(a, "atb_shift_rows", stream);
}

extern "C" int atb_extend_rows(const float *src, int64_t src_row_stride, int nrow, int ncol, int apply_log,
                               double shift, int overlap, int side, float *dst, int64_t dst_row_stride,
                               void *stream) {
  if (!src || !dst) return atb::fail(ATB_EINVAL, "atb_extend_rows: null pointer");
  if (nrow < 1 || ncol < 1) return atb::fail(ATB_EINVAL, "atb_extend_rows: bad shape %dx%d", nrow, ncol);
  if (ncol > kMaxCols) return atb::fail(ATB_ERANGE, "atb_extend_rows: ncol=%d > %d", ncol, kMaxCols);
  if (overlap < 1 || overlap > ncol || (side != 0 && side != 1))
    return atb::fail(ATB_EINVAL, "atb_extend_rows: overlap %d / side %d invalid for %d columns", overlap, side, ncol);
  if (!std::isfinite(shift)) return atb::fail(ATB_EINVAL, "atb_extend_rows: shift is not finite");
  RowArgs a;
  a.src = src; a.srs = src_row_stride; a.nrow = nrow; a.ncol = ncol; a.ncol_src = ncol;
  a.flip = 0; a.apply_log = apply_log ? 1 : 0; a.shift = shift; a.ov = overlap; a.side = side;
  a.dst = dst; a.drs = dst_row_stride;
  return launch_rows(a, "atb_extend_rows", stream);
}

extern "C" int atb_shift_rows_ext(const float *src, int64_t src_row_stride, int nrow, int ncol_src, int ncol,
                                  double shift, float *dst, int64_t dst_row_stride, void *stream) {
  if (!src || !dst) return atb::fail(ATB_EINVAL, "atb_shift_rows_ext: null pointer");
  if (nrow < 1 || ncol_src < 1 || ncol < ncol_src)
    return atb::fail(ATB_EINVAL, "atb_shift_rows_ext: bad shape %dx%d -> %d columns", nrow, ncol_src, ncol);
  if (ncol > kMaxCols) return atb::fail(ATB_ERANGE, "atb_shift_rows_ext: ncol=%d > %d", ncol, kMaxCols);
  if (!std::isfinite(shift)) return atb::fail(ATB_EINVAL, "atb_shift_rows_ext: shift is not finite");
  RowArgs a;
  a.src = src; a.srs = src_row_stride; a.nrow = nrow; a.ncol = ncol; a.ncol_src = ncol_src;
  a.flip = 0; a.apply_log = 0; a.shift = shift; a.ov = 0; a.side = 0;
  a.dst = dst; a.drs = dst_row_stride;
  return launch_rows(a, "atb_shift_rows_ext", stream);
}
