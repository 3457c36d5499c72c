// Direct Fourier inversion (DFI), sm_100a: the B-spline prefilter and the
// polar-to-Cartesian regridding of algotom's dfi_reconstruction
// (algotom/rec/reconstruction.py:687-907).  The row transform of the
// sinogram and the inverse 2-D transform of the regridded spectrum are
// library FFTs; these two kernels are the rest.
//
// - atb_spline_prefilter: B-spline coefficients (order 3 or 5) of many
//   strided lines, real or interleaved complex.  The published recursive
//   filter (gain prod (1 - z)(1 - 1/z), per pole a causal and an anti-causal
//   pass, start values of the symmetric extension) is linear and
//   shift-invariant on the symmetric extension of the line, so it equals the
//   convolution of that extension with its symmetric impulse response, which
//   decays as |z1|^|k| (0.43^|k| for the quintic, 0.27^|k| for the cubic).
//   The kernel applies it as a 2 x 48 (2 x 32) tap FIR, one thread per
//   output sample -- exact to below 1e-17 relative, and fully parallel where
//   the recursion is a serial chain along each line.  Extension: half-sample
//   symmetric ("reflect": scipy's "reflect" and, after 12 edge samples of
//   padding, "nearest") or whole-sample symmetric ("mirror": scipy's
//   "mirror" and "wrap").
// - atb_dfi_regrid: for every pixel of the W x W Cartesian frequency grid,
//   the polar coordinates of generate_mapping_coordinate
//   (reconstruction.py:687-728: radius clipped to floor((W-1)/2), the half
//   plane folded by the Hermitian symmetry of a real image's spectrum, angle
//   scaled to the sinogram's rows), then the quintic B-spline interpolation
//   of the complex row spectra at that point with half-sample symmetric
//   taps (map_coordinates(order=5, mode="reflect")), times the unit circle
//   mask of make_circle_mask(W, 1.0).  FP64 throughout.
#include <cmath>

#include "common.cuh"

namespace {

constexpr int kFirThreads = 256;
constexpr int kGridThreads = 256;
constexpr int kMaxTaps = 48;  // |z1|^48 < 1e-17 for the quintic spline

struct Taps {
  double h[kMaxTaps + 1];  // symmetric impulse response h[|k|], k <= ntaps
  int ntaps;
};

double host_pole(int order, int k) {
  if (order == 3) return std::sqrt(3.0) - 2.0;
  const double a = std::sqrt(17745.0 / 4.0), b = std::sqrt(105.0 / 4.0);
  return k == 0 ? std::sqrt(135.0 / 2.0 - a) + b - 13.0 / 2.0 : std::sqrt(135.0 / 2.0 + a) - b - 13.0 / 2.0;
}

// Impulse response of the B-spline prefilter (gain, then per pole a causal
// and an anti-causal pass), from the recursion run on a unit impulse in the
// middle of a long zero line: the ends are 2 kMaxTaps samples away, where
// the response has decayed below 1e-34.
Taps make_taps(int order) {
  constexpr int kLen = 4 * kMaxTaps + 1, kMid = 2 * kMaxTaps;
  double c[kLen] = {0.0};
  c[kMid] = 1.0;
  const int npoles = order == 5 ? 2 : 1;
  double gain = 1.0;
  for (int k = 0; k < npoles; ++k) {
    const double z = host_pole(order, k);
    gain *= (1.0 - z) * (1.0 - 1.0 / z);
  }
  for (double &v : c) v *= gain;
  for (int k = 0; k < npoles; ++k) {
    const double z = host_pole(order, k);
    for (int i = 1; i < kLen; ++i) c[i] += z * c[i - 1];
    c[kLen - 1] *= z / (z - 1.0);
    for (int i = kLen - 2; i >= 0; --i) c[i] = z * (c[i + 1] - c[i]);
  }
  Taps t;
  t.ntaps = order == 5 ? kMaxTaps : 32;  // |z|^32 < 1e-18 for the cubic
  for (int k = 0; k <= kMaxTaps; ++k) t.h[k] = c[kMid + k];
  return t;
}

// index of sample i of a line of n under the symmetric extension
// (boundary 0: half-sample "reflect", 1: whole-sample "mirror")
__device__ __forceinline__ int sym_index(int i, int n, int boundary) {
  if (i >= 0 && i < n) return i;  // inside: no remainder
  if (boundary == 0) {
    const int p = 2 * n;
    int r = i % p;
    if (r < 0) r += p;
    return r >= n ? p - 1 - r : r;
  }
  if (n == 1) return 0;
  const int p = 2 * (n - 1);
  int r = i % p;
  if (r < 0) r += p;
  return r >= n ? p - r : r;
}

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

// centred quintic B-spline
__device__ __forceinline__ double bspline5(double u) {
  const double a = fabs(u);
  if (a < 1.0) {
    const double a2 = a * a;
    return 11.0 / 20.0 - a2 / 2.0 + a2 * a2 / 4.0 - a2 * a2 * a / 12.0;
  }
  if (a < 2.0) {
    const double a2 = a * a;
    return 17.0 / 40.0 + 5.0 * a / 8.0 - 7.0 * a2 / 4.0 + 5.0 * a2 * a / 4.0 - 3.0 * a2 * a2 / 8.0 +
           a2 * a2 * a / 24.0;
  }
  if (a < 3.0) {
    const double b = 3.0 - a, b2 = b * b;
    return b2 * b2 * b / 120.0;
  }
  return 0.0;
}

// half-sample symmetric index
__device__ __forceinline__ int reflect_index(int i, int n) {
  if (i >= 0 && i < n) return i;
  const int p = 2 * n;
  int r = i % p;
  if (r < 0) r += p;
  return r >= n ? p - 1 - r : r;
}

__global__ void __launch_bounds__(kGridThreads)
    regrid_kernel(const double2 *__restrict__ coef, int nrow, int w, double2 *__restrict__ out) {
  const long long e = blockIdx.x * (long long)kGridThreads + threadIdx.x;
  if (e >= (long long)w * w) return;
  const int i = (int)(e / w), j = (int)(e - (long long)i * w);
  // circle mask of make_circle_mask(w, 1.0): integer grid centred at w // 2
  const long long cm = w / 2, dx = j - cm, dy = i - cm;
  if (dx * dx + dy * dy > cm * cm) {
    out[e] = make_double2(0.0, 0.0);
    return;
  }
  // generate_mapping_coordinate (height_rec = width_rec = width_sino = w)
  const double xc = (w - 1.0) * 0.5;
  const double rmax = floor(xc);
  const double x = (double)(w - 1 - j) - xc, y = (double)i - xc;
  float r = (float)fmin(fmax(sqrt(x * x + y * y), 0.0), rmax);
  double th = M_PI + atan2(y, x);
  if (th > M_PI) r = -r;
  r = (float)fmin(fmax((double)r + rmax, 0.0), (double)(w - 1));
  if (th > M_PI) th -= M_PI;
  const float tf = (float)(th * (nrow - 1.0) / M_PI);
  // quintic B-spline interpolation at (row tf, column r)
  const double rr = (double)tf, cc = (double)r;
  const int fr = (int)floor(rr) - 2, fc = (int)floor(cc) - 2;
  double wr[6], wc[6];
  int ir[6], ic[6];
#pragma unroll
  for (int m = 0; m < 6; ++m) {
    wr[m] = bspline5(rr - (fr + m));
    wc[m] = bspline5(cc - (fc + m));
    ir[m] = reflect_index(fr + m, nrow);
    ic[m] = reflect_index(fc + m, w);
  }
  double re = 0.0, im = 0.0;
#pragma unroll
  for (int a = 0; a < 6; ++a) {
    const double2 *row = coef + (long long)ir[a] * w;
    double sr = 0.0, si = 0.0;
#pragma unroll
    for (int b = 0; b < 6; ++b) {
      const double2 v = row[ic[b]];
      sr += wc[b] * v.x;
      si += wc[b] * v.y;
    }
    re += wr[a] * sr;
    im += wr[a] * si;
  }
  out[e] = make_double2(re, im);
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
  const long long total = (long long)nlines * ncomp * n;
  const long long blocks = (total + kFirThreads - 1) / kFirThreads;
  if (blocks > 2147483647LL) return atb::fail(ATB_ERANGE, "atb_spline_prefilter: too many samples");
  prefilter_kernel<<<(int)blocks, kFirThreads, 0, atb::as_stream(stream)>>>(
      src, dst, line_stride, elem_stride, nlines, ncomp, n, boundary, order == 5 ? taps5 : taps3);
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
