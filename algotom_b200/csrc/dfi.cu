// Direct Fourier inversion (DFI), sm_100a: the B-spline prefilter and the
// polar-to-Cartesian regridding of algotom's dfi_reconstruction
// (algotom/rec/reconstruction.py:687-907).  The row transform of the
// sinogram and the inverse 2-D transform of the regridded spectrum are
// library FFTs; these two kernels are the rest.
//
// - atb_spline_prefilter: B-spline coefficients (order 3 or 5) of many
//   strided lines in place, real or interleaved complex, one thread per line:
//   the published recursive filter -- gain prod (1 - z)(1 - 1/z), then per
//   pole a causal pass and an anti-causal pass -- with the start values of
//   the half-sample symmetric extension ("reflect": scipy's "reflect" and,
//   after 12 edge samples of padding, "nearest") or of the whole-sample
//   symmetric one ("mirror": scipy's "mirror" and "wrap").
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

constexpr int kLineThreads = 128;
constexpr int kGridThreads = 256;

__device__ __forceinline__ double pole(int order, int k) {
  if (order == 3) return sqrt(3.0) - 2.0;
  const double a = sqrt(17745.0 / 4.0), b = sqrt(105.0 / 4.0);
  return k == 0 ? sqrt(135.0 / 2.0 - a) + b - 13.0 / 2.0 : sqrt(135.0 / 2.0 + a) - b - 13.0 / 2.0;
}

__global__ void __launch_bounds__(kLineThreads)
    prefilter_kernel(double *data, long long line_stride, long long es, int nlines, int ncomp, int n, int order,
                     int boundary) {
  const int line = blockIdx.x * kLineThreads + threadIdx.x;
  if (line >= nlines * ncomp) return;
  double *c = data + (long long)(line / ncomp) * line_stride + (line % ncomp);
  const int npoles = order == 5 ? 2 : 1;
  double gain = 1.0;
  for (int k = 0; k < npoles; ++k) {
    const double z = pole(order, k);
    gain = __dmul_rn(gain, __dmul_rn(1.0 - z, 1.0 - 1.0 / z));
  }
  for (int i = 0; i < n; ++i) c[i * es] = __dmul_rn(c[i * es], gain);
  if (n == 1) return;
  for (int k = 0; k < npoles; ++k) {
    const double z = pole(order, k);
    // causal start value
    double s, z_i = z;
    if (boundary == 0) {  // half-sample symmetric
      const double z_n = pow(z, (double)n), c0 = c[0];
      s = __dadd_rn(c[0], __dmul_rn(z_n, c[(n - 1) * es]));
      for (int i = 1; i < n; ++i) {
        s = __dadd_rn(s, __dmul_rn(z_i, __dadd_rn(c[i * es], __dmul_rn(z_n, c[(n - 1 - i) * es]))));
        z_i = __dmul_rn(z_i, z);
      }
      c[0] = __dadd_rn(__dmul_rn(s, z / (1.0 - __dmul_rn(z_n, z_n))), c0);
    } else {  // whole-sample symmetric
      const double z_n1 = pow(z, (double)(n - 1));
      s = __dadd_rn(c[0], __dmul_rn(z_n1, c[(n - 1) * es]));
      for (int i = 1; i < n - 1; ++i) {
        s = __dadd_rn(s, __dmul_rn(z_i, __dadd_rn(c[i * es], __dmul_rn(z_n1, c[(n - 1 - i) * es]))));
        z_i = __dmul_rn(z_i, z);
      }
      c[0] = s / (1.0 - __dmul_rn(z_n1, z_n1));
    }
    for (int i = 1; i < n; ++i) c[i * es] = __dadd_rn(c[i * es], __dmul_rn(z, c[(i - 1) * es]));
    // anti-causal start value
    if (boundary == 0)
      c[(n - 1) * es] = __dmul_rn(c[(n - 1) * es], z / (z - 1.0));
    else
      c[(n - 1) * es] =
          __dmul_rn(__dadd_rn(__dmul_rn(z, c[(n - 2) * es]), c[(n - 1) * es]), z / (__dmul_rn(z, z) - 1.0));
    for (int i = n - 2; i >= 0; --i) c[i * es] = __dmul_rn(z, __dsub_rn(c[(i + 1) * es], c[i * es]));
  }
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

extern "C" int atb_spline_prefilter(double *data, int64_t line_stride, int64_t elem_stride, int nlines, int ncomp,
                                    int n, int order, int boundary, void *stream) {
  if (!data) return atb::fail(ATB_EINVAL, "atb_spline_prefilter: null pointer");
  if (nlines < 1 || n < 1 || (ncomp != 1 && ncomp != 2))
    return atb::fail(ATB_EINVAL, "atb_spline_prefilter: bad shape nlines=%d n=%d ncomp=%d", nlines, n, ncomp);
  if ((order != 3 && order != 5) || (boundary != 0 && boundary != 1))
    return atb::fail(ATB_EINVAL, "atb_spline_prefilter: order %d / boundary %d unsupported", order, boundary);
  const long long lines = (long long)nlines * ncomp;
  const long long blocks = (lines + kLineThreads - 1) / kLineThreads;
  if (blocks > 2147483647LL) return atb::fail(ATB_ERANGE, "atb_spline_prefilter: too many lines");
  prefilter_kernel<<<(int)blocks, kLineThreads, 0, atb::as_stream(stream)>>>(data, line_stride, elem_stride, nlines,
                                                                             ncomp, n, order, boundary);
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
