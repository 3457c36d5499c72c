// One point of DFI's polar-to-Cartesian regridding (shared by
// atb_dfi_regrid and the inverse transform that regrids its rows on the
// fly, so both compute the same values bit for bit).
//
// For Cartesian frequency (i, j) of the w x w grid: the unit-circle mask
// of make_circle_mask(w, 1.0) (algotom/util/utility.py, integer grid
// centred at w // 2), the polar coordinates of generate_mapping_coordinate
// (algotom/rec/reconstruction.py:687-728, height_rec = width_rec =
// width_sino = w: radius clipped to floor((w - 1) / 2), the half plane
// folded by the Hermitian symmetry of a real image's spectrum, angle
// scaled to the sinogram's rows, both rounded to float32 as the reference's
// maps are), then map_coordinates(order=5, mode="reflect") of the complex
// row spectra: 6 x 6 quintic B-spline taps of the coefficients with
// half-sample symmetric indices.  FP64.
#pragma once

#include <cmath>

namespace atb {
namespace dfi {

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

// coef: complex B-spline coefficients [nrow][w], rows crs double2 apart
__device__ __forceinline__ double2 regrid_point(const double2 *__restrict__ coef, long long crs, int nrow, int w,
                                                int i, int j) {
  const long long cm = w / 2, dx = j - cm, dy = i - cm;
  if (dx * dx + dy * dy > cm * cm) return make_double2(0.0, 0.0);
  const double xc = (w - 1.0) * 0.5;
  const double rmax = floor(xc);
  const double x = (double)(w - 1 - j) - xc, y = (double)i - xc;
  float r = (float)fmin(fmax(sqrt(x * x + y * y), 0.0), rmax);
  double th = M_PI + atan2(y, x);
  if (th > M_PI) r = -r;
  r = (float)fmin(fmax((double)r + rmax, 0.0), (double)(w - 1));
  if (th > M_PI) th -= M_PI;
  const float tf = (float)(th * (nrow - 1.0) / M_PI);
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
    const double2 *row = coef + (long long)ir[a] * crs;
    double sr = 0.0, si = 0.0;
#pragma unroll
    for (int b = 0; b < 6; ++b) {
      const double2 v = __ldg(row + ic[b]);
      sr += wc[b] * v.x;
      si += wc[b] * v.y;
    }
    re += wr[a] * sr;
    im += wr[a] * si;
  }
  return make_double2(re, im);
}

}  // namespace dfi
}  // namespace atb
