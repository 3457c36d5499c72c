// Forward projection that is the exact adjoint of the back-projector.
//
// The back-projector (algotom/rec/reconstruction.py:156-190, 307-359) adds,
// for every angle i and pixel (y, x) whose detector position
// p = (x - ic) cos(-a_i) + (y - ic) sin(-a_i) + center lies in [0, ncol-1],
// (1 - f) s[i, d] + f s[i, d+1] with d = floor(p), f = p - d (f = 0 at the
// last bin).  As a matrix B: image <- sinogram its entries are these hat
// weights, so the adjoint B^T: sinogram <- image is
//     r[i, d] = sum over pixels of g(y, x) * hat(p_i(y, x) - d)
// restricted to positions inside [0, ncol-1].  This kernel evaluates that
// sum ray by ray: one thread per (angle, detector bin, slice) walks the
// pixel rows (or columns, whichever axis the ray crosses more steeply) and
// visits the two or three pixels per row whose position lies within one bin
// of d.  Positions are formed in FP64 with the reference's expression, so
// the weights are those of the reference back-projector and the dot-product
// identity <B s, g> = <s, B^T g> holds to rounding.
//
// Edge padding (BPF) is not part of this adjoint: a back-projection with
// edge padding would put the edge bins' weight on whole half-planes.
#include "common.cuh"

namespace {

struct RadonArgs {
  const float *img;   // [ncol][nslice][ncol] (y, slice, x)
  long long irs, iss;
  int nrow, nslice, ncol;
  const double2 *trig;
  double center;
  float *out;         // [nrow][nslice][ncol]
  long long ors, oss;
};

__global__ void __launch_bounds__(256) radon_kernel(RadonArgs a) {
  const int ncol = a.ncol;
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const long long total = (long long)a.nrow * a.nslice * ncol;
  if (t >= total) return;
  const int d = (int)(t % ncol);
  const long long rest = t / ncol;
  const int ks = (int)(rest % a.nslice);
  const int i = (int)(rest / a.nslice);
  const double2 cs = a.trig[i];
  const double c = cs.x, s = cs.y;
  const double ic = 0.5 * (double)(ncol - 1);
  const double w1 = (double)(ncol - 1);
  const float *img = a.img + ks * a.iss;
  double acc = 0.0;
  // weight of a pixel at position p for bin d
  auto weight = [&](double p) -> double {
    if (!(p >= 0.0 && p <= w1)) return 0.0;
    const double fl = floor(p);
    const double f = p - fl;
    const int dl = (int)fl;
    if (dl == d) return 1.0 - f;
    if (dl == d - 1) return f;
    return 0.0;
  };
  if (fabs(c) >= fabs(s)) {
    // walk rows y: p is linear in x with slope c, |c| >= 1/sqrt(2)
    const double inv = 1.0 / c;
    for (int y = 0; y < ncol; ++y) {
      const double yc = (double)y - ic;
      const double ys = __dmul_rn(yc, s);
      // x where p = d: (d - center - ys) / c + ic; neighbours within 1/|c|
      const double xm = ((double)d - a.center - ys) * inv + ic;
      const double span = fabs(inv);
      int xa = (int)ceil(xm - span - 1e-9), xb = (int)floor(xm + span + 1e-9);
      xa = max(xa, 0);
      xb = min(xb, ncol - 1);
      for (int x = xa; x <= xb; ++x) {
        const double p = __dadd_rn(__dadd_rn(__dmul_rn((double)x - ic, c), ys), a.center);
        const double w = weight(p);
        if (w != 0.0) acc += w * (double)__ldg(img + y * a.irs + x);
      }
    }
  } else {
    // walk columns x: p is linear in y with slope s, |s| > 1/sqrt(2)
    const double inv = 1.0 / s;
    for (int x = 0; x < ncol; ++x) {
      const double xcc = __dmul_rn((double)x - ic, c);
      const double ym = ((double)d - a.center - xcc) * inv + ic;
      const double span = fabs(inv);
      int ya = (int)ceil(ym - span - 1e-9), yb = (int)floor(ym + span + 1e-9);
      ya = max(ya, 0);
      yb = min(yb, ncol - 1);
      for (int y = ya; y <= yb; ++y) {
        const double p = __dadd_rn(__dadd_rn(xcc, __dmul_rn((double)y - ic, s)), a.center);
        const double w = weight(p);
        if (w != 0.0) acc += w * (double)__ldg(img + y * a.irs + x);
      }
    }
  }
  a.out[i * a.ors + ks * a.oss + d] = (float)acc;
}

}  // namespace

extern "C" int atb_radon_adjoint(const float *img, int64_t img_row_stride, int64_t img_slice_stride, int nrow,
                                 int nslice, int ncol, const double *trig, double center, float *out,
                                 int64_t out_row_stride, int64_t out_slice_stride, void *stream) {
  if (!img || !trig || !out) return atb::fail(ATB_EINVAL, "atb_radon_adjoint: null pointer");
  if (nrow < 1 || nslice < 1 || ncol < 1)
    return atb::fail(ATB_EINVAL, "atb_radon_adjoint: bad shape nrow=%d nslice=%d ncol=%d", nrow, nslice, ncol);
  if (!(center >= 0.0) || center >= (double)ncol)
    return atb::fail(ATB_EINVAL, "atb_radon_adjoint: center %g outside [0, %d)", center, ncol);
  RadonArgs a;
  a.img = img; a.irs = img_row_stride; a.iss = img_slice_stride;
  a.nrow = nrow; a.nslice = nslice; a.ncol = ncol;
  a.trig = reinterpret_cast<const double2 *>(trig);
  a.center = center;
  a.out = out; a.ors = out_row_stride; a.oss = out_slice_stride;
  const long long total = (long long)nrow * nslice * ncol;
  const long long blocks = (total + 255) / 256;
  if (blocks > 0x7fffffffLL) return atb::fail(ATB_ERANGE, "atb_radon_adjoint: too large");
  radon_kernel<<<(unsigned)blocks, 256, 0, atb::as_stream(stream)>>>(a);
  return atb::check_launch("atb_radon_adjoint");
}
