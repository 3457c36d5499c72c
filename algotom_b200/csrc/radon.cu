// Forward projection that is the exact adjoint of the back-projector.
//
// The back-projector (algotom/rec/reconstruction.py:156-190, 307-359) adds,
// for every angle i and pixel (y, x) whose detector position
// p = (x - ic) cos(-a_i) + (y - ic) sin(-a_i) + center lies in [0, ncol-1],
// (1 - f) s[i, d] + f s[i, d+1] with d = floor(p), f = p - d (f = 0 at the
// last bin).  As a matrix B: image <- sinogram its entries are these hat
// weights, so the adjoint B^T: sinogram <- image is
//     r[i, d] = sum over pixels of g(y, x) * max(0, 1 - |p_i(y, x) - d|)
// restricted to positions inside [0, ncol-1] (bin 0 takes no pixel with
// p < 0, bin ncol-1 none with p > ncol-1).
//
// Ray-driven gather.  A CTA owns 32 consecutive bins of one angle and one
// slice; its 8 warps split the walk along the image axis the ray crosses
// more steeply, and every lane is one bin.  For |cos| >= |sin| the walk
// goes down the rows y: bin d meets row y at x_d(y) = A_d + y r with
// r = -sin/cos, and only the (at most three) pixels within 1/|cos| of it
// carry weight.  Neighbouring lanes' x_d are 1/|cos| <= 1.42 pixels apart,
// so a warp reads one short contiguous run of a row per step.  For
// |sin| > |cos| the same walk runs over a transposed copy of the image
// (rows of the copy are image columns), made by transpose_kernel into the
// caller's workspace, so that reads stay contiguous there too.
//
// Positions: x_d(y) is anchored in FP64 every 32 rows and advanced in FP32
// inside the run (|offset| <= 32 pixels), so each weight carries ~1e-6 of a
// bin of position error, less than the back-projector's own FP32 in-tile
// offsets.  Sums: FP32 over each 32-row run, FP64 across runs and warps,
// added in a fixed order (the result does not depend on scheduling).
//
// Edge padding (BPF) is not part of this adjoint: a back-projection with
// edge padding would put the edge bins' weight on whole half-planes.
#include "common.cuh"

namespace {

constexpr int kBins = 32;       // detector bins per CTA (one per lane)
constexpr int kWalkWarps = 8;   // warps per CTA, each walks a share of the rows
constexpr int kRun = 32;        // rows between FP64 anchors

struct RadonArgs {
  const float *img;   // [ncol][nslice][ncol] (y, slice, x)
  long long irs, iss;
  const float *imgt;  // transposed copy [nslice][ncol x][ncol y], or null
  int nrow, nslice, ncol;
  const double2 *trig;
  double center;
  float *out;         // [nrow][nslice][ncol]
  long long ors, oss;
};

// floor(v) for |v| < 2^22: the round-down add leaves floor(v) in the low
// mantissa bits of 1.5 * 2^23 + floor(v)
__device__ __forceinline__ int floor_small(float v) {
  return __float_as_int(__fadd_rd(v, 12582912.0f)) - 0x4B400000;
}

__global__ void __launch_bounds__(256) transpose_kernel(const float *img, long long irs, long long iss, int ncol,
                                                        float *dst) {
  __shared__ float tile[32][33];
  const int ks = blockIdx.z;
  const int bx = blockIdx.x * 32, by = blockIdx.y * 32;
  const float *src = img + ks * iss;
  for (int r = threadIdx.y; r < 32; r += 8) {
    const int y = by + r, x = bx + threadIdx.x;
    if (y < ncol && x < ncol) tile[r][threadIdx.x] = __ldg(src + (long long)y * irs + x);
  }
  __syncthreads();
  float *d = dst + (long long)ks * ncol * ncol;
  for (int r = threadIdx.y; r < 32; r += 8) {
    const int x = bx + r, y = by + threadIdx.x;
    if (x < ncol && y < ncol) d[(long long)x * ncol + y] = tile[threadIdx.x][r];
  }
}

// Sum of one bin's weighted pixels over walk lines [v0, v1).  kEdge: the
// bin is 0 or ncol-1, where a pixel's inclusion depends on the side of the
// detector edge its position falls; positions within kEdgeTol bins of the
// edge are re-decided in FP64 with the reference's expression and rounding
// order, (x - ic) cos + (y - ic) sin + center, as the back-projector
// decides them, so that the two stay exact transposes at angles such as
// 90 degrees, where whole pixel rows sit ~1e-8 bins from the edge.
template <bool kEdge>
__device__ __forceinline__ double walk_bin(const float *src, long long rs, int v0, int v1, double A, double r,
                                           float cf, float spanf, int d, int ncol, bool rows, double c64,
                                           double s64, double center) {
  constexpr float kEdgeTol = 2e-3f;
  const float rf = (float)r;
  const double ic = 0.5 * (double)(ncol - 1);
  double acc = 0.0;
  const float c2 = 2.0f * cf, c3 = 3.0f * cf;
  for (int va = v0; va < v1; va += kRun) {
    const double X0 = fma((double)va, r, A);
    const double xid = floor(X0);
    const int xi = (int)xid;
    const float xf = (float)(X0 - xid);
    const int nrun = min(kRun, v1 - va);
    const float *line = src + (long long)va * rs;
    float run = 0.0f;
    if constexpr (!kEdge) {
      // a full run whose candidate pixels all lie inside the line: no
      // bounds logic, weights clamped at zero (a zero weight adds exactly 0,
      // the same sum as the checked loop below)
      const float xe = fmaf((float)(kRun - 1), rf, xf);  // xr is monotonic in j
      if (nrun == kRun && xi + floor_small(fminf(xf, xe) - spanf) + 1 >= 0 &&
          xi + floor_small(fmaxf(xf, xe) - spanf) + 3 <= ncol - 1) {
        const float *base = line + xi;
#pragma unroll 8
        for (int j = 0; j < kRun; ++j, base += rs) {
          const float xr = fmaf((float)j, rf, xf);
          const float tq = __fadd_rd(xr - spanf, 12582912.0f);
          const int xb = __float_as_int(tq) - 0x4B400000;
          const float d0 = (tq - 12582912.0f) - xr;  // floor(xr - span) - xr
          const float *px = base + xb;
          const float w1 = fmaxf(0.0f, 1.0f - fabsf(fmaf(d0, cf, cf)));
          const float w2 = fmaxf(0.0f, 1.0f - fabsf(fmaf(d0, cf, c2)));
          const float w3 = fmaxf(0.0f, 1.0f - fabsf(fmaf(d0, cf, c3)));
          run = fmaf(w1, __ldg(px + 1), run);
          run = fmaf(w2, __ldg(px + 2), run);
          run = fmaf(w3, __ldg(px + 3), run);
        }
        acc += (double)run;
        continue;
      }
    }
    for (int j = 0; j < nrun; ++j, line += rs) {
      const float xr = fmaf((float)j, rf, xf);
      const int xb = floor_small(xr - spanf);
#pragma unroll
      const float d0 = (float)xb - xr;
      for (int k = 1; k <= 3; ++k) {
        const float q = fmaf(d0, cf, (float)k * cf);  // p - d
        const float w = 1.0f - fabsf(q);
        const int x = xi + xb + k;
        bool in = w > 0.0f && x >= 0 && x < ncol;
        if constexpr (kEdge) {
          // bin 0 takes no p < 0, bin ncol-1 no p > ncol-1
          const bool low = d == 0;
          if (fabsf(q) < kEdgeTol) {
            const double xc = (double)(rows ? x : va + j) - ic;
            const double yc = (double)(rows ? va + j : x) - ic;
            const double pe = __dadd_rn(__dadd_rn(__dmul_rn(xc, c64), __dmul_rn(yc, s64)), center);
            in = in && (low ? pe >= 0.0 : pe <= (double)(ncol - 1));
          } else {
            in = in && (low ? q >= 0.0f : q <= 0.0f);
          }
        }
        if (in) run = fmaf(w, __ldg(line + x), run);
      }
    }
    acc += (double)run;
  }
  return acc;
}

__global__ void __launch_bounds__(kBins * kWalkWarps) radon_kernel(RadonArgs a) {
  __shared__ double part[kWalkWarps][kBins];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int i = blockIdx.y, ks = blockIdx.z;
  const int ncol = a.ncol;
  const int d = blockIdx.x * kBins + lane;
  const double2 cs = a.trig[i];
  // walk the rows of the image (|cos| >= |sin|) or of its transposed copy,
  // where the roles of cos and sin swap: p = (u - ic) sin + (v - ic) cos + c
  // for the copy's row v = x and column u = y
  const bool rows = fabs(cs.x) >= fabs(cs.y);
  const double cw = rows ? cs.x : cs.y;   // coefficient of the contiguous axis
  const double sw = rows ? cs.y : cs.x;   // coefficient of the walk axis
  const float *src;
  long long rs;
  if (rows) {
    src = a.img + ks * a.iss;
    rs = a.irs;
  } else {
    src = a.imgt + (long long)ks * ncol * ncol;
    rs = ncol;
  }
  const double ic = 0.5 * (double)(ncol - 1);
  const double inv = 1.0 / cw;
  const double r = -sw * inv;
  const double span = fabs(inv);
  // bin d meets walk line v at u = A + v r
  const double A = ((double)d - a.center + ic * sw) * inv + ic;
  const bool live = d < ncol;

  // walk lines where some lane's window [u - span, u + span] reaches
  // [0, ncol-1]; union over the CTA's bins, split evenly over the warps
  int vlo = ncol, vhi = -1;
  if (live) {
    if (r == 0.0) {
      if (A + span > 0.0 && A - span < (double)(ncol - 1)) {
        vlo = 0;
        vhi = ncol - 1;
      }
    } else {
      double t0 = (-span - A) / r, t1 = ((double)(ncol - 1) + span - A) / r;
      if (t0 > t1) {
        const double t = t0;
        t0 = t1;
        t1 = t;
      }
      t0 = fmax(floor(t0) - 1.0, 0.0);
      t1 = fmin(ceil(t1) + 1.0, (double)(ncol - 1));
      if (t0 <= t1) {
        vlo = (int)t0;
        vhi = (int)t1;
      }
    }
  }
  vlo = __reduce_min_sync(0xffffffffu, vlo);
  vhi = __reduce_max_sync(0xffffffffu, vhi);
  // every warp holds the same 32 bins, so every warp finds the same range
  const int nv = vhi - vlo + 1;
  double acc = 0.0;
  if (nv > 0 && live) {
    const int per = (nv + kWalkWarps - 1) / kWalkWarps;
    const int v0 = vlo + warp * per, v1 = min(vhi + 1, v0 + per);
    const float cf = (float)cw, spanf = (float)span;
    if (d == 0 || d == ncol - 1)
      acc = walk_bin<true>(src, rs, v0, v1, A, r, cf, spanf, d, ncol, rows, cs.x, cs.y, a.center);
    else
      acc = walk_bin<false>(src, rs, v0, v1, A, r, cf, spanf, d, ncol, rows, cs.x, cs.y, a.center);
  }
  part[warp][lane] = acc;
  __syncthreads();
  if (warp == 0 && live) {
    double sum = 0.0;
#pragma unroll
    for (int g = 0; g < kWalkWarps; ++g) sum += part[g][lane];
    a.out[i * a.ors + ks * a.oss + d] = (float)sum;
  }
}

}  // namespace

extern "C" int64_t atb_radon_workspace(int nslice, int ncol) {
  if (nslice < 1 || ncol < 1) return atb::fail(ATB_EINVAL, "atb_radon_workspace: bad shape");
  return (int64_t)nslice * ncol * ncol * (int64_t)sizeof(float);
}

extern "C" int atb_radon_adjoint(const float *img, int64_t img_row_stride, int64_t img_slice_stride, int nrow,
                                 int nslice, int ncol, const double *trig, double center, float *out,
                                 int64_t out_row_stride, int64_t out_slice_stride, void *workspace,
                                 int64_t workspace_bytes, void *stream) {
  if (!img || !trig || !out) return atb::fail(ATB_EINVAL, "atb_radon_adjoint: null pointer");
  if (nrow < 1 || nslice < 1 || ncol < 1)
    return atb::fail(ATB_EINVAL, "atb_radon_adjoint: bad shape nrow=%d nslice=%d ncol=%d", nrow, nslice, ncol);
  if (nrow > 65535 || nslice > 65535 || ncol > 1 << 20)
    return atb::fail(ATB_ERANGE, "atb_radon_adjoint: nrow=%d nslice=%d ncol=%d too large", nrow, nslice, ncol);
  if (!(center >= 0.0) || center >= (double)ncol)
    return atb::fail(ATB_EINVAL, "atb_radon_adjoint: center %g outside [0, %d)", center, ncol);
  const int64_t need = (int64_t)nslice * ncol * ncol * (int64_t)sizeof(float);
  if (!workspace || workspace_bytes < need)
    return atb::fail(ATB_EINVAL, "atb_radon_adjoint: workspace of %lld bytes needed (atb_radon_workspace)",
                     (long long)need);
  cudaStream_t st = atb::as_stream(stream);
  float *imgt = static_cast<float *>(workspace);
  const int tiles = (ncol + 31) / 32;
  transpose_kernel<<<dim3(tiles, tiles, nslice), dim3(32, 8), 0, st>>>(img, img_row_stride, img_slice_stride, ncol,
                                                                       imgt);
  int rc = atb::check_launch("atb_radon_adjoint (transpose)");
  if (rc != ATB_OK) return rc;
  RadonArgs a;
  a.img = img; a.irs = img_row_stride; a.iss = img_slice_stride;
  a.imgt = imgt;
  a.nrow = nrow; a.nslice = nslice; a.ncol = ncol;
  a.trig = reinterpret_cast<const double2 *>(trig);
  a.center = center;
  a.out = out; a.ors = out_row_stride; a.oss = out_slice_stride;
  radon_kernel<<<dim3((ncol + kBins - 1) / kBins, nrow, nslice), kBins * kWalkWarps, 0, st>>>(a);
  return atb::check_launch("atb_radon_adjoint");
}
