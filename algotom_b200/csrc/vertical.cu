// Vertical-slice back-projection, sm_100a: the gather of algotom's
// vertical_back_projection_{cpu,gpu}{,_chunk} (algotom/rec/vertrec.py:53-335)
// and the flat-field / -log pre-step of vertical_reconstruction*
// (vertrec.py:594-606).
//
// A vertical slice is a line of points (x_j, y_j) in the horizontal plane,
// reconstructed at every detector row i of the projections
// proj[n][i][0..width-1]:
//     ver[s][i][j] += sum_n value(proj[n][i], x_sj cos a_n + y_sj sin a_n + c)
// with the slice back-projector's interpolation: for 0 <= p <= width-1,
// d = floor(p), u = ceil(p), y[d] + (y[u] - y[d]) (p - d) (y[d] when u == d);
// outside, y[0] (p < 0) or y[width-1] with edge padding, else nothing.
//
// The position depends on (point, angle) only, not on the detector row, so
// a CTA (64 points x 32 rows) forms the positions of a chunk of 32 angles
// once, in FP64, into a shared-memory table of (bin, fraction) entries, and
// every thread reuses each entry for its 8 rows.  Samples are read through
// L1: a warp's 32 consecutive points touch a short run of bins of each row.
// Interpolation is FP32; the sums over each table's 32 angles are FP32
// partials, folded into FP64 registers and finally added to a caller FP64
// accumulator, so that chunks of projections streamed through the device
// sum without FP32 rounding across chunks.  When the tile grid alone would
// not fill the GPU, the angles are also split over CTAs (grid z): each group
// writes its FP64 partial sums to caller scratch and a second kernel adds
// the groups in a fixed order, so results do not depend on scheduling.  The
// grid runs all (line, point block) CTAs of one row block next to each
// other, so the lines resident together share a row block's projection
// rows through L2 (with 64 lines about 8 slices' CTAs fit at once, and the
// rows are read from HBM about 6 times rather than 64).
#include <cmath>

#include "common.cuh"

namespace {

constexpr int kPts = 64;      // points per CTA
constexpr int kRowsPerThread = 8;
constexpr int kRows = 4 * kRowsPerThread;  // rows per CTA (4 row groups)
constexpr int kAng = 32;      // angles per position table
constexpr int kThreads = 256;

struct VArgs {
  const float *proj;
  long long ps, rs;  // projection and row strides (elements)
  int nproj, height, width;
  const double2 *trig;    // (cos a, sin a) per projection
  const double2 *points;  // (x, y) per point, line-major
  long long pls;          // point stride between lines
  int npts, nline, npb;   // points per line, lines, point blocks per line
  double center;
  const double *line_centers;  // per-line centre, or null (all `center`)
  int edge_pad;
  double *acc;
  long long als, ars;  // accumulator line / row strides
  int apg;             // angles per group (blockIdx.z)
  double *part;        // group partials [ngroups][nline][height][npts], or null
};

// table entry of one (point, angle): the two taps d0 <= d1 (equal for a
// single sample), the fraction f, and live = 1 when the point receives a
// value (else 0: d0 = d1 = 0 keeps the reads in bounds and the value is
// discarded by a select, so no NaN or inf sample can leak in)
struct __align__(16) VPos {
  int d0, d1;
  float f, live;
};

__device__ __forceinline__ VPos make_pos(const VArgs &a, const double2 *pts, int n, int je, double center) {
  VPos v = {0, 0, 0.0f, 0.0f};
  const double2 cs = a.trig[n];
  const double2 xy = pts[je];
  // same expression and rounding order as the reference: (x cos + y sin) + center
  const double p = __dadd_rn(__dadd_rn(__dmul_rn(xy.x, cs.x), __dmul_rn(xy.y, cs.y)), center);
  const int width1 = a.width - 1;
  if (p >= 0.0 && p <= (double)width1) {
    const double fl = floor(p);
    v.d0 = (int)fl;
    v.f = (float)(p - fl);  // exact difference; 0 when ceil(p) == floor(p)
    v.d1 = v.f > 0.0f ? v.d0 + 1 : v.d0;
    v.live = 1.0f;
  } else if (a.edge_pad) {
    v.d0 = v.d1 = p < 0.0 ? 0 : width1;
    v.live = 1.0f;
  }
  return v;
}

// the angles [0, nang) of the current table for this thread's rows; kFull:
// all kRowsPerThread rows exist (no predicates)
template <bool kFull>
__device__ __forceinline__ void accumulate(const VPos (*tab)[kPts], int pl, int nang, const float *base,
                                           long long ps, const int *roff, int nr, float *part) {
  int an = 0;
  for (; an + 1 < nang; an += 2, base += 2 * ps) {
    // both angles' samples are requested before any is used
    const VPos v0 = tab[an][pl], v1 = tab[an + 1][pl];
    const float *b1 = base + ps;
    float y[2][kRowsPerThread][2];
#pragma unroll
    for (int r = 0; r < kRowsPerThread; ++r) {
      if (kFull || r < nr) {
        y[0][r][0] = __ldg(base + roff[r] + v0.d0);
        y[0][r][1] = __ldg(base + roff[r] + v0.d1);
        y[1][r][0] = __ldg(b1 + roff[r] + v1.d0);
        y[1][r][1] = __ldg(b1 + roff[r] + v1.d1);
      }
    }
#pragma unroll
    for (int r = 0; r < kRowsPerThread; ++r) {
      if (kFull || r < nr) {
        const float a0 = y[0][r][0] + (y[0][r][1] - y[0][r][0]) * v0.f;
        const float a1 = y[1][r][0] + (y[1][r][1] - y[1][r][0]) * v1.f;
        part[r] += (v0.live != 0.0f ? a0 : 0.0f) + (v1.live != 0.0f ? a1 : 0.0f);
      }
    }
  }
  if (an < nang) {
    const VPos v0 = tab[an][pl];
#pragma unroll
    for (int r = 0; r < kRowsPerThread; ++r) {
      if (kFull || r < nr) {
        const float y0 = __ldg(base + roff[r] + v0.d0), y1 = __ldg(base + roff[r] + v0.d1);
        const float a0 = y0 + (y1 - y0) * v0.f;
        part[r] += v0.live != 0.0f ? a0 : 0.0f;
      }
    }
  }
}

__global__ void __launch_bounds__(kThreads, 2) vbp_kernel(VArgs a) {
  __shared__ VPos tab[kAng][kPts];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int line = blockIdx.x / a.npb, pb = blockIdx.x - line * a.npb;
  const int j0 = pb * kPts;
  const int pl = lane + 32 * (warp & 1);  // this thread's point in the block
  const int j = j0 + pl;
  const int r0 = blockIdx.y * kRows + (warp >> 1) * kRowsPerThread;
  const int nr = min(kRowsPerThread, a.height - r0);  // live rows (may be <= 0)
  const double2 *pts = a.points + line * a.pls;
  const double center = a.line_centers ? a.line_centers[line] : a.center;
  const int g0 = blockIdx.z * a.apg, g1 = min(a.nproj, g0 + a.apg);
  // 32-bit row offsets: one projection holds fewer than 2^31 samples
  int roff[kRowsPerThread];
#pragma unroll
  for (int r = 0; r < kRowsPerThread; ++r) roff[r] = r < nr ? (r0 + r) * (int)a.rs : 0;
  double acc[kRowsPerThread];
#pragma unroll
  for (int r = 0; r < kRowsPerThread; ++r) acc[r] = 0.0;

  for (int n0 = g0; n0 < g1; n0 += kAng) {
    const int nang = min(kAng, g1 - n0);
    __syncthreads();  // the previous table is no longer read
    for (int e = tid; e < kAng * kPts; e += kThreads) {
      const int an = e / kPts, pe = e - an * kPts, je = j0 + pe;
      tab[an][pe] = (an < nang && je < a.npts) ? make_pos(a, pts, n0 + an, je, center) : VPos{0, 0, 0.0f, 0.0f};
    }
    __syncthreads();
    if (j < a.npts && nr > 0) {
      // FP32 partial sums over this table's angles, folded into FP64 below
      float part[kRowsPerThread];
#pragma unroll
      for (int r = 0; r < kRowsPerThread; ++r) part[r] = 0.0f;
      const float *base = a.proj + (long long)n0 * a.ps;
      if (nr == kRowsPerThread)
        accumulate<true>(tab, pl, nang, base, a.ps, roff, nr, part);
      else
        accumulate<false>(tab, pl, nang, base, a.ps, roff, nr, part);
#pragma unroll
      for (int r = 0; r < kRowsPerThread; ++r) acc[r] += (double)part[r];
    }
  }
  if (j < a.npts) {
#pragma unroll
    for (int r = 0; r < kRowsPerThread; ++r) {
      if (r < nr) {
        const long long i = r0 + r;
        if (a.part)
          a.part[((long long)blockIdx.z * a.nline + line) * a.height * (long long)a.npts + i * a.npts + j] = acc[r];
        else
          a.acc[line * a.als + i * a.ars + j] += acc[r];
      }
    }
  }
}

// acc += the angle groups' partial sums, added in group order
__global__ void vbp_reduce_kernel(const double *__restrict__ part, int ngroups, int nline, int height, int npts,
                                  double *acc, long long als, long long ars) {
  const long long total = (long long)nline * height * npts;
  const long long gs = total;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const int j = (int)(e % npts);
    const long long t = e / npts;
    const int i = (int)(t % height), line = (int)(t / height);
    double s = 0.0;
    for (int g = 0; g < ngroups; ++g) s += part[g * gs + e];
    acc[line * als + (long long)i * ars + j] += s;
  }
}

// angle groups for a launch of `base` CTAs: enough for about 1776 CTAs
// (six waves of 2 CTAs per SM), at least one 32-angle table per group
int vbp_groups(int nproj, long long base) {
  const long long want = 4LL * 148 * 3;
  long long g = (want + base - 1) / base;
  const long long gmax = (nproj + kAng - 1) / kAng;
  if (g > gmax) g = gmax;
  return (int)(g < 1 ? 1 : g);
}

// dst = -log((src - dark) / flat_dark) with the reference's <= 0 -> 1
// replacement; counts the replaced values in *nonpos
template <typename T>
__global__ void flat_log_kernel(const T *__restrict__ src, long long sps, long long srs, int nproj, int height,
                                int width, const float *__restrict__ dark, const float *__restrict__ flat_dark,
                                long long frs, int apply_log, float *__restrict__ dst, long long dps, long long drs,
                                unsigned *nonpos) {
  const long long total = (long long)nproj * height * width;
  unsigned bad = 0;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const int c = (int)(e % width);
    const long long t = e / width;
    const int i = (int)(t % height), n = (int)(t / height);
    float v = atb::to_float(src[n * sps + i * srs + c]);
    if (flat_dark) v = __fdiv_rn(__fsub_rn(v, dark[i * frs + c]), flat_dark[i * frs + c]);
    if (apply_log) {
      if (v <= 0.0f) {
        ++bad;
        v = 1.0f;
      }
      v = -logf(v);
    }
    dst[n * dps + i * drs + c] = v;
  }
  for (int o = 16; o > 0; o >>= 1) bad += __shfl_xor_sync(0xffffffffu, bad, o);
  if ((threadIdx.x & 31) == 0 && bad) atomicAdd(nonpos, bad);
}

}  // namespace

extern "C" int64_t atb_vertical_workspace(int nproj, int height, int npts, int nline) {
  if (nproj < 1 || height < 1 || npts < 1 || nline < 1) return 0;
  const long long base = (long long)((npts + kPts - 1) / kPts) * nline * ((height + kRows - 1) / kRows);
  const int g = vbp_groups(nproj, base);
  return g > 1 ? (int64_t)g * nline * height * (int64_t)npts * (int64_t)sizeof(double) : 0;
}

extern "C" int atb_vertical_backproject(const float *proj, int64_t proj_stride, int64_t row_stride, int nproj,
                                        int height, int width, const double *trig, const double *points,
                                        int64_t line_stride, int npts, int nline, double center,
                                        const double *line_centers, int edge_pad, double *acc,
                                        int64_t acc_line_stride, int64_t acc_row_stride, void *work,
                                        int64_t work_bytes, void *stream) {
  if (!proj || !trig || !points || !acc) return atb::fail(ATB_EINVAL, "atb_vertical_backproject: null pointer");
  if (nproj < 1 || height < 1 || width < 1 || npts < 1 || nline < 1)
    return atb::fail(ATB_EINVAL, "atb_vertical_backproject: bad shape nproj=%d height=%d width=%d npts=%d nline=%d",
                     nproj, height, width, npts, nline);
  const int npb = (npts + kPts - 1) / kPts, nrb = (height + kRows - 1) / kRows;
  if ((long long)npb * nline > 2147483647LL || nrb > 65535)
    return atb::fail(ATB_ERANGE, "atb_vertical_backproject: %d lines x %d points x %d rows too large", nline, npts,
                     height);
  if ((long long)height * row_stride > 2147483647LL)
    return atb::fail(ATB_ERANGE, "atb_vertical_backproject: one projection spans more than 2^31 samples");
  if (!std::isfinite(center)) return atb::fail(ATB_EINVAL, "atb_vertical_backproject: center is not finite");
  VArgs a;
  a.proj = proj; a.ps = proj_stride; a.rs = row_stride;
  a.nproj = nproj; a.height = height; a.width = width;
  a.trig = reinterpret_cast<const double2 *>(trig);
  a.points = reinterpret_cast<const double2 *>(points);
  a.pls = line_stride; a.npts = npts; a.nline = nline; a.npb = npb;
  a.center = center; a.line_centers = line_centers; a.edge_pad = edge_pad ? 1 : 0;
  a.acc = acc; a.als = acc_line_stride; a.ars = acc_row_stride;
  // split the angles over CTAs when the caller's scratch holds the partials
  const long long elems = (long long)nline * height * npts;
  int g = vbp_groups(nproj, (long long)npb * nline * nrb);
  if (work == nullptr) g = 1;
  while (g > 1 && (long long)g * elems * (long long)sizeof(double) > work_bytes) --g;
  if (g > 65535) g = 65535;
  a.apg = (nproj + g - 1) / g;
  g = (nproj + a.apg - 1) / a.apg;
  a.part = g > 1 ? static_cast<double *>(work) : nullptr;
  cudaStream_t st = atb::as_stream(stream);
  vbp_kernel<<<dim3(npb * nline, nrb, g), kThreads, 0, st>>>(a);
  int rc = atb::check_launch("atb_vertical_backproject");
  if (rc != ATB_OK || g == 1) return rc;
  long long blocks = (elems + 255) / 256;
  if (blocks > 148LL * 8) blocks = 148LL * 8;
  vbp_reduce_kernel<<<(int)blocks, 256, 0, st>>>(a.part, g, nline, height, npts, acc, acc_line_stride,
                                                  acc_row_stride);
  return atb::check_launch("atb_vertical_backproject");
}

extern "C" int atb_flat_log(const void *src, int src_dtype, int64_t src_proj_stride, int64_t src_row_stride,
                            int nproj, int height, int width, const float *dark, const float *flat_dark,
                            int64_t field_row_stride, int apply_log, float *dst, int64_t dst_proj_stride,
                            int64_t dst_row_stride, unsigned *nonpos, void *stream) {
  if (!src || !dst || !nonpos) return atb::fail(ATB_EINVAL, "atb_flat_log: null pointer");
  if ((dark == nullptr) != (flat_dark == nullptr))
    return atb::fail(ATB_EINVAL, "atb_flat_log: dark and flat_dark go together");
  if (nproj < 1 || height < 1 || width < 1)
    return atb::fail(ATB_EINVAL, "atb_flat_log: bad shape nproj=%d height=%d width=%d", nproj, height, width);
  cudaStream_t st = atb::as_stream(stream);
  const long long total = (long long)nproj * height * width;
  long long blocks = (total + 255) / 256;
  if (blocks > 148LL * 16) blocks = 148LL * 16;
  switch (src_dtype) {
    case ATB_F32:
      flat_log_kernel<float><<<(int)blocks, 256, 0, st>>>(static_cast<const float *>(src), src_proj_stride,
                                                         src_row_stride, nproj, height, width, dark, flat_dark,
                                                         field_row_stride, apply_log, dst, dst_proj_stride,
                                                         dst_row_stride, nonpos);
      break;
    case ATB_U16:
      flat_log_kernel<unsigned short><<<(int)blocks, 256, 0, st>>>(
          static_cast<const unsigned short *>(src), src_proj_stride, src_row_stride, nproj, height, width, dark,
          flat_dark, field_row_stride, apply_log, dst, dst_proj_stride, dst_row_stride, nonpos);
      break;
    default:
      return atb::fail(ATB_EINVAL, "atb_flat_log: unsupported src_dtype %d", src_dtype);
  }
  return atb::check_launch("atb_flat_log");
}
