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
// sum without FP32 rounding across chunks.  The grid runs all (line, point
// block) CTAs of one row block next to each other, so a row block's
// projection rows are read from HBM about once per launch however many
// lines share them.
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
  int edge_pad;
  double *acc;
  long long als, ars;  // accumulator line / row strides
};

// table entry: bin d and fraction f >= 0 (f == 0: the single sample y[d]),
// or f < 0: no contribution
struct __align__(8) VPos {
  int d;
  float f;
};

__global__ void __launch_bounds__(kThreads) vbp_kernel(VArgs a) {
  __shared__ VPos tab[kAng][kPts];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int line = blockIdx.x / a.npb, pb = blockIdx.x - line * a.npb;
  const int j0 = pb * kPts;
  const int pl = lane + 32 * (warp & 1);  // this thread's point in the block
  const int j = j0 + pl;
  const int r0 = blockIdx.y * kRows + (warp >> 1) * kRowsPerThread;
  const int width1 = a.width - 1;
  const double2 *pts = a.points + line * a.pls;
  double acc[kRowsPerThread];
#pragma unroll
  for (int r = 0; r < kRowsPerThread; ++r) acc[r] = 0.0;

  for (int n0 = 0; n0 < a.nproj; n0 += kAng) {
    const int nang = min(kAng, a.nproj - n0);
    __syncthreads();  // the previous table is no longer read
    for (int e = tid; e < kAng * kPts; e += kThreads) {
      const int an = e / kPts, pe = e - an * kPts, je = j0 + pe;
      VPos v = {0, -1.0f};
      if (an < nang && je < a.npts) {
        const double2 cs = a.trig[n0 + an];
        const double2 xy = pts[je];
        // same expression and rounding order as the reference:
        // (x cos + y sin) + center
        const double p = __dadd_rn(__dadd_rn(__dmul_rn(xy.x, cs.x), __dmul_rn(xy.y, cs.y)), a.center);
        if (p >= 0.0 && p <= (double)width1) {
          const double fl = floor(p);
          v.d = (int)fl;
          v.f = (float)(p - fl);  // exact difference; 0 when u == d
        } else if (a.edge_pad) {
          v.d = p < 0.0 ? 0 : width1;
          v.f = 0.0f;
        }
      }
      tab[an][pe] = v;
    }
    __syncthreads();
    if (j < a.npts) {
      // FP32 partial sums over this table's angles, folded into FP64 below
      float part[kRowsPerThread];
#pragma unroll
      for (int r = 0; r < kRowsPerThread; ++r) part[r] = 0.0f;
#pragma unroll 2
      for (int an = 0; an < nang; ++an) {
        const VPos v = tab[an][pl];
        if (v.f < 0.0f) continue;
        const int d1 = v.f > 0.0f ? v.d + 1 : v.d;
        const float *base = a.proj + (long long)(n0 + an) * a.ps;
#pragma unroll
        for (int r = 0; r < kRowsPerThread; ++r) {
          const int i = r0 + r;
          if (i < a.height) {
            const float *row = base + (long long)i * a.rs;
            const float y0 = __ldg(row + v.d), y1 = __ldg(row + d1);
            part[r] += y0 + (y1 - y0) * v.f;
          }
        }
      }
#pragma unroll
      for (int r = 0; r < kRowsPerThread; ++r) acc[r] += (double)part[r];
    }
  }
  if (j < a.npts) {
#pragma unroll
    for (int r = 0; r < kRowsPerThread; ++r) {
      const int i = r0 + r;
      if (i < a.height) a.acc[line * a.als + (long long)i * a.ars + j] += acc[r];
    }
  }
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

extern "C" int atb_vertical_backproject(const float *proj, int64_t proj_stride, int64_t row_stride, int nproj,
                                        int height, int width, const double *trig, const double *points,
                                        int64_t line_stride, int npts, int nline, double center, int edge_pad,
                                        double *acc, int64_t acc_line_stride, int64_t acc_row_stride,
                                        void *stream) {
  if (!proj || !trig || !points || !acc) return atb::fail(ATB_EINVAL, "atb_vertical_backproject: null pointer");
  if (nproj < 1 || height < 1 || width < 1 || npts < 1 || nline < 1)
    return atb::fail(ATB_EINVAL, "atb_vertical_backproject: bad shape nproj=%d height=%d width=%d npts=%d nline=%d",
                     nproj, height, width, npts, nline);
  const int npb = (npts + kPts - 1) / kPts, nrb = (height + kRows - 1) / kRows;
  if ((long long)npb * nline > 2147483647LL || nrb > 65535)
    return atb::fail(ATB_ERANGE, "atb_vertical_backproject: %d lines x %d points x %d rows too large", nline, npts,
                     height);
  if (!std::isfinite(center)) return atb::fail(ATB_EINVAL, "atb_vertical_backproject: center is not finite");
  VArgs a;
  a.proj = proj; a.ps = proj_stride; a.rs = row_stride;
  a.nproj = nproj; a.height = height; a.width = width;
  a.trig = reinterpret_cast<const double2 *>(trig);
  a.points = reinterpret_cast<const double2 *>(points);
  a.pls = line_stride; a.npts = npts; a.nline = nline; a.npb = npb;
  a.center = center; a.edge_pad = edge_pad ? 1 : 0;
  a.acc = acc; a.als = acc_line_stride; a.ars = acc_row_stride;
  vbp_kernel<<<dim3(npb * nline, nrb), kThreads, 0, atb::as_stream(stream)>>>(a);
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
