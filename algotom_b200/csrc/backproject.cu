// Linear-interpolation back-projection (pixel-driven gather), sm_100a.
//
// Same mathematics as algotom's back-projectors
// (algotom/rec/reconstruction.py:156-190, 229-264, 307-359): pixel (y, x)
// of an ncol x ncol slice reads detector position
//     p = (x - ic) cos(-a) + (y - ic) sin(-a) + center,  ic = (ncol - 1) / 2
// and adds s[d] + (s[d+1] - s[d]) (p - d), d = floor(p), when
// 0 <= p <= ncol - 1; outside it adds nothing, or with edge padding the
// nearest edge sample.
//
// Work decomposition.  A CTA of 256 threads owns a 64 x 64 pixel tile of one
// slice and walks the angles in chunks of kChunk.  For every angle of a chunk
// the tile only sees detector bins [lo, lo + kWin) (its footprint is at most
// 63 (|cos| + |sin|) + 2 < 92 bins wide), so the CTA stages just that window
// into shared memory, as interpolation pairs
//     (a_j, D_j) = (s[lo+j] - (j-H) D_j, s[lo+j+1] - s[lo+j]),  H = kWin/2
// so that the value at the window-centred local position q = p - lo - H,
// bin j = floor(q) + H, is the single FMA a_j + D_j q.  Centring keeps |q|
// and |j-H| below 48, which bounds the rounding of both terms.  Bins outside the detector hold (0, 0) (or the edge
// value with D = 0 when edge padding), which reproduces the reference's
// bounds exactly wherever the interpolant is continuous.  The two detector
// edges of FBP (no edge padding) are discontinuities: positions just inside
// count, positions just outside add nothing.  Angles whose tile footprint
// reaches either edge take a checked path (a CTA-uniform branch) that tests
// every position against both edges and re-decides, in FP64 with the
// reference's own expression, any position within 2e-3 bins of an edge --
// e.g. at 90 degrees whole pixel rows sit 1e-8 bins from position 0, which
// no FP32 local coordinate can resolve.
//
// Positions: the tile-origin position is formed in FP64 per (tile, angle)
// from FP64 trigonometry of the float32-rounded angle; inside the tile each
// thread adds its small offset in FP32, so q is accurate to ~1e-5 bins.
// floor(q) is taken with one round-down add of 1.5 * 2^23, whose bit pattern
// is the shared-memory index.
//
// Accumulation: FP32 partial sums over each chunk of angles, added across
// chunks with Kahan compensation (flag bit 0 switches to per-angle Kahan).
// Each thread holds 4 x 4 pixels laid out so that one warp instruction
// covers an 8 x 4 pixel block: its 32 lanes read a compact run of <= 12
// neighbouring pairs, which shared memory serves without bank conflicts.
#include "common.cuh"

namespace {

constexpr int kThreads = 256;
constexpr int kTile = 64;   // tile edge (pixels)
constexpr int kChunk = 32;  // angles per staged chunk
constexpr int kWin = 96;    // staged pairs per angle (>= 63 sqrt(2) + 4)
constexpr int kHalf = kWin / 2;
constexpr float kMagic = 12582912.0f;  // 1.5 * 2^23
constexpr int kMagicBits = 0x4B400000;
constexpr int kPX = 4, kPY = 4;  // pixels per thread along x, y

struct BPArgs {
  const void *sino;
  long long srs, sss;
  int nrow, nslice, ncol;
  const double2 *trig;
  double center;
  int edge_pad;
  double mask_r2;
  float scale;
  float *out;
  long long ors, oss;
  int per_angle_kahan;
};

struct __align__(16) AngleParam {
  float qbase;  // local position of the tile-origin pixel, q = p - lo - kHalf
  float c, s;   // cos(-a), sin(-a) in FP32 for in-tile offsets
  float qmax;   // local position of detector bin ncol - 1
  float qlo;    // local position of detector bin 0
  int j0;       // window index of detector bin 0 (= -lo)
  double c64, s64;  // FP64 trigonometry, for the exact edge decision
};

constexpr float kEdgeTol = 2e-3f;  // bins; FP32 error of q is < 3e-5

__device__ __forceinline__ void kahan_add(float &sum, float &comp, float v) {
  const float y = __fsub_rn(v, comp);
  const float t = __fadd_rn(sum, y);
  comp = __fsub_rn(__fsub_rn(t, sum), y);
  sum = t;
}

template <typename T, bool kPerAngleKahan>
__global__ void __launch_bounds__(kThreads, 2) bp_tile_kernel(BPArgs a) {
  __shared__ float2 pairs[kChunk * kWin];
  __shared__ AngleParam prm[kChunk];
  __shared__ int lo_s[kChunk];
  __shared__ int flag_s[kChunk];  // bit 0: skip angle, bit 1: checked path

  const int tid = threadIdx.x;
  const int warp = tid >> 5, lane = tid & 31;
  const int x0 = blockIdx.x * kTile, y0 = blockIdx.y * kTile;
  const int slice = blockIdx.z;
  const int ncol = a.ncol;
  const T *sino = reinterpret_cast<const T *>(a.sino) + slice * a.sss;

  // thread -> pixel offsets inside the tile: warp w covers 32 x 16 pixels,
  // lane (lx, ly) of an 8 x 4 block, replicated 4 x 4 times
  const int tx = (warp & 1) * 32 + (lane & 7);
  const int ty = (warp >> 1) * 16 + (lane >> 3);

  float acc[kPY][kPX], sum[kPY][kPX], comp[kPY][kPX];
#pragma unroll
  for (int b = 0; b < kPY; ++b)
#pragma unroll
    for (int c = 0; c < kPX; ++c) { acc[b][c] = 0.f; sum[b][c] = 0.f; comp[b][c] = 0.f; }

  const double ic = 0.5 * (double)(ncol - 1);
  const double ext = (double)(kTile - 1);

  for (int i0 = 0; i0 < a.nrow; i0 += kChunk) {
    // (1) per-angle window and local-position parameters, FP64
    if (tid < kChunk) {
      const int i = i0 + tid;
      int flag = 1, lo = 0;
      AngleParam p = {0.f, 0.f, 0.f, 0.f, 0.f, 0, 0.0, 0.0};
      if (i < a.nrow) {
        const double2 cs = a.trig[i];
        const double P0 = ((double)x0 - ic) * cs.x + ((double)y0 - ic) * cs.y + a.center;
        const double ec = ext * cs.x, es = ext * cs.y;
        // non-finite trig (rejected by the host) is skipped, never indexed
        if (isfinite(P0) && isfinite(ec) && isfinite(es)) {
          const double pmin = P0 + fmin(0.0, ec) + fmin(0.0, es);
          const double pmax = P0 + fmax(0.0, ec) + fmax(0.0, es);
          lo = (int)floor(pmin) - 1;
          p.qbase = (float)(P0 - (double)(lo + kHalf));
          p.c = (float)cs.x;
          p.s = (float)cs.y;
          p.qmax = (float)((double)(ncol - 1) - (double)(lo + kHalf));
          p.qlo = (float)(-(lo + kHalf));
          p.j0 = -lo;
          p.c64 = cs.x;
          p.s64 = cs.y;
          flag = 0;
          if (!a.edge_pad) {
            if (pmin > (double)(ncol - 1) + 1e-2 || pmax < -1e-2) flag = 1;
            else if (pmin < 1e-2 || pmax > (double)(ncol - 1) - 1e-2) flag = 2;
          }
        }
      }
      prm[tid] = p;
      lo_s[tid] = lo;
      flag_s[tid] = flag;
    }
    __syncthreads();

    // (2) stage interpolation pairs of every angle of the chunk
    for (int e = tid; e < kChunk * kWin; e += kThreads) {
      const int ai = e / kWin, j = e - ai * kWin;
      const int i = i0 + ai;
      float2 pr = make_float2(0.f, 0.f);
      if (i < a.nrow && !(flag_s[ai] & 1)) {
        const T *row = sino + i * a.srs;
        const int d = lo_s[ai] + j;
        float v, dv;
        if (a.edge_pad) {
          const int d0 = min(max(d, 0), ncol - 1), d1 = min(max(d + 1, 0), ncol - 1);
          v = atb::load_as_float(row + d0);
          dv = atb::load_as_float(row + d1) - v;
        } else if (d < 0 || d > ncol - 1) {
          v = 0.f; dv = 0.f;
        } else if (d == ncol - 1) {
          v = atb::load_as_float(row + d); dv = 0.f;
        } else {
          v = atb::load_as_float(row + d);
          dv = atb::load_as_float(row + d + 1) - v;
        }
        pr = make_float2(fmaf(-(float)(j - kHalf), dv, v), dv);
      }
      pairs[e] = pr;
    }
    __syncthreads();

    // (3) accumulate
    const int nang = min(kChunk, a.nrow - i0);
    for (int ai = 0; ai < nang; ++ai) {
      const int flag = flag_s[ai];
      if (flag & 1) continue;
      const AngleParam p = prm[ai];
      const float qt = fmaf((float)tx, p.c, fmaf((float)ty, p.s, p.qbase));
      const float c8 = 8.f * p.c, s4 = 4.f * p.s;
      const float2 *w = pairs + ai * kWin + kHalf;  // indexed by floor(q)
      if (!(flag & 2)) {
#pragma unroll
        for (int b = 0; b < kPY; ++b) {
          const float qr = fmaf((float)b, s4, qt);
#pragma unroll
          for (int c = 0; c < kPX; ++c) {
            const float q = fmaf((float)c, c8, qr);
            const int j = __float_as_int(__fadd_rd(q, kMagic)) - kMagicBits;
            const float2 pr = w[j];
            const float v = fmaf(pr.y, q, pr.x);
            if (kPerAngleKahan) kahan_add(sum[b][c], comp[b][c], v);
            else acc[b][c] += v;
          }
        }
      } else {
        // checked path: the footprint reaches a detector edge
#pragma unroll
        for (int b = 0; b < kPY; ++b) {
          const float qr = fmaf((float)b, s4, qt);
#pragma unroll
          for (int c = 0; c < kPX; ++c) {
            const float q = fmaf((float)c, c8, qr);
            int j = __float_as_int(__fadd_rd(q, kMagic)) - kMagicBits;
            const float dl = q - p.qlo, dr = q - p.qmax;
            bool inr = (dl >= 0.f) && (dr <= 0.f);
            if (fabsf(dl) < kEdgeTol || fabsf(dr) < kEdgeTol) {
              // same expression and rounding order as the reference's
              // (x - ic) cos + (y - ic) sin + center, in FP64
              const double xc = (double)(x0 + tx + 8 * c) - ic;
              const double yc = (double)(y0 + ty + 4 * b) - ic;
              const double pe = __dadd_rn(__dadd_rn(__dmul_rn(xc, p.c64), __dmul_rn(yc, p.s64)), a.center);
              inr = (pe >= 0.0) && (pe <= (double)(ncol - 1));
              j = max(j, p.j0 - kHalf);
            }
            const float2 pr = w[j];
            const float v = inr ? fmaf(pr.y, q, pr.x) : 0.f;
            if (kPerAngleKahan) kahan_add(sum[b][c], comp[b][c], v);
            else acc[b][c] += v;
          }
        }
      }
    }
    if (!kPerAngleKahan) {
#pragma unroll
      for (int b = 0; b < kPY; ++b)
#pragma unroll
        for (int c = 0; c < kPX; ++c) { kahan_add(sum[b][c], comp[b][c], acc[b][c]); acc[b][c] = 0.f; }
    }
    __syncthreads();
  }

  // (4) epilogue: compensated total, circle mask, scale, store
  const int cm = ncol / 2;
#pragma unroll
  for (int b = 0; b < kPY; ++b) {
    const int y = y0 + ty + 4 * b;
#pragma unroll
    for (int c = 0; c < kPX; ++c) {
      const int x = x0 + tx + 8 * c;
      if (x < ncol && y < ncol) {
        float v = __fsub_rn(sum[b][c], comp[b][c]) * a.scale;
        if (a.mask_r2 >= 0.0) {
          const long long dx = x - cm, dy = y - cm;
          if ((double)(dx * dx + dy * dy) > a.mask_r2) v = 0.f;
        }
        a.out[y * a.ors + slice * a.oss + x] = v;
      }
    }
  }
}

template <typename T>
int launch_bp(const BPArgs &a, cudaStream_t st) {
  dim3 grid((a.ncol + kTile - 1) / kTile, (a.ncol + kTile - 1) / kTile, a.nslice);
  if (a.per_angle_kahan) bp_tile_kernel<T, true><<<grid, kThreads, 0, st>>>(a);
  else bp_tile_kernel<T, false><<<grid, kThreads, 0, st>>>(a);
  return atb::check_launch("atb_backproject");
}

}  // namespace

extern "C" int atb_backproject(const void *sino, int sino_dtype, int64_t sino_row_stride, int64_t sino_slice_stride,
                               int nrow, int nslice, int ncol, const double *trig, double center, int edge_pad,
                               double mask_r2, float scale, float *out, int64_t out_row_stride,
                               int64_t out_slice_stride, int flags, void *stream) {
  if (!sino || !trig || !out) return atb::fail(ATB_EINVAL, "atb_backproject: null pointer");
  if (nrow < 1 || nslice < 1 || ncol < 1)
    return atb::fail(ATB_EINVAL, "atb_backproject: bad shape nrow=%d nslice=%d ncol=%d", nrow, nslice, ncol);
  if (nslice > 65535) return atb::fail(ATB_ERANGE, "atb_backproject: nslice=%d > 65535", nslice);
  if (ncol > (1 << 20)) return atb::fail(ATB_ERANGE, "atb_backproject: ncol=%d too large", ncol);
  if (!(center >= 0.0) || center >= (double)ncol)
    return atb::fail(ATB_EINVAL, "atb_backproject: center %g outside [0, %d)", center, ncol);
  BPArgs a;
  a.sino = sino; a.srs = sino_row_stride; a.sss = sino_slice_stride;
  a.nrow = nrow; a.nslice = nslice; a.ncol = ncol;
  a.trig = reinterpret_cast<const double2 *>(trig);
  a.center = center; a.edge_pad = edge_pad ? 1 : 0; a.mask_r2 = mask_r2; a.scale = scale;
  a.out = out; a.ors = out_row_stride; a.oss = out_slice_stride;
  a.per_angle_kahan = flags & 1;
  cudaStream_t st = atb::as_stream(stream);
  switch (sino_dtype) {
    case ATB_F32: return launch_bp<float>(a, st);
    case ATB_F16: return launch_bp<__half>(a, st);
    case ATB_BF16: return launch_bp<__nv_bfloat16>(a, st);
    default: return atb::fail(ATB_EINVAL, "atb_backproject: unknown sino_dtype %d", sino_dtype);
  }
}
