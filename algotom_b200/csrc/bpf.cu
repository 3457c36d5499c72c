// 2-D circular ramp filter of BPF (algotom/rec/reconstruction.py:527-560,
// applied per slice by bpf_reconstruction at :675-684), with the mask and
// pi/(nrow-1) scale of :679-684 fused in.
//
// The reference pads each back-projected slice to N x N (N = ncol + 2 pad,
// numpy's pad modes), takes fft2, multiplies by the fftshifted circular
// window W2, inverts and keeps the real part of the crop [pad, pad+ncol)^2.
// W2 is real, so only the even part Hh(k) = (H(k) + H(-k)) / 2 of
// H = ifftshift(W2) reaches the real part: the filter is the circular
// convolution on the N x N torus with the real, even kernel ifft2(Hh).  A
// real operator maps real images to real images, so two slices travel as
// one complex image a + i b and come back as the real and imaginary parts.
//
// Transform length T: N itself when its prime factors are all in
// {2, 3, 5, 7, 11, 13} (2860 = 4 5 11 13 at 2560 detector pixels);
// otherwise (1324 = 4 331 at 1024) the smallest 7-smooth M >= N + ncol - 1.
// A circular convolution of length M with the kernel's lags
// [pad - N + 1, pad + ncol - 1] reproduces the N-periodic one exactly on the
// crop (the same embedding as the row filter), per axis.  The host builds
// the spectrum for T in FP64: the real Hh for T = N, the complex transform
// of the embedded kernel otherwise, scaled by 1 / T^2, stored transposed
// ([kx][ky]) so that a column transform reads it contiguously.
//
// Three kernels per group of slice pairs, all FP64 in shared memory
// (atb::fft, mixed-radix Stockham):
//   rows:    pad (on the fly, all ten numpy modes) + forward row transform
//            of each padded row -> workspace [pair][ry < N][kx < T]
//   columns: forward column transform, product with the spectrum, inverse
//            column transform; only the crop rows [pad, pad+ncol) are
//            written back (rows >= N of an embedded transform are zero and
//            never stored)
//   output:  inverse row transform of each crop row, crop, mask, scale,
//            written into the [ncol][nslice][ncol] reconstruction layout
// The ramp amplifies rounding of the smooth back-projection by about 140x
// at 2560^2, which is why the transforms run in FP64 (FP32 gave 2.2e-5
// relative L2 against the FP64 oracle).
#include <cmath>
#include <mutex>

#include "common.cuh"
#include "fft.cuh"

namespace {

using atb::fft::Plan;

constexpr int kThreads = 256;
constexpr int kMaxLen = 7168;        // two buffers of T complex doubles + twiddles fit 227 KB
constexpr int kStatThreads = 1024;
constexpr int kMaxStatLen = 8192;    // lines sorted in shared memory (median)

struct BpfArgs {
  const float *src;    // back-projection stack [ncol y][nslice][ncol x]
  long long srs, sss;
  int nslice, ncol, pad, n;  // n = ncol + 2 pad
  int mode;                  // ATB_PAD_*
  int slice0;                // first slice of this group (pair g: slice0 + 2g, +1)
  float *dst;
  long long drs, dss;
  double mask_r2;
  float scale;
  double2 *work;             // [pairs][n][T]
  const void *spec;          // [T][T] transposed, real (double) or complex
  int spec_complex;
  const double *colstat;     // [2 pairs][ncol] column statistics (stat modes)
  const double *rowstat;     // [2 pairs][ncol] row statistics
  const double *padstat;     // [2 pairs] statistic of the padded rows
};

__device__ __forceinline__ int index_map(int i, int n, int mode) {
  // numpy's index modes as periodic maps, valid for any pad width
  if (mode == ATB_PAD_EDGE) return min(max(i, 0), n - 1);
  if (mode == ATB_PAD_WRAP) {
    const int r = i % n;
    return r < 0 ? r + n : r;
  }
  if (mode == ATB_PAD_SYMMETRIC) {
    const int p = 2 * n;
    int r = i % p;
    if (r < 0) r += p;
    return r >= n ? p - 1 - r : r;
  }
  if (n == 1) return 0;  // reflect: period 2 (n - 1), edges not repeated
  const int p = 2 * (n - 1);
  int r = i % p;
  if (r < 0) r += p;
  return r >= n ? p - r : r;
}

// np.pad(slice, pad, mode) at padded (ry, rx): numpy pads axis 0 over the
// original columns first, then axis 1 over all rows, which fixes the
// corners of the ramp and statistic modes.  ks: slice index within the
// group (statistics).
__device__ double pad_value(const BpfArgs &a, const float *X, int ks, int ry, int rx) {
  const int n = a.ncol, y = ry - a.pad, x = rx - a.pad;
  const long long rs = a.srs;
  switch (a.mode) {
    case ATB_PAD_EDGE:
    case ATB_PAD_REFLECT:
    case ATB_PAD_SYMMETRIC:
    case ATB_PAD_WRAP:
      return (double)__ldg(X + index_map(y, n, a.mode) * rs + index_map(x, n, a.mode));
    case ATB_PAD_CONSTANT:
      return (y >= 0 && y < n && x >= 0 && x < n) ? (double)__ldg(X + y * rs + x) : 0.0;
    case ATB_PAD_LINEAR_RAMP: {
      // ramps from 0 at the ends to the edge sample, endpoint excluded:
      // position k of a pad of width w holds k * (edge / w)
      const double w = (double)a.pad;
      auto column = [&](int xx) -> double {  // value after the axis-0 stage
        if (y < 0) return (double)ry * ((double)__ldg(X + xx) / w);
        if (y >= n) return (double)(a.pad - 1 - (y - n)) * ((double)__ldg(X + (n - 1) * rs + xx) / w);
        return (double)__ldg(X + y * rs + xx);
      };
      if (x < 0) return (double)rx * (column(0) / w);
      if (x >= n) return (double)(a.pad - 1 - (x - n)) * (column(n - 1) / w);
      return column(x);
    }
    default: {  // mean, maximum, minimum, median over the whole line
      const bool yin = y >= 0 && y < n, xin = x >= 0 && x < n;
      if (xin) return yin ? (double)__ldg(X + y * rs + x) : a.colstat[(long long)ks * n + x];
      return yin ? a.rowstat[(long long)ks * n + y] : a.padstat[ks];
    }
  }
}

// Grids put the slice pair on x, so that the CTAs of one row / column of
// every pair run together (the columns kernel then reads each spectrum
// column once from DRAM).  Shared memory: two buffers of T values, then
// the twiddle table.
__global__ void __launch_bounds__(kThreads) bpf_rows_kernel(BpfArgs a, const __grid_constant__ Plan pl) {
  extern __shared__ double2 sm[];
  const int ry = blockIdx.y, g = blockIdx.x, T = pl.n;
  double2 *tws = sm + 2 * T;
  atb::fft::load_twiddles(pl, tws);
  const int sa = a.slice0 + 2 * g, sb = sa + 1;
  const bool hb = sb < a.nslice;
  const float *Xa = a.src + (long long)sa * a.sss;
  const float *Xb = a.src + (long long)(hb ? sb : sa) * a.sss;
  for (int rx = threadIdx.x; rx < T; rx += blockDim.x) {
    double2 z = make_double2(0.0, 0.0);
    if (rx < a.n) {
      z.x = pad_value(a, Xa, 2 * g, ry, rx);
      if (hb) z.y = pad_value(a, Xb, 2 * g + 1, ry, rx);
    }
    sm[rx] = z;
  }
  __syncthreads();
  const double2 *res = atb::fft::run<false>(sm, sm + T, pl, tws);
  double2 *w = a.work + ((long long)g * a.n + ry) * T;
  for (int kx = threadIdx.x; kx < T; kx += blockDim.x) w[kx] = res[kx];
}

__global__ void __launch_bounds__(kThreads) bpf_cols_kernel(BpfArgs a, const __grid_constant__ Plan pl) {
  extern __shared__ double2 sm[];
  const int kx = blockIdx.y, g = blockIdx.x, T = pl.n, n = a.n;
  double2 *tws = sm + 2 * T;
  atb::fft::load_twiddles(pl, tws);
  double2 *w = a.work + (long long)g * n * T + kx;
  for (int ry = threadIdx.x; ry < T; ry += blockDim.x)
    sm[ry] = ry < n ? w[(long long)ry * T] : make_double2(0.0, 0.0);
  __syncthreads();
  double2 *res = atb::fft::run<false>(sm, sm + T, pl, tws);
  double2 *other = res == sm ? sm + T : sm;
  if (a.spec_complex) {
    const double2 *S = static_cast<const double2 *>(a.spec) + (long long)kx * T;
    for (int ky = threadIdx.x; ky < T; ky += blockDim.x) res[ky] = atb::fft::cmul(res[ky], __ldg(S + ky));
  } else {
    const double *S = static_cast<const double *>(a.spec) + (long long)kx * T;
    for (int ky = threadIdx.x; ky < T; ky += blockDim.x) {
      const double h = __ldg(S + ky);
      res[ky].x *= h;
      res[ky].y *= h;
    }
  }
  __syncthreads();
  const double2 *out = atb::fft::run<true>(res, other, pl, tws);
  for (int u = a.pad + threadIdx.x; u < a.pad + a.ncol; u += blockDim.x) w[(long long)u * T] = out[u];
}

__global__ void __launch_bounds__(kThreads) bpf_out_kernel(BpfArgs a, const __grid_constant__ Plan pl) {
  extern __shared__ double2 sm[];
  const int y = blockIdx.y, g = blockIdx.x, T = pl.n;
  double2 *tws = sm + 2 * T;
  atb::fft::load_twiddles(pl, tws);
  const double2 *w = a.work + ((long long)g * a.n + y + a.pad) * T;
  for (int kx = threadIdx.x; kx < T; kx += blockDim.x) sm[kx] = w[kx];
  __syncthreads();
  const double2 *res = atb::fft::run<true>(sm, sm + T, pl, tws);
  const int sa = a.slice0 + 2 * g, sb = sa + 1;
  const bool hb = sb < a.nslice;
  const int c = a.ncol / 2;
  const double dy = (double)(y - c);
  float *oa = a.dst + (long long)y * a.drs + (long long)sa * a.dss;
  float *ob = a.dst + (long long)y * a.drs + (long long)(hb ? sb : sa) * a.dss;
  const double sc = (double)a.scale;
  for (int x = threadIdx.x; x < a.ncol; x += blockDim.x) {
    const double dx = (double)(x - c);
    const bool in = a.mask_r2 < 0.0 || dx * dx + dy * dy <= a.mask_r2;
    const double2 v = res[x + a.pad];
    oa[x] = in ? (float)(v.x * sc) : 0.0f;
    if (hb) ob[x] = in ? (float)(v.y * sc) : 0.0f;
  }
}

// ---- FP64 row filter: the ramp filter a vertical reconstruction applies
// after its back-projection (algotom/rec/vertrec.py:677-684, 697-706),
// real(ifft(fft(pad(row)) * ifftshift(|W|))) cropped to [pad, pad + ncol),
// on FP64 rows, with the same transform lengths and FP64 Stockham FFT as the
// 2-D filter above.  Each row is transformed on its own: packing two rows
// into one complex transform would give equal rows unequal round-off (the
// real and the imaginary slot round differently), and the centre search
// normalises by a maximum that such equal rows reach exactly.  An even
// length T is done as a real transform: the row's even and odd samples are
// the real and imaginary parts of one length-T/2 transform Z, split into the
// row's spectrum X[k] = A[k] + W^k B[k] (W = exp(-2 pi i / T);
// A[k] = (Z[k] + conj Z[-k]) / 2, B[k] = (Z[k] - conj Z[-k]) / 2i), multiplied
// by the filter's spectrum S (Hermitian: the kernel is real), and merged back
// into one length-T/2 inverse, U[k] = (Y[k] + conj Y[H-k])
// + i W^-k (Y[k] - conj Y[H-k]), whose output holds y[2m] + i y[2m+1].  An
// odd T takes one complex transform with a zero imaginary part.
struct Row64Args {
  const double *src;
  long long srs;
  int nrows, ncol, pad, n, mode;
  const double *rowstat;  // [nrows] statistic of each row (statistic modes)
  const double2 *spec;    // [T] spectrum of the embedded kernel, / T
  const double2 *tw;      // [T] exp(-2 pi i t / T)
  double *dst;
  long long drs;
};

__device__ __forceinline__ double row64_value(const Row64Args &a, const double *x, double stat, int rx) {
  const int n = a.ncol, i = rx - a.pad;
  if (rx >= a.n) return 0.0;  // the embedding's zeros
  if (i >= 0 && i < n) return __ldg(x + i);
  switch (a.mode) {
    case ATB_PAD_EDGE:
    case ATB_PAD_REFLECT:
    case ATB_PAD_SYMMETRIC:
    case ATB_PAD_WRAP: return __ldg(x + index_map(i, n, a.mode));
    case ATB_PAD_CONSTANT: return 0.0;
    case ATB_PAD_LINEAR_RAMP: {  // k (edge / pad), endpoint excluded, reversed on the right
      const double w = (double)a.pad;
      return i < 0 ? (double)rx * (__ldg(x) / w) : (double)(a.pad - 1 - (i - n)) * (__ldg(x + n - 1) / w);
    }
    default: return stat;  // mean, maximum, minimum, median of the row
  }
}

// Twiddle table of the plan (the length-L transforms) from the length-T
// table a.tw: every entry when L = T, every second when L = T / 2.
template <bool HALF>
__device__ __forceinline__ void row64_twiddles(const double2 *tw, int L, double2 *tws) {
  constexpr int st = HALF ? 2 : 1, lo = atb::fft::kTwLo;
  const int nhi = (L + lo - 1) / lo;
  for (int i = threadIdx.x; i < lo + nhi; i += blockDim.x)
    tws[i] = i < lo ? (i < L ? __ldg(tw + st * i) : make_double2(1.0, 0.0)) : __ldg(tw + st * (i - lo) * lo);
}

// Between the forward and the inverse half-length transforms of a real row
// (res: Z, the transform of x[2m] + i x[2m+1], m < H): the row's spectrum
// X[k], k = 0 .. H, the product Y[k] = prod(X[k], k), and U, whose inverse
// holds y[2m] + i y[2m+1] for the real y with the Hermitian spectrum Y.
// Pairs (k, H - k) are disjoint, so each thread works in place.
template <class Prod>
__device__ __forceinline__ void real_split_merge(double2 *res, int H, const double2 *tw, Prod prod) {
  for (int k = threadIdx.x; 2 * k <= H; k += blockDim.x) {
    const int kc = k == 0 ? 0 : H - k;
    const double2 zk = res[k], zc = res[kc];
    if (k == 0) {
      // X[0] = Re Z0 + Im Z0, X[H] = Re Z0 - Im Z0; U[0] = (Y0 + conj YH) + i (Y0 - conj YH)
      const double2 y0 = prod(make_double2(zk.x + zk.y, 0.0), 0), yh = prod(make_double2(zk.x - zk.y, 0.0), H);
      const double2 s = make_double2(y0.x + yh.x, y0.y - yh.y), d = make_double2(y0.x - yh.x, y0.y + yh.y);
      res[0] = make_double2(s.x - d.y, s.y + d.x);
      continue;
    }
    const double2 w = __ldg(tw + k);
    // A = (Zk + conj Zc) / 2, B = (Zk - conj Zc) / 2i, X[k] = A + W^k B, X[H-k] = conj(A - W^k B)
    const double2 A = make_double2(0.5 * (zk.x + zc.x), 0.5 * (zk.y - zc.y));
    const double2 B = make_double2(0.5 * (zk.y + zc.y), -0.5 * (zk.x - zc.x));
    const double2 wb = atb::fft::cmul(w, B);
    const double2 yk = prod(make_double2(A.x + wb.x, A.y + wb.y), k);
    const double2 yc = prod(make_double2(A.x - wb.x, wb.y - A.y), H - k);
    // U[k] = (Yk + conj Yc) + i W^-k (Yk - conj Yc); U[H-k] = (Yc + conj Yk) - i W^k (Yc - conj Yk)
    const double2 s1 = make_double2(yk.x + yc.x, yk.y - yc.y), d1 = make_double2(yk.x - yc.x, yk.y + yc.y);
    const double2 t1 = atb::fft::cmulc(d1, w);
    res[k] = make_double2(s1.x - t1.y, s1.y + t1.x);
    if (kc != k) {
      const double2 s2 = make_double2(yc.x + yk.x, yc.y - yk.y), d2 = make_double2(yc.x - yk.x, yc.y + yk.y);
      const double2 t2 = atb::fft::cmul(d2, w);
      res[kc] = make_double2(s2.x + t2.y, s2.y - t2.x);
    }
  }
}

// y[q] of the inverse's output (real transform: packed two per entry)
template <bool HALF>
__device__ __forceinline__ double real_out(const double2 *out, int q) {
  return HALF ? ((q & 1) ? out[q >> 1].y : out[q >> 1].x) : out[q].x;
}

// row blockIdx.x; HALF: the plan is for H = T / 2
template <bool HALF>
__global__ void __launch_bounds__(kThreads) row64_kernel(const __grid_constant__ Row64Args a,
                                                         const __grid_constant__ Plan pl) {
  extern __shared__ double2 sm[];
  const int L = pl.n, r = blockIdx.x;  // L: the length of the complex transforms
  double2 *tws = sm + 2 * L;
  row64_twiddles<HALF>(a.tw, L, tws);
  const double *x = a.src + (long long)r * a.srs;
  const double st = a.rowstat ? a.rowstat[r] : 0.0;
  for (int m = threadIdx.x; m < L; m += blockDim.x)
    sm[m] = HALF ? make_double2(row64_value(a, x, st, 2 * m), row64_value(a, x, st, 2 * m + 1))
                 : make_double2(row64_value(a, x, st, m), 0.0);
  __syncthreads();
  double2 *res = atb::fft::run<false>(sm, sm + L, pl, tws);
  double2 *other = res == sm ? sm + L : sm;
  if constexpr (HALF) {
    real_split_merge(res, L, a.tw, [&](double2 v, int k) { return atb::fft::cmul(v, __ldg(a.spec + k)); });
  } else {
    for (int k = threadIdx.x; k < L; k += blockDim.x) res[k] = atb::fft::cmul(res[k], __ldg(a.spec + k));
  }
  __syncthreads();
  const double2 *out = atb::fft::run<true>(res, other, pl, tws);
  double *d = a.dst + (long long)r * a.drs;
  for (int j = threadIdx.x; j < a.ncol; j += blockDim.x) d[j] = real_out<HALF>(out, a.pad + j);
}

// ---- row autocorrelation maximum of the vertical centre search's
// "autocorrelation" metric (algotom/rec/vertrec.py:1255-1261):
// max over lags of |ifft(|fft(row)|^2)|, the circular autocorrelation of
// the float32 row, in FP64.  Transform length T = ncol when it has no prime
// factor above 13; else the row is zero-padded to a 7-smooth T >= 2 ncol - 1
// and the linear autocorrelation folded back onto the circle,
// r[l] = y[l] + y[T - ncol + l] (l >= 1).  One row per CTA, a real transform
// of half length when T is even.
struct AcArgs {
  const float *src;
  long long srs;
  int nrows, ncol;
  const double2 *tw;  // [T] exp(-2 pi i t / T)
  double *out;        // [nrows] maximum of each row
};

template <bool HALF>
__global__ void __launch_bounds__(kThreads) autocorr_kernel(const __grid_constant__ AcArgs a,
                                                            const __grid_constant__ Plan pl) {
  extern __shared__ double2 sm[];
  __shared__ double red[kThreads / 32];
  const int L = pl.n, T = HALF ? 2 * L : L, r = blockIdx.x, n = a.ncol;
  double2 *tws = sm + 2 * L;
  row64_twiddles<HALF>(a.tw, L, tws);
  const float *x = a.src + (long long)r * a.srs;
  for (int m = threadIdx.x; m < L; m += blockDim.x) {
    const int i0 = HALF ? 2 * m : m, i1 = i0 + 1;
    const double v0 = i0 < n ? (double)__ldg(x + i0) : 0.0;
    const double v1 = HALF && i1 < n ? (double)__ldg(x + i1) : 0.0;
    sm[m] = make_double2(v0, v1);
  }
  __syncthreads();
  double2 *res = atb::fft::run<false>(sm, sm + L, pl, tws);
  double2 *other = res == sm ? sm + L : sm;
  if constexpr (HALF) {
    real_split_merge(res, L, a.tw, [](double2 v, int) { return make_double2(fma(v.x, v.x, v.y * v.y), 0.0); });
  } else {
    for (int k = threadIdx.x; k < L; k += blockDim.x) {
      const double2 v = res[k];
      res[k] = make_double2(fma(v.x, v.x, v.y * v.y), 0.0);
    }
  }
  __syncthreads();
  const double2 *out = atb::fft::run<true>(res, other, pl, tws);
  const double inv = 1.0 / (double)T;  // the inverse's 1 / T
  double m = 0.0;
  for (int l = threadIdx.x; l < n; l += blockDim.x) {
    double v = real_out<HALF>(out, l);
    if (T != n && l > 0) v += real_out<HALF>(out, T - n + l);
    m = fmax(m, fabs(v * inv));
  }
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_down_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < (int)(blockDim.x >> 5); ++w) m = fmax(m, red[w]);
    a.out[r] = m;
  }
}

// ---- statistics of the statistic pad modes (mean, maximum, minimum, median)

template <typename K>
__device__ void bitonic_sort(K *v, int m) {  // m a power of two, ascending
  for (int size = 2; size <= m; size <<= 1) {
    for (int stride = size >> 1; stride > 0; stride >>= 1) {
      for (int i = threadIdx.x; i < m; i += blockDim.x) {
        const int j = i ^ stride;
        if (j > i) {
          const bool up = (i & size) == 0;
          const K vi = v[i], vj = v[j];
          if ((vi > vj) == up) {
            v[i] = vj;
            v[j] = vi;
          }
        }
      }
      __syncthreads();
    }
  }
}

// sum in a fixed order: per-thread strided partials, then a tree
__device__ double block_sum(double v, double *red) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) red[warp] = v;
  __syncthreads();
  double t = 0.0;
  if (threadIdx.x == 0)
    for (int k = 0; k < (int)(blockDim.x >> 5); ++k) t += red[k];
  __syncthreads();
  return t;
}

template <typename K>
__device__ double line_stat(int mode, int n, K *buf, double *red) {
  // buf holds the n values (sorted in place for the median)
  if (mode == ATB_PAD_MEDIAN) {
    int m = 1;
    while (m < n) m <<= 1;
    for (int i = n + threadIdx.x; i < m; i += blockDim.x) buf[i] = (K)INFINITY;
    __syncthreads();
    bitonic_sort(buf, m);
    return 0.5 * ((double)buf[(n - 1) / 2] + (double)buf[n / 2]);
  }
  double acc = mode == ATB_PAD_MEAN ? 0.0 : (mode == ATB_PAD_MAXIMUM ? -INFINITY : INFINITY);
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    const double v = (double)buf[i];
    acc = mode == ATB_PAD_MEAN ? acc + v : (mode == ATB_PAD_MAXIMUM ? fmax(acc, v) : fmin(acc, v));
  }
  if (mode == ATB_PAD_MEAN) return block_sum(acc, red) / (double)n;
  for (int o = 16; o > 0; o >>= 1) {
    const double u = __shfl_down_sync(0xffffffffu, acc, o);
    acc = mode == ATB_PAD_MAXIMUM ? fmax(acc, u) : fmin(acc, u);
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) red[warp] = acc;
  __syncthreads();
  double t = red[0];
  if (threadIdx.x == 0)
    for (int k = 1; k < (int)(blockDim.x >> 5); ++k) t = mode == ATB_PAD_MAXIMUM ? fmax(t, red[k]) : fmin(t, red[k]);
  __syncthreads();
  return t;
}

// blockIdx.x < ncol: statistic of column x over the rows; else of row
// blockIdx.x - ncol over the columns; blockIdx.y: slice within the group
__global__ void __launch_bounds__(kStatThreads) bpf_stats_kernel(BpfArgs a, double *colstat, double *rowstat) {
  __shared__ float buf[kMaxStatLen];
  __shared__ double red[32];
  const int n = a.ncol, ks = blockIdx.y, s = a.slice0 + ks;
  const bool col = (int)blockIdx.x < n;
  const int line = col ? blockIdx.x : blockIdx.x - n;
  const float *X = a.src + (long long)s * a.sss;
  for (int k = threadIdx.x; k < n; k += blockDim.x)
    buf[k] = col ? __ldg(X + (long long)k * a.srs + line) : __ldg(X + (long long)line * a.srs + k);
  __syncthreads();
  const double v = line_stat<float>(a.mode, n, buf, red);
  if (threadIdx.x == 0) (col ? colstat : rowstat)[(long long)ks * n + line] = v;
}

// statistic of a padded row: its original-column part holds colstat, so
// the row statistic is the statistic of colstat; one CTA per slice
__global__ void __launch_bounds__(kStatThreads) bpf_padstat_kernel(BpfArgs a, const double *colstat,
                                                                   double *padstat) {
  extern __shared__ double dbuf[];
  __shared__ double red[32];
  const int n = a.ncol, ks = blockIdx.x;
  for (int k = threadIdx.x; k < n; k += blockDim.x) dbuf[k] = colstat[(long long)ks * n + k];
  __syncthreads();
  const double v = line_stat<double>(a.mode, n, dbuf, red);
  if (threadIdx.x == 0) padstat[ks] = v;
}

bool smooth(int t, const int *primes, int np) {
  for (int k = 0; k < np; ++k)
    while (t % primes[k] == 0) t /= primes[k];
  return t == 1;
}

int transform_length(int ncol, int pad) {
  static const int p13[] = {2, 3, 5, 7, 11, 13};
  static const int p7[] = {2, 3, 5, 7};
  const int n = ncol + 2 * pad;
  if (n <= kMaxLen && smooth(n, p13, 6)) return n;
  for (int m = n + ncol - 1; m <= kMaxLen; ++m)
    if (smooth(m, p7, 4)) return m;
  return -1;
}

// radices of t, 8s and 4s first, then the odd ones, then a last 2
bool make_plan(int t, const double2 *tw, Plan &pl) {
  pl.n = t;
  pl.tw = tw;
  pl.nstages = 0;
  int r = t;
  auto push = [&](int p) {
    if (pl.nstages >= atb::fft::kMaxStages) return false;
    pl.radix[pl.nstages++] = p;
    r /= p;
    return true;
  };
  while (r % 8 == 0)
    if (!push(8)) return false;
  while (r % 4 == 0)
    if (!push(4)) return false;
  static const int odd[] = {13, 11, 7, 5, 3};
  for (int p : odd)
    while (r % p == 0)
      if (!push(p)) return false;
  while (r % 2 == 0)
    if (!push(2)) return false;
  if (r != 1) return false;
  static const int op[atb::fft::kOddRadices] = {3, 5, 7, 11, 13};
  for (int k = 0; k < atb::fft::kOddRadices; ++k)
    for (int q = 1; q <= (op[k] - 1) / 2; ++q) {
      const double ang = 2.0 * M_PI * (double)q / (double)op[k];
      pl.rc[k][q - 1] = make_double2(std::cos(ang), std::sin(ang));
    }
  return true;
}

size_t align256(size_t b) { return (b + 255) / 256 * 256; }

}  // namespace

extern "C" int atb_bpf_filter2d_length(int ncol, int pad) {
  if (ncol < 1 || pad < 0) return atb::fail(ATB_EINVAL, "atb_bpf_filter2d_length: ncol=%d pad=%d", ncol, pad);
  const int t = transform_length(ncol, pad);
  if (t < 0)
    return atb::fail(ATB_ERANGE, "atb_bpf_filter2d_length: no transform length <= %d for ncol=%d pad=%d", kMaxLen,
                     ncol, pad);
  return t;
}

extern "C" int64_t atb_bpf_filter2d_workspace(int ncol, int pad, int pairs) {
  const int t = atb_bpf_filter2d_length(ncol, pad);
  if (t < 0) return t;
  if (pairs < 1) return atb::fail(ATB_EINVAL, "atb_bpf_filter2d_workspace: pairs=%d", pairs);
  const size_t n = (size_t)ncol + 2 * (size_t)pad;
  const size_t work = align256((size_t)pairs * n * (size_t)t * sizeof(double2));
  const size_t stats = align256((size_t)2 * pairs * (2 * (size_t)ncol + 1) * sizeof(double));
  return (int64_t)(work + stats);
}

extern "C" int atb_bpf_filter2d(const float *src, int64_t src_row_stride, int64_t src_slice_stride, int nslice,
                                int ncol, int pad, int pad_mode, const void *spectrum, int spectrum_complex,
                                const void *twiddle, double mask_r2, float scale, float *dst, int64_t dst_row_stride,
                                int64_t dst_slice_stride, void *workspace, int64_t workspace_bytes, void *stream) {
  if (!src || !spectrum || !twiddle || !dst || !workspace)
    return atb::fail(ATB_EINVAL, "atb_bpf_filter2d: null pointer");
  if (nslice < 1 || ncol < 1 || pad < 0)
    return atb::fail(ATB_EINVAL, "atb_bpf_filter2d: bad shape nslice=%d ncol=%d pad=%d", nslice, ncol, pad);
  if (pad_mode < ATB_PAD_EDGE || pad_mode > ATB_PAD_MEDIAN)
    return atb::fail(ATB_EINVAL, "atb_bpf_filter2d: unknown pad mode %d", pad_mode);
  if (pad_mode == ATB_PAD_LINEAR_RAMP && pad == 0) pad_mode = ATB_PAD_CONSTANT;  // nothing to ramp
  const bool stat = pad_mode >= ATB_PAD_MEAN;
  if (stat && ncol > kMaxStatLen)
    return atb::fail(ATB_ERANGE, "atb_bpf_filter2d: statistic pad modes support ncol <= %d", kMaxStatLen);
  const int t = atb_bpf_filter2d_length(ncol, pad);
  if (t < 0) return t;
  Plan pl;
  if (!make_plan(t, static_cast<const double2 *>(twiddle), pl))
    return atb::fail(ATB_ERANGE, "atb_bpf_filter2d: no radix plan for length %d", t);
  const int64_t per_pair = atb_bpf_filter2d_workspace(ncol, pad, 1);
  if (workspace_bytes < per_pair)
    return atb::fail(ATB_EINVAL, "atb_bpf_filter2d: workspace of %lld bytes needed for one slice pair",
                     (long long)per_pair);
  // as many slice pairs per group as the workspace holds
  const int npairs = (nslice + 1) / 2;
  int pairs = npairs < 32768 ? npairs : 32768;
  while (pairs > 1 && atb_bpf_filter2d_workspace(ncol, pad, pairs) > workspace_bytes) pairs = (pairs + 1) / 2;
  while (pairs < npairs && pairs < 32768 && atb_bpf_filter2d_workspace(ncol, pad, pairs + 1) <= workspace_bytes)
    ++pairs;

  const size_t smem = (2 * (size_t)t + atb::fft::twiddle_entries(t)) * sizeof(double2);
  int rc = atb::ensure_smem(bpf_rows_kernel, smem, "atb_bpf_filter2d");
  if (rc == ATB_OK) rc = atb::ensure_smem(bpf_cols_kernel, smem, "atb_bpf_filter2d");
  if (rc == ATB_OK) rc = atb::ensure_smem(bpf_out_kernel, smem, "atb_bpf_filter2d");
  int m2 = 1;  // the median sorts a power-of-two line
  while (m2 < ncol) m2 <<= 1;
  const size_t stat_smem = (size_t)m2 * sizeof(double);
  if (rc == ATB_OK && stat) rc = atb::ensure_smem(bpf_padstat_kernel, stat_smem, "atb_bpf_filter2d");
  if (rc != ATB_OK) return rc;

  const int n = ncol + 2 * pad;
  BpfArgs a;
  a.src = src;
  a.srs = src_row_stride;
  a.sss = src_slice_stride;
  a.nslice = nslice;
  a.ncol = ncol;
  a.pad = pad;
  a.n = n;
  a.mode = pad_mode;
  a.dst = dst;
  a.drs = dst_row_stride;
  a.dss = dst_slice_stride;
  a.mask_r2 = mask_r2;
  a.scale = scale;
  unsigned char *ws = static_cast<unsigned char *>(workspace);
  a.work = reinterpret_cast<double2 *>(ws);
  double *stats = reinterpret_cast<double *>(ws + align256((size_t)pairs * n * (size_t)t * sizeof(double2)));
  double *colstat = stats, *rowstat = stats + (size_t)2 * pairs * ncol, *padstat = rowstat + (size_t)2 * pairs * ncol;
  a.colstat = colstat;
  a.rowstat = rowstat;
  a.padstat = padstat;
  a.spec = spectrum;
  a.spec_complex = spectrum_complex ? 1 : 0;
  cudaStream_t st = atb::as_stream(stream);
  for (int p0 = 0; p0 < npairs; p0 += pairs) {
    const int gp = npairs - p0 < pairs ? npairs - p0 : pairs;
    a.slice0 = 2 * p0;
    const int gs = nslice - a.slice0 < 2 * gp ? nslice - a.slice0 : 2 * gp;  // slices in this group
    if (stat) {
      bpf_stats_kernel<<<dim3(2 * ncol, gs), kStatThreads, 0, st>>>(a, colstat, rowstat);
      bpf_padstat_kernel<<<gs, kStatThreads, stat_smem, st>>>(a, colstat, padstat);
    }
    bpf_rows_kernel<<<dim3(gp, n), kThreads, smem, st>>>(a, pl);
    bpf_cols_kernel<<<dim3(gp, t), kThreads, smem, st>>>(a, pl);
    bpf_out_kernel<<<dim3(gp, ncol), kThreads, smem, st>>>(a, pl);
    rc = atb::check_launch("atb_bpf_filter2d");
    if (rc != ATB_OK) return rc;
  }
  return ATB_OK;
}

extern "C" int atb_filter_rows64_length(int ncol, int pad) {
  if (ncol < 1 || pad < 0) return atb::fail(ATB_EINVAL, "atb_filter_rows64_length: ncol=%d pad=%d", ncol, pad);
  const int t = transform_length(ncol, pad);
  if (t < 0)
    return atb::fail(ATB_ERANGE, "atb_filter_rows64_length: no transform length <= %d for ncol=%d pad=%d", kMaxLen,
                     ncol, pad);
  return t;
}

extern "C" int atb_filter_rows64(const double *src, int64_t src_row_stride, int nrows, int ncol, int pad,
                                 int pad_mode, const double *rowstat, const void *spectrum, const void *twiddle,
                                 int fft_len, double *dst, int64_t dst_row_stride, void *stream) {
  if (!src || !spectrum || !twiddle || !dst) return atb::fail(ATB_EINVAL, "atb_filter_rows64: null pointer");
  if (nrows < 1 || ncol < 1 || pad < 0)
    return atb::fail(ATB_EINVAL, "atb_filter_rows64: bad shape nrows=%d ncol=%d pad=%d", nrows, ncol, pad);
  if (pad_mode < ATB_PAD_EDGE || pad_mode > ATB_PAD_MEDIAN)
    return atb::fail(ATB_EINVAL, "atb_filter_rows64: unknown pad mode %d", pad_mode);
  if (pad_mode >= ATB_PAD_MEAN && pad > 0 && !rowstat)
    return atb::fail(ATB_EINVAL, "atb_filter_rows64: statistic pad modes need the row statistics");
  if (pad_mode == ATB_PAD_LINEAR_RAMP && pad == 0) pad_mode = ATB_PAD_CONSTANT;
  const int t = atb_filter_rows64_length(ncol, pad);
  if (t < 0) return t;
  if (fft_len != t)
    return atb::fail(ATB_EINVAL, "atb_filter_rows64: fft_len=%d, atb_filter_rows64_length gives %d", fft_len, t);
  const bool half = (t & 1) == 0;
  const int len = half ? t / 2 : t;
  Plan pl;
  if (!make_plan(len, static_cast<const double2 *>(twiddle), pl))
    return atb::fail(ATB_ERANGE, "atb_filter_rows64: no radix plan for length %d", len);
  const size_t smem = (2 * (size_t)len + atb::fft::twiddle_entries(len)) * sizeof(double2);
  const int rc = half ? atb::ensure_smem(row64_kernel<true>, smem, "atb_filter_rows64")
                      : atb::ensure_smem(row64_kernel<false>, smem, "atb_filter_rows64");
  if (rc != ATB_OK) return rc;
  Row64Args a;
  a.src = src; a.srs = src_row_stride; a.nrows = nrows; a.ncol = ncol; a.pad = pad; a.n = ncol + 2 * pad;
  a.mode = pad_mode; a.rowstat = rowstat; a.spec = static_cast<const double2 *>(spectrum);
  a.tw = static_cast<const double2 *>(twiddle); a.dst = dst; a.drs = dst_row_stride;
  if (half)
    row64_kernel<true><<<nrows, kThreads, smem, atb::as_stream(stream)>>>(a, pl);
  else
    row64_kernel<false><<<nrows, kThreads, smem, atb::as_stream(stream)>>>(a, pl);
  return atb::check_launch("atb_filter_rows64");
}

extern "C" int atb_autocorr_length(int ncol) {
  static const int p13[] = {2, 3, 5, 7, 11, 13};
  static const int p7[] = {2, 3, 5, 7};
  if (ncol < 1) return atb::fail(ATB_EINVAL, "atb_autocorr_length: ncol=%d", ncol);
  if (ncol <= kMaxLen && smooth(ncol, p13, 6)) return ncol;
  for (int m = 2 * ncol - 1; m <= kMaxLen; ++m)
    if (smooth(m, p7, 4)) return m;
  return atb::fail(ATB_ERANGE, "atb_autocorr_length: no transform length <= %d for ncol=%d", kMaxLen, ncol);
}

extern "C" int atb_autocorr_rowmax(const float *src, int64_t src_row_stride, int nrows, int ncol,
                                   const void *twiddle, int fft_len, double *out, void *stream) {
  if (!src || !twiddle || !out) return atb::fail(ATB_EINVAL, "atb_autocorr_rowmax: null pointer");
  if (nrows < 1 || ncol < 1 || src_row_stride < ncol)
    return atb::fail(ATB_EINVAL, "atb_autocorr_rowmax: bad shape nrows=%d ncol=%d", nrows, ncol);
  const int t = atb_autocorr_length(ncol);
  if (t < 0) return t;
  if (fft_len != t)
    return atb::fail(ATB_EINVAL, "atb_autocorr_rowmax: fft_len=%d, atb_autocorr_length gives %d", fft_len, t);
  const bool half = (t & 1) == 0;
  const int len = half ? t / 2 : t;
  Plan pl;
  if (!make_plan(len, static_cast<const double2 *>(twiddle), pl))
    return atb::fail(ATB_ERANGE, "atb_autocorr_rowmax: no radix plan for length %d", len);
  const size_t smem = (2 * (size_t)len + atb::fft::twiddle_entries(len)) * sizeof(double2);
  const int rc = half ? atb::ensure_smem(autocorr_kernel<true>, smem, "atb_autocorr_rowmax")
                      : atb::ensure_smem(autocorr_kernel<false>, smem, "atb_autocorr_rowmax");
  if (rc != ATB_OK) return rc;
  AcArgs a;
  a.src = src; a.srs = src_row_stride; a.nrows = nrows; a.ncol = ncol;
  a.tw = static_cast<const double2 *>(twiddle); a.out = out;
  if (half)
    autocorr_kernel<true><<<nrows, kThreads, smem, atb::as_stream(stream)>>>(a, pl);
  else
    autocorr_kernel<false><<<nrows, kThreads, smem, atb::as_stream(stream)>>>(a, pl);
  return atb::check_launch("atb_autocorr_rowmax");
}
