// The Fourier transforms of direct Fourier inversion (dfi_reconstruction,
// algotom/rec/reconstruction.py:752-907), sm_100a, FP64.
//
// The reference pads every centred sinogram row (np.pad, :774-776), takes
// -log (:885-890), transforms it (fftshift(fft(ifftshift(row))) times the
// window, :767-770), regrids the polar spectrum (:776-785) and inverts it
// (fftshift(ifft2(.)), :786-787), at the padded width w = ncol1 + 2 pad
// that its algorithm fixes: 3841 = 23 x 167 at 2560 detector pixels, a
// length without small factors.  Both transforms run here as Bluestein
// transforms: with b_m = exp(i pi m^2 / w),
//     X_k = conj(b_k) sum_n (x_n conj(b_n)) b_(k-n),
// a circular convolution of length M >= 2 w - 1 (a power of two) computed
// with this library's in-place FFT (atb::fft::ip_run) in one shared-memory
// buffer: forward transform (digit-reversed order), product with the
// chirp's transform (made once per w by the same code, so the orders
// match), inverse transform.  The inverse DFT uses the conjugate chirp.
//
// Three kernels, each one CTA per transform:
// - dfi_rows_kernel: two sinogram rows per complex transform (the spectra
//   of real rows a and b separate as the Hermitian and anti-Hermitian parts
//   of the transform of a + i b), with the padding (NumPy's ten modes), the
//   -log (values <= 0 give 0 and are counted, the reference's warning), the
//   ifftshift, the fftshift and the window in the same pass;
// - dfi_inv_rows_kernel: rows k and -k of the Cartesian spectrum,
//   regridded on the fly from the B-spline coefficients of the polar
//   spectrum (dfi_grid.cuh) in ifftshift order; one inverse transform of
//   the Hermitian part's row k gives both rows' transforms (the output is
//   the real part, which only the Hermitian part feeds); only the ncol
//   columns the final crop keeps are stored;
// - dfi_inv_cols_kernel: two of those columns per transform (the real
//   parts of the inverses of z1 and z2 are the real and imaginary parts of
//   the inverse of H(z1) + i H(z2), H the Hermitian part), the ncol rows
//   the crop keeps, / w^2, circle mask, float64 or float32 out.
#include <cmath>

#include "common.cuh"
#include "dfi_grid.cuh"
#include "fft.cuh"

namespace {

using atb::fft::cmul;
using atb::fft::cmulc;
using atb::fft::IpPlan;

constexpr int kThreads = 512;
constexpr int kMaxM = 8192;  // one buffer of M complex doubles + twiddles in 227 KB

struct Tables {
  const double2 *chirp;  // [w] b_m = exp(i pi m^2 / w)
  const double2 *tw;     // [M] exp(-2 pi i m / M)
  const double2 *bfwd;   // [M] forward transform of the chirp kernel / M (digit-reversed)
  const double2 *binv;   // [M] the same for the conjugate chirp
};

// x[0 .. w) holds the input (natural order) on entry and its DFT (inverse
// DFT, unnormalised, when INV) on return; x[w .. M) is scratch.  Every
// thread calls it after a barrier; a barrier follows.
template <bool INV>
__device__ void bluestein(double2 *x, int w, const IpPlan &pl, const double2 *tws, const Tables &t) {
  const int M = pl.n;
  for (int n = threadIdx.x; n < M; n += blockDim.x) {
    if (n < w) {
      const double2 b = __ldg(t.chirp + n);
      x[n] = INV ? cmul(x[n], b) : cmulc(x[n], b);
    } else {
      x[n] = make_double2(0.0, 0.0);
    }
  }
  __syncthreads();
  atb::fft::ip_run<false>(x, pl, tws);
  const double2 *B = INV ? t.binv : t.bfwd;
  for (int p = threadIdx.x; p < M; p += blockDim.x) x[p] = cmul(x[p], __ldg(B + p));
  __syncthreads();
  atb::fft::ip_run<true>(x, pl, tws);
  for (int k = threadIdx.x; k < w; k += blockDim.x) {
    const double2 b = __ldg(t.chirp + k);
    x[k] = INV ? cmul(x[k], b) : cmulc(x[k], b);
  }
  __syncthreads();
}

// bfwd / binv: the chirp kernel bb (bb[m] = b_m for m < w, bb[M - m] = b_m
// for 0 < m < w, else 0) and its conjugate, forward-transformed in place,
// divided by M.  blockIdx.x 0: bfwd, 1: binv.
__global__ void __launch_bounds__(kThreads) chirp_setup_kernel(int w, const __grid_constant__ IpPlan pl, Tables t,
                                                               double2 *bfwd, double2 *binv) {
  extern __shared__ double2 sm[];
  const int M = pl.n;
  double2 *tws = sm + M;
  atb::fft::load_twiddles_n(t.tw, M, tws);
  const bool conj = blockIdx.x == 1;
  for (int m = threadIdx.x; m < M; m += blockDim.x) {
    double2 v = make_double2(0.0, 0.0);
    if (m < w) v = __ldg(t.chirp + m);
    else if (M - m < w) v = __ldg(t.chirp + (M - m));
    if (conj) v.y = -v.y;
    sm[m] = v;
  }
  __syncthreads();
  atb::fft::ip_run<false>(sm, pl, tws);
  double2 *out = conj ? binv : bfwd;
  const double s = 1.0 / (double)M;
  for (int p = threadIdx.x; p < M; p += blockDim.x) out[p] = make_double2(sm[p].x * s, sm[p].y * s);
}

// ---- padding (np.pad(row, pad, mode), numpy's ten modes, float32)

struct RowsArgs {
  const float *src;  // rows of n samples: row r of slice k at src + k sss + r srs
  long long srs, sss;
  int nrow, n, pad, mode, apply_log;
  const double *window;  // [w] or null
  int *nonpositive;      // += padded values <= 0 (apply_log), or null
  double2 *dst;          // row r of slice k at dst + k dss + r drs, w values
  long long drs, dss;
};

__device__ __forceinline__ float padded(const float *x, int p, const RowsArgs &a, float stat) {
  const int n = a.n, i = p - a.pad;
  if (i >= 0 && i < n) return __ldg(x + i);
  switch (a.mode) {
    case ATB_PAD_EDGE: return __ldg(x + (i < 0 ? 0 : n - 1));
    case ATB_PAD_CONSTANT: return 0.0f;
    case ATB_PAD_WRAP: {
      const int r = i % n;
      return __ldg(x + (r < 0 ? r + n : r));
    }
    case ATB_PAD_SYMMETRIC: {
      const int q = 2 * n;
      int r = i % q;
      if (r < 0) r += q;
      return __ldg(x + (r >= n ? q - 1 - r : r));
    }
    case ATB_PAD_REFLECT: {
      if (n == 1) return __ldg(x);
      const int q = 2 * (n - 1);
      int r = i % q;
      if (r < 0) r += q;
      return __ldg(x + (r >= n ? q - r : r));
    }
    case ATB_PAD_LINEAR_RAMP: {
      // np.linspace(0, edge, pad, endpoint=False) in float32: k * (edge / pad);
      // reversed on the right
      const float step = (i < 0 ? __ldg(x) : __ldg(x + n - 1)) / (float)a.pad;
      const int k = i < 0 ? p : a.pad - 1 - (i - n);
      return (float)k * step;
    }
    default: return stat;  // mean, maximum, minimum, median of the row
  }
}

// ascending bitonic sort of v[0 .. total) as independent segments of seg
// (a power of two) values
__device__ void sort_segments(float *v, int total, int seg) {
  for (int size = 2; size <= seg; size <<= 1) {
    for (int stride = size >> 1; stride > 0; stride >>= 1) {
      for (int i = threadIdx.x; i < total; i += blockDim.x) {
        const int j = i ^ stride;
        if (j > i) {
          const bool up = (i & (seg - 1) & size) == 0;
          const float vi = v[i], vj = v[j];
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

// statistic of each of the (one or two) rows into stat[0..1]; scratch: the
// transform buffer as floats.  Every thread calls it; a barrier follows.
__device__ void row_stats(const float *xa, const float *xb, const RowsArgs &a, float *scratch, float *stat,
                          double *red) {
  const int n = a.n;
  if (a.mode == ATB_PAD_MEDIAN) {
    int seg = 1;
    while (seg < n) seg <<= 1;
    for (int i = threadIdx.x; i < 2 * seg; i += blockDim.x) {
      const int r = i >= seg, c = i - r * seg;
      const float *x = r ? xb : xa;
      scratch[i] = (c < n && x) ? __ldg(x + c) : INFINITY;
    }
    __syncthreads();
    sort_segments(scratch, 2 * seg, seg);
    if (threadIdx.x < 2) {
      const float *s = scratch + threadIdx.x * seg;
      stat[threadIdx.x] = 0.5f * (s[(n - 1) / 2] + s[n / 2]);
    }
    __syncthreads();
    return;
  }
  const int op = a.mode == ATB_PAD_MEAN ? 0 : (a.mode == ATB_PAD_MAXIMUM ? 1 : 2);
  double acc[2];
  for (int r = 0; r < 2; ++r) {
    const float *x = r ? xb : xa;
    double v = op == 0 ? 0.0 : (op == 1 ? -INFINITY : INFINITY);
    if (x) {
      for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const double u = (double)__ldg(x + i);
        v = op == 0 ? v + u : (op == 1 ? fmax(v, u) : fmin(v, u));
      }
    }
    for (int o = 16; o > 0; o >>= 1) {
      const double u = __shfl_down_sync(0xffffffffu, v, o);
      v = op == 0 ? v + u : (op == 1 ? fmax(v, u) : fmin(v, u));
    }
    acc[r] = v;
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  if (lane == 0) {
    red[warp] = acc[0];
    red[32 + warp] = acc[1];
  }
  __syncthreads();
  if (threadIdx.x < 2) {
    double v = red[threadIdx.x * 32];
    for (int k = 1; k < nw; ++k) {
      const double u = red[threadIdx.x * 32 + k];
      v = op == 0 ? v + u : (op == 1 ? fmax(v, u) : fmin(v, u));
    }
    stat[threadIdx.x] = (float)(op == 0 ? v / (double)n : v);
  }
  __syncthreads();
}

// rows 2 blockIdx.x and 2 blockIdx.x + 1 of slice blockIdx.y
__global__ void __launch_bounds__(kThreads) dfi_rows_kernel(const __grid_constant__ RowsArgs a,
                                                            const __grid_constant__ IpPlan pl, Tables t) {
  extern __shared__ double2 sm[];
  __shared__ float stat[2];
  __shared__ double red[64];
  const int M = pl.n, w = a.n + 2 * a.pad, h = w / 2;
  double2 *tws = sm + M;
  atb::fft::load_twiddles_n(t.tw, M, tws);
  const int r0 = 2 * blockIdx.x, k = blockIdx.y;
  const bool two = r0 + 1 < a.nrow;
  const float *xa = a.src + k * a.sss + r0 * a.srs;
  const float *xb = two ? xa + a.srs : nullptr;
  if (a.pad > 0 && a.mode >= ATB_PAD_MEAN) {
    row_stats(xa, xb, a, reinterpret_cast<float *>(sm), stat, red);
  } else if (threadIdx.x < 2) {
    stat[threadIdx.x] = 0.0f;
  }
  __syncthreads();
  int bad = 0;
  for (int m = threadIdx.x; m < w; m += blockDim.x) {
    const int p = m + h >= w ? m + h - w : m + h;  // ifftshift: y_m = xpad[(m + w/2) mod w]
    float va = padded(xa, p, a, stat[0]);
    float vb = two ? padded(xb, p, a, stat[1]) : 0.0f;
    if (a.apply_log) {
      bad += (va <= 0.0f) + (two && vb <= 0.0f);
      va = atb::neg_log(va);
      vb = two ? atb::neg_log(vb) : 0.0f;
    }
    sm[m] = make_double2((double)va, (double)vb);
  }
  if (a.apply_log && a.nonpositive) {
    bad = __reduce_add_sync(0xffffffffu, bad);
    if ((threadIdx.x & 31) == 0 && bad) atomicAdd(a.nonpositive, bad);
  }
  __syncthreads();
  bluestein<false>(sm, w, pl, tws, t);
  // spectra of the two rows from Y = DFT(a + i b): A_k = (Y_k + conj Y_-k) / 2,
  // B_k = (Y_k - conj Y_-k) / 2i; fftshift: out[q] = X[(q - w/2) mod w]
  double2 *oa = a.dst + k * a.dss + r0 * a.drs;
  double2 *ob = oa + a.drs;
  for (int q = threadIdx.x; q < w; q += blockDim.x) {
    const int m = q - h < 0 ? q - h + w : q - h, mm = m == 0 ? 0 : w - m;
    const double2 Y = sm[m], Z = sm[mm];
    double2 A = make_double2(0.5 * (Y.x + Z.x), 0.5 * (Y.y - Z.y));
    double2 B = make_double2(0.5 * (Y.y + Z.y), 0.5 * (Z.x - Y.x));
    if (a.window) {
      const double g = __ldg(a.window + q);
      A.x *= g;
      A.y *= g;
      B.x *= g;
      B.y *= g;
    }
    oa[q] = A;
    if (two) ob[q] = B;
  }
}

// crop index of the fftshifted inverse: output a <- inverse[(pad + a - w/2) mod w]
__device__ __forceinline__ int crop_index(int a, int pad, int w) {
  int m = (pad + a - w / 2) % w;
  return m < 0 ? m + w : m;
}

struct InvArgs {
  const double2 *coef;  // polar B-spline coefficients: row r of slice k at coef + k css + r crs
  long long crs, css;
  int nrow, w, pad, ncol;
  double2 *z;           // [slice][w][ncol] pass-1 result
  double mask_r2;       // < 0: no mask; centre ncol / 2
  void *out;            // pixel (a, b) of slice k at out + k oss + a ors + b
  long long ors, oss;
  int out_f32;
};

// pass 1: rows oi and w - oi (oi <= w / 2) of the (ifftshift-ordered)
// Cartesian spectrum G of slice blockIdx.y, regridded into shared memory.
// The output is Re(IDFT2(G)) = IDFT2(U) with U = (G + conj G(-k)) / 2, and
// U is Hermitian, so the inverse row transform of U's row -oi is the
// conjugate of that of its row oi: one transform per pair of rows.
__global__ void __launch_bounds__(kThreads) dfi_inv_rows_kernel(const __grid_constant__ InvArgs a,
                                                                const __grid_constant__ IpPlan pl, Tables t) {
  extern __shared__ double2 sm[];
  const int M = pl.n, w = a.w, oi = blockIdx.x, k = blockIdx.y;
  const int oi2 = oi == 0 ? 0 : w - oi;
  double2 *tws = sm + M;
  atb::fft::load_twiddles_n(t.tw, M, tws);
  auto grid_row = [&](int o) { return o + w / 2 >= w ? o + w / 2 - w : o + w / 2; };
  const int i = grid_row(oi), i2 = grid_row(oi2);
  const double2 *coef = a.coef + k * a.css;
  // rows oi and -oi (2 w <= M: the second one in sm[w .. 2 w))
  for (int t2 = threadIdx.x; t2 < 2 * w; t2 += blockDim.x) {
    const int second = t2 >= w, oj = t2 - second * w;
    sm[t2] = atb::dfi::regrid_point(coef, a.crs, a.nrow, w, second ? i2 : i, grid_row(oj));
  }
  __syncthreads();
  // U[oi][oj] = (G[oi][oj] + conj G[-oi][-oj]) / 2, in place (thread per oj)
  for (int oj = threadIdx.x; oj < w; oj += blockDim.x) {
    const double2 g = sm[oj], h = sm[w + (oj == 0 ? 0 : w - oj)];
    sm[oj] = make_double2(0.5 * (g.x + h.x), 0.5 * (g.y - h.y));
  }
  __syncthreads();
  bluestein<true>(sm, w, pl, tws, t);
  double2 *out = a.z + ((long long)k * w + oi) * a.ncol;
  double2 *out2 = a.z + ((long long)k * w + oi2) * a.ncol;
  for (int b = threadIdx.x; b < a.ncol; b += blockDim.x) {
    const double2 v = sm[crop_index(b, a.pad, w)];
    out[b] = v;
    if (oi2 != oi) out2[b] = make_double2(v.x, -v.y);
  }
}

// pass 2: columns 2 blockIdx.x and 2 blockIdx.x + 1 of slice blockIdx.y
__global__ void __launch_bounds__(kThreads) dfi_inv_cols_kernel(const __grid_constant__ InvArgs a,
                                                                const __grid_constant__ IpPlan pl, Tables t) {
  extern __shared__ double2 sm[];
  const int M = pl.n, w = a.w, ncol = a.ncol, b0 = 2 * blockIdx.x, k = blockIdx.y;
  const bool two = b0 + 1 < ncol;
  double2 *tws = sm + M;
  atb::fft::load_twiddles_n(t.tw, M, tws);
  const double2 *z = a.z + (long long)k * w * ncol + b0;
  for (int n = threadIdx.x; n < w; n += blockDim.x) {
    const double2 *p = z + (long long)n * ncol;
    sm[n] = p[0];
    sm[w + n] = two ? p[1] : make_double2(0.0, 0.0);
  }
  __syncthreads();
  // u = H(z1) + i H(z2), H(z)_k = (z_k + conj z_-k) / 2; thread per pair (k, w - k)
  for (int q = threadIdx.x; q <= w / 2; q += blockDim.x) {
    const int qq = q == 0 ? 0 : w - q;
    const double2 p1 = sm[q], m1 = sm[qq], p2 = sm[w + q], m2 = sm[w + qq];
    sm[q] = make_double2(0.5 * ((p1.x + m1.x) - (p2.y - m2.y)), 0.5 * ((p1.y - m1.y) + (p2.x + m2.x)));
    if (qq != q)
      sm[qq] = make_double2(0.5 * ((m1.x + p1.x) - (m2.y - p2.y)), 0.5 * ((m1.y - p1.y) + (m2.x + p2.x)));
  }
  __syncthreads();
  bluestein<true>(sm, w, pl, tws, t);
  const double s = 1.0 / ((double)w * (double)w);
  const int c = ncol / 2;
  const double dx1 = (double)(b0 - c), dx2 = (double)(b0 + 1 - c);
  for (int r = threadIdx.x; r < ncol; r += blockDim.x) {
    const double dy = (double)(r - c);
    const double2 v = sm[crop_index(r, a.pad, w)];
    const bool in1 = a.mask_r2 < 0.0 || dx1 * dx1 + dy * dy <= a.mask_r2;
    const bool in2 = a.mask_r2 < 0.0 || dx2 * dx2 + dy * dy <= a.mask_r2;
    const double v1 = in1 ? v.x * s : 0.0, v2 = in2 ? v.y * s : 0.0;
    const long long o = k * a.oss + r * a.ors + b0;
    if (a.out_f32) {
      float *out = static_cast<float *>(a.out) + o;
      out[0] = (float)v1;
      if (two) out[1] = (float)v2;
    } else {
      double *out = static_cast<double *>(a.out) + o;
      out[0] = v1;
      if (two) out[1] = v2;
    }
  }
}

bool plan_for(int w, IpPlan &pl, int &M) {
  M = 16;
  while (M < 2 * w - 1) M <<= 1;
  return M <= kMaxM && atb::fft::ip_radices(M, pl);
}

size_t smem_bytes(int M) { return ((size_t)M + (size_t)atb::fft::twiddle_entries(M)) * sizeof(double2); }

int prepare(int w, const char *what, IpPlan &pl, int &M) {
  if (w < 2) return atb::fail(ATB_EINVAL, "%s: width %d", what, w);
  if (!plan_for(w, pl, M))
    return atb::fail(ATB_ERANGE, "%s: width %d needs a transform of more than %d points", what, w, kMaxM);
  const size_t sm = smem_bytes(M);
  int rc = atb::ensure_smem(chirp_setup_kernel, sm, what);
  if (rc == ATB_OK) rc = atb::ensure_smem(dfi_rows_kernel, sm, what);
  if (rc == ATB_OK) rc = atb::ensure_smem(dfi_inv_rows_kernel, sm, what);
  if (rc == ATB_OK) rc = atb::ensure_smem(dfi_inv_cols_kernel, sm, what);
  return rc;
}

Tables tables(const void *chirp, const void *twiddle, const void *bfwd, const void *binv) {
  return Tables{static_cast<const double2 *>(chirp), static_cast<const double2 *>(twiddle),
                static_cast<const double2 *>(bfwd), static_cast<const double2 *>(binv)};
}

}  // namespace

extern "C" int atb_dfi_fft_length(int w) {
  IpPlan pl;
  int M = 0;
  if (w < 2) return atb::fail(ATB_EINVAL, "atb_dfi_fft_length: width %d", w);
  if (!plan_for(w, pl, M))
    return atb::fail(ATB_ERANGE, "atb_dfi_fft_length: width %d needs more than %d points", w, kMaxM);
  return M;
}

extern "C" int atb_dfi_fft_setup(int w, const void *chirp, const void *twiddle, void *bfwd, void *binv,
                                 void *stream) {
  if (!chirp || !twiddle || !bfwd || !binv) return atb::fail(ATB_EINVAL, "atb_dfi_fft_setup: null pointer");
  IpPlan pl;
  int M = 0;
  const int rc = prepare(w, "atb_dfi_fft_setup", pl, M);
  if (rc != ATB_OK) return rc;
  chirp_setup_kernel<<<2, kThreads, smem_bytes(M), atb::as_stream(stream)>>>(
      w, pl, tables(chirp, twiddle, nullptr, nullptr), static_cast<double2 *>(bfwd), static_cast<double2 *>(binv));
  return atb::check_launch("atb_dfi_fft_setup");
}

extern "C" int atb_dfi_rows(const float *src, int64_t src_row_stride, int64_t src_slice_stride, int nrow,
                            int nslice, int n, int pad, int pad_mode, int apply_log, const double *window,
                            int *nonpositive, const void *chirp, const void *twiddle, const void *bfwd,
                            const void *binv, void *dst, int64_t dst_row_stride, int64_t dst_slice_stride,
                            void *stream) {
  if (!src || !dst || !chirp || !twiddle || !bfwd || !binv) return atb::fail(ATB_EINVAL, "atb_dfi_rows: null pointer");
  if (nrow < 1 || nslice < 1 || nslice > 65535 || n < 1 || pad < 0)
    return atb::fail(ATB_EINVAL, "atb_dfi_rows: bad shape nrow=%d nslice=%d n=%d pad=%d", nrow, nslice, n, pad);
  if (pad_mode < ATB_PAD_EDGE || pad_mode > ATB_PAD_MEDIAN)
    return atb::fail(ATB_EINVAL, "atb_dfi_rows: pad_mode %d", pad_mode);
  const int w = n + 2 * pad;
  IpPlan pl;
  int M = 0;
  const int rc = prepare(w, "atb_dfi_rows", pl, M);
  if (rc != ATB_OK) return rc;
  cudaStream_t st = atb::as_stream(stream);
  if (apply_log && nonpositive && cudaMemsetAsync(nonpositive, 0, sizeof(int), st) != cudaSuccess)
    return atb::check_launch("atb_dfi_rows (counter)");
  RowsArgs a;
  a.src = src; a.srs = src_row_stride; a.sss = src_slice_stride;
  a.nrow = nrow; a.n = n; a.pad = pad; a.mode = pad_mode; a.apply_log = apply_log ? 1 : 0;
  a.window = window; a.nonpositive = nonpositive;
  a.dst = static_cast<double2 *>(dst); a.drs = dst_row_stride; a.dss = dst_slice_stride;
  const dim3 grid((nrow + 1) / 2, nslice);
  dfi_rows_kernel<<<grid, kThreads, smem_bytes(M), st>>>(a, pl, tables(chirp, twiddle, bfwd, binv));
  return atb::check_launch("atb_dfi_rows");
}

extern "C" int64_t atb_dfi_inverse_workspace(int w, int ncol, int nslice) {
  if (w < 2 || ncol < 1 || ncol > w || nslice < 1)
    return atb::fail(ATB_EINVAL, "atb_dfi_inverse_workspace: w=%d ncol=%d nslice=%d", w, ncol, nslice);
  return (int64_t)nslice * w * ncol * (int64_t)sizeof(double2);
}

extern "C" int atb_dfi_inverse(const void *coef, int64_t coef_row_stride, int64_t coef_slice_stride, int nrow,
                               int nslice, int w, int pad, int ncol, double mask_r2, const void *chirp,
                               const void *twiddle, const void *bfwd, const void *binv, void *out,
                               int64_t out_row_stride, int64_t out_slice_stride, int out_f32, void *workspace,
                               int64_t workspace_bytes, void *stream) {
  if (!coef || !out || !chirp || !twiddle || !bfwd || !binv || !workspace)
    return atb::fail(ATB_EINVAL, "atb_dfi_inverse: null pointer");
  if (nrow < 1 || nslice < 1 || nslice > 65535)
    return atb::fail(ATB_EINVAL, "atb_dfi_inverse: bad shape nrow=%d nslice=%d", nrow, nslice);
  if (ncol < 1 || pad < 0 || pad + ncol > w)
    return atb::fail(ATB_EINVAL, "atb_dfi_inverse: crop [%d, %d) outside width %d", pad, pad + ncol, w);
  const int64_t need = (int64_t)nslice * w * ncol * (int64_t)sizeof(double2);
  if (workspace_bytes < need)
    return atb::fail(ATB_EINVAL, "atb_dfi_inverse: workspace of %lld bytes needed", (long long)need);
  IpPlan pl;
  int M = 0;
  const int rc = prepare(w, "atb_dfi_inverse", pl, M);
  if (rc != ATB_OK) return rc;
  InvArgs a;
  a.coef = static_cast<const double2 *>(coef); a.crs = coef_row_stride; a.css = coef_slice_stride;
  a.nrow = nrow; a.w = w; a.pad = pad; a.ncol = ncol;
  a.z = static_cast<double2 *>(workspace); a.mask_r2 = mask_r2;
  a.out = out; a.ors = out_row_stride; a.oss = out_slice_stride; a.out_f32 = out_f32 ? 1 : 0;
  const Tables t = tables(chirp, twiddle, bfwd, binv);
  cudaStream_t st = atb::as_stream(stream);
  dfi_inv_rows_kernel<<<dim3(w / 2 + 1, nslice), kThreads, smem_bytes(M), st>>>(a, pl, t);
  const int r = atb::check_launch("atb_dfi_inverse (rows)");
  if (r != ATB_OK) return r;
  dfi_inv_cols_kernel<<<dim3((ncol + 1) / 2, nslice), kThreads, smem_bytes(M), st>>>(a, pl, t);
  return atb::check_launch("atb_dfi_inverse (columns)");
}
