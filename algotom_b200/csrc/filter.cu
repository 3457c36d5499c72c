// Fused padded ramp-and-window filter of sinogram rows.
//
// Replaces apply_ramp_filter (algotom/rec/reconstruction.py:118-153), whose
// FFT / shift / window / inverse-FFT / real / crop chain is a real circular
// convolution of the padded row of length N = ncol + 2 pad with a periodic
// kernel kappa, cropped to [pad, pad + ncol).  Those ncol outputs only see
// kernel lags in [pad - N + 1, pad + ncol - 1], so the same numbers come out
// of a circular convolution of any length M >= N + ncol - 1 whose kernel b
// holds kappa at those lags (b[u mod M] = kappa[u mod N]) and zero elsewhere.
// The host builds b's spectrum in FP64 for a power-of-two M; this kernel
// then needs nothing but power-of-two FFTs: radix-16 Stockham stages (and
// one radix-2/4/8 stage) with every thread holding 32 elements in
// registers, twiddles from two short tables in shared memory.
//
// One CTA filters two rows at once: real rows x1, x2 travel as the complex
// row x1 + i x2 through one forward FFT, a product with the (real-kernel)
// spectrum and one inverse FFT (done as conj(FFT(conj(.))) with 1/M folded
// into the spectrum); the real and imaginary parts of the result are the
// two filtered rows.  Each row is read from HBM once (with the -log folded
// in) and written once; padding, both transforms and the spectral product
// stay in shared memory.
#include <cfloat>

#include "common.cuh"

namespace {

constexpr int kMinLog2M = 4;
constexpr int kMaxLog2M = 14;  // 16384 complex (+1/16 padding) = 136 KiB of shared memory

// Shared-memory index of complex element i: one padding word per 16
// elements keeps the strided Stockham writes free of bank conflicts.
__device__ __forceinline__ int pidx(int i) { return i + (i >> 4); }

struct FilterArgs {
  const float *src;
  long long srs, sss;  // src row / slice strides (elements)
  int nrow, nslice, ncol, pad, mode, apply_log;
  const float2 *spec;
  int spec_rows;
  const float2 *tw;
  int log2m;
  void *dst;
  long long drs, dss;
  int pair_within_angle;  // 1: a CTA takes slices 2q, 2q+1 of one angle
  int pairs_per_angle;
};

__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 mul_mi(float2 a) { return make_float2(a.y, -a.x); }  // a * (-i)

// forward DFTs of length 2, 4, 8, 16 in registers (natural order in/out)
__device__ __forceinline__ void dft2(float2 *v) {
  const float2 a = v[0], b = v[1];
  v[0] = cadd(a, b);
  v[1] = csub(a, b);
}
__device__ __forceinline__ void dft4(float2 &v0, float2 &v1, float2 &v2, float2 &v3) {
  const float2 a = cadd(v0, v2), b = csub(v0, v2), c = cadd(v1, v3), d = mul_mi(csub(v1, v3));
  v0 = cadd(a, c);
  v2 = csub(a, c);
  v1 = cadd(b, d);
  v3 = csub(b, d);
}
// exp(-2 pi i m / 16) for m = 1, 2, 3 (cos(pi/8), sin(pi/8), sqrt(1/2))
constexpr float kC1 = 0.92387953251128674f, kS1 = 0.38268343236508978f, kR2 = 0.70710678118654752f;
__device__ __forceinline__ float2 w16_1(float2 a) { return cmul(a, make_float2(kC1, -kS1)); }
__device__ __forceinline__ float2 w16_2(float2 a) { return make_float2(kR2 * (a.x + a.y), kR2 * (a.y - a.x)); }
__device__ __forceinline__ float2 w16_3(float2 a) { return cmul(a, make_float2(kS1, -kC1)); }
__device__ __forceinline__ float2 w16_6(float2 a) { return make_float2(kR2 * (a.y - a.x), -kR2 * (a.x + a.y)); }
__device__ __forceinline__ float2 w16_9(float2 a) { return cmul(a, make_float2(-kC1, kS1)); }
__device__ __forceinline__ void dft8(float2 *v) {
  // 8 = 2 x 4: radix-4 over the even / odd halves, then W8 twiddles
  dft4(v[0], v[2], v[4], v[6]);
  dft4(v[1], v[3], v[5], v[7]);
  const float2 o1 = w16_2(v[3]), o2 = mul_mi(v[5]), o3 = w16_6(v[7]);
  const float2 e0 = v[0], e1 = v[2], e2 = v[4], e3 = v[6], o0 = v[1];
  v[0] = cadd(e0, o0); v[4] = csub(e0, o0);
  v[1] = cadd(e1, o1); v[5] = csub(e1, o1);
  v[2] = cadd(e2, o2); v[6] = csub(e2, o2);
  v[3] = cadd(e3, o3); v[7] = csub(e3, o3);
}
__device__ __forceinline__ void dft16(float2 *v) {
  // 16 = 4 x 4: radix-4 DFTs over n2 (stride 4), W16^(n1 k2) twiddles,
  // radix-4 DFTs over n1; output index k2 + 4 k1
#pragma unroll
  for (int n1 = 0; n1 < 4; ++n1) dft4(v[n1], v[n1 + 4], v[n1 + 8], v[n1 + 12]);
  v[5] = w16_1(v[5]);  v[9] = w16_2(v[9]);  v[13] = w16_3(v[13]);
  v[6] = w16_2(v[6]);  v[10] = mul_mi(v[10]); v[14] = w16_6(v[14]);
  v[7] = w16_3(v[7]);  v[11] = w16_6(v[11]); v[15] = w16_9(v[15]);
  float2 t[16];
#pragma unroll
  for (int k2 = 0; k2 < 4; ++k2) {
    float2 a0 = v[4 * k2], a1 = v[4 * k2 + 1], a2 = v[4 * k2 + 2], a3 = v[4 * k2 + 3];
    dft4(a0, a1, a2, a3);
    t[k2] = a0; t[k2 + 4] = a1; t[k2 + 8] = a2; t[k2 + 12] = a3;
  }
#pragma unroll
  for (int r = 0; r < 16; ++r) v[r] = t[r];
}
template <int R> __device__ __forceinline__ void dft(float2 *v) {
  if constexpr (R == 2) dft2(v);
  else if constexpr (R == 4) dft4(v[0], v[1], v[2], v[3]);
  else if constexpr (R == 8) dft8(v);
  else dft16(v);
}

// Stockham stage of radix R after sub-transforms of length Ns = 2^logNs:
// butterfly j reads x[j + r M/R], twiddles input r by w^(r k)
// (k = j mod Ns, w = exp(-2 pi i / (Ns R))), does an R-point DFT and writes
// output r to x[(j - k) R + k + r Ns].  Every thread reads all of its inputs
// before the barrier and writes after it, so one buffer suffices.
// Twiddles exp(-2 pi i t / M) = ta[t >> L] * tb[t & (2^L - 1)] come from two
// short tables in shared memory.
template <int R, int T>
__device__ __forceinline__ void fft_stage(float2 *x, int log2m, int logNs, const float2 *ta, const float2 *tb,
                                          int L) {
  constexpr int logR = R == 2 ? 1 : (R == 4 ? 2 : (R == 8 ? 3 : 4));
  const int M = 1 << log2m, Q = M >> logR;
  constexpr int kMaxB = 32 / R;  // T >= M / 32 threads: at most 32 elements each
  const int nb = (Q + T - 1) / T;
  const int Ns = 1 << logNs;
  const int tsh = log2m - logR - logNs;
  const int lmask = (1 << L) - 1;
  float2 v[kMaxB][R];
#pragma unroll
  for (int b = 0; b < kMaxB; ++b) {
    const int j = threadIdx.x + b * T;
    if (b < nb && j < Q) {
#pragma unroll
      for (int r = 0; r < R; ++r) v[b][r] = x[pidx(j + r * Q)];
    }
  }
  __syncthreads();
#pragma unroll
  for (int b = 0; b < kMaxB; ++b) {
    const int j = threadIdx.x + b * T;
    if (b < nb && j < Q) {
      const int k = j & (Ns - 1);
      if (k) {
        // w^(r k) for r = 1 .. R-1: the powers 1, 2, 4, 8 of w^k from the
        // tables, each other one the product of those of its set bits (at
        // most three roundings), against 2 (R - 1) table reads per butterfly
        auto tw = [&](int c) {
          const int t = (c * k) << tsh;
          return cmul(ta[t >> L], tb[t & lmask]);
        };
        const float2 w1 = tw(1);
        const float2 w2 = R >= 4 ? tw(2) : w1;
        const float2 w4 = R >= 8 ? tw(4) : w1;
        const float2 w8 = R >= 16 ? tw(8) : w1;
#pragma unroll
        for (int r = 1; r < R; ++r) {
          float2 w = (r & 1) ? w1 : ((r & 2) ? w2 : ((r & 4) ? w4 : w8));
          if ((r & 1) && (r & 2)) w = cmul(w, w2);
          if ((r & 3) && (r & 4)) w = cmul(w, w4);
          if ((r & 7) && (r & 8)) w = cmul(w, w8);
          v[b][r] = cmul(v[b][r], w);
        }
      }
      dft<R>(v[b]);
      const int o = ((j - k) << logR) + k;
#pragma unroll
      for (int r = 0; r < R; ++r) x[pidx(o + r * Ns)] = v[b][r];
    }
  }
  __syncthreads();
}

// In-place forward FFT of length M = 2^log2m: one radix-2/4/8 stage for
// the remainder of log2m / 4, then radix-16 stages.  Force-inlined: called
// from two kernels, the compiler otherwise emits it as a real call whose
// ABI costs a 672-byte stack frame and a third of the filter's speed.
template <int T>
__device__ __forceinline__ void fft_forward(float2 *x, int log2m, const float2 *ta, const float2 *tb, int L) {
  int logNs = 0;
  switch (log2m & 3) {
    case 1: fft_stage<2, T>(x, log2m, 0, ta, tb, L); logNs = 1; break;
    case 2: fft_stage<4, T>(x, log2m, 0, ta, tb, L); logNs = 2; break;
    case 3: fft_stage<8, T>(x, log2m, 0, ta, tb, L); logNs = 3; break;
    default: break;
  }
  for (; logNs < log2m; logNs += 4) fft_stage<16, T>(x, log2m, logNs, ta, tb, L);
}

// Block-wide reduction over T threads (op: 0 sum, 1 max, 2 min).
template <int T>
__device__ float2 block_reduce2(float2 v, int op, float2 *scratch) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    float2 u = make_float2(__shfl_xor_sync(0xffffffffu, v.x, o), __shfl_xor_sync(0xffffffffu, v.y, o));
    if (op == 0) { v.x += u.x; v.y += u.y; }
    else if (op == 1) { v.x = fmaxf(v.x, u.x); v.y = fmaxf(v.y, u.y); }
    else { v.x = fminf(v.x, u.x); v.y = fminf(v.y, u.y); }
  }
  __syncthreads();
  if (lane == 0) scratch[warp] = v;
  __syncthreads();
  if (warp == 0) {
    v = lane < T / 32 ? scratch[lane]
                      : (op == 0 ? make_float2(0.f, 0.f)
                                 : (op == 1 ? make_float2(-FLT_MAX, -FLT_MAX) : make_float2(FLT_MAX, FLT_MAX)));
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      float2 u = make_float2(__shfl_xor_sync(0xffffffffu, v.x, o), __shfl_xor_sync(0xffffffffu, v.y, o));
      if (op == 0) { v.x += u.x; v.y += u.y; }
      else if (op == 1) { v.x = fmaxf(v.x, u.x); v.y = fmaxf(v.y, u.y); }
      else { v.x = fminf(v.x, u.x); v.y = fminf(v.y, u.y); }
    }
    if (lane == 0) scratch[0] = v;
  }
  __syncthreads();
  float2 r = scratch[0];
  __syncthreads();
  return r;
}

// Order-preserving map of a float to an unsigned key.
__device__ __forceinline__ unsigned fkey(float f) {
  unsigned u = __float_as_uint(f);
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float fkey_inv(unsigned k) {
  return __uint_as_float((k & 0x80000000u) ? (k & 0x7fffffffu) : ~k);
}

// Order statistic `rank` (0-based) of each of the two rows held in
// x[pad .. pad+ncol) (.x and .y), by bisection on the float keys.
template <int T>
__device__ float2 block_select2(const float2 *x, int pad, int ncol, int rank, float2 *scratch) {
  unsigned lo1 = 0u, hi1 = 0xffffffffu, lo2 = 0u, hi2 = 0xffffffffu;
  for (int it = 0; it < 32; ++it) {
    const unsigned m1 = lo1 + ((hi1 - lo1) >> 1), m2 = lo2 + ((hi2 - lo2) >> 1);
    float c1 = 0.f, c2 = 0.f;
    for (int j = threadIdx.x; j < ncol; j += T) {
      const float2 v = x[pidx(pad + j)];
      c1 += fkey(v.x) <= m1 ? 1.f : 0.f;
      c2 += fkey(v.y) <= m2 ? 1.f : 0.f;
    }
    const float2 c = block_reduce2<T>(make_float2(c1, c2), 0, scratch);
    if (c.x >= (float)(rank + 1)) hi1 = m1; else lo1 = m1 + 1;
    if (c.y >= (float)(rank + 1)) hi2 = m2; else lo2 = m2 + 1;
  }
  return make_float2(fkey_inv(lo1), fkey_inv(lo2));
}

// Filters row pair `pair` of a (CTA-uniform).
template <typename OutT, int T>
__device__ __forceinline__ void filter_rows_body(const FilterArgs &a, int pair) {
  extern __shared__ float2 sm[];  // M complex, padded by pidx
  __shared__ float2 scratch[T / 32 > 0 ? T / 32 : 1];
  __shared__ float2 ta[128], tb[128];
  const int log2m = a.log2m, M = 1 << log2m;
  const int L = (log2m + 1) >> 1;
  const int ncol = a.ncol, pad = a.pad, N = ncol + 2 * pad;
  const int tid = threadIdx.x;

  // twiddle tables: ta[u] = w^(u 2^L), tb[v] = w^v, w = exp(-2 pi i / M)
  for (int u = tid; u < (M >> L); u += T) ta[u] = __ldg(a.tw + (u << L));
  for (int v = tid; v < (1 << L); v += T) tb[v] = __ldg(a.tw + v);

  // the two rows (angle, slice) of this CTA
  int i1, k1, i2, k2;
  bool ok2;
  if (a.pair_within_angle) {
    i1 = pair / a.pairs_per_angle;
    k1 = 2 * (pair % a.pairs_per_angle);
    i2 = i1;
    k2 = k1 + 1;
    ok2 = k2 < a.nslice;
  } else {
    // rows 2 pair and 2 pair + 1 in [angle][slice] order; the host caps
    // the pairs at 2^31, so the row index fits 32-bit unsigned arithmetic
    // (a 64-bit division here made the kernel spill to the stack)
    const unsigned r1 = 2u * (unsigned)pair, r2 = r1 + 1u, ns = (unsigned)a.nslice;
    i1 = (int)(r1 / ns);
    k1 = (int)(r1 % ns);
    i2 = (int)(r2 / ns);
    k2 = (int)(r2 % ns);
    ok2 = (unsigned long long)r2 < (unsigned long long)a.nrow * (unsigned long long)a.nslice;
  }
  const float *s1 = a.src + i1 * a.srs + k1 * a.sss;
  const float *s2 = a.src + (ok2 ? i2 * a.srs + k2 * a.sss : 0);

  // 1. the two logged rows into the middle of the complex buffer
  for (int j = tid; j < ncol; j += T) {
    float v1 = __ldg(s1 + j);
    float v2 = ok2 ? __ldg(s2 + j) : 0.0f;
    if (a.apply_log) { v1 = atb::neg_log(v1); v2 = ok2 ? atb::neg_log(v2) : 0.0f; }
    sm[pidx(pad + j)] = make_float2(v1, v2);
  }
  for (int m = N + tid; m < M; m += T) sm[pidx(m)] = make_float2(0.f, 0.f);
  __syncthreads();

  // 2. padding (numpy.pad semantics along the row)
  if (pad > 0) {
    float2 stat = make_float2(0.f, 0.f);
    if (a.mode == ATB_PAD_MEAN || a.mode == ATB_PAD_MAXIMUM || a.mode == ATB_PAD_MINIMUM) {
      const int op = a.mode == ATB_PAD_MEAN ? 0 : (a.mode == ATB_PAD_MAXIMUM ? 1 : 2);
      float2 acc = op == 0 ? make_float2(0.f, 0.f)
                           : (op == 1 ? make_float2(-FLT_MAX, -FLT_MAX) : make_float2(FLT_MAX, FLT_MAX));
      for (int j = tid; j < ncol; j += T) {
        const float2 v = sm[pidx(pad + j)];
        if (op == 0) { acc.x += v.x; acc.y += v.y; }
        else if (op == 1) { acc.x = fmaxf(acc.x, v.x); acc.y = fmaxf(acc.y, v.y); }
        else { acc.x = fminf(acc.x, v.x); acc.y = fminf(acc.y, v.y); }
      }
      stat = block_reduce2<T>(acc, op, scratch);
      if (op == 0) { stat.x /= (float)ncol; stat.y /= (float)ncol; }
    } else if (a.mode == ATB_PAD_MEDIAN) {
      const float2 lo = block_select2<T>(sm, pad, ncol, (ncol - 1) / 2, scratch);
      if (ncol & 1) {
        stat = lo;
      } else {
        const float2 hi = block_select2<T>(sm, pad, ncol, ncol / 2, scratch);
        stat = make_float2(0.5f * (lo.x + hi.x), 0.5f * (lo.y + hi.y));
      }
    }
    for (int t = tid; t < 2 * pad; t += T) {
      const bool left = t < pad;
      const int m = left ? t : ncol + t;   // position in the padded row
      const int q = m - pad;               // position relative to the row
      float2 v;
      switch (a.mode) {
        case ATB_PAD_EDGE: v = sm[pidx(pad + (left ? 0 : ncol - 1))]; break;
        case ATB_PAD_CONSTANT: v = make_float2(0.f, 0.f); break;
        case ATB_PAD_WRAP: v = sm[pidx(pad + ((q % ncol) + ncol) % ncol)]; break;
        case ATB_PAD_REFLECT: {
          int r = 0;
          if (ncol > 1) {
            const int P = 2 * (ncol - 1);
            r = ((q % P) + P) % P;
            if (r >= ncol) r = P - r;
          }
          v = sm[pidx(pad + r)];
          break;
        }
        case ATB_PAD_SYMMETRIC: {
          const int P = 2 * ncol;
          int r = ((q % P) + P) % P;
          if (r >= ncol) r = P - 1 - r;
          v = sm[pidx(pad + r)];
          break;
        }
        case ATB_PAD_LINEAR_RAMP: {
          // numpy: linspace(end=0, edge, pad, endpoint=False) on each side
          const float2 e = sm[pidx(pad + (left ? 0 : ncol - 1))];
          const float f = left ? (float)m / (float)pad : (float)(pad - 1 - (q - ncol)) / (float)pad;
          v = make_float2(e.x * f, e.y * f);
          break;
        }
        default: v = stat; break;  // mean / maximum / minimum / median
      }
      sm[pidx(m)] = v;
    }
  }
  __syncthreads();

  // 3. forward transform, spectral product (conjugated), second forward
  //    transform = conjugated inverse
  fft_forward<T>(sm, log2m, ta, tb, L);
  const float2 *spec = a.spec + (a.spec_rows > 1 ? (long long)i1 * M : 0LL);
  for (int k = tid; k < M; k += T) {
    const float2 y = cmul(sm[pidx(k)], __ldg(spec + k));
    sm[pidx(k)] = make_float2(y.x, -y.y);
  }
  __syncthreads();
  fft_forward<T>(sm, log2m, ta, tb, L);

  // 4. crop: real part -> row 1, -imag part -> row 2
  OutT *d1 = reinterpret_cast<OutT *>(a.dst) + i1 * a.drs + k1 * a.dss;
  OutT *d2 = reinterpret_cast<OutT *>(a.dst) + (ok2 ? i2 * a.drs + k2 * a.dss : 0);
  for (int j = tid; j < ncol; j += T) {
    const float2 w = sm[pidx(pad + j)];
    atb::store_from_float(d1 + j, w.x);
    if (ok2) atb::store_from_float(d2 + j, -w.y);
  }
}

template <typename OutT, int T>
__global__ void __launch_bounds__(T, T <= 256 ? 2 : 1) filter_rows_kernel(FilterArgs a) {
  filter_rows_body<OutT, T>(a, (int)blockIdx.x);
}

// One launch over the row pairs of several single-slice sinograms that
// share the FFT length: CTA p finds the item whose pair range holds p
// (binary search on pair_offset) and filters that pair.
template <typename OutT, int T>
__global__ void __launch_bounds__(T, T <= 256 ? 2 : 1)
    filter_batch_kernel(FilterArgs a, const atb_filter_item *items, int nitems) {
  const int p = blockIdx.x;
  int lo = 0, hi = nitems - 1;
  while (lo < hi) {  // last item with pair_offset <= p
    const int mid = (lo + hi + 1) >> 1;
    if (items[mid].pair_offset <= p) lo = mid; else hi = mid - 1;
  }
  const atb_filter_item it = items[lo];
  const int pair = p - it.pair_offset;
  if (pair < 0 || pair >= (it.nrow + 1) / 2) return;  // CTA-uniform
  FilterArgs b = a;
  b.src = it.src; b.srs = it.src_row_stride; b.sss = 0;
  b.nrow = it.nrow; b.nslice = 1; b.ncol = it.ncol; b.pad = it.pad;
  b.spec = reinterpret_cast<const float2 *>(it.spec); b.spec_rows = 1;
  b.dst = it.dst; b.drs = it.dst_row_stride; b.dss = 0;
  b.pair_within_angle = 0;
  b.pairs_per_angle = 0;
  filter_rows_body<OutT, T>(b, pair);
}

__global__ void neg_log_kernel(const float *__restrict__ src, long long srs, long long sss, int nrow,
                               int nslice, int ncol, float *dst, long long drs, long long dss) {
  const long long total = (long long)nrow * nslice * ncol;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    const int j = (int)(t % ncol);
    const long long rk = t / ncol;
    const int k = (int)(rk % nslice), i = (int)(rk / nslice);
    dst[i * drs + k * dss + j] = atb::neg_log(__ldg(src + i * srs + k * sss + j));
  }
}

template <typename OutT, int T>
int launch_filter_t(const FilterArgs &a, long long npairs, cudaStream_t st) {
  const size_t smem = sizeof(float2) * (size_t)((1 << a.log2m) + ((1 << a.log2m) >> 4));
  const int rc = atb::ensure_smem(filter_rows_kernel<OutT, T>, smem, "atb_filter_rows");
  if (rc != ATB_OK) return rc;
  filter_rows_kernel<OutT, T><<<(unsigned)npairs, T, smem, st>>>(a);
  return atb::check_launch("atb_filter_rows");
}

template <typename OutT, int T>
int launch_batch_t(const FilterArgs &a, const atb_filter_item *items, int nitems, int npairs, cudaStream_t st) {
  const size_t smem = sizeof(float2) * (size_t)((1 << a.log2m) + ((1 << a.log2m) >> 4));
  const int rc = atb::ensure_smem(filter_batch_kernel<OutT, T>, smem, "atb_filter_rows_batch");
  if (rc != ATB_OK) return rc;
  filter_batch_kernel<OutT, T><<<(unsigned)npairs, T, smem, st>>>(a, items, nitems);
  return atb::check_launch("atb_filter_rows_batch");
}

template <typename OutT>
int launch_batch(const FilterArgs &a, const atb_filter_item *items, int nitems, int npairs, cudaStream_t st) {
  switch (a.log2m) {
    case 14: return launch_batch_t<OutT, 512>(a, items, nitems, npairs, st);
    case 13: return launch_batch_t<OutT, 256>(a, items, nitems, npairs, st);
    case 12: return launch_batch_t<OutT, 128>(a, items, nitems, npairs, st);
    case 11: return launch_batch_t<OutT, 64>(a, items, nitems, npairs, st);
    default: return launch_batch_t<OutT, 32>(a, items, nitems, npairs, st);
  }
}

// T = max(32, M / 32): every thread holds 32 complex values per stage
template <typename OutT>
int launch_filter(const FilterArgs &a, long long npairs, cudaStream_t st) {
  switch (a.log2m) {
    case 14: return launch_filter_t<OutT, 512>(a, npairs, st);
    case 13: return launch_filter_t<OutT, 256>(a, npairs, st);
    case 12: return launch_filter_t<OutT, 128>(a, npairs, st);
    case 11: return launch_filter_t<OutT, 64>(a, npairs, st);
    default: return launch_filter_t<OutT, 32>(a, npairs, st);
  }
}

}  // namespace

extern "C" {

int atb_filter_log2m(int ncol, int pad) {
  if (ncol < 1 || pad < 0) return atb::fail(ATB_EINVAL, "atb_filter_log2m: ncol=%d pad=%d", ncol, pad);
  const long long need = (long long)ncol + 2LL * pad + ncol - 1;
  int l = kMinLog2M;
  while ((1LL << l) < need) ++l;
  if (l > kMaxLog2M)
    return atb::fail(ATB_ERANGE, "atb_filter_log2m: ncol=%d pad=%d needs FFT length 2^%d > 2^%d", ncol, pad, l,
                     kMaxLog2M);
  return l;
}

int atb_filter_rows(const float *src, int64_t src_row_stride, int64_t src_slice_stride, int nrow, int nslice,
                    int ncol, int pad, int pad_mode, int apply_log, const void *spec, int spec_rows,
                    const void *twiddle, int log2m, void *dst, int dst_dtype, int64_t dst_row_stride,
                    int64_t dst_slice_stride, void *stream) {
  if (!src || !dst || !spec || !twiddle) return atb::fail(ATB_EINVAL, "atb_filter_rows: null pointer");
  if (nrow < 1 || nslice < 1 || ncol < 1 || pad < 0)
    return atb::fail(ATB_EINVAL, "atb_filter_rows: bad shape nrow=%d nslice=%d ncol=%d pad=%d", nrow, nslice,
                     ncol, pad);
  if (pad_mode < ATB_PAD_EDGE || pad_mode > ATB_PAD_MEDIAN)
    return atb::fail(ATB_EINVAL, "atb_filter_rows: unknown pad_mode %d", pad_mode);
  if (log2m < kMinLog2M || log2m > kMaxLog2M)
    return atb::fail(ATB_ERANGE, "atb_filter_rows: log2m=%d outside [%d, %d]", log2m, kMinLog2M, kMaxLog2M);
  if ((1LL << log2m) < (long long)ncol + 2LL * pad + ncol - 1)
    return atb::fail(ATB_EINVAL, "atb_filter_rows: 2^%d < ncol + 2 pad + ncol - 1", log2m);
  if (spec_rows != 1 && spec_rows != nrow)
    return atb::fail(ATB_EINVAL, "atb_filter_rows: spec_rows=%d must be 1 or nrow=%d", spec_rows, nrow);
  FilterArgs a;
  a.src = src; a.srs = src_row_stride; a.sss = src_slice_stride;
  a.nrow = nrow; a.nslice = nslice; a.ncol = ncol; a.pad = pad; a.mode = pad_mode; a.apply_log = apply_log;
  a.spec = reinterpret_cast<const float2 *>(spec); a.spec_rows = spec_rows;
  a.tw = reinterpret_cast<const float2 *>(twiddle); a.log2m = log2m;
  a.dst = dst; a.drs = dst_row_stride; a.dss = dst_slice_stride;
  long long npairs;
  if (spec_rows > 1) {
    a.pair_within_angle = 1;
    a.pairs_per_angle = (nslice + 1) / 2;
    npairs = (long long)nrow * a.pairs_per_angle;
  } else {
    a.pair_within_angle = 0;
    a.pairs_per_angle = 0;
    npairs = ((long long)nrow * nslice + 1) / 2;
  }
  if (npairs > 0x7fffffffLL) return atb::fail(ATB_ERANGE, "atb_filter_rows: too many rows");
  cudaStream_t st = atb::as_stream(stream);
  switch (dst_dtype) {
    case ATB_F32: return launch_filter<float>(a, npairs, st);
    case ATB_F16: return launch_filter<__half>(a, npairs, st);
    case ATB_BF16: return launch_filter<__nv_bfloat16>(a, npairs, st);
    default: return atb::fail(ATB_EINVAL, "atb_filter_rows: unknown dst_dtype %d", dst_dtype);
  }
}

int atb_filter_rows_batch(const atb_filter_item *items, int nitems, int npairs, int pad_mode, int apply_log,
                          const void *twiddle, int log2m, int dst_dtype, void *stream) {
  if (!items || !twiddle) return atb::fail(ATB_EINVAL, "atb_filter_rows_batch: null pointer");
  if (nitems < 1 || npairs < 1) return atb::fail(ATB_EINVAL, "atb_filter_rows_batch: empty batch");
  if (pad_mode < ATB_PAD_EDGE || pad_mode > ATB_PAD_MEDIAN)
    return atb::fail(ATB_EINVAL, "atb_filter_rows_batch: unknown pad_mode %d", pad_mode);
  if (log2m < kMinLog2M || log2m > kMaxLog2M)
    return atb::fail(ATB_ERANGE, "atb_filter_rows_batch: log2m=%d outside [%d, %d]", log2m, kMinLog2M, kMaxLog2M);
  FilterArgs a;
  a.src = nullptr; a.srs = 0; a.sss = 0;
  a.nrow = 0; a.nslice = 1; a.ncol = 0; a.pad = 0; a.mode = pad_mode; a.apply_log = apply_log;
  a.spec = nullptr; a.spec_rows = 1;
  a.tw = reinterpret_cast<const float2 *>(twiddle); a.log2m = log2m;
  a.dst = nullptr; a.drs = 0; a.dss = 0;
  a.pair_within_angle = 0;
  a.pairs_per_angle = 0;
  cudaStream_t st = atb::as_stream(stream);
  switch (dst_dtype) {
    case ATB_F32: return launch_batch<float>(a, items, nitems, npairs, st);
    case ATB_F16: return launch_batch<__half>(a, items, nitems, npairs, st);
    case ATB_BF16: return launch_batch<__nv_bfloat16>(a, items, nitems, npairs, st);
    default: return atb::fail(ATB_EINVAL, "atb_filter_rows_batch: unknown dst_dtype %d", dst_dtype);
  }
}

int atb_neg_log(const float *src, int64_t src_row_stride, int64_t src_slice_stride, int nrow, int nslice, int ncol,
                float *dst, int64_t dst_row_stride, int64_t dst_slice_stride, void *stream) {
  if (!src || !dst) return atb::fail(ATB_EINVAL, "atb_neg_log: null pointer");
  if (nrow < 1 || nslice < 1 || ncol < 1) return atb::fail(ATB_EINVAL, "atb_neg_log: bad shape");
  const long long total = (long long)nrow * nslice * ncol;
  long long blocks = (total + 255) / 256;
  if (blocks > 148LL * 32) blocks = 148LL * 32;
  neg_log_kernel<<<(unsigned)blocks, 256, 0, atb::as_stream(stream)>>>(
      src, src_row_stride, src_slice_stride, nrow, nslice, ncol, dst, dst_row_stride, dst_slice_stride);
  return atb::check_launch("atb_neg_log");
}

}  // extern "C"
