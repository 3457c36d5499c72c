// Fused padded ramp-and-window filter of sinogram rows.
//
// Replaces apply_ramp_filter (algotom/rec/reconstruction.py:118-153), whose
// FFT / shift / window / inverse-FFT / real / crop chain is a real circular
// convolution of the padded row of length N = ncol + 2 pad with a periodic
// kernel kappa, cropped to [pad, pad + ncol).  The transform length n is
// the cheaper of two exact forms (by a flop count of the stages):
// - n = N itself when N has no prime factor above 13 (2860 = 4 5 11 13 at
//   2560 detector pixels and the reference's pad of 150), the reference's
//   own transform length;
// - otherwise the smallest 7-smooth n >= N + ncol - 1: the ncol outputs
//   only see kernel lags in [pad - N + 1, pad + ncol - 1], so a circular
//   convolution of that length whose kernel holds kappa at those lags
//   (b[u mod n] = kappa[u mod N]) and zero elsewhere gives the same numbers.
// The host builds the kernel's spectrum in FP64.  The transforms are
// mixed-radix Stockham FFTs in FP32 (radices 16, 8, 4, 2, 13, 11, 7, 5, 3),
// every thread holding its butterflies' inputs in registers across a
// barrier so one shared-memory buffer suffices; twiddles come from two
// short tables in shared memory.
//
// One CTA filters two rows at once: real rows x1, x2 travel as the complex
// row x1 + i x2 through one forward FFT, a product with the (real-kernel)
// spectrum and one inverse FFT (done as conj(FFT(conj(.))) with 1/n folded
// into the spectrum); the real and imaginary parts of the result are the
// two filtered rows.  Each row is read from HBM once (with the -log folded
// in) and written once; padding, both transforms and the spectral product
// stay in shared memory.
#include <algorithm>
#include <cfloat>
#include <cmath>

#include "common.cuh"

namespace {

constexpr int kMaxLen = 16384;  // 16384 complex (+1/16 padding) = 136 KiB of shared memory
constexpr int kMaxStages = 14;
constexpr int kTwLo = 64;       // two-level twiddle tables: w^t = ta[t / 64] tb[t % 64]

// Shared-memory index of complex element i: one padding word per 16
// elements keeps the strided Stockham writes free of bank conflicts.
__device__ __forceinline__ int pidx(int i) { return i + (i >> 4); }

// What every CTA of a launch shares: the transform plan and the pad / log
// settings (read from parameter space; the plan arrays are indexed at run
// time, so kernels take it as a __grid_constant__ parameter).
struct FilterPlan {
  int mode, apply_log;
  const float2 *tw;    // [n] exp(-2 pi i t / n)
  int n, nstages;      // transform length and its radices, in stage order
  int radix[kMaxStages];
  float2 rc[5][6];     // (cos, sin)(2 pi q / p), q = 1 .. (p-1)/2, p = 3, 5, 7, 11, 13
};

// The rows one launch (or one batch item) filters.
struct FilterRows {
  const float *src;
  long long srs, sss;  // src row / slice strides (elements)
  int nrow, nslice, ncol, pad;
  const float2 *spec;
  int spec_rows;
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
// odd P, forward: y_q = A_q - i B_q, y_{P-q} = A_q + i B_q with
// A_q = v_0 + sum_r (v_r + v_{P-r}) cos(2 pi q r / P),
// B_q = sum_r (v_r - v_{P-r}) sin(2 pi q r / P)
template <int P>
__device__ __forceinline__ void dft_odd(float2 *v, const float2 *rc) {
  constexpr int H = (P - 1) / 2;
  float2 s[H], d[H];
  const float2 v0 = v[0];
  float2 y0 = v0;
#pragma unroll
  for (int r = 1; r <= H; ++r) {
    s[r - 1] = cadd(v[r], v[P - r]);
    d[r - 1] = csub(v[r], v[P - r]);
    y0 = cadd(y0, s[r - 1]);
  }
  v[0] = y0;
#pragma unroll
  for (int q = 1; q <= H; ++q) {
    float2 A = v0, B = make_float2(0.f, 0.f);
#pragma unroll
    for (int r = 1; r <= H; ++r) {
      int t = (q * r) % P;
      float sg = 1.f;
      if (t > H) {  // sin(2 pi t / P) = -sin(2 pi (P - t) / P)
        t = P - t;
        sg = -1.f;
      }
      const float c = rc[t - 1].x, sn = sg * rc[t - 1].y;
      A.x = fmaf(s[r - 1].x, c, A.x);
      A.y = fmaf(s[r - 1].y, c, A.y);
      B.x = fmaf(d[r - 1].x, sn, B.x);
      B.y = fmaf(d[r - 1].y, sn, B.y);
    }
    v[q] = make_float2(A.x + B.y, A.y - B.x);      // A - i B
    v[P - q] = make_float2(A.x - B.y, A.y + B.x);  // A + i B
  }
}
template <int R> __device__ __forceinline__ void dft(float2 *v, const float2 *rc) {
  if constexpr (R == 2) dft2(v);
  else if constexpr (R == 4) dft4(v[0], v[1], v[2], v[3]);
  else if constexpr (R == 8) dft8(v);
  else if constexpr (R == 16) dft16(v);
  else dft_odd<R>(v, rc);
}

__host__ __device__ constexpr int odd_slot(int p) { return p == 3 ? 0 : p == 5 ? 1 : p == 7 ? 2 : p == 11 ? 3 : 4; }

// butterflies a thread holds per stage of radix R (at most ~32 values)
__host__ __device__ constexpr int max_butterflies(int r) { return r >= 11 ? 2 : (r >= 5 ? 4 : 32 / r); }

// Stockham stage of radix R after sub-transforms of length Ns: butterfly
// j (< Q = n / R) reads x[j + r Q], twiddles input r by w^(r k)
// (k = j mod Ns, w = exp(-2 pi i / (Ns R))), does an R-point DFT and writes
// output q to x[(j - k) R + k + q Ns].  Every thread reads all of its
// inputs before the barrier and writes after it, so one buffer suffices.
// Twiddles exp(-2 pi i t / n) = ta[t / 64] * tb[t % 64] come from two short
// tables in shared memory; w^r is the product of the table values of the
// powers 1, 2, 4, 8 in r (at most three roundings, against 2 (R - 1) table
// reads per butterfly).
template <int R, int T>
__device__ __forceinline__ void fft_stage(float2 *x, const FilterPlan &a, int Ns, const float2 *ta,
                                          const float2 *tb) {
  constexpr int kB = max_butterflies(R);
  const int n = a.n, Q = n / R, tstep = n / (Ns * R);
  float2 rc[6];
  if constexpr (R % 2 == 1) {
#pragma unroll
    for (int t = 0; t < (R - 1) / 2; ++t) rc[t] = a.rc[odd_slot(R)][t];
  }
  float2 v[kB][R];
#pragma unroll
  for (int b = 0; b < kB; ++b) {
    const int j = threadIdx.x + b * T;
    if (j < Q) {
#pragma unroll
      for (int r = 0; r < R; ++r) v[b][r] = x[pidx(j + r * Q)];
    }
  }
  __syncthreads();
#pragma unroll
  for (int b = 0; b < kB; ++b) {
    const int j = threadIdx.x + b * T;
    if (j < Q) {
      const int k = j % Ns;
      if (k) {
        const int e = k * tstep;  // w^r = exp(-2 pi i r e / n)
        auto tw = [&](int c) {
          const int t = c * e;
          return cmul(ta[t >> 6], tb[t & (kTwLo - 1)]);
        };
        const float2 w1 = tw(1);
        const float2 w2 = R >= 3 ? tw(2) : w1;
        const float2 w4 = R >= 5 ? tw(4) : w1;
        const float2 w8 = R >= 9 ? tw(8) : w1;
#pragma unroll
        for (int r = 1; r < R; ++r) {
          float2 w = (r & 1) ? w1 : ((r & 2) ? w2 : ((r & 4) ? w4 : w8));
          if ((r & 1) && (r & 2)) w = cmul(w, w2);
          if ((r & 3) && (r & 4)) w = cmul(w, w4);
          if ((r & 7) && (r & 8)) w = cmul(w, w8);
          v[b][r] = cmul(v[b][r], w);
        }
      }
      dft<R>(v[b], rc);
      const int o = (j - k) * R + k;
#pragma unroll
      for (int r = 0; r < R; ++r) x[pidx(o + r * Ns)] = v[b][r];
    }
  }
  __syncthreads();
}

// In-place forward FFT of length a.n through the plan's stages, which come
// in a fixed order (16s, one 8 / 4 / 2, then 13s, 11s, 7s, 5s, 3s): one
// inlined copy of each stage kind in sequence (a switch inside a loop over
// the stages makes the compiler spill).  Force-inlined: called twice per
// kernel, the compiler otherwise emits it as a real call whose ABI costs a
// large stack frame and much of the speed.
template <int T>
__device__ __forceinline__ void fft_forward(float2 *x, const FilterPlan &a, const float2 *ta, const float2 *tb) {
  int s = 0, Ns = 1;
  const int ns = a.nstages;
  for (; s < ns && a.radix[s] == 16; ++s, Ns *= 16) fft_stage<16, T>(x, a, Ns, ta, tb);
  if (s < ns && a.radix[s] == 8) { fft_stage<8, T>(x, a, Ns, ta, tb); ++s; Ns *= 8; }
  if (s < ns && a.radix[s] == 4) { fft_stage<4, T>(x, a, Ns, ta, tb); ++s; Ns *= 4; }
  if (s < ns && a.radix[s] == 2) { fft_stage<2, T>(x, a, Ns, ta, tb); ++s; Ns *= 2; }
  for (; s < ns && a.radix[s] == 13; ++s, Ns *= 13) fft_stage<13, T>(x, a, Ns, ta, tb);
  for (; s < ns && a.radix[s] == 11; ++s, Ns *= 11) fft_stage<11, T>(x, a, Ns, ta, tb);
  for (; s < ns && a.radix[s] == 7; ++s, Ns *= 7) fft_stage<7, T>(x, a, Ns, ta, tb);
  for (; s < ns && a.radix[s] == 5; ++s, Ns *= 5) fft_stage<5, T>(x, a, Ns, ta, tb);
  for (; s < ns && a.radix[s] == 3; ++s, Ns *= 3) fft_stage<3, T>(x, a, Ns, ta, tb);
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

// Filters row pair `pair` of the rows a with the plan p (CTA-uniform).
template <typename OutT, int T>
__device__ __forceinline__ void filter_rows_body(const FilterPlan &p, const FilterRows &a, int pair) {
  extern __shared__ float2 sm[];  // n complex, padded by pidx
  __shared__ float2 scratch[T / 32 > 0 ? T / 32 : 1];
  __shared__ float2 ta[kMaxLen / kTwLo], tb[kTwLo];
  const int M = p.n;
  const int ncol = a.ncol, pad = a.pad, N = ncol + 2 * pad;
  const int tid = threadIdx.x;
  if (N > M) return;  // not a length for these rows (CTA-uniform)

  // twiddle tables: ta[u] = w^(64 u), tb[v] = w^v, w = exp(-2 pi i / n)
  for (int u = tid; u < (M + kTwLo - 1) / kTwLo; u += T) ta[u] = __ldg(p.tw + u * kTwLo);
  for (int v = tid; v < kTwLo; v += T) tb[v] = v < M ? __ldg(p.tw + v) : make_float2(1.f, 0.f);

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
    if (p.apply_log) { v1 = atb::neg_log(v1); v2 = ok2 ? atb::neg_log(v2) : 0.0f; }
    sm[pidx(pad + j)] = make_float2(v1, v2);
  }
  for (int m = N + tid; m < M; m += T) sm[pidx(m)] = make_float2(0.f, 0.f);
  __syncthreads();

  // 2. padding (numpy.pad semantics along the row)
  if (pad > 0) {
    float2 stat = make_float2(0.f, 0.f);
    if (p.mode == ATB_PAD_MEAN || p.mode == ATB_PAD_MAXIMUM || p.mode == ATB_PAD_MINIMUM) {
      const int op = p.mode == ATB_PAD_MEAN ? 0 : (p.mode == ATB_PAD_MAXIMUM ? 1 : 2);
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
    } else if (p.mode == ATB_PAD_MEDIAN) {
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
      switch (p.mode) {
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
  fft_forward<T>(sm, p, ta, tb);
  const float2 *spec = a.spec + (a.spec_rows > 1 ? (long long)i1 * M : 0LL);
  for (int k = tid; k < M; k += T) {
    const float2 y = cmul(sm[pidx(k)], __ldg(spec + k));
    sm[pidx(k)] = make_float2(y.x, -y.y);
  }
  __syncthreads();
  fft_forward<T>(sm, p, ta, tb);

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
__global__ void __launch_bounds__(T, T <= 256 ? 2 : 1)
    filter_rows_kernel(const __grid_constant__ FilterPlan p, const __grid_constant__ FilterRows a) {
  filter_rows_body<OutT, T>(p, a, (int)blockIdx.x);
}

// One launch over the row pairs of several single-slice sinograms that
// share the transform length: CTA q finds the item whose pair range holds q
// (binary search on pair_offset) and filters that pair.
template <typename OutT, int T>
__global__ void __launch_bounds__(T, T <= 256 ? 2 : 1)
    filter_batch_kernel(const __grid_constant__ FilterPlan p, const atb_filter_item *items, int nitems) {
  const int q = blockIdx.x;
  int lo = 0, hi = nitems - 1;
  while (lo < hi) {  // last item with pair_offset <= q
    const int mid = (lo + hi + 1) >> 1;
    if (items[mid].pair_offset <= q) lo = mid; else hi = mid - 1;
  }
  const atb_filter_item it = items[lo];
  const int pair = q - it.pair_offset;
  if (pair < 0 || pair >= (it.nrow + 1) / 2) return;  // CTA-uniform
  FilterRows b;
  b.src = it.src; b.srs = it.src_row_stride; b.sss = 0;
  b.nrow = it.nrow; b.nslice = 1; b.ncol = it.ncol; b.pad = it.pad;
  b.spec = reinterpret_cast<const float2 *>(it.spec); b.spec_rows = 1;
  b.dst = it.dst; b.drs = it.dst_row_stride; b.dss = 0;
  b.pair_within_angle = 0;
  b.pairs_per_angle = 0;
  filter_rows_body<OutT, T>(p, b, pair);
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

// ---- host side: transform length, plan, launches

bool smooth(int t, const int *primes, int np) {
  for (int k = 0; k < np; ++k)
    while (t % primes[k] == 0) t /= primes[k];
  return t == 1;
}

// radices of n in stage order: 16s, one 8 / 4 / 2 for the rest of the
// power of two, then the odd ones
bool make_radices(int n, int *radix, int &nstages) {
  nstages = 0;
  int r = n;
  auto push = [&](int p) {
    if (nstages >= kMaxStages) return false;
    radix[nstages++] = p;
    r /= p;
    return true;
  };
  while (r % 16 == 0)
    if (!push(16)) return false;
  for (int p : {8, 4, 2})
    if (r % p == 0 && !push(p)) return false;
  static const int odd[] = {13, 11, 7, 5, 3};
  for (int p : odd)
    while (r % p == 0)
      if (!push(p)) return false;
  return r == 1;
}

// approximate flops per point of a stage of radix r (butterfly + twiddles)
double stage_cost(int r) {
  switch (r) {
    case 2: return 5.0;
    case 4: return 8.5;
    case 8: return 13.3;
    case 16: return 16.6;
    case 3: return 9.3;
    case 5: return 15.2;
    case 7: return 19.7;
    case 11: return 28.2;
    default: return 32.3;  // 13
  }
}

double transform_cost(int n) {
  int radix[kMaxStages], ns = 0;
  if (!make_radices(n, radix, ns)) return INFINITY;
  double c = 0.0;
  for (int k = 0; k < ns; ++k) c += stage_cost(radix[k]);
  return c * n;
}

// threads per CTA: the fewest (a multiple of 32, at least 64) for which
// every stage's butterflies fit the per-thread register budget
int threads_for(int n, const int *radix, int ns) {
  int need = 64;
  for (int k = 0; k < ns; ++k) {
    const int q = n / radix[k], b = max_butterflies(radix[k]);
    const int t = (q + b - 1) / b;
    if (t > need) need = t;
  }
  for (int t : {64, 128, 256, 512})
    if (t >= need) return t;
  return -1;
}

int filter_length(int ncol, int pad) {
  static const int p13[] = {2, 3, 5, 7, 11, 13};
  static const int p7[] = {2, 3, 5, 7};
  const long long n = (long long)ncol + 2LL * pad;
  int best = -1;
  double best_cost = INFINITY;
  if (n >= 2 && n <= kMaxLen && smooth((int)n, p13, 6)) {
    best = (int)n;
    best_cost = transform_cost(best);
  }
  // the embedding: 7-smooth lengths from N + ncol - 1 up to the next power of two
  const long long lo = std::max(16LL, n + ncol - 1);
  long long hi = 16;
  while (hi < lo) hi <<= 1;
  for (long long m = lo; m <= hi && m <= kMaxLen; ++m) {
    if (!smooth((int)m, p7, 4)) continue;
    const double c = transform_cost((int)m);
    if (c < best_cost) {
      best_cost = c;
      best = (int)m;
    }
  }
  return best;
}

// whether n is an exact transform length for rows of ncol + 2 pad samples
bool valid_length(int n, int ncol, int pad) {
  const long long N = (long long)ncol + 2LL * pad;
  return n >= 2 && n <= kMaxLen && (n == N || n >= N + ncol - 1);
}

// the plan of length n (false: no radix plan or thread count for it)
bool make_plan(int n, int mode, int apply_log, const void *twiddle, FilterPlan &p, int &threads) {
  if (n < 2 || n > kMaxLen) return false;
  p.mode = mode;
  p.apply_log = apply_log ? 1 : 0;
  p.tw = reinterpret_cast<const float2 *>(twiddle);
  p.n = n;
  if (!make_radices(n, p.radix, p.nstages)) return false;
  static const int op[5] = {3, 5, 7, 11, 13};
  for (int k = 0; k < 5; ++k)
    for (int q = 0; q < 6; ++q) {
      const double ang = 2.0 * M_PI * (double)(q + 1) / (double)op[k];
      p.rc[k][q] = q < (op[k] - 1) / 2 ? make_float2((float)std::cos(ang), (float)std::sin(ang)) : make_float2(0.f, 0.f);
    }
  threads = threads_for(n, p.radix, p.nstages);
  return threads > 0;
}

size_t smem_bytes(int n) { return sizeof(float2) * (size_t)(n + (n >> 4) + 1); }

template <typename OutT, int T>
int launch_filter_t(const FilterPlan &p, const FilterRows &a, long long npairs, cudaStream_t st) {
  const size_t smem = smem_bytes(p.n);
  const int rc = atb::ensure_smem(filter_rows_kernel<OutT, T>, smem, "atb_filter_rows");
  if (rc != ATB_OK) return rc;
  filter_rows_kernel<OutT, T><<<(unsigned)npairs, T, smem, st>>>(p, a);
  return atb::check_launch("atb_filter_rows");
}

template <typename OutT>
int launch_filter(const FilterPlan &p, const FilterRows &a, int threads, long long npairs, cudaStream_t st) {
  switch (threads) {
    case 512: return launch_filter_t<OutT, 512>(p, a, npairs, st);
    case 256: return launch_filter_t<OutT, 256>(p, a, npairs, st);
    case 128: return launch_filter_t<OutT, 128>(p, a, npairs, st);
    default: return launch_filter_t<OutT, 64>(p, a, npairs, st);
  }
}

template <typename OutT, int T>
int launch_batch_t(const FilterPlan &p, const atb_filter_item *items, int nitems, int npairs, cudaStream_t st) {
  const size_t smem = smem_bytes(p.n);
  const int rc = atb::ensure_smem(filter_batch_kernel<OutT, T>, smem, "atb_filter_rows_batch");
  if (rc != ATB_OK) return rc;
  filter_batch_kernel<OutT, T><<<(unsigned)npairs, T, smem, st>>>(p, items, nitems);
  return atb::check_launch("atb_filter_rows_batch");
}

template <typename OutT>
int launch_batch(const FilterPlan &p, int threads, const atb_filter_item *items, int nitems, int npairs,
                 cudaStream_t st) {
  switch (threads) {
    case 512: return launch_batch_t<OutT, 512>(p, items, nitems, npairs, st);
    case 256: return launch_batch_t<OutT, 256>(p, items, nitems, npairs, st);
    case 128: return launch_batch_t<OutT, 128>(p, items, nitems, npairs, st);
    default: return launch_batch_t<OutT, 64>(p, items, nitems, npairs, st);
  }
}

}  // namespace

extern "C" {

int atb_filter_length(int ncol, int pad) {
  if (ncol < 1 || pad < 0) return atb::fail(ATB_EINVAL, "atb_filter_length: ncol=%d pad=%d", ncol, pad);
  const int n = filter_length(ncol, pad);
  if (n < 0)
    return atb::fail(ATB_ERANGE, "atb_filter_length: ncol=%d pad=%d needs a transform longer than %d", ncol, pad,
                     kMaxLen);
  return n;
}

int atb_filter_rows(const float *src, int64_t src_row_stride, int64_t src_slice_stride, int nrow, int nslice,
                    int ncol, int pad, int pad_mode, int apply_log, const void *spec, int spec_rows,
                    const void *twiddle, int fft_len, void *dst, int dst_dtype, int64_t dst_row_stride,
                    int64_t dst_slice_stride, void *stream) {
  if (!src || !dst || !spec || !twiddle) return atb::fail(ATB_EINVAL, "atb_filter_rows: null pointer");
  if (nrow < 1 || nslice < 1 || ncol < 1 || pad < 0)
    return atb::fail(ATB_EINVAL, "atb_filter_rows: bad shape nrow=%d nslice=%d ncol=%d pad=%d", nrow, nslice,
                     ncol, pad);
  if (pad_mode < ATB_PAD_EDGE || pad_mode > ATB_PAD_MEDIAN)
    return atb::fail(ATB_EINVAL, "atb_filter_rows: unknown pad_mode %d", pad_mode);
  if (spec_rows != 1 && spec_rows != nrow)
    return atb::fail(ATB_EINVAL, "atb_filter_rows: spec_rows=%d must be 1 or nrow=%d", spec_rows, nrow);
  FilterPlan p;
  int threads = 0;
  if (!valid_length(fft_len, ncol, pad) || !make_plan(fft_len, pad_mode, apply_log, twiddle, p, threads))
    return atb::fail(ATB_EINVAL, "atb_filter_rows: fft_len=%d is not a transform length for ncol=%d pad=%d "
                     "(atb_filter_length gives one)", fft_len, ncol, pad);
  FilterRows a;
  a.src = src; a.srs = src_row_stride; a.sss = src_slice_stride;
  a.nrow = nrow; a.nslice = nslice; a.ncol = ncol; a.pad = pad;
  a.spec = reinterpret_cast<const float2 *>(spec); a.spec_rows = spec_rows;
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
    case ATB_F32: return launch_filter<float>(p, a, threads, npairs, st);
    case ATB_F16: return launch_filter<__half>(p, a, threads, npairs, st);
    case ATB_BF16: return launch_filter<__nv_bfloat16>(p, a, threads, npairs, st);
    default: return atb::fail(ATB_EINVAL, "atb_filter_rows: unknown dst_dtype %d", dst_dtype);
  }
}

int atb_filter_rows_batch(const atb_filter_item *items, int nitems, int npairs, int pad_mode, int apply_log,
                          const void *twiddle, int fft_len, int dst_dtype, void *stream) {
  if (!items || !twiddle) return atb::fail(ATB_EINVAL, "atb_filter_rows_batch: null pointer");
  if (nitems < 1 || npairs < 1) return atb::fail(ATB_EINVAL, "atb_filter_rows_batch: empty batch");
  if (pad_mode < ATB_PAD_EDGE || pad_mode > ATB_PAD_MEDIAN)
    return atb::fail(ATB_EINVAL, "atb_filter_rows_batch: unknown pad_mode %d", pad_mode);
  FilterPlan p;
  int threads = 0;
  // every item needs fft_len == its N or fft_len >= N + ncol - 1; the
  // kernel skips items longer than fft_len
  if (!make_plan(fft_len, pad_mode, apply_log, twiddle, p, threads))
    return atb::fail(ATB_ERANGE, "atb_filter_rows_batch: fft_len=%d has no plan", fft_len);
  cudaStream_t st = atb::as_stream(stream);
  switch (dst_dtype) {
    case ATB_F32: return launch_batch<float>(p, threads, items, nitems, npairs, st);
    case ATB_F16: return launch_batch<__half>(p, threads, items, nitems, npairs, st);
    case ATB_BF16: return launch_batch<__nv_bfloat16>(p, threads, items, nitems, npairs, st);
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
