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
// A CTA filters two rows at once: real rows x1, x2 travel as the complex
// row x1 + i x2 through one forward FFT, a product with the (real-kernel)
// spectrum and one inverse FFT (done as conj(FFT(conj(.))) with 1/n folded
// into the spectrum); the real and imaginary parts of the result are the
// two filtered rows.  Each row is read from HBM once (with the -log folded
// in) and written once; padding, both transforms and the spectral product
// stay in shared memory.  The kernel is persistent: each CTA loops over row
// pairs, the next pair's rows travel into shared memory (cp.async) while
// the current pair is transformed, and a spectrum shared by all rows is
// read once per CTA.
#include <algorithm>
#include <cfloat>
#include <cmath>

#include "common.cuh"

namespace {

constexpr int kMaxLen = 16384;  // 16384 complex (+1/16 padding) = 136 KiB of shared memory
constexpr int kMaxStages = 14;

// Shared-memory index of complex element i.  (A padding word every 16 or
// 32 elements trims the bank conflicts of the first stages' strided
// writes, but its index arithmetic cost more than the conflicts: 0.84 and
// 0.83 against 0.78 ms per 16-slice launch at 2560 pixels.)
__device__ __forceinline__ int pidx(int i) { return i; }

// What every CTA of a launch shares: the transform plan and the pad / log
// settings (read from parameter space; the plan arrays are indexed at run
// time, so kernels take it as a __grid_constant__ parameter).
struct FilterPlan {
  int mode, apply_log;
  const float2 *tw;    // [n] the stages' twiddles (atb_filter_twiddles)
  int n, nstages;      // transform length and its radices, in stage order
  int radix[kMaxStages];
  unsigned magic[kMaxStages];  // ceil(2^32 / Ns) for Ns > 1: j / Ns = umulhi(j, magic) for j, Ns < 2^14
  float2 rc[5][6];     // (cos, sin)(2 pi q / p), q = 1 .. (p-1)/2, p = 3, 5, 7, 11, 13
};

// The plan's stage data as each CTA keeps it in shared memory: the stages
// read it there after barriers, so the compiler does not hoist it into
// registers across the pair loop.
struct StagePlan {
  int n, nstages;
  int radix[kMaxStages];
  unsigned magic[kMaxStages];
  float2 rc[5][6];
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

// butterflies a thread holds per stage of radix r, for a budget of about e
// complex values per thread
__host__ __device__ constexpr int butterflies(int r, int e) { return (e + r - 1) / r; }

// Stockham stage of radix R after sub-transforms of length Ns: butterfly
// j (< Q = n / R) reads x[j + r Q], twiddles input r by w^(r k)
// (k = j mod Ns, w = exp(-2 pi i / (Ns R))), does an R-point DFT and writes
// output q to x[(j - k) R + k + q Ns].  Every thread reads all of its
// inputs before the barrier and writes after it, so one buffer suffices.
// The twiddles w^(r k), r = 1 .. R-1, of butterfly k are R - 1
// consecutive entries of the stage's table (tw + Ns - 1 + k (R - 1)),
// computed in FP64 on the host: one read each, no index arithmetic beyond
// the base, no products.  The launch's thread count is a run-time value
// (blockDim.x); a thread holds up to kB butterflies of the stage.  Values
// of butterflies a thread skips are zeroed, not left undefined: undefined
// values on predicated paths made the compiler keep them alive across the
// pair loop and spill.
template <int R, int E>
__device__ __forceinline__ void fft_stage(float2 *x, const StagePlan &a, int Ns, unsigned magic,
                                          const float2 *tw) {
  constexpr int kB = butterflies(R, E);
  const int n = a.n, Q = n / R;
  const int nt = blockDim.x, nb = (Q + nt - 1) / nt;  // butterflies per thread (<= kB; CTA-uniform)
  float2 rc[6];
  if constexpr (R % 2 == 1) {
#pragma unroll
    for (int t = 0; t < (R - 1) / 2; ++t) rc[t] = a.rc[odd_slot(R)][t];
  }
  float2 v[kB][R];
#pragma unroll
  for (int b = 0; b < kB; ++b) {
    const int j = threadIdx.x + b * nt;
#pragma unroll
    for (int r = 0; r < R; ++r) v[b][r] = b < nb && j < Q ? x[pidx(j + r * Q)] : make_float2(0.f, 0.f);
  }
  __syncthreads();
#pragma unroll
  for (int b = 0; b < kB; ++b) {
    const int j = threadIdx.x + b * nt;
    if (b < nb && j < Q) {
      const int k = Ns == 1 ? 0 : j - (int)__umulhi((unsigned)j, magic) * Ns;  // j mod Ns
      if (k) {
        const float2 *w = tw + (Ns - 1) + k * (R - 1);
#pragma unroll
        for (int r = 1; r < R; ++r) v[b][r] = cmul(v[b][r], w[r - 1]);
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
// the stages makes the compiler spill).
template <int E>
__device__ __forceinline__ void fft_forward(float2 *x, const StagePlan &a, const float2 *tw) {
  int s = 0, Ns = 1;
  const int ns = a.nstages;
  for (; s < ns && a.radix[s] == 16; ++s, Ns *= 16) fft_stage<16, E>(x, a, Ns, a.magic[s], tw);
  if (s < ns && a.radix[s] == 8) { fft_stage<8, E>(x, a, Ns, a.magic[s], tw); ++s; Ns *= 8; }
  if (s < ns && a.radix[s] == 4) { fft_stage<4, E>(x, a, Ns, a.magic[s], tw); ++s; Ns *= 4; }
  if (s < ns && a.radix[s] == 2) { fft_stage<2, E>(x, a, Ns, a.magic[s], tw); ++s; Ns *= 2; }
  for (; s < ns && a.radix[s] == 13; ++s, Ns *= 13) fft_stage<13, E>(x, a, Ns, a.magic[s], tw);
  for (; s < ns && a.radix[s] == 11; ++s, Ns *= 11) fft_stage<11, E>(x, a, Ns, a.magic[s], tw);
  for (; s < ns && a.radix[s] == 7; ++s, Ns *= 7) fft_stage<7, E>(x, a, Ns, a.magic[s], tw);
  for (; s < ns && a.radix[s] == 5; ++s, Ns *= 5) fft_stage<5, E>(x, a, Ns, a.magic[s], tw);
  for (; s < ns && a.radix[s] == 3; ++s, Ns *= 3) fft_stage<3, E>(x, a, Ns, a.magic[s], tw);
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
    v = lane < (int)(blockDim.x >> 5) ? scratch[lane]
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
    for (int j = threadIdx.x; j < ncol; j += (int)blockDim.x) {
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

// The two rows (angle, slice) of row pair `pair`.
struct PairIdx {
  int i1, k1, i2, k2;
  bool ok2;
};

__device__ __forceinline__ PairIdx pair_rows(const FilterRows &a, int pair) {
  PairIdx r;
  if (a.pair_within_angle) {
    r.i1 = pair / a.pairs_per_angle;
    r.k1 = 2 * (pair % a.pairs_per_angle);
    r.i2 = r.i1;
    r.k2 = r.k1 + 1;
    r.ok2 = r.k2 < a.nslice;
  } else {
    // rows 2 pair and 2 pair + 1 in [angle][slice] order; the host caps
    // the pairs at 2^31, so the row index fits 32-bit unsigned arithmetic
    // (a 64-bit division here made the kernel spill to the stack)
    const unsigned r1 = 2u * (unsigned)pair, r2 = r1 + 1u, ns = (unsigned)a.nslice;
    r.i1 = (int)(r1 / ns);
    r.k1 = (int)(r1 % ns);
    r.i2 = (int)(r2 / ns);
    r.k2 = (int)(r2 % ns);
    r.ok2 = (unsigned long long)r2 < (unsigned long long)a.nrow * (unsigned long long)a.nslice;
  }
  return r;
}

// The stage plan into shared memory, visible after the next barrier.
__device__ __forceinline__ void load_tables(const FilterPlan &p, StagePlan &sp) {
  const int nt = blockDim.x;
  for (int i = threadIdx.x; i < kMaxStages; i += nt) {
    sp.radix[i] = p.radix[i];
    sp.magic[i] = p.magic[i];
  }
  for (int i = threadIdx.x; i < 30; i += nt) sp.rc[i / 6][i % 6] = p.rc[i / 6][i % 6];
  if (threadIdx.x == 0) {
    sp.n = p.n;
    sp.nstages = p.nstages;
  }
}

// Padding, transforms and store for one row pair whose (logged) rows sit
// in sm[pad .. pad + ncol) with zeros in [N, n): the padding, the forward
// transform, the product with spec (global or shared memory), the
// conjugated inverse, crop and store.  Starts after a barrier; its last
// reads of sm are not followed by one.
template <typename OutT, int T, int E>
__device__ __forceinline__ void pad_transform_store(const FilterPlan &p, const StagePlan &sp, const FilterRows &a,
                                                    float2 *sm, const float2 *spec, const float2 *tw,
                                                    float2 *scratch, const PairIdx &r) {
  const int M = p.n, ncol = a.ncol, pad = a.pad, tid = threadIdx.x;
  // padding (numpy.pad semantics along the row)
  if (pad > 0) {
    float2 stat = make_float2(0.f, 0.f);
    if (p.mode == ATB_PAD_MEAN || p.mode == ATB_PAD_MAXIMUM || p.mode == ATB_PAD_MINIMUM) {
      const int op = p.mode == ATB_PAD_MEAN ? 0 : (p.mode == ATB_PAD_MAXIMUM ? 1 : 2);
      float2 acc = op == 0 ? make_float2(0.f, 0.f)
                           : (op == 1 ? make_float2(-FLT_MAX, -FLT_MAX) : make_float2(FLT_MAX, FLT_MAX));
      for (int j = tid; j < ncol; j += (int)blockDim.x) {
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
    for (int t = tid; t < 2 * pad; t += (int)blockDim.x) {
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

  // forward transform, spectral product (conjugated), second forward
  // transform = conjugated inverse, from one call site (two inlined copies
  // would double the code the SMs fetch)
#pragma unroll 1
  for (int pass = 0; pass < 2; ++pass) {
    fft_forward<E>(sm, sp, tw);
    if (pass == 1) break;
    for (int k = tid; k < M; k += (int)blockDim.x) {
      const float2 y = cmul(sm[pidx(k)], spec[k]);
      sm[pidx(k)] = make_float2(y.x, -y.y);
    }
    __syncthreads();
  }

  // crop: real part -> row 1, -imag part -> row 2
  OutT *d1 = reinterpret_cast<OutT *>(a.dst) + r.i1 * a.drs + r.k1 * a.dss;
  OutT *d2 = reinterpret_cast<OutT *>(a.dst) + (r.ok2 ? r.i2 * a.drs + r.k2 * a.dss : 0);
  for (int j = tid; j < ncol; j += (int)blockDim.x) {
    const float2 w = sm[pidx(pad + j)];
    atb::store_from_float(d1 + j, w.x);
    if (r.ok2) atb::store_from_float(d2 + j, -w.y);
  }
}

// Filters row pair `pair` of the rows a with the plan p (CTA-uniform),
// reading the rows straight from global memory.
template <typename OutT, int T, int E>
__device__ __forceinline__ void filter_rows_body(const FilterPlan &p, const FilterRows &a, int pair) {
  extern __shared__ float2 sm[];  // n complex
  __shared__ float2 scratch[T / 32 > 0 ? T / 32 : 1];
  __shared__ StagePlan sp;
  const int M = p.n;
  const int ncol = a.ncol, pad = a.pad, N = ncol + 2 * pad;
  const int tid = threadIdx.x, nt = blockDim.x;
  if (N > M) return;  // not a length for these rows (CTA-uniform)
  load_tables(p, sp);
  const PairIdx r = pair_rows(a, pair);
  const float *s1 = a.src + r.i1 * a.srs + r.k1 * a.sss;
  const float *s2 = a.src + (r.ok2 ? r.i2 * a.srs + r.k2 * a.sss : 0);
  for (int j = tid; j < ncol; j += nt) {
    float v1 = __ldg(s1 + j);
    float v2 = r.ok2 ? __ldg(s2 + j) : 0.0f;
    if (p.apply_log) { v1 = atb::neg_log(v1); v2 = r.ok2 ? atb::neg_log(v2) : 0.0f; }
    sm[pidx(pad + j)] = make_float2(v1, v2);
  }
  for (int m = N + tid; m < M; m += nt) sm[pidx(m)] = make_float2(0.f, 0.f);
  __syncthreads();
  const float2 *spec = a.spec + (a.spec_rows > 1 ? (long long)r.i1 * M : 0LL);
  pad_transform_store<OutT, T, E>(p, sp, a, sm, spec, p.tw, scratch, r);  // twiddles through L1
}

// ---- asynchronous copies global -> shared (cp.async; completion is waited
// for with cp.async.wait_all, a hardware wait)
__device__ __forceinline__ void cp_async16(void *dst, const void *src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"((unsigned)__cvta_generic_to_shared(dst)),
               "l"(src)
               : "memory");
}
__device__ __forceinline__ void cp_async8(void *dst, const void *src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"((unsigned)__cvta_generic_to_shared(dst)),
               "l"(src)
               : "memory");
}
__device__ __forceinline__ void cp_async4(void *dst, const void *src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"((unsigned)__cvta_generic_to_shared(dst)),
               "l"(src)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// the rows of pair r into stage[0 .. ncol) and stage[ncol4 .. ncol4 + ncol)
__device__ __forceinline__ void stage_rows(const FilterRows &a, const PairIdx &r, float *stage, int ncol4) {
  const int ncol = a.ncol, nt = blockDim.x;
  const float *s1 = a.src + r.i1 * a.srs + r.k1 * a.sss;
  const float *s2 = a.src + (r.ok2 ? r.i2 * a.srs + r.k2 * a.sss : 0);
  const bool vec = (ncol & 3) == 0 && ((reinterpret_cast<uintptr_t>(s1) | reinterpret_cast<uintptr_t>(s2)) & 15) == 0;
  if (vec) {
    const int q = ncol >> 2;
    for (int t = threadIdx.x; t < 2 * q; t += nt) {
      const int row = t >= q, c = (t - row * q) << 2;
      if (row == 0) cp_async16(stage + c, s1 + c);
      else if (r.ok2) cp_async16(stage + ncol4 + c, s2 + c);
    }
  } else {
    for (int t = threadIdx.x; t < 2 * ncol; t += nt) {
      const int row = t >= ncol, c = t - row * ncol;
      if (row == 0) cp_async4(stage + c, s1 + c);
      else if (r.ok2) cp_async4(stage + ncol4 + c, s2 + c);
    }
  }
  cp_async_commit();
}

// CTAs per SM the register budget aims at (T: the most threads a launch of
// the instantiation uses): 3 for the 16-value budget at up to 256
// threads, 2 up to 384, else 1
constexpr int min_blocks(int t, int e) { return t > 384 ? 1 : (t > 256 || e > 16 ? 2 : 3); }

// Shared-memory layout of the persistent kernel (bytes): the transform
// buffer, the staged rows of the next pair, the twiddle table, the
// spectrum (one kernel for every row, when it fits without costing a CTA
// per SM).
__host__ __device__ constexpr size_t buf_bytes(int n) { return sizeof(float2) * (size_t)((n + 1) & ~1); }
__host__ __device__ constexpr int ncol4_of(int ncol) { return (ncol + 3) & ~3; }
__host__ __device__ constexpr size_t stage_bytes(int ncol) { return sizeof(float) * 2 * (size_t)ncol4_of(ncol); }

// Persistent: CTA b filters pairs b, b + grid, ...  While a pair is
// transformed, the next pair's rows are already on their way into shared
// memory, so row loads do not stall the transforms; a shared spectrum is
// read once per CTA.
template <typename OutT, int T, int E>
__global__ void __launch_bounds__(T, min_blocks(T, E))
    filter_rows_kernel(const __grid_constant__ FilterPlan p, const __grid_constant__ FilterRows a, int npairs,
                       int spec_in_smem) {
  extern __shared__ __align__(16) unsigned char smraw[];
  __shared__ float2 scratch[T / 32 > 0 ? T / 32 : 1];
  __shared__ StagePlan sp;
  const int M = p.n, ncol = a.ncol, pad = a.pad, N = ncol + 2 * pad, ncol4 = ncol4_of(ncol);
  const int tid = threadIdx.x, nt = blockDim.x;
  float2 *sm = reinterpret_cast<float2 *>(smraw);
  float *stage = reinterpret_cast<float *>(smraw + buf_bytes(M));
  float2 *tw_s = reinterpret_cast<float2 *>(smraw + buf_bytes(M) + stage_bytes(ncol));
  float2 *spec_s = tw_s + ((M + 1) & ~1);
  const bool shared_spec = spec_in_smem && a.spec_rows == 1;
  load_tables(p, sp);
  for (int k = tid; k < M; k += nt) cp_async8(tw_s + k, p.tw + k);
  if (shared_spec)
    for (int k = tid; k < M; k += nt) cp_async8(spec_s + k, a.spec + k);
  int pair = blockIdx.x;
  if (pair < npairs) stage_rows(a, pair_rows(a, pair), stage, ncol4);
  for (; pair < npairs; pair += gridDim.x) {
    const PairIdx r = pair_rows(a, pair);
    cp_async_wait_all();
    __syncthreads();  // the staged rows (and the spectrum) are visible; sm is free
    for (int j = tid; j < ncol; j += nt) {
      float v1 = stage[j];
      float v2 = r.ok2 ? stage[ncol4 + j] : 0.0f;
      if (p.apply_log) { v1 = atb::neg_log(v1); v2 = r.ok2 ? atb::neg_log(v2) : 0.0f; }
      sm[pidx(pad + j)] = make_float2(v1, v2);
    }
    for (int m = N + tid; m < M; m += nt) sm[pidx(m)] = make_float2(0.f, 0.f);
    __syncthreads();  // stage is consumed
    const int next = pair + gridDim.x;
    if (next < npairs) stage_rows(a, pair_rows(a, next), stage, ncol4);
    const float2 *spec = shared_spec ? spec_s : a.spec + (a.spec_rows > 1 ? (long long)r.i1 * M : 0LL);
    pad_transform_store<OutT, T, E>(p, sp, a, sm, spec, tw_s, scratch, r);
  }
}

// One CTA per pair, rows read straight from global memory: rows too long
// for the persistent kernel's staging buffer.
template <typename OutT, int T, int E>
__global__ void __launch_bounds__(T, min_blocks(T, E))
    filter_rows_direct_kernel(const __grid_constant__ FilterPlan p, const __grid_constant__ FilterRows a) {
  filter_rows_body<OutT, T, E>(p, a, (int)blockIdx.x);
}

// One launch over the row pairs of several single-slice sinograms that
// share the transform length: CTA q finds the item whose pair range holds q
// (binary search on pair_offset) and filters that pair.
template <typename OutT, int T, int E>
__global__ void __launch_bounds__(T, min_blocks(T, E))
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
  filter_rows_body<OutT, T, E>(p, b, pair);
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

// Launch shape of a plan: threads per CTA and per-thread value budget:
// the fewest of 64, 128, 256 or 512 threads for which every stage's
// butterflies fit a budget of 16 values, else 512 threads with a budget of
// 32.  (In between counts that waste fewer butterfly slots cost more in
// residency: 288 threads for 2860 points, two CTAs per SM, took 0.90 ms
// per 16-slice launch against 0.78 ms for 256 threads, three per SM.)
bool threads_for(int n, const int *radix, int ns, int &threads, int &budget) {
  for (int e : {16, 32}) {
    for (int t : {64, 128, 256, 512}) {
      if (e == 32 && t != 512) continue;
      bool ok = true;
      for (int k = 0; k < ns && ok; ++k) ok = (n / radix[k] + t - 1) / t <= butterflies(radix[k], e);
      if (ok) {
        threads = t;
        budget = e;
        return true;
      }
    }
  }
  return false;
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
bool make_plan(int n, int mode, int apply_log, const void *twiddle, FilterPlan &p, int &threads, int &budget) {
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
  for (int k = 0, ns = 1; k < p.nstages; ns *= p.radix[k], ++k)
    p.magic[k] = ns == 1 ? 0u : (unsigned)((0x100000000ULL + (unsigned long long)ns - 1) / (unsigned long long)ns);
  return threads_for(n, p.radix, p.nstages, threads, budget);
}

int sm_count() {
  int dev = 0, n = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
    return 148;
  return n;
}

int max_smem() {
  int dev = 0, v = 0;
  if (cudaGetDevice(&dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess)
    return 227 * 1024;
  return v;
}

template <typename OutT, int T, int E>
int launch_filter_t(const FilterPlan &p, const FilterRows &a, int nt, long long npairs, cudaStream_t st) {
  // shared memory besides the dynamic part: plan, scratch
  const size_t fixed = sizeof(float2) * 32 + sizeof(StagePlan);
  const size_t limit = (size_t)max_smem() - fixed;
  const size_t base = buf_bytes(p.n) + stage_bytes(a.ncol) + buf_bytes(p.n), spec = sizeof(float2) * p.n;
  if (base > limit) {  // no room to stage rows: one CTA per pair
    const size_t smem = buf_bytes(p.n);
    const int rc = atb::ensure_smem(filter_rows_direct_kernel<OutT, T, E>, smem, "atb_filter_rows");
    if (rc != ATB_OK) return rc;
    filter_rows_direct_kernel<OutT, T, E><<<(unsigned)npairs, nt, smem, st>>>(p, a);
    return atb::check_launch("atb_filter_rows");
  }
  // the spectrum in shared memory only if that costs no CTA per SM
  auto resident = [&](size_t bytes) {
    int n = 0;
    if (atb::ensure_smem(filter_rows_kernel<OutT, T, E>, bytes, "atb_filter_rows") != ATB_OK ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, filter_rows_kernel<OutT, T, E>, nt, bytes) != cudaSuccess)
      return 0;
    return n;
  };
  int per_sm = resident(base);
  if (per_sm < 1) return atb::fail(ATB_ECUDA, "atb_filter_rows: no CTA of %d bytes fits an SM", (int)base);
  const int spec_in_smem = a.spec_rows == 1 && base + spec <= limit && resident(base + spec) >= per_sm;
  const size_t smem = base + (spec_in_smem ? spec : 0);
  const int rc = atb::ensure_smem(filter_rows_kernel<OutT, T, E>, smem, "atb_filter_rows");
  if (rc != ATB_OK) return rc;
  const long long grid = std::min<long long>(npairs, (long long)per_sm * sm_count());
  filter_rows_kernel<OutT, T, E><<<(unsigned)grid, nt, smem, st>>>(p, a, (int)npairs, spec_in_smem);
  return atb::check_launch("atb_filter_rows");
}

template <typename OutT>
int launch_filter(const FilterPlan &p, const FilterRows &a, int threads, int budget, long long npairs,
                  cudaStream_t st) {
  if (budget > 16) return launch_filter_t<OutT, 512, 32>(p, a, threads, npairs, st);
  if (threads <= 128) return launch_filter_t<OutT, 128, 16>(p, a, threads, npairs, st);
  if (threads <= 256) return launch_filter_t<OutT, 256, 16>(p, a, threads, npairs, st);
  if (threads <= 384) return launch_filter_t<OutT, 384, 16>(p, a, threads, npairs, st);
  return launch_filter_t<OutT, 512, 16>(p, a, threads, npairs, st);
}

template <typename OutT, int T, int E>
int launch_batch_t(const FilterPlan &p, const atb_filter_item *items, int nitems, int nt, int npairs,
                   cudaStream_t st) {
  const size_t smem = buf_bytes(p.n);
  const int rc = atb::ensure_smem(filter_batch_kernel<OutT, T, E>, smem, "atb_filter_rows_batch");
  if (rc != ATB_OK) return rc;
  filter_batch_kernel<OutT, T, E><<<(unsigned)npairs, nt, smem, st>>>(p, items, nitems);
  return atb::check_launch("atb_filter_rows_batch");
}

template <typename OutT>
int launch_batch(const FilterPlan &p, int threads, int budget, const atb_filter_item *items, int nitems,
                 int npairs, cudaStream_t st) {
  if (budget > 16) return launch_batch_t<OutT, 512, 32>(p, items, nitems, threads, npairs, st);
  if (threads <= 128) return launch_batch_t<OutT, 128, 16>(p, items, nitems, threads, npairs, st);
  if (threads <= 256) return launch_batch_t<OutT, 256, 16>(p, items, nitems, threads, npairs, st);
  if (threads <= 384) return launch_batch_t<OutT, 384, 16>(p, items, nitems, threads, npairs, st);
  return launch_batch_t<OutT, 512, 16>(p, items, nitems, threads, npairs, st);
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

int atb_filter_twiddles(int n, void *host_out) {
  if (!host_out) return atb::fail(ATB_EINVAL, "atb_filter_twiddles: null pointer");
  int radix[kMaxStages], ns = 0;
  if (n < 2 || n > kMaxLen || !make_radices(n, radix, ns))
    return atb::fail(ATB_EINVAL, "atb_filter_twiddles: %d is not a transform length of the filter", n);
  float *out = static_cast<float *>(host_out);
  // stage s of radix R after sub-transforms of length Ns: entries
  // Ns - 1 + k (R - 1) + (r - 1) = exp(-2 pi i r k / (Ns R)), k < Ns, 0 < r < R
  // (the stages' Ns (R - 1) add up to n - 1; entry n - 1 is unused)
  int Ns = 1;
  for (int st = 0; st < ns; ++st) {
    const int R = radix[st];
    for (int k = 0; k < Ns; ++k)
      for (int r = 1; r < R; ++r) {
        const long long e = (long long)r * k;
        const double ang = -2.0 * M_PI * (double)e / (double)(Ns * R);
        float *o = out + 2 * (Ns - 1 + k * (R - 1) + (r - 1));
        o[0] = (float)std::cos(ang);
        o[1] = (float)std::sin(ang);
      }
    Ns *= R;
  }
  out[2 * (n - 1)] = 1.0f;
  out[2 * (n - 1) + 1] = 0.0f;
  return ATB_OK;
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
  int threads = 0, budget = 0;
  if (!valid_length(fft_len, ncol, pad) || !make_plan(fft_len, pad_mode, apply_log, twiddle, p, threads, budget))
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
    case ATB_F32: return launch_filter<float>(p, a, threads, budget, npairs, st);
    case ATB_F16: return launch_filter<__half>(p, a, threads, budget, npairs, st);
    case ATB_BF16: return launch_filter<__nv_bfloat16>(p, a, threads, budget, npairs, st);
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
  int threads = 0, budget = 0;
  // every item needs fft_len == its N or fft_len >= N + ncol - 1; the
  // kernel skips items longer than fft_len
  if (!make_plan(fft_len, pad_mode, apply_log, twiddle, p, threads, budget))
    return atb::fail(ATB_ERANGE, "atb_filter_rows_batch: fft_len=%d has no plan", fft_len);
  cudaStream_t st = atb::as_stream(stream);
  switch (dst_dtype) {
    case ATB_F32: return launch_batch<float>(p, threads, budget, items, nitems, npairs, st);
    case ATB_F16: return launch_batch<__half>(p, threads, budget, items, nitems, npairs, st);
    case ATB_BF16: return launch_batch<__nv_bfloat16>(p, threads, budget, items, nitems, npairs, st);
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
