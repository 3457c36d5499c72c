// Mixed-radix complex FFT in shared memory, FP64, for the 2-D filters.
//
// Stockham auto-sort: a transform of length n = p_0 p_1 ... p_{s-1} runs s
// stages; the stage of radix p with L = p_0 ... p_{k-1} takes the p inputs
// of butterfly j (j in [0, n/p)) at j + r n/p, multiplies input r by
// w_n^(r (j mod L) n/(L p)), transforms them with a p-point DFT and writes
// output q to (j / L) L p + (j mod L) + q L.  Each stage reads one buffer
// and writes the other, so the result ends in natural order with one CTA
// barrier per stage.  Radices 2, 4 and 8 use the usual butterflies; the odd
// radices 3, 5, 7, 11 and 13 use the symmetric form of the DFT (sums and
// differences of inputs r and p - r against cos and sin of 2 pi t / p).
// Forward: w = exp(-2 pi i / n); inverse: its conjugate, unnormalised.
#pragma once

#include <cuda_runtime.h>

namespace atb {
namespace fft {

constexpr int kMaxStages = 24;
constexpr int kOddRadices = 5;  // 3, 5, 7, 11, 13

struct Plan {
  int n;                 // transform length
  int nstages;
  int radix[kMaxStages];
  const double2 *tw;     // exp(-2 pi i m / n), m in [0, n)
  // cos / sin (2 pi t / p), t = 1 .. (p-1)/2, for p = 3, 5, 7, 11, 13
  double2 rc[kOddRadices][6];
};

__host__ __device__ constexpr int odd_slot(int p) {
  return p == 3 ? 0 : p == 5 ? 1 : p == 7 ? 2 : p == 11 ? 3 : 4;
}

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(fma(a.x, b.x, -a.y * b.y), fma(a.x, b.y, a.y * b.x));
}
__device__ __forceinline__ double2 cmulc(double2 a, double2 b) {  // a * conj(b)
  return make_double2(fma(a.x, b.x, a.y * b.y), fma(a.y, b.x, -a.x * b.y));
}
__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
// -i z (forward quarter turn) and +i z
__device__ __forceinline__ double2 mul_mi(double2 z) { return make_double2(z.y, -z.x); }
__device__ __forceinline__ double2 mul_pi(double2 z) { return make_double2(-z.y, z.x); }

template <bool INV>
__device__ __forceinline__ double2 quarter(double2 z) {  // w_4 z
  return INV ? mul_pi(z) : mul_mi(z);
}

template <bool INV>
__device__ __forceinline__ void dft4(double2 &v0, double2 &v1, double2 &v2, double2 &v3) {
  const double2 a = cadd(v0, v2), b = csub(v0, v2);
  const double2 c = cadd(v1, v3), d = quarter<INV>(csub(v1, v3));
  v0 = cadd(a, c);
  v2 = csub(a, c);
  v1 = cadd(b, d);
  v3 = csub(b, d);
}

template <int P, bool INV>
__device__ __forceinline__ void dft(double2 (&v)[P], const double2 (&rc)[6]) {
  if constexpr (P == 2) {
    const double2 a = v[0];
    v[0] = cadd(a, v[1]);
    v[1] = csub(a, v[1]);
  } else if constexpr (P == 4) {
    dft4<INV>(v[0], v[1], v[2], v[3]);
  } else if constexpr (P == 8) {
    // two 4-point DFTs of the even and odd inputs, then w_8^q combinations
    double2 e0 = v[0], e1 = v[2], e2 = v[4], e3 = v[6];
    double2 o0 = v[1], o1 = v[3], o2 = v[5], o3 = v[7];
    dft4<INV>(e0, e1, e2, e3);
    dft4<INV>(o0, o1, o2, o3);
    constexpr double h = 0.70710678118654752440;  // sqrt(1/2)
    // w_8 = (h, -h) forward, (h, h) inverse; w_8^2 = -+i; w_8^3 = (-h, -+h)
    const double2 t1 = INV ? make_double2(h * (o1.x - o1.y), h * (o1.x + o1.y))
                           : make_double2(h * (o1.x + o1.y), h * (o1.y - o1.x));
    const double2 t2 = quarter<INV>(o2);
    const double2 t3 = INV ? make_double2(-h * (o3.x + o3.y), h * (o3.x - o3.y))
                           : make_double2(h * (o3.y - o3.x), -h * (o3.x + o3.y));
    v[0] = cadd(e0, o0);
    v[4] = csub(e0, o0);
    v[1] = cadd(e1, t1);
    v[5] = csub(e1, t1);
    v[2] = cadd(e2, t2);
    v[6] = csub(e2, t2);
    v[3] = cadd(e3, t3);
    v[7] = csub(e3, t3);
  } else {
    // odd P: y_q = A_q -+ i B_q, y_{P-q} = A_q +- i B_q with
    // A_q = v_0 + sum_r (v_r + v_{P-r}) cos(2 pi q r / P),
    // B_q = sum_r (v_r - v_{P-r}) sin(2 pi q r / P)
    constexpr int H = (P - 1) / 2;
    double2 s[H], d[H];
    const double2 v0 = v[0];
    double2 y0 = v0;
#pragma unroll
    for (int r = 1; r <= H; ++r) {
      s[r - 1] = cadd(v[r], v[P - r]);
      d[r - 1] = csub(v[r], v[P - r]);
      y0 = cadd(y0, s[r - 1]);
    }
    v[0] = y0;
#pragma unroll
    for (int q = 1; q <= H; ++q) {
      double2 A = v0, B = make_double2(0.0, 0.0);
#pragma unroll
      for (int r = 1; r <= H; ++r) {
        int t = (q * r) % P;
        double sg = 1.0;
        if (t > H) {  // sin(2 pi t / P) = -sin(2 pi (P - t) / P)
          t = P - t;
          sg = -1.0;
        }
        const double c = rc[t - 1].x, sn = sg * rc[t - 1].y;
        A.x = fma(s[r - 1].x, c, A.x);
        A.y = fma(s[r - 1].y, c, A.y);
        B.x = fma(d[r - 1].x, sn, B.x);
        B.y = fma(d[r - 1].y, sn, B.y);
      }
      // forward: A - i B and A + i B; inverse: the other way round
      const double2 mB = mul_mi(B), pB = mul_pi(B);
      v[q] = INV ? cadd(A, pB) : cadd(A, mB);
      v[P - q] = INV ? cadd(A, mB) : cadd(A, pB);
    }
  }
}

// Twiddles w_n^e in shared memory as a two-level table: e = 64 h + l,
// w^e = hi[h] lo[l] (one complex product, within two roundings of the
// correctly rounded value); 64 + ceil(n / 64) entries instead of n.
constexpr int kTwLo = 64;
__host__ __device__ constexpr int twiddle_entries(int n) { return kTwLo + (n + kTwLo - 1) / kTwLo; }

// Fills the table from the plan's full table; call before the first run
// (a CTA barrier separates them).
__device__ __forceinline__ void load_twiddles(const Plan &pl, double2 *tws) {
  const int nhi = (pl.n + kTwLo - 1) / kTwLo;
  for (int i = threadIdx.x; i < kTwLo + nhi; i += blockDim.x)
    tws[i] = i < kTwLo ? (i < pl.n ? __ldg(pl.tw + i) : make_double2(1.0, 0.0)) : __ldg(pl.tw + (i - kTwLo) * kTwLo);
}

__device__ __forceinline__ double2 twiddle(const double2 *tws, int e) {
  return cmul(tws[kTwLo + (e >> 6)], tws[e & (kTwLo - 1)]);
}

template <int P, bool INV>
__device__ __forceinline__ void stage(const double2 *__restrict__ in, double2 *__restrict__ out, const Plan &pl,
                                      const double2 *tws, int L) {
  const int n = pl.n, m = n / P;
  const int tstep = n / (L * P);  // twiddle index step per unit of r * k
  // the odd radix's cos / sin in registers for the whole stage (read
  // through a pointer the compiler would reload them for every butterfly)
  double2 rc[6];
  if constexpr (P % 2 == 1) {
#pragma unroll
    for (int t = 0; t < (P - 1) / 2; ++t) rc[t] = pl.rc[odd_slot(P)][t];
  }
  for (int j = threadIdx.x; j < m; j += blockDim.x) {
    const int i = j / L, k = j - i * L;
    double2 v[P];
#pragma unroll
    for (int r = 0; r < P; ++r) v[r] = in[j + r * m];
    if (k > 0) {
#pragma unroll
      for (int r = 1; r < P; ++r) {
        const double2 w = twiddle(tws, r * k * tstep);
        v[r] = INV ? cmulc(v[r], w) : cmul(v[r], w);
      }
    }
    dft<P, INV>(v, rc);
    double2 *o = out + i * L * P + k;
#pragma unroll
    for (int q = 0; q < P; ++q) o[q * L] = v[q];
  }
}

// Transform of the n values in a[] (b[] is scratch of the same size; tws
// the table of load_twiddles); returns the buffer holding the result.
// Every thread of the CTA calls it.
template <bool INV>
__device__ double2 *run(double2 *a, double2 *b, const Plan &pl, const double2 *tws) {
  int L = 1;
  for (int s = 0; s < pl.nstages; ++s) {
    const int p = pl.radix[s];
    switch (p) {
      case 2: stage<2, INV>(a, b, pl, tws, L); break;
      case 3: stage<3, INV>(a, b, pl, tws, L); break;
      case 4: stage<4, INV>(a, b, pl, tws, L); break;
      case 5: stage<5, INV>(a, b, pl, tws, L); break;
      case 7: stage<7, INV>(a, b, pl, tws, L); break;
      case 8: stage<8, INV>(a, b, pl, tws, L); break;
      case 11: stage<11, INV>(a, b, pl, tws, L); break;
      default: stage<13, INV>(a, b, pl, tws, L); break;
    }
    __syncthreads();
    double2 *t = a;
    a = b;
    b = t;
    L *= p;
  }
  return a;
}

}  // namespace fft
}  // namespace atb

namespace atb {
namespace fft {

// ---------------------------------------------------------------------------
// In-place transforms of n = 2^m values (m <= 13) in one shared-memory
// buffer, for lengths whose two Stockham buffers would not fit.  Radices 8,
// then 4, then 2 (the sequence ip_radices gives).  The forward transform
// decimates in frequency: the stage of radix r on blocks of length L takes,
// for each n1 < L / r, the r values at n1 + j L / r, transforms them and
// multiplies output k by w_L^(k n1), in place; its output is in digit-
// reversed order.  The inverse runs the same stages in reverse order, each
// undoing its forward twin (conjugate twiddles, then the inverse r-point
// DFT), so it takes digit-reversed input to natural order, unnormalised.
// A product of two forward outputs is therefore a circular convolution
// after the inverse, with no reordering pass.

struct IpPlan {
  int n, nstages;
  int radix[16];
};

__host__ __device__ inline bool ip_radices(int n, IpPlan &p) {
  p.n = n;
  p.nstages = 0;
  int r = n;
  while (r > 1 && r % 8 == 0) { p.radix[p.nstages++] = 8; r /= 8; }
  while (r > 1 && r % 4 == 0) { p.radix[p.nstages++] = 4; r /= 4; }
  while (r > 1 && r % 2 == 0) { p.radix[p.nstages++] = 2; r /= 2; }
  return r == 1 && p.nstages <= 16;
}

// the two-level twiddle table of a length-n transform from the full table
__device__ __forceinline__ void load_twiddles_n(const double2 *tw, int n, double2 *tws) {
  const int nhi = (n + kTwLo - 1) / kTwLo;
  for (int i = threadIdx.x; i < kTwLo + nhi; i += blockDim.x)
    tws[i] = i < kTwLo ? (i < n ? __ldg(tw + i) : make_double2(1.0, 0.0)) : __ldg(tw + (i - kTwLo) * kTwLo);
}

// One in-place stage on two butterflies per thread at a time: both load
// before either computes (a stage's butterflies touch disjoint elements),
// which doubles the independent work in flight per thread.  The twiddles
// of a butterfly are w, w^2, ..., w^(R-1) of one table value w by repeated
// products (at most R - 2 extra roundings in FP64, against R - 1 table
// lookups of two shared-memory reads each).  n and L are powers of two, so
// the butterfly's block and offset come from a shift and a mask.
template <int R, bool INV>
__device__ __forceinline__ void ip_butterfly(double2 (&v)[R], int n1, int tstep, const double2 *tws) {
  const double2 rc[6] = {};
  if constexpr (!INV) dft<R, false>(v, rc);
  if (n1) {
    const double2 w = twiddle(tws, n1 * tstep);
    double2 wk = w;
#pragma unroll
    for (int k = 1; k < R; ++k) {
      v[k] = INV ? cmulc(v[k], wk) : cmul(v[k], wk);
      if (k + 1 < R) wk = cmul(wk, w);
    }
  }
  if constexpr (INV) dft<R, true>(v, rc);
}

template <int R, bool INV>
__device__ __forceinline__ void ip_stage(double2 *x, int n, int L, const double2 *tws) {
  const int s = L / R, tstep = n / L, nq = n / R, nt = blockDim.x;
  const int sh = __ffs(s) - 1;  // s = 2^sh
  for (int q0 = threadIdx.x; q0 < nq; q0 += 2 * nt) {
    const int q1 = q0 + nt;
    const bool two = q1 < nq;
    const int n10 = q0 & (s - 1), n11 = q1 & (s - 1);
    double2 *p0 = x + (q0 >> sh) * L + n10;
    double2 *p1 = x + (q1 >> sh) * L + n11;
    double2 v0[R], v1[R];
#pragma unroll
    for (int j = 0; j < R; ++j) {
      v0[j] = p0[j * s];
      v1[j] = two ? p1[j * s] : make_double2(0.0, 0.0);
    }
    ip_butterfly<R, INV>(v0, n10, tstep, tws);
    ip_butterfly<R, INV>(v1, n11, tstep, tws);
#pragma unroll
    for (int j = 0; j < R; ++j) {
      p0[j * s] = v0[j];
      if (two) p1[j * s] = v1[j];
    }
  }
}

// every thread of the CTA calls these; a barrier separates the stages and
// follows the last one
template <bool INV>
__device__ void ip_run(double2 *x, const IpPlan &pl, const double2 *tws) {
  if constexpr (!INV) {
    int L = pl.n;
    for (int s = 0; s < pl.nstages; ++s) {
      const int r = pl.radix[s];
      if (r == 8) ip_stage<8, false>(x, pl.n, L, tws);
      else if (r == 4) ip_stage<4, false>(x, pl.n, L, tws);
      else ip_stage<2, false>(x, pl.n, L, tws);
      __syncthreads();
      L /= r;
    }
  } else {
    int L = 1;
    for (int s = pl.nstages - 1; s >= 0; --s) {
      const int r = pl.radix[s];
      L *= r;
      if (r == 8) ip_stage<8, true>(x, pl.n, L, tws);
      else if (r == 4) ip_stage<4, true>(x, pl.n, L, tws);
      else ip_stage<2, true>(x, pl.n, L, tws);
      __syncthreads();
    }
  }
}

}  // namespace fft
}  // namespace atb
