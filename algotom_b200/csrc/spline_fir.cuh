// B-spline prefilter as a finite impulse response, shared by the DFI and
// 360-degree kernels.
//
// The published prefilter of cubic / quintic B-spline interpolation (gain
// prod (1 - z)(1 - 1/z), then per pole a causal and an anti-causal
// recursion, started from the values of a symmetric extension of the line)
// is linear and shift-invariant on that symmetric extension, so it equals
// the convolution of the extended line with its symmetric impulse response,
// which decays as |z1|^|k| (0.43^|k| for the quintic, 0.27^|k| for the
// cubic).  Applied as a 2 x 48 (quintic) or 2 x 32 (cubic) tap FIR it is
// exact to below 1e-17 relative and fully parallel, where the recursion is
// a serial chain along each line.
#pragma once

#include <cmath>

namespace atb {
namespace spline {

constexpr int kMaxTaps = 48;  // |z1|^48 < 1e-17 for the quintic spline

struct Taps {
  double h[kMaxTaps + 1];  // symmetric impulse response h[|k|], k <= ntaps
  int ntaps;
};

inline double host_pole(int order, int k) {
  if (order == 3) return std::sqrt(3.0) - 2.0;
  const double a = std::sqrt(17745.0 / 4.0), b = std::sqrt(105.0 / 4.0);
  return k == 0 ? std::sqrt(135.0 / 2.0 - a) + b - 13.0 / 2.0 : std::sqrt(135.0 / 2.0 + a) - b - 13.0 / 2.0;
}

// Impulse response of the prefilter (gain, then per pole a causal and an
// anti-causal pass), from the recursion run on a unit impulse in the middle
// of a long zero line: the ends are 2 kMaxTaps samples away, where the
// response has decayed below 1e-34.
inline Taps make_taps(int order) {
  constexpr int kLen = 4 * kMaxTaps + 1, kMid = 2 * kMaxTaps;
  double c[kLen] = {0.0};
  c[kMid] = 1.0;
  const int npoles = order == 5 ? 2 : 1;
  double gain = 1.0;
  for (int k = 0; k < npoles; ++k) {
    const double z = host_pole(order, k);
    gain *= (1.0 - z) * (1.0 - 1.0 / z);
  }
  for (double &v : c) v *= gain;
  for (int k = 0; k < npoles; ++k) {
    const double z = host_pole(order, k);
    for (int i = 1; i < kLen; ++i) c[i] += z * c[i - 1];
    c[kLen - 1] *= z / (z - 1.0);
    for (int i = kLen - 2; i >= 0; --i) c[i] = z * (c[i + 1] - c[i]);
  }
  Taps t;
  t.ntaps = order == 5 ? kMaxTaps : 32;  // |z|^32 < 1e-18 for the cubic
  for (int k = 0; k <= kMaxTaps; ++k) t.h[k] = c[kMid + k];
  return t;
}

// index of sample i of a line of n under the symmetric extension
// (boundary 0: half-sample "reflect", 1: whole-sample "mirror")
__device__ __forceinline__ int sym_index(int i, int n, int boundary) {
  if (i >= 0 && i < n) return i;  // inside: no remainder
  if (boundary == 0) {
    const int p = 2 * n;
    int r = i % p;
    if (r < 0) r += p;
    return r >= n ? p - 1 - r : r;
  }
  if (n == 1) return 0;
  const int p = 2 * (n - 1);
  int r = i % p;
  if (r < 0) r += p;
  return r >= n ? p - r : r;
}

// Register-blocked FIR: acc[r] = sum_k h[|k|] x(r + k + NT), |k| <= NT,
// for BLK consecutive outputs from one sliding window of BLK + 2 NT values
// x(0), x(1), ... (each read once, feeding up to BLK outputs).  NT is a
// template parameter, so the loops unroll with the taps as constants.
template <int NT, int BLK, typename Load>
__device__ __forceinline__ void fir_block(const Taps &taps, Load load, double (&acc)[BLK]) {
#pragma unroll
  for (int r = 0; r < BLK; ++r) acc[r] = 0.0;
#pragma unroll
  for (int t = 0; t < BLK + 2 * NT; ++t) {
    const double x = load(t);
#pragma unroll
    for (int r = 0; r < BLK; ++r) {
      const int k = t - NT - r;
      if (k >= -NT && k <= NT) acc[r] = fma(taps.h[k < 0 ? -k : k], x, acc[r]);
    }
  }
}

// index of value q in a strip padded by one word every 8 (threads 8 values
// apart then hit distinct shared-memory banks)
__device__ __forceinline__ int fir_pad(int q) { return q + (q >> 3); }

}  // namespace spline
}  // namespace atb
