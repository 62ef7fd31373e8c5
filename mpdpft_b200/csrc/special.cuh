// special.cuh -- the special functions of the reference's finite-temperature
// gradient-corrected density (DensityExpression 5, getDenEnAt,
// mpDPFT.cpp:3363-3453) and its Airy-averaged branch
// (AdaptiveBoole_nAiT / nAiTintegrand, mpDPFT.cpp:3553-3620).
//
// fd_li(o, x) = Li_s(-e^x) for s = 5/2, 3/2, 1/2, -1/2, -3/2 (the
// reference's polylog("5half" .. "m3half", x), mpDPFT.cpp:7000-7027, whose
// spline tables are not in its checkout): the alternating series below
// x = -2, Chebyshev series on unit intervals up to 60, the Sommerfeld
// expansion above, and the reference's leading term -x^s/Gamma(s+1) above
// 699 and 0 below -699, as its polylog() does.
// curly_a(x) = int_x^inf Ai(t) dt (CurlyA, mpDPFT.h:231-237): Chebyshev
// series of width 1/4 on [-150, 16), the reference's leading asymptotic
// below -149.99, 1 below -1e50, and e^{-z}/(2 sqrt(pi) x^{3/4}),
// z = 2 x^{3/2}/3, from 16 up (the reference returns 0 from 99.99).
// The tables are generated by gen_special_tables.py (mpmath, 30 digits).
#pragma once
#include <cmath>

namespace mpdpft {

#include "special_tables.inc"

static __device__ const double kFdTab[5 * (MPDPFT_FD_X1 - MPDPFT_FD_X0) * MPDPFT_FD_DEG] = MPDPFT_FD_TABLE;
static __device__ const double kFdAsym[5 * MPDPFT_FD_ASYM] = MPDPFT_FD_ASYM_TABLE;
static __device__ const double kFdRGamma[5] = MPDPFT_FD_RGAMMA;
static __device__ const double kCaTab[MPDPFT_CA_N * MPDPFT_CA_DEG] = MPDPFT_CA_TABLE;

// orders of fd_li
enum { FD_5HALF = 0, FD_3HALF = 1, FD_1HALF = 2, FD_M1HALF = 3, FD_M3HALF = 4 };

// Clenshaw sum of a Chebyshev series c[0..n-1] at t in [-1, 1].
__device__ __forceinline__ double cheb_sum(const double* c, int n, double t) {
  double b1 = 0.0, b2 = 0.0;
  for (int j = n - 1; j >= 1; --j) {
    const double b0 = fma(2.0 * t, b1, __ldg(c + j) - b2);
    b2 = b1;
    b1 = b0;
  }
  return fma(t, b1, __ldg(c) - b2);
}

// k^{-s} for the order o.
__device__ __forceinline__ double fd_kpow(int o, double k) {
  const double r = sqrt(k);
  switch (o) {
    case FD_5HALF: return 1.0 / (k * k * r);
    case FD_3HALF: return 1.0 / (k * r);
    case FD_1HALF: return 1.0 / r;
    case FD_M1HALF: return r;
    default: return k * r;
  }
}

// x^s for the order o (x > 0).
__device__ __forceinline__ double fd_xpow(int o, double x) {
  const double r = sqrt(x);
  switch (o) {
    case FD_5HALF: return x * x * r;
    case FD_3HALF: return x * r;
    case FD_1HALF: return r;
    case FD_M1HALF: return 1.0 / r;
    default: return 1.0 / (x * r);
  }
}

__device__ __forceinline__ double fd_li(int o, double x) {
  if (!(x >= -699.0)) return x != x ? x : 0.0;
  if (x > 699.0) return -fd_xpow(o, x) * kFdRGamma[o];
  if (x < (double)MPDPFT_FD_X0) {
    // sum_{k>=1} (-1)^k e^{kx} k^{-s}; e^{x} <= e^{-2}: 40 terms reach 1e-35
    const double z = exp(x);
    double zk = z, sum = 0.0;
    for (int k = 1; k <= 40; ++k) {
      const double t = zk * fd_kpow(o, (double)k);
      sum += (k & 1) ? -t : t;
      zk *= z;
      if (zk < 1.0e-18 * fabs(sum)) break;
    }
    return sum;
  }
  if (x < (double)MPDPFT_FD_X1) {
    const double m = floor(x);
    const int i = (int)m - MPDPFT_FD_X0;
    const double* c = kFdTab + ((long)o * (MPDPFT_FD_X1 - MPDPFT_FD_X0) + i) * MPDPFT_FD_DEG;
    return cheb_sum(c, MPDPFT_FD_DEG, 2.0 * (x - m) - 1.0);
  }
  const double y = 1.0 / (x * x);
  const double* t = kFdAsym + o * MPDPFT_FD_ASYM;
  double s = 0.0;
  for (int k = MPDPFT_FD_ASYM - 1; k >= 0; --k) s = fma(s, y, __ldg(t + k));
  return -fd_xpow(o, x) * kFdRGamma[o] * s;
}

__device__ __forceinline__ double curly_a(double y) {
  if (y < -1.0e50) return 1.0;
  if (y < -149.99) {
    const double a = -y * sqrt(-y);
    return 1.0 - cos(0.25 * 3.141592653589793 + 0.6666666666666666666 * a) / sqrt(3.141592653589793 * a);
  }
  if (y < MPDPFT_CA_X1) {
    const double u = (y - MPDPFT_CA_X0) / MPDPFT_CA_W;
    int i = (int)floor(u);
    i = i < 0 ? 0 : i;  // [-150, -149.99): the first interval
    return cheb_sum(kCaTab + (long)i * MPDPFT_CA_DEG, MPDPFT_CA_DEG, 2.0 * (u - (double)i) - 1.0);
  }
  const double z = 2.0 / 3.0 * y * sqrt(y);
  return exp(-z) / (2.0 * sqrt(3.141592653589793) * sqrt(sqrt(y)) * sqrt(y));
}

// Ai(y) and Ai'(y) (gsl_sf_airy_Ai / _Ai_deriv at mpDPFT.cpp:3589, 5616,
// 5666): on the CurlyA table's range [-150, 16) the first and second
// derivatives of its Chebyshev series (Ai = -CurlyA', Ai' = -CurlyA''; the
// derivative series by the recurrence d_{k-1} = d_{k+1} + 2 k c_k); outside
// it the asymptotic expansions to third order in 1/zeta, zeta = 2 |y|^{3/2}/3
// (Ai(x) ~ e^{-zeta} sum (-1)^k u_k zeta^{-k} / (2 sqrt(pi) x^{1/4}); for
// negative arguments the sine and cosine series); 0 above 100, as the
// reference sets there.
// coefficients u_k = Gamma(3k + 1/2) / (54^k k! Gamma(k + 1/2)) and
// v_k = -(6k + 1) u_k / (6k - 1) of the asymptotic series, k = 1 .. 3
constexpr double kAiU1 = 0.069444444444444444, kAiU2 = 0.037133487654320988, kAiU3 = 0.037993059127800655;
constexpr double kAiV1 = -0.097222222222222222, kAiV2 = -0.043885030864197531, kAiV3 = -0.042462830789894850;

__device__ __forceinline__ void airy_ai_d(double y, double& ai, double& aip) {
  constexpr double kSqrtPi = 1.7724538509055159;
  if (y > 100.0) { ai = 0.0; aip = 0.0; return; }
  if (y < MPDPFT_CA_X0 || y >= MPDPFT_CA_X1) {
    const double x = fabs(y), r4 = sqrt(sqrt(x)), z = 2.0 / 3.0 * x * sqrt(x);
    if (y < 0.0) {
      const double sn = sin(z + 0.25 * 3.141592653589793), cs = cos(z + 0.25 * 3.141592653589793);
      const double iz = 1.0 / z, iz2 = iz * iz;
      ai = (sn * (1.0 - kAiU2 * iz2) - cs * iz * (kAiU1 - kAiU3 * iz2)) / (kSqrtPi * r4);
      aip = r4 * (-cs * (1.0 - kAiV2 * iz2) - sn * iz * (kAiV1 - kAiV3 * iz2)) / kSqrtPi;
    } else {
      const double e = exp(-z), iz = 1.0 / z;
      ai = e * (1.0 - iz * (kAiU1 - iz * (kAiU2 - iz * kAiU3))) / (2.0 * kSqrtPi * r4);
      aip = -r4 * e * (1.0 - iz * (kAiV1 - iz * (kAiV2 - iz * kAiV3))) / (2.0 * kSqrtPi);
    }
    return;
  }
  const double u = (y - MPDPFT_CA_X0) / MPDPFT_CA_W;
  int i = (int)floor(u);
  i = i < 0 ? 0 : i;
  const double* c = kCaTab + (long)i * MPDPFT_CA_DEG;
  const double t = 2.0 * (u - (double)i) - 1.0;
  double d1[MPDPFT_CA_DEG], d2[MPDPFT_CA_DEG];
  const int n = MPDPFT_CA_DEG;
  d1[n - 1] = 0.0;
  d1[n - 2] = 2.0 * (n - 1) * __ldg(c + n - 1);
  for (int k = n - 2; k >= 1; --k) d1[k - 1] = (k + 1 < n ? d1[k + 1] : 0.0) + 2.0 * k * __ldg(c + k);
  d1[0] *= 0.5;
  d2[n - 1] = 0.0;
  d2[n - 2] = 2.0 * (n - 1) * d1[n - 1];
  for (int k = n - 2; k >= 1; --k) d2[k - 1] = (k + 1 < n ? d2[k + 1] : 0.0) + 2.0 * k * d1[k];
  d2[0] *= 0.5;
  double b1 = 0.0, b2 = 0.0, e1 = 0.0, e2 = 0.0;
  for (int j = n - 1; j >= 1; --j) {
    const double b0 = fma(2.0 * t, b1, d1[j] - b2);
    b2 = b1;
    b1 = b0;
    const double f0 = fma(2.0 * t, e1, d2[j] - e2);
    e2 = e1;
    e1 = f0;
  }
  const double s1 = fma(t, b1, d1[0] - b2), s2 = fma(t, e1, d2[0] - e2);
  const double g = 2.0 / MPDPFT_CA_W;  // dt/dy
  ai = -g * s1;
  aip = -g * g * s2;
}

}  // namespace mpdpft
