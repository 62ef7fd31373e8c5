// common.cuh -- shared device helpers of the B200 DPFT engine.
#pragma once
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>

#include "../../include/mpdpft_gpu.h"

namespace mpdpft {

constexpr double kPi = 3.141592653589793;
constexpr int kThreads = 256;
constexpr int kMaxS = MPDPFT_MAX_SPECIES;
constexpr int kMaxP = MPDPFT_MAX_PULAY;
constexpr int kMuCand = 8;           // candidates per mu-search pass
constexpr int kMuMaxPasses = 24;     // device mu-search pass cap
constexpr int kMaxBlocks = 148 * 8;  // 148 SMs x 8 resident 256-thread blocks

// Device error bits (ScState::status_bits), bit k = mpdpft_status k.
constexpr int kBitNonfinite = 1 << MPDPFT_ERR_NONFINITE;
constexpr int kBitBracket = 1 << MPDPFT_ERR_MU_BRACKET;
constexpr int kBitPulay = 1 << MPDPFT_ERR_PULAY_SINGULAR;
constexpr int kBitTimeout = 1 << MPDPFT_ERR_TIMEOUT;
constexpr int kBitTrapped = 1 << MPDPFT_WARN_MU_TRAPPED;

inline int grid_blocks(long n) {
  long b = (n + kThreads - 1) / kThreads;
  if (b > kMaxBlocks) b = kMaxBlocks;
  if (b < 1) b = 1;
  return (int)b;
}

// Geometry of the periodic grid.
struct Geom {
  int dim;
  int s;
  long n;       // s^dim
  double L, dx, dk;
  double dvol;  // dx^dim: trapezoid weight of every periodic point
};

// Multiplicity of a periodic point in the reference's (s+1)^D storage: plane
// 0 of every axis is stored twice (mpDPFT.cpp:863), so VecMult over that
// storage (mpDPFT.cpp:7103-7107) counts it twice.
// Grid indices use 32-bit arithmetic: grids hold at most 2^30 points.
__device__ __forceinline__ double ref_multiplicity(long p, int s, int dim) {
  const unsigned us = (unsigned)s, pp = (unsigned)p;
  const unsigned q = pp / us, k = pp - q * us;
  const unsigned i = q / us, j = q - i * us;
  double w = (k == 0 ? 2.0 : 1.0) * (j == 0 ? 2.0 : 1.0);
  if (dim == 3) w *= (i == 0 ? 2.0 : 1.0);
  return w;
}

// One 16-byte vector of a field per thread: NP = 16 / sizeof(R) values at
// p0 (a multiple of NP); scalar accesses at the ragged end or when the
// field length is not a multiple of 4 (vec = 0).
template <typename R>
constexpr int kVecPts = 16 / (int)sizeof(R);

template <typename R>
__device__ __forceinline__ void vload(const R* f, long p0, long n, int vec, R (&o)[kVecPts<R>]) {
  constexpr int NP = kVecPts<R>;
  if (vec && p0 + NP - 1 < n) {
    if constexpr (NP == 4) {
      const float4 t = __ldcg(reinterpret_cast<const float4*>(f + p0));
      o[0] = t.x; o[1] = t.y; o[2] = t.z; o[3] = t.w;
    } else {
      const double2 t = __ldcg(reinterpret_cast<const double2*>(f + p0));
      o[0] = t.x; o[1] = t.y;
    }
  } else {
#pragma unroll
    for (int i = 0; i < NP; ++i) o[i] = (p0 + i < n) ? __ldcg(f + p0 + i) : R(0);
  }
}

template <typename R>
__device__ __forceinline__ void vstore(R* f, long p0, long n, int vec, const R (&o)[kVecPts<R>]) {
  constexpr int NP = kVecPts<R>;
  if (vec && p0 + NP - 1 < n) {
    if constexpr (NP == 4) *reinterpret_cast<float4*>(f + p0) = make_float4(o[0], o[1], o[2], o[3]);
    else *reinterpret_cast<double2*>(f + p0) = make_double2(o[0], o[1]);
  } else {
#pragma unroll
    for (int i = 0; i < NP; ++i)
      if (p0 + i < n) f[p0 + i] = o[i];
  }
}

// Trapezoid weight of point q of the reference's (s+1)^D storage (el = s + 1
// points per axis): 1/2 on the first and the last plane of every axis, as in
// Riemann (mpDPFT.cpp:7981-8026).  Indices fit 32 bits (el <= 1025 in 3D).
__device__ __forceinline__ double riemann_weight(unsigned q, unsigned el, int dim) {
  const unsigned t = q / el, k = q - t * el;
  double w = (k == 0 || k == el - 1) ? 0.5 : 1.0;
  if (dim == 3) {
    const unsigned i = t / el, j = t - i * el;
    w *= (j == 0 || j == el - 1) ? 0.5 : 1.0;
    w *= (i == 0 || i == el - 1) ? 0.5 : 1.0;
  } else {
    w *= (t == 0 || t == el - 1) ? 0.5 : 1.0;
  }
  return w;
}

__device__ __forceinline__ void point_coords(long p, const Geom& g, double& x, double& y, double& z) {
  const unsigned us = (unsigned)g.s, pp = (unsigned)p;
  const unsigned q = pp / us, k = pp - q * us;
  if (g.dim == 3) {
    const unsigned i = q / us, j = q - i * us;
    x = -0.5 * g.L + g.dx * i; y = -0.5 * g.L + g.dx * j; z = -0.5 * g.L + g.dx * k;
  } else {
    x = -0.5 * g.L + g.dx * q; y = -0.5 * g.L + g.dx * k; z = 0.0;
  }
}

// Order-preserving 64-bit image of a double (atomicMax of doubles).
__device__ __forceinline__ unsigned long long ordered_bits(double v) {
  unsigned long long b = (unsigned long long)__double_as_longlong(v);
  return (b & 0x8000000000000000ull) ? ~b : (b | 0x8000000000000000ull);
}
__device__ __forceinline__ double from_ordered_bits(unsigned long long b) {
  b = (b & 0x8000000000000000ull) ? (b & 0x7fffffffffffffffull) : ~b;
  return __longlong_as_double((long long)b);
}

// |r - r0| < w from r^2, without the square root (the DelField taper shell).
__device__ __forceinline__ bool in_shell(double r2, double r0, double w) {
  const double lo = r0 - w, hi = r0 + w;
  return r2 < hi * hi && (lo <= 0.0 || r2 > lo * lo);
}

// ---------------------------------------------------------- reductions --
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Reduce NV per-thread accumulators over the block; thread t < NV writes
// the block total of accumulator t to out[t].  Deterministic order.
template <int NV>
__device__ __forceinline__ void block_reduce_store(double (&acc)[NV], double* out) {
  __shared__ double sh[32][NV];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  __syncthreads();  // a previous call may still be reading sh
#pragma unroll
  for (int v = 0; v < NV; ++v) {
    double t = warp_sum(acc[v]);
    if (lane == 0) sh[warp][v] = t;
  }
  __syncthreads();
  for (int v = threadIdx.x; v < NV; v += blockDim.x) {
    double t = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += sh[w][v];
    out[v] = t;
  }
}

// Pairwise sum of n partial values (one block, deterministic), returned to
// every thread of the block.
__device__ inline double block_sum_partials(const double* part, int n, int stride) {
  __shared__ double sh[kThreads];
  double t = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) t += part[(long)i * stride];
  sh[threadIdx.x] = t;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
    __syncthreads();
  }
  double r = sh[0];
  __syncthreads();
  return r;
}

// ---------------------------------------------------- density functionals --
// Parameters of n[V] for one species.  Numbering follows DensityExpression.
struct DensParams {
  int expr;
  int dim;
  double g;        // degeneracy
  double tau;      // tauVec (TF-inspired)
  double T;        // temperature (TF-inspired T>0, gradient 2D)
  double floor_u;  // floor of mu - V in the 3D gradient terms
  double c2;       // |grad V|^2 coefficient (3D gradient form)
  int cut;         // 1: n and dn/dmu vanish wherever mu - V <= 0
  // 3D gradient form at finite T (the reference's getDenEnAt)
  int finite_t;        // 1: Fermi-Dirac form with the Airy-averaged branch
  double airy_thr;     // Airy branch where |grad V|^{2/3}/2 >= airy_thr
  int boole_pairs;     // Boole pairs per half interval
  int boole_max_iter;  // bisection depth
  double rtpna;        // relative accuracy of the Airy integral
  double avg_density;  // AverageDensity = N* / L^D (NegligibleMagnitudeQ scale)
};

// Functionals with a classically forbidden region where n = 0 exactly (TF,
// TF-inspired, 3D gradient-corrected T -> 0 form); the finite-temperature
// forms are positive everywhere.
inline int density_has_cut(int expr, int dim, int finite_t = 0) {
  return expr == MPDPFT_DENS_TF || expr == MPDPFT_DENS_TF_INSPIRED ||
         (expr == MPDPFT_DENS_GRADIENT && dim == 3 && !finite_t);
}

}  // namespace mpdpft

#include "special.cuh"

namespace mpdpft {

// ------------------------------------ 3D gradient form at finite T --------
// getDenEnAt (EnergyQ = 0, Units 1: alpha = 1, tweak = 1; mpDPFT.cpp:
// 3363-3453) with U = V - mu, tau = 1/T, beta0 = -g/(2 pi)^{3/2},
// beta1 = (alpha tau)^{-3/2}, beta2 = -lap/(12 sqrt(alpha tau)),
// ar = |grad V|^{2/3}/2:
//   ar <  threshold  n = beta0 (beta1 Li_{3/2}(-e^{-tau U}) + beta2 Li_{-1/2}(-e^{-tau U}))
//   ar >= threshold  n = int CurlyA(x) prefactor (Li_{1/2} + prefactor2 Li_{-3/2})(-e^{-(U - x ar)/T}) dx
//                    over [2 x0, x0] and [x0, 100] by the reference's adaptive
//                    Boole rule, x0 the first of -2, -4, ... where the
//                    integrand falls below MP = 1e-12 (or -2^27 at most).
// beta2 is taken exactly as the reference writes it (sqrt(T) where the
// Wigner-Kirkwood correction has 1/sqrt(T): the reference's gradient term
// is T times the textbook one); a NaN result counts as 0.
struct AiryArgs {
  double pre, pre2, U, ar, T;
};

__device__ __forceinline__ double airy_integrand(const AiryArgs& A, double x) {
  // nAiTintegrand, 3D, EnergyQ = 0 (mpDPFT.cpp:3614-3619)
  const double arg = -(A.U - x * A.ar) / A.T;
  return A.pre * curly_a(x) * (fd_li(FD_1HALF, arg) + A.pre2 * fd_li(FD_M3HALF, arg));
}

// BooleRule1D (mpDPFT.cpp:8050-8058) over the 4 bp + 1 nodes
// (a + i delta) + off of AdaptiveBoole_nAiT.
__device__ __forceinline__ double airy_boole(const AiryArgs& A, int bp, double a, double delta, double off) {
  const int n = 4 * bp + 1;
  double res = 7.0 * airy_integrand(A, a + 0.0 * delta + off);
  double last = 0.0;
  for (int i = 1; i <= n - 4; i += 4) {
    const double f1 = airy_integrand(A, (a + (double)i * delta) + off);
    const double f2 = airy_integrand(A, (a + (double)(i + 1) * delta) + off);
    const double f3 = airy_integrand(A, (a + (double)(i + 2) * delta) + off);
    const double f4 = airy_integrand(A, (a + (double)(i + 3) * delta) + off);
    res += (32.0 * f1 + 12.0 * f2 + 32.0 * f3 + 14.0 * f4);
    last = f4;
  }
  res -= 14.0 * last;
  res += 7.0 * last;
  return res * (2.0 * delta / 45.0);
}

// NegligibleMagnitudeQ (mpDPFT.cpp:7094-7101)
__device__ __forceinline__ bool negligible_magnitude(double big, double small, double max_exp) {
  if (small == 0.0) return true;
  if (big == 0.0 || big < small) return false;
  return log10(fabs(big)) - log10(fabs(small)) > max_exp;
}

constexpr int kAiryMaxDepth = 24;  // boole_max_iter <= kAiryMaxDepth - 3

// AdaptiveBoole_nAiT (mpDPFT.cpp:3553-3578) without recursion: a stack of
// frames (a, b, previous integral, depth); a frame that does not return
// evaluates its left half, then its right half, and returns their sum, in
// the reference's order.
static __device__ __noinline__ double airy_adaptive(const AiryArgs& A, const DensParams& d, double a0, double b0) {
  struct Frame {
    double a, b, prev, ib, left;
    int iter, stage;
  };
  Frame st[kAiryMaxDepth];
  int sp = 0;
  double ret = 0.0;
  const double mexp = -log10(d.rtpna);
  st[0] = Frame{a0, b0, 0.0, 0.0, 0.0, 0, 0};
  while (sp >= 0) {
    Frame& f = st[sp];
    const double half = 0.5 * (f.b - f.a);
    if (f.stage == 0) {
      const double delta = 0.25 * half / (double)d.boole_pairs;
      const double ia = airy_boole(A, d.boole_pairs, f.a, delta, 0.0);
      const double ib = airy_boole(A, d.boole_pairs, f.a, delta, half);
      const double in = ia + ib;
      bool done;
      if (f.iter > 1 && fabs(in) > 0.0 && fabs((in - f.prev) / in) < d.rtpna) done = true;
      else if (f.iter > d.boole_max_iter) done = true;
      else if (negligible_magnitude(d.avg_density, pow(2.0, (double)f.iter) * in, mexp)) done = true;
      else if (delta < 1.0e-12) done = true;
      else done = sp + 1 >= kAiryMaxDepth;
      if (done) {
        ret = in;
        --sp;
        continue;
      }
      f.ib = ib;
      f.stage = 1;
      st[sp + 1] = Frame{f.a, f.a + half, ia, 0.0, 0.0, f.iter + 1, 0};
      ++sp;
    } else if (f.stage == 1) {
      f.left = ret;
      f.stage = 2;
      st[sp + 1] = Frame{f.a + half, f.b, f.ib, 0.0, 0.0, f.iter + 1, 0};
      ++sp;
    } else {
      ret = f.left + ret;
      --sp;
    }
  }
  return ret;
}

static __device__ __noinline__ double finite_t_density(const DensParams& d, double u, double lap, double g2) {
  const double T = d.T, tau = 1.0 / T, U = -u;
  const double beta0 = -d.g / 15.749609945722419;  // (2 pi)^{3/2}
  const double beta1 = T * sqrt(T);
  const double beta2 = -lap / (12.0 * sqrt(tau));
  const double ar = 0.5 * cbrt(g2 > 0.0 ? g2 : 0.0);
  double res;
  if (ar < d.airy_thr) {
    const double arg = -tau * U;
    res = beta0 * (beta1 * fd_li(FD_3HALF, arg) + beta2 * fd_li(FD_M1HALF, arg));
  } else {
    const AiryArgs A{beta0 * ar * tau * beta1, beta2 / beta1, U, ar, T};
    double x = -1.0, test;
    do {  // lower integration limit (mpDPFT.cpp:3424-3433)
      x *= 2.0;
      const double arg = -tau * (U - x * ar);
      test = beta0 * curly_a(x) * ar * tau * (beta1 * fd_li(FD_1HALF, arg) + beta2 * fd_li(FD_M3HALF, arg));
      if (x < -1.0e8) break;
    } while (fabs(test) > 1.0e-12);
    res = airy_adaptive(A, d, 2.0 * x, x);
    res += airy_adaptive(A, d, x, 100.0);
  }
  return res != res ? 0.0 : res;
}

// dn/dmu of the small-gradient finite-T form, beta0 (beta1 Li_{1/2} +
// beta2 Li_{-3/2}) / T (also used at Airy points: it only places mu
// candidates).
static __device__ __noinline__ double finite_t_slope(const DensParams& d, double u, double lap) {
  const double T = d.T, tau = 1.0 / T;
  const double beta0 = -d.g / 15.749609945722419;
  const double beta1 = T * sqrt(T);
  const double beta2 = -lap / (12.0 * sqrt(tau));
  const double arg = tau * u;
  const double r = beta0 * (beta1 * fd_li(FD_1HALF, arg) + beta2 * fd_li(FD_M3HALF, arg)) * tau;
  return r == r ? r : 0.0;
}

// Pointwise density at u = mu - V (R = float or double arithmetic).
//  7: GetTFdensity (mpDPFT.cpp:4415-4436)
//  1/2: GetTFinspireddensity (mpDPFT.cpp:3318-3347)
//  5: small-gradient branch of getDenEnAt (mpDPFT.cpp:3376-3388): finite-T
//     form in 2D; its T -> 0 limit in 3D,
//     n = g (2u)^{3/2}/(6 pi^2) - g sqrt2/(48 pi^2) [lap u^{-1/2} + c2/4 |gradV|^2 u^{-3/2}],
//     with the singular factors continued linearly to 0 below u = floor.
template <typename R>
__device__ __forceinline__ R density_at(const DensParams& d, R u, R lap, R g2) {
  if (d.expr == MPDPFT_DENS_TF) {
    if (!(u > R(0))) return R(0);
    if (d.dim == 3) return R(1.4142135623730951 * d.g / (3.0 * kPi * kPi)) * u * sqrt(u);
    return R(d.g / (2.0 * kPi)) * u;
  }
  if (d.expr == MPDPFT_DENS_TF_INSPIRED) {
    R t = u / R(d.tau);
    if (!(t > R(0))) return R(0);
    if (d.dim == 3) return t * sqrt(t) * R(sqrt(d.tau));
    return t;
  }
  if (d.expr == MPDPFT_DENS_TF_INSPIRED_T) {
    R pref = R(1.0 / d.tau);
    R t = u * pref;
    R t2 = t / R(d.T);
    if (fabs(t2) < R(40)) return pref * R(d.T) * log(R(1) + exp(t2));
    if (t2 <= R(-40) || t2 != t2) return R(0);
    return pref * t;
  }
  // MPDPFT_DENS_GRADIENT
  if (d.finite_t) return R(finite_t_density(d, (double)u, (double)lap, (double)g2));
  if (d.dim == 2) {
    const R tau = R(1.0 / d.T);
    const R arg = tau * u;  // -tau (V - mu)
    R zeta, LOG;
    if (arg > R(700)) zeta = R(0);
    else zeta = exp(-arg);
    if (arg < R(-100)) LOG = R(1) / zeta;
    else if (arg > R(100)) LOG = arg;
    else LOG = log(R(1) + R(1) / zeta);
    R opz = R(1) + zeta;
    R r = R(d.g / (2.0 * kPi)) * (LOG / tau - tau * lap / R(12) * zeta / (opz * opz));
    return (r != r) ? R(0) : r;
  }
  if (!(u > R(0))) return R(0);
  const R f = R(d.floor_u);
  R m1, m3;
  if (u >= f) { m1 = R(1) / sqrt(u); m3 = m1 / u; }
  else { m1 = u * R(1.0 / (d.floor_u * sqrt(d.floor_u))); m3 = m1 / f; }
  const R ctf = R(2.0 * 1.4142135623730951 * d.g / (6.0 * kPi * kPi));
  const R cg = R(1.4142135623730951 * d.g / (48.0 * kPi * kPi));
  R r = ctf * u * sqrt(u) - cg * (lap * m1 + R(0.25) * R(d.c2) * g2 * m3);
  return r > R(0) ? r : R(0);
}

// Start value of a double-precision 1/sqrt(u), u > 0 normal: the PTX
// approximation rsqrt.approx.ftz.f64, which reads the double itself (an
// FP32 estimate would need two conversions to and from 64-bit types, which
// issue at a quarter of the FP64 FMA rate).  Its error is squared by each
// Newton step of the callers.
__device__ __forceinline__ double rsqrt_seed(double u) {
  double r;
  asm("rsqrt.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(u));
  return r;
}

// 1/sqrt(u) for u > 0 to double precision: the estimate refined by two
// Newton steps r <- r (3 - u r^2)/2 in double (the error squares each step
// and ends below double rounding).  Inputs outside [1e-30, 1e30] fall back
// to the library division.
__device__ __forceinline__ double rsqrt_d(double u) {
  if (u < 1.0e-30 || u > 1.0e30) return 1.0 / sqrt(u);
  double r = rsqrt_seed(u);
  double h = 0.5 * u;
  r = r * fma(-h * r, r, 1.5);
  r = r * fma(-h * r, r, 1.5);
  return r;
}

// The density functionals in double, for the particle-number integral and
// the mu search (same formulas as density_at; square roots via rsqrt_d).
__device__ __forceinline__ double density_at_d(const DensParams& d, double u, double lap, double g2) {
  if (d.expr == MPDPFT_DENS_TF) {
    if (!(u > 0.0)) return 0.0;
    if (d.dim == 3) return (1.4142135623730951 * d.g / (3.0 * kPi * kPi)) * u * u * rsqrt_d(u);
    return (d.g / (2.0 * kPi)) * u;
  }
  if (d.expr == MPDPFT_DENS_GRADIENT && d.dim == 3) {
    if (d.finite_t) return finite_t_density(d, u, lap, g2);
    if (!(u > 0.0)) return 0.0;
    const double ctf = 2.0 * 1.4142135623730951 * d.g / (6.0 * kPi * kPi);
    const double cg = 1.4142135623730951 * d.g / (48.0 * kPi * kPi);
    const double r = rsqrt_d(u);
    double m1, m3;
    if (u >= d.floor_u) { m1 = r; m3 = r * r * r; }
    else {
      const double rf = rsqrt_d(d.floor_u);
      m1 = u * rf / d.floor_u;
      m3 = m1 / d.floor_u;
    }
    const double v = ctf * u * u * r - cg * (lap * m1 + 0.25 * d.c2 * g2 * m3);
    return v > 0.0 ? v : 0.0;
  }
  return density_at<double>(d, u, lap, g2);
}

// dn/dmu (= dn/du) of each functional, in double, for the Newton placement
// of mu candidates.  Zero where the density is clamped at 0.
__device__ __forceinline__ double density_slope_d(const DensParams& d, double u, double lap, double g2) {
  if (d.expr == MPDPFT_DENS_TF) {
    if (!(u > 0.0)) return 0.0;
    if (d.dim == 3) return 1.5 * (1.4142135623730951 * d.g / (3.0 * kPi * kPi)) * u * rsqrt_d(u);
    return d.g / (2.0 * kPi);
  }
  if (d.expr == MPDPFT_DENS_TF_INSPIRED) {
    const double t = u / d.tau;
    if (!(t > 0.0)) return 0.0;
    if (d.dim == 3) return 1.5 * t * rsqrt_d(t) * sqrt(d.tau) / d.tau;
    return 1.0 / d.tau;
  }
  if (d.expr == MPDPFT_DENS_TF_INSPIRED_T) {
    const double t2 = u / (d.tau * d.T);
    if (t2 <= -40.0 || t2 != t2) return 0.0;
    if (t2 >= 40.0) return 1.0 / (d.tau * d.tau);
    return 1.0 / (1.0 + exp(-t2)) / (d.tau * d.tau);
  }
  // gradient-corrected
  if (d.finite_t) return finite_t_slope(d, u, lap);
  if (d.dim == 2) {
    const double tau = 1.0 / d.T;
    const double arg = tau * u;
    if (arg > 700.0) return d.g / (2.0 * kPi);
    if (arg < -700.0) return 0.0;
    const double z = exp(-arg), opz = 1.0 + z;
    const double r = d.g / (2.0 * kPi) * (1.0 / opz + tau * tau * lap / 12.0 * z * (1.0 - z) / (opz * opz * opz));
    return r == r ? r : 0.0;
  }
  if (!(u > 0.0)) return 0.0;
  const double ctf = 2.0 * 1.4142135623730951 * d.g / (6.0 * kPi * kPi);
  const double cg = 1.4142135623730951 * d.g / (48.0 * kPi * kPi);
  const double r = rsqrt_d(u);
  double m1, m3, dm1, dm3;
  if (u >= d.floor_u) {
    m1 = r; m3 = r * r * r;
    dm1 = -0.5 * m3; dm3 = -1.5 * m3 * r * r;
  } else {
    const double rf = rsqrt_d(d.floor_u);
    dm1 = rf / d.floor_u; m1 = u * dm1;
    dm3 = dm1 / d.floor_u; m3 = u * dm3;
  }
  const double n = ctf * u * u * r - cg * (lap * m1 + 0.25 * d.c2 * g2 * m3);
  if (!(n > 0.0)) return 0.0;
  return 1.5 * ctf * u * r - cg * (lap * dm1 + 0.25 * d.c2 * g2 * dm3);
}

// FP32 evaluation for the mixed-precision mu search: u is formed in double
// from the double candidate mu and then rounded once, so N(mu) keeps the
// resolution of double mu (a staircase of 2M per-point steps of relative size
// ~1e-7 / 2M, far below RelAcc); the sum is accumulated in double.
__device__ __forceinline__ float density_at_f(const DensParams& d, float u, float lap, float g2) {
  if (d.expr == MPDPFT_DENS_TF) {
    if (!(u > 0.f)) return 0.f;
    if (d.dim == 3) return float(1.4142135623730951 * d.g / (3.0 * kPi * kPi)) * u * u * rsqrtf(u);
    return float(d.g / (2.0 * kPi)) * u;
  }
  if (d.expr == MPDPFT_DENS_GRADIENT && d.dim == 3) {
    if (!(u > 0.f)) return 0.f;
    const float ctf = float(2.0 * 1.4142135623730951 * d.g / (6.0 * kPi * kPi));
    const float cg = float(1.4142135623730951 * d.g / (48.0 * kPi * kPi));
    const float fl = float(d.floor_u);
    float m1, m3;
    if (u >= fl) { m1 = rsqrtf(u); m3 = m1 * m1 * m1; }
    else { m1 = u * float(1.0 / (d.floor_u * sqrt(d.floor_u))); m3 = m1 / fl; }
    const float v = ctf * u * u * rsqrtf(u) - cg * (lap * m1 + 0.25f * float(d.c2) * g2 * m3);
    return v > 0.f ? v : 0.f;
  }
  return density_at<float>(d, u, lap, g2);
}

// d n / d mu at u (used to place mu candidates; accuracy is not critical).
template <typename R>
__device__ __forceinline__ R density_slope(const DensParams& d, R u) {
  if (!(u > R(0))) return R(0);
  if (d.dim == 3) return R(1.5 * 1.4142135623730951 * d.g / (3.0 * kPi * kPi)) * sqrt(u);
  return R(d.g / (2.0 * kPi));
}

// Programmatic dependent launch.  A kernel launched with
// cudaLaunchAttributeProgrammaticStreamSerialization may begin while the
// kernel before it on the stream is still running: pdl_wait() returns once
// that kernel has completed and its memory is visible (a no-op for a kernel
// launched without the attribute), pdl_trigger() lets the next kernel begin
// once every block of this one has called it or exited.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

// Kernel launch with programmatic stream serialization (the kernels of the
// SC iteration call pdl_wait before touching memory and pdl_trigger when
// their block is done), process-wide unless a captured graph with
// programmatic edges could not be built (pdl_disable).
bool pdl_enabled();
void pdl_disable();
template <typename... P, typename... A>
inline cudaError_t launch_k(void (*k)(P...), dim3 grid, dim3 block, size_t smem, cudaStream_t st, A&&... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = pdl_enabled() ? 1 : 0;
  return cudaLaunchKernelEx(&cfg, k, static_cast<A&&>(args)...);
}

// e^{-x} I0(x) for x >= 0 (the exponentially scaled modified Bessel function
// of the 2D Coulomb compensation term, mpDPFT.cpp:2659).  Below x = 30 the
// power series I0(x) = sum_k (x^2/4)^k / (k!)^2 (positive terms, no
// cancellation) times e^{-x}; above, the asymptotic expansion
// e^{-x} I0(x) ~ (2 pi x)^{-1/2} sum_k [(2k-1)!!]^2 / (k! (8x)^k), whose
// terms fall below 1e-17 of the sum long before they start to grow.
__host__ __device__ inline double bessel_i0e(double x) {
  if (x < 30.0) {
    const double q = 0.25 * x * x;
    double t = 1.0, sum = 1.0;
    for (int k = 1; k < 200; ++k) {
      t *= q / ((double)k * (double)k);
      sum += t;
      if (t < 1.0e-17 * sum) break;
    }
    return sum * exp(-x);
  }
  double t = 1.0, sum = 1.0;
  for (int k = 1; k < 40; ++k) {
    const double a = 2.0 * k - 1.0;
    t *= a * a / (8.0 * k * x);
    sum += t;
    if (t < 1.0e-17 * sum) break;
  }
  return sum / sqrt(2.0 * kPi * x);
}

}  // namespace mpdpft
