// sc_kernel.cuh -- the kernels of one SC iteration and their block-level
// helpers.  State, parameters and the mu-search decisions are in
// sc_step.cuh.
//
// One iteration is three launches on the context stream:
//   sc_mu_kernel       cooperative, one block per SM: UpdateV (when V is not
//                      assembled by the FFT path) and the mu search, whose
//                      passes are separated by bounded grid barriers;
//   sc_density_kernel  all points at full occupancy: final densities,
//                      residual, convergence dots and the Pulay Gram row; its
//                      last block to finish runs the scalar logic
//                      (CheckConvergence ... InjectSchedule, Pulay solve);
//   sc_mix_kernel      all points: the mixed density into the next ring slot.
// The mu search of a functional that vanishes for mu <= V evaluates only
// the points below the largest candidate: a sweep over V compacts them (in
// grid order) into a list that later passes reuse while their candidates
// stay below the bound, and every thread of the grid takes an equal share of
// the list.  The 3D gradient-corrected and TF functionals are evaluated in a
// branch-free form so that all candidates of a point run side by side.
#pragma once
#include "sc_step.cuh"

namespace mpdpft {

// ---------------------------------------------------------- small solve --
// Inverse of the Pulay Gram matrix (n <= kMaxP) by Gauss-Jordan elimination
// with full pivoting; rank test as Eigen's FullPivHouseholderQR::isInvertible
// (threshold eps * n * max|pivot|), which the reference uses
// (mpDPFT.cpp:5089).  Each pivot is the first maximum, in row-major order,
// among the rows and columns not used yet; rows are never swapped (row pc_k
// of the inverse is row pr_k of R).  Runs on the first `nthr` threads of the
// block (whole warps), synchronised with named barrier 1 so that the other
// warps can work meanwhile: warp 0 finds each pivot, every thread updates
// elements of [M | R].  A matrix with no finite pivot left (NaN or Inf
// entries) is reported singular.
__device__ __forceinline__ void group_bar(int nthr) { asm volatile("bar.sync 1, %0;" ::"r"(nthr) : "memory"); }

__device__ inline bool group_inverse(int n, const double* G, double* M, double* Rm, double* inv, int* colof,
                                     double* s_pv, int* s_pi, int nthr) {
  const int t = threadIdx.x, lane = t & 31;
  const int nn = n * n;
  for (int e = t; e < nn; e += nthr) {
    M[e] = G[e];
    Rm[e] = (e / n == e % n) ? 1.0 : 0.0;
  }
  if (t == 0) { s_pi[2] = 0; s_pi[3] = 0; s_pv[1] = 0.0; s_pv[2] = 1e300; }  // used rows, used cols, max, min pivot
  group_bar(nthr);
  for (int c = 0; c < n; ++c) {
    if (t < 32) {  // first maximum |M| over unused rows and columns, row-major order
      const unsigned ur = (unsigned)s_pi[2], uc = (unsigned)s_pi[3];
      double best = -1.0;
      int be = 0x7fffffff;
      for (int e = lane; e < nn; e += 32) {
        const int i = e / n, j = e % n;
        if (((ur >> i) & 1u) || ((uc >> j) & 1u)) continue;
        const double v = fabs(M[e]);
        if (v > best) { best = v; be = e; }
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        const double ob = __shfl_xor_sync(0xffffffffu, best, o);
        const int oe = __shfl_xor_sync(0xffffffffu, be, o);
        if (ob > best || (ob == best && oe < be)) { best = ob; be = oe; }
      }
      if (lane == 0) {
        if (be >= nn || !(best <= 1.0e300)) {  // no finite pivot: singular
          s_pi[0] = 0;
          s_pi[1] = 0;
          s_pv[0] = 0.0;
        } else {
          const int pr = be / n, pc = be % n;
          s_pi[0] = pr;
          s_pi[1] = pc;
          s_pv[0] = M[be];
          s_pv[1] = fmax(s_pv[1], best);
          s_pv[2] = fmin(s_pv[2], best);
          s_pi[2] |= 1 << pr;
          s_pi[3] |= 1 << pc;
          colof[pr] = pc;
        }
      }
    }
    group_bar(nthr);
    const int pr = s_pi[0], pc = s_pi[1];
    const double piv = s_pv[0];
    if (piv == 0.0) return false;  // same value for every thread
    const double ip = 1.0 / piv;
    // new values of this thread's (at most two) elements: 2 n^2 <= 288 <= 2 nthr
    auto updated = [&](int e) -> double {
      const bool right = e >= nn;
      const int ee = right ? e - nn : e;
      const int i = ee / n, j = ee % n;
      const double* X = right ? Rm : M;
      return (i == pr) ? X[ee] * ip : X[ee] - M[i * n + pc] * ip * X[pr * n + j];
    };
    const int e0 = t, e1 = t + nthr;
    const double v0 = e0 < 2 * nn ? updated(e0) : 0.0;
    const double v1 = e1 < 2 * nn ? updated(e1) : 0.0;
    group_bar(nthr);
    if (e0 < 2 * nn) { if (e0 >= nn) Rm[e0 - nn] = v0; else M[e0] = v0; }
    if (e1 < 2 * nn) { if (e1 >= nn) Rm[e1 - nn] = v1; else M[e1] = v1; }
    group_bar(nthr);
  }
  if (s_pv[2] <= 2.220446049250313e-16 * (double)n * s_pv[1]) return false;
  for (int e = t; e < nn; e += nthr) inv[colof[e / n] * n + e % n] = Rm[e];
  group_bar(nthr);
  return true;
}

// sum_{i,j} ((inv G)_{ij} - delta_ij)^2 on one warp (the reference's
// validation of the inverse, mpDPFT.cpp:5099-5107)
__device__ inline double warp_inverse_defect(int n, const double* G, const double* inv) {
  const int lane = threadIdx.x & 31;
  double test = 0.0;
  for (int e = lane; e < n * n; e += 32) {
    const int i = e / n, j = e % n;
    double t = 0.0;
    for (int k = 0; k < n; ++k) t += inv[i * n + k] * G[k * n + j];
    t -= (i == j) ? 1.0 : 0.0;
    test += t * t;
  }
  return warp_sum(test);
}

// ------------------------------------------------------------ segments --
template <typename R>
__device__ __forceinline__ void load4(const R* f, long p0, long n, int vec4, R (&o)[4]) {
  if (vec4 && p0 + 3 < n) {
    if constexpr (sizeof(R) == sizeof(float)) {
      const float4 t = __ldcg(reinterpret_cast<const float4*>(f + p0));
      o[0] = t.x; o[1] = t.y; o[2] = t.z; o[3] = t.w;
    } else {
      const double2 t0 = __ldcg(reinterpret_cast<const double2*>(f + p0));
      const double2 t1 = __ldcg(reinterpret_cast<const double2*>(f + p0 + 2));
      o[0] = t0.x; o[1] = t0.y; o[2] = t1.x; o[3] = t1.y;
    }
  } else {
#pragma unroll
    for (int i = 0; i < 4; ++i) o[i] = (p0 + i < n) ? __ldcg(f + p0 + i) : R(0);
  }
}

template <typename R>
__device__ __forceinline__ void store4(R* f, long p0, long n, int vec4, const R (&o)[4]) {
  if (vec4 && p0 + 3 < n) {
    if constexpr (sizeof(R) == sizeof(float)) {
      *reinterpret_cast<float4*>(f + p0) = make_float4(o[0], o[1], o[2], o[3]);
    } else {
      *reinterpret_cast<double2*>(f + p0) = make_double2(o[0], o[1]);
      *reinterpret_cast<double2*>(f + p0 + 2) = make_double2(o[2], o[3]);
    }
  } else {
#pragma unroll
    for (int i = 0; i < 4; ++i)
      if (p0 + i < n) f[p0 + i] = o[i];
  }
}

// Reference-storage multiplicities (ref_multiplicity) of points p0 .. p0+NP-1.
template <int NP>
__device__ __forceinline__ void ref_weights(long p0, int s, int dim, double (&w)[NP]) {
  const unsigned us = (unsigned)s;
  unsigned p = (unsigned)p0;
  unsigned k = p % us, q = p / us;
  unsigned j = q % us, i = q / us;
#pragma unroll
  for (int t = 0; t < NP; ++t) {
    w[t] = (k == 0 ? 2.0 : 1.0) * (j == 0 ? 2.0 : 1.0) * ((dim == 3 && i == 0) ? 2.0 : 1.0);
    if (++k == us) {
      k = 0;
      if (++j == us) { j = 0; ++i; }
    }
  }
}

// ------------------------------------------------------- point evaluation --
// Constants of the branch-free forms (fast = 1: 3D gradient-corrected,
// fast = 2: 3D TF, 0: the general density_at_d / density_slope_d).
struct EvalK {
  int fast;
  double ctf;     // TF prefactor
  double cg;      // gradient prefactor (times lap)
  double cg2;     // gradient prefactor times c2 / 4 (times |grad V|^2)
  double floor_u, c1, c3;  // below floor: u^{-1/2} -> u c1, u^{-3/2} -> u c3
  double c2d, T, invT, lt;  // 2D finite-T form: g/(2 pi), T, 1/T, 1/(12 T)
};

__device__ __forceinline__ EvalK eval_constants(const DensParams& d) {
  EvalK k;
  k.fast = 0;
  k.ctf = k.cg = k.cg2 = k.floor_u = k.c1 = k.c3 = 0.0;
  k.c2d = k.T = k.invT = k.lt = 0.0;
  if (d.expr == MPDPFT_DENS_GRADIENT && d.dim == 3) {
    k.fast = 1;
    k.ctf = 2.0 * 1.4142135623730951 * d.g / (6.0 * kPi * kPi);
    k.cg = 1.4142135623730951 * d.g / (48.0 * kPi * kPi);
    k.cg2 = k.cg * 0.25 * d.c2;
    k.floor_u = d.floor_u;
    k.c1 = rsqrt_d(d.floor_u) / d.floor_u;
    k.c3 = k.c1 / d.floor_u;
  } else if (d.expr == MPDPFT_DENS_TF && d.dim == 3) {
    k.fast = 2;
    k.ctf = 1.4142135623730951 * d.g / (3.0 * kPi * kPi);
  } else if (d.expr == MPDPFT_DENS_GRADIENT && d.dim == 2) {
    k.fast = 3;
    k.c2d = d.g / (2.0 * kPi);
    k.T = d.T;
    k.invT = 1.0 / d.T;
    k.lt = 1.0 / (12.0 * d.T);
  }
  return k;
}

// rsqrt_d without its range branch (callers keep u normal and positive).
__device__ __forceinline__ double rsqrt_nr(double u) {
  double r = rsqrt_seed(u);
  const double h = 0.5 * u;
  r = r * fma(-h * r, r, 1.5);
  r = r * fma(-h * r, r, 1.5);
  return r;
}

// n(u) of the 3D gradient-corrected form for A = cg lap, B = cg c2/4 |grad V|^2
// (density_at_d without branches: u^{-1/2}, u^{-3/2} continued linearly below
// the floor, n = 0 for u <= 0 or a negative value).
// HB: the |grad V|^2 term is present (B != 0); without it the u^{-3/2}
// factor is not formed.  u is replaced by 1 where it is not in
// [1e-30, 1e30] before the square root (the result is 0 for u <= 0, and u
// stays far inside the range elsewhere), with selects rather than FP64
// min/max instructions.
template <bool HB = true>
__device__ __forceinline__ double grad3_n(const EvalK& k, double u, double A, double B) {
  const bool pos = u > 0.0;
  const double r = rsqrt_nr(u > 1.0e-30 && u < 1.0e30 ? u : 1.0);
  const bool hi = u >= k.floor_u;
  const double m1 = hi ? r : u * k.c1;
  double v = k.ctf * u * u * r - A * m1;
  if constexpr (HB) v -= B * (hi ? r * r * r : u * k.c3);
  return (pos && v > 0.0) ? v : 0.0;
}

// n(u) and dn/du of the same form with one reciprocal square root.
template <bool HB = true>
__device__ __forceinline__ double grad3_n_slope(const EvalK& k, double u, double A, double B, double& sl) {
  const double r = rsqrt_nr(u > 1.0e-30 && u < 1.0e30 ? u : 1.0);
  const bool hi = u >= k.floor_u;
  const double r3 = r * r * r;
  const double m1 = hi ? r : u * k.c1;
  const double dm1 = hi ? -0.5 * r3 : k.c1;
  double v = k.ctf * u * u * r - A * m1;
  double dv = 1.5 * k.ctf * u * r - A * dm1;
  if constexpr (HB) {
    v -= B * (hi ? r3 : u * k.c3);
    dv -= B * (hi ? -1.5 * r3 * r * r : k.c3);
  }
  const bool pos = u > 0.0 && v > 0.0;
  sl = pos ? dv : 0.0;
  return pos ? v : 0.0;
}

// dn/du of the same form (density_slope_d), zero where n is clamped.
__device__ __forceinline__ double grad3_slope(const EvalK& k, double u, double A, double B) {
  const double r = rsqrt_nr(fmin(fmax(u, 1.0e-30), 1.0e30));
  const bool hi = u >= k.floor_u;
  const double r3 = r * r * r;
  const double m1 = hi ? r : u * k.c1;
  const double m3 = hi ? r3 : u * k.c3;
  const double dm1 = hi ? -0.5 * r3 : k.c1;
  const double dm3 = hi ? -1.5 * r3 * r * r : k.c3;
  const double v = k.ctf * u * u * r - (A * m1 + B * m3);
  const double sl = 1.5 * k.ctf * u * r - (A * dm1 + B * dm3);
  return (u > 0.0 && v > 0.0) ? sl : 0.0;
}

__device__ __forceinline__ double tf3_n(const EvalK& k, double u) {
  const double r = rsqrt_nr(u > 1.0e-30 && u < 1.0e30 ? u : 1.0);
  return u > 0.0 ? k.ctf * u * u * r : 0.0;
}

__device__ __forceinline__ double tf3_slope(const EvalK& k, double u) {
  const double r = rsqrt_nr(u > 1.0e-30 && u < 1.0e30 ? u : 1.0);
  return u > 0.0 ? 1.5 * k.ctf * u * r : 0.0;
}

// 2D gradient-corrected density at finite T (the small-gradient branch of
// getDenEnAt, mpDPFT.cpp:3376-3384) in logistic form.  With a = (mu - V)/T
// and s(a) = 1/(1 + e^{-a}):
//   n      = g/(2 pi) [T softplus(a) - lap/(12 T) s (1 - s)],
//   dn/dmu = g/(2 pi) [s - lap/(12 T^2) s (1 - s)(1 - 2 s)];
// one exponential e = exp(-|a|) gives softplus(a) = max(a, 0) + log1p(e),
// s = (a >= 0 ? 1 : e)/(1 + e) and s (1 - s) = e/(1 + e)^2 (the reference's
// zeta = e^{-a}; its +-100 cut-offs are the two tails of the same forms).
__device__ __forceinline__ double g2d_n(const EvalK& k, double u, double l) {
  const double a = u * k.invT;
  const double e = exp(-fabs(a));
  const double ope = 1.0 + e;
  const double r = k.c2d * (k.T * (fmax(a, 0.0) + log1p(e)) - l * k.lt * (e / (ope * ope)));
  return r == r ? r : 0.0;
}

// n from a = u/T and e = exp(-|a|) given.
__device__ __forceinline__ double g2d_n_e(const EvalK& k, double a, double e, double l) {
  const double ope = 1.0 + e;
  const double r = k.c2d * (k.T * (fmax(a, 0.0) + log1p(e)) - l * k.lt * (e / (ope * ope)));
  return r == r ? r : 0.0;
}

// n and dn/dmu together (one exponential).
__device__ __forceinline__ void g2d_n_slope(const EvalK& k, double u, double l, double& n, double& slope) {
  const double a = u * k.invT;
  const double e = exp(-fabs(a));
  const double ope = 1.0 + e;
  const double rope = 1.0 / ope;
  const double sg = (a >= 0.0 ? 1.0 : e) * rope;
  const double q = e * rope * rope;
  const double r = k.c2d * (k.T * (fmax(a, 0.0) + log1p(e)) - l * k.lt * q);
  const double d = k.c2d * (sg - l * k.lt * k.invT * q * (1.0 - 2.0 * sg));
  n = r == r ? r : 0.0;
  slope = d == d ? d : 0.0;
}

// Functional kind, a template parameter of the kernels so that each
// instantiation carries only its own evaluation code: 1 = 3D
// gradient-corrected, 2 = 3D TF, 3 = 2D gradient-corrected, 0 = any
// (density_at_d).  The point values are FP64 in both precisions: the mu
// search resolves N to RelAcc (1e-10), below the rounding of FP32 values.
inline int functional_kind(int expr, int dim, int finite_t = 0) {
  if (expr == MPDPFT_DENS_GRADIENT && dim == 3 && finite_t) return 0;
  if (expr == MPDPFT_DENS_GRADIENT && dim == 3) return 1;
  if (expr == MPDPFT_DENS_TF && dim == 3) return 2;
  if (expr == MPDPFT_DENS_GRADIENT && dim == 2) return 3;
  return 0;
}

// Density kernel variant for a Pulay window (the PW template argument):
// 1 -> 5, 3 -> 8, 2 -> kMaxP.
inline int density_variant(int window) { return window <= 5 ? 1 : (window <= 8 ? 3 : 2); }

// n at u = mu - V for one point.
template <int FK>
__device__ __forceinline__ double point_density(const DensParams& d, const EvalK& k, double u, double l, double g) {
  if constexpr (FK == 1) return grad3_n(k, u, k.cg * l, k.cg2 * g);
  else if constexpr (FK == 2) return tf3_n(k, u);
  else if constexpr (FK == 3) return g2d_n(k, u, l);
  else return density_at_d(d, u, l, g);
}

// N(mu_c) contributions of one point for the nc candidates, and dN/dmu at
// candidate 0.
// kx (2D form only): per candidate exp(-(mu_c - mu_0)/T) at [c] and its
// inverse at [kMuCand + c], 0 where the step is too large to share the
// exponential of candidate 0 (then exp(-|a_c|) is taken directly).
template <int FK>
__device__ __forceinline__ void mu_point(const DensParams& d, const EvalK& k, const double* cmu, int nc, double v,
                                         double l, double g, double (&acc)[kMuAcc], const double* kx = nullptr) {
  if constexpr (FK == 1) {
    const double A = k.cg * l, B = k.cg2 * g;
    double sl;
    acc[0] += grad3_n_slope(k, cmu[0] - v, A, B, sl);
    acc[kMuCand] += sl;
#pragma unroll
    for (int c = 1; c < kMuCand; ++c) {
      if (c >= nc) break;
      acc[c] += grad3_n(k, cmu[c] - v, A, B);
    }
  } else if constexpr (FK == 2) {
    acc[kMuCand] += tf3_slope(k, cmu[0] - v);
#pragma unroll
    for (int c = 0; c < kMuCand; ++c) {
      if (c >= nc) break;
      acc[c] += tf3_n(k, cmu[c] - v);
    }
  } else if constexpr (FK == 3) {
    const double a0 = (cmu[0] - v) * k.invT;
    const double e0 = exp(-fabs(a0));
    {
      const double ope = 1.0 + e0, rope = 1.0 / ope;
      const double sg = (a0 >= 0.0 ? 1.0 : e0) * rope;
      const double q = e0 * rope * rope;
      const double r = k.c2d * (k.T * (fmax(a0, 0.0) + log1p(e0)) - l * k.lt * q);
      const double dd = k.c2d * (sg - l * k.lt * k.invT * q * (1.0 - 2.0 * sg));
      acc[0] += r == r ? r : 0.0;
      acc[kMuCand] += dd == dd ? dd : 0.0;
    }
    // e_c = e_0 exp(-+(a_c - a_0)) while a_c keeps the sign of a_0
    const int side = a0 >= 0.0 ? 0 : kMuCand;
#pragma unroll
    for (int c = 1; c < kMuCand; ++c) {
      if (c >= nc) break;
      const double a = (cmu[c] - v) * k.invT;
      const double kk = kx[side + c];
      const double e = ((a >= 0.0) == (a0 >= 0.0) && kk > 0.0) ? e0 * kk : exp(-fabs(a));
      acc[c] += g2d_n_e(k, a, e, l);
    }
  } else {
    acc[kMuCand] += density_slope_d(d, cmu[0] - v, l, g);
#pragma unroll
    for (int c = 0; c < kMuCand; ++c) {
      if (c >= nc) break;
      acc[c] += density_at_d(d, cmu[c] - v, l, g);
    }
  }
}

// The 3D gradient-corrected form of mu_points (below), HB as for grad3_n.
template <bool HB, int NPT, typename R>
__device__ __forceinline__ void mu_points_grad3(const EvalK& k, const double* cmu, int nc, const R (&vr)[NPT],
                                                const R (&lr)[NPT], const R (&gr)[NPT], const bool (&ok)[NPT],
                                                double (&acc)[kMuAcc]) {
  double v[NPT], A[NPT], B[NPT];
#pragma unroll
  for (int i = 0; i < NPT; ++i) {
    v[i] = (double)vr[i];
    A[i] = k.cg * (double)lr[i];
    B[i] = HB ? k.cg2 * (double)gr[i] : 0.0;
  }
#pragma unroll
  for (int i = 0; i < NPT; ++i) {
    double sl;
    const double n0 = grad3_n_slope<HB>(k, cmu[0] - v[i], A[i], B[i], sl);
    acc[0] += ok[i] ? n0 : 0.0;
    acc[kMuCand] += ok[i] ? sl : 0.0;
  }
#pragma unroll
  for (int c = 1; c < kMuCand; ++c) {
    if (c >= nc) break;
    double t = 0.0;
#pragma unroll
    for (int i = 0; i < NPT; ++i) {
      const double x = grad3_n<HB>(k, cmu[c] - v[i], A[i], B[i]);
      t += ok[i] ? x : 0.0;
    }
    acc[c] += t;
  }
}

// mu_point for the NPT points of a lane's trip (ok[i]: point i exists):
// the candidate loop is the outer one, so the points' evaluations are NPT
// independent chains.
template <int FK, int NPT, typename R>
__device__ __forceinline__ void mu_points(const DensParams& d, const EvalK& k, const double* cmu, int nc,
                                          const R (&vr)[NPT], const R (&lr)[NPT], const R (&gr)[NPT],
                                          const bool (&ok)[NPT], double (&acc)[kMuAcc], const double* kx) {
  if constexpr (FK == 1) {
    // the reference's small-gradient branch has no |grad V|^2 term
    if (k.cg2 == 0.0) mu_points_grad3<false, NPT>(k, cmu, nc, vr, lr, gr, ok, acc);
    else mu_points_grad3<true, NPT>(k, cmu, nc, vr, lr, gr, ok, acc);
  } else if constexpr (FK == 2) {
    double v[NPT];
#pragma unroll
    for (int i = 0; i < NPT; ++i) v[i] = (double)vr[i];
#pragma unroll
    for (int i = 0; i < NPT; ++i) {
      acc[0] += ok[i] ? tf3_n(k, cmu[0] - v[i]) : 0.0;
      acc[kMuCand] += ok[i] ? tf3_slope(k, cmu[0] - v[i]) : 0.0;
    }
#pragma unroll
    for (int c = 1; c < kMuCand; ++c) {
      if (c >= nc) break;
      double t = 0.0;
#pragma unroll
      for (int i = 0; i < NPT; ++i) t += ok[i] ? tf3_n(k, cmu[c] - v[i]) : 0.0;
      acc[c] += t;
    }
  } else {
#pragma unroll
    for (int i = 0; i < NPT; ++i)
      if (ok[i]) mu_point<FK>(d, k, cmu, nc, (double)vr[i], (double)lr[i], (double)gr[i], acc, kx);
  }
}

// Sum of nb per-block partials (at base + b * stride) on one warp, several
// loads in flight per lane.
__device__ __forceinline__ double warp_sum_rows(const double* base, int nb, int stride) {
  const int lane = threadIdx.x & 31;
  double t = 0.0;
#pragma unroll 4
  for (int b = lane; b < nb; b += 32) t += __ldcg(base + (long)b * stride);
  return warp_sum(t);
}

// Sums over nb per-block rows (row b of value v at
// base[b * stride + (v / per) * pstride + v % per]) of nv values into
// out[(v / per) * pstride + v % per], by all threads of the block with every
// thread's loads in flight together (CH values at a time).
__device__ inline void block_rows_sum(const double* base, int nb, int stride, int nv, int per, int pstride,
                                      double* out) {
  constexpr int CH = 8;
  __shared__ double sh[32][CH];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int c0 = 0; c0 < nv; c0 += CH) {
    double t[CH];
    int off[CH];
#pragma unroll
    for (int u = 0; u < CH; ++u) {
      t[u] = 0.0;
      const int v = c0 + u < nv ? c0 + u : c0;
      off[u] = (v / per) * pstride + v % per;
    }
    for (int b = threadIdx.x; b < nb; b += blockDim.x) {
      const double* row = base + (long)b * stride;
#pragma unroll
      for (int u = 0; u < CH; ++u) t[u] += __ldcg(row + off[u]);
    }
    __syncthreads();  // sh is free
#pragma unroll
    for (int u = 0; u < CH; ++u) {
      const double x = warp_sum(t[u]);
      if (lane == 0) sh[w][u] = x;
    }
    __syncthreads();
    if (threadIdx.x < CH && c0 + (int)threadIdx.x < nv) {
      double x = 0.0;
      for (int i = 0; i < nw; ++i) x += sh[i][threadIdx.x];
      const int v = c0 + threadIdx.x;
      out[(v / per) * pstride + v % per] = x;
    }
  }
  __syncthreads();
}

// Two sources in one pass (all threads, CH2 values at a time): nv1 values of
// nb1 rows as block_rows_sum, then nv2 values (v at base2[b * stride2 + v])
// of nb2 rows into out2.
__device__ inline void block_rows_sum2(const double* base1, int nb1, int stride1, int nv1, int per, int pstride,
                                       double* out1, const double* base2, int nb2, int stride2, int nv2,
                                       double* out2) {
  constexpr int CH2 = 16;
  __shared__ double sh[32][CH2];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const int nv = nv1 + nv2;
  const int nb = nb1 > nb2 ? nb1 : nb2;
  for (int c0 = 0; c0 < nv; c0 += CH2) {
    double t[CH2];
#pragma unroll
    for (int u = 0; u < CH2; ++u) t[u] = 0.0;
    for (int b = threadIdx.x; b < nb; b += blockDim.x) {
#pragma unroll
      for (int u = 0; u < CH2; ++u) {
        const int v = c0 + u;
        if (v < nv1) {
          if (b < nb1) t[u] += __ldcg(base1 + (long)b * stride1 + (v / per) * pstride + v % per);
        } else if (v < nv) {
          if (b < nb2) t[u] += __ldcg(base2 + (long)b * stride2 + (v - nv1));
        }
      }
    }
    __syncthreads();  // sh is free
#pragma unroll
    for (int u = 0; u < CH2; ++u) {
      const double x = warp_sum(t[u]);
      if (lane == 0) sh[w][u] = x;
    }
    __syncthreads();
    if (threadIdx.x < CH2 && c0 + (int)threadIdx.x < nv) {
      double x = 0.0;
      for (int i = 0; i < nw; ++i) x += sh[i][threadIdx.x];
      const int v = c0 + threadIdx.x;
      if (v < nv1) out1[(v / per) * pstride + v % per] = x;
      else out2[v - nv1] = x;
    }
  }
  __syncthreads();
}

// Block-wide sums of two ints, returned to every thread.
__device__ __forceinline__ void block_sum2(int& x, int& y) {
  __shared__ int sh[2][kStepWarps];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  x = __reduce_add_sync(0xffffffffu, x);
  y = __reduce_add_sync(0xffffffffu, y);
  __syncthreads();
  if (lane == 0) { sh[0][w] = x; sh[1][w] = y; }
  __syncthreads();
  x = 0;
  y = 0;
  for (int i = 0; i < (int)(blockDim.x >> 5); ++i) { x += sh[0][i]; y += sh[1][i]; }
}

// ------------------------------------------------------------ mu kernel --
// mode 0: UpdateV + mu search of one SC iteration.  mode 1: mu search of the
// current V (GetDensities for the initial densities, mpDPFT.cpp:195, and the
// standalone mu-search entry point).  Not launched in mode 2 (admix only).
template <typename R, int FK>
__device__ __forceinline__ void sc_mu_body(const StepArgs<R>& a, const int bid, const int nblk) {
  const KParams& kp = a.kp;
  ScState* st = a.st;
  const long n = kp.geom.n;
  const int S = kp.S;
  const long tid = (long)bid * blockDim.x + threadIdx.x;
  const long nthreads = (long)nblk * blockDim.x;
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const long gw = (long)bid * kStepWarps + wib;
  const long nwarps = (long)nblk * kStepWarps;
  __shared__ double red[kNPart];
  __shared__ MuState s_ms[kMaxS];  // every block runs the same search on its own copy
  __shared__ double s_dmm;
  __shared__ double s_kx[kMaxS][2 * kMuCand];  // 2D form: shared exponentials of the candidates
  // active-point lists as this block sees them (identical in every block)
  // list length of each warp of this block (-1: the warp evaluates all the
  // points it owns)
  __shared__ int s_wlen[kMaxS][kStepWarps];
  __shared__ int s_need[kMaxS], s_lok[kMaxS];
  __shared__ double s_cap[kMaxS], s_lcap[kMaxS];

  if (a.mode == 0) {
    const int exited = ldcg(&st->exit_loop);
    if (bid == 0 && threadIdx.x == 0) st->iter_active = exited ? 0 : 1;
    if (exited) return;
  }
  // block 0 runs the scalar logic on a shared-memory copy of the state and
  // writes it back before every grid barrier after which others read it
  __shared__ ScState s_st;
  ScState* const ls = &s_st;
  if (bid == 0) {
    state_load(ls, st);
    __syncthreads();
  }
  const int cur = ldcg(&st->slot);
  double* mypart = a.part + (long)bid * kNPart;
  MPDPFT_TSTAMP_B(0);

  // ---- UpdateV (mpDPFT.cpp:4815-4838) -----------------------------------
  if (a.mode == 0 && a.assemble_v) {
    const double incv = ldcg(&st->inc_v);
    const double fac = incv < 1.0 ? incv : 1.0;
    double acc[kMaxS];
    for (int s = 0; s < kMaxS; ++s) acc[s] = 0.0;
    const R* nin = a.nin + (long)cur * S * n;
    for (long p = tid; p < n; p += nthreads) {
      for (int s = 0; s < S; ++s) {
        R vi = R(0);
        if (kp.contact_self) vi += R(2.0 * kp.beta) * nin[(long)s * n + p];  // type 10 (:2261)
        if (kp.contact_mutual) {                                              // type 1 (:2247)
          R t = R(0);
          for (int q = 0; q < S; ++q)
            if (q != s) t += nin[(long)q * n + p];
          vi += R(kp.beta) * t;
        }
        if (kp.dirac) {  // type 11 (:2768): -gammaH 2 (D n+/pi)^{1/D}/(D-1)
          R ns = nin[(long)s * n + p];
          ns = ns > R(0) ? ns : R(0);
          if (kp.geom.dim == 3) vi += R(-kp.gamma_h) * cbrt(R(3.0 / kPi) * ns);
          else vi += R(-2.0 * kp.gamma_h) * sqrt(R(2.0 / kPi) * ns);
        }
        if (a.vh) vi += a.vh[(long)s * n + p];
        R vnew = a.vext[(long)s * n + p] + R(fac) * vi;
        R vold = a.V[(long)s * n + p];
        double d = (double)vnew - (double)vold;
        acc[s] += d * d;
        a.V[(long)s * n + p] = vnew;
      }
    }
    block_reduce_store<kMaxS>(acc, mypart + kVresOff);
  }

  // ---- mu search (GetDensities + EnforceConstraints) --------------------
  const int active = kp.rel_acc > 1.0e-12 ? 1 : 0;
  if (threadIdx.x == 0) {  // every block derives the pass-0 candidates itself
    double dmm = ldcg(&st->dmm);
    s_dmm = dmm;
    double pn = 0.0;
    for (int s = 0; s < S; ++s) { double pm = ldcg(&st->mu[s]); pn += pm * pm; }
    for (int s = 0; s < S; ++s) {
      double mu = ldcg(&st->mu[s]);
      double pa = sqrt(pn) < 1.0e-12 ? 1.0e-12 : fabs(mu);
      mu_begin(s_ms[s], mu, pa, dmm, active);
      for (int c = s_ms[s].ncand; c < kMuCand; ++c) s_ms[s].cand[c] = s_ms[s].cand[0];
    }
  }
  if (threadIdx.x < kMaxS) {
    s_need[threadIdx.x] = 0;
    s_lok[threadIdx.x] = 0;
  }
  if (lane == 0)
    for (int s = 0; s < kMaxS; ++s) s_wlen[s][wib] = -1;
  // the points a warp owns: the 32-point segments gw, gw + nwarps, ... of
  // the grid (spread over the whole grid, so that the warps' shares of the
  // active points are alike)
  const long nseg = (n + 31) / 32;
  const long own = gw < nseg ? 32 * ((nseg - gw + nwarps - 1) / nwarps) : 0;
  const long wcap = 32 * ((nseg + nwarps - 1) / nwarps);  // list capacity of a warp
  __syncthreads();
  if (bid == 0 && threadIdx.x == 0) {
    for (int s = 0; s < S; ++s) { ls->ms[s] = s_ms[s]; ls->prev_mu[s] = s_ms[s].start; }
    ls->mu_passes = 0;
    ls->iter_bits = 0;
  }
  // V written above is read at other points below
  if (a.mode == 0 && a.assemble_v && !grid_barrier(st, nblk, kp.spin_limit)) return;

  const R* V = a.V;
  MPDPFT_TSTAMP_B(1);
  for (int pass = 0; pass < kp.mu_max_passes; ++pass) {
    if (pass > 0 && threadIdx.x < S) {
      const int s = threadIdx.x;
      for (int c = s_ms[s].ncand; c < kMuCand; ++c) s_ms[s].cand[c] = s_ms[s].cand[0];
    }
    if constexpr (FK == 3) {
      if (threadIdx.x < S) {
        const int s = threadIdx.x;
        const double invT = 1.0 / kp.dens[s].T;
        for (int c = 0; c < kMuCand; ++c) {
          const double dlt = (s_ms[s].cand[c] - s_ms[s].cand[0]) * invT;
          const bool ok = fabs(dlt) < 50.0;
          s_kx[s][c] = ok ? exp(-dlt) : 0.0;
          s_kx[s][kMuCand + c] = ok ? exp(dlt) : 0.0;
        }
      }
    }
    __syncthreads();
    if (threadIdx.x < S) {
      const int s = threadIdx.x;
      double cmax = s_ms[s].cand[0];
      for (int c = 1; c < s_ms[s].ncand; ++c) cmax = fmax(cmax, s_ms[s].cand[c]);
      s_cap[s] = cmax;
      s_need[s] = !s_ms[s].done && kp.dens[s].cut && !(s_lok[s] && cmax <= s_lcap[s]);
    }
    __syncthreads();
    int any = 0, need = 0;
    for (int s = 0; s < S; ++s) { any |= !s_ms[s].done; need |= s_need[s]; }
    if (!any) break;
    if (need) {
      // (re)build the active-point lists: every warp lists the points it owns
      // below the largest candidate, in its own region of plist (no count
      // pass, no offsets, no grid barrier); a warp that finds most of its
      // points active keeps no list and evaluates all of them
      const unsigned lt = (1u << lane) - 1u;
      for (int s = 0; s < S; ++s) {
        if (!s_need[s]) continue;
        const R* Vs = V + (long)s * n;
        int* pl = a.plist + (long)s * a.plist_stride + gw * wcap;
        const double cap = s_cap[s];
        int cnt = 0;
        for (long seg = gw; seg < nseg; seg += 4 * nwarps) {
          R vv[4];
#pragma unroll
          for (int u = 0; u < 4; ++u) {
            const long p = (seg + u * nwarps) * 32 + lane;
            vv[u] = p < n ? __ldcg(Vs + p) : R(0);
          }
#pragma unroll
          for (int u = 0; u < 4; ++u) {
            const long p = (seg + u * nwarps) * 32 + lane;
            const bool f = p < n && cap - (double)vv[u] > 0.0;
            const unsigned m = __ballot_sync(0xffffffffu, f);
            if (f) pl[cnt + __popc(m & lt)] = (int)p;
            cnt += __popc(m);
          }
        }
        __syncwarp();  // the warp's list entries are visible to all its lanes
        if (lane == 0) s_wlen[s][wib] = 2L * cnt > own ? -1 : cnt;
      }
      __syncthreads();
      if (threadIdx.x < S && s_need[threadIdx.x]) {
        const int s = threadIdx.x;
        s_lok[s] = 1;
        s_lcap[s] = s_cap[s];
        s_need[s] = 0;
      }
      __syncthreads();
    }
    for (int s = 0; s < S; ++s) {
      if (s_ms[s].done) continue;
      // N(mu) and dN/dmu in double from the stored fields (FP32 in mixed
      // mode): the particle-number integral and the mu search are FP64 in
      // both modes
      double acc[kMuAcc];
#pragma unroll
      for (int c = 0; c < kMuAcc; ++c) acc[c] = 0.0;
      const DensParams d = kp.dens[s];
      const EvalK k = eval_constants(d);
      const int nc = s_ms[s].ncand;
      const double* cmu = s_ms[s].cand;  // shared memory (broadcast reads)
      const R* Vs = V + (long)s * n;
      const R* Ls = a.lap ? a.lap + (long)s * n : nullptr;
      const R* Gs = a.g2 ? a.g2 + (long)s * n : nullptr;
      const int* pl = a.plist + (long)s * a.plist_stride + gw * wcap;
      const int wl = s_wlen[s][wib];
      const bool listed = d.cut && wl >= 0;  // else every owned point
      const long len = listed ? (long)wl : own;
      // a warp takes 32 NPT consecutive entries of its own list (or of its
      // owned points) per trip, entry lane + 32 i on lane `lane` (coalesced
      // loads), in a three-stage pipeline: the indices of trip t + 2 and the
      // field values of trip t + 1 are loaded while trip t is evaluated
      // (index -1: past the end).  NPT = 4 points per lane for FP32 fields,
      // 2 for FP64 (the registers of two stages of values).
      constexpr int NPT = sizeof(R) == sizeof(float) ? 4 : 2;
      const long step = 32 * NPT;
      auto indices = [&](long jb, int (&q)[NPT]) {
#pragma unroll
        for (int i = 0; i < NPT; ++i) {
          const long j = jb + 32 * i + lane;
          if (j >= len) { q[i] = -1; continue; }
          if (listed) { q[i] = __ldcg(pl + j); continue; }
          const long p = (gw + (j >> 5) * nwarps) * 32 + (j & 31);
          q[i] = p < n ? (int)p : -1;
        }
      };
      auto values = [&](const int (&q)[NPT], R (&v)[NPT], R (&l)[NPT], R (&g)[NPT]) {
#pragma unroll
        for (int i = 0; i < NPT; ++i) {
          const bool ok = q[i] >= 0;
          v[i] = ok ? __ldcg(Vs + q[i]) : R(0);
          l[i] = (ok && Ls) ? __ldcg(Ls + q[i]) : R(0);
          g[i] = (ok && Gs) ? __ldcg(Gs + q[i]) : R(0);
        }
      };
      long jb = 0;
      int qa[NPT], qb[NPT];
      R v[NPT], l[NPT], g[NPT];
      indices(jb, qa);
      values(qa, v, l, g);
      indices(jb + step, qb);
      for (; jb < len; jb += step) {
        R v2[NPT], l2[NPT], g2[NPT];
        int qc[NPT];
        values(qb, v2, l2, g2);
        indices(jb + 2 * step, qc);
        bool ok[NPT];
#pragma unroll
        for (int i = 0; i < NPT; ++i) ok[i] = qa[i] >= 0;
        mu_points<FK, NPT>(d, k, cmu, nc, v, l, g, ok, acc, s_kx[s]);
#pragma unroll
        for (int i = 0; i < NPT; ++i) {
          qa[i] = qb[i];
          qb[i] = qc[i];
          v[i] = v2[i];
          l[i] = l2[i];
          g[i] = g2[i];
        }
      }
      // partial sums double-buffered by pass: a block that has decided may
      // write the next pass's row while others still read this one
      block_reduce_store<kMuAcc>(acc, a.part + ((long)(pass & 1) * nblk + bid) * kNPart + s * kMuAcc);
    }
    if (!grid_barrier(st, nblk, kp.spin_limit)) return;
    // every block sums the partials in the same order and runs the same
    // decision on its own copy of the search state (no broadcast, no second
    // barrier); block 0 keeps the state copy that is written back
    {
      const double* pbase = a.part + (long)(pass & 1) * nblk * kNPart;
      for (int v = wib; v < S * kMuAcc; v += kStepWarps) {
        const double t = warp_sum_rows(pbase + v, nblk, kNPart);
        if (lane == 0) red[v] = t;
      }
      __syncthreads();
      for (int v = threadIdx.x; v < S * kMuAcc; v += blockDim.x) red[v] *= kp.geom.dvol;  // N(mu_c), dN/dmu
      __syncthreads();
      if (threadIdx.x == 0) {
        double dmm = s_dmm;
        int bits = 0;
        for (int s = 0; s < S; ++s) {
          if (s_ms[s].done) continue;
          mu_decide(s_ms[s], red + s * kMuAcc, red[s * kMuAcc + kMuCand], kp.abundance[s], kp.rel_acc, dmm, bits,
                    kp.mu_max_passes);
        }
        s_dmm = dmm;
        if (bid == 0) {
          for (int s = 0; s < S; ++s) ls->ms[s] = s_ms[s];
          ls->dmm = dmm;
          ls->iter_bits |= bits;
          ls->mu_passes++;
        }
      }
      __syncthreads();
    }
  }
  if (bid == 0) {  // the pass-0 set-up when no pass ran
    __syncthreads();
    state_store(st, ls);
  }
  MPDPFT_TSTAMP_B(2);
}

template <typename R, int FK>
__global__ void __launch_bounds__(kStepThreads, 1) sc_mu_kernel(StepArgs<R> a) {
  pdl_wait();
  sc_mu_body<R, FK>(a, blockIdx.x, gridDim.x);
  pdl_trigger();
}

// Batched launches: entry b of the block table names the solve (x), the
// block's index within that solve (y) and the solve's block count (z).
template <typename R, int FK>
__global__ void __launch_bounds__(kStepThreads, 1) sc_mu_kernel_b(const StepArgs<R>* __restrict__ args,
                                                                 const int4* __restrict__ tab) {
  const int4 t = tab[blockIdx.x];
  sc_mu_body<R, FK>(args[t.x], t.y, t.z);
}

// ---- phase D: CheckConvergence, Intercept, PulayMixer, InjectSchedule --
// over the nblk rows of density-kernel partial sums; cur/next: ring slots,
// I: Pulay window of this step, mu_rep: the mu reported per species.
template <typename R, int PW>
__device__ __forceinline__ void sc_phase_d(const StepArgs<R>& a, const int nblk, const int cur, const int next,
                                           const int I, const int hist, const int pulay_now, const double* s_mu_rep) {
  const KParams& kp = a.kp;
  ScState* st = a.st;
  const long n = kp.geom.n;
  const int S = kp.S;
  const int wib = threadIdx.x >> 5;
  __shared__ double red[kNPart];
  __shared__ double red_v[kMaxS];
  if (threadIdx.x == 0) st->tphase[3] = globaltimer();
  __shared__ ScState s_st;
  ScState* const ls = &s_st;
  __shared__ double s_G[kMaxP * kMaxP], s_inv[kMaxP * kMaxP], s_M[kMaxP * kMaxP], s_R[kMaxP * kMaxP];
  __shared__ double s_prm[kMaxP], s_pv[4];
  __shared__ int s_colof[kMaxP], s_pi[4];
  __shared__ double s_grow[kMaxP];
  __shared__ int s_pbits;
  state_load(ls, st);
  if (threadIdx.x == 0) s_pbits = 0;
  const int nv = 4 + I;  // per species: N, three dots, Gram row
  const int vres = (a.mode == 0 && (a.assemble_v || a.vres_part)) ? S : 0;
  if (!vres) block_rows_sum2(a.part2, nblk, kNPart, S * nv, nv, kNF, red, nullptr, 0, 0, 0, red_v);
  else if (a.assemble_v)
    block_rows_sum2(a.part2, nblk, kNPart, S * nv, nv, kNF, red, a.part + kVresOff, kp.mu_blocks, kNPart, S,
                    red_v);
  else
    block_rows_sum2(a.part2, nblk, kNPart, S * nv, nv, kNF, red, a.vres_part, a.vres_blocks, kMaxS, S, red_v);
  if (threadIdx.x < I) {  // Gram row summed over species
    double t = 0.0;
    for (int s = 0; s < S; ++s) t += red[s * kNF + 4 + threadIdx.x];
    s_grow[threadIdx.x] = t;
  }
  __syncthreads();
  // AdmixDensities / PulayMixer (mpDPFT.cpp:4921-5167) on warp 0: the Gram
  // matrix (last row/column new, the rest shifted from before), its inverse
  // (FullPivHouseholderQR + validation in the reference, :5089-5107) and the
  // coefficients c = G^{-1} 1 / (1^T G^{-1} 1) ...
  const int ngrp = blockDim.x - 32;  // warps 0 .. n-2 solve; the last warp does the bookkeeping
  if (a.mode != 1 && pulay_now && (int)threadIdx.x < ngrp) {
    const int shift = (hist + 1 > kp.scope) ? 1 : 0;
    for (int e = threadIdx.x; e < I * I; e += ngrp) {
      const int i = e / I, j = e % I;
      double v;
      if (i == I - 1) v = s_grow[j];
      else if (j == I - 1) v = s_grow[i];
      else v = ls->gram[(i + shift) * kMaxP + (j + shift)];
      s_G[e] = v;
    }
    group_bar(ngrp);
    for (int e = threadIdx.x; e < I * I; e += ngrp) ls->gram[(e / I) * kMaxP + (e % I)] = s_G[e];
    const bool inv_ok = group_inverse(I, s_G, s_M, s_R, s_inv, s_colof, s_pv, s_pi, ngrp);
    double test = 0.0;
    if (inv_ok && wib == 0) test = warp_inverse_defect(I, s_G, s_inv);
    if (threadIdx.x == 0) s_pv[3] = test;
    group_bar(ngrp);
    const bool used = inv_ok && s_pv[3] <= 1.0e-8;
    if (used && (int)threadIdx.x < I) {  // row sums of the inverse
      double x = 0.0;
      for (int k2 = 0; k2 < I; ++k2) x += s_inv[threadIdx.x * I + k2];
      s_prm[threadIdx.x] = x;
    }
    group_bar(ngrp);
    if (threadIdx.x == 0) {
      ls->hist = I;
      if (used) {
        double A = 0.0;
        for (int i = 0; i < I; ++i) A += s_prm[i];
        for (int i = 0; i < I; ++i) ls->coeff[i] = s_prm[i] / A;
      } else {
        s_pbits = kBitPulay;
      }
      ls->pulay_used = used ? 1 : 0;
      ls->ncoeff = used ? I : 0;
    }
  }
  // ... while the last warp does CheckConvergence and Intercept
  if ((int)threadIdx.x == ngrp) {
    if (vres) {
      double w = 0.0;
      for (int s = 0; s < S; ++s) w = fmax(w, sqrt(red_v[s] / (double)n));
      ls->v_res = w;
    }
    const int sc = ls->sc_count;
    double tot = 0.0;
    for (int s = 0; s < S; ++s) {
      ls->mu[s] = s_mu_rep[s];
      ls->ab[s] = red[s * kNF] * kp.geom.dvol;
      if (!isfinite(ls->ab[s])) ls->iter_bits |= kBitNonfinite;
      tot += ls->ab[s];
    }
    if (a.mode != 1) {
      // CheckConvergence (mpDPFT.cpp:4759-4782)
      const double mp = 100.0 * 1.0e-16;
      if (sc > 0) {
        double cc = 0.0, maxtest = 0.0;
        for (int s = 0; s < S; ++s) {
          double oi = red[s * kNF + 1], oo = red[s * kNF + 2], ii = red[s * kNF + 3];
          double rd = (oo + ii > 1.0e-12) ? 1.0 - 2.0 * oi / (oo + ii) : 0.0;
          double t = rd * ls->ab[s] / tot;
          if (t > maxtest) { maxtest = t; cc = maxtest; }
        }
        ls->cc = cc;
        double dab = 0.0, dmu = 0.0;
        for (int s = 0; s < S; ++s) {
          dab += (ls->ab[s] - ls->old_ab[s]) * (ls->ab[s] - ls->old_ab[s]);
          dmu += (ls->mu[s] - ls->old_mu[s]) * (ls->mu[s] - ls->old_mu[s]);
        }
        int steady = (cc < mp && sqrt(dab) < mp && sqrt(dmu) < mp) ? 1 : 0;
        double avth = 0.0;
        for (int s = 0; s < S; ++s) avth += ls->theta[s] / (double)S;
        bool vok = !(kp.pot_tol > 0.0) || ls->v_res <= kp.pot_tol;
        if ((tot > mp || (tot <= mp && (double)sc * avth > 1.0)) && kp.sc_criterion >= 0.0 &&
            (cc < kp.sc_criterion || steady) && vok)
          ls->exit_count++;
        else
          ls->exit_count = 0;
        if (ls->exit_count >= 3) ls->exit_loop = 1;
      } else {
        ls->cc = 1.2345678901234567890;
      }
      if (sc == kp.max_sc) ls->exit_loop = 1;  // Intercept (:4866)
    }
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    const int sc = ls->sc_count;
    // TrappedQ (mpDPFT.cpp:4926-4934): a mu search that ended without
    // meeting the tolerance lowers this iteration's mixing weight theta by
    // min(1, |1 - RelDiff|^30), RelDiff = |N* - N| / |N*| over the species
    int trapped = 0;
    for (int s = 0; s < S; ++s) trapped |= ls->ms[s].trapped;
    double tmod = 1.0;
    if (trapped) {
      double na = 0.0, nd = 0.0;
      for (int s = 0; s < S; ++s) {
        na += kp.abundance[s] * kp.abundance[s];
        nd += (kp.abundance[s] - ls->ab[s]) * (kp.abundance[s] - ls->ab[s]);
      }
      const double rd = sqrt(nd) / sqrt(na);
      if (rd > 1.0e-12) tmod = fmin(1.0, pow(fabs(1.0 - rd), 30.0));
      ls->iter_bits |= kBitTrapped;
    }
    if (a.mode == 1) {
      ls->status_bits |= ls->iter_bits;
      ls->mu_passes_total += ls->mu_passes;
    } else {
      const int used = pulay_now ? ls->pulay_used : 0;
      if (!pulay_now) { ls->pulay_used = 0; ls->ncoeff = 0; }
      ls->iter_bits |= s_pbits;
      for (int s = 0; s < S; ++s) ls->theta_mix[s] = ls->theta[s] * tmod;
      // InjectSchedule (mpDPFT.cpp:5229-5315)
      if (kp.schedule == 5) {
        for (int s = 0; s < S; ++s) {
          double th = ls->theta[s] * (ls->cc < ls->old_cc ? 1.1 : 0.5);
          th = fmin(0.8, th);
          th = fmax(10.0 / (double)kp.max_sc, th);
          ls->theta[s] = th;
        }
      } else if (kp.schedule == 9) {
        for (int s = 0; s < S; ++s)
          if (ls->theta[s] < 0.2)
            ls->theta[s] = ls->theta0[s] + (0.2 - ls->theta0[s]) * (double)sc / (double)kp.max_sc;
      }
      if (a.log && sc >= 0 && sc < a.log_cap) {
        mpdpft_iter_log& L = a.log[sc];
        L.sc_count = sc;
        L.mu_trials = ls->mu_passes;
        L.pulay_used = used;
        L.status_bits = ls->iter_bits;
        L.cc = ls->cc;
        L.v_residual = ls->v_res;
        for (int s = 0; s < kMaxS; ++s) {
          L.mu[s] = s < S ? ls->mu[s] : 0.0;
          L.abundance[s] = s < S ? ls->ab[s] : 0.0;
          L.theta[s] = s < S ? ls->theta_mix[s] : 0.0;
        }
        L.ms = 0.0;
      }
      ls->status_bits |= ls->iter_bits;
      ls->mu_passes_total += ls->mu_passes;
      // StoreCurrentIteration of the next iteration; PrepareNextIteration
      for (int s = 0; s < S; ++s) { ls->old_mu[s] = ls->mu[s]; ls->old_ab[s] = ls->ab[s]; }
      ls->old_cc = ls->cc;
      if (sc > 0) ls->inc_v = fmin(1.0, ls->inc_v + kp.inc_v0);  // (:4833)
      ls->mix_src = cur;
      ls->slot = next;
      ls->sc_count = sc + 1;
    }
  }
  __syncthreads();
  state_store(st, ls);
  if (threadIdx.x == 0) {
    st->k2_done = 0u;
    st->tphase[4] = globaltimer();
  }
}

// ------------------------------------------------------- density kernel --
// Final densities n_out = n[V] at the mu the search chose, residual
// r = n_out - n_in into the ring, and per species [0] N, [1] <n_out, n_in>_w,
// [2] <n_out, n_out>_w, [3] <n_in, n_in>_w, [4 + j] <r_new, r_j>_w (Gram
// row), w = multiplicity in the reference storage.  mode 1 writes n_out
// into the current ring slot instead; mode 2 (admix only) takes n_out from V.
// The last block to finish runs phase D: CheckConvergence, Intercept, the
// Pulay solve (AdmixDensities / PulayMixer) and InjectSchedule.
template <typename R, int FK, int PW>
__device__ __forceinline__ void sc_density_body(const StepArgs<R>& a, const int bid, const int nblk) {
  // PW: the largest Pulay window this instantiation handles (<= kMaxP); a
  // small window keeps the per-thread sums in few registers
  const KParams& kp = a.kp;
  ScState* st = a.st;
  const long n = kp.geom.n;
  const int S = kp.S;
  const int wib = threadIdx.x >> 5;
  __shared__ double s_mu[kMaxS];      // mu of the final density
  __shared__ double s_mu_rep[kMaxS];  // mu reported (the start value after a bracket failure)
  __shared__ int s_flag, s_last;
  __shared__ long s_roff[kMaxP];

  if (a.mode == 0 && !ldcg(&st->iter_active)) return;
  const int cur = ldcg(&st->slot);
  const int ring = kp.ring;
  const int next = (cur + 1) % ring;
  const int active = kp.rel_acc > 1.0e-12 ? 1 : 0;
  if (threadIdx.x < S) {
    const int s = threadIdx.x;
    s_mu[s] = (active && a.mode != 2) ? ldcg(&st->ms[s].dens_mu) : ldcg(&st->mu[s]);
    s_mu_rep[s] = (active && a.mode != 2) ? ldcg(&st->ms[s].best_mu) : ldcg(&st->mu[s]);
  }
  if (threadIdx.x == 0) s_flag = (a.mode != 1 && kp.mixer > 0 && ldcg(&st->sc_count) > 0) ? 1 : 0;
  __syncthreads();
  const int pulay_now = s_flag;
  const int hist = ldcg(&st->hist);
  const int I = pulay_now ? (hist + 1 < kp.scope ? hist + 1 : kp.scope) : 0;
  if (threadIdx.x < I) {
    const int j = threadIdx.x;
    s_roff[j] = (long)((cur - (I - 1) + j + ring) % ring) * S * n;
  }
  __syncthreads();
  R* nin = a.nin + (long)cur * S * n;
  R* rcur = a.res + (long)cur * S * n;
  const long gstride = (long)nblk * blockDim.x;
  for (int s = 0; s < S; ++s) {
    double acc[4 + PW];
#pragma unroll
    for (int j = 0; j < 4 + PW; ++j) acc[j] = 0.0;
    const DensParams d = kp.dens[s];
    const EvalK k = eval_constants(d);
    const double mus = s_mu[s];
    const long so = (long)s * n;
    const R* Vs = a.V + so;
    const R* Ls = a.lap ? a.lap + so : nullptr;
    const R* Gs = a.g2 ? a.g2 + so : nullptr;
    // NP consecutive points per thread and trip, one 16-byte vector per
    // field; every load of a trip (the history residuals of the Gram row
    // included) is issued before its arithmetic.  Every lane of a warp runs
    // every trip (the vote below needs them all).
    constexpr int NP = kVecPts<R>;
    constexpr int NH = PW - 1;  // history residuals of the Gram row
    const int vec4 = kp.vec4;
    const bool in_loads = a.mode == 0 || a.mode == 2;
    for (long base = (long)bid * blockDim.x * NP; base < n; base += gstride * NP) {
      const long p0 = base + (long)NP * threadIdx.x;
      R v[NP], ni[NP], rj[NH][NP], l[NP], g[NP];
      vload(Vs, p0, n, vec4, v);
#pragma unroll
      for (int i = 0; i < NP; ++i) ni[i] = l[i] = g[i] = R(0);
      if (a.mode != 2) {
        if (Ls) vload(Ls, p0, n, vec4, l);
        if (Gs) vload(Gs, p0, n, vec4, g);
      }
      if (in_loads) {
        vload(nin + so, p0, n, vec4, ni);
#pragma unroll
        for (int j = 0; j < NH; ++j)
          if (j < I - 1) vload(a.res + s_roff[j] + so, p0, n, vec4, rj[j]);
      }
      double nod[NP];
#pragma unroll
      for (int i = 0; i < NP; ++i) nod[i] = 0.0;
      if (a.mode == 2) {  // admix only: V holds the output densities
#pragma unroll
        for (int i = 0; i < NP; ++i) nod[i] = (double)v[i];
      } else {
        bool mine[NP], any = false;
#pragma unroll
        for (int i = 0; i < NP; ++i) {
          mine[i] = p0 + i < n && (!d.cut || mus - (double)v[i] > 0.0);
          any |= mine[i];
        }
        if (__any_sync(0xffffffffu, any) && any) {
          if constexpr (FK != 0) {  // branch-free forms: the points are independent chains
#pragma unroll
            for (int i = 0; i < NP; ++i) {
              const double x = point_density<FK>(d, k, mus - (double)v[i], (double)l[i], (double)g[i]);
              nod[i] = mine[i] ? x : 0.0;
            }
          } else {
#pragma unroll
            for (int i = 0; i < NP; ++i)
              if (mine[i]) nod[i] = point_density<FK>(d, k, mus - (double)v[i], (double)l[i], (double)g[i]);
          }
        }
      }
      if (p0 >= n) continue;
      R no[NP];
#pragma unroll
      for (int i = 0; i < NP; ++i) {
        no[i] = R(nod[i]);
        acc[0] += nod[i];  // 0 past the end
      }
      if (a.mode == 1) {
        vstore(nin + so, p0, n, vec4, no);
        vstore(a.cur_copy + so, p0, n, vec4, no);
        continue;
      }
      R r[NP];
      double w[NP], wr[NP];
      ref_weights<NP>(p0, kp.geom.s, kp.geom.dim, w);
#pragma unroll
      for (int i = 0; i < NP; ++i) {
        r[i] = no[i] - ni[i];
        if (p0 + i >= n) w[i] = 0.0;
        const double dno = (double)no[i], dni = (double)ni[i];
        wr[i] = w[i] * (double)r[i];
        acc[1] += w[i] * dno * dni;
        acc[2] += w[i] * dno * dno;
        acc[3] += w[i] * dni * dni;
      }
#pragma unroll
      for (int j = 0; j < PW; ++j) {
        if (j < I - 1) {
#pragma unroll
          for (int i = 0; i < NP; ++i) acc[4 + j] += wr[i] * (double)rj[j < NH ? j : 0][i];
        } else if (j == I - 1) {
#pragma unroll
          for (int i = 0; i < NP; ++i) acc[4 + j] += wr[i] * (double)r[i];
        }
      }
      vstore(rcur + so, p0, n, vec4, r);
    }
    block_reduce_store<4 + PW>(acc, a.part2 + (long)bid * kNPart + s * kNF);
  }
  if (a.split_d) return;  // phase D runs as its own launch
  // the last block to finish takes phase D
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) s_last = atomicAdd(&st->k2_done, 1u) == nblk - 1 ? 1 : 0;
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  sc_phase_d<R, PW>(a, nblk, cur, next, I, hist, pulay_now, s_mu_rep);
}

template <typename R, int FK, int PW>
__global__ void __launch_bounds__(kDensityThreads, 2) sc_density_kernel(StepArgs<R> a) {
  pdl_wait();
  sc_density_body<R, FK, PW>(a, blockIdx.x, gridDim.x);
  pdl_trigger();
}

template <typename R, int FK, int PW>
__global__ void __launch_bounds__(kDensityThreads, 2) sc_density_kernel_b(const StepArgs<R>* __restrict__ args,
                                                                         const int4* __restrict__ tab) {
  const int4 t = tab[blockIdx.x];
  sc_density_body<R, FK, PW>(args[t.x], t.y, t.z);
}

// Phase D as its own launch: one block, no register cap from the streaming
// kernel's occupancy.
template <typename R, int PW>
__global__ void __launch_bounds__(kDensityThreads, 1) sc_phase_d_kernel(StepArgs<R> a, int nblk) {
  pdl_wait();
  const KParams& kp = a.kp;
  ScState* st = a.st;
  const int S = kp.S;
  __shared__ double s_mu_rep[kMaxS];
  __shared__ int s_flag;
  if (a.mode == 0 && !ldcg(&st->iter_active)) return;
  const int cur = ldcg(&st->slot);
  const int next = (cur + 1) % kp.ring;
  const int active = kp.rel_acc > 1.0e-12 ? 1 : 0;
  if (threadIdx.x < S) {
    const int s = threadIdx.x;
    s_mu_rep[s] = (active && a.mode != 2) ? ldcg(&st->ms[s].best_mu) : ldcg(&st->mu[s]);
  }
  if (threadIdx.x == 0) s_flag = (a.mode != 1 && kp.mixer > 0 && ldcg(&st->sc_count) > 0) ? 1 : 0;
  __syncthreads();
  const int pulay_now = s_flag;
  const int hist = ldcg(&st->hist);
  const int I = pulay_now ? (hist + 1 < kp.scope ? hist + 1 : kp.scope) : 0;
  sc_phase_d<R, PW>(a, nblk, cur, next, I, hist, pulay_now, s_mu_rep);
}

// ---------------------------------------------------------- mix kernel --
// The mixed density n = sum_j c_j (n_in,j + theta r_j) (Pulay) or
// n_in + theta r (linear) into the next ring slot (AdmixDensities,
// mpDPFT.cpp:4946-4955 / :4987).
template <typename R>
__device__ __forceinline__ void sc_mix_body(const StepArgs<R>& a, const int bid, const int nblk) {
  const KParams& kp = a.kp;
  ScState* st = a.st;
  const long n = kp.geom.n;
  const int S = kp.S;
  __shared__ long s_off[kMaxP];
  __shared__ double s_c[kMaxP];
  __shared__ int s_nc;
  if (a.mode == 0 && !ldcg(&st->iter_active)) return;
  if (bid == 0 && threadIdx.x == 0) st->tphase[5] = globaltimer();
  const int ring = kp.ring;
  const int cur = ldcg(&st->mix_src), next = ldcg(&st->slot);
  if (threadIdx.x == 0) {
    const int used = ldcg(&st->pulay_used);
    const int nc = used ? ldcg(&st->ncoeff) : 1;
    s_nc = nc;
    for (int j = 0; j < nc; ++j) {
      const int slot = (cur - (nc - 1) + j + ring) % ring;
      s_off[j] = (long)slot * S * n;
      s_c[j] = used ? ldcg(&st->coeff[j]) : 1.0;
    }
  }
  __syncthreads();
  const int nc = s_nc;
  const long gstride = (long)nblk * blockDim.x;
  for (int s = 0; s < S; ++s) {
    const double th = ldcg(&st->theta_mix[s]);
    R* out = a.nin + (long)next * S * n + (long)s * n;
    for (long q = (long)bid * blockDim.x + threadIdx.x; 4 * q < n; q += gstride) {
      const long p0 = 4 * q;
      double v[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll 4
      for (int j = 0; j < nc; ++j) {
        const long o = s_off[j] + (long)s * n;
        R ni[4], ri[4];
        load4(a.nin + o, p0, n, kp.vec4, ni);
        load4(a.res + o, p0, n, kp.vec4, ri);
        const double c = s_c[j];
#pragma unroll
        for (int i = 0; i < 4; ++i) v[i] += c * ((double)ni[i] + th * (double)ri[i]);
      }
      R o4[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) o4[i] = R(v[i]);
      store4(out, p0, n, kp.vec4, o4);
      store4(a.cur_copy + (long)s * n, p0, n, kp.vec4, o4);
    }
  }
  if (bid == 0 && threadIdx.x == 0) st->tphase[6] = globaltimer();
}

template <typename R>
__global__ void __launch_bounds__(kDensThreads, 4) sc_mix_kernel(StepArgs<R> a) {
  pdl_wait();
  sc_mix_body<R>(a, blockIdx.x, gridDim.x);
  pdl_trigger();
}

template <typename R>
__global__ void __launch_bounds__(kDensThreads, 4) sc_mix_kernel_b(const StepArgs<R>* __restrict__ args,
                                                                  const int4* __restrict__ tab) {
  const int4 t = tab[blockIdx.x];
  sc_mix_body<R>(args[t.x], t.y, t.z);
}

}  // namespace mpdpft
