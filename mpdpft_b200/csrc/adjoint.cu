// adjoint.cu -- the adjoint of the converged SC fixed point.
//
// At convergence the density n* of one species satisfies n* = Phi(n*),
// Phi(n) = N_c(V_ext + V_int[n]), where N_c maps a potential to the density
// at the mu that holds the particle number (GetDensities + EnforceConstraints,
// mpDPFT.cpp:3306-3316, 4569-4743) and V_int is the interaction potential
// (UpdateV, :4815-4838).  For a loss L(n*) with gradient g = dL/dn*,
//   dL/dV_ext = J_N^T lambda,   lambda = g + J_W^T J_N^T lambda,
// J_N the Jacobian of N_c at V*, J_W that of V_int at n*.  The linear system
// is solved by the context's own device Pulay mixer (the admix step of the SC
// kernels), iterating lambda -> g + J_W^T J_N^T lambda.
//
// J_N^T, from the pieces of the forward map (all linear operators act on the
// periodic grid with the plain dot product):
//   density    dn = A (dmu - dV) + B dlap + C dg2 pointwise (A = dn/du,
//              B = dn/dlap, C = dn/d|grad V|^2; zero where n is clamped),
//   mu         sum dn = 0  =>  J_N = (I - A 1^T / 1^T A) J0,
//   DelField   f = w (V - V(p*)) (taper weight w, shell maximum at p*),
//              lap = L f, g2 = Pos Sm(sum_j (D_j f)^2), with L, Sm symmetric
//              and D_j antisymmetric spectral operators;
// so  J_N^T y = -A z + T^T [ L(B z) - sum_j D_j(2 d_j Sm(C' z)) ],
//     z = y - (A.y / 1.A),  T^T h = w h - e_{p*} (w.h),  d_j = D_j f,
//     C' = C where the smoothed g2 is positive (the clamp), else 0.
// J_W^T: Hartree = gammaH (K_sym + q 1^T) with K_sym the translation-invariant
// part and q the field of the regularised kernel's total-charge terms
// (q = K e_0 - K_sym e_0 from a unit impulse), Dirac and contact pointwise.
// The iteration is preconditioned by the pointwise part of the map: near the
// density edge the Dirac term's d V / d n ~ n^{-2/3} makes the local gain
// -dx A exceed 1; at points where it exceeds 2, lambda is mixed with
// lambda + (T(lambda) - lambda)/(1 + dx A) (the same fixed point).
// The fixed-point adjoint needs only the converged state, not the forward
// iteration history.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "engine.h"
#include "sc_kernel.cuh"

namespace mpdpft {

#define CU(call)                                                                             \
  do {                                                                                       \
    cudaError_t e_ = (call);                                                                 \
    if (e_ != cudaSuccess)                                                                   \
      return set_error(MPDPFT_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

// device scalars of the adjoint
enum { SC_SUM_A = 0, SC_A_DOT_Y, SC_W_DOT_H, SC_Q_DOT_ETA, SC_R2, SC_O2, SC_VMAX, SC_PSTAR, SC_COUNT = 16 };

struct Adjoint {
  size_t rsize = 8;
  long n = 0;
  void* f[20] = {};  // fields, see the enum below
  double* scal = nullptr;        // SC_COUNT doubles
  double* part = nullptr;        // per-block partials
  int blocks = 0;
  unsigned long long* vmax = nullptr;
  long long* pstar = nullptr;
};
enum { F_VSAVE, F_NSTAR, F_G, F_A, F_B, F_C, F_W, F_D0, F_D1, F_D2, F_DX, F_Q, F_M, F_ETA, F_OUT, F_T1, F_T2,
       F_T3, F_H, F_NF };

// ------------------------------------------------------------ kernels ----
// Per-block partial sums of x.y (y null: sum x).
template <typename R>
__global__ void k_adj_dot(const R* x, const R* y, long n, double* part) {
  double acc[1] = {0.0};
  for (long p = (long)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (long)gridDim.x * blockDim.x)
    acc[0] += (double)x[p] * (y ? (double)y[p] : 1.0);
  block_reduce_store<1>(acc, part + blockIdx.x);
}

// out = sum of nb partials, one warp, fixed order.
__global__ void k_adj_sum(const double* part, int nb, double* out) {
  double t = 0.0;
  for (int b = threadIdx.x; b < nb; b += 32) t += part[b];
  t = warp_sum(t);
  if (threadIdx.x == 0) *out = t;
}

// Taper weight w(r) of DelField (mpDPFT.cpp:7251-7264): 1 inside r0,
// exp(a (r - r0)^2) beyond; 1 everywhere without the taper.
template <typename R>
__global__ void k_adj_weights(Geom g, double r0, double ta, int taper, R* w) {
  for (long p = (long)blockIdx.x * blockDim.x + threadIdx.x; p < g.n; p += (long)gridDim.x * blockDim.x) {
    double wt = 1.0;
    if (taper) {
      double x, y, z;
      point_coords(p, g, x, y, z);
      const double r = sqrt(x * x + y * y + z * z);
      if (r > r0) wt = exp(ta * (r - r0) * (r - r0));
    }
    w[p] = R(wt);
  }
}

// Pointwise derivatives of n at the converged V: A = dn/du, B = dn/dlap,
// C = dn/d|grad V|^2 with |grad V|^2 = max(g2s, 0) and C = 0 where the
// smoothed g2s is not positive (the clamp); dx = d V_int / dn of the
// pointwise terms (Dirac, contact within the species).
template <typename R, int FK>
__global__ void k_adj_prepare(Geom g, DensParams d, double mu, const R* V, const R* lap, const R* g2s, const R* nstar,
                              double gamma_h, int dirac, double beta2, R* A, R* B, R* C, R* dx) {
  const EvalK k = eval_constants(d);
  for (long p = (long)blockIdx.x * blockDim.x + threadIdx.x; p < g.n; p += (long)gridDim.x * blockDim.x) {
    const double u = mu - (double)V[p];
    const double l = lap ? (double)lap[p] : 0.0;
    const double graw = g2s ? (double)g2s[p] : 0.0;
    const double q = graw > 0.0 ? graw : 0.0;
    double a = 0.0, b = 0.0, c = 0.0;
    if constexpr (FK == 1) {
      const double Al = k.cg * l, Bg = k.cg2 * q;
      a = grad3_slope(k, u, Al, Bg);
      const double r = rsqrt_nr(fmin(fmax(u, 1.0e-30), 1.0e30));
      const bool hi = u >= k.floor_u;
      const double m1 = hi ? r : u * k.c1;
      const double m3 = hi ? r * r * r : u * k.c3;
      const double v = k.ctf * u * u * r - (Al * m1 + Bg * m3);
      if (u > 0.0 && v > 0.0) {
        b = -k.cg * m1;
        c = graw > 0.0 ? -k.cg2 * m3 : 0.0;
      }
    } else if constexpr (FK == 2) {
      a = tf3_slope(k, u);
    } else {  // 2D finite-T form
      double nn;
      g2d_n_slope(k, u, l, nn, a);
      const double e = exp(-fabs(u * k.invT));
      const double ope = 1.0 + e;
      b = -k.c2d * k.lt * e / (ope * ope);
    }
    A[p] = R(a);
    B[p] = R(b);
    C[p] = R(c);
    double dv = beta2;
    if (dirac) {
      const double ns = (double)nstar[p];
      if (ns > 0.0) {
        if (g.dim == 3) dv += -gamma_h * cbrt(3.0 / kPi) / 3.0 * pow(ns, -2.0 / 3.0);
        else dv += -gamma_h * sqrt(2.0 / kPi) / sqrt(ns);
      }
    }
    dx[p] = R(dv);
  }
}

// t = d0^2 + d1^2 (+ d2^2)
template <typename R>
__global__ void k_adj_sumsq(long n, int dim, const R* d0, const R* d1, const R* d2, R* t) {
  for (long p = (long)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (long)gridDim.x * blockDim.x) {
    double v = (double)d0[p] * (double)d0[p] + (double)d1[p] * (double)d1[p];
    if (dim == 3) v += (double)d2[p] * (double)d2[p];
    t[p] = R(v);
  }
}

// f = w (V - shift) (the tapered field whose derivatives DelField takes).
template <typename R>
__global__ void k_adj_taper(long n, const R* V, const R* w, const double* scal, R* f) {
  const unsigned long long b = *(const unsigned long long*)(scal + SC_VMAX);
  const double shift = b ? from_ordered_bits(b) : 0.0;
  for (long p = (long)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (long)gridDim.x * blockDim.x)
    f[p] = R(((double)V[p] - shift) * (double)w[p]);
}

// Shell maximum of V (ordered bits) and the first point that attains it.
template <typename R>
__global__ void k_adj_shell_max(Geom g, const R* V, double r0, double width, unsigned long long* vmax) {
  double vm = -1.0e300;
  for (long p = (long)blockIdx.x * blockDim.x + threadIdx.x; p < g.n; p += (long)gridDim.x * blockDim.x) {
    double x, y, z;
    point_coords(p, g, x, y, z);
    if (in_shell(x * x + y * y + z * z, r0, width)) vm = fmax(vm, (double)V[p]);
  }
  for (int o = 16; o > 0; o >>= 1) vm = fmax(vm, __shfl_xor_sync(0xffffffffu, vm, o));
  if ((threadIdx.x & 31) == 0 && vm > -1.0e300) atomicMax(vmax, ordered_bits(vm));
}

template <typename R>
__global__ void k_adj_argmax(Geom g, const R* V, double r0, double width, const unsigned long long* vmax,
                             long long* pstar) {
  const unsigned long long b = *vmax;
  if (!b) return;
  for (long p = (long)blockIdx.x * blockDim.x + threadIdx.x; p < g.n; p += (long)gridDim.x * blockDim.x) {
    double x, y, z;
    point_coords(p, g, x, y, z);
    if (in_shell(x * x + y * y + z * z, r0, width) && ordered_bits((double)V[p]) == b)
      atomicMin((unsigned long long*)pstar, (unsigned long long)p);
  }
}

// z = y - (A.y)/(1.A); t1 = B z; t2 = C z.
template <typename R>
__global__ void k_adj_project(long n, const R* y, const R* A, const R* B, const R* C, const double* scal, R* z,
                              R* t1, R* t2) {
  const double sa = scal[SC_SUM_A];
  const double shift = sa != 0.0 ? scal[SC_A_DOT_Y] / sa : 0.0;
  for (long p = (long)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (long)gridDim.x * blockDim.x) {
    const double zz = (double)y[p] - shift;
    z[p] = R(zz);
    t1[p] = R((double)B[p] * zz);
    t2[p] = R((double)C[p] * zz);
  }
}

// t = 2 d s
template <typename R>
__global__ void k_adj_times2(long n, const R* d, const R* s, R* t) {
  for (long p = (long)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (long)gridDim.x * blockDim.x)
    t[p] = R(2.0 * (double)d[p] * (double)s[p]);
}

// h -= t
template <typename R>
__global__ void k_adj_sub(long n, const R* t, R* h) {
  for (long p = (long)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (long)gridDim.x * blockDim.x)
    h[p] = R((double)h[p] - (double)t[p]);
}

// out = -A z + w h - e_{p*} (w.h)
template <typename R>
__global__ void k_adj_finish_n(long n, const R* A, const R* z, const R* w, const R* h, const double* scal,
                               const long long* pstar, R* out) {
  const long long ps = *pstar;
  const double wh = scal[SC_W_DOT_H];
  for (long p = (long)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (long)gridDim.x * blockDim.x) {
    double v = -(double)A[p] * (double)z[p] + (h ? (double)w[p] * (double)h[p] : 0.0);
    if (h && (long long)p == ps) v -= wh;
    out[p] = R(v);
  }
}

// out = g + kc + (q.eta) + dx eta
template <typename R>
__global__ void k_adj_finish_w(long n, const R* g, const R* kc, const R* dx, const R* eta, const double* scal,
                               int coulomb, R* out) {
  const double qe = coulomb ? scal[SC_Q_DOT_ETA] : 0.0;
  for (long p = (long)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (long)gridDim.x * blockDim.x) {
    double v = (double)g[p] + (double)dx[p] * (double)eta[p];
    if (coulomb) v += (double)kc[p] + qe;
    out[p] = R(v);
  }
}

// Diagonal preconditioner of the adjoint iteration: the pointwise part of
// J_W^T J_N^T is D = -dx A (the local feedback of the Dirac and contact
// terms through the density).  Where that gain exceeds 2 the point is
// unstable under the plain iteration and M = 1 - D; elsewhere M = 1.
template <typename R>
__global__ void k_adj_precond(long n, const R* A, const R* dx, R* M) {
  for (long p = (long)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (long)gridDim.x * blockDim.x) {
    const double d = -(double)dx[p] * (double)A[p];
    M[p] = R(d > 2.0 ? 1.0 - d : 1.0);
  }
}

// Mixer input: lambda + (T(lambda) - lambda) / M (same fixed point as T).
template <typename R>
__global__ void k_adj_step(long n, const R* lam, const R* out, const R* M, R* next) {
  for (long p = (long)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (long)gridDim.x * blockDim.x) {
    const double l = (double)lam[p];
    next[p] = R(l + ((double)out[p] - l) / (double)M[p]);
  }
}

// r2 += (a - b)^2, o2 += a^2 (partials [block][2])
template <typename R>
__global__ void k_adj_resid(long n, const R* a, const R* b, double* part) {
  double acc[2] = {0.0, 0.0};
  for (long p = (long)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (long)gridDim.x * blockDim.x) {
    const double x = (double)a[p], y = (double)b[p];
    acc[0] += (x - y) * (x - y);
    acc[1] += x * x;
  }
  block_reduce_store<2>(acc, part + 2L * blockIdx.x);
}

__global__ void k_adj_sum2(const double* part, int nb, double* out) {
  const int v = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (v >= 2) return;
  double t = 0.0;
  for (int b = lane; b < nb; b += 32) t += part[2L * b + v];
  t = warp_sum(t);
  if (lane == 0) out[v] = t;
}

template <typename R>
__global__ void k_adj_unit(long n, long p0, R* f) {
  for (long p = (long)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (long)gridDim.x * blockDim.x)
    f[p] = R(p == p0 ? 1.0 : 0.0);
}

// q = a - b
template <typename R>
__global__ void k_adj_diff(long n, const R* a, const R* b, R* q) {
  for (long p = (long)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (long)gridDim.x * blockDim.x)
    q[p] = R((double)a[p] - (double)b[p]);
}

// dL/dR of Gaussian nuclei: V_ext = sum_a phi_a(|r - R_a|), phi(rho) =
// -Z erf(rho / (sqrt(2) sigma)) / rho; d V_ext / d R_a = -phi'(rho) (r - R_a) / rho.
__global__ void k_adj_nuclei(Geom g, const double* gv, int nn, const double* Z, const double* pos, double sigma,
                             double* part) {
  const double s2 = sqrt(2.0) * sigma;
  for (int a = 0; a < nn; ++a) {
    double acc[3] = {0.0, 0.0, 0.0};
    for (long p = (long)blockIdx.x * blockDim.x + threadIdx.x; p < g.n; p += (long)gridDim.x * blockDim.x) {
      double x, y, z;
      point_coords(p, g, x, y, z);
      const double dx = x - pos[3 * a], dy = y - pos[3 * a + 1], dz = z - pos[3 * a + 2];
      const double rho = sqrt(dx * dx + dy * dy + dz * dz);
      double fr;  // phi'(rho) / rho
      if (rho < 1.0e-4 * sigma) {
        fr = Z[a] * sqrt(2.0 / kPi) / (3.0 * sigma * sigma * sigma);
      } else {
        const double dphi = -Z[a] * (2.0 / sqrt(kPi) / s2 * exp(-rho * rho / (s2 * s2)) / rho -
                                     erf(rho / s2) / (rho * rho));
        fr = dphi / rho;
      }
      const double gp = gv[p];
      acc[0] -= gp * fr * dx;
      acc[1] -= gp * fr * dy;
      acc[2] -= gp * fr * dz;
    }
    block_reduce_store<3>(acc, part + ((long)blockIdx.x * nn + a) * 3);
  }
}

__global__ void k_adj_sum_rows(const double* part, int nb, int nv, double* out) {
  const int lane = threadIdx.x & 31;
  for (int v = threadIdx.x >> 5; v < nv; v += blockDim.x >> 5) {
    double t = 0.0;
    for (int b = lane; b < nb; b += 32) t += part[(long)b * nv + v];
    t = warp_sum(t);
    if (lane == 0) out[v] = t;
  }
}

// ------------------------------------------------------------- host -----
void Ctx::adjoint_release() {
  if (!adj) return;
  for (void*& p : adj->f) if (p) { cudaFree(p); p = nullptr; }
  cudaFree(adj->scal);
  cudaFree(adj->part);
  cudaFree(adj->vmax);
  cudaFree(adj->pstar);
  delete adj;
  adj = nullptr;
}

template <typename R>
static int adj_dot(Ctx& c, const void* x, const void* y, int slot) {
  Adjoint& a = *c.adj;
  k_adj_dot<R><<<a.blocks, kThreads, 0, c.stream>>>((const R*)x, (const R*)y, a.n, a.part);
  k_adj_sum<<<1, 32, 0, c.stream>>>(a.part, a.blocks, a.scal + slot);
  CU(cudaGetLastError());
  return MPDPFT_OK;
}

// out = J_N^T y
template <typename R>
static int adj_jn_t(Ctx& c, const R* y, R* out) {
  Adjoint& a = *c.adj;
  const long n = a.n;
  const int nb = a.blocks;
  int st;
  R** F = (R**)a.f;
  if ((st = adj_dot<R>(c, F[F_A], y, SC_A_DOT_Y))) return st;
  k_adj_project<R><<<nb, kThreads, 0, c.stream>>>(n, y, F[F_A], F[F_B], F[F_C], a.scal, F[F_T3], F[F_T1], F[F_T2]);
  CU(cudaGetLastError());
  if (!c.gradient) {
    k_adj_finish_n<R><<<nb, kThreads, 0, c.stream>>>(n, F[F_A], F[F_T3], F[F_W], nullptr, a.scal, a.pstar, out);
    CU(cudaGetLastError());
    return MPDPFT_OK;
  }
  const int dim = c.P.dim;
  // h = L(B z)
  if ((st = c.spectral(F[F_T1], SPEC_DERIV, dim, F[F_H], 0.0))) return st;
  if (dim == 3 || c.fk != 3) {  // terms in |grad V|^2 (the 2D finite-T form has none)
    // s1 = Sm(C' z); h -= sum_j D_j(2 d_j s1)
    if ((st = c.spectral(F[F_T2], SPEC_SMOOTH, 0, F[F_T2], 0.0))) return st;
    for (int j = 0; j < dim; ++j) {
      k_adj_times2<R><<<nb, kThreads, 0, c.stream>>>(n, F[F_D0 + j], F[F_T2], F[F_T1]);
      CU(cudaGetLastError());
      if ((st = c.spectral(F[F_T1], SPEC_DERIV, j, F[F_T1], 0.0))) return st;
      k_adj_sub<R><<<nb, kThreads, 0, c.stream>>>(n, F[F_T1], F[F_H]);
      CU(cudaGetLastError());
    }
  }
  if ((st = adj_dot<R>(c, F[F_W], F[F_H], SC_W_DOT_H))) return st;
  k_adj_finish_n<R><<<nb, kThreads, 0, c.stream>>>(n, F[F_A], F[F_T3], F[F_W], F[F_H], a.scal, a.pstar, out);
  CU(cudaGetLastError());
  return MPDPFT_OK;
}

// out = g + J_W^T eta
template <typename R>
static int adj_jw_t(Ctx& c, const R* eta, R* out) {
  Adjoint& a = *c.adj;
  R** F = (R**)a.f;
  int st;
  const int coul = c.has_interaction(MPDPFT_INT_HARTREE);
  if (coul) {
    if ((st = c.spectral(eta, SPEC_COULOMB, 0, F[F_T1], c.P.gamma_h))) return st;
    if ((st = adj_dot<R>(c, F[F_Q], eta, SC_Q_DOT_ETA))) return st;
  }
  k_adj_finish_w<R><<<a.blocks, kThreads, 0, c.stream>>>(a.n, F[F_G], F[F_T1], F[F_DX], eta, a.scal, coul, out);
  CU(cudaGetLastError());
  return MPDPFT_OK;
}

template <typename R>
static int adjoint_impl(Ctx& c, const double* dl_dn, double* dl_dvext, int mem, double tol, int max_iter,
                        int* iters_out, double* resid_out) {
  const long n = c.geom.n;
  int st;
  if (!c.adj) {
    c.adj = new Adjoint;
    Adjoint& a = *c.adj;
    a.rsize = sizeof(R);
    a.n = n;
    a.blocks = grid_blocks(n);
    for (int i = 0; i < F_NF; ++i) CU(cudaMalloc(&a.f[i], sizeof(R) * n));
    CU(cudaMalloc((void**)&a.scal, sizeof(double) * SC_COUNT));
    CU(cudaMalloc((void**)&a.part, sizeof(double) * 2 * a.blocks));
    CU(cudaMalloc((void**)&a.vmax, sizeof(unsigned long long)));
    CU(cudaMalloc((void**)&a.pstar, sizeof(long long)));
  }
  Adjoint& a = *c.adj;
  R** F = (R**)a.f;
  const int nb = a.blocks;
  const int dim = c.P.dim;
  ScState h0;
  if ((st = c.read_state(&h0))) return st;
  // the converged state: V, the density of the current ring slot, mu
  CU(cudaMemcpyAsync(F[F_VSAVE], c.d_V, sizeof(R) * n, cudaMemcpyDeviceToDevice, c.stream));
  R* nslot = (R*)c.d_nin + (long)h0.slot * n;
  CU(cudaMemcpyAsync(F[F_NSTAR], nslot, sizeof(R) * n, cudaMemcpyDeviceToDevice, c.stream));
  if ((st = c.import_field(dl_dn, F[F_G], MPDPFT_LAYOUT_PERIODIC, mem))) return st;
  // taper: shell maximum of V and the point that attains it, weights
  const bool taper = c.gradient && c.P.taper_off;
  const double r0 = c.P.edge * c.P.regularization_threshold, width = 2.0 * c.geom.dx;
  CU(cudaMemsetAsync(a.vmax, 0, sizeof(unsigned long long), c.stream));
  CU(cudaMemsetAsync(a.pstar, 0xff, sizeof(long long), c.stream));
  CU(cudaMemsetAsync(a.scal, 0, sizeof(double) * SC_COUNT, c.stream));
  if (taper) {
    k_adj_shell_max<R><<<nb, kThreads, 0, c.stream>>>(c.geom, F[F_VSAVE], r0, width, a.vmax);
    k_adj_argmax<R><<<nb, kThreads, 0, c.stream>>>(c.geom, F[F_VSAVE], r0, width, a.vmax, a.pstar);
    CU(cudaMemcpyAsync(a.scal + SC_VMAX, a.vmax, sizeof(unsigned long long), cudaMemcpyDeviceToDevice, c.stream));
  }
  k_adj_weights<R><<<nb, kThreads, 0, c.stream>>>(c.geom, r0, -2500.0 / (c.P.edge * c.P.edge), taper ? 1 : 0, F[F_W]);
  CU(cudaGetLastError());
  // DelField of the converged V: d_j = D_j f, Laplacian, smoothed |grad f|^2
  const R* lap = nullptr;
  const R* g2s = nullptr;
  if (c.gradient) {
    k_adj_taper<R><<<nb, kThreads, 0, c.stream>>>(n, F[F_VSAVE], F[F_W], a.scal, F[F_T1]);
    CU(cudaGetLastError());
    for (int j = 0; j < dim; ++j)
      if ((st = c.spectral(F[F_T1], SPEC_DERIV, j, F[F_D0 + j], 0.0))) return st;
    if ((st = c.spectral(F[F_T1], SPEC_DERIV, dim, F[F_T2], 0.0))) return st;
    k_adj_sumsq<R><<<nb, kThreads, 0, c.stream>>>(n, dim, F[F_D0], F[F_D1], F[F_D2], F[F_T3]);
    CU(cudaGetLastError());
    if ((st = c.spectral(F[F_T3], SPEC_SMOOTH, 0, F[F_T3], 0.0))) return st;
    lap = F[F_T2];
    g2s = F[F_T3];
  }
  const double mu = h0.mu[0];
  const DensParams d = c.kparams().dens[0];
  const double beta2 = c.has_interaction(MPDPFT_INT_CONTACT_SELF) ? 2.0 * c.P.beta : 0.0;
  const int dirac = c.has_interaction(MPDPFT_INT_DIRAC);
#define PREP(FKV)                                                                                                \
  k_adj_prepare<R, FKV><<<nb, kThreads, 0, c.stream>>>(c.geom, d, mu, F[F_VSAVE], lap, g2s, F[F_NSTAR], c.P.gamma_h, \
                                                       dirac, beta2, F[F_A], F[F_B], F[F_C], F[F_DX])
  if (c.fk == 1) PREP(1);
  else if (c.fk == 2) PREP(2);
  else if (c.fk == 3) PREP(3);
  else return set_error(MPDPFT_ERR_ARG, "adjoint: functional not supported (3D gradient, 3D TF, 2D gradient)");
#undef PREP
  CU(cudaGetLastError());
  if ((st = adj_dot<R>(c, F[F_A], nullptr, SC_SUM_A))) return st;
  k_adj_precond<R><<<nb, kThreads, 0, c.stream>>>(n, F[F_A], F[F_DX], F[F_M]);
  CU(cudaGetLastError());
  // Hartree: the total-charge field q = K e_0 - K_sym e_0
  if (c.has_interaction(MPDPFT_INT_HARTREE)) {
    k_adj_unit<R><<<nb, kThreads, 0, c.stream>>>(n, 0, F[F_T1]);
    CU(cudaGetLastError());
    if ((st = c.coulomb_field(F[F_T1], F[F_T2]))) return st;
    if ((st = c.spectral(F[F_T1], SPEC_COULOMB, 0, F[F_T3], c.P.gamma_h))) return st;
    k_adj_diff<R><<<nb, kThreads, 0, c.stream>>>(n, F[F_T2], F[F_T3], F[F_Q]);
    CU(cudaGetLastError());
  }
  // lambda = g + J_W^T J_N^T lambda by the device Pulay mixer (admix step)
  if ((st = c.reset_state())) return st;
  ScState hs;
  if ((st = c.read_state(&hs))) return st;
  R* lam = (R*)c.d_nin + (long)hs.slot * n;
  CU(cudaMemcpyAsync(lam, F[F_G], sizeof(R) * n, cudaMemcpyDeviceToDevice, c.stream));
  double resid = 1.0, scal2[2] = {0.0, 0.0};
  int it = 0;
  for (; it < max_iter; ++it) {
    if ((st = adj_jn_t<R>(c, lam, F[F_ETA]))) return st;
    if ((st = adj_jw_t<R>(c, F[F_ETA], F[F_OUT]))) return st;
    k_adj_resid<R><<<nb, kThreads, 0, c.stream>>>(n, F[F_OUT], lam, a.part);
    k_adj_sum2<<<1, 64, 0, c.stream>>>(a.part, nb, a.scal + SC_R2);
    CU(cudaGetLastError());
    CU(cudaMemcpyAsync(scal2, a.scal + SC_R2, sizeof(scal2), cudaMemcpyDeviceToHost, c.stream));
    CU(cudaStreamSynchronize(c.stream));
    resid = scal2[1] > 0.0 ? std::sqrt(scal2[0] / scal2[1]) : 0.0;
    if (!(resid == resid)) return set_error(MPDPFT_ERR_NONFINITE, "adjoint: non-finite residual");
    if (resid <= tol) break;
    // the (preconditioned) map's output in V (species 0); the admix step
    // mixes it with lambda into the next slot
    k_adj_step<R><<<nb, kThreads, 0, c.stream>>>(n, lam, F[F_OUT], F[F_M], (R*)c.d_V);
    CU(cudaGetLastError());
    if ((st = c.launch_step(2))) return st;
    if ((st = c.read_state(&hs))) return st;
    lam = (R*)c.d_nin + (long)hs.slot * n;
  }
  if (iters_out) *iters_out = it + 1;
  if (resid_out) *resid_out = resid;
  // dL/dV_ext = J_N^T lambda
  if ((st = c.export_field(F[F_ETA], dl_dvext, MPDPFT_LAYOUT_PERIODIC, mem))) return st;
  // restore the converged state (the Pulay history restarts)
  CU(cudaMemcpyAsync(c.d_V, F[F_VSAVE], sizeof(R) * n, cudaMemcpyDeviceToDevice, c.stream));
  CU(cudaMemcpyAsync(nslot, F[F_NSTAR], sizeof(R) * n, cudaMemcpyDeviceToDevice, c.stream));
  CU(cudaMemcpyAsync(c.d_cur, F[F_NSTAR], sizeof(R) * n, cudaMemcpyDeviceToDevice, c.stream));
  h0.hist = 0;
  h0.ncoeff = 0;
  h0.pulay_used = 0;
  CU(cudaMemcpyAsync(c.d_state, &h0, sizeof(h0), cudaMemcpyHostToDevice, c.stream));
  CU(cudaStreamSynchronize(c.stream));
  if (resid > tol) return set_error(MPDPFT_ERR_NOT_CONVERGED, "adjoint: iteration cap reached");
  return MPDPFT_OK;
}

int Ctx::adjoint(const double* dl_dn, double* dl_dvext, int layout, int mem, double tol, int max_iter, int* iters,
                 double* resid) {
  if (!initialised) return set_error(MPDPFT_ERR_ARG, "adjoint: no converged state (call sc_run first)");
  if (S != 1) return set_error(MPDPFT_ERR_ARG, "adjoint: one species only");
  if (finite_t) return set_error(MPDPFT_ERR_ARG, "adjoint: the finite-T gradient form is not differentiated");
  if (layout != MPDPFT_LAYOUT_PERIODIC) return set_error(MPDPFT_ERR_ARG, "adjoint: periodic layout only");
  if (!dl_dn || !dl_dvext) return set_error(MPDPFT_ERR_ARG, "adjoint: null array");
  if (max_iter < 1) return set_error(MPDPFT_ERR_ARG, "adjoint: max_iter < 1");
  if (has_interaction(MPDPFT_INT_HARTREE_INTER) || has_interaction(MPDPFT_INT_COULOMB_CHARGED) ||
      has_interaction(MPDPFT_INT_CONTACT_MUTUAL))
    return set_error(MPDPFT_ERR_ARG, "adjoint: interactions 8, 10, 11 only");
  if (adj && adj->rsize != rsize) adjoint_release();
  return rsize == sizeof(double) ? adjoint_impl<double>(*this, dl_dn, dl_dvext, mem, tol, max_iter, iters, resid)
                                 : adjoint_impl<float>(*this, dl_dn, dl_dvext, mem, tol, max_iter, iters, resid);
}

// dL/dR for Gaussian nuclei given dL/dV_ext (periodic layout, double).
int Ctx::adjoint_nuclei(const double* dl_dvext, int mem, int nn, const double* z, const double* pos, double sigma,
                        double* dl_dpos) {
  if (nn < 1 || nn > 64 || !z || !pos || !dl_dpos || !dl_dvext || !(sigma > 0.0))
    return set_error(MPDPFT_ERR_ARG, "adjoint_nuclei: bad arguments (1..64 nuclei, sigma > 0)");
  if (P.dim != 3) return set_error(MPDPFT_ERR_ARG, "adjoint_nuclei: 3D only");
  const long n = geom.n;
  const int nb = std::min(grid_blocks(n), 592);
  double *d_g = nullptr, *d_zp = nullptr, *d_part = nullptr, *d_out = nullptr;
  auto cleanup = [&]() { cudaFree(d_g); cudaFree(d_zp); cudaFree(d_part); cudaFree(d_out); };
  cudaError_t e = cudaSuccess;
  const double* gv = dl_dvext;
  if (mem == MPDPFT_MEM_HOST) {
    if ((e = cudaMalloc((void**)&d_g, sizeof(double) * n)) != cudaSuccess) { cleanup(); CU(e); }
    if ((e = cudaMemcpyAsync(d_g, dl_dvext, sizeof(double) * n, cudaMemcpyHostToDevice, stream)) != cudaSuccess) {
      cleanup(); CU(e);
    }
    gv = d_g;
  }
  std::vector<double> zp(4 * (size_t)nn);
  for (int a = 0; a < nn; ++a) zp[a] = z[a];
  for (int i = 0; i < 3 * nn; ++i) zp[nn + i] = pos[i];
  if ((e = cudaMalloc((void**)&d_zp, sizeof(double) * zp.size())) != cudaSuccess ||
      (e = cudaMemcpyAsync(d_zp, zp.data(), sizeof(double) * zp.size(), cudaMemcpyHostToDevice, stream)) != cudaSuccess ||
      (e = cudaMalloc((void**)&d_part, sizeof(double) * (size_t)nb * 3 * nn)) != cudaSuccess ||
      (e = cudaMalloc((void**)&d_out, sizeof(double) * 3 * nn)) != cudaSuccess) {
    cleanup();
    CU(e);
  }
  k_adj_nuclei<<<nb, kThreads, 0, stream>>>(geom, gv, nn, d_zp, d_zp + nn, sigma, d_part);
  k_adj_sum_rows<<<1, kThreads, 0, stream>>>(d_part, nb, 3 * nn, d_out);
  e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpyAsync(dl_dpos, d_out, sizeof(double) * 3 * nn, cudaMemcpyDeviceToHost, stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
  cleanup();
  CU(e);
  return MPDPFT_OK;
}

}  // namespace mpdpft
