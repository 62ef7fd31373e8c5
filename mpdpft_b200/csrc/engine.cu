// engine.cu -- host side of the B200 DPFT engine and its C ABI.
//
// A context owns every device buffer of one SC solve on one GPU: fields are
// stored on the periodic s^D grid in the compute precision (double for
// MPDPFT_FP64, float for MPDPFT_MIXED); the particle-number integrals, the
// convergence dots, the Pulay Gram matrix and solve, and the energies are
// accumulated in double in every mode.  All work is issued on the context's
// stream; the SC iteration is one persistent kernel (plus the FFT kernels for
// Coulomb and gradient terms) and is replayed as a CUDA graph.
#include <cuda_runtime.h>
#if defined(__x86_64__) && defined(__SSE2__)
#include <immintrin.h>
#endif
#include <cstdint>

#include <algorithm>
#include <atomic>
#include <condition_variable>
#include <functional>
#include <mutex>
#include <chrono>
#include <cstdio>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "../../include/mpdpft_gpu.h"
#include "common.cuh"
#include "engine.h"
#include "sc_kernel.cuh"

namespace mpdpft {

thread_local std::string g_last_error;

// programmatic dependent launch of the SC iteration's kernels (launch_k)
static std::atomic<bool> g_pdl{true};
bool pdl_enabled() { return g_pdl.load(std::memory_order_relaxed); }
void pdl_disable() { g_pdl.store(false, std::memory_order_relaxed); }

int set_error(int status, const std::string& msg) {
  g_last_error = msg;
  return status;
}

#define CU(call)                                                                         \
  do {                                                                                   \
    cudaError_t e_ = (call);                                                             \
    if (e_ != cudaSuccess)                                                               \
      return set_error(MPDPFT_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

// ------------------------------------------------------------- kernels ----
template <typename R, typename S = double>
__global__ void k_import(const S* __restrict__ src, R* __restrict__ dst, Geom g, int layout) {
  const long n = g.n;
  for (long p = (long)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (long)gridDim.x * blockDim.x) {
    long q = p;
    if (layout == MPDPFT_LAYOUT_REFERENCE) {
      const long el = g.s + 1;
      int k = (int)(p % g.s);
      long t = p / g.s;
      if (g.dim == 3) {
        int j = (int)(t % g.s), i = (int)(t / g.s);
        q = ((long)i * el + j) * el + k;
      } else {
        q = t * el + k;
      }
    }
    dst[p] = (R)src[q];
  }
}

template <typename R, typename D = double>
__global__ void k_export(const R* __restrict__ src, D* __restrict__ dst, Geom g, int layout) {
  long total = g.n;
  const long el = g.s + 1;
  if (layout == MPDPFT_LAYOUT_REFERENCE) total = (g.dim == 3) ? el * el * el : el * el;
  for (long q = (long)blockIdx.x * blockDim.x + threadIdx.x; q < total; q += (long)gridDim.x * blockDim.x) {
    long p = q;
    if (layout == MPDPFT_LAYOUT_REFERENCE) {
      int k = (int)(q % el) % g.s;
      long t = q / el;
      if (g.dim == 3) {
        int j = (int)(t % el) % g.s, i = (int)(t / el) % g.s;
        p = ((long)i * g.s + j) * g.s + k;
      } else {
        p = (t % g.s) * g.s + k;
      }
    }
    dst[q] = (D)src[p];
  }
}

// Energy integrands (GetEnergy, mpDPFT.cpp:5414-5436), one block partial per
// accumulator: per species [0] int (mu-V)_+^{(D+2)/2}, [1] int Vext n,
// [2] int n^2, [3] int n_+^{1+1/D}, [4] int n vh/2; pairs [16+...] int n_s n_s'.
// NS = S at compile time: only the accumulators of NS species are held
// (the row's other entries are written as 0), and the powers are products
// with one square or cube root instead of pow.
template <typename R, int NS>
__global__ void k_energy(Geom g, const R* V, const R* vext, const R* dens, const R* vh, const double* mu,
                         double* part) {
  constexpr int NP = NS * (NS - 1) / 2;
  constexpr int NA = 5 * NS + (NP > 0 ? NP : 1);
  double acc[NA];
#pragma unroll
  for (int j = 0; j < NA; ++j) acc[j] = 0.0;
  const long n = g.n;
  const bool d3 = g.dim == 3;
  for (long p = (long)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (long)gridDim.x * blockDim.x) {
    double nsv[NS];
#pragma unroll
    for (int s = 0; s < NS; ++s) {
      const long q = (long)s * n + p;
      const double u = mu[s] - (double)V[q];
      const double ns = (double)dens[q];
      nsv[s] = ns;
      acc[5 * s + 0] += u > 0.0 ? (d3 ? u * u * sqrt(u) : u * u) : 0.0;
      acc[5 * s + 1] += (double)vext[q] * ns;
      acc[5 * s + 2] += ns * ns;
      acc[5 * s + 3] += ns > 0.0 ? (d3 ? ns * cbrt(ns) : ns * sqrt(ns)) : 0.0;
      if (vh) acc[5 * s + 4] += 0.5 * ns * (double)vh[q];
    }
    int k = 5 * NS;
#pragma unroll
    for (int s = 0; s < NS; ++s)
#pragma unroll
      for (int t = s + 1; t < NS; ++t) acc[k++] += nsv[s] * nsv[t];
  }
  __shared__ double red[NA];
  block_reduce_store<NA>(acc, red);
  __syncthreads();
  double* out = part + (long)blockIdx.x * kNEnergy;
  for (int v = threadIdx.x; v < kNEnergy; v += blockDim.x) {
    double x = 0.0;
    if (v < 5 * kMaxS) {
      if (v / 5 < NS) x = red[v];
    } else if (v < kEkinOff) {
      const int s = (v - 5 * kMaxS) / kMaxS, t = (v - 5 * kMaxS) % kMaxS;
      if (s < t && t < NS) x = red[5 * NS + s * NS - s * (s + 1) / 2 + (t - s - 1)];
    }
    out[v] = x;
  }
}

// Kinetic energy integrands of the gradient-corrected density, per species
// (GetDispersalEnergy, DensityExpression 5, mpDPFT.cpp:5606-5703), one block
// partial per accumulator: [s] the point values, [kMaxS + s] V n (2D).
//  2D: g/2 [lap CurlyA(y)/(12 pi) - |grad V|^{4/3} (y^2 CurlyA(y) + Ai(y) +
//      y Ai'(y))/(8 pi)], y = 2 (V - mu)/|grad V|^{2/3}; 0 where |grad V|^2
//      <= MP; Ai = Ai' = 0 from y = 50.
//  3D (EkinAiT03D): (2u)^{5/2}/5 - lap (2u)^{1/2}/6, u = mu - V > 0, where
//      a = |grad V|^{2/3}/2 < thr; else the Airy-weighted integral
//      int_0^{x1} Ai(x + U/a) [(2ax)^{5/2}/5 - lap (2ax)^{1/2}/6] dx by the
//      trapezoid rule on 64, 128, ... points until two agree (ASYMcritABS <
//      MP), or until maxit doublings (the reference's NegligibleMagnitudeQ
//      exit against e_env = int V_ext n).
template <typename R>
__global__ void k_ekin_grad(Geom g, int S, double gdeg, double thr, int maxit, double internal_acc,
                            double area_pref, const R* V, const R* lap, const R* g2, const R* dens,
                            const double* mu, const double* e_env, double* part) {
  double acc[2 * kMaxS];
#pragma unroll
  for (int j = 0; j < 2 * kMaxS; ++j) acc[j] = 0.0;
  const long n = g.n;
  constexpr double kMP = 1.0e-12;
  for (long p = (long)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (long)gridDim.x * blockDim.x) {
    for (int s = 0; s < S; ++s) {
      const long q = (long)s * n + p;
      const double U = (double)V[q] - mu[s], L = (double)lap[q], ab = fabs((double)g2[q]);
      double t = 0.0;
      if (g.dim == 2) {
        if (ab > kMP) {
          const double y = 2.0 * U / cbrt(ab);
          double ai = 0.0, aip = 0.0;
          if (y < 50.0) airy_ai_d(y, ai, aip);
          const double ca = curly_a(y);
          t = 0.5 * gdeg * (L * ca / (12.0 * kPi) - pow(ab, 2.0 / 3.0) * (y * y * ca + ai + y * aip) / (8.0 * kPi));
        }
        acc[kMaxS + s] += (double)V[q] * (double)dens[q];
      } else {
        const double a = 0.5 * cbrt(ab);
        if (a < thr) {
          const double w = -2.0 * U;
          t = w > 0.0 ? w * w * sqrt(w) / 5.0 - L * sqrt(w) / 6.0 : 0.0;
        } else {
          const double x1 = fmax(1.0, 100.0 - U / a);
          double prev = 1.0, res = 0.0;
          for (int it = 0, m = 64;; ++it, m *= 2) {
            const double h = x1 / (double)(m - 1);
            double sum = 0.0;
            for (int j = 0; j < m; ++j) {
              const double x = (double)j * h, y = x + U / a;
              double ai = 0.0, aip;
              if (!(y > 100.0)) {
                if (y > -300.0) airy_ai_d(y, ai, aip);
                else ai = cos(2.0 * (-y) * sqrt(-y) / 3.0 - 0.25 * kPi) / (1.7724538509055159 * sqrt(sqrt(-y)));
              }
              const double w = 2.0 * a * x;
              const double f = ai * (w * w * sqrt(w) / 5.0 - L * sqrt(w) / 6.0);
              sum += (j == 0 || j == m - 1) ? 0.5 * f : f;
            }
            res = sum * h;
            if (it > 0) {
              const bool tiny = fabs(res) < kMP && fabs(prev) < kMP;
              const double da = tiny ? 0.0 : fabs((res - prev) / (res + prev));
              const double dr = (res == 0.0 && prev == 0.0) ? 0.0 : fabs((res - prev) / (res + prev));
              if (da < kMP || (dr < internal_acc && negligible_magnitude(e_env[5 * s + 1], area_pref * res,
                                                                      -log(internal_acc))))
                break;
            }
            if (it == maxit) break;
            prev = res;
          }
          t = res;
        }
      }
      acc[s] += t;
    }
  }
  block_reduce_store<2 * kMaxS>(acc, part + (long)blockIdx.x * 2 * kMaxS);
}

// out[v] = scale * sum over rows b < nb of part[b * nv + v]: block v sums
// column v (each thread a strided share of the rows, then a fixed-order
// tree), so the result is the same in every run.  Launch with nv blocks.
__global__ void k_sum_rows(const double* part, int nb, int nv, double scale, double* out) {
  __shared__ double sh[32];
  const int v = blockIdx.x, lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  double t = 0.0;
  for (int b = threadIdx.x; b < nb; b += blockDim.x) t += part[(long)b * nv + v];
  t = warp_sum(t);
  if (lane == 0) sh[w] = t;
  __syncthreads();
  if (threadIdx.x == 0) {
    double x = 0.0;
    for (int i = 0; i < (int)(blockDim.x >> 5); ++i) x += sh[i];
    out[v] = x * scale;
  }
}

template <typename R>
__global__ void k_integrate(Geom g, const R* f, double* part) {
  double acc[1] = {0.0};
  for (long p = (long)blockIdx.x * blockDim.x + threadIdx.x; p < g.n; p += (long)gridDim.x * blockDim.x)
    acc[0] += (double)f[p];
  block_reduce_store<1>(acc, part + blockIdx.x);
}

// Trapezoid sum over the reference's (s+1)^D storage with its end weights
// (Riemann, mpDPFT.cpp:7981-8026); the duplicate planes need not repeat
// plane 0.
__global__ void k_integrate_ref(Geom g, const double* f, double* part) {
  const unsigned el = (unsigned)g.s + 1;
  const unsigned total = g.dim == 3 ? el * el * el : el * el;
  double acc[1] = {0.0};
  for (unsigned q = blockIdx.x * blockDim.x + threadIdx.x; q < total; q += gridDim.x * blockDim.x)
    acc[0] += riemann_weight(q, el, g.dim) * f[q];
  block_reduce_store<1>(acc, part + blockIdx.x);
}

// n[V] at a fixed mu (GetDensity), no reduction.
template <typename R>
__global__ void k_density(Geom g, DensParams d, double mu, const R* V, const R* lap, const R* g2, R* out) {
  for (long p = (long)blockIdx.x * blockDim.x + threadIdx.x; p < g.n; p += (long)gridDim.x * blockDim.x)
    out[p] = density_at<R>(d, R(mu) - V[p], lap ? lap[p] : R(0), g2 ? g2[p] : R(0));
}

// The mu kernel (which 0) and the density kernel for Pulay windows <= 5
// (which 1), <= 8 (which 3) or up to kMaxP (which 2), of functional kind fk.
template <typename R, int FK>
static const void* sc_kernel_fk(int which) {
  if (which == 0) return (const void*)sc_mu_kernel<R, FK>;
  if (which == 1) return (const void*)sc_density_kernel<R, FK, 5>;
  if (which == 3) return (const void*)sc_density_kernel<R, FK, 8>;
  return (const void*)sc_density_kernel<R, FK, kMaxP>;
}

template <typename R>
static const void* sc_kernel_ptr(int which, int fk) {
  if (fk == 1) return sc_kernel_fk<R, 1>(which);
  if (fk == 2) return sc_kernel_fk<R, 2>(which);
  if (fk == 3) return sc_kernel_fk<R, 3>(which);
  return sc_kernel_fk<R, 0>(which);
}

// ---------------------------------------------------------- the context --
Ctx::~Ctx() { release(); }

void Ctx::release() {
  adjoint_release();
  drop_graphs();
  for (void* p : allocations) cudaFree(p);
  allocations.clear();
  if (pinned) { cudaFreeHost(pinned); pinned = nullptr; }
  for (cudaEvent_t e : copy_events) cudaEventDestroy(e);
  copy_events.clear();
  copy_pool.reset();
  if (stream) { cudaStreamDestroy(stream); stream = nullptr; }
}

int Ctx::alloc(void** p, size_t bytes) {
  if (bytes == 0) bytes = 16;
  cudaError_t e = cudaMalloc(p, bytes);
  if (e != cudaSuccess) return set_error(MPDPFT_ERR_CUDA, std::string("cudaMalloc: ") + cudaGetErrorString(e));
  allocations.push_back(*p);
  return MPDPFT_OK;
}

static int check_params(const mpdpft_params& p) {
  if (p.dim != 2 && p.dim != 3) return set_error(MPDPFT_ERR_ARG, "dim must be 2 or 3");
  if (p.steps < 4 || (p.steps & 1)) return set_error(MPDPFT_ERR_ARG, "steps must be even and >= 4");
  if ((p.dim == 3 && p.steps > 1024) || (p.dim == 2 && p.steps > 32768))
    return set_error(MPDPFT_ERR_ARG, "steps too large (grid indices are 32-bit)");
  if (p.species < 1 || p.species > MPDPFT_MAX_SPECIES) return set_error(MPDPFT_ERR_ARG, "species out of range");
  if (!(p.edge > 0.0)) return set_error(MPDPFT_ERR_ARG, "edge must be positive");
  if (p.mixer < 0 || p.mixer > 1) return set_error(MPDPFT_ERR_ARG, "mixer must be 0 (linear) or 1 (Pulay)");
  if (p.mixer == 1 && (p.pulay_scope < 1 || p.pulay_scope > MPDPFT_MAX_PULAY))
    return set_error(MPDPFT_ERR_ARG, "pulay_scope out of range");
  if (p.n_interactions < 0 || p.n_interactions > MPDPFT_MAX_INTERACTIONS)
    return set_error(MPDPFT_ERR_ARG, "n_interactions out of range");
  int de = p.density_expression;
  if (de != MPDPFT_DENS_TF && de != MPDPFT_DENS_TF_INSPIRED && de != MPDPFT_DENS_TF_INSPIRED_T &&
      de != MPDPFT_DENS_GRADIENT)
    return set_error(MPDPFT_ERR_ARG, "unsupported density_expression");
  for (int a = 0; a < p.n_interactions; ++a) {
    int t = p.interactions[a];
    if (t != 0 && t != 1 && t != 8 && t != 10 && t != 11 && t != 21 && t != 100)
      return set_error(MPDPFT_ERR_ARG, "unsupported interaction type " + std::to_string(t));
    if ((t == 8 || t == 21 || t == 100) && p.dim == 2 && p.coulomb_kernel == MPDPFT_COULOMB_TRUNCATED)
      return set_error(MPDPFT_ERR_ARG, "2D Coulomb interactions use the reference's regularised 2D kernel only");
  }
  if (p.precision != MPDPFT_FP64 && p.precision != MPDPFT_MIXED) return set_error(MPDPFT_ERR_ARG, "bad precision");
  if (p.gradient_form != MPDPFT_GRADIENT_T0 && p.gradient_form != MPDPFT_GRADIENT_FINITE_T)
    return set_error(MPDPFT_ERR_ARG, "bad gradient_form");
  if (p.gradient_form == MPDPFT_GRADIENT_FINITE_T && de == MPDPFT_DENS_GRADIENT) {
    if (p.dim != 3) return set_error(MPDPFT_ERR_ARG, "the finite-T gradient form is 3D (2D uses its own finite-T form)");
    if (p.boole_pairs < 1 || p.boole_pairs > 50)
      return set_error(MPDPFT_ERR_ARG, "boole_pairs must be 1 to 50 (the reference caps Mpp[0] at 50)");
    if (p.boole_max_iter < 0 || p.boole_max_iter > 21) return set_error(MPDPFT_ERR_ARG, "boole_max_iter must be 0 to 21");
    if (!(p.internal_acc > 0.0)) return set_error(MPDPFT_ERR_ARG, "internal_acc must be positive");
    for (int s = 0; s < p.species; ++s)
      if (p.temperature[s] == 0.0)
        return set_error(MPDPFT_ERR_ARG, "the finite-T gradient form needs T > 0 (or T < 0: automatic)");
  }
  if (p.max_sc_count < 0) return set_error(MPDPFT_ERR_ARG, "max_sc_count < 0");
  return MPDPFT_OK;
}

bool Ctx::has_interaction(int t) const {
  for (int a = 0; a < P.n_interactions; ++a)
    if (P.interactions[a] == t) return true;
  return false;
}

KParams Ctx::kparams() const {
  KParams k;
  std::memset(&k, 0, sizeof(k));
  k.geom = geom;
  k.S = P.species;
  for (int s = 0; s < P.species; ++s) {
    DensParams& d = k.dens[s];
    d.expr = P.density_expression;
    d.dim = P.dim;
    d.g = P.degeneracy;
    d.tau = P.tau[s];
    d.T = temperature[s];
    d.floor_u = P.gradient_floor;
    d.c2 = P.gradient_grad2;
    d.finite_t = finite_t ? 1 : 0;
    d.airy_thr = std::fabs(P.airy_threshold);
    d.boole_pairs = P.boole_pairs;
    d.boole_max_iter = P.boole_max_iter;
    d.rtpna = P.internal_acc;
    d.avg_density = P.abundances[s] / std::pow(P.edge, (double)P.dim);  // AverageDensity (mpDPFT.cpp:1003)
    d.cut = density_has_cut(d.expr, d.dim, d.finite_t) && (d.expr != MPDPFT_DENS_TF_INSPIRED || d.tau > 0.0);
    k.abundance[s] = P.abundances[s];
    k.charges[s] = P.charges[s];
  }
  k.rel_acc = P.rel_acc;
  k.beta = P.beta;
  k.gamma_h = P.gamma_h;
  k.contact_self = has_interaction(MPDPFT_INT_CONTACT_SELF);
  k.contact_mutual = has_interaction(MPDPFT_INT_CONTACT_MUTUAL);
  k.dirac = has_interaction(MPDPFT_INT_DIRAC);
  k.has_coulomb = has_coulomb;
  k.mixer = P.mixer;
  k.scope = P.mixer ? P.pulay_scope : 1;
  k.ring = ring;
  k.sc_criterion = P.sc_criterion;
  k.max_sc = P.max_sc_count;
  k.schedule = P.schedule;
  k.pot_tol = P.potential_tol;
  k.inc_v0 = P.incremental_v;
  k.chunk = chunk;
  k.mu_blocks = step_blocks;
  k.vec4 = (geom.n % 4) == 0;
  k.mu_max_passes = mu_max_passes;
  k.spin_limit = spin_limit;
  return k;
}

// Device loop limits of this context: the mu-search pass cap and the grid
// barrier's spin limit (negative: the defaults).  The captured iteration
// carries the old values, so it is rebuilt on the next graph step.
int Ctx::set_limits(int mu_passes, long long spins) {
  if (mu_passes > kMuMaxPasses) return set_error(MPDPFT_ERR_ARG, "mu pass cap above the device maximum");
  if (mu_passes == 0) return set_error(MPDPFT_ERR_ARG, "mu pass cap must be at least 1");
  mu_max_passes = mu_passes < 0 ? kMuMaxPasses : mu_passes;
  spin_limit = spins < 0 ? kBarrierSpinLimit : (long)spins;
  drop_graphs();
  return MPDPFT_OK;
}

int Ctx::init(const mpdpft_params& params, int dev) {
  int st = check_params(params);
  if (st) return st;
  P = params;
  device = dev;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
    return set_error(MPDPFT_ERR_NO_DEVICE, "no CUDA device");
  if (dev < 0 || dev >= ndev) return set_error(MPDPFT_ERR_ARG, "device index out of range");
  CU(cudaSetDevice(dev));
  cudaDeviceProp prop;
  CU(cudaGetDeviceProperties(&prop, dev));
  if (prop.major < 10) return set_error(MPDPFT_ERR_NO_DEVICE, "needs an sm_100 (Blackwell) device");
  num_sms = prop.multiProcessorCount;
  CU(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
  geom.dim = P.dim;
  geom.s = P.steps;
  geom.n = 1;
  for (int d = 0; d < P.dim; ++d) geom.n *= P.steps;
  geom.L = P.edge;
  geom.dx = P.edge / P.steps;
  geom.dk = 2.0 * kPi / P.edge;
  geom.dvol = std::pow(geom.dx, (double)P.dim);
  n_ref = 1;
  for (int d = 0; d < P.dim; ++d) n_ref *= (P.steps + 1);
  rsize = P.precision == MPDPFT_FP64 ? sizeof(double) : sizeof(float);
  S = P.species;
  ring = (P.mixer ? P.pulay_scope : 1) + 1;
  gradient = P.density_expression == MPDPFT_DENS_GRADIENT;
  // |grad V|^2 enters only the 3D form with a |grad V|^2 coefficient; the
  // reference's small-gradient branch (and the 2D form) use the Laplacian
  // alone, so the SC loop's DelField then skips the gradients
  finite_t = gradient && P.dim == 3 && P.gradient_form == MPDPFT_GRADIENT_FINITE_T;
  // the finite-T form reads |grad V|^2 for its Airy-branch test
  need_g2 = gradient && P.dim == 3 && (finite_t || P.gradient_grad2 != 0.0);
  has_coulomb = has_interaction(MPDPFT_INT_HARTREE) || has_interaction(MPDPFT_INT_HARTREE_INTER) ||
                has_interaction(MPDPFT_INT_COULOMB_CHARGED);
  for (int s = 0; s < S; ++s) temperature[s] = P.temperature[s];
  const size_t field = (size_t)geom.n * rsize;
  if ((st = alloc(&d_vext, field * S))) return st;
  if ((st = alloc(&d_V, field * S))) return st;
  if ((st = alloc(&d_nin, field * S * ring))) return st;
  if ((st = alloc(&d_res, field * S * ring))) return st;
  if ((st = alloc(&d_tmp, field * S))) return st;
  if ((st = alloc(&d_cur, field * S))) return st;
  if (gradient) {
    if ((st = alloc(&d_lap, field * S))) return st;
    if ((st = alloc(&d_g2, field * S))) return st;
  }
  if (has_coulomb) {
    if ((st = alloc(&d_vh, field * S))) return st;
  }
  if ((st = alloc((void**)&d_io, sizeof(double) * (size_t)std::max(n_ref, geom.n) * 2))) return st;
  if ((st = alloc((void**)&d_state, sizeof(ScState)))) return st;
  log_cap = P.max_sc_count + 2;
  if ((st = alloc((void**)&d_log, sizeof(mpdpft_iter_log) * log_cap))) return st;
  // persistent-kernel grid: co-resident blocks only
  // grids: the cooperative mu kernel holds co-resident blocks only; the
  // density and mixing kernels fill every SM
  auto occupancy = [&](const void* fn, int threads, int* occ) -> int {
    cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(occ, fn, threads, 0);
    if (e != cudaSuccess) return set_error(MPDPFT_ERR_CUDA, std::string("occupancy: ") + cudaGetErrorString(e));
    if (*occ < 1) return set_error(MPDPFT_ERR_CUDA, "SC kernel cannot be resident");
    return MPDPFT_OK;
  };
  const bool f64 = P.precision == MPDPFT_FP64;
  int occ_mu = 0, occ_dens = 0, occ_mix = 0;
  fk = functional_kind(P.density_expression, P.dim, finite_t);
  if ((st = occupancy(f64 ? sc_kernel_ptr<double>(0, fk) : sc_kernel_ptr<float>(0, fk), kStepThreads, &occ_mu)))
    return st;
  dens_which = density_variant(P.mixer ? P.pulay_scope : 1);
  if ((st = occupancy(f64 ? sc_kernel_ptr<double>(dens_which, fk) : sc_kernel_ptr<float>(dens_which, fk), kDensityThreads,
                      &occ_dens)))
    return st;
  if ((st = occupancy(f64 ? (const void*)sc_mix_kernel<double> : (const void*)sc_mix_kernel<float>, kDensThreads,
                      &occ_mix)))
    return st;
  step_blocks = num_sms * std::min(occ_mu, 2);
  long useful = (geom.n + kStepThreads - 1) / kStepThreads;
  if (step_blocks > useful) step_blocks = (int)std::max(1L, useful);
  const long groups = (geom.n + 3) / 4;  // the mixing kernel takes 4 points a thread
  dens_blocks = (int)std::max(1L, std::min((long)num_sms * occ_dens, (geom.n + 4 * kDensityThreads - 1) / (4 * kDensityThreads)));
  mix_blocks = (int)std::max(1L, std::min((long)num_sms * occ_mix, (groups + kDensThreads - 1) / kDensThreads));
  // the mu kernel's list sweeps: a contiguous chunk of points per warp
  {
    const long warps = (long)step_blocks * kStepWarps;
    chunk = (geom.n + warps - 1) / warps;
    chunk = (chunk + kSegPts - 1) / kSegPts * kSegPts;
    if ((st = alloc((void**)&d_bcount, sizeof(int) * (size_t)kMaxS * step_blocks))) return st;
    // a warp's region holds its owned points, whole 32-point segments
    plist_stride = geom.n + 32L * (warps + 1);
    if ((st = alloc((void**)&d_plist, sizeof(int) * (size_t)S * plist_stride))) return st;
    if ((st = alloc((void**)&d_part2, sizeof(double) * (size_t)dens_blocks * kNPart))) return st;
  }
  part_vals = std::max(kNPart, kNEnergy);
  if ((st = alloc((void**)&d_part, sizeof(double) * (size_t)std::max(step_blocks, kMaxBlocks) * part_vals))) return st;
  // two halves, the second starting on a 16-byte boundary (streaming stores)
  pinned_bytes = sizeof(double) * (size_t)((std::max(n_ref, geom.n) + 1) & ~1L) * 2;
  CU(cudaMallocHost(&pinned, pinned_bytes));
  CU(cudaMemsetAsync(d_V, 0, field * S, stream));
  CU(cudaMemsetAsync(d_vext, 0, field * S, stream));
  CU(cudaMemsetAsync(d_nin, 0, field * S * ring, stream));
  CU(cudaMemsetAsync(d_cur, 0, field * S, stream));
  CU(cudaMemsetAsync(d_res, 0, field * S * ring, stream));
  CU(cudaMemsetAsync(d_log, 0, sizeof(mpdpft_iter_log) * log_cap, stream));
  if (gradient) {
    CU(cudaMemsetAsync(d_g2, 0, field * S, stream));
    CU(cudaMemsetAsync(d_lap, 0, field * S, stream));
  }
  return reset_state();
}

int Ctx::reset_state(bool sync) {
  ScState h;
  std::memset(&h, 0, sizeof(h));
  for (int s = 0; s < S; ++s) {
    h.mu[s] = h.prev_mu[s] = h.old_mu[s] = P.mu[s];
    h.theta[s] = h.theta0[s] = h.theta_mix[s] = P.theta[s];
  }
  h.dmm = P.deltamu_modifier;
  h.inc_v = P.incremental_v;
  h.cc = 0.0;
  h.old_cc = 0.0;  // the reference leaves data.CC indeterminate before iteration 0
  // a pageable source: the copy has read h when the call returns
  CU(cudaMemcpyAsync(d_state, &h, sizeof(h), cudaMemcpyHostToDevice, stream));
  if (sync) CU(cudaStreamSynchronize(stream));
  return MPDPFT_OK;
}

int Ctx::read_state(ScState* h) {
  CU(cudaMemcpyAsync(h, d_state, sizeof(ScState), cudaMemcpyDeviceToHost, stream));
  CU(cudaStreamSynchronize(stream));
  return MPDPFT_OK;
}

// Copy one grid (host or device double pointer, either layout) into the
// compute-precision device array dst.  Host data is staged through half
// `slot` (0 or 1) of the pinned buffer and of d_io; with sync = false the
// caller synchronises the stream before that half is used again.
double* Ctx::host_stage(int slot) { return (double*)pinned + (slot ? ((std::max(n_ref, geom.n) + 1) & ~1L) : 0); }

// Grids between a caller's host array and the device in kCopyChunk pieces,
// pipelined over the context's host copy threads (CopyPool, started once):
// on import the workers copy chunks into the pinned buffer and the calling
// thread queues each chunk's DMA as soon as it is copied (in chunk order);
// on export the calling thread queues every chunk's DMA with an event after
// it, waits for the events in order and releases each chunk to the workers,
// which copy it out.  Only the calling thread makes CUDA calls.
constexpr long kCopyChunk = 1L << 16;  // doubles (512 KB)

// n doubles into pinned staging memory with non-temporal stores where the
// host has them (x86-64): cached stores leave the staged grid dirty in the
// host's caches, and the DMA that reads it next then ran at a fifth of the
// speed it has from memory (measured on the B200 host: 16.8 MB in 1.5 ms vs
// 0.3 ms).
void copy_to_pinned(double* dst, const double* src, long n) {
#if defined(__x86_64__) && defined(__SSE2__)
  if (((uintptr_t)dst & 15) == 0) {
    long i = 0;
    for (; i + 2 <= n; i += 2) _mm_stream_si128((__m128i*)(dst + i), _mm_loadu_si128((const __m128i*)(src + i)));
    for (; i < n; ++i) dst[i] = src[i];
    _mm_sfence();
    return;
  }
#endif
  std::memcpy(dst, src, sizeof(double) * n);
}

// n doubles rounded to float (round to nearest, as the device conversion)
// into pinned staging memory, with non-temporal stores as copy_to_pinned.
static void convert_to_pinned(float* dst, const double* src, long n) {
#if defined(__x86_64__) && defined(__SSE2__)
  if (((uintptr_t)dst & 15) == 0) {
    long i = 0;
    for (; i + 4 <= n; i += 4) {
      const __m128 lo = _mm_cvtpd_ps(_mm_loadu_pd(src + i)), hi = _mm_cvtpd_ps(_mm_loadu_pd(src + i + 2));
      _mm_stream_ps(dst + i, _mm_movelh_ps(lo, hi));
    }
    for (; i < n; ++i) dst[i] = (float)src[i];
    _mm_sfence();
    return;
  }
#endif
  for (long i = 0; i < n; ++i) dst[i] = (float)src[i];
}

CopyPool::CopyPool() {
  const int hw = (int)std::max(1u, std::thread::hardware_concurrency());
  nt = std::max(1, std::min(8, hw - 1));
  for (int t = 0; t < nt; ++t)
    th.emplace_back([this, t] {
      unsigned seen = 0;
      for (;;) {
        std::function<void(int)> f;
        {
          std::unique_lock<std::mutex> l(m);
          cv.wait(l, [&] { return stop || gen != seen; });
          if (stop) return;
          seen = gen;
          f = job;
        }
        f(t);
        std::lock_guard<std::mutex> l(m);
        if (--pending == 0) done.notify_all();
      }
    });
}

CopyPool::~CopyPool() {
  {
    std::lock_guard<std::mutex> l(m);
    stop = true;
  }
  cv.notify_all();
  for (std::thread& x : th) x.join();
}

void CopyPool::begin(std::function<void(int)> f) {
  {
    std::lock_guard<std::mutex> l(m);
    job = std::move(f);
    pending = nt;
    ++gen;
  }
  cv.notify_all();
}

void CopyPool::wait() {
  std::unique_lock<std::mutex> l(m);
  done.wait(l, [&] { return pending == 0; });
}

static void stage_chunk(double* dst, const double* src, long n) { copy_to_pinned(dst, src, n); }
static void stage_chunk(float* dst, const double* src, long n) { convert_to_pinned(dst, src, n); }
static void unstage_chunk(double* dst, const double* src, long n) { std::memcpy(dst, src, sizeof(double) * n); }
static void unstage_chunk(double* dst, const float* src, long n) {
  for (long i = 0; i < n; ++i) dst[i] = (double)src[i];
}

// cnt values of a caller's double array into device memory as T (double,
// or float for FP32 fields: rounded on the host, half the bytes over the
// link) through the pinned buffer hs.
template <typename T>
static int stage_in(Ctx& c, T* dstage, T* hs, const double* src, long cnt) {
  const long nchunk = (cnt + kCopyChunk - 1) / kCopyChunk;
  if (!c.copy_pool) c.copy_pool.reset(new CopyPool());
  CopyPool& P = *c.copy_pool;
  std::vector<std::atomic<int>> ready(nchunk);
  for (auto& r : ready) r.store(0);
  const int nt = P.nt;
  P.begin([&](int t) {
    for (long k = t; k < nchunk; k += nt) {
      const long off = k * kCopyChunk, len = std::min(kCopyChunk, cnt - off);
      stage_chunk(hs + off, src + off, len);
      ready[k].store(1, std::memory_order_release);
    }
  });
  int st = MPDPFT_OK;
  for (long k = 0; k < nchunk; ++k) {
    while (!ready[k].load(std::memory_order_acquire)) std::this_thread::yield();
    const long off = k * kCopyChunk, len = std::min(kCopyChunk, cnt - off);
    if (!st && cudaMemcpyAsync(dstage + off, hs + off, sizeof(T) * len, cudaMemcpyHostToDevice, c.stream) !=
                   cudaSuccess)
      st = set_error(MPDPFT_ERR_CUDA, "host to device copy");
  }
  P.wait();
  return st;
}

// cnt values of type T in device memory out to a caller's double array.
template <typename T>
static int stage_out(Ctx& c, double* dst, T* hs, const T* dsrc, long cnt) {
  const long nchunk = (cnt + kCopyChunk - 1) / kCopyChunk;
  while ((long)c.copy_events.size() < nchunk) {
    cudaEvent_t e;
    CU(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    c.copy_events.push_back(e);
  }
  for (long k = 0; k < nchunk; ++k) {
    const long off = k * kCopyChunk, len = std::min(kCopyChunk, cnt - off);
    CU(cudaMemcpyAsync(hs + off, dsrc + off, sizeof(T) * len, cudaMemcpyDeviceToHost, c.stream));
    CU(cudaEventRecord(c.copy_events[k], c.stream));
  }
  if (!c.copy_pool) c.copy_pool.reset(new CopyPool());
  CopyPool& P = *c.copy_pool;
  std::vector<std::atomic<int>> ready(nchunk);  // 1: copied to the host, 2: failed
  for (auto& r : ready) r.store(0);
  const int nt = P.nt;
  P.begin([&](int t) {
    for (long k = t; k < nchunk; k += nt) {
      int r;
      while (!(r = ready[k].load(std::memory_order_acquire))) std::this_thread::yield();
      if (r != 1) continue;
      const long off = k * kCopyChunk, len = std::min(kCopyChunk, cnt - off);
      unstage_chunk(dst + off, hs + off, len);
    }
  });
  int st = MPDPFT_OK;
  for (long k = 0; k < nchunk; ++k) {
    const bool ok = !st && cudaEventSynchronize(c.copy_events[k]) == cudaSuccess;
    if (!ok && !st) st = set_error(MPDPFT_ERR_CUDA, "device to host copy");
    ready[k].store(ok ? 1 : 2, std::memory_order_release);
  }
  P.wait();
  return st;
}

int Ctx::host_to_device(double* dstage, double* hs, const double* src, long cnt) {
  return stage_in<double>(*this, dstage, hs, src, cnt);
}

int Ctx::device_to_host(double* dst, double* hs, const double* dsrc, long cnt) {
  return stage_out<double>(*this, dst, hs, dsrc, cnt);
}

int Ctx::import_field(const double* src, void* dst, int layout, int mem, int slot, bool sync) {
  if (!src) return set_error(MPDPFT_ERR_ARG, "null input array");
  if (mem != MPDPFT_MEM_HOST) return import_staged(src, dst, layout, slot, sync);
  // host grids cross in chunks, copied and sent by several host threads
  const long cnt = layout == MPDPFT_LAYOUT_REFERENCE ? n_ref : geom.n;
  double* dstage = d_io + (slot ? std::max(n_ref, geom.n) : 0);  // d_io holds two grids
  int st;
  if (rsize == sizeof(float)) {  // FP32 fields: rounded on the host, half the bytes over the link
    float* fstage = reinterpret_cast<float*>(dstage);
    if ((st = stage_in<float>(*this, fstage, reinterpret_cast<float*>(host_stage(slot)), src, cnt))) return st;
    k_import<float, float><<<grid_blocks(geom.n), kThreads, 0, stream>>>(fstage, (float*)dst, geom, layout);
    CU(cudaGetLastError());
    if (sync) CU(cudaStreamSynchronize(stream));  // pinned buffer reuse
    return MPDPFT_OK;
  }
  if ((st = host_to_device(dstage, host_stage(slot), src, cnt))) return st;
  st = import_staged(dstage, dst, layout, slot, false);
  if (st) return st;
  if (sync) CU(cudaStreamSynchronize(stream));  // pinned buffer reuse
  return MPDPFT_OK;
}

// The device half of import_field: src (device) or, when src is null, the
// grid already copied into host_stage(slot).
int Ctx::import_staged(const double* src, void* dst, int layout, int slot, bool sync) {
  const long cnt = layout == MPDPFT_LAYOUT_REFERENCE ? n_ref : geom.n;
  const double* dsrc = src;
  const bool staged = src == nullptr;
  if (staged) {
    double* dstage = d_io + (slot ? std::max(n_ref, geom.n) : 0);  // d_io holds two grids
    CU(cudaMemcpyAsync(dstage, host_stage(slot), sizeof(double) * cnt, cudaMemcpyHostToDevice, stream));
    dsrc = dstage;
  }
  const int blocks = grid_blocks(geom.n);
  if (rsize == sizeof(double)) k_import<double><<<blocks, kThreads, 0, stream>>>(dsrc, (double*)dst, geom, layout);
  else k_import<float><<<blocks, kThreads, 0, stream>>>(dsrc, (float*)dst, geom, layout);
  CU(cudaGetLastError());
  if (staged && sync) CU(cudaStreamSynchronize(stream));  // pinned buffer reuse
  return MPDPFT_OK;
}

// One field of the current state (mpdpft_get_field): the input density of
// the current ring slot, V, V_ext, |grad V|^2 or the Laplacian of species s.
int Ctx::get_field(int which, int s, double* out, int layout, int mem) {
  if (s < 0 || s >= S) return set_error(MPDPFT_ERR_ARG, "species index out of range");
  const size_t off = (size_t)s * geom.n * rsize;
  const void* src = nullptr;
  if (which == MPDPFT_FIELD_DENSITY) {
    ScState h;
    int st = read_state(&h);
    if (st) return st;
    src = (char*)d_nin + (size_t)h.slot * S * geom.n * rsize + off;
  } else if (which == MPDPFT_FIELD_POTENTIAL) {
    src = (char*)d_V + off;
  } else if (which == MPDPFT_FIELD_EXTERNAL) {
    src = (char*)d_vext + off;
  } else if (which == MPDPFT_FIELD_GRAD2 && d_g2) {
    src = (char*)d_g2 + off;
  } else if (which == MPDPFT_FIELD_LAPLACIAN && d_lap) {
    src = (char*)d_lap + off;
  } else {
    return set_error(MPDPFT_ERR_ARG, "field not available");
  }
  return export_field(src, out, layout, mem);
}

int Ctx::export_field(const void* src, double* dst, int layout, int mem) {
  if (!dst) return set_error(MPDPFT_ERR_ARG, "null output array");
  const long cnt = layout == MPDPFT_LAYOUT_REFERENCE ? n_ref : geom.n;
  double* ddst = mem == MPDPFT_MEM_HOST ? d_io : dst;
  const int blocks = grid_blocks(cnt);
  if (mem == MPDPFT_MEM_HOST && rsize == sizeof(float)) {  // FP32 fields cross as floats
    float* fstage = reinterpret_cast<float*>(d_io);
    k_export<float, float><<<blocks, kThreads, 0, stream>>>((const float*)src, fstage, geom, layout);
    CU(cudaGetLastError());
    return stage_out<float>(*this, dst, reinterpret_cast<float*>(pinned), fstage, cnt);
  }
  if (rsize == sizeof(double)) k_export<double><<<blocks, kThreads, 0, stream>>>((const double*)src, ddst, geom, layout);
  else k_export<float><<<blocks, kThreads, 0, stream>>>((const float*)src, ddst, geom, layout);
  CU(cudaGetLastError());
  if (mem == MPDPFT_MEM_HOST) return device_to_host(dst, (double*)pinned, d_io, cnt);
  return MPDPFT_OK;
}

template <typename R>
StepArgs<R> Ctx::step_args(int mode) {
  StepArgs<R> a;
  std::memset(&a, 0, sizeof(a));
  a.kp = kparams();
  a.st = d_state;
  a.vext = (const R*)d_vext;
  a.V = (R*)d_V;
  a.lap = gradient ? (const R*)d_lap : nullptr;
  a.g2 = need_g2 ? (const R*)d_g2 : nullptr;
  a.vh = has_coulomb ? (const R*)d_vh : nullptr;
  a.nin = (R*)d_nin;
  a.res = (R*)d_res;
  a.cur_copy = (R*)d_cur;
  a.part = d_part;
  a.part2 = d_part2;
  a.bcount = d_bcount;
  a.plist = d_plist;
  a.plist_stride = plist_stride;
  a.vres_part = vres_part_ext;
  a.vres_blocks = vres_blocks_ext;
  a.log = d_log;
  a.log_cap = log_cap;
  a.assemble_v = assemble_in_step;
  a.mode = mode;
  a.split_d = 1;
  return a;
}

template StepArgs<double> Ctx::step_args<double>(int);
template StepArgs<float> Ctx::step_args<float>(int);

// parts: bit 0 mu kernel, bit 1 density kernel, bit 2 mixing kernel (a
// mode still runs only the kernels it has)
template <typename R>
static cudaError_t launch_sc_kernels(Ctx& c, int mode, int fk, int parts = 7) {
  StepArgs<R> args = c.step_args<R>(mode);
  void* params[] = {&args};
  // algorithmic bytes per species: the fields each kernel reads and writes,
  // once (the mu search counts one sweep whatever its passes)
  const double fb = c.field_bytes() * c.S;
  const double deriv = (args.lap ? 1.0 : 0.0) + (args.g2 ? 1.0 : 0.0);
  const double m = c.P.mixer ? c.P.pulay_scope : 1;
  if (c.noting) {
    if (mode != 2 && (parts & 1))
      c.note("sc_mu_kernel", ((mode == 0 && args.assemble_v) ? 4.0 * fb : 0.0) + (1.0 + deriv) * fb);
    if (parts & 2) {
      // V, derivatives, n_in, m - 1 history residuals in; the residual out
      c.note("sc_density_kernel", (2.0 + deriv + m) * fb);
      c.note("sc_phase_d_kernel", (double)c.dens_blocks * kNPart * sizeof(double));
    }
    // m input densities and residuals in; the next density and its copy out
    if (mode != 1 && (parts & 4)) c.note("sc_mix_kernel", (2.0 * m + 2.0) * fb);
  }
  if (mode != 2 && (parts & 1)) {
    cudaLaunchConfig_t cfg;
    std::memset(&cfg, 0, sizeof(cfg));
    cfg.gridDim = dim3(c.step_blocks);
    cfg.blockDim = dim3(kStepThreads);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = c.stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    c.cnt[MPDPFT_STAGE_SC_STEP]++;
    cudaError_t e = cudaLaunchKernelExC(&cfg, sc_kernel_ptr<R>(0, fk), params);
    if (e != cudaSuccess) return e;
  }
  cudaError_t e = cudaSuccess;
  if (parts & 2) {
    c.cnt[MPDPFT_STAGE_SC_STEP]++;
    {
      cudaLaunchConfig_t dc;
      std::memset(&dc, 0, sizeof(dc));
      dc.gridDim = dim3(c.dens_blocks);
      dc.blockDim = dim3(kDensityThreads);
      dc.stream = c.stream;
      cudaLaunchAttribute pa[1];
      pa[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
      pa[0].val.programmaticStreamSerializationAllowed = 1;
      dc.attrs = pa;
      dc.numAttrs = pdl_enabled() ? 1 : 0;
      e = cudaLaunchKernelExC(&dc, sc_kernel_ptr<R>(c.dens_which, fk), params);
    }
    if (e != cudaSuccess) return e;
    c.cnt[MPDPFT_STAGE_SC_STEP]++;
    const int nb = c.dens_blocks;
    if (c.dens_which == 1) e = launch_k(sc_phase_d_kernel<R, 5>, dim3(1), dim3(kDensityThreads), 0, c.stream, args, nb);
    else if (c.dens_which == 3) e = launch_k(sc_phase_d_kernel<R, 8>, dim3(1), dim3(kDensityThreads), 0, c.stream, args, nb);
    else e = launch_k(sc_phase_d_kernel<R, kMaxP>, dim3(1), dim3(kDensityThreads), 0, c.stream, args, nb);
    if (e != cudaSuccess) return e;
  }
  if (mode != 1 && (parts & 4)) {
    c.cnt[MPDPFT_STAGE_SC_STEP]++;
    e = launch_k(sc_mix_kernel<R>, dim3(c.mix_blocks), dim3(kDensThreads), 0, c.stream, args);
  }
  return e;
}

// One SC iteration's kernels (mode 0), the densities of the current V
// (mode 1: mu kernel + density kernel) or the admix step alone (mode 2:
// density kernel + mixing kernel).
int Ctx::launch_step(int mode, int parts) {
  cudaError_t e = rsize == sizeof(double) ? launch_sc_kernels<double>(*this, mode, fk, parts)
                                          : launch_sc_kernels<float>(*this, mode, fk, parts);
  if (e != cudaSuccess) return set_error(MPDPFT_ERR_CUDA, std::string("SC kernel launch: ") + cudaGetErrorString(e));
  return MPDPFT_OK;
}

// Everything of one SC iteration, issued on the stream (graph-capturable).
int Ctx::issue_iteration() {
  int st;
  if (has_coulomb || gradient) {
    if ((st = issue_fft_terms())) return st;
  }
  return launch_step(0);
}

int Ctx::status_from_state(const ScState& h) {
  if (h.abort) return set_error(MPDPFT_ERR_TIMEOUT, "grid barrier timed out in the SC step kernel");
  return MPDPFT_OK;
}

int Ctx::sc_init(const double* const* v0, int layout, int mem, bool check) {
  int st;
  if ((st = reset_state())) return st;
  for (int s = 0; s < S; ++s) {
    void* dst = (char*)d_V + (size_t)s * geom.n * rsize;
    if (v0 && v0[s]) {
      if ((st = import_field(v0[s], dst, layout, mem))) return st;
    } else {
      CU(cudaMemcpyAsync(dst, (char*)d_vext + (size_t)s * geom.n * rsize, geom.n * rsize,
                         cudaMemcpyDeviceToDevice, stream));
    }
  }
  // automatic temperature (PreparationsForSCdensity, mpDPFT.cpp:4523-4528)
  // (every solve takes its own from its V_0)
  bool need_t = false;
  for (int s = 0; s < S; ++s) need_t |= P.temperature[s] < 0.0;
  if (need_t) {
    std::vector<double> h(geom.n);
    for (int s = 0; s < S; ++s) {
      if (P.temperature[s] >= 0.0) continue;
      if ((st = export_field((char*)d_V + (size_t)s * geom.n * rsize, h.data(), MPDPFT_LAYOUT_PERIODIC, MPDPFT_MEM_HOST))) return st;
      double vmin = h[0], vmax = h[0];
      for (double x : h) { vmin = std::min(vmin, x); vmax = std::max(vmax, x); }
      temperature[s] = std::max(std::fabs(P.mu[s] - vmin), std::fabs(P.mu[s] - vmax)) / 50.0;
    }
  }
  if (gradient) {
    if ((st = issue_delfield_of_V())) return st;
  }
  if ((st = launch_step(1))) return st;  // initial densities (mpDPFT.cpp:195)
  initialised = true;
  if (!check) return MPDPFT_OK;
  ScState h;
  if ((st = read_state(&h))) return st;  // (synchronises the stream)
  return status_from_state(h);
}

void Ctx::drop_graphs() {
  if (graph_exec) { cudaGraphExecDestroy(graph_exec); graph_exec = nullptr; }
  if (graph) { cudaGraphDestroy(graph); graph = nullptr; }
  if (loop_exec) { cudaGraphExecDestroy(loop_exec); loop_exec = nullptr; }
  if (loop_graph) { cudaGraphDestroy(loop_graph); loop_graph = nullptr; }
  if (loop_state > 0) loop_state = 0;
}

// The captured graphs hold the kernel parameters by value; the only ones
// that change after context creation are the automatic temperatures (set
// per solve from V_0) and the device loop limits, so a graph is kept while
// kparams() is what it was captured with.
void Ctx::check_graphs() {
  if (!graph_exec && !loop_exec) return;
  const KParams k = kparams();
  if (std::memcmp(&k, &graph_kp, sizeof(k)) != 0) drop_graphs();
}

// Last node of the device-side loop's body: loop again unless the exit test
// has been met, a kernel aborted, or `cap` iterations have run.
__global__ void k_loop_cond(cudaGraphConditionalHandle h, const ScState* st, int cap) {
  const bool stop = __ldcg(&st->exit_loop) != 0 || __ldcg(&st->abort) != 0 || __ldcg(&st->sc_count) >= cap;
  cudaGraphSetConditional(h, stop ? 0u : 1u);
}

// The SC loop as one graph: a WHILE node whose body is one captured
// iteration followed by k_loop_cond, so a solve runs without host round
// trips between iterations.  Where the driver cannot build or instantiate
// it (loop_state -1), sc_run replays the one-iteration graph from the host.
int Ctx::build_loop() {
  check_graphs();
  if (loop_exec || loop_state < 0) return MPDPFT_OK;
  cudaGraph_t g = nullptr;
  cudaGraphConditionalHandle h = 0;
  cudaGraphNode_t node = nullptr;
  cudaGraphNodeParams cp = {cudaGraphNodeTypeConditional};
  cudaError_t e = cudaGraphCreate(&g, 0);
  if (e == cudaSuccess) e = cudaGraphConditionalHandleCreate(&h, g, 1u, cudaGraphCondAssignDefault);
  if (e == cudaSuccess) {
    cp.conditional.handle = h;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    e = cudaGraphAddNode(&node, g, nullptr, 0, &cp);
  }
  cudaGraph_t body = e == cudaSuccess ? cp.conditional.phGraph_out[0] : nullptr;
  if (e == cudaSuccess) e = cudaStreamBeginCaptureToGraph(stream, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal);
  if (e != cudaSuccess) {
    if (g) cudaGraphDestroy(g);
    cudaGetLastError();
    loop_state = -1;
    return MPDPFT_OK;
  }
  const KParams k = kparams();
  int st = issue_iteration();
  if (st == MPDPFT_OK) {
    k_loop_cond<<<1, 1, 0, stream>>>(h, d_state, P.max_sc_count + 3);
    if (cudaGetLastError() != cudaSuccess) st = -1;
  }
  cudaGraph_t out = nullptr;
  e = cudaStreamEndCapture(stream, &out);
  if (st == MPDPFT_OK && e == cudaSuccess) e = cudaGraphInstantiate(&loop_exec, g, 0);
  // any failure here (a launch the driver does not take inside a loop body,
  // say) leaves the host-driven loop, which reports real errors itself
  if (st != MPDPFT_OK || e != cudaSuccess || !loop_exec) {
    cudaGraphDestroy(g);
    cudaGetLastError();
    loop_exec = nullptr;
    loop_state = -1;
    g_last_error.clear();
    return MPDPFT_OK;
  }
  loop_graph = g;
  loop_state = 1;
  graph_kp = k;
  return MPDPFT_OK;
}

int Ctx::sc_step(int use_graph) {
  if (!initialised) return set_error(MPDPFT_ERR_ARG, "sc_init has not been called");
  int st;
  if (!use_graph) return issue_iteration();
  check_graphs();
  if (!graph_exec) {
    graph_kp = kparams();
    // a driver that does not take the programmatic launches inside a
    // captured graph gets the iteration captured again without them
    for (int attempt = 0;; ++attempt) {
      CU(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
      for (int i = 0; i < 6; ++i) cnt[i] = 0;
      notes.clear();
      noting = true;
      st = issue_iteration();
      noting = false;
      for (int i = 0; i < 6; ++i) iter_cnt[i] = cnt[i];
      cudaGraph_t g = nullptr;
      cudaError_t e = cudaStreamEndCapture(stream, &g);
      if (st == MPDPFT_OK && e == cudaSuccess) e = cudaGraphInstantiate(&graph_exec, g, 0);
      if (st == MPDPFT_OK && e == cudaSuccess) { graph = g; break; }
      if (g) cudaGraphDestroy(g);
      graph_exec = nullptr;
      if (attempt == 0 && pdl_enabled()) {
        cudaGetLastError();
        g_last_error.clear();
        pdl_disable();
        continue;
      }
      if (st) return st;
      return set_error(MPDPFT_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(e));
    }
  }
  CU(cudaGraphLaunch(graph_exec, stream));
  return MPDPFT_OK;
}

void Ctx::note(const char* name, double bytes) {
  if (!noting) return;
  LaunchNote r;
  std::memset(&r, 0, sizeof(r));
  std::strncpy(r.name, name, sizeof(r.name) - 1);
  r.bytes = bytes;
  notes.push_back(r);
}

// One SC iteration replayed node by node from the captured graph (dependency
// order; a stream capture is a chain), each node as a one-node graph with the
// kernel's launch attributes (the mu kernel stays cooperative), timed with
// CUDA events on the context stream.
int Ctx::iteration_profile(int cap, mpdpft_launch_record* out, int* n_out) {
  if (!graph) return set_error(MPDPFT_ERR_ARG, "no captured iteration (run one graph-mode mpdpft_sc_step first)");
  size_t nn = 0;
  CU(cudaGraphGetNodes(graph, nullptr, &nn));
  std::vector<cudaGraphNode_t> nodes(nn);
  CU(cudaGraphGetNodes(graph, nodes.data(), &nn));
  // topological order: repeatedly take the nodes whose dependencies are taken
  std::vector<cudaGraphNode_t> order;
  std::vector<char> done(nn, 0);
  while (order.size() < nn) {
    bool progress = false;
    for (size_t i = 0; i < nn; ++i) {
      if (done[i]) continue;
      // (the edge-data form: programmatic edges refuse the plain query)
      size_t nd = 0;
      CU(cudaGraphNodeGetDependencies_v2(nodes[i], nullptr, nullptr, &nd));
      std::vector<cudaGraphNode_t> deps(nd);
      std::vector<cudaGraphEdgeData> edata(nd);
      if (nd) CU(cudaGraphNodeGetDependencies_v2(nodes[i], deps.data(), edata.data(), &nd));
      bool ready = true;
      for (cudaGraphNode_t d : deps) {
        size_t j = 0;
        while (j < nn && nodes[j] != d) ++j;
        if (j < nn && !done[j]) ready = false;
      }
      if (!ready) continue;
      done[i] = 1;
      order.push_back(nodes[i]);
      progress = true;
    }
    if (!progress) return set_error(MPDPFT_ERR_CUDA, "captured iteration has a dependency cycle");
  }
  if (order.size() != notes.size())
    return set_error(MPDPFT_ERR_CUDA, "captured iteration: " + std::to_string(order.size()) + " nodes, " +
                                          std::to_string(notes.size()) + " recorded launches");
  cudaEvent_t ev0, ev1;
  CU(cudaEventCreate(&ev0));
  CU(cudaEventCreate(&ev1));
  int st = MPDPFT_OK;
  int k = 0;
  for (size_t i = 0; i < order.size() && st == MPDPFT_OK; ++i) {
    cudaGraphNodeType type;
    if (cudaGraphNodeGetType(order[i], &type) != cudaSuccess) { st = set_error(MPDPFT_ERR_CUDA, "node type"); break; }
    cudaGraph_t g1 = nullptr;
    cudaGraphExec_t x1 = nullptr;
    cudaGraphNode_t n1 = nullptr;
    cudaError_t e = cudaGraphCreate(&g1, 0);
    if (e == cudaSuccess && type == cudaGraphNodeTypeKernel) {
      cudaKernelNodeParams kp;
      e = cudaGraphKernelNodeGetParams(order[i], &kp);
      if (e == cudaSuccess) e = cudaGraphAddKernelNode(&n1, g1, nullptr, 0, &kp);
      if (e == cudaSuccess) e = cudaGraphKernelNodeCopyAttributes(n1, order[i]);
    } else if (e == cudaSuccess && type == cudaGraphNodeTypeMemset) {
      cudaMemsetParams mp;
      e = cudaGraphMemsetNodeGetParams(order[i], &mp);
      if (e == cudaSuccess) e = cudaGraphAddMemsetNode(&n1, g1, nullptr, 0, &mp);
    } else if (e == cudaSuccess) {
      e = cudaErrorNotSupported;
    }
    if (e == cudaSuccess) e = cudaGraphInstantiate(&x1, g1, 0);
    if (e == cudaSuccess) e = cudaEventRecord(ev0, stream);
    if (e == cudaSuccess) e = cudaGraphLaunch(x1, stream);
    if (e == cudaSuccess) e = cudaEventRecord(ev1, stream);
    if (e == cudaSuccess) e = cudaEventSynchronize(ev1);
    float ms = 0.f;
    if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, ev0, ev1);
    if (x1) cudaGraphExecDestroy(x1);
    if (g1) cudaGraphDestroy(g1);
    if (e != cudaSuccess) { st = set_error(MPDPFT_ERR_CUDA, std::string("iteration profile: ") + cudaGetErrorString(e)); break; }
    if (k < cap && out) {
      std::memset(&out[k], 0, sizeof(out[k]));
      std::strncpy(out[k].name, notes[i].name, sizeof(out[k].name) - 1);
      out[k].ms = ms;
      out[k].bytes = notes[i].bytes;
    }
    ++k;
  }
  cudaEventDestroy(ev0);
  cudaEventDestroy(ev1);
  if (n_out) *n_out = k;
  if (st) return st;
  ScState h;
  if ((st = read_state(&h))) return st;
  return status_from_state(h);
}

int Ctx::sc_run(mpdpft_result* result, mpdpft_iter_log* log, int cap, int use_graph) {
  auto t0 = std::chrono::steady_clock::now();
  int st;
  ScState h;
  bool looped = false;
  if (use_graph) {
    if (!initialised) return set_error(MPDPFT_ERR_ARG, "sc_init has not been called");
    if ((st = build_loop())) return st;
    if (loop_exec) {
      CU(cudaGraphLaunch(loop_exec, stream));
      if ((st = read_state(&h))) return st;
      if ((st = status_from_state(h))) return st;
      looped = true;
    }
  }
  const int chunk = 4;
  int issued = 0;
  while (!looped) {
    for (int c = 0; c < chunk; ++c, ++issued)
      if ((st = sc_step(use_graph))) return st;
    CU(cudaStreamSynchronize(stream));
    if ((st = read_state(&h))) return st;
    if ((st = status_from_state(h))) return st;
    if (h.exit_loop || issued > P.max_sc_count + 2) break;
  }
  auto t1 = std::chrono::steady_clock::now();
  if (result) {
    std::memset(result, 0, sizeof(*result));
    if ((st = fill_result(result, h))) return st;
    result->seconds = std::chrono::duration<double>(t1 - t0).count();
    result->device_loop = looped ? 1 : 0;
  }
  if (log && cap > 0) {
    int nlog = std::min(cap, std::min(h.sc_count, log_cap));
    CU(cudaMemcpy(log, d_log, sizeof(mpdpft_iter_log) * nlog, cudaMemcpyDeviceToHost));
  }
  if (h.status_bits & kBitTimeout) return set_error(MPDPFT_ERR_TIMEOUT, "mu search reached its pass cap");
  if (!h.exit_loop || h.exit_count < 3) return set_error(MPDPFT_ERR_NOT_CONVERGED, "maxSCcount reached");
  return MPDPFT_OK;
}

int Ctx::fill_result(mpdpft_result* r, const ScState& h) {
  r->iterations = h.sc_count;
  r->converged = h.exit_count >= 3 ? 1 : 0;
  r->total_mu_trials = h.mu_passes_total;
  r->cc = h.cc;
  r->v_residual = h.v_res;
  for (int s = 0; s < S; ++s) { r->mu[s] = h.mu[s]; r->abundance[s] = h.ab[s]; }
  return energy(r, h);
}

// Energies of the current state (GetEnergy, mpDPFT.cpp:5414-5436): the
// densities are the mixed densities of the last iteration, V and mu those
// of the last density evaluation, as in the reference's ExportData.
// energy_issue leaves the kNEnergy integrals (times dvol) at e_dev on the
// stream; energy_finish forms the energies from them on the host.
template <typename R>
void Ctx::launch_energy(int blocks, const void* dens, const double* d_mu) {
  const R* vh = has_coulomb ? (const R*)d_vh : nullptr;
  auto go = [&](auto kern) {
    kern<<<blocks, kThreads, 0, stream>>>(geom, (const R*)d_V, (const R*)d_vext, (const R*)dens, vh, d_mu, d_part);
  };
  if (S == 1) go(k_energy<R, 1>);
  else if (S == 2) go(k_energy<R, 2>);
  else if (S == 3) go(k_energy<R, 3>);
  else go(k_energy<R, 4>);
}

int Ctx::energy_issue(const ScState& h, double* e_dev, bool g2_current) {
  int st;
  double* d_mu = d_io;  // scratch: mu of the state h was read from (still on the device)
  CU(cudaMemcpyAsync(d_mu, d_state->mu, sizeof(double) * kMaxS, cudaMemcpyDeviceToDevice, stream));
  const void* dens = (char*)d_nin + (size_t)h.slot * S * geom.n * rsize;
  if (gradient && geom.dim == 2 && !need_g2 && !g2_current) {
    // the 2D kinetic energy reads |grad V|^2, which the iterations' DelField
    // leaves out (the 2D density does not use it)
    need_g2 = true;
    st = issue_delfield_of_V();
    need_g2 = false;
    if (st) return st;
  }
  if (has_coulomb) {
    if ((st = issue_coulomb(dens, d_vh, /*for_energy=*/1))) return st;
  }
  const int blocks = grid_blocks(geom.n);
  if (rsize == sizeof(double)) launch_energy<double>(blocks, dens, d_mu);
  else launch_energy<float>(blocks, dens, d_mu);
  k_sum_rows<<<kNEnergy, kThreads, 0, stream>>>(d_part, blocks, kNEnergy, geom.dvol, e_dev);
  CU(cudaGetLastError());
  if (gradient) return ekin_issue(dens, d_mu, e_dev, 4, e_dev + kEkinOff);
  return MPDPFT_OK;
}

// Kinetic integrals of the gradient-corrected density (k_ekin_grad) with
// inner trapezoid cap maxit: 2 kMaxS values (times dvol) to out; mu and
// e_dev (int V_ext n at [5 s + 1]) on the device.
int Ctx::ekin_issue(const void* dens, const double* d_mu, const double* e_dev, int maxit, double* out) {
  const int blocks = grid_blocks(geom.n);
  const double thr = finite_t ? std::fabs(P.airy_threshold) : 1.0e300;
  const double area_pref = std::pow(P.edge, (double)P.dim) * P.degeneracy / (4.0 * kPi * kPi);
  if (rsize == sizeof(double))
    k_ekin_grad<double><<<blocks, kThreads, 0, stream>>>(geom, S, P.degeneracy, thr, maxit, P.internal_acc, area_pref,
                                                          (const double*)d_V, (const double*)d_lap, (const double*)d_g2,
                                                          (const double*)dens, d_mu, e_dev, d_part);
  else
    k_ekin_grad<float><<<blocks, kThreads, 0, stream>>>(geom, S, P.degeneracy, thr, maxit, P.internal_acc, area_pref,
                                                        (const float*)d_V, (const float*)d_lap, (const float*)d_g2,
                                                        (const float*)dens, d_mu, e_dev, d_part);
  k_sum_rows<<<2 * kMaxS, kThreads, 0, stream>>>(d_part, blocks, 2 * kMaxS, geom.dvol, out);
  CU(cudaGetLastError());
  return MPDPFT_OK;
}

int Ctx::energy(mpdpft_result* r, const ScState& h) {
  int st;
  double* e_dev = d_io + kMaxS;
  if ((st = energy_issue(h, e_dev))) return st;
  double E[kNEnergy];
  CU(cudaMemcpyAsync(E, e_dev, sizeof(E), cudaMemcpyDeviceToHost, stream));
  CU(cudaStreamSynchronize(stream));
  if (gradient && geom.dim == 3 && finite_t) {
    // EkinAiT03D's outer loop (mpDPFT.cpp:5651-5700): the Airy-weighted
    // integrals again with MaxIteration 5 .. 10 until a species' kinetic
    // integral agrees with the previous one to max(RelAcc, MP)
    const void* dens = (char*)d_nin + (size_t)h.slot * S * geom.n * rsize;
    double* e2 = e_dev + kNEnergy;  // scratch beside the integrals
    bool done[kMaxS] = {false, false, false, false};
    for (int maxit = 5; maxit <= 10; ++maxit) {
      if ((st = ekin_issue(dens, d_io, e_dev, maxit, e2))) return st;
      double K[2 * kMaxS];
      CU(cudaMemcpyAsync(K, e2, sizeof(K), cudaMemcpyDeviceToHost, stream));
      CU(cudaStreamSynchronize(stream));
      bool all = true;
      for (int s = 0; s < S; ++s) {
        if (done[s]) continue;
        const double a = K[s], b = E[kEkinOff + s];
        const double d = (a == 0.0 && b == 0.0) ? 0.0 : std::fabs((a - b) / (a + b));
        E[kEkinOff + s] = a;
        if (d < std::max(P.rel_acc, 1.0e-12)) done[s] = true;
        else all = false;
      }
      if (all) break;
    }
  }
  energy_finish(r, E);
  return MPDPFT_OK;
}

void Ctx::energy_finish(mpdpft_result* r, const double* E) {
  const double D = P.dim;
  double etot = 0.0;
  for (int a = 0; a < P.n_interactions; ++a) {
    const int t = P.interactions[a];
    double e = 0.0;
    if (t == MPDPFT_INT_CONTACT_MUTUAL) {
      for (int s = 0; s < S; ++s)
        for (int q = s + 1; q < S; ++q) e += E[5 * kMaxS + s * kMaxS + q];
      e *= P.beta;
    } else if (t == MPDPFT_INT_CONTACT_SELF) {
      e = P.beta * E[2];
    } else if (t == MPDPFT_INT_HARTREE || t == MPDPFT_INT_HARTREE_INTER || t == MPDPFT_INT_COULOMB_CHARGED) {
      for (int s = 0; s < S; ++s) e += E[5 * s + 4];
    } else if (t == MPDPFT_INT_DIRAC) {
      const double cXD = 2.0 * std::sqrt(4.0 * kPi) / ((D - 1.0) * kPi) *
                         std::pow(0.5 * std::pow(0.75 * std::sqrt(kPi), D - 2.0), 1.0 / D);
      for (int s = 0; s < S; ++s) e += -P.gamma_h * cXD * D / (1.0 + D) * E[5 * s + 3];
    }
    r->e_interaction[a] = e;
    etot += e;
  }
  const double AF = P.dim == 2 ? 2.0 * kPi : 4.0 * kPi;
  for (int s = 0; s < S; ++s) {
    double ekin;
    if (P.dim == 2 && (P.density_expression == MPDPFT_DENS_TF_INSPIRED ||
                       P.density_expression == MPDPFT_DENS_TF_INSPIRED_T))
      ekin = 0.5 * P.tau[s] * E[5 * s + 2];
    else if (P.density_expression == MPDPFT_DENS_GRADIENT && P.dim == 2)  // E1 - int V n + mu N (:5608-5621)
      ekin = E[kEkinOff + s] - E[kEkinOff + kMaxS + s] + r->mu[s] * r->abundance[s];
    else if (P.density_expression == MPDPFT_DENS_GRADIENT)  // EkinAiT03D (:5647-5703)
      ekin = P.degeneracy / (4.0 * kPi * kPi) * E[kEkinOff + s];
    else
      ekin = P.degeneracy * AF * std::pow(2.0, (D + 2.0) / 2.0) / (std::pow(2.0 * kPi, D) * (2.0 * D + 4.0)) *
             E[5 * s + 0];
    r->e_kinetic[s] = ekin;
    r->e_external[s] = E[5 * s + 1];
    etot += ekin + E[5 * s + 1];
  }
  r->e_total = etot;
}

// -------------------------------------------------- standalone operators --
int Ctx::op_mu_search(int s, const double* v, double target, double* mu_io, double* ab_out, int* trials,
                      double* n_out, int layout, int mem) {
  if (s < 0 || s >= S) return set_error(MPDPFT_ERR_ARG, "species index out of range");
  int st;
  if ((st = reset_state())) return st;
  // the kernel searches every species; others get their own target N from
  // P and the same V, which is harmless (only species s is reported)
  for (int q = 0; q < S; ++q)
    if ((st = import_field(v, (char*)d_V + (size_t)q * geom.n * rsize, layout, mem))) return st;
  ScState h;
  if ((st = read_state(&h))) return st;
  for (int q = 0; q < S; ++q) h.mu[q] = *mu_io;
  P.abundances[s] = target;
  CU(cudaMemcpyAsync(d_state, &h, sizeof(h), cudaMemcpyHostToDevice, stream));
  if (gradient && (st = issue_delfield_of_V())) return st;
  if ((st = launch_step(1))) return st;
  CU(cudaStreamSynchronize(stream));
  if ((st = read_state(&h))) return st;
  if ((st = status_from_state(h))) return st;
  *mu_io = h.mu[s];
  if (ab_out) *ab_out = h.ab[s];
  if (trials) *trials = h.mu_passes;
  if (n_out) {
    const void* src = (char*)d_nin + ((size_t)h.slot * S + s) * geom.n * rsize;
    if ((st = export_field(src, n_out, layout, mem))) return st;
  }
  if (h.status_bits & kBitBracket) return set_error(MPDPFT_ERR_MU_BRACKET, "mu bracket not found; mu reset");
  if (h.status_bits & kBitTimeout) return set_error(MPDPFT_ERR_TIMEOUT, "mu search reached its pass cap");
  if (h.status_bits & kBitTrapped)
    return set_error(MPDPFT_WARN_MU_TRAPPED, "mu search trapped at a step of N(mu) (TrappedQ); mu and N are its end point");
  return MPDPFT_OK;
}

int Ctx::op_density(int s, const double* v, double mu, double* n_out, double* ab_out, int layout, int mem) {
  if (s < 0 || s >= S) return set_error(MPDPFT_ERR_ARG, "species index out of range");
  int st;
  void* Vs = (char*)d_V + (size_t)s * geom.n * rsize;
  if ((st = import_field(v, Vs, layout, mem))) return st;
  if (gradient && (st = issue_delfield_of_V())) return st;
  DensParams d = kparams().dens[s];
  const int blocks = grid_blocks(geom.n);
  void* lap = gradient ? (char*)d_lap + (size_t)s * geom.n * rsize : nullptr;
  void* g2 = gradient ? (char*)d_g2 + (size_t)s * geom.n * rsize : nullptr;
  if (rsize == sizeof(double))
    k_density<double><<<blocks, kThreads, 0, stream>>>(geom, d, mu, (const double*)Vs, (const double*)lap,
                                                        (const double*)g2, (double*)d_tmp);
  else
    k_density<float><<<blocks, kThreads, 0, stream>>>(geom, d, mu, (const float*)Vs, (const float*)lap,
                                                      (const float*)g2, (float*)d_tmp);
  CU(cudaGetLastError());
  if (ab_out && (st = integrate_device(d_tmp, ab_out))) return st;
  if (n_out && (st = export_field(d_tmp, n_out, layout, mem))) return st;
  return MPDPFT_OK;
}

int Ctx::integrate_device(const void* f, double* out) {
  const int blocks = grid_blocks(geom.n);
  if (rsize == sizeof(double)) k_integrate<double><<<blocks, kThreads, 0, stream>>>(geom, (const double*)f, d_part);
  else k_integrate<float><<<blocks, kThreads, 0, stream>>>(geom, (const float*)f, d_part);
  CU(cudaGetLastError());
  std::vector<double> hp(blocks);
  CU(cudaMemcpyAsync(hp.data(), d_part, sizeof(double) * blocks, cudaMemcpyDeviceToHost, stream));
  CU(cudaStreamSynchronize(stream));
  double t = 0.0;
  for (double x : hp) t += x;
  *out = t * geom.dvol;
  return MPDPFT_OK;
}

int Ctx::op_integrate(const double* f, double* out, int layout, int mem) {
  int st;
  if (!f) return set_error(MPDPFT_ERR_ARG, "null input array");
  if (layout == MPDPFT_LAYOUT_REFERENCE) {
    // every stored point with the reference's weights, duplicate planes included
    const double* src = f;
    if (mem == MPDPFT_MEM_HOST) {
      std::memcpy(host_stage(0), f, sizeof(double) * n_ref);
      CU(cudaMemcpyAsync(d_io, host_stage(0), sizeof(double) * n_ref, cudaMemcpyHostToDevice, stream));
      src = d_io;
    }
    const int blocks = grid_blocks(n_ref);
    k_integrate_ref<<<blocks, kThreads, 0, stream>>>(geom, src, d_part);
    CU(cudaGetLastError());
    std::vector<double> hp(blocks);
    CU(cudaMemcpyAsync(hp.data(), d_part, sizeof(double) * blocks, cudaMemcpyDeviceToHost, stream));
    CU(cudaStreamSynchronize(stream));
    double t = 0.0;
    for (double x : hp) t += x;
    *out = t * geom.dvol;
    return MPDPFT_OK;
  }
  if ((st = import_field(f, d_tmp, layout, mem))) return st;
  return integrate_device(d_tmp, out);
}

int Ctx::op_admix(const double* const* n_in, const double* const* n_out, const double* theta, double* const* n_mixed,
                  double* coeffs, int* ncoeff, int layout, int mem) {
  int st;
  ScState h;
  if ((st = read_state(&h))) return st;
  const int cur = h.slot;
  for (int s = 0; s < S; ++s) {
    void* dst = (char*)d_nin + ((size_t)cur * S + s) * geom.n * rsize;
    if ((st = import_field(n_in[s], dst, layout, mem))) return st;
    void* dv = (char*)d_V + (size_t)s * geom.n * rsize;  // n_out staged in V
    if ((st = import_field(n_out[s], dv, layout, mem))) return st;
    if (theta) { h.theta[s] = theta[s]; }
  }
  h.ab[0] = h.ab[0];
  CU(cudaMemcpyAsync(d_state, &h, sizeof(h), cudaMemcpyHostToDevice, stream));
  admix_only = true;
  st = launch_step(2);
  admix_only = false;
  if (st) return st;
  CU(cudaStreamSynchronize(stream));
  if ((st = read_state(&h))) return st;
  if ((st = status_from_state(h))) return st;
  for (int s = 0; s < S; ++s) {
    const void* src = (char*)d_nin + ((size_t)h.slot * S + s) * geom.n * rsize;
    if ((st = export_field(src, n_mixed[s], layout, mem))) return st;
  }
  if (ncoeff) *ncoeff = h.ncoeff;
  if (coeffs)
    for (int i = 0; i < h.ncoeff; ++i) coeffs[i] = h.coeff[i];
  if (h.iter_bits & kBitPulay) return set_error(MPDPFT_ERR_PULAY_SINGULAR, "Pulay Gram matrix rejected; linear mixing");
  return MPDPFT_OK;
}

}  // namespace mpdpft
