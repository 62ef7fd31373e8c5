// sc_step.cuh -- one SC iteration of the DPFT loop as a persistent kernel.
//
// The reference iteration (GetData loop, mpDPFT.cpp:213-224) is
//   StoreCurrentIteration; UpdateV; GetDensities (n[V] + EnforceConstraints);
//   CheckConvergence; Intercept; AdmixDensities; InjectSchedule;
//   PrepareNextIteration.
// Every step that is pointwise or a reduction runs here, in one cooperative
// launch whose phases are separated by bounded grid barriers; the scalar
// logic (mu decisions, convergence test, Pulay solve, schedules) runs on
// block 0 and lives in device memory, so an iteration needs no host
// synchronisation and can be captured in a CUDA graph.  FFT-based terms
// (Hartree, DelField) are produced by the FFT kernels before this launch.
#pragma once
#include <cstddef>

#include "common.cuh"

namespace mpdpft {

constexpr int kStepThreads = 512;
constexpr int kMuAcc = kMuCand + 1;  // candidate sums + dN/dmu at candidate 0
constexpr int kNF = 4 + kMaxP;        // per-species sums of the density/Gram pass
constexpr int kNPart = kMaxS * kNF > kMaxS * kMuAcc ? kMaxS * kNF : kMaxS * kMuAcc;
constexpr long kBarrierSpinLimit = 20000000;  // ~ seconds with nanosleep backoff

// Constant parameters of one solve (kernel argument, by value).
struct KParams {
  Geom geom;
  int S;
  DensParams dens[kMaxS];
  double abundance[kMaxS];
  double rel_acc;
  double beta, gamma_h;
  double charges[kMaxS];
  int contact_self, contact_mutual, dirac;  // pointwise V_int terms present
  int has_coulomb;                          // vh holds the Coulomb terms
  int mixer, scope, ring;                   // ring = scope + 1 slots
  double sc_criterion;
  int max_sc;
  int schedule;
  double pot_tol;
  double inc_v0;
};

struct MuState {
  double start, prev_abs, delta0, delta1, lo, hi, Nlo, Nhi;
  int have_lo, have_hi, done, active, pass;
  int ncand;
  int dir;     // -1: N(start) > N*, step down; +1: step up (reference order)
  int next_c;  // next reference bracket step to place
  double cand[kMuCand];
  double best_mu, best_N, best_err;
  double dens_mu;  // mu at which the final density is evaluated
  double step;     // size of the last Newton step
  double last_mu, last_N;     // last bracket-step position and its N
  double cand_prev0, N_prev0; // candidate 0 of the evaluated pass and its N
};

// SC loop state, resident in device memory.
struct ScState {
  double mu[kMaxS], prev_mu[kMaxS], old_mu[kMaxS];
  double ab[kMaxS], old_ab[kMaxS];
  double theta[kMaxS], theta0[kMaxS], theta_mix[kMaxS];
  double dmm, cc, old_cc, inc_v, v_res;
  int sc_count, exit_count, exit_loop, halted;
  int status_bits, iter_bits;
  int slot;      // ring slot of the current input density
  int mix_src;   // slot the last mix read from
  int hist;      // Pulay history length
  int pulay_used;
  int ncoeff;
  double gram[kMaxP * kMaxP];
  double coeff[kMaxP];
  int mu_passes;
  int mu_passes_total;
  MuState ms[kMaxS];
  unsigned bar_count, bar_gen;
  int abort;
  unsigned long long tphase[8];  // %globaltimer at phase boundaries (block 0)
};

template <typename R>
struct StepArgs {
  KParams kp;
  ScState* st;
  const R* vext;  // [S][n]
  R* V;           // [S][n]
  const R* lap;   // [S][n] or null
  const R* g2;    // [S][n] or null
  const R* vh;    // [S][n] Coulomb terms or null
  R* nin;         // [ring][S][n]
  R* res;         // [ring][S][n]
  double* part;   // [gridDim.x][kNPart]
  const double* vres_part;  // partials of |V_new - V_old|^2 from an external
  int vres_blocks;          //   V assembly (when assemble_v == 0), or null
  mpdpft_iter_log* log;
  int log_cap;
  int assemble_v;  // 1: phase A assembles V from vext, n_in and vh
  int mode;        // 0: SC iteration; 1: densities of the current V only;
                   // 2: admix only (V holds the output densities)
};

__device__ __forceinline__ unsigned long long globaltimer() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
#define MPDPFT_TSTAMP(k) \
  if (blockIdx.x == 0 && threadIdx.x == 0) st->tphase[k] = globaltimer()

__device__ __forceinline__ double ldcg(const double* p) { return __ldcg(p); }

// Block-wide copy of the SC state between global and block 0's shared copy.
// The grid-barrier fields (bar_count onwards) are never copied back.
__device__ __forceinline__ void state_load(ScState* dst, const ScState* src) {
  const unsigned* s = reinterpret_cast<const unsigned*>(src);
  unsigned* d = reinterpret_cast<unsigned*>(dst);
  for (int i = threadIdx.x; i < (int)(sizeof(ScState) / 4); i += blockDim.x) d[i] = __ldcg(s + i);
}
__device__ __forceinline__ void state_store(ScState* dst, const ScState* src) {
  const unsigned* s = reinterpret_cast<const unsigned*>(src);
  unsigned* d = reinterpret_cast<unsigned*>(dst);
  for (int i = threadIdx.x; i < (int)(offsetof(ScState, bar_count) / 4); i += blockDim.x) d[i] = s[i];
}
__device__ __forceinline__ int ldcg(const int* p) { return __ldcg(p); }

// Bounded sense-free generation barrier over all blocks of a cooperative
// launch.  Returns false (and raises the abort flag) if a block does not
// arrive within the spin limit; every block then leaves its loop.
__device__ inline bool grid_barrier(ScState* st) {
  __syncthreads();
  __shared__ int ok;
  if (threadIdx.x == 0) {
    ok = 1;
    volatile unsigned* gen = &st->bar_gen;
    unsigned g = *gen;
    __threadfence();
    unsigned arrived = atomicAdd(&st->bar_count, 1u);
    if (arrived == gridDim.x - 1) {
      atomicExch(&st->bar_count, 0u);
      __threadfence();
      atomicAdd(&st->bar_gen, 1u);
    } else {
      long spins = 0;
      while (*gen == g) {
        if (*(volatile int*)&st->abort) { ok = 0; break; }
        if (++spins > kBarrierSpinLimit) {
          atomicExch(&st->abort, 1);
          atomicOr(&st->status_bits, kBitTimeout);
          ok = 0;
          break;
        }
        __nanosleep(64);
      }
    }
    __threadfence();
  }
  __syncthreads();
  return ok != 0;
}

// ---------------------------------------------------------- mu search ----
// The reference brackets mu by steps Delta_c = e^{DeltamuModifier} (1 + c)
// |mu_prev| away from the start (mpDPFT.cpp:4603, 4633), adapting
// DeltamuModifier once after the first step (:4613, :4643), for at most 20
// steps (:4584), and then bisects until |N - N*| / (2 N*) <= RelAcc.
// Here every pass evaluates N(mu) (in double) for a few candidates in one
// sweep over the grid, plus dN/dmu at the first candidate:
//   pass 0   the start value and the reference's first step both ways;
//   then     a Newton step from the first candidate with a tight pair
//            around it (which usually brackets the root) and the bracket
//            midpoint as a safeguard; while no bracket is known, the
//            reference's remaining bracket steps (adapted modifier) join.
// Every evaluated point tightens the bracket, the Newton point is clipped
// into it, and the search ends with the reference's tolerance test.
__device__ __forceinline__ double tri(int c) { return 0.5 * (double)c * (double)(c + 1); }

// Offset of the reference's c-th bracket step from the start.
__device__ __forceinline__ double step_offset(const MuState& m, int c) {
  return m.delta0 + m.delta1 * (tri(c) - 1.0);
}

__device__ inline void mu_begin(MuState& m, double mu, double prev_abs, double dmm, int active) {
  m.start = mu;
  m.prev_abs = prev_abs;
  m.delta0 = exp(dmm) * prev_abs;
  m.delta1 = m.delta0;
  m.have_lo = m.have_hi = 0;
  m.done = active ? 0 : 1;
  m.active = active;
  m.pass = 0;
  m.dir = 0;
  m.next_c = 2;
  m.best_mu = mu;
  m.dens_mu = mu;
  m.best_N = 0.0;
  m.best_err = 1e300;
  m.step = 0.0;
  m.ncand = 0;
  m.cand[m.ncand++] = mu;
  m.cand[m.ncand++] = mu - m.delta0;  // first reference step, both directions
  m.cand[m.ncand++] = mu + m.delta0;
}

// Bracket [lo, hi] of the reference: the two consecutive bracket-step
// positions around the first crossing of N* in the search direction
// (muVecMIN/muVecMAX, mpDPFT.cpp:4601-4654).  Only candidates inside it take
// part in the search afterwards, so the root found is the one the
// reference's bisection converges to when N(mu) is not monotone.
__device__ inline void set_bracket(MuState& m, double a, double Na, double b, double Nb) {
  if (a > b) { double t = a; a = b; b = t; t = Na; Na = Nb; Nb = t; }
  m.lo = a; m.Nlo = Na; m.hi = b; m.Nhi = Nb;
  m.have_lo = m.have_hi = 1;
}

// Evaluate a pass (block 0, thread 0): N[c] at the candidates, slope =
// dN/dmu at candidate 0.  Finds the bracket, tightens it with every
// candidate inside, and places the next candidates or finishes.
__device__ inline void mu_decide(MuState& m, const double* N, double slope, double target, double rel_acc,
                                 double& dmm, int& bits) {
  const double denom = fabs(2.0 * target);
  for (int c = 0; c < m.ncand; ++c)
    if (!isfinite(N[c])) bits |= kBitNonfinite;
  const bool bracket_before = m.have_lo && m.have_hi;
  m.cand_prev0 = m.cand[0];
  m.N_prev0 = N[0];
  if (m.pass == 0) {
    const double mu0 = m.cand[0], N0 = N[0];
    const double diff0 = fabs(N0 - target);
    m.best_mu = mu0; m.best_N = N0; m.best_err = diff0 / denom;
    m.dir = N0 > target ? -1 : 1;
    if (m.best_err > rel_acc) {
      const double mu1 = m.dir < 0 ? m.cand[1] : m.cand[2];
      const double n1 = m.dir < 0 ? N[1] : N[2];
      dmm -= (fabs(n1 - target) - diff0 < 0.0 ? -1.0 : 1.0) * 0.1 * fabs(dmm);  // (:4613, :4643)
      m.delta1 = exp(dmm) * m.prev_abs;
      const bool cross = m.dir < 0 ? (n1 <= target) : (n1 >= target);
      if (cross) set_bracket(m, mu0, N0, mu1, n1);
      m.last_mu = mu1; m.last_N = n1;
    }
  } else if (!bracket_before) {
    // bracket-step pass: candidates are steps next_c0 .. in the search direction
    double pm = m.last_mu, pN = m.last_N;
    for (int c = 0; c < m.ncand; ++c) {
      const bool cross = m.dir < 0 ? (N[c] <= target) : (N[c] >= target);
      if (cross) { set_bracket(m, pm, pN, m.cand[c], N[c]); break; }
      pm = m.cand[c]; pN = N[c];
    }
    m.last_mu = pm; m.last_N = pN;
  } else {
    // inside the bracket: tighten it and track the best point
    for (int c = 0; c < m.ncand; ++c) {
      const double mu = m.cand[c], n = N[c];
      if (!(mu > m.lo && mu < m.hi) || !isfinite(n)) continue;
      const double err = fabs(n - target) / denom;
      if (err < m.best_err) { m.best_err = err; m.best_mu = mu; m.best_N = n; }
      if (n < target) { m.lo = mu; m.Nlo = n; }
      else if (n > target) { m.hi = mu; m.Nhi = n; }
    }
  }
  m.pass++;
  m.dens_mu = m.best_mu;
  if (m.best_err <= rel_acc) { m.done = 1; return; }
  if (m.pass >= kMuMaxPasses) { m.done = 1; bits |= kBitTimeout; return; }
  m.ncand = 0;
  if (!(m.have_lo && m.have_hi)) {
    if (m.next_c > 20) {
      // no bracket within the reference's 20 steps: it resets mu to the
      // start value but keeps the density of its last trial (:4657-4662)
      m.done = 1;
      m.dens_mu = m.start + m.dir * step_offset(m, 20);
      m.best_mu = m.start;
      m.best_err = 1e300;
      bits |= kBitBracket;
      return;
    }
    while (m.next_c <= 20 && m.ncand < kMuCand) m.cand[m.ncand++] = m.start + m.dir * step_offset(m, m.next_c++);
    return;
  }
  if (!(m.hi - m.lo > 1.0e-12)) { m.done = 1; return; }  // Deltamu below MP (:4711)
  if (!bracket_before) {
    // the reference starts bisecting at the bracket midpoint (:4667-4672);
    // its first evaluation also provides the slope for Newton steps
    m.best_mu = 0.5 * (m.lo + m.hi);
    m.best_err = 1e300;
    m.step = 0.0;
    // Newton from candidate 0 of the bracketing pass (its slope is known)
    if (slope > 0.0 && isfinite(slope) && isfinite(m.N_prev0)) {
      const double est = m.cand_prev0 + (target - m.N_prev0) / slope;
      if (est > m.lo && est < m.hi) {
        const double d = fabs(est - m.cand_prev0);
        const double e = fmax(1e-3 * d, 1e-13 * fabs(est) + 1e-300);
        m.step = d;
        m.cand[m.ncand++] = est;  // candidate 0 carries the slope
        if (est - e > m.lo) m.cand[m.ncand++] = est - e;
        if (est + e < m.hi) m.cand[m.ncand++] = est + e;
      }
    }
    const double rf = m.lo + (target - m.Nlo) * (m.hi - m.lo) / (m.Nhi - m.Nlo);
    if (rf > m.lo && rf < m.hi) m.cand[m.ncand++] = rf;
    m.cand[m.ncand++] = 0.5 * (m.lo + m.hi);
    return;
  }
  // Newton from candidate 0 of this pass, clipped into the bracket; else
  // regula falsi
  const double mu0 = m.cand_prev0, N0 = m.N_prev0;
  double est;
  bool newton = slope > 0.0 && isfinite(slope) && isfinite(N0);
  if (newton) {
    est = mu0 + (target - N0) / slope;
    newton = est > m.lo && est < m.hi;
  }
  if (!newton) est = m.lo + (target - m.Nlo) * (m.hi - m.lo) / (m.Nhi - m.Nlo);
  if (!(est > m.lo && est < m.hi)) est = 0.5 * (m.lo + m.hi);
  const double d = fabs(est - mu0);
  double e = 1e-3 * d;
  if (m.step > 0.0) e = fmax(e, 2.0 * d * d / m.step);
  e = fmax(e, 1e-13 * fabs(est) + 1e-300);
  m.step = d;
  m.cand[m.ncand++] = est;
  if (est - e > m.lo) m.cand[m.ncand++] = est - e;
  if (est + e < m.hi) m.cand[m.ncand++] = est + e;
  if (m.pass > 3) m.cand[m.ncand++] = 0.5 * (m.lo + m.hi);
}

// ---------------------------------------------------------- small solve --
// Inverse of the Pulay Gram matrix by Gauss-Jordan elimination with full
// pivoting; rank test as Eigen's FullPivHouseholderQR::isInvertible
// (threshold eps * n * max|pivot|), which the reference uses (mpDPFT.cpp:5089).
// One warp, matrices in shared memory; pivots are the first maximum in
// row-major order, as in a serial scan.
// G is n x n (row-major, stride n); inv receives the inverse.  Returns the
// rank-test result on every lane.
__device__ inline bool warp_inverse(int n, const double* G, double* M, double* inv, double* fac, int* colperm) {
  const int lane = threadIdx.x & 31;
  for (int i = lane; i < n * n; i += 32) { M[i] = G[i]; inv[i] = 0.0; }
  __syncwarp();
  for (int i = lane; i < n; i += 32) { inv[i * n + i] = 1.0; colperm[i] = i; }
  __syncwarp();
  double maxpiv = 0.0, minpiv = 1e300;
  for (int c = 0; c < n; ++c) {
    const int w = n - c;
    double best = -1.0;
    int bidx = c * n + c;
    for (int e = lane; e < w * w; e += 32) {
      const int i = c + e / w, j = c + e % w;
      const double v = fabs(M[i * n + j]);
      if (v > best) { best = v; bidx = i * n + j; }
    }
    for (int o = 16; o > 0; o >>= 1) {
      const double ob = __shfl_xor_sync(0xffffffffu, best, o);
      const int oi = __shfl_xor_sync(0xffffffffu, bidx, o);
      if (ob > best || (ob == best && oi < bidx)) { best = ob; bidx = oi; }
    }
    const int pr = bidx / n, pc = bidx % n;
    if (pr != c)
      for (int j = lane; j < n; j += 32) {
        double t = M[pr * n + j]; M[pr * n + j] = M[c * n + j]; M[c * n + j] = t;
        t = inv[pr * n + j]; inv[pr * n + j] = inv[c * n + j]; inv[c * n + j] = t;
      }
    __syncwarp();
    if (pc != c) {
      for (int i = lane; i < n; i += 32) { double t = M[i * n + pc]; M[i * n + pc] = M[i * n + c]; M[i * n + c] = t; }
      if (lane == 0) { int t = colperm[pc]; colperm[pc] = colperm[c]; colperm[c] = t; }
    }
    __syncwarp();
    const double piv = M[c * n + c];
    maxpiv = fmax(maxpiv, fabs(piv));
    minpiv = fmin(minpiv, fabs(piv));
    if (piv == 0.0) return false;
    const double ip = 1.0 / piv;
    __syncwarp();
    for (int j = lane; j < n; j += 32) { M[c * n + j] *= ip; inv[c * n + j] *= ip; }
    __syncwarp();
    for (int i = lane; i < n; i += 32) fac[i] = M[i * n + c];
    __syncwarp();
    for (int e = lane; e < n * n; e += 32) {
      const int i = e / n, j = e % n;
      if (i == c) continue;
      const double f = fac[i];
      if (f == 0.0) continue;
      M[i * n + j] -= f * M[c * n + j];
      inv[i * n + j] -= f * inv[c * n + j];
    }
    __syncwarp();
  }
  if (minpiv <= 2.220446049250313e-16 * (double)n * maxpiv) return false;
  // undo the column permutation: row c of the result goes to row colperm[c]
  for (int e = lane; e < n * n; e += 32) M[e] = inv[e];
  __syncwarp();
  for (int e = lane; e < n * n; e += 32) {
    const int c = e / n, j = e % n;
    inv[colperm[c] * n + j] = M[e];
  }
  __syncwarp();
  return true;
}

// Reduce kNPart partials over blocks into red[] (block 0 only).
__device__ inline void reduce_partials(const double* part, int nblocks, int nvals, double* red) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int j = warp; j < nvals; j += nw) {
    double t = 0.0;
    for (int b = lane; b < nblocks; b += 32) t += __ldcg(part + (long)b * kNPart + j);
    t = warp_sum(t);
    if (lane == 0) red[j] = t;
  }
  __syncthreads();
}

// ------------------------------------------------------------ the kernel --
// mode 0: one SC iteration.  mode 1: GetDensities of the current V (mu
// search + n[V]), written into the current ring slot; used for the initial
// densities (mpDPFT.cpp:195) and the standalone mu-search entry point.
template <typename R>
__global__ void __launch_bounds__(kStepThreads, 2) sc_step_kernel(StepArgs<R> a) {
  const KParams& kp = a.kp;
  ScState* st = a.st;
  const long n = kp.geom.n;
  const int S = kp.S;
  const long tid = (long)blockIdx.x * blockDim.x + threadIdx.x;
  const long nthreads = (long)gridDim.x * blockDim.x;
  __shared__ double red[kNPart];
  __shared__ double s_mu[kMaxS];      // mu of the final density
  __shared__ double s_mu_rep[kMaxS];  // mu reported (the start value after a bracket failure)
  __shared__ int s_flag;
  __shared__ MuState s_ms[kMaxS];
  __shared__ double s_G[kMaxP * kMaxP], s_M[kMaxP * kMaxP], s_inv[kMaxP * kMaxP], s_fac[kMaxP];
  __shared__ int s_perm[kMaxP];
  __shared__ int s_ok;
  __shared__ double s_grow[kMaxP];

  if (a.mode != 1 && ldcg(&st->exit_loop)) return;
  // block 0 runs the scalar SC logic on a shared-memory copy of the state
  // (global round trips would serialise it); it writes the copy back before
  // every grid barrier after which other blocks read the state
  __shared__ ScState s_st;
  ScState* const ls = &s_st;
  if (blockIdx.x == 0) {
    state_load(ls, st);
    __syncthreads();
  }
  const int cur = ldcg(&st->slot);
  const int ring = kp.ring;
  const int next = (cur + 1) % ring;
  double* mypart = a.part + (long)blockIdx.x * kNPart;
  MPDPFT_TSTAMP(0);

  // ---- phase A: UpdateV (mpDPFT.cpp:4815-4838) --------------------------
  if (a.mode == 0 && a.assemble_v) {
    const double incv = ldcg(&st->inc_v);
    const double fac = incv < 1.0 ? incv : 1.0;
    double acc[kMaxS];
    for (int s = 0; s < kMaxS; ++s) acc[s] = 0.0;
    const R* nin = a.nin + (long)cur * S * n;
    for (long p = tid; p < n; p += nthreads) {
      for (int s = 0; s < S; ++s) {
        R vi = R(0);
        if (kp.contact_self) vi += R(2.0 * kp.beta) * nin[p];  // type 10 (:2261)
        if (kp.contact_mutual) {                                  // type 1 (:2247)
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
    block_reduce_store<kMaxS>(acc, mypart);
  }

  // ---- phase B: mu search (GetDensities + EnforceConstraints) ----------
  const int active = kp.rel_acc > 1.0e-12 ? 1 : 0;
  if (threadIdx.x == 0) {  // every block derives the pass-0 candidates itself
    double dmm = ldcg(&st->dmm);
    double pn = 0.0;
    for (int s = 0; s < S; ++s) { double pm = ldcg(&st->mu[s]); pn += pm * pm; }
    for (int s = 0; s < S; ++s) {
      double mu = ldcg(&st->mu[s]);
      double pa = sqrt(pn) < 1.0e-12 ? 1.0e-12 : fabs(mu);
      mu_begin(s_ms[s], mu, pa, dmm, active);
    }
  }
  __syncthreads();
  if (!grid_barrier(st)) return;
  if (blockIdx.x == 0) {
    if (a.mode == 0 && (a.assemble_v || a.vres_part)) {
      const double* vp = a.assemble_v ? a.part : a.vres_part;
      const int nb = a.assemble_v ? (int)gridDim.x : a.vres_blocks;
      const int stride = a.assemble_v ? kNPart : kMaxS;
      const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
      if (warp < S) {
        double t = 0.0;
        for (int b = lane; b < nb; b += 32) t += __ldcg(vp + (long)b * stride + warp);
        t = warp_sum(t);
        if (lane == 0) red[warp] = t;
      }
      __syncthreads();
      if (threadIdx.x == 0) {
        double w = 0.0;
        for (int s = 0; s < S; ++s) w = fmax(w, sqrt(red[s] / (double)n));
        ls->v_res = w;
      }
    }
    if (threadIdx.x == 0) {
      for (int s = 0; s < S; ++s) { ls->ms[s] = s_ms[s]; ls->prev_mu[s] = s_ms[s].start; }
      ls->mu_passes = 0;
      ls->iter_bits = 0;
    }
    __syncthreads();
    state_store(st, ls);
  }
  if (!grid_barrier(st)) return;

  const R* V = a.V;
  MPDPFT_TSTAMP(1);
  for (int pass = 0; pass < kMuMaxPasses && a.mode != 2; ++pass) {
    if (pass > 0 && threadIdx.x < S) {
      const int s = threadIdx.x;
      s_ms[s].done = ldcg(&st->ms[s].done);
      s_ms[s].ncand = ldcg(&st->ms[s].ncand);
      for (int c = 0; c < s_ms[s].ncand; ++c) s_ms[s].cand[c] = ldcg(&st->ms[s].cand[c]);
    }
    __syncthreads();
    int any = 0;
    for (int s = 0; s < S; ++s) any |= !s_ms[s].done;
    if (!any) break;
    for (int s = 0; s < S; ++s) {
      if (s_ms[s].done) continue;
      // N(mu) and dN/dmu are evaluated in double from the stored fields
      // (FP32 in mixed mode): the particle-number integral and the mu search
      // are FP64 in both modes
      double acc[kMuAcc];
#pragma unroll
      for (int c = 0; c < kMuAcc; ++c) acc[c] = 0.0;
      const DensParams d = kp.dens[s];
      const int nc = s_ms[s].ncand;
      const double* cmu = s_ms[s].cand;  // shared memory (broadcast reads)
      const R* Vs = V + (long)s * n;
      const R* Ls = a.lap ? a.lap + (long)s * n : nullptr;
      const R* Gs = a.g2 ? a.g2 + (long)s * n : nullptr;
      for (long p = tid; p < n; p += nthreads) {
        const double v = (double)Vs[p];
        const double l = Ls ? (double)Ls[p] : 0.0;
        const double g = Gs ? (double)Gs[p] : 0.0;
        acc[kMuCand] += density_slope_d(d, cmu[0] - v, l, g);
#pragma unroll
        for (int c = 0; c < kMuCand; ++c)
          if (c < nc) acc[c] += density_at_d(d, cmu[c] - v, l, g);
      }
      block_reduce_store<kMuAcc>(acc, mypart + s * kMuAcc);
    }
    if (!grid_barrier(st)) return;
    if (blockIdx.x == 0) {
      reduce_partials(a.part, gridDim.x, S * kMuAcc, red);
      if (threadIdx.x == 0) {
        double dmm = ls->dmm;
        int bits = 0;
        for (int s = 0; s < S; ++s) {
          if (s_ms[s].done) continue;
          MuState ms = ls->ms[s];
          double N[kMuCand];
          for (int c = 0; c < ms.ncand; ++c) N[c] = red[s * kMuAcc + c] * kp.geom.dvol;
          mu_decide(ms, N, red[s * kMuAcc + kMuCand] * kp.geom.dvol, kp.abundance[s], kp.rel_acc, dmm, bits);
          ls->ms[s] = ms;
        }
        ls->dmm = dmm;
        ls->iter_bits |= bits;
        ls->mu_passes++;
      }
      __syncthreads();
      state_store(st, ls);
    }
    if (!grid_barrier(st)) return;
  }

  MPDPFT_TSTAMP(2);
  // ---- phase C: final densities, residual, CC dots, Gram row -----------
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
  {
    // per species: [0] N, [1] <n_out, n_in>_w, [2] <n_out, n_out>_w,
    // [3] <n_in, n_in>_w, [4 + j] <r_new, r_j>_w (Gram row, summed over
    // species in phase D); w = multiplicity in the reference storage
    __shared__ long s_roff[kMaxP];
    if (threadIdx.x < I) {
      const int j = threadIdx.x;
      s_roff[j] = (long)((cur - (I - 1) + j + ring) % ring) * S * n;
    }
    __syncthreads();
    R* nin = a.nin + (long)cur * S * n;
    R* rcur = a.res + (long)cur * S * n;
    for (int s = 0; s < S; ++s) {
      double acc[kNF];
#pragma unroll
      for (int j = 0; j < kNF; ++j) acc[j] = 0.0;
      const DensParams d = kp.dens[s];
      const double mus = s_mu[s];
      const long so = (long)s * n;
      for (long p = tid; p < n; p += nthreads) {
        const long q = so + p;
        const R v = V[q];
        const double l = a.lap ? (double)a.lap[q] : 0.0;
        const double g = a.g2 ? (double)a.g2[q] : 0.0;
        // mode 2 (admix only): V holds the output densities
        const double nod = a.mode == 2 ? (double)v : density_at_d(d, mus - (double)v, l, g);
        const R no = R(nod);
        acc[0] += nod;
        if (a.mode == 1) { nin[q] = no; continue; }
        const R ni = nin[q];
        const R r = no - ni;
        rcur[q] = r;
        const double w = ref_multiplicity(p, kp.geom.s, kp.geom.dim);
        const double dno = (double)no, dni = (double)ni, dr = (double)r, wr = w * dr;
        acc[1] += w * dno * dni;
        acc[2] += w * dno * dno;
        acc[3] += w * dni * dni;
        for (int j = 0; j < I - 1; ++j) acc[4 + j] += wr * (double)a.res[s_roff[j] + q];
        if (I > 0) acc[4 + I - 1] += wr * dr;
      }
      block_reduce_store<kNF>(acc, mypart + s * kNF);
    }
  }
  if (!grid_barrier(st)) return;

  // ---- phase D: CheckConvergence, Intercept, PulayMixer, InjectSchedule --
  MPDPFT_TSTAMP(3);
  if (blockIdx.x == 0) {
    reduce_partials(a.part, gridDim.x, S * kNF, red);
    if (threadIdx.x < kMaxP) {  // Gram row summed over species
      double t = 0.0;
      for (int s = 0; s < S; ++s) t += red[s * kNF + 4 + threadIdx.x];
      s_grow[threadIdx.x] = t;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      const int sc = ls->sc_count;
      double tot = 0.0;
      for (int s = 0; s < S; ++s) {
        ls->mu[s] = s_mu_rep[s];
        ls->ab[s] = red[s * kNF] * kp.geom.dvol;
        if (!isfinite(ls->ab[s])) ls->iter_bits |= kBitNonfinite;
        tot += ls->ab[s];
      }
      if (a.mode == 1) {
        ls->status_bits |= ls->iter_bits;
        ls->mu_passes_total += ls->mu_passes;
      } else {
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
        // AdmixDensities / PulayMixer (mpDPFT.cpp:4921-5167): assemble the
        // Gram matrix (last row/column new, the rest shifted from before)
        if (pulay_now) {
          const int shift = (hist + 1 > kp.scope) ? 1 : 0;
          for (int i = 0; i < I; ++i)
            for (int j = 0; j < I; ++j) {
              double v;
              if (i == I - 1) v = s_grow[j];
              else if (j == I - 1) v = s_grow[i];
              else v = ls->gram[(i + shift) * kMaxP + (j + shift)];
              s_G[i * I + j] = v;
            }
          for (int i = 0; i < I; ++i)
            for (int j = 0; j < I; ++j) ls->gram[i * kMaxP + j] = s_G[i * I + j];
          ls->hist = I;
        }
      }
    }
    __syncthreads();
    // the small inverse on warp 0 (FullPivHouseholderQR + validation in the
    // reference, mpDPFT.cpp:5089-5107)
    if (a.mode != 1 && pulay_now && threadIdx.x < 32) {
      bool ok = warp_inverse(I, s_G, s_M, s_inv, s_fac, s_perm);
      double test = 0.0;
      if (ok) {
        for (int e = threadIdx.x; e < I * I; e += 32) {
          const int i = e / I, j = e % I;
          double t = 0.0;
          for (int k = 0; k < I; ++k) t += s_inv[i * I + k] * s_G[k * I + j];
          t -= (i == j) ? 1.0 : 0.0;
          test += t * t;
        }
        test = warp_sum(test);
      }
      if (threadIdx.x == 0) s_ok = ok && test <= 1.0e-8;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      const int sc = ls->sc_count;
      if (a.mode != 1) {
        int used = 0;
        if (pulay_now) {
          if (s_ok) {
            double x[kMaxP], A = 0.0;
            for (int i = 0; i < I; ++i) {
              x[i] = 0.0;
              for (int k = 0; k < I; ++k) x[i] += s_inv[i * I + k];
              A += x[i];
            }
            for (int i = 0; i < I; ++i) ls->coeff[i] = x[i] / A;
            used = 1;
          }
          if (!used) ls->iter_bits |= kBitPulay;
        }
        ls->pulay_used = used;
        ls->ncoeff = used ? I : 0;
        for (int s = 0; s < S; ++s) ls->theta_mix[s] = ls->theta[s];
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
        if (a.log && sc < a.log_cap) {
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
  }
  if (a.mode == 1) return;
  MPDPFT_TSTAMP(4);
  if (!grid_barrier(st)) return;
  MPDPFT_TSTAMP(5);

  // ---- phase E: mixed density -> ring[next] ----------------------------
  // n = sum_j c_j (n_in,j + theta r_j) (Pulay) or n_in + theta r (linear),
  // AdmixDensities mpDPFT.cpp:4946-4955 / :4987
  {
    __shared__ long s_off[kMaxP];
    __shared__ double s_c[kMaxP];
    __shared__ int s_nc;
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
    for (int s = 0; s < S; ++s) {
      const double th = ldcg(&st->theta_mix[s]);
      R* out = a.nin + (long)next * S * n + (long)s * n;
      if (sizeof(R) == sizeof(float) && (n & 3) == 0) {
        const long n4 = n >> 2;
        for (long p4 = tid; p4 < n4; p4 += nthreads) {
          double v0 = 0.0, v1 = 0.0, v2 = 0.0, v3 = 0.0;
          for (int j = 0; j < nc; ++j) {
            const long q = s_off[j] + (long)s * n + 4 * p4;
            const float4 ni = *reinterpret_cast<const float4*>(a.nin + q);
            const float4 ri = *reinterpret_cast<const float4*>(a.res + q);
            const double c = s_c[j];
            v0 += c * ((double)ni.x + th * (double)ri.x);
            v1 += c * ((double)ni.y + th * (double)ri.y);
            v2 += c * ((double)ni.z + th * (double)ri.z);
            v3 += c * ((double)ni.w + th * (double)ri.w);
          }
          *reinterpret_cast<float4*>(out + 4 * p4) = make_float4((float)v0, (float)v1, (float)v2, (float)v3);
        }
      } else {
        for (long p = tid; p < n; p += nthreads) {
          double v = 0.0;
          for (int j = 0; j < nc; ++j) {
            const long q = s_off[j] + (long)s * n + p;
            v += s_c[j] * ((double)a.nin[q] + th * (double)a.res[q]);
          }
          out[p] = R(v);
        }
      }
    }
  }
  MPDPFT_TSTAMP(6);
}

}  // namespace mpdpft
