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
constexpr int kStepWarps = kStepThreads / 32;
constexpr int kSegPts = 128;          // points of one warp step (4 per lane)
constexpr int kDensThreads = 256;     // mixing kernel
constexpr int kDensityThreads = 256;  // density kernel
constexpr int kMuAcc = kMuCand + 1;  // candidate sums + dN/dmu at candidate 0
constexpr int kNF = 4 + kMaxP;        // per-species sums of the density/Gram pass
// per-block partial sums: [0, kVresOff) the mu-pass or density-pass sums,
// [kVresOff, kVresOff + kMaxS) |V_new - V_old|^2 of the in-kernel V update
constexpr int kVresOff = kMaxS * kNF > kMaxS * kMuAcc ? kMaxS * kNF : kMaxS * kMuAcc;
constexpr int kNPart = kVresOff + kMaxS;
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
  long chunk;     // points per warp in the mu kernel's sweeps (multiple of kSegPts)
  int mu_blocks;  // grid of the mu kernel (rows of its partial sums)
  int vec4;       // n % 4 == 0: a lane loads 4 points as one vector
  int mu_max_passes;  // mu-search pass cap (1 .. kMuMaxPasses)
  long spin_limit;    // grid-barrier spin limit
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
  int trapped;  // ended inside a bracket without meeting the tolerance
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
  // not part of the state copies (written by one kernel, read by the next)
  int iter_active;    // 0: the loop had already exited when this iteration began
  unsigned k2_done;   // blocks of the density kernel that have finished
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
  R* cur_copy;    // [S][n] copy of the current input densities (fixed address)
  double* part;   // [mu_blocks][kNPart]: mu-pass sums, V-update residual
  double* part2;  // [density blocks][kNPart]: density-pass sums
  // active-point lists of the mu search (functionals that vanish for
  // mu <= V): every warp's list of the points it owns below the largest
  // candidate of the pass that built the lists; later passes whose
  // candidates stay below that bound visit only those
  int* bcount;  // [kMaxS][mu_blocks] (unused by the mu search)
  int* plist;   // [S][plist_stride]: per species, one region per warp
  long plist_stride;
  const double* vres_part;  // partials of |V_new - V_old|^2 from an external
  int vres_blocks;          //   V assembly (when assemble_v == 0), or null
  mpdpft_iter_log* log;
  int log_cap;
  int assemble_v;  // 1: phase A assembles V from vext, n_in and vh
  int mode;        // 0: SC iteration; 1: densities of the current V only;
                   // 2: admix only (V holds the output densities)
  int split_d;     // 1: phase D runs as its own one-block launch after the
                   // density kernel; 0: the density kernel's last block runs it
};

__device__ __forceinline__ unsigned long long globaltimer() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
// phase timestamp from block 0 of a solve (bid: the block's index within it)
#define MPDPFT_TSTAMP_B(k) \
  if (bid == 0 && threadIdx.x == 0) st->tphase[k] = globaltimer()

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
// arrive within `limit` spins; every block then leaves its loop.
__device__ inline bool grid_barrier(ScState* st, const int nblk, const long limit) {
  __syncthreads();
  __shared__ int ok;
  if (threadIdx.x == 0) {
    ok = 1;
    volatile unsigned* gen = &st->bar_gen;
    unsigned g = *gen;
    __threadfence();
    unsigned arrived = atomicAdd(&st->bar_count, 1u);
    if (arrived == (unsigned)nblk - 1u) {
      atomicExch(&st->bar_count, 0u);
      __threadfence();
      atomicAdd(&st->bar_gen, 1u);
    } else {
      long spins = 0;
      while (*gen == g) {
        if (*(volatile int*)&st->abort) { ok = 0; break; }
        if (++spins > limit) {
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
  m.trapped = 0;
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
                                 double& dmm, int& bits, int max_passes) {
  const double denom = fabs(2.0 * target);
  for (int c = 0; c < m.ncand; ++c)
    if (!isfinite(N[c])) bits |= kBitNonfinite;
  const bool bracket_before = m.have_lo && m.have_hi;
  bool poor = false;  // an in-bracket pass that left more than a quarter of the bracket
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
    const double w0 = m.hi - m.lo;
    for (int c = 0; c < m.ncand; ++c) {
      const double mu = m.cand[c], n = N[c];
      if (!(mu > m.lo && mu < m.hi) || !isfinite(n)) continue;
      const double err = fabs(n - target) / denom;
      if (err < m.best_err) { m.best_err = err; m.best_mu = mu; m.best_N = n; }
      if (n < target) { m.lo = mu; m.Nlo = n; }
      else if (n > target) { m.hi = mu; m.Nhi = n; }
    }
    poor = !(m.hi - m.lo <= 0.25 * w0);
  }
  m.pass++;
  m.dens_mu = m.best_mu;
  if (m.best_err <= rel_acc) { m.done = 1; return; }
  if (m.pass >= max_passes) {
    m.done = 1;
    m.trapped = m.have_lo && m.have_hi;
    bits |= kBitTimeout;
    return;
  }
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
  // the bracket has closed to MP (1e-12) without meeting the tolerance.  The
  // reference's bisection stops either on Deltamu < MP (:4711, a warning:
  // N(mu) too steep for the tolerance) or, earlier, on its trap test
  // (:4690-4703: abundances repeating within RelAcc N*, i.e. N(mu) changes
  // by less than that over the remaining steps while a step of N straddles
  // the target), which sets TrappedQ: the latter where the local slope
  // moves N by less than RelAcc N* over MP
  if (!(m.hi - m.lo > 1.0e-12)) {
    m.done = 1;
    m.trapped = !(slope * 1.0e-12 >= rel_acc * fabs(target));
    return;
  }
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
  // a pass that left more than a quarter of the bracket (N(mu) too rough
  // for the Newton placement, e.g. where the adaptive Airy quadrature
  // changes its subdivision with mu), and every pass after the third, puts
  // the free candidates on an even subdivision of the bracket, so such a
  // pass shrinks it at least (free + 1)-fold
  if (poor || m.pass > 3) {
    const int nfree = kMuCand - m.ncand;
    for (int k = 1; k <= nfree; ++k) m.cand[m.ncand++] = m.lo + (m.hi - m.lo) * ((double)k / (double)(nfree + 1));
  }
}

}  // namespace mpdpft
