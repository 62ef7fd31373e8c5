// mpdpft_oracle.cpp -- CPU oracle for the SC loop of mpDPFT.
//
// TEST INFRASTRUCTURE ONLY.  This file is the checker: the parity tests, the
// smoke check and the CPU-baseline leg of bench.py call it to produce the
// expected results.  The product (mpdpft_b200/) never links, loads or calls it.
//
// A fresh FP64 restatement of the reference algorithm, written from the
// mathematics of mpDPFT.cpp (cited as MD:line) without copying its source.
// It keeps the reference's storage conventions on purpose: fields live on the
// (s+1)^D grid whose last plane along each axis duplicates plane 0 (MD:863),
// integrals are trapezoid sums over that grid (MD:7981-8026), dot products run
// over every stored point (VecMult, MD:7103-7107), and transforms use the
// centred-k convention of fftParallel (MD:8173-8335).  The FFT is this file's
// own mixed-radix Stockham transform (FFTW is absent here); it is validated
// against numpy.fft by the tests.
//
// Parity of the SC loop is unpinned by the reference itself (it ships no
// tests and cannot be built in this container); this oracle is pinned by
// known-answer tests (Gaussian transform pair, harmonic-oscillator TF mu and
// energy, Poisson of a Gaussian charge, Pulay on a linear map) in tests/.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstring>
#include <limits>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "../include/mpdpft_gpu.h"

namespace {

using cplx = std::complex<double>;
constexpr double PI = 3.141592653589793;
constexpr double MP = 1.0e-12;               // MD:111
constexpr double MACHINE_PRECISION = 1.0e-16; // MD:111

inline double POS(double x) { return x > 0. ? x : 0.; }
inline double SIGN(double x) { return x < 0. ? -1. : 1.; }
// EXP with the reference's clamps (mpDPFT.h:266)
inline double EXPc(double x) {
  if (x < -700.) return 0.;
  if (x < 700.) return std::exp(x);
  return 1.0142320547350045e+304;
}

// ---------------------------------------------------------------- FFT ----
// Stockham autosort, decimation in frequency, radices 4/2/3/5 and a direct
// DFT for any other prime factor.  Unnormalised, sign -1 = e^{-2 pi i jk/n}.
struct Plan1D {
  int n = 0;
  std::vector<int> radix;
  std::vector<cplx> tw_fwd, tw_bwd;  // e^{-+2 pi i t/n}, t = 0..n-1
};

Plan1D make_plan(int n) {
  Plan1D p;
  p.n = n;
  int m = n;
  while (m % 4 == 0) { p.radix.push_back(4); m /= 4; }
  while (m % 2 == 0) { p.radix.push_back(2); m /= 2; }
  while (m % 3 == 0) { p.radix.push_back(3); m /= 3; }
  while (m % 5 == 0) { p.radix.push_back(5); m /= 5; }
  for (int f = 7; m > 1; f += 2)
    while (m % f == 0) { p.radix.push_back(f); m /= f; }
  p.tw_fwd.resize(n);
  p.tw_bwd.resize(n);
  for (int t = 0; t < n; ++t) {
    double a = 2. * PI * (double)t / (double)n;
    p.tw_fwd[t] = cplx(std::cos(a), -std::sin(a));
    p.tw_bwd[t] = cplx(std::cos(a), std::sin(a));
  }
  return p;
}

// One length-n transform of x (contiguous); y is scratch of length n.
void fft_line(const Plan1D& p, int sign, cplx* x, cplx* y) {
  const int n = p.n;
  const std::vector<cplx>& tw = sign < 0 ? p.tw_fwd : p.tw_bwd;
  cplx* src = x;
  cplx* dst = y;
  int len = n;   // current sub-transform length
  int stride = 1;
  cplx a[64], b[64];
  for (int r : p.radix) {
    const int m = len / r;
    const int twstep = n / len;  // twiddle e^{-+2 pi i p u/len} = tw[p*u*twstep]
    const int rstep = n / r;     // r-th roots: tw[(t*u mod r) * rstep]
    for (int q = 0; q < m; ++q) {
      for (int k = 0; k < stride; ++k) {
        for (int t = 0; t < r; ++t) a[t] = src[k + stride * (q + t * m)];
        for (int u = 0; u < r; ++u) {
          cplx acc = 0.;
          for (int t = 0; t < r; ++t) acc += a[t] * tw[((t * u) % r) * rstep];
          b[u] = acc;
        }
        for (int u = 0; u < r; ++u)
          dst[k + stride * (r * q + u)] = b[u] * tw[((long)q * u * twstep) % n];
      }
    }
    std::swap(src, dst);
    len = m;
    stride *= r;
  }
  if (src != x) std::memcpy(x, src, sizeof(cplx) * n);
}

// Unnormalised D-dimensional transform of a contiguous s^D complex array.
void fft_nd(int dim, int s, int sign, cplx* data) {
  Plan1D p = make_plan(s);
  const long s2 = (long)s * s;
  const long lines = (dim == 3) ? s2 : (dim == 2 ? s : 1);
  for (int axis = dim - 1; axis >= 0; --axis) {
    long axstride = 1;
    for (int d = dim - 1; d > axis; --d) axstride *= s;
#pragma omp parallel
    {
      std::vector<cplx> line(s), scratch(s);
#pragma omp for schedule(static)
      for (long l = 0; l < lines; ++l) {
        // enumerate the lines along `axis`: l -> base offset
        long base;
        if (dim == 1) base = 0;
        else if (dim == 2) base = (axis == 1) ? l * s : l;
        else {
          long a = l / s, b = l % s;
          if (axis == 2) base = a * s2 + b * s;
          else if (axis == 1) base = a * s2 + b;
          else base = a * s + b;
        }
        for (int t = 0; t < s; ++t) line[t] = data[base + t * axstride];
        fft_line(p, sign, line.data(), scratch.data());
        for (int t = 0; t < s; ++t) data[base + t * axstride] = line[t];
      }
    }
  }
}

// ------------------------------------------------------------- state ----
struct State {
  mpdpft_params P;
  int D, s, EL, S;
  long G;        // (s+1)^D stored points
  double L, dx, k0, dk, sigma_c;
  int centre;    // CentreIndex = (G-1)/2
  std::vector<double> lattice;  // x_i, i = 0..s
  std::vector<double> klattice; // k_i, i = 0..s
  std::vector<std::vector<double>> Env, Den, V, OldDen, OldV, Grad2, Lap;
  std::vector<cplx> CF, TmpCF;
  std::vector<double> mu, prev_mu, old_mu, tmp_ab, old_ab, theta, theta0, T;
  double relacc_orig, dmm, cc = 0., old_cc = 0., incV, incV0;
  int sc_count = 0, exit_count = 0, exit_loop = 0;
  bool trapped = false;
  long mu_trials = 0;
  unsigned del_valid = 0;  // bit s: DelField(V[s]) cached for the current V[s]
  // Pulay
  std::vector<std::vector<std::vector<double>>> nin, nout, res;
  std::vector<std::vector<double>> gram;
  std::vector<double> coeff;
  int status_bits = 0;
};

void coords(const State& st, long idx, double* r) {
  if (st.D == 3) {
    long i = idx / ((long)st.EL * st.EL), j = (idx / st.EL) % st.EL, k = idx % st.EL;
    r[0] = st.lattice[i]; r[1] = st.lattice[j]; r[2] = st.lattice[k];
  } else {
    long i = idx / st.EL, j = idx % st.EL;
    r[0] = st.lattice[i]; r[1] = st.lattice[j]; r[2] = 0.;
  }
}
double knorm2(const State& st, long idx) {
  if (st.D == 3) {
    long i = idx / ((long)st.EL * st.EL), j = (idx / st.EL) % st.EL, k = idx % st.EL;
    return st.klattice[i] * st.klattice[i] + st.klattice[j] * st.klattice[j] +
           st.klattice[k] * st.klattice[k];
  }
  long i = idx / st.EL, j = idx % st.EL;
  return st.klattice[i] * st.klattice[i] + st.klattice[j] * st.klattice[j];
}
double kcomp(const State& st, long idx, int axis) {
  long c;
  if (st.D == 3) {
    if (axis == 0) c = idx / ((long)st.EL * st.EL);
    else if (axis == 1) c = (idx / st.EL) % st.EL;
    else c = idx % st.EL;
  } else {
    c = axis == 0 ? idx / st.EL : idx % st.EL;
  }
  return st.klattice[c];
}

void init_state(State& st, const mpdpft_params& P) {
  st.P = P;
  st.D = P.dim; st.s = P.steps; st.EL = P.steps + 1; st.S = P.species;
  st.G = 1; for (int d = 0; d < st.D; ++d) st.G *= st.EL;
  st.centre = (int)((st.G - 1) / 2);
  st.L = P.edge;
  st.dx = st.L / (double)st.s;                 // MD:887
  st.k0 = -PI / st.dx;                         // MD:889
  st.dk = 2. * PI / st.L;                      // MD:890
  double smear = P.smearing_extent > 0. ? P.smearing_extent : 6. * st.dx;  // MD:1105
  st.sigma_c = -0.5 * smear * smear;           // MD:1106
  st.lattice.resize(st.EL); st.klattice.resize(st.EL);
  for (int i = 0; i <= st.s; ++i) {
    st.lattice[i] = -st.L / 2. + st.dx * (double)i;  // rGrid MD:7130
    st.klattice[i] = st.k0 + st.dk * (double)i;      // kframe MD:891-895
  }
  auto fields = [&](std::vector<std::vector<double>>& f) { f.assign(st.S, std::vector<double>(st.G, 0.)); };
  fields(st.Env); fields(st.Den); fields(st.V); fields(st.OldDen); fields(st.OldV);
  fields(st.Grad2); fields(st.Lap);
  st.CF.assign(st.G, 0.); st.TmpCF.assign(st.G, 0.);
  st.mu.assign(P.mu, P.mu + st.S);
  st.prev_mu = st.mu; st.old_mu = st.mu;
  st.tmp_ab.assign(st.S, 0.); st.old_ab.assign(st.S, 0.);
  st.theta.assign(P.theta, P.theta + st.S); st.theta0 = st.theta;
  st.T.assign(P.temperature, P.temperature + st.S);
  st.relacc_orig = P.rel_acc;
  st.dmm = P.deltamu_modifier;
  st.incV = P.incremental_v; st.incV0 = P.incremental_v;
}

// --------------------------------------------------- fftParallel MD:8173 --
void fft_parallel(State& st, int sign, std::vector<cplx>& CF) {
  const int s = st.s, EL = st.EL, D = st.D;
  const double L = st.L, x0 = -L / 2., dx = L / (double)s, k0 = -PI / dx, dk = 2. * PI / L;
  const double argPref = (sign < 0) ? PI : x0 * dk;
  long n = 1; for (int d = 0; d < D; ++d) n *= s;
  std::vector<cplx> buf(n);
  // pre-modulation (MD:8188-8218)
#pragma omp parallel for schedule(static)
  for (long p = 0; p < n; ++p) {
    long i, j, k, src;
    if (D == 3) { i = p / ((long)s * s); j = (p / s) % s; k = p % s; src = (i * EL + j) * EL + k; }
    else { i = p / s; j = p % s; k = 0; src = i * EL + j; }
    double arg = argPref * (double)(i + j + k);
    buf[p] = CF[src] * cplx(std::cos(arg), std::sin(arg));
  }
  fft_nd(D, s, sign, buf.data());
  double factor, c1, c2;
  if (sign < 0) { factor = std::pow(dx, (double)D); c1 = -x0 * (double)D * k0; c2 = -x0 * dk; }
  else { factor = std::pow(1. / L, (double)D); c1 = k0 * (double)D * x0; c2 = k0 * dx; }
#pragma omp parallel for schedule(static)
  for (long p = 0; p < n; ++p) {
    long i, j, k, dst;
    if (D == 3) { i = p / ((long)s * s); j = (p / s) % s; k = p % s; dst = (i * EL + j) * EL + k; }
    else { i = p / s; j = p % s; k = 0; dst = i * EL + j; }
    double arg = c1 + c2 * (double)(i + j + k);
    CF[dst] = factor * (cplx(std::cos(arg), std::sin(arg)) * buf[p]);
  }
  // refill of the duplicate planes (MD:8266-8324)
  if (D == 2) {
    for (int j = 0; j <= s; ++j) CF[(long)s * EL + j] = CF[j % s];
    for (int i = 0; i < s; ++i) CF[(long)i * EL + s] = CF[(long)i * EL];
  } else {
    for (int i = 0; i <= s; ++i)
      for (int j = 0; j <= s; ++j)
        for (int k = 0; k <= s; ++k) {
          if (i < s && j < s && k < s) continue;
          CF[((long)i * EL + j) * EL + k] = CF[((long)(i % s) * EL + (j % s)) * EL + (k % s)];
        }
  }
}

// ---------------------------------------------------- Integrate MD:7981 --
double integrate(const State& st, const std::vector<double>& f) {
  const int I = st.EL;
  std::vector<double> RES(I, 0.);
  if (st.D == 2) {
    for (int i = 0; i < I; ++i) {
      double ip = (i == 0 || i == I - 1) ? 0.5 : 1.;
      for (int j = 0; j < I; ++j) {
        double jp = (j == 0 || j == I - 1) ? 0.5 : 1.;
        RES[i] += ip * jp * f[(long)i * I + j];
      }
    }
  } else {
#pragma omp parallel for schedule(static)
    for (int i = 0; i < I; ++i) {
      double ip = (i == 0 || i == I - 1) ? 0.5 : 1.;
      for (int j = 0; j < I; ++j) {
        double jp = (j == 0 || j == I - 1) ? 0.5 : 1.;
        for (int k = 0; k < I; ++k) {
          double kp = (k == 0 || k == I - 1) ? 0.5 : 1.;
          RES[i] += ip * jp * kp * f[((long)i * I + j) * I + k];
        }
      }
    }
  }
  double res = 0.;
  for (int i = 0; i < I; ++i) res += RES[i];
  for (int d = 0; d < st.D; ++d) res *= st.L / ((double)I - 1.);
  return res;
}

double vecmult(const std::vector<double>& a, const std::vector<double>& b) {  // MD:7103
  double r = 0.;
  for (size_t i = 0; i < a.size(); ++i) r += a[i] * b[i];
  return r;
}

// ------------------------------------------------------ DelField MD:7243 --
// method 5 (FFT derivatives + Gaussian smoothing) with the boundary taper.
void delfield(State& st, const std::vector<double>& f, std::vector<double>& grad2,
              std::vector<double>& lap) {
  const long G = st.G;
  const int D = st.D;
  std::vector<double> t3(f);
  double r3[3];
  if (st.P.taper_off) {  // MD:7251-7264
    const double shell = st.L * st.P.regularization_threshold;
    double mx = 0.;
    bool first = true;
    for (long i = 0; i < G; ++i) {
      coords(st, i, r3);
      double r = std::sqrt(r3[0] * r3[0] + r3[1] * r3[1] + r3[2] * r3[2]);
      if (std::fabs(r - shell) < 2. * st.dx) {
        if (first) { mx = f[i]; first = false; }
        if (f[i] > mx) mx = f[i];
      }
    }
    const double a = -2500. / (st.L * st.L);  // Regularize procedure 2, MD:12269-12275
#pragma omp parallel for schedule(static)
    for (long i = 0; i < G; ++i) {
      double r3l[3];
      coords(st, i, r3l);
      double r = std::sqrt(r3l[0] * r3l[0] + r3l[1] * r3l[1] + r3l[2] * r3l[2]);
      t3[i] -= mx;
      if (r > shell) t3[i] *= EXPc(a * (r - shell) * (r - shell));
    }
  }
  std::vector<std::vector<double>> d1(D, std::vector<double>(G)), d2(D, std::vector<double>(G));
  for (long i = 0; i < G; ++i) st.CF[i] = cplx(t3[i], 0.);
  fft_parallel(st, -1, st.CF);
  st.TmpCF = st.CF;
  for (int deriv = 1; deriv <= 2; ++deriv)
    for (int j = 0; j < D; ++j) {  // MD:7431-7451
      st.CF = st.TmpCF;
      for (long i = 0; i < G; ++i) {
        double kj = kcomp(st, i, j);
        double fac = deriv == 1 ? -kj : -kj * kj;
        st.CF[i] *= fac;
      }
      fft_parallel(st, +1, st.CF);
      std::vector<double>& dst = deriv == 1 ? d1[j] : d2[j];
      for (long i = 0; i < G; ++i) dst[i] = deriv == 1 ? st.CF[i].imag() : st.CF[i].real();
    }
  auto smooth = [&](std::vector<double>& fld) {  // MD:7473-7478 and repeats
    for (long i = 0; i < G; ++i) st.CF[i] = cplx(fld[i], 0.);
    fft_parallel(st, -1, st.CF);
    for (long i = 0; i < G; ++i) st.CF[i] *= EXPc(st.sigma_c * knorm2(st, i));
    fft_parallel(st, +1, st.CF);
    for (long i = 0; i < G; ++i) fld[i] = st.CF[i].real();
  };
  for (int j = 0; j < D; ++j) { smooth(d1[j]); smooth(d2[j]); }
  grad2.assign(G, 0.);
  lap.assign(G, 0.);
  for (int j = 0; j < D; ++j)
    for (long i = 0; i < G; ++i) { grad2[i] += d1[j][i] * d1[j][i]; lap[i] += d2[j][i]; }
  smooth(grad2);
  for (long i = 0; i < G; ++i) grad2[i] = POS(grad2[i]);  // MD:7559
  smooth(lap);
}

// ---------------------------------------------- densities MD:2142-2238 --
// ------------------------- finite-T gradient form, MD:3363-3453, 3553-3620 --
// Special functions from the same Chebyshev tables as the product
// (mpdpft_b200/csrc/special_tables.inc, generated from mpmath and pinned by
// tests/test_special_functions.py against mpmath and the reference's own
// TabFunc_CurlyA.dat); the density algorithm around them is restated here.
#include "../mpdpft_b200/csrc/special_tables.inc"
const double kFdTab[5 * (MPDPFT_FD_X1 - MPDPFT_FD_X0) * MPDPFT_FD_DEG] = MPDPFT_FD_TABLE;
const double kFdAsym[5 * MPDPFT_FD_ASYM] = MPDPFT_FD_ASYM_TABLE;
const double kFdRGamma[5] = MPDPFT_FD_RGAMMA;
const double kCaTab[MPDPFT_CA_N * MPDPFT_CA_DEG] = MPDPFT_CA_TABLE;
const double kFdOrder[5] = {2.5, 1.5, 0.5, -0.5, -1.5};

double cheb(const double* c, int n, double t) {
  double b1 = 0., b2 = 0.;
  for (int j = n - 1; j >= 1; --j) {
    double b0 = std::fma(2. * t, b1, c[j] - b2);
    b2 = b1;
    b1 = b0;
  }
  return std::fma(t, b1, c[0] - b2);
}

// polylog(order, x) of MD:7000-7027 = Li_s(-e^x): 0 below -699, the leading
// term -x^s/Gamma(s+1) above 699, else the series / table / Sommerfeld forms.
double polylog(int o, double x) {
  const double s = kFdOrder[o];
  if (!(x >= -699.)) return x != x ? x : 0.;
  if (x > 699.) return -std::pow(x, s) * kFdRGamma[o];
  if (x < MPDPFT_FD_X0) {
    const double z = std::exp(x);
    double zk = z, sum = 0.;
    for (int k = 1; k <= 40; ++k) {
      const double t = zk * std::pow((double)k, -s);
      sum += (k & 1) ? -t : t;
      zk *= z;
      if (zk < 1e-18 * std::fabs(sum)) break;
    }
    return sum;
  }
  if (x < MPDPFT_FD_X1) {
    const double m = std::floor(x);
    const double* c = kFdTab + ((long)o * (MPDPFT_FD_X1 - MPDPFT_FD_X0) + ((int)m - MPDPFT_FD_X0)) * MPDPFT_FD_DEG;
    return cheb(c, MPDPFT_FD_DEG, 2. * (x - m) - 1.);
  }
  const double y = 1. / (x * x);
  double sum = 0.;
  for (int k = MPDPFT_FD_ASYM - 1; k >= 0; --k) sum = std::fma(sum, y, kFdAsym[o * MPDPFT_FD_ASYM + k]);
  return -std::pow(x, s) * kFdRGamma[o] * sum;
}

// CurlyA(y) = int_y^inf Ai (mpDPFT.h:231-237), the reference's own forms
// outside the table's range
double CurlyA(double y) {
  if (y < -1.0e50) return 1.;
  if (y < -149.99) return 1. - std::cos(0.25 * PI + 0.6666666666666666666 * (-y) * std::sqrt(-y)) /
                                   std::sqrt(PI * (-y) * std::sqrt(-y));
  if (y < MPDPFT_CA_X1) {
    const double u = (y - MPDPFT_CA_X0) / MPDPFT_CA_W;
    int i = (int)std::floor(u);
    if (i < 0) i = 0;
    return cheb(kCaTab + (long)i * MPDPFT_CA_DEG, MPDPFT_CA_DEG, 2. * (u - i) - 1.);
  }
  const double z = 2. / 3. * y * std::sqrt(y);
  return std::exp(-z) / (2. * std::sqrt(PI) * std::pow(y, 0.75));
}

// Ai(y), Ai'(y) (gsl_sf_airy_Ai / _Ai_deriv, MD:3589, 5616, 5666): on the
// CurlyA table's range the negated first and second derivatives of its
// Chebyshev series, outside it the asymptotic expansions with their first
// correction terms; 0 above 100.
void airy_ai_d(double y, double& ai, double& aip) {
  const double sp = std::sqrt(PI);
  if (y > 100.) { ai = aip = 0.; return; }
  if (y < MPDPFT_CA_X0 || y >= MPDPFT_CA_X1) {
    const double x = std::fabs(y), r4 = std::pow(x, 0.25), z = 2. / 3. * x * std::sqrt(x);
    // u_k = Gamma(3k + 1/2) / (54^k k! Gamma(k + 1/2)), v_k = -(6k+1) u_k/(6k-1)
    const double u1 = 5. / 72., u2 = 385. / 10368., u3 = 0.037993059127800655;
    const double v1 = -7. / 72., v2 = -455. / 10368., v3 = -19. / 17. * u3;
    const double iz = 1. / z, iz2 = iz * iz;
    if (y < 0.) {
      const double sn = std::sin(z + 0.25 * PI), cs = std::cos(z + 0.25 * PI);
      ai = (sn * (1. - u2 * iz2) - cs * iz * (u1 - u3 * iz2)) / (sp * r4);
      aip = r4 * (-cs * (1. - v2 * iz2) - sn * iz * (v1 - v3 * iz2)) / sp;
    } else {
      const double e = std::exp(-z);
      ai = e * (1. - u1 * iz + u2 * iz2 - u3 * iz2 * iz) / (2. * sp * r4);
      aip = -r4 * e * (1. - v1 * iz + v2 * iz2 - v3 * iz2 * iz) / (2. * sp);
    }
    return;
  }
  const double u = (y - MPDPFT_CA_X0) / MPDPFT_CA_W;
  int i = (int)std::floor(u);
  if (i < 0) i = 0;
  const double* c = kCaTab + (long)i * MPDPFT_CA_DEG;
  const int n = MPDPFT_CA_DEG;
  std::vector<double> d1(n + 1, 0.), d2(n + 1, 0.);
  for (int k = n - 1; k >= 1; --k) d1[k - 1] = d1[k + 1] + 2. * k * c[k];
  d1[0] *= 0.5;
  for (int k = n - 1; k >= 1; --k) d2[k - 1] = d2[k + 1] + 2. * k * d1[k];
  d2[0] *= 0.5;
  const double t = 2. * (u - i) - 1., g = 2. / MPDPFT_CA_W;
  ai = -g * cheb(d1.data(), n, t);
  aip = -g * g * cheb(d2.data(), n, t);
}

struct NAiT {  // the arguments nAiTintegrand takes beside x (MD:3580)
  double prefactor, U, ar, prefactor2, T, compare, rtpna;
  int bp, max_iter;
};

double nAiT_integrand(const NAiT& a, double x) {  // MD:3614-3619, EnergyQ = 0
  const double arg = -(a.U - x * a.ar) / a.T;
  return a.prefactor * CurlyA(x) * (polylog(2, arg) + a.prefactor2 * polylog(4, arg));
}

double boole_1d(const std::vector<double>& f, int Lf, double a1, double b1, int bp) {  // MD:8050-8058
  const double h = (b1 - a1) / (bp * 4.);
  double res = 7. * f[0];
  for (int i = 1; i <= Lf - 4; i += 4) res += (32. * f[i] + 12. * f[i + 1] + 32. * f[i + 2] + 14. * f[i + 3]);
  res -= 14. * f[Lf - 1];
  res += 7. * f[Lf - 1];
  return res * (2. * h / 45.);
}

bool negligible_magnitude_q(double big, double small, double max_exp) {  // MD:7094-7101
  if (small == 0.) return true;
  if (big == 0. || big < small) return false;
  return std::log10(std::fabs(big)) - std::log10(std::fabs(small)) > max_exp;
}

// AdaptiveBoole_nAiT (MD:3553-3578), recursive as the reference
double adaptive_boole(const NAiT& A, double a, double b, double prev, int iter) {
  const int BP = A.bp, n = 4 * BP + 1;
  const double half = 0.5 * (b - a), Delta = 0.25 * half / (double)BP;
  std::vector<double> fa(n), fb(n);
  for (int yi = 0; yi < n; ++yi) {
    const double x = a + (double)yi * Delta;
    fa[yi] = nAiT_integrand(A, x);
    fb[yi] = nAiT_integrand(A, x + half);
  }
  const double Inta = boole_1d(fa, n, a, a + half, BP);
  const double Intb = boole_1d(fb, n, a + half, b, BP);
  const double Int = Inta + Intb;
  if (iter > 1 && std::fabs(Int) > 0. && std::fabs((Int - prev) / Int) < A.rtpna) return Int;
  if (iter > A.max_iter) return Int;
  if (negligible_magnitude_q(A.compare, std::pow(2., (double)iter) * Int, -std::log10(A.rtpna))) return Int;
  if (Delta < MP) return Int;
  return adaptive_boole(A, a, a + half, Inta, iter + 1) + adaptive_boole(A, a + half, b, Intb, iter + 1);
}

// getDenEnAt, DIM 3, EnergyQ = 0, Units 1 (alpha = 1, tweak = 1), MD:3365-3441
double den_nAiT(const State& st, int s, long i, double mu) {
  const mpdpft_params& P = st.P;
  const double T = st.T[s], tau = 1. / T;
  const double beta0 = -P.degeneracy / std::pow(2. * PI, 1.5), beta1 = std::pow(tau, -1.5);
  const double U = st.V[s][i] - mu, ar = 0.5 * std::cbrt(st.Grad2[s][i]);
  const double beta2 = -st.Lap[s][i] / (12. * std::sqrt(tau));
  double res;
  if (ar < std::fabs(P.airy_threshold)) {
    const double arg = -tau * U;
    res = beta0 * (beta1 * polylog(1, arg) + beta2 * polylog(3, arg));
  } else {
    NAiT A;
    A.prefactor = beta0 * ar * tau * beta1;
    A.prefactor2 = beta2 / beta1;
    A.U = U;
    A.ar = ar;
    A.T = T;
    A.compare = P.abundances[s] / std::pow(P.edge, (double)P.dim);  // AverageDensity (MD:1003)
    A.rtpna = P.internal_acc;
    A.bp = P.boole_pairs;
    A.max_iter = P.boole_max_iter;
    double test = 1., x = -1.;
    while (std::fabs(test) > MP) {  // lower integration limit (MD:3424-3433)
      x *= 2.;
      const double arg = -tau * (U - x * ar);
      test = beta0 * CurlyA(x) * ar * tau * (beta1 * polylog(2, arg) + beta2 * polylog(4, arg));
      if (x < -1.0e8) break;
    }
    res = adaptive_boole(A, 2. * x, x, 0., 0);
    res += adaptive_boole(A, x, 100., 0., 0);
  }
  return res != res ? 0. : res;
}

void density(State& st, int s) {
  const mpdpft_params& P = st.P;
  const long G = st.G;
  const int D = st.D;
  const double g = P.degeneracy;
  std::vector<double>& n = st.Den[s];
  const std::vector<double>& V = st.V[s];
  const double mu = st.mu[s];
  if (P.density_expression == MPDPFT_DENS_TF) {  // GetTFdensity MD:4415-4436
    double pref = D == 1 ? std::sqrt(2.) * g / PI : (D == 2 ? g / (2. * PI) : std::sqrt(2.) * g / (3. * PI * PI));
#pragma omp parallel for schedule(static)
    for (long i = 0; i < G; ++i) {
      double t = mu - V[i];
      n[i] = t > 0. ? (D == 2 ? pref * t : pref * t * std::sqrt(t)) : 0.;
    }
  } else if (P.density_expression == MPDPFT_DENS_TF_INSPIRED ||
             P.density_expression == MPDPFT_DENS_TF_INSPIRED_T) {  // MD:3318-3347
    const double pref = 1. / P.tau[s];
    const double T = st.T[s];
#pragma omp parallel for schedule(static)
    for (long i = 0; i < G; ++i) {
      double t = (mu - V[i]) * pref;
      if (!std::isfinite(t)) t = 0.;
      if (P.density_expression == MPDPFT_DENS_TF_INSPIRED) {
        if (t > 0.) n[i] = D == 2 ? t : (D == 3 ? t * std::sqrt(t) / std::sqrt(pref) : std::sqrt(pref * t));
        else n[i] = 0.;
      } else {
        double t2 = t / T;
        if (std::fabs(t2) < 40.) n[i] = pref * T * std::log(1. + EXPc(t2));
        else if (t2 <= -40. || t2 != t2) n[i] = 0.;
        else n[i] = pref * t;
      }
    }
  } else if (P.density_expression == MPDPFT_DENS_GRADIENT) {
    if (!(st.del_valid >> s & 1u)) {  // DelField(V[s]) is independent of mu: computed once per V[s]
      delfield(st, V, st.Grad2[s], st.Lap[s]);
      st.del_valid |= 1u << s;
    }
    const std::vector<double>& lap = st.Lap[s];
    const std::vector<double>& g2 = st.Grad2[s];
    if (D == 2) {  // getDenEnAt small-gradient branch, 2D (MD:3376-3384)
      const double tau = 1. / st.T[s];
#pragma omp parallel for schedule(static)
      for (long i = 0; i < G; ++i) {
        double U = V[i] - mu, arg = -tau * U;
        double zeta = EXPc(-arg), LOG;
        if (arg < -100.) LOG = 1. / zeta;
        else if (arg > 100.) LOG = arg;
        else LOG = std::log(1. + 1. / zeta);
        double r = g / (2. * PI) * (LOG / tau - tau * lap[i] / 12. * zeta / ((1. + zeta) * (1. + zeta)));
        n[i] = (r != r) ? 0. : r;
      }
    } else if (P.gradient_form == MPDPFT_GRADIENT_FINITE_T) {  // MD:3365-3441
#pragma omp parallel for schedule(dynamic, 256)
      for (long i = 0; i < G; ++i) n[i] = den_nAiT(st, s, i, mu);
    } else {  // T -> 0 limit of the small-gradient branch in 3D (MD:3385-3386)
      const double floor_u = P.gradient_floor;
      const double c2 = P.gradient_grad2;
      const double ctf = g * 2. * std::sqrt(2.) / (6. * PI * PI);
      const double cg = g * std::sqrt(2.) / (48. * PI * PI);
#pragma omp parallel for schedule(static)
      for (long i = 0; i < G; ++i) {
        double u = mu - V[i];
        if (u <= 0.) { n[i] = 0.; continue; }
        // Below the floor f the singular factors continue linearly to 0 at the
        // turning point: u^{-1/2} -> u f^{-3/2}, u^{-3/2} -> u f^{-5/2}.
        double m1, m3;
        if (u >= floor_u) { m1 = 1. / std::sqrt(u); m3 = m1 / u; }
        else { double rf = 1. / std::sqrt(floor_u); m1 = u * rf / floor_u; m3 = m1 / floor_u; }
        double r = ctf * u * std::sqrt(u) - cg * (lap[i] * m1 + 0.25 * c2 * g2[i] * m3);
        n[i] = (r > 0.) ? r : 0.;
      }
    }
  }
}

void get_density_and_abundance(State& st, int s) {
  density(st, s);
  st.tmp_ab[s] = integrate(st, st.Den[s]);
  st.mu_trials++;
}

// e^{-x} I0(x), x >= 0, for the 2D compensation term (gsl_sf_bessel_I0 times
// EXP(-x) at MD:2659): the power series of I0 below x = 30 (positive terms),
// the asymptotic series (2 pi x)^{-1/2} sum [(2k-1)!!]^2 / (k! (8x)^k) above.
double i0e(double x) {
  if (x < 30.) {
    const double q = 0.25 * x * x;
    double t = 1., sum = 1.;
    for (int k = 1; k < 200 && t >= 1e-17 * sum; ++k) {
      t *= q / ((double)k * k);
      sum += t;
    }
    return sum * std::exp(-x);
  }
  double t = 1., sum = 1.;
  for (int k = 1; k < 40 && t >= 1e-17 * sum; ++k) {
    t *= (2. * k - 1.) * (2. * k - 1.) / (8. * k * x);
    sum += t;
  }
  return sum / std::sqrt(2. * PI * x);
}

// ------------------------------------------ Hartree MD:2583-2717 --------
// Coulomb potential of rho, gammaH * int rho(r')/|r-r'| (no prefactor here).
// 2D (HartreeType 0, MD:2636-2665): n~ -> (n~ - n~0 e^{-k^2})/k (imaginary
// part / k), k = 0 -> 0, then 2 pi (IFT + n~0 e^{-z^2/8} I0(z^2/8)/(4 sqrt pi)).
void coulomb(State& st, const std::vector<double>& rho, std::vector<double>& out) {
  const long G = st.G;
  for (long i = 0; i < G; ++i) st.CF[i] = cplx(rho[i], 0.);
  fft_parallel(st, -1, st.CF);
  const double f0 = st.CF[st.centre].real();
  if (st.D == 2) {
    const double kmin = 0.00001 * st.dk;
#pragma omp parallel for schedule(static)
    for (long i = 0; i < G; ++i) {
      double k = std::sqrt(knorm2(st, i));
      if (k > kmin) st.CF[i] = cplx((st.CF[i].real() - f0 * EXPc(-k * k)) / k, st.CF[i].imag() / k);
      else st.CF[i] = cplx(0., 0.);
    }
    fft_parallel(st, +1, st.CF);
    out.resize(G);
#pragma omp parallel for schedule(static)
    for (long i = 0; i < G; ++i) {
      double r3[3];
      coords(st, i, r3);
      const double z2 = r3[0] * r3[0] + r3[1] * r3[1];
      const double x = z2 / 8.;
      const double ebi = x < 1.0e+300 ? i0e(x) : 1. / std::sqrt(2. * PI * x);
      out[i] = 2. * PI * (st.CF[i].real() + f0 * ebi / (4. * std::sqrt(PI)));
    }
    return;
  }
  if (st.P.coulomb_kernel == MPDPFT_COULOMB_REGULARISED) {
    const double kzero = 0.000001 * st.dk * st.dk;
#pragma omp parallel for schedule(static)
    for (long i = 0; i < G; ++i) {
      double q2 = knorm2(st, i);
      if (q2 > kzero) st.CF[i] = cplx((st.CF[i].real() - f0 * EXPc(-q2)) / q2, st.CF[i].imag() / q2);
      else st.CF[i] = cplx(f0, 0.);
    }
    fft_parallel(st, +1, st.CF);
    out.resize(G);
#pragma omp parallel for schedule(static)
    for (long i = 0; i < G; ++i) {
      double r3[3];
      coords(st, i, r3);
      double z = std::sqrt(r3[0] * r3[0] + r3[1] * r3[1] + r3[2] * r3[2]);
      double zf = z > 1.0e-10 ? PI * std::erf(z / 2.) / z : std::sqrt(PI);
      out[i] = 4. * PI * (st.CF[i].real() + f0 * zf / (4. * PI * PI));
    }
  } else {  // truncated kernel 4 pi (1 - cos kR)/k^2, K(0) = 2 pi R^2
    const double R = st.P.coulomb_cutoff > 0. ? st.P.coulomb_cutoff : 0.5 * st.L;
#pragma omp parallel for schedule(static)
    for (long i = 0; i < G; ++i) {
      double q2 = knorm2(st, i);
      double K = q2 > 0. ? 4. * PI * (1. - std::cos(std::sqrt(q2) * R)) / q2 : 2. * PI * R * R;
      st.CF[i] *= K;
    }
    fft_parallel(st, +1, st.CF);
    out.resize(G);
    for (long i = 0; i < G; ++i) out[i] = st.CF[i].real();
  }
}

// ------------------------------------------------ getVint MD:2240-2318 --
void vint(State& st, int type, int ss, std::vector<double>& out) {
  const mpdpft_params& P = st.P;
  const long G = st.G;
  out.assign(G, 0.);
  if (type == MPDPFT_INT_CONTACT_MUTUAL) {
    for (int s = 0; s < st.S; ++s)
      if (s != ss)
        for (long i = 0; i < G; ++i) out[i] += st.Den[s][i];
    for (long i = 0; i < G; ++i) out[i] *= P.beta;
  } else if (type == MPDPFT_INT_CONTACT_SELF) {
    for (long i = 0; i < G; ++i) out[i] = st.Den[0][i] * 2. * P.beta;
  } else if (type == MPDPFT_INT_HARTREE) {
    coulomb(st, st.Den[ss], out);
    for (long i = 0; i < G; ++i) out[i] *= P.gamma_h;
  } else if (type == MPDPFT_INT_HARTREE_INTER) {
    std::vector<double> tmp;
    for (int s = 0; s < st.S; ++s)
      if (s != ss) {
        coulomb(st, st.Den[s], tmp);
        for (long i = 0; i < G; ++i) out[i] += P.gamma_h * tmp[i];
      }
  } else if (type == MPDPFT_INT_COULOMB_CHARGED) {
    std::vector<double> rho(G, 0.), tmp;
    for (int s = 0; s < st.S; ++s)
      for (long i = 0; i < G; ++i) rho[i] += P.charges[s] * st.Den[s][i];
    coulomb(st, rho, tmp);
    for (long i = 0; i < G; ++i) out[i] = P.charges[ss] * P.gamma_h * tmp[i];
  } else if (type == MPDPFT_INT_DIRAC) {
    const double DD = (double)st.D;
    for (long i = 0; i < G; ++i)
      out[i] = -P.gamma_h * (2. * std::pow(POS(st.Den[ss][i]) * DD / PI, 1. / DD)) / (DD - 1.);
  }
}

// --------------------------------------------------- UpdateV MD:4815 ----
void update_v(State& st) {
  std::vector<double> tmp;
  for (int s = 0; s < st.S; ++s) {
    std::vector<double>& V = st.V[s];
    std::fill(V.begin(), V.end(), 0.);
    for (int a = 0; a < st.P.n_interactions; ++a) {
      vint(st, st.P.interactions[a], s, tmp);
      for (long i = 0; i < st.G; ++i) V[i] += tmp[i];
    }
    if (st.incV < 1.)
      for (long i = 0; i < st.G; ++i) V[i] *= st.incV;
    for (long i = 0; i < st.G; ++i) V[i] += st.Env[s][i];
  }
  if (st.sc_count > 0) st.incV += st.incV0;  // MD:4833
  st.incV = std::min(1., st.incV);
  st.del_valid = 0;
}

// ------------------------------------ EnforceConstraints MD:4569-4743 --
void enforce_constraints(State& st) {
  st.trapped = false;
  if (!(st.P.rel_acc > MP)) return;
  const int S = st.S;
  double relacc = st.P.rel_acc;
  st.prev_mu = st.mu;
  {
    double nrm = 0.;
    for (int s = 0; s < S; ++s) nrm += st.prev_mu[s] * st.prev_mu[s];
    if (std::sqrt(nrm) < MP)
      for (int s = 0; s < S; ++s) st.prev_mu[s] = SIGN(st.prev_mu[s]) * MP;
  }
  double min_dmu = std::fabs(st.mu[0]);
  const int MAXRANGE = 20;
  std::vector<double> muMIN = st.mu, muMAX = st.mu, Dmu = st.mu;
  std::vector<int> minF(S, 0), maxF(S, 0);
  bool abort = false;
  const double* Ab = st.P.abundances;
  for (int s = 0; s < S; ++s) {
    double diff0 = std::fabs(st.tmp_ab[s] - Ab[s]);
    if (diff0 / std::fabs(2. * Ab[s]) > relacc) {
      int rc = 0;
      while (st.tmp_ab[s] > Ab[s] && rc < MAXRANGE) {
        maxF[s] = 1;
        if (st.mu[s] < muMAX[s]) muMAX[s] = st.mu[s];
        Dmu[s] = EXPc(st.dmm) * (1. + (double)rc) * std::fabs(st.prev_mu[s]);
        st.mu[s] -= Dmu[s];
        if (std::fabs(st.mu[s]) > 1.0e+20) { st.mu[s] = st.prev_mu[s]; break; }
        get_density_and_abundance(st, s);
        rc++;
        if (rc == 1) {
          double diff1 = std::fabs(st.tmp_ab[s] - Ab[s]);
          st.dmm -= SIGN(diff1 - diff0) * 0.1 * std::fabs(st.dmm);
        }
        muMIN[s] = st.mu[s];
      }
      if (st.tmp_ab[s] <= Ab[s]) minF[s] = 1;
      rc = 0;
      if (!maxF[s]) {
        while (st.tmp_ab[s] < Ab[s] && rc < MAXRANGE) {
          minF[s] = 1;
          if (std::fabs(st.mu[s]) > 1.0e+100) { st.mu[s] = st.prev_mu[s]; break; }
          if (st.mu[s] > muMIN[s]) muMIN[s] = st.mu[s];
          Dmu[s] = EXPc(st.dmm) * (1. + (double)rc) * std::fabs(st.prev_mu[s]);
          st.mu[s] += Dmu[s];
          if (std::fabs(st.mu[s]) > 1.0e+20) { st.mu[s] = st.prev_mu[s]; break; }
          get_density_and_abundance(st, s);
          rc++;
          if (rc == 1) {
            double diff1 = std::fabs(st.tmp_ab[s] - Ab[s]);
            st.dmm -= SIGN(diff1 - diff0) * 0.1 * std::fabs(st.dmm);
          }
          muMAX[s] = st.mu[s];
        }
      }
      if (st.tmp_ab[s] >= Ab[s]) maxF[s] = 1;
      if (!maxF[s] || !minF[s]) {
        st.mu[s] = st.prev_mu[s];
        abort = true;
        st.status_bits |= 1 << MPDPFT_ERR_MU_BRACKET;
        break;
      }
    }
  }
  if (!abort) {
    for (int s = 0; s < S; ++s) {
      Dmu[s] = 0.5 * (muMAX[s] - muMIN[s]);
      st.mu[s] = 0.5 * (muMIN[s] + muMAX[s]);
    }
    for (int s = 0; s < S; ++s) {
      double diff0 = std::fabs(st.tmp_ab[s] - Ab[s]);
      if (diff0 / std::fabs(2. * Ab[s]) > st.relacc_orig) {
        bool success = false, too_small = false;
        std::vector<double> hist;
        while (!success && !too_small) {
          success = true;
          get_density_and_abundance(st, s);
          if (st.tmp_ab[s] > 0.) hist.push_back(st.tmp_ab[s]);
          int trap = 0;
          if (hist.size() > 5) {
            int hs = (int)hist.size();
            for (int h = hs - 5; h < hs - 1 && !trap; ++h)
              for (int hp = hs - 5; hp < hs - 1; ++hp)
                if (h >= 0 && hp > h && std::fabs(hist[h] - hist[hp]) < st.relacc_orig * Ab[s]) {
                  trap++;
                  st.trapped = true;
                  st.status_bits |= 1 << MPDPFT_WARN_MU_TRAPPED;
                  break;
                }
          }
          if (trap) break;
          for (int sg = -1; sg < 2; sg += 2) {
            if ((double)sg * (st.tmp_ab[s] - Ab[s]) / std::fabs(2. * Ab[s]) > st.relacc_orig) {
              double old = st.mu[s];
              st.mu[s] -= (double)sg * 0.5 * Dmu[s];
              if (std::fabs(st.mu[s]) > 1.0e+20) { st.mu[s] = st.prev_mu[s]; break; }
              Dmu[s] = std::fabs(st.mu[s] - old);
              if (Dmu[s] < min_dmu) min_dmu = Dmu[s];
              if (std::fabs(Dmu[s]) < MP) { too_small = true; break; }
              success = false;
            }
          }
        }
      }
    }
  }
  for (int s = 0; s < S; ++s)
    if (!std::isfinite(st.mu[s])) st.mu[s] = st.prev_mu[s];
  (void)relacc;
}

void get_densities(State& st) {  // MD:3306-3316
  for (int s = 0; s < st.S; ++s) get_density_and_abundance(st, s);
  enforce_constraints(st);
}

// ------------------------------------------- CheckConvergence MD:4759 --
double reldev(const std::vector<double>& a, const std::vector<double>& b) {  // MD:4784
  double aa = vecmult(a, a), bb = vecmult(b, b);
  if (aa + bb > MP) return 1. - 2. * vecmult(a, b) / (aa + bb);
  return 0.;
}

double v_residual(const State& st) {  // rms of V - OldV over the periodic points
  double worst = 0.;
  for (int s = 0; s < st.S; ++s) {
    double acc = 0.;
    long cnt = 0;
    for (long i = 0; i < st.G; ++i) {
      double r3[3];
      long ii = st.D == 3 ? i / ((long)st.EL * st.EL) : i / st.EL;
      long jj = st.D == 3 ? (i / st.EL) % st.EL : i % st.EL;
      long kk = st.D == 3 ? i % st.EL : 0;
      (void)r3;
      if (ii == st.s || jj == st.s || kk == st.s) continue;
      double d = st.V[s][i] - st.OldV[s][i];
      acc += d * d;
      cnt++;
    }
    worst = std::max(worst, std::sqrt(acc / (double)cnt));
  }
  return worst;
}

void check_convergence(State& st, double vres) {
  const double mp = 100. * MACHINE_PRECISION;
  if (st.sc_count > 0) {
    st.cc = 0.;
    double tot = 0.;
    for (int s = 0; s < st.S; ++s) tot += st.tmp_ab[s];
    double maxtest = 0.;
    for (int s = 0; s < st.S; ++s) {
      double t = reldev(st.Den[s], st.OldDen[s]) * st.tmp_ab[s] / tot;
      if (t > maxtest) { maxtest = t; st.cc = maxtest; }
    }
    double dab = 0., dmu = 0.;
    for (int s = 0; s < st.S; ++s) {
      dab += (st.tmp_ab[s] - st.old_ab[s]) * (st.tmp_ab[s] - st.old_ab[s]);
      dmu += (st.mu[s] - st.old_mu[s]) * (st.mu[s] - st.old_mu[s]);
    }
    int steady = (st.cc < mp && std::sqrt(dab) < mp && std::sqrt(dmu) < mp) ? 1 : 0;
    double avtheta = 0.;
    for (int s = 0; s < st.S; ++s) avtheta += st.theta[s] / st.S;
    bool vres_ok = !(st.P.potential_tol > 0.) || vres <= st.P.potential_tol;
    if ((tot > mp || (tot <= mp && (double)st.sc_count * avtheta > 1.)) && st.P.sc_criterion >= 0. &&
        (st.cc < st.P.sc_criterion || steady) && vres_ok)
      st.exit_count++;
    else
      st.exit_count = 0;
    if (st.exit_count >= 3) st.exit_loop = 1;
  } else {
    st.cc = 1.2345678901234567890;
  }
}

// ------------------------------------------------- Pulay MD:5005-5167 ---
// Inverse of a small matrix by Gaussian elimination with full pivoting.
// Rank test as Eigen's FullPivHouseholderQR::isInvertible: every pivot
// above eps * n * |largest pivot|.
bool small_inverse(int n, const std::vector<double>& A, std::vector<double>& inv) {
  std::vector<double> M(A);
  inv.assign(n * n, 0.);
  for (int i = 0; i < n; ++i) inv[i * n + i] = 1.;
  std::vector<int> colperm(n);
  for (int i = 0; i < n; ++i) colperm[i] = i;
  double maxpiv = 0.;
  std::vector<double> piv(n);
  for (int c = 0; c < n; ++c) {
    int pr = c, pc = c;
    double best = -1.;
    for (int i = c; i < n; ++i)
      for (int j = c; j < n; ++j)
        if (std::fabs(M[i * n + j]) > best) { best = std::fabs(M[i * n + j]); pr = i; pc = j; }
    if (pr != c) {
      for (int j = 0; j < n; ++j) { std::swap(M[pr * n + j], M[c * n + j]); std::swap(inv[pr * n + j], inv[c * n + j]); }
    }
    if (pc != c) {
      for (int i = 0; i < n; ++i) std::swap(M[i * n + pc], M[i * n + c]);
      std::swap(colperm[pc], colperm[c]);
    }
    piv[c] = M[c * n + c];
    maxpiv = std::max(maxpiv, std::fabs(piv[c]));
    if (piv[c] == 0.) return false;
    double ip = 1. / piv[c];
    for (int j = 0; j < n; ++j) { M[c * n + j] *= ip; inv[c * n + j] *= ip; }
    for (int i = 0; i < n; ++i) {
      if (i == c) continue;
      double f = M[i * n + c];
      if (f == 0.) continue;
      for (int j = 0; j < n; ++j) { M[i * n + j] -= f * M[c * n + j]; inv[i * n + j] -= f * inv[c * n + j]; }
    }
  }
  const double thr = std::numeric_limits<double>::epsilon() * (double)n * maxpiv;
  for (int c = 0; c < n; ++c)
    if (std::fabs(piv[c]) <= thr) return false;
  // undo the column permutation: rows of the inverse follow colperm
  std::vector<double> out(n * n);
  for (int c = 0; c < n; ++c)
    for (int j = 0; j < n; ++j) out[colperm[c] * n + j] = inv[c * n + j];
  inv.swap(out);
  return true;
}

int pulay_mixer(State& st) {
  const int S = st.S;
  st.nin.push_back(st.OldDen);
  st.nout.push_back(st.Den);
  int I = (int)st.nout.size();
  std::vector<std::vector<double>> r(S, std::vector<double>(st.G));
  for (int s = 0; s < S; ++s)
    for (long i = 0; i < st.G; ++i) r[s][i] = st.nout[I - 1][s][i] - st.nin[I - 1][s][i];
  st.res.push_back(r);
  int shift = 0;
  if (I > st.P.pulay_scope) {
    st.res.erase(st.res.begin());
    st.nin.erase(st.nin.begin());
    st.nout.erase(st.nout.begin());
    I--;
    shift = 1;
  }
  std::vector<std::vector<double>> copy = st.gram;
  st.gram.assign(I, std::vector<double>(I, 0.));
  std::vector<double> B(I * I);
  for (int i = 0; i < I; ++i)
    for (int j = 0; j < I; ++j) {
      if (i == I - 1 || j == I - 1) {
        double acc = 0.;
        for (int s = 0; s < S; ++s) acc += vecmult(st.res[i][s], st.res[j][s]);
        st.gram[i][j] = acc;
      } else {
        st.gram[i][j] = copy[i + shift][j + shift];
      }
      B[i * I + j] = st.gram[i][j];
    }
  std::vector<double> inv;
  int success = 1;
  st.coeff.assign(I, 0.);
  if (small_inverse(I, B, inv)) {
    double test = 0.;
    for (int i = 0; i < I; ++i)
      for (int j = 0; j < I; ++j) {
        double acc = 0.;
        for (int k = 0; k < I; ++k) acc += inv[i * I + k] * B[k * I + j];
        double d = acc - (i == j ? 1. : 0.);
        test += d * d;
      }
    if (test > 1.0e-8) success = 0;
    if (success) {
      std::vector<double> x(I, 0.);
      double A = 0.;
      for (int i = 0; i < I; ++i) {
        for (int k = 0; k < I; ++k) x[i] += inv[i * I + k];
        A += x[i];
      }
      for (int i = 0; i < I; ++i) st.coeff[i] = x[i] / A;
    }
  } else {
    success = 0;
  }
  return success;
}

int admix(State& st) {  // AdmixDensities MD:4921-4992
  const int S = st.S;
  double nrmA = 0., nrmD = 0.;
  for (int s = 0; s < S; ++s) {
    nrmA += st.P.abundances[s] * st.P.abundances[s];
    nrmD += (st.P.abundances[s] - st.tmp_ab[s]) * (st.P.abundances[s] - st.tmp_ab[s]);
  }
  double reldiff = std::sqrt(nrmD) / std::sqrt(nrmA), mod = 1.;
  if (reldiff > MP) mod = std::min(1., std::pow(std::fabs(1. - reldiff), 30.));
  if (st.trapped)
    for (int s = 0; s < S; ++s) st.theta[s] *= mod;
  int pulay = 0;
  if (st.P.mixer > 0 && st.sc_count > 0) pulay = pulay_mixer(st);
  if (pulay > 0) {
    const int I = (int)st.coeff.size();
#pragma omp parallel for schedule(static)
    for (long i = 0; i < st.G; ++i)
      for (int s = 0; s < S; ++s) {
        double acc = 0.;
        for (int p = 0; p < I; ++p)
          acc += st.coeff[p] * ((1. - st.theta[s]) * st.nin[p][s][i] + st.theta[s] * st.nout[p][s][i]);
        st.Den[s][i] = acc;
      }
  } else {
    if (st.P.mixer > 0 && st.sc_count > 0) st.status_bits |= 1 << MPDPFT_ERR_PULAY_SINGULAR;
#pragma omp parallel for schedule(static)
    for (long i = 0; i < st.G; ++i)
      for (int s = 0; s < S; ++s)
        st.Den[s][i] = st.theta[s] * st.Den[s][i] + (1. - st.theta[s]) * st.OldDen[s][i];
  }
  if (st.trapped)
    for (int s = 0; s < S; ++s) st.theta[s] /= mod;
  return pulay;
}

void inject_schedule(State& st) {  // MD:5229-5315, schedules 5 and 9
  if (st.P.schedule == 5) {
    for (int s = 0; s < st.S; ++s) {
      if (st.cc < st.old_cc) st.theta[s] *= 1.1;
      else st.theta[s] *= 0.5;
      st.theta[s] = std::max(10. / (double)st.P.max_sc_count, std::min(0.8, st.theta[s]));
    }
  } else if (st.P.schedule == 9) {
    const double maxTheta = 0.2;
    for (int s = 0; s < st.S; ++s)
      if (st.theta[s] < maxTheta)
        st.theta[s] = st.theta0[s] + (maxTheta - st.theta0[s]) * (double)st.sc_count / (double)st.P.max_sc_count;
  }
}

// --------------------------------------------------------- energies ----
// Kinetic energy of the gradient-corrected density (GetDispersalEnergy,
// DensityExpression 5, MD:5606-5703), units 1 (alpha = 1).
//  2D (MD:5608-5621): E1 - int V n + mu N, E1 = int g/2 [lap CurlyA(y)/(12 pi)
//     - |grad V|^{4/3} (y^2 CurlyA(y) + Ai(y) + y Ai'(y))/(8 pi)],
//     y = 2 (V - mu) / |grad V|^{2/3}, 0 where |grad V|^2 <= MP, Ai = Ai' = 0
//     from y = 50.
//  3D EkinAiT03D (MD:5647-5703): g/(4 pi^2) int T, T = (2u)^{5/2}/5 -
//     lap (2u)^{1/2}/6 (u = mu - V > 0, else 0) where a = |grad V|^{2/3}/2 <
//     Mpp[2] (the T -> 0 form: everywhere), else the Airy-weighted integral
//     int_0^{x1} Ai(x + U/a) [(2ax)^{5/2}/5 - lap (2ax)^{1/2}/6] dx, U = V - mu,
//     x1 = max(1, 100 - U/a), by the trapezoid rule on 64, 128, ... points
//     until two agree (ASYMcritABS < MP) or MaxIteration doublings; the whole
//     integral again with MaxIteration + 1 ... (4 .. 10) until two agree to
//     max(RelAcc, MP).
double ekin_gradient(State& st, int s, double e_env) {
  const mpdpft_params& P = st.P;
  const long G = st.G;
  const double g = P.degeneracy, mu = st.mu[s];
  const std::vector<double>& V = st.V[s];
  const std::vector<double>& lap = st.Lap[s];
  const std::vector<double>& g2 = st.Grad2[s];
  std::vector<double> tmp(G);
  if (st.D == 2) {
    for (long i = 0; i < G; ++i) {
      const double U = V[i] - mu, ab = std::fabs(g2[i]);
      if (ab > MP) {
        const double y = 2. * U / std::cbrt(ab);
        double ai = 0., aip = 0.;
        if (y < 50.) airy_ai_d(y, ai, aip);
        const double ca = CurlyA(y);
        tmp[i] = 0.5 * g * (lap[i] * ca / (12. * PI) - std::pow(ab, 2. / 3.) * (y * y * ca + ai + y * aip) / (8. * PI));
      } else {
        tmp[i] = 0.;
      }
    }
    const double e1 = integrate(st, tmp);
    for (long i = 0; i < G; ++i) tmp[i] = V[i] * st.Den[s][i];
    return e1 - integrate(st, tmp) + mu * st.tmp_ab[s];
  }
  const bool airy = P.gradient_form == MPDPFT_GRADIENT_FINITE_T;
  const double thr = airy ? std::fabs(P.airy_threshold) : 1.0e300;
  const double pref = g / (4. * PI * PI), area = std::pow(P.edge, 3.);
  auto asym = [](double x, double y) { return (x == 0. && y == 0.) ? 0. : (x - y) / (x + y); };
  auto asym_abs = [](double x, double y, double crit) {
    return (std::fabs(x) < crit && std::fabs(y) < crit) ? 0. : std::fabs((x - y) / (x + y));
  };
  auto negligible = [](double big, double small, double max_exp) {
    if (small == 0.) return true;
    if (big == 0. || big < small) return false;
    return std::log10(std::fabs(big)) - std::log10(std::fabs(small)) > max_exp;
  };
  double e = 0., eprev = 0.;
  for (int outer = 0, maxit = 4;; ++outer, ++maxit) {
#pragma omp parallel for schedule(dynamic, 256)
    for (long i = 0; i < G; ++i) {
      const double U = V[i] - mu, a = 0.5 * std::cbrt(std::fabs(g2[i]));
      if (a < thr) {
        const double w = 2. * (-U);
        tmp[i] = -U > 0. ? w * w * std::sqrt(w) / 5. - lap[i] * std::sqrt(w) / 6. : 0.;
        continue;
      }
      const double x1 = std::max(1., 100. - U / a);
      double prev = 1., res = 0.;
      for (int it = 0, n = 64;; ++it, n *= 2) {
        const double h = x1 / (double)(n - 1);
        double sum = 0.;
        for (int j = 0; j < n; ++j) {
          const double x = (double)j * h, y = x + U / a;
          double ai = 0., aip;
          if (!(y > 100.)) {
            if (y > -300.) airy_ai_d(y, ai, aip);
            else ai = std::cos(2. * (-y) * std::sqrt(-y) / 3. - 0.25 * PI) / (std::sqrt(PI) * std::pow(-y, 0.25));
          }
          const double w = 2. * a * x;
          const double f = ai * (w * w * std::sqrt(w) / 5. - lap[i] * std::sqrt(w) / 6.);
          sum += (j == 0 || j == n - 1) ? 0.5 * f : f;
        }
        res = sum * h;
        if (it > 0 && (asym_abs(res, prev, MP) < MP ||
                       (std::fabs(asym(res, prev)) < P.internal_acc &&
                        negligible(e_env, area * pref * res, -std::log(P.internal_acc)))))
          break;
        if (it == maxit) break;
        prev = res;
      }
      tmp[i] = res;
    }
    e = pref * integrate(st, tmp);
    if (!airy) break;  // no Airy points: MaxIteration does not enter
    if (outer > 0 && std::fabs(asym(e, eprev)) < std::max(P.rel_acc, MP)) break;
    if (maxit >= 10) break;
    eprev = e;
  }
  return e;
}

void energy(State& st, mpdpft_result* res) {
  const mpdpft_params& P = st.P;
  const int D = st.D;
  const long G = st.G;
  std::vector<double> tmp(G), vh;
  double etot = 0.;
  for (int a = 0; a < P.n_interactions && a < MPDPFT_MAX_INTERACTIONS; ++a) {
    int type = P.interactions[a];
    double e = 0.;
    if (type == MPDPFT_INT_CONTACT_MUTUAL) {
      for (int s = 0; s < st.S; ++s)
        for (int sp = s + 1; sp < st.S; ++sp) {
          for (long i = 0; i < G; ++i) tmp[i] = st.Den[s][i] * st.Den[sp][i];
          e += integrate(st, tmp);
        }
      e *= P.beta;
    } else if (type == MPDPFT_INT_CONTACT_SELF) {
      for (long i = 0; i < G; ++i) tmp[i] = st.Den[0][i] * st.Den[0][i];
      e = P.beta * integrate(st, tmp);
    } else if (type == MPDPFT_INT_HARTREE) {
      std::fill(tmp.begin(), tmp.end(), 0.);
      for (int s = 0; s < st.S; ++s) {
        coulomb(st, st.Den[s], vh);
        for (long i = 0; i < G; ++i) tmp[i] += 0.5 * P.gamma_h * vh[i] * st.Den[s][i];
      }
      e = integrate(st, tmp);
    } else if (type == MPDPFT_INT_HARTREE_INTER) {
      std::fill(tmp.begin(), tmp.end(), 0.);
      for (int s = 0; s < st.S; ++s)
        for (int sp = 0; sp < st.S; ++sp)
          if (sp != s) {
            coulomb(st, st.Den[sp], vh);
            for (long i = 0; i < G; ++i) tmp[i] += 0.5 * P.gamma_h * vh[i] * st.Den[s][i];
          }
      e = integrate(st, tmp);
    } else if (type == MPDPFT_INT_COULOMB_CHARGED) {
      std::vector<double> rho(G, 0.);
      for (int s = 0; s < st.S; ++s)
        for (long i = 0; i < G; ++i) rho[i] += P.charges[s] * st.Den[s][i];
      coulomb(st, rho, vh);
      for (long i = 0; i < G; ++i) tmp[i] = 0.5 * P.gamma_h * vh[i] * rho[i];
      e = integrate(st, tmp);
    } else if (type == MPDPFT_INT_DIRAC) {
      const double DD = (double)D;
      const double cXD = 2. * std::sqrt(4. * PI) / ((DD - 1.) * PI) *
                         std::pow(0.5 * std::pow(0.75 * std::sqrt(PI), DD - 2.), 1. / DD);
      std::fill(tmp.begin(), tmp.end(), 0.);
      for (int s = 0; s < st.S; ++s)
        for (long i = 0; i < G; ++i)
          tmp[i] += -P.gamma_h * cXD * DD / (1. + DD) * std::pow(POS(st.Den[s][i]), 1. + 1. / DD);
      e = integrate(st, tmp);
    }
    res->e_interaction[a] = e;
    etot += e;
  }
  const double DD = (double)D;
  const double AF = D == 2 ? 2. * PI : 4. * PI;
  for (int s = 0; s < st.S; ++s) {
    for (long i = 0; i < G; ++i) tmp[i] = st.Env[s][i] * st.Den[s][i];
    double eenv = integrate(st, tmp);
    double ekin;
    if (D == 2 && (P.density_expression == MPDPFT_DENS_TF_INSPIRED || P.density_expression == MPDPFT_DENS_TF_INSPIRED_T)) {
      for (long i = 0; i < G; ++i) tmp[i] = st.Den[s][i] * st.Den[s][i];
      ekin = 0.5 * P.tau[s] * integrate(st, tmp);
    } else if (P.density_expression == MPDPFT_DENS_GRADIENT) {
      ekin = ekin_gradient(st, s, eenv);
    } else {  // TF potential functional, MD:5741-5750 (U = 1)
      for (long i = 0; i < G; ++i) {
        double t = st.mu[s] - st.V[s][i];
        tmp[i] = t > 0. ? std::pow(t, (DD + 2.) / 2.) : 0.;
      }
      ekin = P.degeneracy * AF * std::pow(2., (DD + 2.) / 2.) /
             (std::pow(2. * PI, DD) * (2. * DD + 4.)) * integrate(st, tmp);
    }
    res->e_kinetic[s] = ekin;
    res->e_external[s] = eenv;
    etot += ekin + eenv;
  }
  res->e_total = etot;
}

void fill_result(State& st, mpdpft_result* r) {
  r->iterations = st.sc_count;
  r->cc = st.cc;
  for (int s = 0; s < st.S; ++s) { r->mu[s] = st.mu[s]; r->abundance[s] = st.tmp_ab[s]; }
  energy(st, r);
}

}  // namespace

// ======================================================== C interface ====
extern "C" {

// fftParallel on a complex field in the reference layout ((s+1)^D,
// interleaved re/im), in place.
void oracle_fft(const mpdpft_params* p, int sign, double* field) {
  State st;
  init_state(st, *p);
  std::vector<cplx> cf(st.G);
  for (long i = 0; i < st.G; ++i) cf[i] = cplx(field[2 * i], field[2 * i + 1]);
  fft_parallel(st, sign, cf);
  for (long i = 0; i < st.G; ++i) { field[2 * i] = cf[i].real(); field[2 * i + 1] = cf[i].imag(); }
}

// Plain unnormalised s^D transform (the oracle's own FFT engine).
void oracle_fft_raw(int dim, int s, int sign, double* data) {
  fft_nd(dim, s, sign, reinterpret_cast<cplx*>(data));
}

double oracle_integrate(const mpdpft_params* p, const double* f) {
  State st;
  init_state(st, *p);
  std::vector<double> v(f, f + st.G);
  return integrate(st, v);
}

void oracle_delfield(const mpdpft_params* p, const double* f, double* grad2, double* lap) {
  State st;
  init_state(st, *p);
  std::vector<double> v(f, f + st.G), g2, l;
  delfield(st, v, g2, l);
  std::memcpy(grad2, g2.data(), sizeof(double) * st.G);
  std::memcpy(lap, l.data(), sizeof(double) * st.G);
}

// n[V] at mu for species s; returns N = Integrate(n).
double oracle_density(const mpdpft_params* p, int s, const double* v, double mu, double* n_out) {
  State st;
  init_state(st, *p);
  st.V[s].assign(v, v + st.G);
  st.mu[s] = mu;
  density(st, s);
  std::memcpy(n_out, st.Den[s].data(), sizeof(double) * st.G);
  return integrate(st, st.Den[s]);
}

// getVint for focal species s; dens holds S consecutive grids.
void oracle_vint(const mpdpft_params* p, int type, int s, const double* dens, double* out) {
  State st;
  init_state(st, *p);
  for (int q = 0; q < st.S; ++q) st.Den[q].assign(dens + q * st.G, dens + (q + 1) * st.G);
  std::vector<double> o;
  vint(st, type, s, o);
  std::memcpy(out, o.data(), sizeof(double) * st.G);
}

// EnforceConstraints for all species from potentials v (S grids) and the
// starting mu in p->mu.  Writes mu, N, trials and densities.
static int g_last_status_bits = 0;

// status bits of the last oracle_mu_search (MPDPFT_WARN_MU_TRAPPED: the
// bisection ended on the reference's trap test)
int oracle_last_status_bits() { return g_last_status_bits; }

int oracle_mu_search(const mpdpft_params* p, const double* v, double* mu_out, double* ab_out,
                     double* dens_out, double* deltamu_modifier_io) {
  State st;
  init_state(st, *p);
  st.status_bits = 0;
  if (deltamu_modifier_io) st.dmm = *deltamu_modifier_io;
  for (int q = 0; q < st.S; ++q) st.V[q].assign(v + q * st.G, v + (q + 1) * st.G);
  get_densities(st);
  for (int q = 0; q < st.S; ++q) {
    mu_out[q] = st.mu[q];
    ab_out[q] = st.tmp_ab[q];
    if (dens_out) std::memcpy(dens_out + q * st.G, st.Den[q].data(), sizeof(double) * st.G);
  }
  if (deltamu_modifier_io) *deltamu_modifier_io = st.dmm;
  g_last_status_bits = st.status_bits;
  return (int)st.mu_trials;
}

// Full SC solve (GetData's loop).  vext, v0: S grids each (v0 may be NULL).
// Outputs: result, per-iteration log, final densities and potentials.
int oracle_sc_run(const mpdpft_params* p, const double* vext, const double* v0,
                  mpdpft_result* result, mpdpft_iter_log* log, int log_cap,
                  double* dens_out, double* v_out) {
  State st;
  init_state(st, *p);
  for (int q = 0; q < st.S; ++q) {
    st.Env[q].assign(vext + q * st.G, vext + (q + 1) * st.G);
    if (v0) st.V[q].assign(v0 + q * st.G, v0 + (q + 1) * st.G);
    else st.V[q] = st.Env[q];
  }
  for (int q = 0; q < st.S; ++q)  // automatic temperature (MD:4523-4528) from the start V
    if (st.T[q] < 0.) {
      double vmin = st.V[q][0], vmax = st.V[q][0];
      for (long i = 0; i < st.G; ++i) { vmin = std::min(vmin, st.V[q][i]); vmax = std::max(vmax, st.V[q][i]); }
      st.T[q] = std::max(std::fabs(st.mu[q] - vmin), std::fabs(st.mu[q] - vmax)) / 50.;
    }
  std::memset(result, 0, sizeof(*result));
  st.del_valid = 0;
  get_densities(st);  // initial densities, MD:195
  long total_trials = st.mu_trials;
  int logged = 0;
  while (!st.exit_loop) {
    st.status_bits = 0;
    long trials0 = st.mu_trials;
    auto t_iter = std::chrono::steady_clock::now();
    st.OldDen = st.Den; st.OldV = st.V;   // StoreCurrentIteration MD:4804
    st.old_mu = st.mu; st.old_ab = st.tmp_ab; st.old_cc = st.cc;
    update_v(st);
    double vres = v_residual(st);
    get_densities(st);
    check_convergence(st, vres);
    if (st.sc_count == st.P.max_sc_count) st.exit_loop = 1;  // Intercept MD:4866
    int pul = admix(st);
    inject_schedule(st);
    if (log && logged < log_cap) {
      mpdpft_iter_log& L = log[logged++];
      std::memset(&L, 0, sizeof(L));
      L.sc_count = st.sc_count;
      L.mu_trials = (int)(st.mu_trials - trials0);
      L.pulay_used = pul;
      L.status_bits = st.status_bits;
      L.cc = st.cc;
      L.v_residual = vres;
      L.ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_iter).count();
      for (int q = 0; q < st.S; ++q) { L.mu[q] = st.mu[q]; L.abundance[q] = st.tmp_ab[q]; L.theta[q] = st.theta[q]; }
    }
    result->v_residual = vres;
    st.sc_count++;  // PrepareNextIteration MD:5317
  }
  total_trials = st.mu_trials;
  fill_result(st, result);
  result->iterations = st.sc_count;
  result->converged = st.exit_count >= 3 ? 1 : 0;
  result->total_mu_trials = (int)total_trials;
  for (int q = 0; q < st.S; ++q) {
    if (dens_out) std::memcpy(dens_out + q * st.G, st.Den[q].data(), sizeof(double) * st.G);
    if (v_out) std::memcpy(v_out + q * st.G, st.V[q].data(), sizeof(double) * st.G);
  }
  return logged;
}

// Energies of given densities/potentials/mu (GetEnergy MD:5414).
void oracle_energy(const mpdpft_params* p, const double* vext, const double* dens,
                   const double* v, const double* mu, mpdpft_result* result) {
  State st;
  init_state(st, *p);
  for (int q = 0; q < st.S; ++q) {
    st.Env[q].assign(vext + q * st.G, vext + (q + 1) * st.G);
    st.Den[q].assign(dens + q * st.G, dens + (q + 1) * st.G);
    st.V[q].assign(v + q * st.G, v + (q + 1) * st.G);
    st.mu[q] = mu[q];
    st.tmp_ab[q] = integrate(st, st.Den[q]);
    if (p->density_expression == MPDPFT_DENS_GRADIENT) delfield(st, st.V[q], st.Grad2[q], st.Lap[q]);
  }
  std::memset(result, 0, sizeof(*result));
  energy(st, result);
}

// Pulay mixing sequence: feed `iters` pairs (n_in, n_out) of one species
// (each a grid) through AdmixDensities with sc_count = 1.. and return the
// mixed densities and the last coefficients.
int oracle_pulay_sequence(const mpdpft_params* p, int iters, const double* nin, const double* nout,
                          double* mixed, double* coeffs, int* ncoeff, int* used) {
  State st;
  init_state(st, *p);
  const long G = st.G;
  const int S = st.S;
  for (int t = 0; t < iters; ++t) {
    for (int q = 0; q < S; ++q) {
      st.OldDen[q].assign(nin + ((long)t * S + q) * G, nin + ((long)t * S + q + 1) * G);
      st.Den[q].assign(nout + ((long)t * S + q) * G, nout + ((long)t * S + q + 1) * G);
      st.tmp_ab[q] = st.P.abundances[q];
    }
    st.sc_count = t;
    used[t] = admix(st);
    for (int q = 0; q < S; ++q) std::memcpy(mixed + ((long)t * S + q) * G, st.Den[q].data(), sizeof(double) * G);
  }
  *ncoeff = (int)st.coeff.size();
  for (size_t i = 0; i < st.coeff.size(); ++i) coeffs[i] = st.coeff[i];
  return 0;
}

int oracle_num_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

// The special functions and one point of the finite-T gradient density
// (species 0 of p, temperature T, u = mu - V), for the known-answer tests.
double oracle_polylog(int order, double x) { return polylog(order, x); }
double oracle_curly_a(double x) { return CurlyA(x); }
double oracle_i0e(double x) { return i0e(x); }
void oracle_airy(double x, double* ai, double* aip) { airy_ai_d(x, *ai, *aip); }
double oracle_finite_t_point(const mpdpft_params* p, double T, double u, double lap, double grad2) {
  State st;
  mpdpft_params q = *p;
  q.steps = 2;
  q.dim = 3;
  init_state(st, q);
  st.T[0] = T;
  st.V[0].assign(st.G, 0.);
  st.Lap[0].assign(st.G, lap);
  st.Grad2[0].assign(st.G, grad2);
  st.P.edge = p->edge;
  st.P.dim = p->dim;
  return den_nAiT(st, 0, 0, u);
}

// OpenMP threads of later oracle calls (<= 0: all host threads).
void oracle_set_threads(int n) {
#ifdef _OPENMP
  omp_set_num_threads(n > 0 ? n : omp_get_num_procs());
#else
  (void)n;
#endif
}

}  // extern "C"
