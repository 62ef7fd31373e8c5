// fft.cu -- FFT kernels and the FFT-based operators of the engine:
// Coulomb (Hartree) potentials, DelField (spectral gradient, Laplacian and
// Gaussian smoothing with the boundary taper) and the reference-convention
// complex transform of fftParallel.
//
// A D-dimensional real transform is split into passes over global memory:
//   Z  R2C along the contiguous axis (s reals -> s/2+1 complex per row), with
//      a fused prologue (taper, species charge sum) and the row sums needed
//      for the k = 0 mode;
//   Y  C2C along y (3D only), in place, batched over fields;
//   X  C2C along x as a round trip: forward FFT, k-space multiplier(s),
//      inverse FFT, without leaving shared memory;
//   Y  inverse, then Z C2R with a fused epilogue (|grad f|^2 + Laplacian,
//      positivity clamp, Coulomb compensation term).
// The half spectrum is stored [x][y][kz], kz = 0..s/2.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdlib>
#include <cstring>
#include <array>
#include <cstdio>
#include <map>
#include <mutex>
#include <set>
#include <tuple>
#include <string>
#include <vector>

#include "batch.h"
#include "engine.h"
#include "fft.cuh"

namespace mpdpft {

#define CU(call)                                                                         \
  do {                                                                                   \
    cudaError_t e_ = (call);                                                             \
    if (e_ != cudaSuccess)                                                               \
      return set_error(MPDPFT_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

constexpr int kFftThreads = 256;

// Raise a kernel's dynamic shared memory limit to the device's per-block
// opt-in maximum minus the kernel's static shared memory (once per kernel).
template <typename F>
static cudaError_t smem_optin(F* fn) {
  static std::mutex mu;
  static std::set<const void*> done;
  std::lock_guard<std::mutex> lock(mu);
  if (done.count((const void*)fn)) return cudaSuccess;
  int dev = 0, optin = 0;
  cudaGetDevice(&dev);
  cudaError_t e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  if (e != cudaSuccess) return e;
  cudaFuncAttributes at;
  if ((e = cudaFuncGetAttributes(&at, fn)) != cudaSuccess) return e;
  e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, optin - (int)at.sharedSizeBytes);
  if (e == cudaSuccess) done.insert((const void*)fn);
  return e;
}

// ------------------------------------------------------------ plan ------
static bool factor(int len, RadixPlan& p) {
  p.len = len;
  p.n = 0;
  int m = len;
  while (m % 4 == 0 && p.n < kMaxRadixStages) { p.r[p.n++] = 4; m /= 4; }
  while (m % 2 == 0 && p.n < kMaxRadixStages) { p.r[p.n++] = 2; m /= 2; }
  while (m % 3 == 0 && p.n < kMaxRadixStages) { p.r[p.n++] = 3; m /= 3; }
  return m == 1;
}

struct FftPlan {
  int dim, s, M, H;     // M = s/2, H = s/2 + 1
  long rows;            // s^{dim-1} rows of the contiguous axis
  long nspec;           // complex elements of one half spectrum
  RadixPlan plan_s, plan_m;
  void* tw_s_f = nullptr;  // forward / inverse twiddles of length s (compute precision)
  void* tw_s_b = nullptr;
  void* tw_m_f = nullptr;  // of length M
  void* tw_m_b = nullptr;
  void* tw_n_f = nullptr;  // e^{-2 pi i q/s}, q < s  (R2C split)
  int zl;                  // rows per block in the Z passes
  int tk;                  // lines per tile in the Y/X passes
  void* spec[4] = {nullptr, nullptr, nullptr, nullptr};  // half spectra
  void* rtmp = nullptr;    // real scratch field
  double* zpart = nullptr; // per-block sums of the Z pass input
  int zblocks = 0;
  unsigned long long* vmax = nullptr;  // ordered-bits max of the taper shell
  double* vres_part = nullptr;         // V assembly |dV|^2 partials
  int vblocks = 0;
  void* cbuf = nullptr;    // complex s^D field for the fftParallel op
  int zparts = 0;          // block sums in zpart written by the last forward pass
  bool plane = false;      // 3D transforms by x-planes (k_plane_fwd / k_plane_inv)
  double tune_ms[2] = {0.0, 0.0};  // autotuner: transforms of one iteration, plane / pass path
  int tuned = 0;                   // 0: one path only, 1: measured now, 2: from the cache, 3: forced
};


// ---------------------------------------------------------- prologues ----
enum { PRO_NONE = 0, PRO_TAPER = 1, PRO_CHARGE = 2 };
// EPI_COULOMB_V: the Coulomb epilogue followed by the V assembly of one
// species (k_assemble_v fused into the transform; plane kernels only)
enum { EPI_STORE = 0, EPI_POS = 1, EPI_GRAD = 2, EPI_COULOMB = 3, EPI_SCALE = 4, EPI_COULOMB_V = 5 };
// MUL_LAP: the Laplacian output of MUL_DERIV alone (one output)
// MUL_COULOMB_2D: the reference's 2D kernel (n~ - n~0 e^{-k^2})/k, k = 0 -> 0
enum { MUL_COULOMB_REG = 0, MUL_COULOMB_TRUNC = 1, MUL_DERIV = 2, MUL_SMOOTH = 3, MUL_LAP = 4, MUL_COULOMB_2D = 5 };

template <typename R>
struct ZArgs {
  Geom g;
  int M, H, zl;
  long rows;
  RadixPlan plan;
  const typename Cx<R>::T* tw_m;  // length-M table (forward for R2C, inverse for C2R)
  const typename Cx<R>::T* tw_n;  // e^{-2 pi i q/s}
  // R2C
  const R* in;                    // real input [nsrc][n] (PRO_CHARGE sums nsrc)
  int nsrc;
  double qcoef[kMaxS];
  int pro;
  double taper_r0, taper_a;       // taper: r > r0 -> * exp(a (r - r0)^2)
  const unsigned long long* vmax; // shift for the taper
  typename Cx<R>::T* out;         // half spectrum
  double* part;                   // per-block input sums (may be null)
  // C2R
  const typename Cx<R>::T* cin[4];
  int nin;
  int epi;
  R* rout[2];
  double scale;
  double coul_coef;               // Coulomb epilogue: out = coef (x + f0 erf(r/2)/(4 pi r))
  const double* f0_part;          // Z-pass partials giving f0 = dvol * sum(input)
  int f0_blocks;
  // plane kernels
  const typename Cx<R>::T* tw_s;  // length-s table for the y transforms
  int* err;                       // raised when a bulk copy does not complete
  // EPI_COULOMB_V (one species): V = vext + min(1, inc_v) (vh + pointwise
  // terms of ncur); |V_new - V_old|^2 block sums and the shell maximum of V
  const ScState* st;
  const R* vext;
  const R* ncur;
  R* vpot;
  double beta, gamma_h;
  int contact_self, dirac;
  double shell_r, shell_w;
  double* vres_part;              // [blocks][kMaxS]
  unsigned long long* vmax_out;
  int coul_reg;                   // 1: regularised kernel (erf term), 0: truncated (plain scale)
  const int* skip;                // batched launches: nonzero -> this solve has finished (no work)
};

// R2C along the contiguous axis.  Block = zl rows; each row of s reals is
// read as M complex z_m = x_2m + i x_2m+1, transformed (length M) and split
// into the s/2 + 1 outputs X_q = E_q + e^{-2 pi i q/s} O_q.
// Input value of the R2C pass at element p (prologue: taper or charge sum).
// DelField boundary taper (mpDPFT.cpp:7251-7264) of value x at (px, py, pz).
template <typename R>
__device__ __forceinline__ R taper_xyz(const ZArgs<R>& a, double px, double py, double pz, R x, double shift) {
  if constexpr (sizeof(R) == sizeof(float)) {  // FP32 fields: the factor in FP32
    const float r = sqrtf(float(px) * float(px) + float(py) * float(py) + float(pz) * float(pz));
    float f = x - float(shift);
    const float dr = r - float(a.taper_r0);
    if (dr > 0.f) f *= expf(float(a.taper_a) * dr * dr);
    return R(f);
  } else {
    const double r = sqrt(px * px + py * py + pz * pz);
    double f = (double)x - shift;
    if (r > a.taper_r0) f *= exp(a.taper_a * (r - a.taper_r0) * (r - a.taper_r0));
    return R(f);
  }
}

template <typename R>
__device__ __forceinline__ R taper_value(const ZArgs<R>& a, long p, R x, double shift) {
  double px, py, pz;
  point_coords(p, a.g, px, py, pz);
  return taper_xyz<R>(a, px, py, pz, x, shift);
}

// Coulomb epilogue value at (x, y, z): coef (v + f0 pi erf(r/2)/r / (4 pi^2))
// (mpDPFT.cpp:2704-2711).
// 2D (mpDPFT.cpp:2657-2662): coef (v + f0 e^{-r^2/8} I0(r^2/8) / (4 sqrt pi)).
template <typename R>
__device__ __forceinline__ R coulomb_xyz(const ZArgs<R>& a, double x, double y, double z, R v, double f0) {
  if (a.g.dim == 2) {
    const double q = 0.125 * (x * x + y * y);
    return R(a.coul_coef * ((double)v + f0 * bessel_i0e(q) / (4.0 * 1.7724538509055159)));
  }
  if constexpr (sizeof(R) == sizeof(float)) {  // FP32 fields: the term in FP32
    const float r = sqrtf(float(x) * float(x) + float(y) * float(y) + float(z) * float(z));
    const float zf = r > 1.0e-10f ? float(kPi) * erff(0.5f * r) / r : float(1.7724538509055159);
    return R(float(a.coul_coef) * (v + float(f0 / (4.0 * kPi * kPi)) * zf));
  } else {
    const double r = sqrt(x * x + y * y + z * z);
    const double zf = r > 1.0e-10 ? kPi * erf(0.5 * r) / r : sqrt(kPi);
    return R(a.coul_coef * ((double)v + f0 * zf / (4.0 * kPi * kPi)));
  }
}

template <typename R>
__device__ __forceinline__ R z_input(const ZArgs<R>& a, long p, double shift) {
  R x;
  if (a.pro == PRO_CHARGE) {
    double t = 0.0;
    for (int q = 0; q < a.nsrc; ++q) t += a.qcoef[q] * (double)a.in[(long)q * a.g.n + p];
    x = R(t);
  } else {
    x = a.in[p];
  }
  if (a.pro == PRO_TAPER) x = taper_value<R>(a, p, x, shift);
  return x;
}

// R2C along the contiguous axis.  Block = zl rows; each row of s reals is
// read as M complex z_m = x_2m + i x_2m+1, transformed (length M) and split
// into the s/2 + 1 outputs X_q = E_q + e^{-2 pi i q/s} O_q.
template <typename R, int NC, int NL>
__device__ __forceinline__ void z_r2c_body(const ZArgs<R>& a, const long blk) {
  using C = typename Cx<R>::T;
  extern __shared__ unsigned char smem_raw[];
  const int M = NC > 0 ? NC : a.M;
  const int zl = NC > 0 ? NL : a.zl;
  const int H = M + 1;
  const long row0 = blk * zl;
  const int s = a.g.s;
  double shift = 0.0;  // no shell points: no shift
  if (a.pro == PRO_TAPER && *a.vmax != 0ull) shift = from_ordered_bits(*a.vmax);
  double rowsum = 0.0;
  C* Z;
  if constexpr (NC > 0) {
    C* A = reinterpret_cast<C*>(smem_raw);
    C* B = A + NC * (NL + 1);
    Z = B + NC * (NL + 1);
    C* tws = Z + NC * (NL + 1);
    for (int i = threadIdx.x; i < NC; i += blockDim.x) tws[i] = a.tw_m[i];
    __syncthreads();
    auto load = [&](int m, int l) -> C {
      const long row = row0 + l;
      if (row >= a.rows) return C{R(0), R(0)};
      const long p0 = row * s + 2 * m;
      R x0, x1;
      if (a.pro == PRO_NONE) {
        const C v = *reinterpret_cast<const C*>(a.in + p0);  // 2 reals, aligned (s even)
        x0 = v.x;
        x1 = v.y;
      } else {
        x0 = z_input<R>(a, p0, shift);
        x1 = z_input<R>(a, p0 + 1, shift);
      }
      rowsum += (double)x0 + (double)x1;
      return C{x0, x1};
    };
    auto store = [&](int m, int l, C v) { Z[m * (NL + 1) + l] = v; };
    fft_lines<C, NC, NL, true>(A, B, tws, -1, load, store);
    if (a.part) {
      double acc[1] = {rowsum};
      block_reduce_store<1>(acc, a.part + blk);
    }
  } else {
    C* A = reinterpret_cast<C*>(smem_raw);
    C* B = A + M * zl;
    for (int w = threadIdx.x; w < M * zl; w += blockDim.x) {
      const int l = w / M, m = w % M;
      const long row = row0 + l;
      C z = {R(0), R(0)};
      if (row < a.rows) {
        const long p0 = row * s + 2 * m;
        R x0 = z_input<R>(a, p0, shift), x1 = z_input<R>(a, p0 + 1, shift);
        rowsum += (double)x0 + (double)x1;
        z = {x0, x1};
      }
      A[m * zl + l] = z;
    }
    if (a.part) {
      double acc[1] = {rowsum};
      block_reduce_store<1>(acc, a.part + blk);
    }
    __syncthreads();
    Z = tile_fft<C>(A, B, a.plan, zl, a.tw_m, -1);
  }
  const int zld = NC > 0 ? NL + 1 : zl;  // row stride of the Z tile
  for (int w = threadIdx.x; w < H * zl; w += blockDim.x) {
    const int l = w / H, q = w % H;
    const long row = row0 + l;
    if (row >= a.rows) continue;
    C zq = Z[(q % M) * zld + l];
    C zc = cconj(Z[((M - q) % M) * zld + l]);
    C E = cscale(cadd(zq, zc), R(0.5));
    C D = csub(zq, zc);             // 2 i O_q
    C O = {D.y * R(0.5), -D.x * R(0.5)};
    C t = a.tw_n[q];               // e^{-2 pi i q/s}, q <= M < s
    a.out[row * H + q] = cadd(E, cmul(t, O));
  }
}

template <typename R, int NC, int NL>
__global__ void __launch_bounds__(kFftThreads) k_z_r2c(ZArgs<R> a) {
  pdl_wait();
  z_r2c_body<R, NC, NL>(a, blockIdx.x);
  pdl_trigger();
}

// Batched launch: blockIdx.y selects the transform's arguments (one solve
// and species of a batch, all with the same grid size).
__device__ __forceinline__ bool batch_skip(const int* skip) { return skip && __ldcg(skip) != 0; }

template <typename R, int NC, int NL>
__global__ void __launch_bounds__(kFftThreads) k_z_r2c_b(const ZArgs<R>* __restrict__ args) {
  const ZArgs<R>& a = args[blockIdx.y];
  if (batch_skip(a.skip)) return;
  z_r2c_body<R, NC, NL>(a, blockIdx.x);
}

// Epilogue value of the C2R pass at element p (single-field epilogues).
template <typename R>
__device__ __forceinline__ R z_output(const ZArgs<R>& a, long p, R v, double f0) {
  if (a.epi == EPI_POS) return v > R(0) ? v : R(0);
  if (a.epi == EPI_SCALE) return R(a.coul_coef * (double)v);
  if (a.epi == EPI_COULOMB) {
    double x, y, z;
    point_coords(p, a.g, x, y, z);
    return coulomb_xyz<R>(a, x, y, z, v, f0);
  }
  return v;
}

// C2R along the contiguous axis for nin half-spectrum rows, with epilogue.
template <typename R, int NC, int NL>
__device__ __forceinline__ void z_c2r_body(const ZArgs<R>& a, const long blk) {
  using C = typename Cx<R>::T;
  extern __shared__ unsigned char smem_raw[];
  const int M = NC > 0 ? NC : a.M;
  const int zl = NC > 0 ? NL : a.zl;
  const int H = M + 1;
  const long row0 = blk * zl;
  const int s = a.g.s;
  double f0 = 0.0;
  if (a.epi == EPI_COULOMB) {  // f0 = dvol * sum of the R2C pass's block sums (same order in every block)
    __shared__ double s_f0[kFftThreads / 32];
    double t = 0.0;
    for (int b = threadIdx.x; b < a.f0_blocks; b += blockDim.x) t += a.f0_part[b];
    t = warp_sum(t);
    if ((threadIdx.x & 31) == 0) s_f0[threadIdx.x >> 5] = t;
    __syncthreads();
    t = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += s_f0[w];
    f0 = t * a.g.dvol;
  }
  if constexpr (NC > 0) {
    C* A = reinterpret_cast<C*>(smem_raw);
    C* B = A + NC * (NL + 1);
    C* tws = B + NC * (NL + 1);
    R* acc = reinterpret_cast<R*>(tws + NC);  // [NL][s] (EPI_GRAD)
    for (int i = threadIdx.x; i < NC; i += blockDim.x) tws[i] = a.tw_m[i];
    __syncthreads();
    for (int f = 0; f < a.nin; ++f) {
      const C* X = a.cin[f];
      auto load = [&](int q, int l) -> C {
        const long row = row0 + l;
        if (row >= a.rows) return C{R(0), R(0)};
        C xq = X[row * H + q];
        C xc = cconj(X[row * H + (NC - q)]);
        C E = cadd(xq, xc);   // 2 E_q
        C D = csub(xq, xc);   // 2 e^{-2 pi i q/s} O_q
        C O = cmul(cconj(a.tw_n[q]), D);  // 2 O_q
        return C{E.x - O.y, E.y + O.x};   // 2 (E_q + i O_q)
      };
      auto store = [&](int m, int l, C z) {
        const long row = row0 + l;
        if (row >= a.rows) return;
        const R x0 = z.x * R(a.scale), x1 = z.y * R(a.scale);
        const long p0 = row * s + 2 * m;
        if (a.epi == EPI_GRAD) {
          R* dst = acc + (long)l * s + 2 * m;
          if (f == 0) { dst[0] = x0 * x0; dst[1] = x1 * x1; }
          else if (f < a.nin - 1) { dst[0] += x0 * x0; dst[1] += x1 * x1; }
          else {
            *reinterpret_cast<C*>(a.rout[0] + p0) = C{dst[0], dst[1]};
            *reinterpret_cast<C*>(a.rout[1] + p0) = C{x0, x1};
          }
        } else {
          *reinterpret_cast<C*>(a.rout[0] + p0) = C{z_output<R>(a, p0, x0, f0), z_output<R>(a, p0 + 1, x1, f0)};
        }
      };
      fft_lines<C, NC, NL, true>(A, B, tws, +1, load, store);
    }
  } else {
    C* A = reinterpret_cast<C*>(smem_raw);
    C* B = A + M * zl;
    R* acc = reinterpret_cast<R*>(B + M * zl);  // [zl][s]
    for (int f = 0; f < a.nin; ++f) {
      const C* X = a.cin[f];
      for (int w = threadIdx.x; w < M * zl; w += blockDim.x) {
        const int l = w / M, q = w % M;
        const long row = row0 + l;
        C z = {R(0), R(0)};
        if (row < a.rows) {
          C xq = X[row * H + q];
          C xc = cconj(X[row * H + (M - q)]);
          C E = cadd(xq, xc);
          C D = csub(xq, xc);
          C O = cmul(cconj(a.tw_n[q]), D);
          z = {E.x - O.y, E.y + O.x};
        }
        A[q * zl + l] = z;
      }
      __syncthreads();
      C* Z = tile_fft<C>(A, B, a.plan, zl, a.tw_m, +1);
      for (int w = threadIdx.x; w < M * zl; w += blockDim.x) {
        const int l = w / M, m = w % M;
        C z = Z[m * zl + l];
        R x0 = z.x * R(a.scale), x1 = z.y * R(a.scale);
        R* dst = acc + (long)l * s + 2 * m;
        if (a.epi == EPI_GRAD) {
          if (f == 0) { dst[0] = x0 * x0; dst[1] = x1 * x1; }
          else if (f < a.nin - 1) { dst[0] += x0 * x0; dst[1] += x1 * x1; }
          else {
            const long row = row0 + l;
            if (row < a.rows) {
              a.rout[0][row * s + 2 * m] = dst[0];
              a.rout[0][row * s + 2 * m + 1] = dst[1];
              a.rout[1][row * s + 2 * m] = x0;
              a.rout[1][row * s + 2 * m + 1] = x1;
            }
          }
        } else {
          dst[0] = x0;
          dst[1] = x1;
        }
      }
      __syncthreads();
    }
    if (a.epi == EPI_GRAD) return;
    for (int w = threadIdx.x; w < s * zl; w += blockDim.x) {
      const int l = w / s, k = w % s;
      const long row = row0 + l;
      if (row >= a.rows) continue;
      const long p = row * s + k;
      a.rout[0][p] = z_output<R>(a, p, acc[(long)l * s + k], f0);
    }
  }
}

template <typename R, int NC, int NL>
__global__ void __launch_bounds__(kFftThreads) k_z_c2r(ZArgs<R> a) {
  pdl_wait();
  z_c2r_body<R, NC, NL>(a, blockIdx.x);
  pdl_trigger();
}

template <typename R, int NC, int NL>
__global__ void __launch_bounds__(kFftThreads) k_z_c2r_b(const ZArgs<R>* __restrict__ args) {
  const ZArgs<R>& a = args[blockIdx.y];
  if (batch_skip(a.skip)) return;
  z_c2r_body<R, NC, NL>(a, blockIdx.x);
}

// Y or X pass arguments.  Lines run along an axis of stride `astride`
// (complex elements); a line is identified by (outer, col) with base
// outer * ostride + col, col in [0, H).  Blocks [0, nbulk) take tk adjacent
// columns of one outer index; the remaining blocks take the Nyquist column
// col = M of tk consecutive outer indices.
template <typename R>
struct AxisArgs {
  int s, M, H, tk, dim;
  long nouter, ostride, astride;
  int ntile;   // column tiles per outer index (M / tk)
  long nbulk;  // nouter * ntile
  RadixPlan plan;
  const typename Cx<R>::T* twf;
  const typename Cx<R>::T* twb;
  typename Cx<R>::T* data[4];  // Y pass: per field (blockIdx.y); X pass: input in data[0]
  int dir;                     // Y pass direction
  // X round trip
  int nout;
  typename Cx<R>::T* out[4];
  int mul;
  double sigma_c;       // Gaussian smoothing exponent (k^2 multiplier)
  double scale;         // 1 / s^D
  double dk;
  double cutoff;        // truncated Coulomb radius
  const double* f0_part;  // Z-pass input sums (Coulomb, k = 0 mode)
  int f0_blocks;
  const int* skip;        // batched launches: nonzero -> this solve has finished (no work)
  int o0;                 // output o uses multiplier o0 + o (one derivative or the Laplacian alone)
};

template <typename R>
__device__ __forceinline__ bool axis_line(const AxisArgs<R>& a, long b, int l, long& base, long& outer, int& col) {
  if (b < a.nbulk) {
    outer = b / a.ntile;
    col = (int)(b % a.ntile) * a.tk + l;
  } else {
    outer = (b - a.nbulk) * a.tk + l;
    col = a.M;
    if (l > 0 && a.nouter == 1) return false;
  }
  if (outer >= a.nouter) return false;
  base = outer * a.ostride + col;
  return true;
}

template <typename R, int NC, int NL>
__global__ void __launch_bounds__(kFftThreads) k_axis_c2c(AxisArgs<R> a) {
  pdl_wait();
  using C = typename Cx<R>::T;
  extern __shared__ unsigned char smem_raw[];
  const long blk = blockIdx.x;
  C* data = a.data[blockIdx.y];
  const C* twg = a.dir < 0 ? a.twf : a.twb;
  if constexpr (NC > 0) {
    C* A = reinterpret_cast<C*>(smem_raw);
    C* B = A + NC * (NL + 1);
    C* tws = B + NC * (NL + 1);
    __shared__ long s_base[NL];
    __shared__ int s_ok[NL];
    for (int i = threadIdx.x; i < NC; i += blockDim.x) tws[i] = twg[i];
    if (threadIdx.x < NL) {
      long base, outer;
      int col;
      s_ok[threadIdx.x] = axis_line(a, blk, threadIdx.x, base, outer, col) ? 1 : 0;
      s_base[threadIdx.x] = base;
    }
    __syncthreads();
    const long as = a.astride;
    auto load = [&](int t, int l) -> C {
      return s_ok[l] ? data[s_base[l] + t * as] : C{R(0), R(0)};
    };
    auto store = [&](int t, int l, C v) {
      if (s_ok[l]) data[s_base[l] + t * as] = v;
    };
    fft_lines<C, NC, NL, false>(A, B, tws, a.dir, load, store);
  } else {
    const int n = a.s;
    const int tk = a.tk;
    C* A = reinterpret_cast<C*>(smem_raw);
    C* B = A + n * tk;
    for (int w = threadIdx.x; w < n * tk; w += blockDim.x) {
      const int t = w / tk, l = w % tk;
      long base, outer;
      int col;
      C v = {R(0), R(0)};
      if (axis_line(a, blk, l, base, outer, col)) v = data[base + t * a.astride];
      A[t * tk + l] = v;
    }
    __syncthreads();
    C* res = tile_fft<C>(A, B, a.plan, tk, twg, a.dir);
    for (int w = threadIdx.x; w < n * tk; w += blockDim.x) {
      const int t = w / tk, l = w % tk;
      long base, outer;
      int col;
      if (axis_line(a, blk, l, base, outer, col)) data[base + t * a.astride] = res[t * tk + l];
    }
  }
}

// Signed frequency of stored index t of a length-s axis: t < s/2 -> t,
// else t - s.  The reference's k grid runs over -s/2 .. s/2 - 1, so the
// Nyquist index s/2 carries k = -pi/dx (mpDPFT.cpp:889-895).
__device__ __forceinline__ int signed_freq(int t, int s) { return t < s / 2 ? t : t - s; }

// k-space multiplier of the x round trip for element (t along x, line of
// outer index `outer`, column `col`) and output o; v is the forward
// transform value, the return value what the inverse transform receives.
template <typename R>
__device__ __forceinline__ typename Cx<R>::T apply_multiplier(const AxisArgs<R>& a, typename Cx<R>::T v, int t,
                                                             long outer, int col, int o, double f0) {
  using C = typename Cx<R>::T;
  const int qx = signed_freq(t, a.s);
  const int qy = a.dim == 3 ? signed_freq((int)outer, a.s) : 0;
  const double kx = a.dk * (t == a.s / 2 ? -(double)(a.s / 2) : (double)qx);
  const double ky = a.dk * (double)qy;
  const double kz = a.dk * (col == a.M ? -(double)a.M : (double)col);  // col M: Nyquist
  const double k2 = kx * kx + ky * ky + kz * kz;  // 2D: ky = 0, kz is the contiguous axis
  if (a.mul == MUL_COULOMB_2D) {
    // (n~ - n~0 e^{-k^2})/k on the real part, n~/k on the imaginary part,
    // k <= 1e-5 dk -> 0 (mpDPFT.cpp:2647-2657); phase as below
    const double k = sqrt(k2);
    if (k > 0.00001 * a.dk) {
      const int par = (t + col) & 1;
      const double g = exp(-k2) * f0 * (par ? -1.0 : 1.0);
      return C{R(((double)v.x - g) / k * a.scale), R((double)v.y / k * a.scale)};
    }
    return C{R(0), R(0)};
  }
  if (a.mul == MUL_COULOMB_REG) {
    // (n~ - n~0 e^{-k^2})/k^2, k = 0 -> n~0 (mpDPFT.cpp:2686-2701); the
    // centred transform's phase (-1)^{qx+qy+qz} carries over to the
    // subtracted Gaussian in this frame
    if (k2 > 1.0e-6 * a.dk * a.dk) {
      const int par = (t + (int)outer * (a.dim == 3) + col) & 1;
      const double g = exp(-k2) * f0 * (par ? -1.0 : 1.0);
      return C{R(((double)v.x - g) / k2 * a.scale), R((double)v.y / k2 * a.scale)};
    }
    return C{R(f0 * a.scale), R(0)};
  }
  double fr;
  bool imag = false;
  if (a.mul == MUL_COULOMB_TRUNC) {
    fr = k2 > 0.0 ? (1.0 - cos(sqrt(k2) * a.cutoff)) / k2 : 0.5 * a.cutoff * a.cutoff;
  } else if (a.mul == MUL_SMOOTH) {
    fr = exp(a.sigma_c * k2);
  } else {  // MUL_DERIV: outputs d/dx, d/dy (, d/dz), Laplacian; MUL_LAP: Laplacian
    const double sm = exp(a.sigma_c * k2);
    if (a.mul == MUL_DERIV && o < a.dim) {
      // i k_j: the reference takes Im of IFT(-k f~), which drops the
      // Nyquist index of axis j (mpDPFT.cpp:7442-7444)
      double kj;
      if (a.dim == 3) kj = (o == 0) ? (t == a.s / 2 ? 0.0 : kx) : (o == 1 ? ((int)outer == a.s / 2 ? 0.0 : ky) : (col == a.M ? 0.0 : kz));
      else kj = (o == 0) ? (t == a.s / 2 ? 0.0 : kx) : (col == a.M ? 0.0 : kz);
      fr = kj * sm;
      imag = true;
    } else {
      fr = -k2 * sm * sm;  // Laplacian smoothed twice (mpDPFT.cpp:7477, 7577)
    }
  }
  fr *= a.scale;
  if (imag) return C{R(-fr * (double)v.y), R(fr * (double)v.x)};
  return C{R(fr * (double)v.x), R(fr * (double)v.y)};
}

// Separable factors of the multipliers for one tile: per x index t (kx,
// e^{sigma kx^2}, e^{-kx^2}) and per line (ky, kz, the y-z parts of k^2,
// e^{sigma k^2} and e^{-k^2}, and the parity of qy + qz).
template <typename R, int NC, int NL>
struct MulTables {
  R kx[NC], ex[NC], gx[NC];
  R ky[NL], kz[NL], k2yz[NL], eyz[NL], gyz[NL];
  int par[NL];
};

template <typename R, int NC, int NL>
__device__ __forceinline__ typename Cx<R>::T apply_multiplier_tab(const AxisArgs<R>& a, const MulTables<R, NC, NL>& T,
                                                                 typename Cx<R>::T v, int t, int l, int o, double f0,
                                                                 long outer, int col) {
  using C = typename Cx<R>::T;
  const R sc = R(a.scale);
  if (a.mul == MUL_COULOMB_TRUNC) return apply_multiplier<R>(a, v, t, outer, col, o, f0);
  const R kx = T.kx[t];
  const R k2 = kx * kx + T.k2yz[l];
  if (a.mul == MUL_COULOMB_2D) {
    const R k = sqrt(k2);
    if ((double)k > 0.00001 * a.dk) {
      const int par = (t + T.par[l]) & 1;
      const R g = T.gx[t] * T.gyz[l] * R(f0) * (par ? R(-1) : R(1));
      const R ik = sc / k;
      return C{(v.x - g) * ik, v.y * ik};
    }
    return C{R(0), R(0)};
  }
  if (a.mul == MUL_COULOMB_REG) {
    if ((double)k2 > 1.0e-6 * a.dk * a.dk) {
      const int par = (t + T.par[l]) & 1;
      const R g = T.gx[t] * T.gyz[l] * R(f0) * (par ? R(-1) : R(1));
      const R ik = sc / k2;
      return C{(v.x - g) * ik, v.y * ik};
    }
    return C{R(f0) * sc, R(0)};
  }
  const R e = T.ex[t] * T.eyz[l];  // e^{sigma k^2}
  if (a.mul == MUL_SMOOTH) return C{v.x * e * sc, v.y * e * sc};
  // MUL_DERIV: i k_j e^{sigma k^2} (Nyquist of axis j dropped), Laplacian
  // -k^2 e^{2 sigma k^2}; MUL_LAP: the Laplacian alone
  if (a.mul == MUL_DERIV && o < a.dim) {
    R kj;
    if (o == 0) kj = (t == a.s / 2) ? R(0) : kx;
    else if (o == 1 && a.dim == 3) kj = T.ky[l];
    else kj = T.kz[l];
    const R fr = kj * e * sc;
    return C{-fr * v.y, fr * v.x};
  }
  const R fr = -k2 * e * e * sc;
  return C{fr * v.x, fr * v.y};
}

template <typename R, int NC, int NL>
__device__ __forceinline__ void x_roundtrip_body(const AxisArgs<R>& a, const long blk) {
  using C = typename Cx<R>::T;
  extern __shared__ unsigned char smem_raw[];
  __shared__ double s_f0;
  if (a.mul == MUL_COULOMB_REG || a.mul == MUL_COULOMB_2D) {
    if (threadIdx.x < 32) {
      double t = 0.0;
      for (int b = threadIdx.x; b < a.f0_blocks; b += 32) t += a.f0_part[b];
      t = warp_sum(t);
      if (threadIdx.x == 0) s_f0 = t;  // unnormalised k = 0 mode: sum of the input
    }
  }
  C* data = a.data[0];
  if constexpr (NC > 0) {
    C* A = reinterpret_cast<C*>(smem_raw);
    C* B = A + NC * (NL + 1);
    C* F = B + NC * (NL + 1);
    C* twf = F + NC * (NL + 1);
    C* twb = twf + NC;
    __shared__ long s_base[NL];
    __shared__ long s_outer[NL];
    __shared__ int s_col[NL];
    __shared__ int s_ok[NL];
    __shared__ MulTables<R, NC, NL> T;
    for (int i = threadIdx.x; i < NC; i += blockDim.x) {
      twf[i] = a.twf[i];
      twb[i] = a.twb[i];
      const double kx = a.dk * (i == NC / 2 ? -(double)(NC / 2) : (double)signed_freq(i, NC));
      T.kx[i] = R(kx);
      T.ex[i] = R(exp(a.sigma_c * kx * kx));
      T.gx[i] = R(exp(-kx * kx));
    }
    if (threadIdx.x < NL) {
      const int l = threadIdx.x;
      long base, outer;
      int col;
      s_ok[l] = axis_line(a, blk, l, base, outer, col) ? 1 : 0;
      s_base[l] = base;
      s_outer[l] = outer;
      s_col[l] = col;
      const double ky = a.dim == 3 ? a.dk * (double)signed_freq((int)outer, a.s) : 0.0;
      const double kz = a.dk * (col == a.M ? -(double)a.M : (double)col);  // col M: Nyquist
      const double k2 = ky * ky + (a.dim == 3 ? kz * kz : 0.0);
      // 2D: the single-outer layout puts the contiguous axis in col (its k
      // is "kz" here); the y slot is unused
      const double kyy = a.dim == 3 ? ky : kz;
      T.ky[l] = R(a.dim == 3 ? (((int)outer == a.s / 2) ? 0.0 : ky) : 0.0);
      T.kz[l] = R(col == a.M ? 0.0 : kz);
      T.k2yz[l] = R(a.dim == 3 ? k2 : kyy * kyy);
      T.eyz[l] = R(exp(a.sigma_c * (a.dim == 3 ? k2 : kyy * kyy)));
      T.gyz[l] = R(exp(-(a.dim == 3 ? k2 : kyy * kyy)));
      T.par[l] = ((a.dim == 3 ? (int)outer : 0) + col) & 1;
    }
    __syncthreads();
    const long as = a.astride;
    auto gload = [&](int t, int l) -> C { return s_ok[l] ? data[s_base[l] + t * as] : C{R(0), R(0)}; };
    auto fstore = [&](int t, int l, C v) { F[t * (NL + 1) + l] = v; };
    fft_lines<C, NC, NL, false>(A, B, twf, -1, gload, fstore);
    const double f0 = (a.mul == MUL_COULOMB_REG || a.mul == MUL_COULOMB_2D) ? s_f0 : 0.0;
    for (int o = 0; o < a.nout; ++o) {
      C* dst = a.out[o];
      auto mload = [&](int t, int l) -> C {
        C v = F[t * (NL + 1) + l];
        return s_ok[l] ? apply_multiplier_tab<R, NC, NL>(a, T, v, t, l, a.o0 + o, f0, s_outer[l], s_col[l]) : v;
      };
      auto gstore = [&](int t, int l, C v) { if (s_ok[l]) dst[s_base[l] + t * as] = v; };
      fft_lines<C, NC, NL, false>(A, B, twb, +1, mload, gstore);
    }
  } else {
    const int n = a.s;
    const int tk = a.tk;
    C* A = reinterpret_cast<C*>(smem_raw);
    C* B = A + n * tk;
    C* W = B + n * tk;
    for (int w = threadIdx.x; w < n * tk; w += blockDim.x) {
      const int t = w / tk, l = w % tk;
      long base, outer;
      int col;
      C v = {R(0), R(0)};
      if (axis_line(a, blk, l, base, outer, col)) v = data[base + t * a.astride];
      A[t * tk + l] = v;
    }
    __syncthreads();
    C* F = tile_fft<C>(A, B, a.plan, tk, a.twf, -1);
    C* spare = (F == A) ? B : A;  // two free buffers: spare and W
    const double f0 = (a.mul == MUL_COULOMB_REG || a.mul == MUL_COULOMB_2D) ? s_f0 : 0.0;
    for (int o = 0; o < a.nout; ++o) {
      for (int w = threadIdx.x; w < n * tk; w += blockDim.x) {
        const int t = w / tk, l = w % tk;
        long base, outer;
        int col;
        C v = F[t * tk + l];
        if (axis_line(a, blk, l, base, outer, col)) v = apply_multiplier<R>(a, v, t, outer, col, a.o0 + o, f0);
        spare[t * tk + l] = v;
      }
      __syncthreads();
      C* res = tile_fft<C>(spare, W, a.plan, tk, a.twb, +1);
      C* dst = a.out[o];
      for (int w = threadIdx.x; w < n * tk; w += blockDim.x) {
        const int t = w / tk, l = w % tk;
        long base, outer;
        int col;
        if (axis_line(a, blk, l, base, outer, col)) dst[base + t * a.astride] = res[t * tk + l];
      }
      __syncthreads();
    }
  }
}

template <typename R, int NC, int NL>
__global__ void __launch_bounds__(kFftThreads) k_x_roundtrip(AxisArgs<R> a) {
  pdl_wait();
  x_roundtrip_body<R, NC, NL>(a, blockIdx.x);
  pdl_trigger();
}

template <typename R, int NC, int NL>
__global__ void __launch_bounds__(kFftThreads) k_x_roundtrip_b(const AxisArgs<R>* __restrict__ args) {
  const AxisArgs<R>& a = args[blockIdx.y];
  if (batch_skip(a.skip)) return;
  x_roundtrip_body<R, NC, NL>(a, blockIdx.x);
}

// V assembly (UpdateV, mpDPFT.cpp:4815-4838) when Coulomb terms exist:
// V_s = Vext_s + incV (vh_s + contact + Dirac); partial sums of |dV|^2 and
// the maximum of V over the taper shell (DelField, mpDPFT.cpp:7253-7259).

// Body of the V assembly over blocks blk of nblk: species s < nmax also
// update their taper-shell maximum vmax[s]; update = 0 only takes the
// shell maxima of the current V (the DelField of the start potential).
template <typename R>
__device__ __forceinline__ void assemble_v_body(const KParams& kp, const ScState* st, const R* vext, const R* vh,
                                                const R* nin_ring, R* V, double* vres_part, unsigned long long* vmax,
                                                double shell_r, double shell_w, int nmax, int update, long blk,
                                                long nblk) {
  const long n = kp.geom.n;
  const int S = kp.S;
  if (__ldcg(&st->exit_loop)) return;
  const int cur = __ldcg(&st->slot);
  const double incv = __ldcg(&st->inc_v);
  const double fac = incv < 1.0 ? incv : 1.0;
  const R* nin = nin_ring + (long)cur * S * n;
  double acc[kMaxS], vm[kMaxS];
  for (int s = 0; s < kMaxS; ++s) { acc[s] = 0.0; vm[s] = -1.0e300; }
  // one 16-byte vector per field and thread per trip (NP points), every
  // load of a species issued before its arithmetic
  constexpr int NP = kVecPts<R>;
  const int vec = kp.vec4;
  for (long p0 = (blk * blockDim.x + threadIdx.x) * NP; p0 < n; p0 += nblk * blockDim.x * NP) {
    bool shell[NP];
#pragma unroll
    for (int t = 0; t < NP; ++t) {
      double x, y, z;
      point_coords(p0 + t, kp.geom, x, y, z);
      shell[t] = p0 + t < n && in_shell(x * x + y * y + z * z, shell_r, shell_w);
    }
    for (int s = 0; s < S; ++s) {
      R vnew[NP];
      if (update) {
        R vi[NP], ve[NP], vo[NP];
#pragma unroll
        for (int t = 0; t < NP; ++t) vi[t] = R(0);
        if (vh) vload(vh + (long)s * n, p0, n, vec, vi);
        vload(vext + (long)s * n, p0, n, vec, ve);
        vload(V + (long)s * n, p0, n, vec, vo);
        if (kp.contact_self) {  // type 10 (:2261)
          R a[NP];
          vload(nin, p0, n, vec, a);
#pragma unroll
          for (int t = 0; t < NP; ++t) vi[t] += R(2.0 * kp.beta) * a[t];
        }
        if (kp.contact_mutual) {  // type 1 (:2247)
          R tsum[NP];
#pragma unroll
          for (int t = 0; t < NP; ++t) tsum[t] = R(0);
          for (int q = 0; q < S; ++q) {
            if (q == s) continue;
            R a[NP];
            vload(nin + (long)q * n, p0, n, vec, a);
#pragma unroll
            for (int t = 0; t < NP; ++t) tsum[t] += a[t];
          }
#pragma unroll
          for (int t = 0; t < NP; ++t) vi[t] += R(kp.beta) * tsum[t];
        }
        if (kp.dirac) {  // type 11 (:2768)
          R a[NP];
          vload(nin + (long)s * n, p0, n, vec, a);
#pragma unroll
          for (int t = 0; t < NP; ++t) {
            const R ns = a[t] > R(0) ? a[t] : R(0);
            if (kp.geom.dim == 3) vi[t] += R(-kp.gamma_h) * cbrt(R(3.0 / kPi) * ns);
            else vi[t] += R(-2.0 * kp.gamma_h) * sqrt(R(2.0 / kPi) * ns);
          }
        }
#pragma unroll
        for (int t = 0; t < NP; ++t) {
          vnew[t] = ve[t] + R(fac) * vi[t];
          const double d = (double)vnew[t] - (double)vo[t];
          acc[s] += p0 + t < n ? d * d : 0.0;
        }
        vstore(V + (long)s * n, p0, n, vec, vnew);
      } else {
        vload(V + (long)s * n, p0, n, vec, vnew);
      }
      if (s < nmax) {
#pragma unroll
        for (int t = 0; t < NP; ++t)
          if (shell[t]) vm[s] = fmax(vm[s], (double)vnew[t]);
      }
    }
  }
  if (update) block_reduce_store<kMaxS>(acc, vres_part + blk * kMaxS);
  // block max -> global ordered max (order independent, so deterministic)
  __shared__ double sm[32];
  for (int s = 0; s < nmax; ++s) {
    double t = vm[s];
    for (int o = 16; o > 0; o >>= 1) t = fmax(t, __shfl_xor_sync(0xffffffffu, t, o));
    __syncthreads();
    if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = t;
    __syncthreads();
    if (threadIdx.x == 0) {
      double b = sm[0];
      for (int w = 1; w < (int)(blockDim.x >> 5); ++w) b = fmax(b, sm[w]);
      if (b > -1.0e300) atomicMax(vmax + s, ordered_bits(b));
    }
  }
}

// V assembly of one solve; the taper shift of species 0 (the others take
// k_shell_max before their DelField).
template <typename R>
__global__ void k_assemble_v(KParams kp, const ScState* st, const R* vext, const R* vh, const R* nin_ring, R* V,
                             double* vres_part, unsigned long long* vmax, double shell_r, double shell_w) {
  assemble_v_body<R>(kp, st, vext, vh, nin_ring, V, vres_part, vmax, shell_r, shell_w, 1, 1, blockIdx.x, gridDim.x);
}

// Shell maximum of a standalone field (the DelField entry point).
template <typename R>
__global__ void k_shell_max(Geom g, const R* f, unsigned long long* vmax, double shell_r, double shell_w) {
  double vm = -1.0e300;
  // four points per thread and trip; a value is read only inside the shell
  for (long p0 = ((long)blockIdx.x * blockDim.x + threadIdx.x) * 4; p0 < g.n; p0 += (long)gridDim.x * blockDim.x * 4) {
#pragma unroll
    for (int t = 0; t < 4; ++t) {
      const long p = p0 + t;
      double x, y, z;
      point_coords(p, g, x, y, z);
      if (p < g.n && in_shell(x * x + y * y + z * z, shell_r, shell_w)) vm = fmax(vm, (double)f[p]);
    }
  }
  for (int o = 16; o > 0; o >>= 1) vm = fmax(vm, __shfl_xor_sync(0xffffffffu, vm, o));
  if ((threadIdx.x & 31) == 0 && vm > -1.0e300) atomicMax(vmax, ordered_bits(vm));
}

// fftParallel phase factors on an s^D complex field: multiply by
// c * (-1)^{i+j+k}, c complex.
template <typename R>
__global__ void k_alternate(typename Cx<R>::T* f, Geom g, double cr, double ci) {
  for (long p = (long)blockIdx.x * blockDim.x + threadIdx.x; p < g.n; p += (long)gridDim.x * blockDim.x) {
    int k = (int)(p % g.s);
    long q = p / g.s;
    int par = k + (int)(q % g.s) + (g.dim == 3 ? (int)(q / g.s) : 0);
    double sg = (par & 1) ? -1.0 : 1.0;
    typename Cx<R>::T v = f[p];
    double x = (double)v.x, y = (double)v.y;
    f[p] = {R(sg * (cr * x - ci * y)), R(sg * (cr * y + ci * x))};
  }
}

template <typename R>
__global__ void k_cx_import(const double* src, typename Cx<R>::T* dst, long n) {
  for (long p = (long)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (long)gridDim.x * blockDim.x)
    dst[p] = {R(src[2 * p]), R(src[2 * p + 1])};
}
template <typename R>
__global__ void k_cx_export(const typename Cx<R>::T* src, double* dst, long n) {
  for (long p = (long)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (long)gridDim.x * blockDim.x) {
    dst[2 * p] = (double)src[p].x;
    dst[2 * p + 1] = (double)src[p].y;
  }
}

template <typename R>
__global__ void k_scale_copy(const R* src, R* dst, long n, double a) {
  for (long p = (long)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (long)gridDim.x * blockDim.x)
    dst[p] = R(a * (double)src[p]);
}

template <typename R>
__global__ void k_axpy(const R* x, R* y, long n, double a, int accumulate) {
  constexpr int NP = kVecPts<R>;
  const int vec = (n % 4) == 0;
  for (long p0 = ((long)blockIdx.x * blockDim.x + threadIdx.x) * NP; p0 < n; p0 += (long)gridDim.x * blockDim.x * NP) {
    R xv[NP], yv[NP];
    vload(x, p0, n, vec, xv);
    if (accumulate) vload(y, p0, n, vec, yv);
#pragma unroll
    for (int t = 0; t < NP; ++t)
      yv[t] = accumulate ? R((double)yv[t] + a * (double)xv[t]) : R(a * (double)xv[t]);
    vstore(y, p0, n, vec, yv);
  }
}

#include "fft_plane.cuh"

// ------------------------------------------------- size dispatch --------
// Compile-time instantiations for the grid sizes the engine is run at; any
// other size uses the runtime radix plan (tile_fft).  NL is the tile width:
// 16 lines in FP32 and 8 in FP64 (128-byte rows).

#define MPDPFT_CT_LENGTHS(X) X(16) X(32) X(48) X(64) X(96) X(128) X(192) X(256) X(384) X(512)

template <typename R, int NL>
static bool launch_z_r2c_ct(int M, unsigned grid, size_t smem, cudaStream_t st, const ZArgs<R>& a) {
  switch (M) {
#define CASE(N)                                                                                   \
  case N:                                                                                         \
    smem_optin(k_z_r2c<R, N, NL>); \
    launch_k(k_z_r2c<R, N, NL>, dim3(grid), dim3(kFftThreads), smem, st, a);                                        \
    return true;
    MPDPFT_CT_LENGTHS(CASE)
#undef CASE
    default: return false;
  }
}

template <typename R, int NL>
static bool launch_z_c2r_ct(int M, unsigned grid, size_t smem, cudaStream_t st, const ZArgs<R>& a) {
  switch (M) {
#define CASE(N)                                                                                   \
  case N:                                                                                         \
    smem_optin(k_z_c2r<R, N, NL>); \
    launch_k(k_z_c2r<R, N, NL>, dim3(grid), dim3(kFftThreads), smem, st, a);                                        \
    return true;
    MPDPFT_CT_LENGTHS(CASE)
#undef CASE
    default: return false;
  }
}

template <typename R, int NL>
static bool launch_axis_ct(int n, dim3 grid, size_t smem, cudaStream_t st, const AxisArgs<R>& a) {
  switch (n) {
#define CASE(N)                                                                                      \
  case N:                                                                                            \
    smem_optin(k_axis_c2c<R, N, NL>); \
    launch_k(k_axis_c2c<R, N, NL>, dim3(grid), dim3(kFftThreads), smem, st, a);                                        \
    return true;
    MPDPFT_CT_LENGTHS(CASE)
#undef CASE
    default: return false;
  }
}

template <typename R, int NL>
static bool launch_x_ct(int n, unsigned grid, size_t smem, cudaStream_t st, const AxisArgs<R>& a) {
  switch (n) {
#define CASE(N)                                                                                         \
  case N:                                                                                               \
    smem_optin(k_x_roundtrip<R, N, NL>); \
    launch_k(k_x_roundtrip<R, N, NL>, dim3(grid), dim3(kFftThreads), smem, st, a);                                        \
    return true;
    MPDPFT_CT_LENGTHS(CASE)
#undef CASE
    default: return false;
  }
}

template <typename R>
constexpr int ct_width() { return sizeof(R) == sizeof(double) ? 8 : 16; }

// Batched launches (grid.y = argument sets of one grid size).
template <typename R, int NL>
static bool launch_z_r2c_b_ct(int M, dim3 grid, size_t smem, cudaStream_t st, const ZArgs<R>* a) {
  switch (M) {
#define CASE(N)                                                   \
  case N:                                                         \
    smem_optin(k_z_r2c_b<R, N, NL>);                              \
    k_z_r2c_b<R, N, NL><<<grid, kFftThreads, smem, st>>>(a);      \
    return true;
    MPDPFT_CT_LENGTHS(CASE)
#undef CASE
    default: return false;
  }
}

template <typename R, int NL>
static bool launch_z_c2r_b_ct(int M, dim3 grid, size_t smem, cudaStream_t st, const ZArgs<R>* a) {
  switch (M) {
#define CASE(N)                                                   \
  case N:                                                         \
    smem_optin(k_z_c2r_b<R, N, NL>);                              \
    k_z_c2r_b<R, N, NL><<<grid, kFftThreads, smem, st>>>(a);      \
    return true;
    MPDPFT_CT_LENGTHS(CASE)
#undef CASE
    default: return false;
  }
}

template <typename R, int NL>
static bool launch_x_b_ct(int n, dim3 grid, size_t smem, cudaStream_t st, const AxisArgs<R>* a) {
  switch (n) {
#define CASE(N)                                                       \
  case N:                                                             \
    smem_optin(k_x_roundtrip_b<R, N, NL>);                            \
    k_x_roundtrip_b<R, N, NL><<<grid, kFftThreads, smem, st>>>(a);    \
    return true;
    MPDPFT_CT_LENGTHS(CASE)
#undef CASE
    default: return false;
  }
}

// ------------------------------------------------------------ host side --
template <typename R>
static int make_twiddles(Ctx& c, FftPlan& f) {
  using C = typename Cx<R>::T;
  auto table = [&](int len, int sign, void** dst) -> int {
    std::vector<C> h(len);
    for (int t = 0; t < len; ++t) {
      double a = 2.0 * kPi * (double)t / (double)len;
      h[t] = C{R(std::cos(a)), R(sign * std::sin(a))};
    }
    int st = c.alloc(dst, sizeof(C) * len);
    if (st) return st;
    CU(cudaMemcpy(*dst, h.data(), sizeof(C) * len, cudaMemcpyHostToDevice));
    return MPDPFT_OK;
  };
  int st;
  if ((st = table(f.s, -1, &f.tw_s_f))) return st;
  if ((st = table(f.s, +1, &f.tw_s_b))) return st;
  if ((st = table(f.M, -1, &f.tw_m_f))) return st;
  if ((st = table(f.M, +1, &f.tw_m_b))) return st;
  if ((st = table(f.s, -1, &f.tw_n_f))) return st;
  return MPDPFT_OK;
}

int Ctx::fft_setup() {
  fft = new FftPlan;
  FftPlan& f = *fft;
  f.dim = P.dim;
  f.s = P.steps;
  f.M = P.steps / 2;
  f.H = f.M + 1;
  f.rows = geom.n / P.steps;
  f.nspec = f.rows * f.H;
  if (!factor(f.s, f.plan_s) || !factor(f.M, f.plan_m))
    return set_error(MPDPFT_ERR_ARG, "steps must factor into 2s and 3s for the FFT");
  int st = rsize == sizeof(double) ? make_twiddles<double>(*this, f) : make_twiddles<float>(*this, f);
  if (st) return st;
  const size_t csz = 2 * rsize;
  f.tk = rsize == sizeof(double) ? 8 : 16;
  while (f.tk > 1 && f.M % f.tk) f.tk /= 2;
  f.zl = 16;
  f.zblocks = (int)((f.rows + f.zl - 1) / f.zl);
  const bool need = has_coulomb || gradient;
  const int nspec_buf = gradient ? 4 : 1;
  for (int i = 0; i < nspec_buf; ++i)
    if ((st = alloc(&f.spec[i], csz * f.nspec))) return st;
  if ((st = alloc(&f.rtmp, rsize * geom.n))) return st;
  // (room for the autotuner's narrower z tiles: 8 rows per block)
  if ((st = alloc((void**)&f.zpart, sizeof(double) * ((f.rows + 7) / 8 + 1)))) return st;
  if ((st = alloc((void**)&f.vmax, sizeof(unsigned long long)))) return st;
  f.vblocks = grid_blocks(geom.n);
  if ((st = alloc((void**)&f.vres_part, sizeof(double) * f.vblocks * kMaxS))) return st;
  (void)need;
  {
    int dev = 0, optin = 0;
    CU(cudaGetDevice(&dev));
    CU(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    const bool f64 = rsize == sizeof(double);
    const bool inst = f64 ? plane_size_instantiated<double>(f.s) : plane_size_instantiated<float>(f.s);
    const size_t need_smem = f64 ? plane_inv_smem<double>(f.s, plane_nly<double>(f.s), plane_nlz<double>(f.s), true)
                                 : plane_inv_smem<float>(f.s, plane_nly<float>(f.s), plane_nlz<float>(f.s), true);
    f.plane = f.dim == 3 && inst && need_smem + 1024 <= (size_t)optin;
  }
  // shared memory opt-in of the runtime-plan kernels (any grid size)
  if (rsize == sizeof(double)) {
    CU(smem_optin(k_z_r2c<double, 0, 0>));
    CU(smem_optin(k_z_c2r<double, 0, 0>));
    CU(smem_optin(k_axis_c2c<double, 0, 0>));
    CU(smem_optin(k_x_roundtrip<double, 0, 0>));
  } else {
    CU(smem_optin(k_z_r2c<float, 0, 0>));
    CU(smem_optin(k_z_c2r<float, 0, 0>));
    CU(smem_optin(k_axis_c2c<float, 0, 0>));
    CU(smem_optin(k_x_roundtrip<float, 0, 0>));
  }
  return fft_autotune();
}

void Ctx::fft_release() {
  delete fft;
  fft = nullptr;
}

// --- pass launchers ---------------------------------------------------------
template <typename R>
static ZArgs<R> zargs(Ctx& c) {
  FftPlan& f = *c.fft;
  ZArgs<R> a;
  std::memset(&a, 0, sizeof(a));
  a.g = c.geom;
  a.M = f.M;
  a.H = f.H;
  a.zl = f.zl;
  a.rows = f.rows;
  a.plan = f.plan_m;
  a.tw_n = (const typename Cx<R>::T*)f.tw_n_f;
  a.nsrc = 1;
  return a;
}

// Arguments of the R2C pass (vmax: the taper shift slot).
template <typename R>
static ZArgs<R> r2c_args(Ctx& c, const R* in, int pro, int nsrc, const double* qcoef, void* out, bool sums,
                         unsigned long long* vmax) {
  FftPlan& f = *c.fft;
  ZArgs<R> a = zargs<R>(c);
  a.tw_m = (const typename Cx<R>::T*)f.tw_m_f;
  a.in = in;
  a.pro = pro;
  a.nsrc = nsrc;
  for (int q = 0; q < nsrc && qcoef; ++q) a.qcoef[q] = qcoef[q];
  a.vmax = vmax;
  a.taper_r0 = c.P.regularization_threshold * c.P.edge;
  a.taper_a = -2500.0 / (c.P.edge * c.P.edge);
  a.out = (typename Cx<R>::T*)out;
  a.part = sums ? f.zpart : nullptr;
  return a;
}

template <typename R>
static size_t r2c_smem(const FftPlan& f) {
  return (3 * (size_t)f.M * (f.zl + 1) + f.M) * sizeof(typename Cx<R>::T);
}

template <typename R>
static int launch_z_r2c(Ctx& c, const R* in, int pro, int nsrc, const double* qcoef, void* out, bool sums) {
  FftPlan& f = *c.fft;
  ZArgs<R> a = r2c_args<R>(c, in, pro, nsrc, qcoef, out, sums, f.vmax);
  if (sums) f.zparts = f.zblocks;
  const size_t smem = r2c_smem<R>(f);
  c.cnt[MPDPFT_STAGE_FFT_Z_R2C]++;
  c.note("k_z_r2c", nsrc * c.field_bytes() + c.spec_bytes());
  if (!(f.zl == 16 ? launch_z_r2c_ct<R, 16>(f.M, f.zblocks, smem, c.stream, a)
                   : f.zl == 8 && launch_z_r2c_ct<R, 8>(f.M, f.zblocks, smem, c.stream, a)))
    launch_k(k_z_r2c<R, 0, 0>, dim3(f.zblocks), dim3(kFftThreads), smem, c.stream, a);
  CU(cudaGetLastError());
  return MPDPFT_OK;
}

// Arguments of the C2R pass.
template <typename R>
static ZArgs<R> c2r_args(Ctx& c, void* const* in, int nin, int epi, R* out0, R* out1, double coul_coef) {
  FftPlan& f = *c.fft;
  ZArgs<R> a = zargs<R>(c);
  a.tw_m = (const typename Cx<R>::T*)f.tw_m_b;
  for (int i = 0; i < nin; ++i) a.cin[i] = (const typename Cx<R>::T*)in[i];
  a.nin = nin;
  a.epi = epi;
  a.rout[0] = out0;
  a.rout[1] = out1;
  a.scale = 1.0;
  a.coul_coef = coul_coef;
  a.f0_part = f.zpart;
  a.f0_blocks = f.zparts;
  return a;
}

template <typename R>
static size_t c2r_smem(const FftPlan& f) {
  return (2 * (size_t)f.M * (f.zl + 1) + f.M) * sizeof(typename Cx<R>::T) + sizeof(R) * (size_t)f.s * f.zl;
}

template <typename R>
static int launch_z_c2r(Ctx& c, void* const* in, int nin, int epi, R* out0, R* out1, double coul_coef) {
  FftPlan& f = *c.fft;
  ZArgs<R> a = c2r_args<R>(c, in, nin, epi, out0, out1, coul_coef);
  const size_t smem = c2r_smem<R>(f);
  c.cnt[MPDPFT_STAGE_FFT_Z_C2R]++;
  c.note("k_z_c2r", nin * c.spec_bytes() + ((out0 ? 1 : 0) + (out1 ? 1 : 0)) * c.field_bytes());
  if (!(f.zl == 16 ? launch_z_c2r_ct<R, 16>(f.M, f.zblocks, smem, c.stream, a)
                   : f.zl == 8 && launch_z_c2r_ct<R, 8>(f.M, f.zblocks, smem, c.stream, a)))
    launch_k(k_z_c2r<R, 0, 0>, dim3(f.zblocks), dim3(kFftThreads), smem, c.stream, a);
  CU(cudaGetLastError());
  return MPDPFT_OK;
}

template <typename R>
static AxisArgs<R> axis_args(Ctx& c, int axis) {
  FftPlan& f = *c.fft;
  AxisArgs<R> a;
  std::memset(&a, 0, sizeof(a));
  a.s = f.s;
  a.M = f.M;
  a.H = f.H;
  a.tk = f.tk;
  a.dim = f.dim;
  a.plan = f.plan_s;
  a.twf = (const typename Cx<R>::T*)f.tw_s_f;
  a.twb = (const typename Cx<R>::T*)f.tw_s_b;
  if (f.dim == 3 && axis == 1) {        // Y: outer = x index, lines along y
    a.nouter = f.s;
    a.ostride = (long)f.s * f.H;
    a.astride = f.H;
  } else if (f.dim == 3) {              // X: outer = y index, lines along x
    a.nouter = f.s;
    a.ostride = f.H;
    a.astride = (long)f.s * f.H;
  } else {                              // 2D X: single outer
    a.nouter = 1;
    a.ostride = 0;
    a.astride = f.H;
  }
  a.ntile = f.M / f.tk;
  a.nbulk = a.nouter * a.ntile;
  a.dk = c.geom.dk;
  a.scale = 1.0 / (double)c.geom.n;
  return a;
}

template <typename R>
static int launch_y(Ctx& c, void* const* data, int nfield, int dir) {
  FftPlan& f = *c.fft;
  AxisArgs<R> a = axis_args<R>(c, 1);
  for (int i = 0; i < nfield; ++i) a.data[i] = (typename Cx<R>::T*)data[i];
  a.dir = dir;
  const long nyq_blocks = (a.nouter + a.tk - 1) / a.tk;
  dim3 grid((unsigned)(a.nbulk + nyq_blocks), nfield);
  const size_t smem = (2 * (size_t)f.s * (f.tk + 1) + f.s) * sizeof(typename Cx<R>::T);
  c.cnt[MPDPFT_STAGE_FFT_Y]++;
  c.note("k_axis_c2c", 2.0 * nfield * c.spec_bytes());
  constexpr int W = ct_width<R>();
  if (!(f.tk == W ? launch_axis_ct<R, W>(f.s, grid, smem, c.stream, a)
                  : f.tk == W / 2 && launch_axis_ct<R, W / 2>(f.s, grid, smem, c.stream, a)))
    launch_k(k_axis_c2c<R, 0, 0>, dim3(grid), dim3(kFftThreads), smem, c.stream, a);
  CU(cudaGetLastError());
  return MPDPFT_OK;
}

// Arguments of the X round trip.
template <typename R>
static AxisArgs<R> x_args(Ctx& c, void* in, void* const* out, int nout, int mul, double sigma_c) {
  FftPlan& f = *c.fft;
  AxisArgs<R> a = axis_args<R>(c, 0);
  a.data[0] = (typename Cx<R>::T*)in;
  for (int i = 0; i < nout; ++i) a.out[i] = (typename Cx<R>::T*)out[i];
  a.nout = nout;
  a.mul = mul;
  a.sigma_c = sigma_c;
  a.cutoff = c.P.coulomb_cutoff > 0.0 ? c.P.coulomb_cutoff : 0.5 * c.P.edge;
  a.f0_part = f.zpart;
  a.f0_blocks = f.zparts;
  return a;
}

template <typename R>
static unsigned x_grid(const AxisArgs<R>& a) {
  const long nyq_blocks = (a.nouter + a.tk - 1) / a.tk;
  return (unsigned)(a.nbulk + nyq_blocks);
}

// Compile-time tile of the X round trip: shared memory, and whether it fits.
template <typename R>
static size_t x_smem_ct(const FftPlan& f) {
  return (3 * (size_t)f.s * (f.tk + 1) + 2 * f.s) * sizeof(typename Cx<R>::T);
}
template <typename R>
static size_t x_smem_rt(const FftPlan& f) {
  return 3 * (size_t)f.s * f.tk * sizeof(typename Cx<R>::T);
}
template <typename R>
static bool x_ct_fits(const FftPlan& f) {
  return x_smem_ct<R>(f) + sizeof(MulTables<R, 512, 16>) <= 227 * 1024;
}

// The compile-time x round trip for the plan's tile width (the width of
// ct_width or half of it); false: the runtime kernel runs instead.
template <typename R>
static bool launch_x_tiles(const FftPlan& f, unsigned grid, cudaStream_t st, const AxisArgs<R>& a) {
  constexpr int W = ct_width<R>();
  if (!x_ct_fits<R>(f)) return false;
  if (f.tk == W) return launch_x_ct<R, W>(f.s, grid, x_smem_ct<R>(f), st, a);
  if (f.tk == W / 2) return launch_x_ct<R, W / 2>(f.s, grid, x_smem_ct<R>(f), st, a);
  return false;
}

template <typename R>
static int launch_x_args(Ctx& c, const AxisArgs<R>& a) {
  FftPlan& f = *c.fft;
  const unsigned grid = x_grid<R>(a);
  c.cnt[MPDPFT_STAGE_FFT_X]++;
  c.note("k_x_roundtrip", (1.0 + a.nout) * c.spec_bytes());
  if (!launch_x_tiles<R>(f, grid, c.stream, a))
    launch_k(k_x_roundtrip<R, 0, 0>, dim3(grid), dim3(kFftThreads), x_smem_rt<R>(f), c.stream, a);
  CU(cudaGetLastError());
  return MPDPFT_OK;
}

template <typename R>
static int launch_x(Ctx& c, void* in, void* const* out, int nout, int mul, double sigma_c) {
  FftPlan& f = *c.fft;
  AxisArgs<R> a = x_args<R>(c, in, out, nout, mul, sigma_c);
  const unsigned grid = x_grid<R>(a);
  c.cnt[MPDPFT_STAGE_FFT_X]++;
  c.note("k_x_roundtrip", (1.0 + a.nout) * c.spec_bytes());
  if (!launch_x_tiles<R>(f, grid, c.stream, a))
    launch_k(k_x_roundtrip<R, 0, 0>, dim3(grid), dim3(kFftThreads), x_smem_rt<R>(f), c.stream, a);
  CU(cudaGetLastError());
  return MPDPFT_OK;
}

// ---- plane passes (3D): instantiated (s, lines per tile) per precision ----
template <typename R, int S, int PRO>
static void plane_fwd_pro(unsigned grid, size_t smem, cudaStream_t st, const ZArgs<R>& a) {
  constexpr int NLY = plane_nly<R>(S), NLZ = plane_nlz<R>(S);
  smem_optin(k_plane_fwd<R, S, NLY, NLZ, PRO>);
  launch_k(k_plane_fwd<R, S, NLY, NLZ, PRO>, dim3(grid), dim3(kPlaneThreads), smem, st, a);
}
template <typename R, int S>
static void plane_fwd_ct(unsigned grid, size_t smem, cudaStream_t st, const ZArgs<R>& a) {
  if (a.pro == PRO_TAPER) plane_fwd_pro<R, S, PRO_TAPER>(grid, smem, st, a);
  else plane_fwd_pro<R, S, PRO_NONE>(grid, smem, st, a);
}
template <typename R, int S, int EPI>
static void plane_inv_epi(unsigned grid, size_t smem, cudaStream_t st, const ZArgs<R>& a) {
  constexpr int NLY = plane_nly<R>(S), NLZ = plane_nlz<R>(S);
  smem_optin(k_plane_inv<R, S, NLY, NLZ, EPI>);
  launch_k(k_plane_inv<R, S, NLY, NLZ, EPI>, dim3(grid), dim3(kPlaneThreads), smem, st, a);
}
template <typename R, int S>
static void plane_inv_ct(unsigned grid, size_t smem, cudaStream_t st, const ZArgs<R>& a) {
  switch (a.epi) {
    case EPI_POS: plane_inv_epi<R, S, EPI_POS>(grid, smem, st, a); break;
    case EPI_GRAD: plane_inv_epi<R, S, EPI_GRAD>(grid, smem, st, a); break;
    case EPI_COULOMB: plane_inv_epi<R, S, EPI_COULOMB>(grid, smem, st, a); break;
    case EPI_SCALE: plane_inv_epi<R, S, EPI_SCALE>(grid, smem, st, a); break;
    case EPI_COULOMB_V: plane_inv_epi<R, S, EPI_COULOMB_V>(grid, smem, st, a); break;
    default: plane_inv_epi<R, S, EPI_STORE>(grid, smem, st, a); break;
  }
}

template <typename R>
static void plane_dispatch(bool fwd, int s, size_t smem, cudaStream_t st, const ZArgs<R>& a) {
  const unsigned grid = (unsigned)s;
  if (s == 32) { fwd ? plane_fwd_ct<R, 32>(grid, smem, st, a) : plane_inv_ct<R, 32>(grid, smem, st, a); }
  else if (s == 64) { fwd ? plane_fwd_ct<R, 64>(grid, smem, st, a) : plane_inv_ct<R, 64>(grid, smem, st, a); }
  else if constexpr (sizeof(R) == sizeof(float)) {
    if (s == 128) { fwd ? plane_fwd_ct<R, 128>(grid, smem, st, a) : plane_inv_ct<R, 128>(grid, smem, st, a); }
  }
}

// Forward 3D transform of `in` (prologue PRO_NONE or PRO_TAPER) into the
// half spectrum `out`: plane pass (z R2C + y C2C); the x pass follows.
template <typename R>
static int launch_plane_fwd(Ctx& c, const R* in, int pro, void* out, bool sums) {
  FftPlan& f = *c.fft;
  ZArgs<R> a = zargs<R>(c);
  a.tw_m = (const typename Cx<R>::T*)f.tw_m_f;
  a.tw_s = (const typename Cx<R>::T*)f.tw_s_f;
  a.in = in;
  a.pro = pro;
  a.vmax = f.vmax;
  a.taper_r0 = c.P.regularization_threshold * c.P.edge;
  a.taper_a = -2500.0 / (c.P.edge * c.P.edge);
  a.out = (typename Cx<R>::T*)out;
  a.part = sums ? f.zpart : nullptr;
  a.err = &c.d_state->abort;
  if (sums) f.zparts = f.s;
  c.cnt[MPDPFT_STAGE_FFT_Z_R2C]++;
  c.note("k_plane_fwd", c.field_bytes() + c.spec_bytes());
  plane_dispatch<R>(true, f.s, plane_fwd_smem<R>(f.s, plane_nly<R>(f.s), plane_nlz<R>(f.s)), c.stream, a);
  CU(cudaGetLastError());
  return MPDPFT_OK;
}

// Inverse 3D transform after the x pass: y C2C inverse + z C2R with epilogue.
template <typename R>
static int launch_plane_inv(Ctx& c, void* const* in, int nin, int epi, R* out0, R* out1, double coul_coef) {
  FftPlan& f = *c.fft;
  ZArgs<R> a = zargs<R>(c);
  a.tw_m = (const typename Cx<R>::T*)f.tw_m_b;
  a.tw_s = (const typename Cx<R>::T*)f.tw_s_b;
  for (int i = 0; i < nin; ++i) a.cin[i] = (const typename Cx<R>::T*)in[i];
  a.nin = nin;
  a.epi = epi;
  a.rout[0] = out0;
  a.rout[1] = out1;
  a.scale = 1.0;
  a.coul_coef = coul_coef;
  a.f0_part = f.zpart;
  a.f0_blocks = f.zparts;
  a.err = &c.d_state->abort;
  a.coul_reg = c.P.coulomb_kernel != MPDPFT_COULOMB_TRUNCATED;
  if (epi == EPI_COULOMB_V) {  // V assembly of species 0 fused into the epilogue
    a.st = c.d_state;
    a.vext = (const R*)c.d_vext;
    a.ncur = (const R*)c.d_cur;
    a.vpot = (R*)c.d_V;
    a.beta = c.P.beta;
    a.gamma_h = c.P.gamma_h;
    a.contact_self = c.has_interaction(MPDPFT_INT_CONTACT_SELF);
    a.dirac = c.has_interaction(MPDPFT_INT_DIRAC);
    a.shell_r = c.P.edge * c.P.regularization_threshold;
    a.shell_w = 2.0 * c.geom.dx;
    a.vres_part = f.vres_part;
    a.vmax_out = f.vmax;
  }
  c.cnt[MPDPFT_STAGE_FFT_Z_C2R]++;
  {
    // spectra in, outputs out; the fused V assembly also reads V_ext, the
    // density and the old V and writes V
    double b = nin * c.spec_bytes() + ((out0 ? 1 : 0) + (out1 ? 1 : 0)) * c.field_bytes();
    if (epi == EPI_COULOMB_V) b += (3.0 + ((a.contact_self || a.dirac) ? 1.0 : 0.0)) * c.field_bytes();
    c.note("k_plane_inv", b);
  }
  plane_dispatch<R>(false, f.s, plane_inv_smem<R>(f.s, plane_nly<R>(f.s), plane_nlz<R>(f.s), epi == EPI_GRAD || epi == EPI_COULOMB || epi == EPI_COULOMB_V), c.stream, a);
  CU(cudaGetLastError());
  return MPDPFT_OK;
}

// Coulomb potential of `src` (nsrc species combined with weights qcoef)
// into out: out = coef * phi, phi = int rho(r')/|r - r'|.
// fuse_v: also assemble V of species 0 in the final pass (plane path only;
// the caller checked that this Coulomb term is species 0's whole vh).
template <typename R>
static int coulomb_into(Ctx& c, const R* src, int nsrc, const double* qcoef, R* out, double coef,
                        bool fuse_v = false) {
  FftPlan& f = *c.fft;
  int st;
  const int pro = nsrc > 1 || (qcoef && qcoef[0] != 1.0) ? PRO_CHARGE : PRO_NONE;
  if (f.dim == 2) {  // HartreeRepulsion 2D (mpDPFT.cpp:2636-2665): V = 2 pi gammaH (...)
    if ((st = launch_z_r2c<R>(c, src, pro, nsrc, qcoef, f.spec[0], true))) return st;
    if ((st = launch_x<R>(c, f.spec[0], &f.spec[0], 1, MUL_COULOMB_2D, 0.0))) return st;
    return launch_z_c2r<R>(c, &f.spec[0], 1, EPI_COULOMB, out, nullptr, 2.0 * kPi * coef);
  }
  const int mul = c.P.coulomb_kernel == MPDPFT_COULOMB_TRUNCATED ? MUL_COULOMB_TRUNC : MUL_COULOMB_REG;
  if (f.plane && pro == PRO_NONE) {
    if ((st = launch_plane_fwd<R>(c, src, pro, f.spec[0], true))) return st;
    if ((st = launch_x<R>(c, f.spec[0], &f.spec[0], 1, mul, 0.0))) return st;
    if (fuse_v) return launch_plane_inv<R>(c, &f.spec[0], 1, EPI_COULOMB_V, out, nullptr, 4.0 * kPi * coef);
    if (mul == MUL_COULOMB_REG)
      return launch_plane_inv<R>(c, &f.spec[0], 1, EPI_COULOMB, out, nullptr, 4.0 * kPi * coef);
    return launch_plane_inv<R>(c, &f.spec[0], 1, EPI_SCALE, out, nullptr, 4.0 * kPi * coef);
  }
  if ((st = launch_z_r2c<R>(c, src, pro, nsrc, qcoef, f.spec[0], true))) return st;
  if (f.dim == 3 && (st = launch_y<R>(c, &f.spec[0], 1, -1))) return st;
  if ((st = launch_x<R>(c, f.spec[0], &f.spec[0], 1, mul, 0.0))) return st;
  if (f.dim == 3 && (st = launch_y<R>(c, &f.spec[0], 1, +1))) return st;
  // regularised: V = 4 pi gammaH (x + f0 erf(r/2)/(4 pi r)); truncated: V = 4 pi gammaH x
  if (mul == MUL_COULOMB_REG)
    return launch_z_c2r<R>(c, &f.spec[0], 1, EPI_COULOMB, out, nullptr, 4.0 * kPi * coef);
  // truncated kernel: out = 4 pi coef x
  return launch_z_c2r<R>(c, &f.spec[0], 1, EPI_SCALE, out, nullptr, 4.0 * kPi * coef);
}


int Ctx::scale_copy(const void* src, void* dst, double a) {
  const int blocks = grid_blocks(geom.n);
  cnt[5]++;
  note("k_scale_copy", 2.0 * field_bytes());
  if (rsize == sizeof(double)) k_scale_copy<double><<<blocks, kThreads, 0, stream>>>((const double*)src, (double*)dst, geom.n, a);
  else k_scale_copy<float><<<blocks, kThreads, 0, stream>>>((const float*)src, (float*)dst, geom.n, a);
  CU(cudaGetLastError());
  return MPDPFT_OK;
}

// Coulomb terms of every species for densities `dens` ([S][n]) into out
// ([S][n]): types 8, 21 and 100 (mpDPFT.cpp:2266-2285).
template <typename R>
static int coulomb_terms(Ctx& c, const R* dens, R* out) {
  const long n = c.geom.n;
  const int S = c.S;
  int st;
  std::vector<int> touched(S, 0);
  for (int a = 0; a < c.P.n_interactions; ++a) {
    const int t = c.P.interactions[a];
    if (t == MPDPFT_INT_HARTREE) {
      for (int s = 0; s < S; ++s) {
        double one = 1.0;
        if (!touched[s]) {  // first term of species s: straight into its output
          if ((st = coulomb_into<R>(c, dens + (long)s * n, 1, &one, out + (long)s * n, c.P.gamma_h))) return st;
        } else {
          if ((st = coulomb_into<R>(c, dens + (long)s * n, 1, &one, (R*)c.fft->rtmp, c.P.gamma_h))) return st;
          if ((st = c.axpy(c.fft->rtmp, out + (long)s * n, 1.0, 1))) return st;
        }
        touched[s] = 1;
      }
    } else if (t == MPDPFT_INT_HARTREE_INTER) {
      for (int s = 0; s < S; ++s)
        for (int q = 0; q < S; ++q) {
          if (q == s) continue;
          double one = 1.0;
          if ((st = coulomb_into<R>(c, dens + (long)q * n, 1, &one, (R*)c.fft->rtmp, c.P.gamma_h))) return st;
          if ((st = c.axpy(c.fft->rtmp, out + (long)s * n, 1.0, touched[s]))) return st;
          touched[s] = 1;
        }
    } else if (t == MPDPFT_INT_COULOMB_CHARGED) {
      if ((st = coulomb_into<R>(c, dens, S, c.P.charges, (R*)c.fft->rtmp, c.P.gamma_h))) return st;
      for (int s = 0; s < S; ++s) {
        if ((st = c.axpy(c.fft->rtmp, out + (long)s * n, c.P.charges[s], touched[s]))) return st;
        touched[s] = 1;
      }
    }
  }
  for (int s = 0; s < S; ++s)
    if (!touched[s]) {
      CU(cudaMemsetAsync(out + (long)s * n, 0, sizeof(R) * n, c.stream));
      c.note("memset", c.field_bytes());
    }
  return MPDPFT_OK;
}


int Ctx::axpy(const void* x, void* y, double a, int accumulate) {
  const int blocks = grid_blocks(geom.n);
  cnt[5]++;
  note("k_axpy", (accumulate ? 3.0 : 2.0) * field_bytes());
  if (rsize == sizeof(double)) k_axpy<double><<<blocks, kThreads, 0, stream>>>((const double*)x, (double*)y, geom.n, a, accumulate);
  else k_axpy<float><<<blocks, kThreads, 0, stream>>>((const float*)x, (float*)y, geom.n, a, accumulate);
  CU(cudaGetLastError());
  return MPDPFT_OK;
}

// DelField of species-0 field f (already in compute precision): g2 and lap.
// want_g2 = false: the Laplacian alone (a density functional without a
// |grad V|^2 term needs no gradients; g2 is left as it is).
template <typename R>
static int delfield_into(Ctx& c, const R* f, R* g2, R* lap, bool want_g2 = true) {
  FftPlan& F = *c.fft;
  int st;
  const double smear = c.P.smearing_extent > 0.0 ? c.P.smearing_extent : 6.0 * c.geom.dx;
  const double sigma_c = -0.5 * smear * smear;  // ConvolutionSigma (mpDPFT.cpp:1106)
  const int pro = c.P.taper_off ? PRO_TAPER : PRO_NONE;
  if (!want_g2) {  // in place, as the smoothing pass below
    void* out = F.spec[0];
    if (F.plane) {
      if ((st = launch_plane_fwd<R>(c, f, pro, F.spec[0], false))) return st;
      if ((st = launch_x<R>(c, F.spec[0], &out, 1, MUL_LAP, sigma_c))) return st;
      return launch_plane_inv<R>(c, &out, 1, EPI_STORE, lap, nullptr, 0.0);
    }
    if ((st = launch_z_r2c<R>(c, f, pro, 1, nullptr, F.spec[0], false))) return st;
    if (F.dim == 3 && (st = launch_y<R>(c, &F.spec[0], 1, -1))) return st;
    if ((st = launch_x<R>(c, F.spec[0], &out, 1, MUL_LAP, sigma_c))) return st;
    if (F.dim == 3 && (st = launch_y<R>(c, &out, 1, +1))) return st;
    return launch_z_c2r<R>(c, &out, 1, EPI_STORE, lap, nullptr, 0.0);
  }
  if (F.plane) {
    void* outs[4] = {F.spec[0], F.spec[1], F.spec[2], F.spec[3]};
    if ((st = launch_plane_fwd<R>(c, f, pro, F.spec[0], false))) return st;
    if ((st = launch_x<R>(c, F.spec[0], outs, 4, MUL_DERIV, sigma_c))) return st;
    // |grad f|^2 (raw) -> rtmp, Laplacian -> lap
    if ((st = launch_plane_inv<R>(c, outs, 4, EPI_GRAD, (R*)F.rtmp, lap, 0.0))) return st;
    // smooth |grad f|^2 and clamp at 0 (mpDPFT.cpp:7550-7560)
    if ((st = launch_plane_fwd<R>(c, (const R*)F.rtmp, PRO_NONE, F.spec[0], false))) return st;
    if ((st = launch_x<R>(c, F.spec[0], &F.spec[0], 1, MUL_SMOOTH, sigma_c))) return st;
    return launch_plane_inv<R>(c, &F.spec[0], 1, EPI_POS, g2, nullptr, 0.0);
  }
  if ((st = launch_z_r2c<R>(c, f, pro, 1, nullptr, F.spec[0], false))) return st;
  if (F.dim == 3 && (st = launch_y<R>(c, &F.spec[0], 1, -1))) return st;
  const int nout = F.dim + 1;  // gradients + Laplacian
  void* outs[4] = {F.spec[0], F.spec[1], F.spec[2], F.spec[3]};
  if (F.dim == 2) { outs[0] = F.spec[1]; outs[1] = F.spec[2]; outs[2] = F.spec[3]; }
  if ((st = launch_x<R>(c, F.spec[0], outs, nout, MUL_DERIV, sigma_c))) return st;
  if (F.dim == 3 && (st = launch_y<R>(c, outs, nout, +1))) return st;
  // |grad f|^2 (raw) -> rtmp, Laplacian -> lap
  if ((st = launch_z_c2r<R>(c, outs, nout, EPI_GRAD, (R*)F.rtmp, lap, 0.0))) return st;
  // smooth |grad f|^2 and clamp at 0 (mpDPFT.cpp:7550-7560)
  if ((st = launch_z_r2c<R>(c, (const R*)F.rtmp, PRO_NONE, 1, nullptr, F.spec[0], false))) return st;
  if (F.dim == 3 && (st = launch_y<R>(c, &F.spec[0], 1, -1))) return st;
  if ((st = launch_x<R>(c, F.spec[0], &F.spec[0], 1, MUL_SMOOTH, sigma_c))) return st;
  if (F.dim == 3 && (st = launch_y<R>(c, &F.spec[0], 1, +1))) return st;
  if ((st = launch_z_c2r<R>(c, &F.spec[0], 1, EPI_POS, g2, nullptr, 0.0))) return st;
  return MPDPFT_OK;
}

static double shell_width(const Ctx& c) { return 2.0 * c.geom.dx; }
static double shell_radius(const Ctx& c) { return c.P.edge * c.P.regularization_threshold; }

template <typename R>
static int fft_terms_impl(Ctx& c) {
  FftPlan& F = *c.fft;
  int st;
  const long n = c.geom.n;
  // the current input densities: the ring slot state.slot is only known on
  // the device, so the kernels that write a new input density also store a
  // copy at the fixed address d_cur
  const R* dens = (const R*)c.d_cur;
  // one species whose only Coulomb term is the Hartree potential: V is
  // assembled in the epilogue of that transform
  const bool fuse = F.plane && c.S == 1 && c.has_interaction(MPDPFT_INT_HARTREE) &&
                    !c.has_interaction(MPDPFT_INT_HARTREE_INTER) && !c.has_interaction(MPDPFT_INT_COULOMB_CHARGED);
  CU(cudaMemsetAsync(F.vmax, 0, sizeof(unsigned long long), c.stream));
  c.note("memset", sizeof(unsigned long long));
  if (fuse) {
    if ((st = coulomb_into<R>(c, dens, 1, nullptr, (R*)c.d_vh, c.P.gamma_h, true))) return st;
    c.assemble_in_step = 0;
    c.vres_part_ext = F.vres_part;
    c.vres_blocks_ext = F.s;
  } else {
    if (c.has_coulomb) {
      if ((st = coulomb_terms<R>(c, dens, (R*)c.d_vh))) return st;
    }
  }
  KParams kp = c.kparams();
  if (!fuse) {
    c.cnt[5]++;
    // per species V_ext, the density, the Coulomb term and the old V in,
    // the new V out
    c.note("k_assemble_v", c.S * (4.0 + (c.has_coulomb ? 1.0 : 0.0)) * c.field_bytes());
    k_assemble_v<R><<<F.vblocks, kThreads, 0, c.stream>>>(kp, c.d_state, (const R*)c.d_vext,
                                                           c.has_coulomb ? (const R*)c.d_vh : nullptr,
                                                           (const R*)c.d_nin, (R*)c.d_V, F.vres_part, F.vmax,
                                                           shell_radius(c), shell_width(c));
    CU(cudaGetLastError());
    c.assemble_in_step = 0;
    c.vres_part_ext = F.vres_part;
    c.vres_blocks_ext = F.vblocks;
  }
  if (c.gradient) {
    for (int s = 0; s < c.S; ++s) {
      if (s > 0) {  // taper shift of species s
        CU(cudaMemsetAsync(F.vmax, 0, sizeof(unsigned long long), c.stream));
        c.note("memset", sizeof(unsigned long long));
        c.cnt[5]++;
        c.note("k_shell_max", c.field_bytes());
        k_shell_max<R><<<grid_blocks(n), kThreads, 0, c.stream>>>(c.geom, (const R*)c.d_V + (long)s * n, F.vmax,
                                                                  shell_radius(c), shell_width(c));
        CU(cudaGetLastError());
      }
      if ((st = delfield_into<R>(c, (const R*)c.d_V + (long)s * n, (R*)c.d_g2 + (long)s * n,
                                 (R*)c.d_lap + (long)s * n, c.need_g2)))
        return st;
    }
  }
  return MPDPFT_OK;
}

// Copy the current input densities (ring slot held on the device) into
// d_tmp, so FFT passes can read them from a fixed address.
template <typename R>
__global__ void k_copy_slot(const ScState* st, const R* ring, R* dst, long count) {
  if (__ldcg(&st->exit_loop)) return;
  const int cur = __ldcg(&st->slot);
  const R* src = ring + (long)cur * count;
  for (long p = (long)blockIdx.x * blockDim.x + threadIdx.x; p < count; p += (long)gridDim.x * blockDim.x)
    dst[p] = src[p];
}

int Ctx::copy_current_density() {
  const long count = geom.n * S;
  const int blocks = grid_blocks(count);
  cnt[5]++;
  if (rsize == sizeof(double)) k_copy_slot<double><<<blocks, kThreads, 0, stream>>>(d_state, (const double*)d_nin, (double*)d_tmp, count);
  else k_copy_slot<float><<<blocks, kThreads, 0, stream>>>(d_state, (const float*)d_nin, (float*)d_tmp, count);
  CU(cudaGetLastError());
  return MPDPFT_OK;
}

int Ctx::issue_fft_terms() {
  return rsize == sizeof(double) ? fft_terms_impl<double>(*this) : fft_terms_impl<float>(*this);
}

int Ctx::issue_coulomb(const void* dens, void* out, int for_energy) {
  (void)for_energy;
  if (rsize == sizeof(double)) return coulomb_terms<double>(*this, (const double*)dens, (double*)out);
  return coulomb_terms<float>(*this, (const float*)dens, (float*)out);
}

template <typename R>
static int delfield_of_v_impl(Ctx& c) {
  FftPlan& F = *c.fft;
  const long n = c.geom.n;
  int st;
  for (int s = 0; s < c.S; ++s) {
    CU(cudaMemsetAsync(F.vmax, 0, sizeof(unsigned long long), c.stream));
    k_shell_max<R><<<grid_blocks(n), kThreads, 0, c.stream>>>(c.geom, (const R*)c.d_V + (long)s * n, F.vmax,
                                                              shell_radius(c), shell_width(c));
    CU(cudaGetLastError());
    if ((st = delfield_into<R>(c, (const R*)c.d_V + (long)s * n, (R*)c.d_g2 + (long)s * n, (R*)c.d_lap + (long)s * n,
                               c.need_g2)))
      return st;
  }
  return MPDPFT_OK;
}

int Ctx::issue_delfield_of_V() {
  return rsize == sizeof(double) ? delfield_of_v_impl<double>(*this) : delfield_of_v_impl<float>(*this);
}

// ------------------------------------------------- standalone operators --
int Ctx::op_delfield(const double* f, double* grad2, double* lap, int layout, int mem) {
  if (!gradient) return set_error(MPDPFT_ERR_ARG, "context was not created with density_expression 5");
  int st;
  void* V0 = d_V;  // species 0 slot is used as staging
  if ((st = import_field(f, V0, layout, mem))) return st;
  const int S_save = S;
  const bool g2_save = need_g2;
  S = 1;
  need_g2 = true;  // the caller asks for |grad f|^2 as well
  st = issue_delfield_of_V();
  S = S_save;
  need_g2 = g2_save;
  if (st) return st;
  if (grad2 && (st = export_field(d_g2, grad2, layout, mem))) return st;
  if (lap && (st = export_field(d_lap, lap, layout, mem))) return st;
  return MPDPFT_OK;
}

int Ctx::op_vint(int type, int s, const double* const* nn, double* v_out, int layout, int mem) {
  if (s < 0 || s >= S) return set_error(MPDPFT_ERR_ARG, "species index out of range");
  if (!nn || !v_out) return set_error(MPDPFT_ERR_ARG, "null arrays");
  int st;
  for (int q = 0; q < S; ++q)
    if ((st = import_field(nn[q], (char*)d_tmp + (size_t)q * geom.n * rsize, layout, mem))) return st;
  const mpdpft_params saved = P;
  P.n_interactions = 1;
  P.interactions[0] = type;
  P.incremental_v = 1.0;
  const bool coul = type == MPDPFT_INT_HARTREE || type == MPDPFT_INT_HARTREE_INTER || type == MPDPFT_INT_COULOMB_CHARGED;
  if (coul && (!fft || !fft->spec[0])) {
    P = saved;
    return set_error(MPDPFT_ERR_ARG, "Coulomb terms need a context created with a Coulomb interaction");
  }
  void* out = (char*)d_V + (size_t)s * geom.n * rsize;  // staging
  if (coul) {
    st = rsize == sizeof(double) ? coulomb_terms<double>(*this, (const double*)d_tmp, (double*)d_vh)
                                 : coulomb_terms<float>(*this, (const float*)d_tmp, (float*)d_vh);
    if (!st) st = export_field((char*)d_vh + (size_t)s * geom.n * rsize, v_out, layout, mem);
  } else if (type == MPDPFT_INT_CONTACT_SELF || type == MPDPFT_INT_CONTACT_MUTUAL || type == MPDPFT_INT_DIRAC ||
             type == MPDPFT_INT_NONE) {
    st = pointwise_vint(type, s, out);
    if (!st) st = export_field(out, v_out, layout, mem);
  } else {
    st = set_error(MPDPFT_ERR_ARG, "unsupported interaction type");
  }
  P = saved;
  return st;
}

template <typename R>
__global__ void k_pointwise_vint(KParams kp, int type, int s, const R* dens, R* out) {
  const long n = kp.geom.n;
  for (long p = (long)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (long)gridDim.x * blockDim.x) {
    R v = R(0);
    if (type == MPDPFT_INT_CONTACT_SELF) v = R(2.0 * kp.beta) * dens[p];
    else if (type == MPDPFT_INT_CONTACT_MUTUAL) {
      R t = R(0);
      for (int q = 0; q < kp.S; ++q)
        if (q != s) t += dens[(long)q * n + p];
      v = R(kp.beta) * t;
    } else if (type == MPDPFT_INT_DIRAC) {
      R ns = dens[(long)s * n + p];
      ns = ns > R(0) ? ns : R(0);
      if (kp.geom.dim == 3) v = R(-kp.gamma_h) * cbrt(R(3.0 / kPi) * ns);
      else v = R(-2.0 * kp.gamma_h) * sqrt(R(2.0 / kPi) * ns);
    }
    out[p] = v;
  }
}

int Ctx::pointwise_vint(int type, int s, void* out) {
  KParams kp = kparams();
  const int blocks = grid_blocks(geom.n);
  if (rsize == sizeof(double)) k_pointwise_vint<double><<<blocks, kThreads, 0, stream>>>(kp, type, s, (const double*)d_tmp, (double*)out);
  else k_pointwise_vint<float><<<blocks, kThreads, 0, stream>>>(kp, type, s, (const float*)d_tmp, (float*)out);
  CU(cudaGetLastError());
  return MPDPFT_OK;
}

int Ctx::op_update_v(const double* const* nn, double incremental, double* const* v_out, int layout, int mem) {
  if (!nn || !v_out) return set_error(MPDPFT_ERR_ARG, "null arrays");
  int st;
  ScState h;
  if ((st = read_state(&h))) return st;
  const int cur = h.slot;
  for (int q = 0; q < S; ++q)
    if ((st = import_field(nn[q], (char*)d_nin + ((size_t)cur * S + q) * geom.n * rsize, layout, mem))) return st;
  h.inc_v = incremental;
  h.exit_loop = 0;
  CU(cudaMemcpyAsync(d_state, &h, sizeof(h), cudaMemcpyHostToDevice, stream));
  if (has_coulomb || gradient) {
    if ((st = issue_fft_terms())) return st;
  } else {
    const int blocks = grid_blocks(geom.n);
    KParams kp = kparams();
    if (!fft) return set_error(MPDPFT_ERR_ARG, "no FFT plan");
    if (rsize == sizeof(double))
      k_assemble_v<double><<<fft->vblocks, kThreads, 0, stream>>>(kp, d_state, (const double*)d_vext, nullptr,
                                                                  (const double*)d_nin, (double*)d_V, fft->vres_part,
                                                                  fft->vmax, 0.0, -1.0);
    else
      k_assemble_v<float><<<fft->vblocks, kThreads, 0, stream>>>(kp, d_state, (const float*)d_vext, nullptr,
                                                                 (const float*)d_nin, (float*)d_V, fft->vres_part,
                                                                 fft->vmax, 0.0, -1.0);
    (void)blocks;
    CU(cudaGetLastError());
  }
  for (int s = 0; s < S; ++s)
    if ((st = export_field((char*)d_V + (size_t)s * geom.n * rsize, v_out[s], layout, mem))) return st;
  return MPDPFT_OK;
}

// fftParallel semantics on an interleaved complex s^D field (see header).
int Ctx::op_fft(int sign, const double* in, double* out, int mem) {
  if (sign != -1 && sign != 1) return set_error(MPDPFT_ERR_ARG, "sign must be -1 or +1");
  if (!in || !out) return set_error(MPDPFT_ERR_ARG, "null arrays");
  FftPlan& F = *fft;
  int st;
  if (!F.cbuf && (st = alloc(&F.cbuf, 2 * rsize * geom.n))) return st;
  const long n = geom.n;
  double* din = d_io;
  double* dout = d_io;
  std::vector<double> stage;
  if (mem == MPDPFT_MEM_HOST) {  // d_io holds 2 * max(n_ref, n) doubles: one complex field
    CU(cudaMemcpyAsync(d_io, in, sizeof(double) * 2 * n, cudaMemcpyHostToDevice, stream));
  } else {
    din = (double*)in;
    dout = out;
  }
  const int blocks = grid_blocks(n);
  const double D = geom.dim;
  const double ph = -0.5 * D * kPi * geom.s;  // e^{-i D pi s/2} (mpDPFT.cpp:8228-8262)
  double cr_pre = 1.0, ci_pre = 0.0, cr_post, ci_post;
  if (sign < 0) {
    const double fac = std::pow(geom.dx, D);
    cr_post = fac * std::cos(ph);
    ci_post = fac * std::sin(ph);
  } else {
    const double fac = std::pow(1.0 / geom.L, D);
    cr_post = fac * std::cos(-ph);
    ci_post = fac * std::sin(-ph);
  }
  if (rsize == sizeof(double)) {
    using C = double2;
    k_cx_import<double><<<blocks, kThreads, 0, stream>>>(din, (C*)F.cbuf, n);
    k_alternate<double><<<blocks, kThreads, 0, stream>>>((C*)F.cbuf, geom, cr_pre, ci_pre);
    st = full_c2c(F.cbuf, sign);
    if (st) return st;
    k_alternate<double><<<blocks, kThreads, 0, stream>>>((C*)F.cbuf, geom, cr_post, ci_post);
    k_cx_export<double><<<blocks, kThreads, 0, stream>>>((const C*)F.cbuf, dout, n);
  } else {
    using C = float2;
    k_cx_import<float><<<blocks, kThreads, 0, stream>>>(din, (C*)F.cbuf, n);
    k_alternate<float><<<blocks, kThreads, 0, stream>>>((C*)F.cbuf, geom, cr_pre, ci_pre);
    st = full_c2c(F.cbuf, sign);
    if (st) return st;
    k_alternate<float><<<blocks, kThreads, 0, stream>>>((C*)F.cbuf, geom, cr_post, ci_post);
    k_cx_export<float><<<blocks, kThreads, 0, stream>>>((const C*)F.cbuf, dout, n);
  }
  CU(cudaGetLastError());
  if (mem == MPDPFT_MEM_HOST) {
    CU(cudaMemcpyAsync(out, d_io, sizeof(double) * 2 * n, cudaMemcpyDeviceToHost, stream));
    CU(cudaStreamSynchronize(stream));
  }
  return MPDPFT_OK;
}

// Unnormalised full complex transform of an s^D field along every axis,
// using the tile kernel with all s columns of each axis.
template <typename R>
static int full_c2c_impl(Ctx& c, void* buf, int sign) {
  FftPlan& F = *c.fft;
  const int s = F.s;
  const int dim = F.dim;
  for (int axis = 0; axis < dim; ++axis) {
    AxisArgs<R> a;
    std::memset(&a, 0, sizeof(a));
    a.s = s;
    a.tk = F.tk;
    a.dim = dim;
    a.plan = F.plan_s;
    a.twf = (const typename Cx<R>::T*)F.tw_s_f;
    a.twb = (const typename Cx<R>::T*)F.tw_s_b;
    a.dir = sign;
    a.data[0] = (typename Cx<R>::T*)buf;
    // treat the field as H = s columns with no separate Nyquist column
    a.M = s;  // columns 0..s-1 are all bulk
    a.H = s;
    long astride, ostride, nouter;
    if (dim == 3) {
      if (axis == 0) { astride = (long)s * s; ostride = s; nouter = s; }       // lines along x: (y, z)
      else if (axis == 1) { astride = s; ostride = (long)s * s; nouter = s; }  // along y: (x, z)
      else { astride = 1; ostride = s; nouter = (long)s * s; }                 // along z: rows
    } else {
      if (axis == 0) { astride = s; ostride = 0; nouter = 1; }
      else { astride = 1; ostride = s; nouter = s; }
    }
    a.astride = astride;
    a.ostride = ostride;
    a.nouter = nouter;
    if ((dim == 3 && axis == 2) || (dim == 2 && axis == 1)) {
      // contiguous lines: one column per outer row
      a.M = 1;
      a.ntile = 1;
      a.tk = 1;
    } else {
      a.ntile = s / a.tk;
      a.M = s;
    }
    a.nbulk = a.nouter * a.ntile;
    const size_t smem = 2 * sizeof(typename Cx<R>::T) * s * a.tk;
    // no Nyquist blocks: columns cover 0..s-1
    k_axis_c2c<R, 0, 0><<<dim3((unsigned)a.nbulk, 1), kFftThreads, smem, c.stream>>>(a);
    CU(cudaGetLastError());
  }
  return MPDPFT_OK;
}

int Ctx::full_c2c(void* buf, int sign) {
  return rsize == sizeof(double) ? full_c2c_impl<double>(*this, buf, sign) : full_c2c_impl<float>(*this, buf, sign);
}

// Stage timing with CUDA events (see mpdpft_profile_stage).
template <typename R>
static int profile_impl(Ctx& c, int stage, int reps, double* ms, double* bytes) {
  FftPlan& F = *c.fft;
  const double n = (double)c.geom.n;
  const double spec = (double)F.nspec * 2.0 * c.rsize;
  const double field = n * c.rsize;
  const int S = c.S;
  cudaEvent_t e0, e1;
  CU(cudaEventCreate(&e0));
  CU(cudaEventCreate(&e1));
  int st = MPDPFT_OK;
  double b = 0.0;
  const bool sc_stage = stage == MPDPFT_STAGE_SC_STEP || stage == MPDPFT_STAGE_ITERATION ||
                        stage == MPDPFT_STAGE_SC_MU || stage == MPDPFT_STAGE_SC_DENSITY || stage == MPDPFT_STAGE_SC_MIX;
  if ((stage == MPDPFT_STAGE_FFT_PLANE_FWD || stage == MPDPFT_STAGE_FFT_PLANE_INV) && !F.plane)
    return set_error(MPDPFT_ERR_ARG, "this grid does not use the plane kernels");
  if (!sc_stage) {
    if (!F.spec[0]) return set_error(MPDPFT_ERR_ARG, "context has no FFT buffers");
    CU(cudaMemsetAsync(F.spec[0], 0, (size_t)spec, c.stream));
    CU(cudaMemsetAsync(F.rtmp, 0, (size_t)field, c.stream));
  }
  auto one = [&]() -> int {
    switch (stage) {
      case MPDPFT_STAGE_SC_STEP: return c.launch_step(0);
      case MPDPFT_STAGE_FFT_Z_R2C: return launch_z_r2c<R>(c, (const R*)F.rtmp, PRO_NONE, 1, nullptr, F.spec[0], false);
      case MPDPFT_STAGE_FFT_Y: return F.dim == 3 ? launch_y<R>(c, &F.spec[0], 1, -1) : set_error(MPDPFT_ERR_ARG, "no y pass in 2D");
      case MPDPFT_STAGE_FFT_X: return launch_x<R>(c, F.spec[0], &F.spec[0], 1, MUL_SMOOTH, -0.01);
      case MPDPFT_STAGE_FFT_Z_C2R: return launch_z_c2r<R>(c, &F.spec[0], 1, EPI_STORE, (R*)F.rtmp, nullptr, 0.0);
      case MPDPFT_STAGE_ITERATION: return c.sc_step(1);
      case MPDPFT_STAGE_SC_MU: return c.launch_step(0, 1);
      case MPDPFT_STAGE_SC_DENSITY: return c.launch_step(0, 2);
      case MPDPFT_STAGE_SC_MIX: return c.launch_step(0, 4);
      case MPDPFT_STAGE_FFT_PLANE_FWD: return launch_plane_fwd<R>(c, (const R*)F.rtmp, PRO_NONE, F.spec[0], false);
      case MPDPFT_STAGE_FFT_PLANE_INV: return launch_plane_inv<R>(c, &F.spec[0], 1, EPI_STORE, (R*)F.rtmp, nullptr, 0.0);
      default: return set_error(MPDPFT_ERR_ARG, "unknown stage");
    }
  };
  if ((st = one())) return st;  // warm-up (and graph instantiation)
  CU(cudaEventRecord(e0, c.stream));
  for (int r = 0; r < reps && !st; ++r) st = one();
  CU(cudaEventRecord(e1, c.stream));
  CU(cudaEventSynchronize(e1));
  float t = 0.f;
  CU(cudaEventElapsedTime(&t, e0, e1));
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (st) return st;
  *ms = (double)t / reps;
  const int I = c.P.mixer ? c.P.pulay_scope : 1;
  switch (stage) {
    case MPDPFT_STAGE_SC_STEP:
      // V (+ Laplacian, |grad V|^2) read once by the mu search, n_in read,
      // residual written, I-1 older residuals read for the Gram row, 2I
      // history fields read and 1 written by the mix
      b = field * S * ((c.gradient ? 3 : 1) + 1 + 1 + (I - 1) + 2 * I + 1);
      if (c.assemble_in_step) b += field * S * 3;
      break;
    case MPDPFT_STAGE_SC_MU:  // V (+ Laplacian, |grad V|^2) read once
      b = field * S * (c.gradient ? 3 : 1);
      break;
    case MPDPFT_STAGE_SC_DENSITY:  // V, n_in, I-1 older residuals read; residual written
      b = field * S * (1 + 1 + (I - 1) + 1);
      break;
    case MPDPFT_STAGE_SC_MIX:  // I input densities and residuals read; mix and its copy written
      b = field * S * (2 * I + 2);
      break;
    case MPDPFT_STAGE_FFT_PLANE_FWD: b = field + spec; break;
    case MPDPFT_STAGE_FFT_PLANE_INV: b = spec + field; break;
    case MPDPFT_STAGE_FFT_Z_R2C: b = field + spec; break;
    case MPDPFT_STAGE_FFT_Y: b = 2.0 * spec; break;
    case MPDPFT_STAGE_FFT_X: b = 2.0 * spec; break;
    case MPDPFT_STAGE_FFT_Z_C2R: b = spec + field; break;
    default: b = 0.0; break;
  }
  if (bytes) *bytes = b;
  return MPDPFT_OK;
}

int Ctx::profile_stage(int stage, int reps, double* ms, double* bytes) {
  return rsize == sizeof(double) ? profile_impl<double>(*this, stage, reps, ms, bytes)
                                 : profile_impl<float>(*this, stage, reps, ms, bytes);
}

// ================================================================ batches ==
// DelField of a 2D field as the six argument sets of delfield_into's row
// and column passes: z[0] R2C (taper), x[0] derivatives + Laplacian, z[1]
// C2R -> |grad f|^2 (raw) and Laplacian, z[2] R2C of |grad f|^2, x[1]
// smoothing, z[3] C2R with the clamp at 0.
template <typename R>
struct Delfield2D {
  ZArgs<R> z[4];
  AxisArgs<R> x[2];
};

template <typename R>
static Delfield2D<R> delfield2d_args(Ctx& c, const R* f, R* g2, R* lap, void* const* spec, void* rtmp,
                                     unsigned long long* vmax) {
  const double smear = c.P.smearing_extent > 0.0 ? c.P.smearing_extent : 6.0 * c.geom.dx;
  const double sigma_c = -0.5 * smear * smear;
  const int pro = c.P.taper_off ? PRO_TAPER : PRO_NONE;
  void* outs[3] = {spec[1], spec[2], spec[3]};
  Delfield2D<R> d;
  d.z[0] = r2c_args<R>(c, f, pro, 1, nullptr, spec[0], false, vmax);
  d.x[0] = x_args<R>(c, spec[0], outs, 3, MUL_DERIV, sigma_c);
  d.z[1] = c2r_args<R>(c, outs, 3, EPI_GRAD, (R*)rtmp, lap, 0.0);
  d.z[2] = r2c_args<R>(c, (const R*)rtmp, PRO_NONE, 1, nullptr, spec[0], false, vmax);
  d.x[1] = x_args<R>(c, spec[0], &spec[0], 1, MUL_SMOOTH, sigma_c);
  d.z[3] = c2r_args<R>(c, &spec[0], 1, EPI_POS, g2, nullptr, 0.0);
  return d;
}

struct BatchFftClass {
  size_t rsize = 8;
  int count = 0;        // argument sets (members x species)
  int M = 0, s = 0, zl = 0, tk = 0, zblocks = 0;
  unsigned xgrid = 0;
  size_t smem_r2c = 0, smem_c2r = 0, smem_xct = 0, smem_xrt = 0;
  bool xct = false;
  void* d_z[4] = {nullptr, nullptr, nullptr, nullptr};  // ZArgs<R>[count]
  void* d_x[2] = {nullptr, nullptr};                    // AxisArgs<R>[count]
  // Coulomb terms (2D kernel): per argument set one transform of the
  // weighted densities sum_q w_q n_q into that species' vh
  bool coulomb = false;
  void* d_cz[2] = {nullptr, nullptr};  // ZArgs<R>[count]: R2C, C2R
  void* d_cx = nullptr;                // AxisArgs<R>[count]
};

// Weights w_q of the densities whose Coulomb potential is species s's
// Coulomb term, V_s = gammaH V_H[sum_q w_q n_q] (V_H linear): type 8 its
// own density, 21 the other species' (mpDPFT.cpp:2266-2285), 100 the
// charge density times q_s.
static void coulomb_weights(const Ctx& c, int s, double* w) {
  for (int q = 0; q < kMaxS; ++q) w[q] = 0.0;
  for (int a = 0; a < c.P.n_interactions; ++a) {
    const int t = c.P.interactions[a];
    if (t == MPDPFT_INT_HARTREE) w[s] += 1.0;
    else if (t == MPDPFT_INT_HARTREE_INTER)
      for (int q = 0; q < c.S; ++q) w[q] += q == s ? 0.0 : 1.0;
    else if (t == MPDPFT_INT_COULOMB_CHARGED)
      for (int q = 0; q < c.S; ++q) w[q] += c.P.charges[s] * c.P.charges[q];
  }
}

template <typename R>
static int batch_fft_build(const std::vector<BatchMember>& members, unsigned long long* vmax_all, BatchFftClass* b) {
  std::vector<ZArgs<R>> z[4], cz[2];
  std::vector<AxisArgs<R>> x[2], cx;
  const bool coul = members[0].c->has_coulomb;
  for (const BatchMember& m : members) {
    Ctx& c = *m.c;
    FftPlan& f = *c.fft;
    const long n = c.geom.n;
    for (int s = 0; s < c.S; ++s) {
      void* spec[4];
      void* rtmp;
      double* zpart = f.zpart;
      if (s == 0) {
        for (int i = 0; i < 4; ++i) spec[i] = f.spec[i];
        rtmp = f.rtmp;
      } else {  // the species run concurrently: scratch of their own
        int st;
        for (int i = 0; i < 4; ++i)
          if ((st = c.alloc(&spec[i], 2 * c.rsize * f.nspec))) return st;
        if ((st = c.alloc(&rtmp, c.rsize * n))) return st;
        if (coul && (st = c.alloc((void**)&zpart, sizeof(double) * (f.zblocks + 1)))) return st;
      }
      Delfield2D<R> d = delfield2d_args<R>(c, (const R*)c.d_V + (long)s * n, (R*)c.d_g2 + (long)s * n,
                                           (R*)c.d_lap + (long)s * n, spec, rtmp,
                                           vmax_all + (long)m.index * kMaxS + s);
      const int* skip = &c.d_state->exit_loop;
      for (int i = 0; i < 4; ++i) { d.z[i].skip = skip; z[i].push_back(d.z[i]); }
      for (int i = 0; i < 2; ++i) { d.x[i].skip = skip; x[i].push_back(d.x[i]); }
      if (coul) {  // HartreeRepulsion 2D of the weighted current densities into vh of species s
        double w[kMaxS];
        coulomb_weights(c, s, w);
        const bool plain = c.S == 1 && w[0] == 1.0;
        ZArgs<R> a0 = r2c_args<R>(c, (const R*)c.d_cur, plain ? PRO_NONE : PRO_CHARGE, c.S, w, spec[0], true,
                                  vmax_all + (long)m.index * kMaxS + s);
        a0.part = zpart;
        AxisArgs<R> ax = x_args<R>(c, spec[0], &spec[0], 1, MUL_COULOMB_2D, 0.0);
        ax.f0_part = zpart;
        ax.f0_blocks = f.zblocks;
        ZArgs<R> a1 = c2r_args<R>(c, &spec[0], 1, EPI_COULOMB, (R*)c.d_vh + (long)s * n, nullptr,
                                  2.0 * kPi * c.P.gamma_h);
        a1.f0_part = zpart;
        a1.f0_blocks = f.zblocks;
        a0.skip = skip;
        ax.skip = skip;
        a1.skip = skip;
        cz[0].push_back(a0);
        cz[1].push_back(a1);
        cx.push_back(ax);
      }
    }
  }
  Ctx& c0 = *members[0].c;
  FftPlan& f = *c0.fft;
  b->rsize = sizeof(R);
  b->count = (int)z[0].size();
  b->M = f.M;
  b->s = f.s;
  b->zl = f.zl;
  b->tk = f.tk;
  b->zblocks = f.zblocks;
  b->xgrid = x_grid<R>(x[0][0]);
  b->smem_r2c = r2c_smem<R>(f);
  b->smem_c2r = c2r_smem<R>(f);
  b->smem_xct = x_smem_ct<R>(f);
  b->smem_xrt = x_smem_rt<R>(f);
  b->xct = f.tk == ct_width<R>() && x_ct_fits<R>(f);
  for (int i = 0; i < 4; ++i) {
    CU(cudaMalloc(&b->d_z[i], sizeof(ZArgs<R>) * b->count));
    CU(cudaMemcpy(b->d_z[i], z[i].data(), sizeof(ZArgs<R>) * b->count, cudaMemcpyHostToDevice));
  }
  for (int i = 0; i < 2; ++i) {
    CU(cudaMalloc(&b->d_x[i], sizeof(AxisArgs<R>) * b->count));
    CU(cudaMemcpy(b->d_x[i], x[i].data(), sizeof(AxisArgs<R>) * b->count, cudaMemcpyHostToDevice));
  }
  b->coulomb = coul;
  if (coul) {
    for (int i = 0; i < 2; ++i) {
      CU(cudaMalloc(&b->d_cz[i], sizeof(ZArgs<R>) * b->count));
      CU(cudaMemcpy(b->d_cz[i], cz[i].data(), sizeof(ZArgs<R>) * b->count, cudaMemcpyHostToDevice));
    }
    CU(cudaMalloc(&b->d_cx, sizeof(AxisArgs<R>) * b->count));
    CU(cudaMemcpy(b->d_cx, cx.data(), sizeof(AxisArgs<R>) * b->count, cudaMemcpyHostToDevice));
  }
  return MPDPFT_OK;
}

int batch_fft_create(const std::vector<BatchMember>& members, unsigned long long* vmax_all, BatchFftClass** out) {
  *out = nullptr;
  if (members.empty()) return set_error(MPDPFT_ERR_ARG, "empty batch class");
  for (const BatchMember& m : members) {
    const Ctx& c = *m.c;
    if (c.P.dim != 2 || !c.gradient || !c.fft || c.fft->plane)
      return set_error(MPDPFT_ERR_ARG, "batched DelField: 2D gradient-corrected solves only");
    if (c.P.steps != members[0].c->P.steps || c.rsize != members[0].c->rsize)
      return set_error(MPDPFT_ERR_ARG, "batched DelField: one grid size and precision per class");
  }
  BatchFftClass* b = new BatchFftClass;
  const int st = members[0].c->rsize == sizeof(double) ? batch_fft_build<double>(members, vmax_all, b)
                                                       : batch_fft_build<float>(members, vmax_all, b);
  if (st) {
    batch_fft_destroy(b);
    return st;
  }
  *out = b;
  return MPDPFT_OK;
}

template <typename R>
static int batch_fft_issue_t(BatchFftClass* b, cudaStream_t st, bool coulomb_only) {
  const ZArgs<R>* z[4];
  const AxisArgs<R>* x[2];
  for (int i = 0; i < 4; ++i) z[i] = (const ZArgs<R>*)b->d_z[i];
  for (int i = 0; i < 2; ++i) x[i] = (const AxisArgs<R>*)b->d_x[i];
  const dim3 zg(b->zblocks, b->count), xg(b->xgrid, b->count);
  auto r2c = [&](const ZArgs<R>* a) {
    if (b->zl != 16 || !launch_z_r2c_b_ct<R, 16>(b->M, zg, b->smem_r2c, st, a))
      k_z_r2c_b<R, 0, 0><<<zg, kFftThreads, b->smem_r2c, st>>>(a);
  };
  auto c2r = [&](const ZArgs<R>* a) {
    if (b->zl != 16 || !launch_z_c2r_b_ct<R, 16>(b->M, zg, b->smem_c2r, st, a))
      k_z_c2r_b<R, 0, 0><<<zg, kFftThreads, b->smem_c2r, st>>>(a);
  };
  auto xrt = [&](const AxisArgs<R>* a) {
    if (!b->xct || !launch_x_b_ct<R, ct_width<R>()>(b->s, xg, b->smem_xct, st, a))
      k_x_roundtrip_b<R, 0, 0><<<xg, kFftThreads, b->smem_xrt, st>>>(a);
  };
  if (coulomb_only) {
    r2c((const ZArgs<R>*)b->d_cz[0]);
    xrt((const AxisArgs<R>*)b->d_cx);
    c2r((const ZArgs<R>*)b->d_cz[1]);
    CU(cudaGetLastError());
    return MPDPFT_OK;
  }
  r2c(z[0]);
  xrt(x[0]);
  c2r(z[1]);
  r2c(z[2]);
  xrt(x[1]);
  c2r(z[3]);
  CU(cudaGetLastError());
  return MPDPFT_OK;
}

int batch_fft_issue(BatchFftClass* b, cudaStream_t st) {
  return b->rsize == sizeof(double) ? batch_fft_issue_t<double>(b, st, false) : batch_fft_issue_t<float>(b, st, false);
}

bool batch_fft_has_coulomb(const BatchFftClass* b) { return b && b->coulomb; }

int batch_fft_issue_coulomb(BatchFftClass* b, cudaStream_t st) {
  if (!b->coulomb) return MPDPFT_OK;
  return b->rsize == sizeof(double) ? batch_fft_issue_t<double>(b, st, true) : batch_fft_issue_t<float>(b, st, true);
}

void batch_fft_destroy(BatchFftClass* b) {
  if (!b) return;
  for (int i = 0; i < 4; ++i) cudaFree(b->d_z[i]);
  for (int i = 0; i < 2; ++i) cudaFree(b->d_x[i]);
  for (int i = 0; i < 2; ++i) cudaFree(b->d_cz[i]);
  cudaFree(b->d_cx);
  delete b;
}

// ============================================================ adjoint ops ==
// out = IFFT(m(k) FFT(in)) on the pass kernels, one output:
//   SPEC_DERIV   j < dim: d/dx_j with the DelField smoothing e^{sigma k^2} and
//                the Nyquist index of axis j dropped; j = dim: the Laplacian
//                smoothed twice (the multipliers of DelField's outputs);
//   SPEC_SMOOTH  e^{sigma k^2};
//   SPEC_COULOMB the Coulomb multiplier of the context's kernel times
//                4 pi coef, with the regularised kernel's terms in the total
//                charge left out (k = 0 mode, Gaussian subtraction,
//                compensation term): a translation-invariant symmetric part.
template <typename R>
static int spectral_impl(Ctx& c, const R* in, int kind, int j, R* out, double coef) {
  FftPlan& f = *c.fft;
  int st;
  const double smear = c.P.smearing_extent > 0.0 ? c.P.smearing_extent : 6.0 * c.geom.dx;
  const double sigma_c = -0.5 * smear * smear;
  int mul = MUL_SMOOTH;
  if (kind == SPEC_DERIV) mul = MUL_DERIV;
  else if (kind == SPEC_COULOMB) mul = c.P.coulomb_kernel == MPDPFT_COULOMB_TRUNCATED ? MUL_COULOMB_TRUNC : MUL_COULOMB_REG;
  if ((st = launch_z_r2c<R>(c, in, PRO_NONE, 1, nullptr, f.spec[0], false))) return st;
  if (f.dim == 3 && (st = launch_y<R>(c, &f.spec[0], 1, -1))) return st;
  AxisArgs<R> a = x_args<R>(c, f.spec[0], &f.spec[0], 1, mul, sigma_c);
  a.f0_blocks = 0;  // no k = 0 / total-charge terms
  a.o0 = kind == SPEC_DERIV ? j : 0;
  if ((st = launch_x_args<R>(c, a))) return st;
  if (f.dim == 3 && (st = launch_y<R>(c, &f.spec[0], 1, +1))) return st;
  if (kind == SPEC_COULOMB) return launch_z_c2r<R>(c, &f.spec[0], 1, EPI_SCALE, out, nullptr, 4.0 * kPi * coef);
  return launch_z_c2r<R>(c, &f.spec[0], 1, EPI_STORE, out, nullptr, 0.0);
}

int Ctx::spectral(const void* in, int kind, int j, void* out, double coef) {
  if (!fft) return set_error(MPDPFT_ERR_ARG, "no FFT plan");
  return rsize == sizeof(double) ? spectral_impl<double>(*this, (const double*)in, kind, j, (double*)out, coef)
                                 : spectral_impl<float>(*this, (const float*)in, kind, j, (float*)out, coef);
}

// The forward Hartree operator (coefficient gammaH, the context's kernel) on
// one field.
int Ctx::coulomb_field(const void* in, void* out) {
  double one = 1.0;
  return rsize == sizeof(double)
             ? coulomb_into<double>(*this, (const double*)in, 1, &one, (double*)out, P.gamma_h)
             : coulomb_into<float>(*this, (const float*)in, 1, &one, (float*)out, P.gamma_h);
}

// ============================================================ autotuner ==
// 3D grids whose x-plane kernels are instantiated have two complete
// transform paths: x-plane kernels (z and y passes fused per plane, TMA bulk
// copies) and one pass per axis.  Which is faster depends on the grid size,
// precision and the mix of transforms an iteration runs, so the first
// context of each (grid, precision, functional, Coulomb) kind times the
// transforms of one SC iteration (DelField of every species and the Coulomb
// terms) both ways on its own buffers and keeps the faster; later contexts
// of the same kind reuse the choice.  MPDPFT_FFT_PATH=plane|pass forces a path.
// Every 3D grid also tunes the tile widths: lines per tile of the Y and X
// passes (16 or 8 in FP32, 8 or 4 in FP64) and rows per block of the Z
// passes (16 or 8, pass path); each width has compile-time kernels, and a
// line's arithmetic does not depend on the width, so every configuration
// gives the same bits.  MPDPFT_FFT_TILES=<lines>,<rows> forces the widths.
template <typename R>
static int tune_transforms(Ctx& c) {
  int st;
  FftPlan& F = *c.fft;
  const long n = c.geom.n;
  if (c.has_coulomb) {
    double one = 1.0;
    if ((st = coulomb_into<R>(c, (const R*)c.d_V, 1, &one, (R*)c.d_tmp, c.P.gamma_h))) return st;
  }
  if (c.gradient)
    for (int s = 0; s < c.S; ++s) {
      CU(cudaMemsetAsync(F.vmax, 0, sizeof(unsigned long long), c.stream));
      if ((st = delfield_into<R>(c, (const R*)c.d_V + (long)s * n, (R*)c.d_g2 + (long)s * n,
                                 (R*)c.d_lap + (long)s * n, c.need_g2)))
        return st;
    }
  return MPDPFT_OK;
}

int Ctx::fft_autotune() {
  FftPlan& F = *fft;
  F.tuned = 0;
  if (F.dim != 3 || !(gradient || has_coulomb)) return MPDPFT_OK;  // no transforms in the iteration
  // candidate configurations: path (plane where instantiated, pass) x tile
  // width of the Y/X passes (tk0, tk0/2) x rows per block of the Z passes
  // (16, 8; pass path only)
  struct Cfg { bool plane; int tk, zl; };
  const int tk0 = F.tk;
  Cfg cfg[6];
  int ncfg = 0;
  const char* env = std::getenv("MPDPFT_FFT_PATH");
  const bool forced = env && (!std::strcmp(env, "pass") || !std::strcmp(env, "plane"));
  for (int path = 0; path < 2; ++path) {
    const bool plane = path == 0;
    if (plane && !F.plane) continue;
    if (forced && plane != !std::strcmp(env, "plane")) continue;
    for (int t = 0; t < 2; ++t) {
      const int tk = t ? tk0 / 2 : tk0;
      if (tk < 4 && t) continue;
      for (int z = 0; z < (plane ? 1 : 2); ++z) cfg[ncfg++] = Cfg{plane, tk, z ? 8 : 16};
    }
  }
  // MPDPFT_FFT_TILES=<tk>,<zl> keeps only that tile configuration
  const char* tiles = std::getenv("MPDPFT_FFT_TILES");
  int want_tk = 0, want_zl = 0;
  if (tiles && std::sscanf(tiles, "%d,%d", &want_tk, &want_zl) == 2) {
    int k = 0;
    for (int i = 0; i < ncfg; ++i)
      if (cfg[i].tk == want_tk && (cfg[i].plane || cfg[i].zl == want_zl)) cfg[k++] = cfg[i];
    ncfg = k;
    if (ncfg == 0) return set_error(MPDPFT_ERR_ARG, "MPDPFT_FFT_TILES: no such configuration for this grid");
  }
  auto apply = [&](const Cfg& c) {
    F.plane = c.plane;
    F.tk = c.tk;
    F.zl = c.zl;
    F.zblocks = (int)((F.rows + F.zl - 1) / F.zl);
  };
  using Key = std::tuple<int, size_t, int, int, int, int, int>;
  static std::mutex mu;
  static std::map<Key, std::array<double, 5>> cache;  // plane ms, pass ms, plane, tk, zl
  const Key key{F.s, rsize, gradient ? 1 : 0, has_coulomb, S, forced ? 1 + (env[1] == 'l') : 0, want_tk * 64 + want_zl};
  {
    std::lock_guard<std::mutex> lock(mu);
    auto it = cache.find(key);
    if (it != cache.end()) {
      F.tune_ms[0] = it->second[0];
      F.tune_ms[1] = it->second[1];
      apply(Cfg{it->second[2] != 0.0, (int)it->second[3], (int)it->second[4]});
      F.tuned = forced ? 3 : 2;
      return MPDPFT_OK;
    }
  }
  if (ncfg == 1) {  // nothing to choose
    apply(cfg[0]);
    F.tuned = forced ? 3 : 0;
    return MPDPFT_OK;
  }
  cudaEvent_t e0, e1;
  CU(cudaEventCreate(&e0));
  CU(cudaEventCreate(&e1));
  int st = MPDPFT_OK;
  double best = 1e300;
  int ibest = 0;
  F.tune_ms[0] = F.tune_ms[1] = 0.0;
  for (int i = 0; i < ncfg && !st; ++i) {
    apply(cfg[i]);
    for (int rep = 0; rep < 2 && !st; ++rep)  // warm-up
      st = rsize == sizeof(double) ? tune_transforms<double>(*this) : tune_transforms<float>(*this);
    if (st) break;
    const int reps = 5;
    cudaEventRecord(e0, stream);
    for (int rep = 0; rep < reps && !st; ++rep)
      st = rsize == sizeof(double) ? tune_transforms<double>(*this) : tune_transforms<float>(*this);
    cudaEventRecord(e1, stream);
    if (cudaEventSynchronize(e1) != cudaSuccess) st = set_error(MPDPFT_ERR_CUDA, "autotuner timing");
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    const double t = ms / reps;
    double& slot = F.tune_ms[cfg[i].plane ? 0 : 1];
    if (slot == 0.0 || t < slot) slot = t;
    if (t < best) { best = t; ibest = i; }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  for (int i = 0; i < 6; ++i) cnt[i] = 0;
  if (st) return st;
  apply(cfg[ibest]);
  F.tuned = forced ? 3 : 1;
  std::lock_guard<std::mutex> lock(mu);
  cache[key] = {F.tune_ms[0], F.tune_ms[1], F.plane ? 1.0 : 0.0, (double)F.tk, (double)F.zl};
  return MPDPFT_OK;
}

int Ctx::fft_tiles(int* axis_lines, int* z_rows) {
  if (!fft) return set_error(MPDPFT_ERR_ARG, "no FFT plan");
  if (axis_lines) *axis_lines = fft->tk;
  if (z_rows) *z_rows = fft->zl;
  return MPDPFT_OK;
}

int Ctx::fft_config(int* path, double* ms_plane, double* ms_pass, int* how) {
  if (!fft) return set_error(MPDPFT_ERR_ARG, "no FFT plan");
  if (path) *path = fft->plane ? 1 : 0;
  if (ms_plane) *ms_plane = fft->tune_ms[0];
  if (ms_pass) *ms_pass = fft->tune_ms[1];
  if (how) *how = fft->tuned;
  return MPDPFT_OK;
}

double* batch_vres_part(const Ctx& c) { return c.fft ? c.fft->vres_part : nullptr; }

// ---- batched V assembly: one launch over every member, block table ------
template <typename R>
struct AssembleArgs {
  KParams kp;
  const ScState* st;
  const R* vext;
  const R* vh;  // Coulomb terms [S][n] or null
  const R* nin;
  R* V;
  double* vres_part;
  unsigned long long* vmax;  // [kMaxS]
  double shell_r, shell_w;
};

template <typename R>
__global__ void k_assemble_v_b(const AssembleArgs<R>* __restrict__ args, const int4* __restrict__ tab, int update) {
  const int4 t = tab[blockIdx.x];  // (member, block, blocks)
  const AssembleArgs<R>& a = args[t.x];
  assemble_v_body<R>(a.kp, a.st, a.vext, a.vh, a.nin, a.V, a.vres_part, a.vmax, a.shell_r, a.shell_w, a.kp.S,
                     update, t.y, t.z);
}

struct BatchAssemble {
  size_t rsize = 8;
  void* d_args = nullptr;
  int4* d_tab = nullptr;
  int blocks = 0;
};

template <typename R>
static int batch_assemble_build(const std::vector<BatchMember>& members, unsigned long long* vmax_all,
                                BatchAssemble* b, std::vector<int>* blocks_out) {
  std::vector<AssembleArgs<R>> args;
  std::vector<int4> tab;
  blocks_out->clear();
  for (size_t k = 0; k < members.size(); ++k) {
    Ctx& c = *members[k].c;
    AssembleArgs<R> a;
    std::memset(&a, 0, sizeof(a));
    a.kp = c.kparams();
    a.st = c.d_state;
    a.vext = (const R*)c.d_vext;
    a.vh = c.has_coulomb ? (const R*)c.d_vh : nullptr;
    a.nin = (const R*)c.d_nin;
    a.V = (R*)c.d_V;
    a.vres_part = c.fft->vres_part;
    a.vmax = vmax_all + (long)members[k].index * kMaxS;
    a.shell_r = shell_radius(c);
    a.shell_w = shell_width(c);
    args.push_back(a);
    // 8 points a thread, at most the rows of the residual partials
    int nb = (int)std::min<long>((c.geom.n + 8L * kThreads - 1) / (8L * kThreads), c.fft->vblocks);
    nb = std::max(nb, 1);
    for (int i = 0; i < nb; ++i) tab.push_back(make_int4((int)k, i, nb, 0));
    blocks_out->push_back(nb);
  }
  b->rsize = sizeof(R);
  b->blocks = (int)tab.size();
  CU(cudaMalloc(&b->d_args, sizeof(AssembleArgs<R>) * args.size()));
  CU(cudaMemcpy(b->d_args, args.data(), sizeof(AssembleArgs<R>) * args.size(), cudaMemcpyHostToDevice));
  CU(cudaMalloc((void**)&b->d_tab, sizeof(int4) * tab.size()));
  CU(cudaMemcpy(b->d_tab, tab.data(), sizeof(int4) * tab.size(), cudaMemcpyHostToDevice));
  return MPDPFT_OK;
}

int batch_assemble_create(const std::vector<BatchMember>& members, unsigned long long* vmax_all,
                          BatchAssemble** out, std::vector<int>* blocks_out) {
  *out = nullptr;
  if (members.empty()) return set_error(MPDPFT_ERR_ARG, "empty batch");
  for (const BatchMember& m : members)
    if (!m.c->fft || m.c->has_coulomb != members[0].c->has_coulomb)
      return set_error(MPDPFT_ERR_ARG, "batched V assembly: the solves share their interactions");
  BatchAssemble* b = new BatchAssemble;
  const int st = members[0].c->rsize == sizeof(double) ? batch_assemble_build<double>(members, vmax_all, b, blocks_out)
                                                       : batch_assemble_build<float>(members, vmax_all, b, blocks_out);
  if (st) {
    batch_assemble_destroy(b);
    return st;
  }
  *out = b;
  return MPDPFT_OK;
}

int batch_assemble_issue(BatchAssemble* b, int update, cudaStream_t st) {
  if (b->rsize == sizeof(double))
    k_assemble_v_b<double><<<b->blocks, kThreads, 0, st>>>((const AssembleArgs<double>*)b->d_args, b->d_tab, update);
  else
    k_assemble_v_b<float><<<b->blocks, kThreads, 0, st>>>((const AssembleArgs<float>*)b->d_args, b->d_tab, update);
  CU(cudaGetLastError());
  return MPDPFT_OK;
}

void batch_assemble_destroy(BatchAssemble* b) {
  if (!b) return;
  cudaFree(b->d_args);
  cudaFree(b->d_tab);
  delete b;
}

}  // namespace mpdpft
