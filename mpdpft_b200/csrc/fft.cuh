// fft.cuh -- shared-memory Stockham FFT building blocks (sm_100a).
//
// Transforms of length len are done by the threads of one block on a tile of
// nl lines held in shared memory as element (t, l) at t * nl + l, so that
// adjacent threads work on adjacent lines and the tile loads from global
// memory are coalesced across lines.  Stages are radix 4, 2 and 3 (3 covers
// 192 = 2^6 * 3); the Stockham form needs no bit reversal.  Twiddles come
// from a per-length table tw[t] = exp(-+2 pi i t / len).
#pragma once
#include "common.cuh"

namespace mpdpft {

template <typename R>
struct Cx;
template <>
struct Cx<float> { using T = float2; };
template <>
struct Cx<double> { using T = double2; };

template <typename C>
__device__ __forceinline__ C cadd(C a, C b) { return {a.x + b.x, a.y + b.y}; }
template <typename C>
__device__ __forceinline__ C csub(C a, C b) { return {a.x - b.x, a.y - b.y}; }
template <typename C>
__device__ __forceinline__ C cmul(C a, C b) { return {a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x}; }
template <typename C, typename R>
__device__ __forceinline__ C cscale(C a, R s) { return {a.x * s, a.y * s}; }
template <typename C>
__device__ __forceinline__ C cconj(C a) { return {a.x, -a.y}; }
// multiply by +i (dir > 0) or -i (dir < 0)
template <typename C>
__device__ __forceinline__ C cmul_i(C a, int dir) { return dir > 0 ? C{-a.y, a.x} : C{a.y, -a.x}; }

constexpr int kMaxRadixStages = 12;

struct RadixPlan {
  int len;
  int n;                      // number of stages
  int r[kMaxRadixStages];     // radices in order
};

// One Stockham stage sweep over the tile.  dir = -1 forward, +1 inverse.
template <typename C>
__device__ __forceinline__ void stockham_stage(const C* __restrict__ src, C* __restrict__ dst, int len, int nl,
                                               int r, int stride, const C* __restrict__ tw, int dir) {
  const int L = len / stride;
  const int m = L / r;
  const int nbf = (len / r) * nl;
  using R = decltype(C{}.x);
  for (int w = threadIdx.x; w < nbf; w += blockDim.x) {
    const int l = w % nl;
    const int b = w / nl;
    const int q = b / stride, k = b % stride;
    C a[4];
#pragma unroll
    for (int t = 0; t < 4; ++t)
      if (t < r) a[t] = src[(k + stride * (q + t * m)) * nl + l];
    C o[4];
    if (r == 4) {
      C s02 = cadd(a[0], a[2]), d02 = csub(a[0], a[2]);
      C s13 = cadd(a[1], a[3]), d13 = csub(a[1], a[3]);
      C j13 = cmul_i(d13, dir);  // W = e^{dir 2 pi i/4}: a1 W + a3 W^3 = dir*i (a1 - a3)
      o[0] = cadd(s02, s13);
      o[1] = cadd(d02, j13);
      o[2] = csub(s02, s13);
      o[3] = csub(d02, j13);
    } else if (r == 2) {
      o[0] = cadd(a[0], a[1]);
      o[1] = csub(a[0], a[1]);
    } else {  // r == 3
      const R c = R(-0.5);
      const R sd = R(dir) * R(0.8660254037844386);
      C t1 = cadd(a[1], a[2]), t2 = csub(a[1], a[2]);
      C base = {a[0].x + c * t1.x, a[0].y + c * t1.y};
      C rot = {-sd * t2.y, sd * t2.x};  // i * sd * t2
      o[0] = cadd(a[0], t1);
      o[1] = cadd(base, rot);
      o[2] = csub(base, rot);
    }
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      if (u >= r) break;
      C v = o[u];
      if (u > 0 && q > 0) v = cmul(v, tw[q * u * stride]);
      dst[(k + stride * (r * q + u)) * nl + l] = v;
    }
  }
}

// Full transform of the tile; returns the buffer holding the result.
template <typename C>
__device__ __forceinline__ C* tile_fft(C* A, C* B, const RadixPlan& plan, int nl, const C* tw, int dir) {
  C* src = A;
  C* dst = B;
  int stride = 1;
  for (int st = 0; st < plan.n; ++st) {
    stockham_stage<C>(src, dst, plan.len, nl, plan.r[st], stride, tw, dir);
    __syncthreads();
    C* t = src; src = dst; dst = t;
    stride *= plan.r[st];
  }
  return src;
}

// ------------------------------------------------ compile-time lengths ----
// Radix sequence for a length known at compile time: 8 while possible, then
// 4, 2 and 3.  All index arithmetic of a stage then folds to constants.
__host__ __device__ constexpr int ct_radix(int m) {
  return (m % 8 == 0) ? 8 : (m % 4 == 0) ? 4 : (m % 2 == 0) ? 2 : (m % 3 == 0) ? 3 : 1;
}
__host__ __device__ constexpr int ct_stage_radix(int n, int i) {
  int m = n;
  for (int k = 0; k < i; ++k) m /= ct_radix(m);
  return ct_radix(m);
}
__host__ __device__ constexpr int ct_num_stages(int n) {
  int m = n, k = 0;
  while (m > 1 && ct_radix(m) > 1) { m /= ct_radix(m); ++k; }
  return m == 1 ? k : -1;
}

// In-register DFT of R points, W = e^{dir 2 pi i / R}.
template <int R, typename C>
__device__ __forceinline__ void reg_dft(C (&a)[8], int dir) {
  using T = decltype(C{}.x);
  if constexpr (R == 2) {
    C t = a[0];
    a[0] = cadd(t, a[1]);
    a[1] = csub(t, a[1]);
  } else if constexpr (R == 3) {
    const T c = T(-0.5), sd = T(dir) * T(0.8660254037844386);
    C t1 = cadd(a[1], a[2]), t2 = csub(a[1], a[2]);
    C base = {a[0].x + c * t1.x, a[0].y + c * t1.y};
    C rot = {-sd * t2.y, sd * t2.x};
    a[0] = cadd(a[0], t1);
    a[1] = cadd(base, rot);
    a[2] = csub(base, rot);
  } else if constexpr (R == 4) {
    C s02 = cadd(a[0], a[2]), d02 = csub(a[0], a[2]);
    C s13 = cadd(a[1], a[3]), j13 = cmul_i(csub(a[1], a[3]), dir);
    a[0] = cadd(s02, s13);
    a[1] = cadd(d02, j13);
    a[2] = csub(s02, s13);
    a[3] = csub(d02, j13);
  } else {  // R == 8: two 4-point DFTs (even/odd) and W8^u combinations
    C e0 = cadd(a[0], a[4]), e1 = csub(a[0], a[4]);
    C e2 = cadd(a[2], a[6]), e3 = cmul_i(csub(a[2], a[6]), dir);
    C E0 = cadd(e0, e2), E2 = csub(e0, e2), E1 = cadd(e1, e3), E3 = csub(e1, e3);
    C o0 = cadd(a[1], a[5]), o1 = csub(a[1], a[5]);
    C o2 = cadd(a[3], a[7]), o3 = cmul_i(csub(a[3], a[7]), dir);
    C O0 = cadd(o0, o2), O2 = csub(o0, o2), O1 = cadd(o1, o3), O3 = csub(o1, o3);
    const T h = T(0.7071067811865476);
    // W8 = h (1 + dir i), W8^2 = dir i, W8^3 = h (-1 + dir i)
    C w1 = {h * (O1.x - T(dir) * O1.y), h * (O1.y + T(dir) * O1.x)};
    C w2 = cmul_i(O2, dir);
    C w3 = {h * (-O3.x - T(dir) * O3.y), h * (-O3.y + T(dir) * O3.x)};
    a[0] = cadd(E0, O0);
    a[4] = csub(E0, O0);
    a[1] = cadd(E1, w1);
    a[5] = csub(E1, w1);
    a[2] = cadd(E2, w2);
    a[6] = csub(E2, w2);
    a[3] = cadd(E3, w3);
    a[7] = csub(E3, w3);
  }
}

// Element (t, l) of an NL-line tile: rows padded to NL + 1, and the line
// index XOR-ed with (t / 8) mod NL.  The element-fastest first stage writes
// the radix-8 outputs of consecutive threads 8 rows apart, which padding
// alone maps onto two banks (8-way conflicts); the swizzle spreads them over
// all banks while line-fastest accesses stay conflict-free (NL a power of 2).
template <int NL>
__device__ __forceinline__ int tile_at(int t, int l) {
  static_assert((NL & (NL - 1)) == 0, "tile width must be a power of two");
  return t * (NL + 1) + (l ^ ((t >> 3) & (NL - 1)));
}

// Stockham stages STAGE .. END-1 of a length-N transform of an NL-line tile
// (element (t, l) at tile_at<NL>(t, l)).
template <typename C, int N, int NL, int STAGE, int STRIDE, int END = ct_num_stages(N)>
__device__ __forceinline__ void ct_stages(C* __restrict__ src, C* __restrict__ dst, const C* __restrict__ tw,
                                          int dir) {
  if constexpr (STAGE < END) {
    constexpr int R = ct_stage_radix(N, STAGE);
    constexpr int L = N / STRIDE;
    constexpr int M = L / R;
    constexpr int NBF = (N / R) * NL;
    for (int w = threadIdx.x; w < NBF; w += blockDim.x) {
      const int l = w % NL;
      const int b = w / NL;
      const int q = b / STRIDE, k = b % STRIDE;
      C a[8];
#pragma unroll
      for (int t = 0; t < R; ++t) a[t] = src[tile_at<NL>(k + STRIDE * (q + t * M), l)];
      reg_dft<R>(a, dir);
#pragma unroll
      for (int u = 0; u < R; ++u) {
        C v = a[u];
        if (u > 0) v = cmul(v, tw[q * u * STRIDE]);
        dst[tile_at<NL>(k + STRIDE * (R * q + u), l)] = v;
      }
    }
    __syncthreads();
    ct_stages<C, N, NL, STAGE + 1, STRIDE * R, END>(dst, src, tw, dir);
  }
}

__host__ __device__ constexpr int ct_stride_before(int n, int stage) {
  int st = 1;
  for (int k = 0; k < stage; ++k) st *= ct_stage_radix(n, k);
  return st;
}

// Length-N transforms of NL lines with the first stage reading its inputs
// from `load(t, l)` straight into registers and the last stage handing its
// outputs to `store(t, l, v)`; only the middle stages exchange through the
// shared-memory tile A/B (layout tile_at<NL>).  ELEM_FAST maps consecutive
// threads to consecutive elements of a line in the first and last stages
// (contiguous rows); otherwise to consecutive lines (strided columns).
// The twiddle table tw (length N) holds e^{dir 2 pi i t/N}.  Ends with
// __syncthreads().
template <typename C, int N, int NL, bool ELEM_FAST, class Load, class Store>
__device__ __forceinline__ void fft_lines(C* __restrict__ A, C* __restrict__ B, const C* __restrict__ tw, int dir,
                                          const Load& load, const Store& store) {
  constexpr int S = ct_num_stages(N);
  static_assert(S >= 1, "unsupported length");
  if constexpr (S == 1) {
    constexpr int R = N;
    for (int w = threadIdx.x; w < NL; w += blockDim.x) {
      C a[8];
#pragma unroll
      for (int t = 0; t < R; ++t) a[t] = load(t, w);
      reg_dft<R>(a, dir);
#pragma unroll
      for (int u = 0; u < R; ++u) store(u, w, a[u]);
    }
    __syncthreads();
  } else {
    // stage 0: global -> registers -> shared
    constexpr int R0 = ct_stage_radix(N, 0);
    constexpr int M0 = N / R0;
    for (int w = threadIdx.x; w < M0 * NL; w += blockDim.x) {
      const int l = ELEM_FAST ? w / M0 : w % NL;
      const int q = ELEM_FAST ? w % M0 : w / NL;
      C a[8];
#pragma unroll
      for (int t = 0; t < R0; ++t) a[t] = load(q + t * M0, l);
      reg_dft<R0>(a, dir);
#pragma unroll
      for (int u = 0; u < R0; ++u) {
        C v = a[u];
        if (u > 0) v = cmul(v, tw[q * u]);
        A[tile_at<NL>(R0 * q + u, l)] = v;
      }
    }
    __syncthreads();
    // middle stages 1 .. S-2 in shared memory
    ct_stages<C, N, NL, 1, R0, S - 1>(A, B, tw, dir);
    C* src = ((S - 2) & 1) ? B : A;
    // last stage: shared -> registers -> store (q = 0, no twiddles)
    constexpr int RL = ct_stage_radix(N, S - 1);
    constexpr int SL = ct_stride_before(N, S - 1);  // = N / RL
    for (int w = threadIdx.x; w < SL * NL; w += blockDim.x) {
      const int l = ELEM_FAST ? w / SL : w % NL;
      const int k = ELEM_FAST ? w % SL : w / NL;
      C a[8];
#pragma unroll
      for (int t = 0; t < RL; ++t) a[t] = src[tile_at<NL>(k + SL * t, l)];
      reg_dft<RL>(a, dir);
#pragma unroll
      for (int u = 0; u < RL; ++u) store(k + SL * u, l, a[u]);
    }
    __syncthreads();
  }
}


}  // namespace mpdpft
