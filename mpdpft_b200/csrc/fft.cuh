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

}  // namespace mpdpft
