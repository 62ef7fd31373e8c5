// noalloc.cu -- a trapezoid integral that allocates no device memory.
//
// mpdpft_integrate needs a context, and a context allocates its fields and
// its reduction scratch with cudaMalloc.  Some callers cannot do that: a
// plug-in whose host application owns all device memory through its own
// pool, or a latency-critical loop that must not hit cudaMalloc's implicit
// device synchronisation.  mpdpft_integrate_noalloc serves them: the caller
// passes the field and the result slot (both device memory), and the per-tile
// partial sums live in the file-scope array below, which every GPU that loads
// this library holds until the process exits.
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "../../include/mpdpft_gpu.h"
#include "common.cuh"

namespace mpdpft {

int set_error(int status, const std::string& msg);

// One block sums one tile of kTile consecutive grid points; the tile count
// (and so the summation order) depends only on the grid, never on the GPU.
constexpr int kNoAllocThreads = 256;
constexpr int kNoAllocTile = kNoAllocThreads * 16;  // 4096 points per tile
constexpr int kNoAllocMaxTiles = MPDPFT_NOALLOC_MAX_POINTS / kNoAllocTile;
static_assert(MPDPFT_NOALLOC_MAX_POINTS % kNoAllocTile == 0, "whole tiles");

// The scratch: one partial sum per tile (32 KiB).  Every call writes the
// partials it later reads, so nothing has to be cleared between calls.
static __device__ __align__(256) double g_noalloc_partials[kNoAllocMaxTiles];

// Periodic point p -> its index in the caller's layout.
__device__ __forceinline__ long noalloc_index(long p, int dim, int s, int layout) {
  if (layout != MPDPFT_LAYOUT_REFERENCE) return p;
  const long el = s + 1;
  const int k = (int)(p % s);
  const long t = p / s;
  if (dim == 3) return ((t / s) * el + (t % s)) * el + k;
  return t * el + k;
}

__global__ void __launch_bounds__(kNoAllocThreads) k_noalloc_tiles(const double* __restrict__ f, long n, int dim,
                                                                    int s, int layout, double* partials) {
  __shared__ double sh[kNoAllocThreads];
  const long base = (long)blockIdx.x * kNoAllocTile;
  double t = 0.0;
  for (int i = threadIdx.x; i < kNoAllocTile; i += kNoAllocThreads) {
    const long p = base + i;
    if (p < n) t += f[noalloc_index(p, dim, s, layout)];
  }
  sh[threadIdx.x] = t;
  __syncthreads();
  for (int w = kNoAllocThreads / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) partials[blockIdx.x] = sh[0];
}

__global__ void __launch_bounds__(kNoAllocThreads) k_noalloc_finish(const double* partials, int ntiles, double dvol,
                                                                     double* out) {
  __shared__ double sh[kNoAllocThreads];
  double t = 0.0;
  for (int i = threadIdx.x; i < ntiles; i += kNoAllocThreads) t += partials[i];
  sh[threadIdx.x] = t;
  __syncthreads();
  for (int w = kNoAllocThreads / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) *out = sh[0] * dvol;
}

// Device address of the scratch, looked up once per device (the symbol's
// name in host code is only a stand-in, not a device pointer).
namespace {
constexpr int kNoAllocMaxDevices = 64;
std::mutex g_noalloc_mutex;
double* g_noalloc_ptr[kNoAllocMaxDevices] = {};

int noalloc_scratch(int dev, double** out) {
  if (dev < 0 || dev >= kNoAllocMaxDevices) return set_error(MPDPFT_ERR_ARG, "device ordinal out of range");
  std::lock_guard<std::mutex> lock(g_noalloc_mutex);
  if (!g_noalloc_ptr[dev]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_partials);
    if (e != cudaSuccess)
      return set_error(MPDPFT_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
    g_noalloc_ptr[dev] = static_cast<double*>(p);
  }
  *out = g_noalloc_ptr[dev];
  return MPDPFT_OK;
}
}  // namespace

}  // namespace mpdpft

extern "C" int mpdpft_integrate_noalloc(int dim, int steps, double edge, const double* f, double* out, int layout,
                                        void* stream) {
  using namespace mpdpft;
  if (dim != 2 && dim != 3) return set_error(MPDPFT_ERR_ARG, "dim must be 2 or 3");
  if (steps < 1) return set_error(MPDPFT_ERR_ARG, "steps must be positive");
  if (!(edge > 0.0)) return set_error(MPDPFT_ERR_ARG, "edge must be positive");
  if (layout != MPDPFT_LAYOUT_PERIODIC && layout != MPDPFT_LAYOUT_REFERENCE)
    return set_error(MPDPFT_ERR_ARG, "bad layout");
  if (!f || !out) return set_error(MPDPFT_ERR_ARG, "null field or result pointer");
  // 2^24 points: s <= 256 in 3D, s <= 4096 in 2D
  if ((dim == 3 && steps > 256) || (dim == 2 && steps > 4096))
    return set_error(MPDPFT_ERR_ARG, "grid larger than MPDPFT_NOALLOC_MAX_POINTS (16777216 points, 256^3): "
                                     "use mpdpft_integrate with a context");
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return set_error(MPDPFT_ERR_NO_DEVICE, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
  const long n = dim == 3 ? (long)steps * steps * steps : (long)steps * steps;
  double* scratch = nullptr;
  int st = noalloc_scratch(dev, &scratch);
  if (st) return st;
  const int ntiles = (int)((n + kNoAllocTile - 1) / kNoAllocTile);
  const double dx = edge / steps;
  const double dvol = dim == 3 ? dx * dx * dx : dx * dx;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  k_noalloc_tiles<<<ntiles, kNoAllocThreads, 0, s>>>(f, n, dim, steps, layout, scratch);
  k_noalloc_finish<<<1, kNoAllocThreads, 0, s>>>(scratch, ntiles, dvol, out);
  e = cudaGetLastError();
  if (e != cudaSuccess) return set_error(MPDPFT_ERR_CUDA, std::string("integrate_noalloc launch: ") + cudaGetErrorString(e));
  return MPDPFT_OK;
}
