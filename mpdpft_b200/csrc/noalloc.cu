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
#include <cuda.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>

#include <mutex>
#include <string>

#include "../../include/mpdpft_gpu.h"
#include "common.cuh"

namespace mpdpft {

int set_error(int status, const std::string& msg);

// One block sums one tile of kTile consecutive stored points; the tile count
// (and so the summation order) depends only on the grid, never on the GPU.
constexpr int kNoAllocThreads = 256;
constexpr int kNoAllocTile = kNoAllocThreads * 16;  // 4096 points per tile
// The largest accepted grids are s = 256 in 3D and s = 4096 in 2D; in the
// reference layout they store (s+1)^D points, 257^3 = 16974593 at most.
constexpr long kNoAllocMaxStored = 257L * 257L * 257L;
constexpr int kNoAllocMaxTiles = (int)((kNoAllocMaxStored + kNoAllocTile - 1) / kNoAllocTile);  // 4145
static_assert(4097L * 4097L <= kNoAllocMaxStored, "2D reference grids fit the scratch");

// The scratch: one partial sum per tile (33160 bytes).  Every call writes the
// partials it later reads, so nothing has to be cleared between calls.
static __device__ __align__(256) double g_noalloc_partials[kNoAllocMaxTiles];

// Sum of tile blockIdx.x: periodic layout, every point weight 1; reference
// layout, the trapezoid end weights 1/2 per axis (Riemann,
// mpDPFT.cpp:7981-8026), so the duplicate planes count as stored.
__global__ void __launch_bounds__(kNoAllocThreads) k_noalloc_tiles(const double* __restrict__ f, unsigned total,
                                                                    int dim, unsigned el, int layout,
                                                                    double* partials) {
  __shared__ double sh[kNoAllocThreads];
  const unsigned base = blockIdx.x * (unsigned)kNoAllocTile;
  double t = 0.0;
  for (int i = threadIdx.x; i < kNoAllocTile; i += kNoAllocThreads) {
    const unsigned q = base + i;
    if (q < total) t += (layout == MPDPFT_LAYOUT_REFERENCE ? riemann_weight(q, el, dim) : 1.0) * f[q];
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

// Device address of the scratch.  The symbol's name in host code is only a
// stand-in, and its device address belongs to a CUDA context, not to a
// device ordinal: a caller may make its own driver context current, and a
// device reset replaces the primary context.  So the address is looked up
// once per context, keyed by the context's process-unique id (cuCtxGetId,
// reached through the runtime's driver entry points so that the library
// does not link the driver).
namespace {
constexpr int kNoAllocCache = 32;
std::mutex g_noalloc_mutex;
struct NoAllocEntry {
  unsigned long long ctx_id;
  double* ptr;
};
NoAllocEntry g_noalloc_cache[kNoAllocCache] = {};
int g_noalloc_next = 0;
PFN_cuCtxGetCurrent_v4000 g_ctx_get_current = nullptr;
PFN_cuCtxGetId_v12000 g_ctx_get_id = nullptr;

int current_context_id(unsigned long long* id, bool* have) {
  *have = false;
  if (!g_ctx_get_current || !g_ctx_get_id) {
    void* f1 = nullptr;
    void* f2 = nullptr;
    cudaDriverEntryPointQueryResult q1, q2;
    cudaError_t e1 = cudaGetDriverEntryPoint("cuCtxGetCurrent", &f1, cudaEnableDefault, &q1);
    cudaError_t e2 = cudaGetDriverEntryPoint("cuCtxGetId", &f2, cudaEnableDefault, &q2);
    if (e1 != cudaSuccess || e2 != cudaSuccess || q1 != cudaDriverEntryPointSuccess ||
        q2 != cudaDriverEntryPointSuccess || !f1 || !f2)
      return set_error(MPDPFT_ERR_CUDA, "cuCtxGetCurrent/cuCtxGetId not available from the driver");
    g_ctx_get_current = reinterpret_cast<PFN_cuCtxGetCurrent_v4000>(f1);
    g_ctx_get_id = reinterpret_cast<PFN_cuCtxGetId_v12000>(f2);
  }
  CUcontext ctx = nullptr;
  if (g_ctx_get_current(&ctx) != CUDA_SUCCESS)
    return set_error(MPDPFT_ERR_CUDA, "cuCtxGetCurrent failed");
  if (!ctx) return MPDPFT_OK;  // no context yet: the runtime creates one below
  if (g_ctx_get_id(ctx, id) != CUDA_SUCCESS) return set_error(MPDPFT_ERR_CUDA, "cuCtxGetId failed");
  *have = true;
  return MPDPFT_OK;
}

int noalloc_scratch(double** out) {
  std::lock_guard<std::mutex> lock(g_noalloc_mutex);
  unsigned long long id = 0;
  bool have = false;
  int st = current_context_id(&id, &have);
  if (st) return st;
  if (have)
    for (const NoAllocEntry& e : g_noalloc_cache)
      if (e.ptr && e.ctx_id == id) {
        *out = e.ptr;
        return MPDPFT_OK;
      }
  // first call in this context: cudaGetSymbolAddress also initialises the
  // runtime's context when none is current yet
  void* p = nullptr;
  cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_partials);
  if (e != cudaSuccess)
    return set_error(MPDPFT_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
  if (!have) {
    if ((st = current_context_id(&id, &have))) return st;
    if (!have) return set_error(MPDPFT_ERR_CUDA, "no current CUDA context after cudaGetSymbolAddress");
  }
  g_noalloc_cache[g_noalloc_next] = NoAllocEntry{id, static_cast<double*>(p)};
  g_noalloc_next = (g_noalloc_next + 1) % kNoAllocCache;
  *out = static_cast<double*>(p);
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
  // 2^24 periodic points: s <= 256 in 3D, s <= 4096 in 2D
  if ((dim == 3 && steps > 256) || (dim == 2 && steps > 4096))
    return set_error(MPDPFT_ERR_ARG, "grid larger than MPDPFT_NOALLOC_MAX_POINTS (16777216 points, 256^3): "
                                     "use mpdpft_integrate with a context");
  const unsigned el = layout == MPDPFT_LAYOUT_REFERENCE ? (unsigned)steps + 1 : (unsigned)steps;
  const unsigned total = dim == 3 ? el * el * el : el * el;
  double* scratch = nullptr;
  int st = noalloc_scratch(&scratch);
  if (st) return st;
  const int ntiles = (int)((total + kNoAllocTile - 1) / kNoAllocTile);
  const double dx = edge / steps;
  const double dvol = dim == 3 ? dx * dx * dx : dx * dx;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  // each launch's own return code: an error the caller left pending is
  // neither reported as ours nor cleared
  {
    void* args[] = {(void*)&f, (void*)&total, (void*)&dim, (void*)&el, (void*)&layout, (void*)&scratch};
    cudaError_t e = cudaLaunchKernel((const void*)k_noalloc_tiles, dim3(ntiles), dim3(kNoAllocThreads), args, 0, s);
    if (e != cudaSuccess) {
      cudaGetLastError();
      return set_error(MPDPFT_ERR_CUDA, std::string("k_noalloc_tiles launch: ") + cudaGetErrorString(e));
    }
  }
  {
    const double* cp = scratch;
    void* args[] = {(void*)&cp, (void*)&ntiles, (void*)&dvol, (void*)&out};
    cudaError_t e = cudaLaunchKernel((const void*)k_noalloc_finish, dim3(1), dim3(kNoAllocThreads), args, 0, s);
    if (e != cudaSuccess) {
      cudaGetLastError();
      return set_error(MPDPFT_ERR_CUDA, std::string("k_noalloc_finish launch: ") + cudaGetErrorString(e));
    }
  }
  return MPDPFT_OK;
}
