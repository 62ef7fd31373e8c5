// batch.cu -- many independent SC solves advanced together on one GPU.
//
// Each solve keeps its own context (buffers, FFT plans, SC state); the
// batch adds device tables that let one launch of each SC kernel serve every
// solve, and captures one iteration of all of them as a CUDA graph:
//   memset of the taper-shift slots
//   V assembly of every solve                          (one launch)
//   DelField of every species, one branch per grid size (six launches each,
//     the branches run concurrently)
//   mu search: a persistent kernel whose blocks claim gangs of blocks of one
//     solve from a queue, largest solves first        (one launch)
//   densities, residuals, Gram rows and the per-solve Pulay solve (the last
//     block of each solve)                              (one launch)
//   mixing                                              (one launch)
// A solve that has met its exit test skips all of it.  The mu search of one
// solve needs its gang's blocks to wait for one another; gangs are claimed
// in queue order by the co-resident blocks of a cooperative launch and no
// gang is larger than the grid, so every gang that has a member waiting is
// completed by blocks that are running.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "batch.h"
#include "sc_kernel.cuh"

namespace mpdpft {

#define CU(call)                                                                             \
  do {                                                                                       \
    cudaError_t e_ = (call);                                                                 \
    if (e_ != cudaSuccess)                                                                   \
      return set_error(MPDPFT_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

// Gang queue of the batched mu search: claim c of nclaims is block tab[c].y
// of the tab[c].z blocks of solve tab[c].x.
template <typename R, int FK>
__global__ void __launch_bounds__(kStepThreads, 1) sc_mu_gangs(const StepArgs<R>* __restrict__ args,
                                                              const int4* __restrict__ tab, int nclaims,
                                                              unsigned* queue) {
  __shared__ int s_claim;
  for (;;) {
    __syncthreads();  // the previous gang's use of shared memory is over
    if (threadIdx.x == 0) s_claim = (int)atomicAdd(queue, 1u);
    __syncthreads();
    const int c = s_claim;
    if (c >= nclaims) return;
    const int4 t = tab[c];
    sc_mu_body<R, FK>(args[t.x], t.y, t.z);
  }
}

// Minimum and maximum of field b (of counts[b] points) into out[2b], out[2b+1].
template <typename R>
__global__ void k_minmax_b(const R* const* fields, const long* counts, double* out) {
  const R* f = fields[blockIdx.x];
  const long n = counts[blockIdx.x];
  double lo = 1.0e300, hi = -1.0e300;
  for (long p = threadIdx.x; p < n; p += blockDim.x) {
    const double v = (double)__ldcg(f + p);
    lo = fmin(lo, v);
    hi = fmax(hi, v);
  }
  for (int o = 16; o > 0; o >>= 1) {
    lo = fmin(lo, __shfl_xor_sync(0xffffffffu, lo, o));
    hi = fmax(hi, __shfl_xor_sync(0xffffffffu, hi, o));
  }
  __shared__ double sl[32], sh[32];
  if ((threadIdx.x & 31) == 0) { sl[threadIdx.x >> 5] = lo; sh[threadIdx.x >> 5] = hi; }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < (int)(blockDim.x >> 5); ++w) { lo = fmin(lo, sl[w]); hi = fmax(hi, sh[w]); }
    out[2 * blockIdx.x] = fmin(lo, sl[0]);
    out[2 * blockIdx.x + 1] = fmax(hi, sh[0]);
  }
}

// Solves that have not met their exit test.
__global__ void k_count_active(ScState* const* states, int count, int* out) {
  __shared__ int sh;
  if (threadIdx.x == 0) sh = 0;
  __syncthreads();
  int c = 0;
  for (int i = threadIdx.x; i < count; i += blockDim.x) c += __ldcg(&states[i]->exit_loop) ? 0 : 1;
  atomicAdd(&sh, c);
  __syncthreads();
  if (threadIdx.x == 0) *out = sh;
}

struct Batch {
  std::vector<Ctx*> members;
  int count = 0, S = 1, device = 0, fk = 0, dens_which = 1, num_sms = 148;
  size_t rsize = 8;
  cudaStream_t stream = nullptr;
  std::vector<cudaStream_t> side;  // one per grid size
  std::vector<cudaEvent_t> events;
  unsigned long long* d_vmax = nullptr;  // [count][kMaxS]
  std::vector<BatchFftClass*> classes;
  BatchAssemble* assemble = nullptr;
  void* d_args[2] = {nullptr, nullptr};  // StepArgs<R>[count], modes 0 and 1
  int4* d_tab_mu = nullptr;
  int n_mu = 0, mu_grid = 0;
  unsigned* d_queue = nullptr;
  int4* d_tab_dens = nullptr;
  int n_dens = 0;
  int4* d_tab_mix = nullptr;
  int n_mix = 0;
  ScState** d_states = nullptr;
  int* d_active = nullptr;
  int* h_active = nullptr;  // pinned
  double* d_energy = nullptr;  // [count][kNEnergy]
  void** d_vfields = nullptr;  // [count * S] potential of each species (automatic temperature)
  long* d_vcounts = nullptr;
  double* d_minmax = nullptr;  // [count * S][2]
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  bool initialised = false;
  std::vector<int> asm_blocks;

  ~Batch() { release(); }
  void release();
  int init(const mpdpft_params* params, int n, int dev);
  int build_tables();
  template <typename R>
  int upload_args();
  int issue_sc(int mode);
  int issue_iteration();
  int sc_init(const double* const* v0, int layout, int mem);
  int step(int iterations);
  int run(mpdpft_result* results, int* status);
};

void Batch::release() {
  if (exec) { cudaGraphExecDestroy(exec); exec = nullptr; }
  if (graph) { cudaGraphDestroy(graph); graph = nullptr; }
  for (BatchFftClass* b : classes) batch_fft_destroy(b);
  classes.clear();
  batch_assemble_destroy(assemble);
  assemble = nullptr;
  for (Ctx* c : members) {
    c->stream = nullptr;  // the batch's stream
    delete c;
  }
  members.clear();
  void* bufs[] = {d_vmax, d_args[0], d_args[1], d_tab_mu, d_queue, d_tab_dens, d_tab_mix, d_states,
                  d_active, d_energy, d_vfields, d_vcounts, d_minmax};
  for (void* p : bufs) if (p) cudaFree(p);
  d_vmax = nullptr; d_args[0] = d_args[1] = nullptr; d_tab_mu = nullptr; d_queue = nullptr;
  d_tab_dens = nullptr; d_tab_mix = nullptr; d_states = nullptr; d_active = nullptr; d_energy = nullptr;
  d_vfields = nullptr; d_vcounts = nullptr; d_minmax = nullptr;
  if (h_active) { cudaFreeHost(h_active); h_active = nullptr; }
  for (cudaEvent_t e : events) cudaEventDestroy(e);
  events.clear();
  for (cudaStream_t s : side) cudaStreamDestroy(s);
  side.clear();
  if (stream) { cudaStreamDestroy(stream); stream = nullptr; }
}

template <typename R, int FK>
static const void* density_b_ptr(int which) {
  if (which == 1) return (const void*)sc_density_kernel_b<R, FK, 5>;
  if (which == 3) return (const void*)sc_density_kernel_b<R, FK, 8>;
  return (const void*)sc_density_kernel_b<R, FK, kMaxP>;
}

template <typename R>
static const void* batch_kernel(int which, int fk) {
  // which: 0 mu gangs, 1/2/3 density (Pulay window variant), 4 mixing;
  // batches are 2D gradient-corrected: functional kind 3
  if (which == 4) return (const void*)sc_mix_kernel_b<R>;
  if (fk != 3) return nullptr;
  if (which == 0) return (const void*)sc_mu_gangs<R, 3>;
  return density_b_ptr<R, 3>(which);
}

int Batch::init(const mpdpft_params* params, int n, int dev) {
  if (!params || n < 1) return set_error(MPDPFT_ERR_ARG, "batch: no parameter sets");
  count = n;
  device = dev;
  const mpdpft_params& p0 = params[0];
  for (int i = 0; i < n; ++i) {
    const mpdpft_params& p = params[i];
    if (p.dim != 2 || p.species != p0.species || p.precision != p0.precision ||
        p.density_expression != MPDPFT_DENS_GRADIENT || p.mixer != p0.mixer ||
        (p.mixer && p.pulay_scope != p0.pulay_scope) || p.n_interactions != p0.n_interactions)
      return set_error(MPDPFT_ERR_ARG, "batch: solves must share dim 2, species, precision, density "
                                       "functional 5, mixer and interactions");
    for (int a = 0; a < p.n_interactions; ++a) {
      const int t = p.interactions[a];
      if (t != p0.interactions[a] || (t != MPDPFT_INT_CONTACT_MUTUAL && t != MPDPFT_INT_CONTACT_SELF &&
                                      t != MPDPFT_INT_DIRAC && t != MPDPFT_INT_HARTREE &&
                                      t != MPDPFT_INT_HARTREE_INTER && t != MPDPFT_INT_COULOMB_CHARGED))
        return set_error(MPDPFT_ERR_ARG, "batch: interaction types 1, 8, 10, 11, 21 and 100 only");
    }
  }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return set_error(MPDPFT_ERR_NO_DEVICE, "no CUDA device");
  CU(cudaSetDevice(dev));
  CU(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
  for (int i = 0; i < n; ++i) {
    Ctx* c = new Ctx;
    members.push_back(c);
    int st = c->init(params[i], dev);
    if (st) return st;
    cudaStreamDestroy(c->stream);  // every member works on the batch's stream
    c->stream = stream;
    if ((st = c->fft_setup())) return st;
    c->assemble_in_step = 0;
  }
  S = p0.species;
  rsize = members[0]->rsize;
  fk = members[0]->fk;
  dens_which = members[0]->dens_which;
  num_sms = members[0]->num_sms;
  if (fk != 3) return set_error(MPDPFT_ERR_ARG, "batch: unsupported functional kind");
  CU(cudaMalloc((void**)&d_vmax, sizeof(unsigned long long) * kMaxS * count));
  // grid-size classes
  std::vector<int> sizes;
  for (Ctx* c : members) sizes.push_back(c->P.steps);
  std::sort(sizes.begin(), sizes.end());
  sizes.erase(std::unique(sizes.begin(), sizes.end()), sizes.end());
  for (int s : sizes) {
    std::vector<BatchMember> cls;
    for (int i = 0; i < count; ++i)
      if (members[i]->P.steps == s) cls.push_back({members[i], i});
    BatchFftClass* b = nullptr;
    int st = batch_fft_create(cls, d_vmax, &b);
    if (st) return st;
    classes.push_back(b);
    cudaStream_t ss;
    CU(cudaStreamCreateWithFlags(&ss, cudaStreamNonBlocking));
    side.push_back(ss);
  }
  for (size_t i = 0; i < 2 * classes.size() + 1; ++i) {
    cudaEvent_t e;
    CU(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    events.push_back(e);
  }
  {
    std::vector<BatchMember> all;
    for (int i = 0; i < count; ++i) all.push_back({members[i], i});
    int st = batch_assemble_create(all, d_vmax, &assemble, &asm_blocks);
    if (st) return st;
  }
  std::vector<ScState*> states;
  for (Ctx* c : members) states.push_back(c->d_state);
  CU(cudaMalloc((void**)&d_states, sizeof(ScState*) * count));
  CU(cudaMemcpy(d_states, states.data(), sizeof(ScState*) * count, cudaMemcpyHostToDevice));
  CU(cudaMalloc((void**)&d_active, sizeof(int)));
  CU(cudaMallocHost((void**)&h_active, sizeof(int)));
  CU(cudaMalloc((void**)&d_energy, sizeof(double) * kNEnergy * count));
  {
    std::vector<void*> f;
    std::vector<long> nn;
    for (Ctx* c : members)
      for (int s = 0; s < S; ++s) {
        f.push_back((char*)c->d_V + (size_t)s * c->geom.n * rsize);
        nn.push_back(c->geom.n);
      }
    CU(cudaMalloc((void**)&d_vfields, sizeof(void*) * f.size()));
    CU(cudaMemcpy(d_vfields, f.data(), sizeof(void*) * f.size(), cudaMemcpyHostToDevice));
    CU(cudaMalloc((void**)&d_vcounts, sizeof(long) * nn.size()));
    CU(cudaMemcpy(d_vcounts, nn.data(), sizeof(long) * nn.size(), cudaMemcpyHostToDevice));
    CU(cudaMalloc((void**)&d_minmax, sizeof(double) * 2 * f.size()));
  }
  CU(cudaMalloc((void**)&d_queue, sizeof(unsigned)));
  return build_tables();
}

// Block tables of the SC kernels.  Gangs of the mu search get one block per
// 16384 points (8192 per species of a two-species solve), the density
// kernel one per 1024 points, the mixing kernel one per 2048; gangs are
// queued largest first.
int Batch::build_tables() {
  const bool f64 = rsize == sizeof(double);
  int occ = 0;
  const void* mu_fn = f64 ? batch_kernel<double>(0, fk) : batch_kernel<float>(0, fk);
  CU(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, mu_fn, kStepThreads, 0));
  if (occ < 1) return set_error(MPDPFT_ERR_CUDA, "batch: mu kernel cannot be resident");
  mu_grid = num_sms * occ;
  std::vector<int> order(count);
  for (int i = 0; i < count; ++i) order[i] = i;
  std::stable_sort(order.begin(), order.end(),
                   [&](int a, int b) { return members[a]->geom.n > members[b]->geom.n; });
  std::vector<int4> mu, dens, mix;
  for (int i : order) {
    Ctx& c = *members[i];
    const long pts = c.geom.n * (long)S;
    int g = (int)std::min<long>((pts + 16383) / 16384, std::min(c.step_blocks, mu_grid));
    g = std::max(g, 1);
    // the member's kernels see a gang of g blocks
    c.step_blocks = g;
    const long warps = (long)g * kStepWarps;
    c.chunk = (c.geom.n + warps - 1) / warps;
    c.chunk = (c.chunk + kSegPts - 1) / kSegPts * kSegPts;
    for (int b = 0; b < g; ++b) mu.push_back(make_int4(i, b, g, 0));
  }
  for (int i = 0; i < count; ++i) {
    Ctx& c = *members[i];
    int d = (int)std::min<long>((c.geom.n + 1023) / 1024, c.dens_blocks);
    d = std::max(d, 1);
    c.dens_blocks = d;
    for (int b = 0; b < d; ++b) dens.push_back(make_int4(i, b, d, 0));
    int m = (int)std::min<long>((c.geom.n + 2047) / 2048, c.mix_blocks);
    m = std::max(m, 1);
    c.mix_blocks = m;
    for (int b = 0; b < m; ++b) mix.push_back(make_int4(i, b, m, 0));
  }
  n_mu = (int)mu.size();
  n_dens = (int)dens.size();
  n_mix = (int)mix.size();
  CU(cudaMalloc((void**)&d_tab_mu, sizeof(int4) * n_mu));
  CU(cudaMemcpy(d_tab_mu, mu.data(), sizeof(int4) * n_mu, cudaMemcpyHostToDevice));
  CU(cudaMalloc((void**)&d_tab_dens, sizeof(int4) * n_dens));
  CU(cudaMemcpy(d_tab_dens, dens.data(), sizeof(int4) * n_dens, cudaMemcpyHostToDevice));
  CU(cudaMalloc((void**)&d_tab_mix, sizeof(int4) * n_mix));
  CU(cudaMemcpy(d_tab_mix, mix.data(), sizeof(int4) * n_mix, cudaMemcpyHostToDevice));
  const size_t asz = f64 ? sizeof(StepArgs<double>) : sizeof(StepArgs<float>);
  CU(cudaMalloc(&d_args[0], asz * count));
  CU(cudaMalloc(&d_args[1], asz * count));
  return MPDPFT_OK;
}

// Step arguments of every member (after the temperatures are known).
template <typename R>
int Batch::upload_args() {
  for (int mode = 0; mode < 2; ++mode) {
    std::vector<StepArgs<R>> a(count);
    for (int i = 0; i < count; ++i) {
      Ctx& c = *members[i];
      c.vres_part_ext = batch_vres_part(c);
      c.vres_blocks_ext = asm_blocks[i];
      a[i] = c.step_args<R>(mode);
      a[i].split_d = 0;  // the last block of each solve runs its phase D
    }
    CU(cudaMemcpyAsync(d_args[mode], a.data(), sizeof(StepArgs<R>) * count, cudaMemcpyHostToDevice, stream));
    CU(cudaStreamSynchronize(stream));
  }
  return MPDPFT_OK;
}

// The SC kernels of every member: mu search + densities (mode 1), or mu
// search + densities + mixing (mode 0).
int Batch::issue_sc(int mode) {
  const bool f64 = rsize == sizeof(double);
  void* args = d_args[mode];
  CU(cudaMemsetAsync(d_queue, 0, sizeof(unsigned), stream));
  {
    void* params[] = {&args, &d_tab_mu, &n_mu, &d_queue};
    cudaLaunchConfig_t cfg;
    std::memset(&cfg, 0, sizeof(cfg));
    cfg.gridDim = dim3(mu_grid);
    cfg.blockDim = dim3(kStepThreads);
    cfg.stream = stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    CU(cudaLaunchKernelExC(&cfg, f64 ? batch_kernel<double>(0, fk) : batch_kernel<float>(0, fk), params));
  }
  {
    void* params[] = {&args, &d_tab_dens};
    const void* fn = f64 ? batch_kernel<double>(dens_which, fk) : batch_kernel<float>(dens_which, fk);
    CU(cudaLaunchKernel(fn, dim3(n_dens), dim3(kDensityThreads), params, 0, stream));
  }
  if (mode == 0) {
    void* params[] = {&args, &d_tab_mix};
    const void* fn = f64 ? batch_kernel<double>(4, fk) : batch_kernel<float>(4, fk);
    CU(cudaLaunchKernel(fn, dim3(n_mix), dim3(kDensThreads), params, 0, stream));
  }
  return MPDPFT_OK;
}

int Batch::issue_iteration() {
  int st;
  CU(cudaMemsetAsync(d_vmax, 0, sizeof(unsigned long long) * kMaxS * count, stream));
  // Coulomb terms of the current densities, every grid size on its own stream
  if (!classes.empty() && batch_fft_has_coulomb(classes[0])) {
    CU(cudaEventRecord(events[0], stream));
    for (size_t k = 0; k < classes.size(); ++k) {
      CU(cudaStreamWaitEvent(side[k], events[0], 0));
      if ((st = batch_fft_issue_coulomb(classes[k], side[k]))) return st;
      CU(cudaEventRecord(events[1 + k], side[k]));
      CU(cudaStreamWaitEvent(stream, events[1 + k], 0));
    }
  }
  if ((st = batch_assemble_issue(assemble, 1, stream))) return st;
  // DelField of every grid size on its own stream
  CU(cudaEventRecord(events[0], stream));
  for (size_t k = 0; k < classes.size(); ++k) {
    CU(cudaStreamWaitEvent(side[k], events[0], 0));
    if ((st = batch_fft_issue(classes[k], side[k]))) return st;
    CU(cudaEventRecord(events[1 + k], side[k]));
    CU(cudaStreamWaitEvent(stream, events[1 + k], 0));
  }
  return issue_sc(0);
}

int Batch::sc_init(const double* const* v0, int layout, int mem) {
  int st;
  CU(cudaSetDevice(device));
  CU(cudaStreamSynchronize(stream));
  // host arrays: copied into the members' pinned staging halves (one per
  // species) by several host threads, then sent by one stream
  const bool staged = v0 && mem == MPDPFT_MEM_HOST && S <= 2;
  if (staged) {
    const int nt = (int)std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
    std::vector<std::thread> pool;
    for (int t = 0; t < nt; ++t)
      pool.emplace_back([&, t]() {
        for (int i = t; i < count; i += nt) {
          Ctx& c = *members[i];
          const long cnt = layout == MPDPFT_LAYOUT_REFERENCE ? c.n_ref : c.geom.n;
          for (int s = 0; s < S; ++s)
            if (v0[(size_t)i * S + s]) copy_to_pinned(c.host_stage(s), v0[(size_t)i * S + s], cnt);
        }
      });
    for (std::thread& th : pool) th.join();
  }
  for (int i = 0; i < count; ++i) {
    Ctx& c = *members[i];
    if ((st = c.reset_state(false))) return st;
    for (int s = 0; s < S; ++s) {
      void* dst = (char*)c.d_V + (size_t)s * c.geom.n * rsize;
      const double* src = v0 ? v0[(size_t)i * S + s] : nullptr;
      if (src && staged) {
        if ((st = c.import_staged(nullptr, dst, layout, s, false))) return st;
      } else if (src) {  // device arrays, or host data staged in half s % 2
        if ((st = c.import_field(src, dst, layout, mem, s & 1, mem == MPDPFT_MEM_HOST && (s & 1)))) return st;
      } else {
        CU(cudaMemcpyAsync(dst, (char*)c.d_vext + (size_t)s * c.geom.n * rsize, c.geom.n * rsize,
                           cudaMemcpyDeviceToDevice, stream));
      }
    }
  }
  // automatic temperature (PreparationsForSCdensity, mpDPFT.cpp:4523-4528)
  // from the extremes of every start potential
  bool need_t = false;
  for (Ctx* c : members)
    for (int s = 0; s < S; ++s) need_t |= c->P.temperature[s] < 0.0;
  std::vector<double> mm(2 * (size_t)count * S);
  if (need_t) {
    if (rsize == sizeof(double))
      k_minmax_b<double><<<count * S, 256, 0, stream>>>((const double* const*)d_vfields, d_vcounts, d_minmax);
    else
      k_minmax_b<float><<<count * S, 256, 0, stream>>>((const float* const*)d_vfields, d_vcounts, d_minmax);
    CU(cudaGetLastError());
    CU(cudaMemcpyAsync(mm.data(), d_minmax, sizeof(double) * mm.size(), cudaMemcpyDeviceToHost, stream));
  }
  CU(cudaStreamSynchronize(stream));
  for (int i = 0; i < count; ++i) {
    Ctx& c = *members[i];
    for (int s = 0; s < S; ++s) {
      if (c.P.temperature[s] >= 0.0) { c.temperature[s] = c.P.temperature[s]; continue; }
      const double vmin = mm[2 * ((size_t)i * S + s)], vmax = mm[2 * ((size_t)i * S + s) + 1];
      c.temperature[s] = std::max(std::fabs(c.P.mu[s] - vmin), std::fabs(c.P.mu[s] - vmax)) / 50.0;
    }
  }
  if ((st = (rsize == sizeof(double) ? upload_args<double>() : upload_args<float>()))) return st;
  // DelField of the start potentials, then the initial densities (mpDPFT.cpp:195)
  CU(cudaMemsetAsync(d_vmax, 0, sizeof(unsigned long long) * kMaxS * count, stream));
  if ((st = batch_assemble_issue(assemble, 0, stream))) return st;
  for (BatchFftClass* b : classes)
    if ((st = batch_fft_issue(b, stream))) return st;
  if ((st = issue_sc(1))) return st;
  CU(cudaStreamSynchronize(stream));
  for (Ctx* c : members) c->initialised = true;
  initialised = true;
  return MPDPFT_OK;
}

int Batch::step(int iterations) {
  if (!initialised) return set_error(MPDPFT_ERR_ARG, "batch: sc_init has not been called");
  int st;
  if (!exec) {
    CU(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
    st = issue_iteration();
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamEndCapture(stream, &g);
    if (st) { if (g) cudaGraphDestroy(g); return st; }
    if (e != cudaSuccess) return set_error(MPDPFT_ERR_CUDA, std::string("batch graph capture: ") + cudaGetErrorString(e));
    graph = g;
    CU(cudaGraphInstantiate(&exec, graph, 0));
  }
  for (int k = 0; k < iterations; ++k) CU(cudaGraphLaunch(exec, stream));
  return MPDPFT_OK;
}

int Batch::run(mpdpft_result* results, int* status) {
  int st;
  int max_sc = 0;
  for (Ctx* c : members) max_sc = std::max(max_sc, c->P.max_sc_count);
  auto t0 = std::chrono::steady_clock::now();
  int issued = 0;
  const int chunk = 4;
  for (;;) {
    if ((st = step(chunk))) return st;
    issued += chunk;
    k_count_active<<<1, 256, 0, stream>>>(d_states, count, d_active);
    CU(cudaGetLastError());
    CU(cudaMemcpyAsync(h_active, d_active, sizeof(int), cudaMemcpyDeviceToHost, stream));
    CU(cudaStreamSynchronize(stream));
    if (*h_active == 0 || issued > max_sc + 2) break;
  }
  // states, energies and results of every member
  std::vector<ScState> h(count);
  for (int i = 0; i < count; ++i)
    CU(cudaMemcpyAsync(&h[i], members[i]->d_state, sizeof(ScState), cudaMemcpyDeviceToHost, stream));
  CU(cudaStreamSynchronize(stream));
  for (int i = 0; i < count; ++i)
    if ((st = members[i]->energy_issue(h[i], d_energy + (size_t)i * kNEnergy, /*g2_current=*/true))) return st;
  std::vector<double> E((size_t)count * kNEnergy);
  CU(cudaMemcpyAsync(E.data(), d_energy, sizeof(double) * E.size(), cudaMemcpyDeviceToHost, stream));
  CU(cudaStreamSynchronize(stream));
  const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  int worst = MPDPFT_OK;
  for (int i = 0; i < count; ++i) {
    Ctx& c = *members[i];
    const ScState& s = h[i];
    int code = MPDPFT_OK;
    if (s.abort) code = MPDPFT_ERR_TIMEOUT;
    else if (s.status_bits & kBitTimeout) code = MPDPFT_ERR_TIMEOUT;
    else if (!s.exit_loop || s.exit_count < 3) code = MPDPFT_ERR_NOT_CONVERGED;
    if (status) status[i] = code;
    if (code && !worst) worst = code;
    if (results) {
      mpdpft_result& r = results[i];
      std::memset(&r, 0, sizeof(r));
      r.iterations = s.sc_count;
      r.converged = s.exit_count >= 3 ? 1 : 0;
      r.total_mu_trials = s.mu_passes_total;
      r.cc = s.cc;
      r.v_residual = s.v_res;
      for (int q = 0; q < S; ++q) { r.mu[q] = s.mu[q]; r.abundance[q] = s.ab[q]; }
      c.energy_finish(&r, E.data() + (size_t)i * kNEnergy);
      r.seconds = secs;
    }
  }
  if (worst == MPDPFT_ERR_TIMEOUT) return set_error(worst, "batch: a solve's mu search or barrier timed out");
  if (worst == MPDPFT_ERR_NOT_CONVERGED) return set_error(worst, "batch: a solve reached maxSCcount");
  return MPDPFT_OK;
}

}  // namespace mpdpft

// ------------------------------------------------------------- C ABI ------
using mpdpft::Batch;
using mpdpft::set_error;

struct mpdpft_batch {
  Batch impl;
};

#define CHECK_BATCH(b) \
  if (!(b)) return set_error(MPDPFT_ERR_ARG, "null batch")

extern "C" {

int mpdpft_batch_create(const mpdpft_params* params, int count, int device, mpdpft_batch** out) {
  if (!out) return set_error(MPDPFT_ERR_ARG, "null output handle");
  *out = nullptr;
  mpdpft_batch* b = new (std::nothrow) mpdpft_batch;
  if (!b) return set_error(MPDPFT_ERR_CUDA, "out of host memory");
  int st = b->impl.init(params, count, device);
  if (st) {
    delete b;
    return st;
  }
  *out = b;
  return MPDPFT_OK;
}

int mpdpft_batch_destroy(mpdpft_batch* batch) {
  if (!batch) return MPDPFT_OK;
  cudaSetDevice(batch->impl.device);
  if (batch->impl.stream) cudaStreamSynchronize(batch->impl.stream);
  delete batch;
  return MPDPFT_OK;
}

int mpdpft_batch_set_external_potential(mpdpft_batch* batch, int i, int s, const double* v_ext, int layout, int mem) {
  CHECK_BATCH(batch);
  Batch& b = batch->impl;
  if (i < 0 || i >= b.count) return set_error(MPDPFT_ERR_ARG, "solve index out of range");
  if (s < 0 || s >= b.S) return set_error(MPDPFT_ERR_ARG, "species index out of range");
  cudaSetDevice(b.device);
  mpdpft::Ctx& c = *b.members[i];
  return c.import_field(v_ext, (char*)c.d_vext + (size_t)s * c.geom.n * c.rsize, layout, mem);
}

int mpdpft_batch_sc_init(mpdpft_batch* batch, const double* const* v0, int layout, int mem) {
  CHECK_BATCH(batch);
  return batch->impl.sc_init(v0, layout, mem);
}

int mpdpft_batch_sc_step(mpdpft_batch* batch, int iterations) {
  CHECK_BATCH(batch);
  if (iterations < 0) return set_error(MPDPFT_ERR_ARG, "negative iteration count");
  cudaSetDevice(batch->impl.device);
  return batch->impl.step(iterations);
}

int mpdpft_batch_sc_run(mpdpft_batch* batch, const double* const* v0, int layout, int mem, mpdpft_result* results,
                        int* status) {
  CHECK_BATCH(batch);
  int st = batch->impl.sc_init(v0, layout, mem);
  if (st) return st;
  return batch->impl.run(results, status);
}

int mpdpft_batch_get_field(mpdpft_batch* batch, int i, int which, int s, double* out, int layout, int mem) {
  CHECK_BATCH(batch);
  Batch& b = batch->impl;
  if (i < 0 || i >= b.count) return set_error(MPDPFT_ERR_ARG, "solve index out of range");
  if (s < 0 || s >= b.S) return set_error(MPDPFT_ERR_ARG, "species index out of range");
  cudaSetDevice(b.device);
  mpdpft::Ctx& c = *b.members[i];
  const size_t off = (size_t)s * c.geom.n * c.rsize;
  const void* src = nullptr;
  if (which == MPDPFT_FIELD_DENSITY) {
    mpdpft::ScState h;
    int st = c.read_state(&h);
    if (st) return st;
    src = (char*)c.d_nin + (size_t)h.slot * c.S * c.geom.n * c.rsize + off;
  } else if (which == MPDPFT_FIELD_POTENTIAL) {
    src = (char*)c.d_V + off;
  } else if (which == MPDPFT_FIELD_EXTERNAL) {
    src = (char*)c.d_vext + off;
  } else if (which == MPDPFT_FIELD_GRAD2) {
    src = (char*)c.d_g2 + off;
  } else if (which == MPDPFT_FIELD_LAPLACIAN) {
    src = (char*)c.d_lap + off;
  } else {
    return set_error(MPDPFT_ERR_ARG, "field not available");
  }
  return c.export_field(src, out, layout, mem);
}

int mpdpft_batch_get_log(mpdpft_batch* batch, int i, mpdpft_iter_log* log, int log_cap, int* n_out) {
  CHECK_BATCH(batch);
  Batch& b = batch->impl;
  if (i < 0 || i >= b.count) return set_error(MPDPFT_ERR_ARG, "solve index out of range");
  cudaSetDevice(b.device);
  mpdpft::Ctx& c = *b.members[i];
  mpdpft::ScState h;
  int st = c.read_state(&h);
  if (st) return st;
  const int n = std::max(0, std::min(log_cap, std::min(h.sc_count, c.log_cap)));
  if (n > 0 && log) {
    cudaError_t e = cudaMemcpy(log, c.d_log, sizeof(mpdpft_iter_log) * n, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return set_error(MPDPFT_ERR_CUDA, std::string("log copy: ") + cudaGetErrorString(e));
  }
  if (n_out) *n_out = n;
  return MPDPFT_OK;
}

int mpdpft_batch_sync(mpdpft_batch* batch) {
  CHECK_BATCH(batch);
  cudaSetDevice(batch->impl.device);
  cudaError_t e = cudaStreamSynchronize(batch->impl.stream);
  if (e != cudaSuccess) return set_error(MPDPFT_ERR_CUDA, std::string("batch sync: ") + cudaGetErrorString(e));
  return MPDPFT_OK;
}

}  // extern "C"
