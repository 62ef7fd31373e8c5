// engine.h -- the context object behind the C ABI (host side).
#pragma once
#include <cuda_runtime.h>

#include <condition_variable>
#include <functional>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/mpdpft_gpu.h"
#include "common.cuh"
#include "sc_step.cuh"

namespace mpdpft {

int set_error(int status, const std::string& msg);
extern thread_local std::string g_last_error;

struct FftPlan;  // fft.cu
struct Adjoint;  // adjoint.cu

// n doubles from a caller's array into pinned staging memory (engine.cu).
void copy_to_pinned(double* dst, const double* src, long n);

// Host threads for the copies between callers' host arrays and the pinned
// staging buffer (engine.cu): begin() hands every worker t the job f(t)
// and returns; wait() returns when all have finished it.
struct CopyPool {
  int nt = 1;
  CopyPool();
  ~CopyPool();
  void begin(std::function<void(int)> f);
  void wait();

 private:
  std::vector<std::thread> th;
  std::mutex m;
  std::condition_variable cv, done;
  std::function<void(int)> job;
  unsigned gen = 0;
  int pending = 0;
  bool stop = false;
};

// kinds of Ctx::spectral
enum { SPEC_DERIV = 0, SPEC_SMOOTH = 1, SPEC_COULOMB = 2 };

// energy integrals per solve (k_energy)
// [5 s + k] per species, [5 kMaxS + s kMaxS + t] pairs, then the kinetic
// integrals of the gradient-corrected density: [kEkinOff + s] its point
// values, [kEkinOff + kMaxS + s] int V n (2D)
constexpr int kEkinOff = 5 * kMaxS + kMaxS * kMaxS;
constexpr int kNEnergy = kEkinOff + 2 * kMaxS;

struct Ctx {
  mpdpft_params P;
  int device = 0;
  int num_sms = 148;
  cudaStream_t stream = nullptr;
  Geom geom;
  long n_ref = 0;
  size_t rsize = 8;
  int S = 1;
  int ring = 2;
  bool gradient = false;
  bool need_g2 = false;  // the SC loop's functional reads |grad V|^2
  bool finite_t = false; // 3D gradient form at finite T (MPDPFT_GRADIENT_FINITE_T)
  int has_coulomb = 0;
  double temperature[kMaxS];
  bool initialised = false;
  bool admix_only = false;

  // device buffers (compute precision unless noted)
  void* d_vext = nullptr;  // [S][n]
  void* d_V = nullptr;     // [S][n]
  void* d_nin = nullptr;   // [ring][S][n]
  void* d_res = nullptr;   // [ring][S][n]
  void* d_tmp = nullptr;   // [S][n]
  void* d_cur = nullptr;   // [S][n] copy of the current input densities
  void* d_lap = nullptr;   // [S][n]
  void* d_g2 = nullptr;    // [S][n]
  void* d_vh = nullptr;    // [S][n] Coulomb terms of V
  double* d_io = nullptr;  // staging, double
  double* d_part = nullptr;
  int part_vals = 0;
  ScState* d_state = nullptr;
  mpdpft_iter_log* d_log = nullptr;
  int log_cap = 0;
  int step_blocks = 0;
  int fk = 0;            // functional kind of the SC kernels (functional_kind)
  int dens_which = 1;    // density kernel variant: 1 Pulay window <= 5, 3 <= 8, 2 up to kMaxP
  int dens_blocks = 0;   // grid of the density kernel
  int mix_blocks = 0;    // grid of the mixing kernel
  long chunk = kSegPts;  // points per warp in the mu kernel's list sweeps
  int* d_bcount = nullptr;    // [kMaxS][step_blocks] active points per block
  int* d_plist = nullptr;     // [S][plist_stride] active-point lists (a region per warp)
  long plist_stride = 0;      // >= n + 32 (warps of the largest mu grid + 1)
  double* d_part2 = nullptr;  // [dens_blocks][kNPart] density-kernel partial sums
  int assemble_in_step = 1;
  const double* vres_part_ext = nullptr;
  int vres_blocks_ext = 0;
  void* pinned = nullptr;
  std::vector<cudaEvent_t> copy_events;  // per-chunk events of device_to_host
  std::unique_ptr<CopyPool> copy_pool;    // host copy threads, started at the first host copy
  size_t pinned_bytes = 0;
  std::vector<void*> allocations;
  cudaGraph_t graph = nullptr;          // one SC iteration (mpdpft_sc_step)
  cudaGraphExec_t graph_exec = nullptr;
  // the whole SC loop on the device: a WHILE conditional node around one
  // iteration whose last kernel clears the condition at the exit test
  cudaGraph_t loop_graph = nullptr;
  cudaGraphExec_t loop_exec = nullptr;
  int loop_state = 0;  // 0: not built yet, 1: built, -1: not available (host loop)
  KParams graph_kp;    // kernel parameters the captured graphs were built with
  FftPlan* fft = nullptr;
  Adjoint* adj = nullptr;  // adjoint work fields (allocated on first use)
  // launches of the iteration being captured, in issue order: kernel name
  // and algorithmic bytes (each input and output field counted once)
  struct LaunchNote {
    char name[32];
    double bytes;
  };
  std::vector<LaunchNote> notes;
  bool noting = false;
  void note(const char* name, double bytes);
  double field_bytes() const { return (double)geom.n * (double)rsize; }
  double spec_bytes() const { return (double)geom.n * (double)rsize * (geom.s + 2) / geom.s; }
  int iteration_profile(int cap, mpdpft_launch_record* out, int* n_out);
  int mu_max_passes = kMuMaxPasses;     // device loop limits (mpdpft_set_limits)
  long spin_limit = kBarrierSpinLimit;
  int cnt[6] = {0, 0, 0, 0, 0, 0};       // launches issued, by stage
  int iter_cnt[6] = {0, 0, 0, 0, 0, 0};  // launches in the captured iteration

  ~Ctx();
  void release();
  int alloc(void** p, size_t bytes);
  int init(const mpdpft_params& params, int dev);
  int reset_state(bool sync = true);
  int read_state(ScState* h);
  int status_from_state(const ScState& h);
  int set_limits(int mu_passes, long long spins);
  bool has_interaction(int t) const;
  KParams kparams() const;
  int import_field(const double* src, void* dst, int layout, int mem, int slot = 0, bool sync = true);
  int import_staged(const double* src, void* dst, int layout, int slot, bool sync);
  double* host_stage(int slot);  // half slot of the pinned staging buffer
  int export_field(const void* src, double* dst, int layout, int mem);
  int get_field(int which, int s, double* out, int layout, int mem);
  template <typename R>
  StepArgs<R> step_args(int mode);
  int launch_step(int mode, int parts = 7);  // parts: 1 mu, 2 density, 4 mixing kernel
  int issue_iteration();
  // check: wait for the initial densities and report a device abort now
  // (false when the SC loop follows at once and reads the state itself)
  int sc_init(const double* const* v0, int layout, int mem, bool check = true);
  int sc_step(int use_graph);
  void drop_graphs();
  void check_graphs();  // drop captured graphs whose kernel parameters changed
  int build_loop();
  int sc_run(mpdpft_result* result, mpdpft_iter_log* log, int cap, int use_graph);
  int fill_result(mpdpft_result* r, const ScState& h);
  int energy(mpdpft_result* r, const ScState& h);
  // kNEnergy integrals to e_dev (device); g2_current: d_g2 already holds
  // |grad V|^2 of the current V (the batch's 2D transforms always write it)
  int energy_issue(const ScState& h, double* e_dev, bool g2_current = false);
  void energy_finish(mpdpft_result* r, const double* E);
  int ekin_issue(const void* dens, const double* d_mu, const double* e_dev, int maxit, double* out);
  template <typename R>
  void launch_energy(int blocks, const void* dens, const double* d_mu);
  int integrate_device(const void* f, double* out);
  // standalone operators
  int op_mu_search(int s, const double* v, double target, double* mu_io, double* ab_out, int* trials,
                   double* n_out, int layout, int mem);
  int op_density(int s, const double* v, double mu, double* n_out, double* ab_out, int layout, int mem);
  int op_integrate(const double* f, double* out, int layout, int mem);
  int op_admix(const double* const* n_in, const double* const* n_out, const double* theta, double* const* n_mixed,
               double* coeffs, int* ncoeff, int layout, int mem);
  // FFT-based terms (fft.cu)
  int fft_setup();
  int fft_autotune();  // plane or pass path for 3D transforms (timed, cached per kind)
  int fft_config(int* path, double* ms_plane, double* ms_pass, int* how);
  int fft_tiles(int* axis_lines, int* z_rows);
  // cnt doubles between a host array and device memory through the pinned
  // buffer hs, pipelined over several host threads
  int host_to_device(double* dstage, double* hs, const double* src, long cnt);
  int device_to_host(double* dst, double* hs, const double* dsrc, long cnt);
  void fft_release();
  int issue_fft_terms();                      // Coulomb terms + V assembly + DelField(V)
  int issue_coulomb(const void* dens, void* out, int for_energy);
  int issue_delfield_of_V();
  int op_vint(int type, int s, const double* const* n, double* v_out, int layout, int mem);
  int op_update_v(const double* const* n, double incremental, double* const* v_out, int layout, int mem);
  int op_delfield(const double* f, double* grad2, double* lap, int layout, int mem);
  int op_fft(int sign, const double* in, double* out, int mem);
  // helpers (fft.cu)
  int scale_copy(const void* src, void* dst, double a);
  int axpy(const void* x, void* y, double a, int accumulate);
  int copy_current_density();
  int pointwise_vint(int type, int s, void* out);
  int full_c2c(void* buf, int sign);
  int profile_stage(int stage, int reps, double* ms, double* bytes);
  // linear spectral operators and the Hartree operator of one field (fft.cu)
  int spectral(const void* in, int kind, int j, void* out, double coef);
  int coulomb_field(const void* in, void* out);
  // adjoint of the converged fixed point (adjoint.cu)
  int adjoint(const double* dl_dn, double* dl_dvext, int layout, int mem, double tol, int max_iter, int* iters,
              double* resid);
  int adjoint_nuclei(const double* dl_dvext, int mem, int nn, const double* z, const double* pos, double sigma,
                     double* dl_dpos);
  void adjoint_release();
};

// the reference's files (refio.cu)
int write_field_files(Ctx& c, const char* v_path, const char* den_path);
int interpolate_v_file(Ctx& c, const char* path, double* const* v_out, int layout, int mem, int* n_file);

}  // namespace mpdpft
