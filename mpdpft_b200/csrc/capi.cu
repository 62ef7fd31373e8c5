// capi.cu -- extern "C" entry points of include/mpdpft_gpu.h.
#include <chrono>
#include <cstring>
#include <new>

#include "../../include/mpdpft_gpu.h"
#include "engine.h"

using mpdpft::Ctx;
using mpdpft::set_error;

struct mpdpft_ctx {
  Ctx impl;
};

#define CHECK_CTX(c) \
  if (!(c)) return set_error(MPDPFT_ERR_ARG, "null context")

extern "C" {

void mpdpft_params_default(mpdpft_params* p) {
  if (!p) return;
  std::memset(p, 0, sizeof(*p));
  p->dim = 3;
  p->steps = 64;
  p->species = 1;
  p->edge = 16.0;
  p->rel_acc = 1.0e-10;
  p->density_expression = MPDPFT_DENS_TF;
  for (int s = 0; s < MPDPFT_MAX_SPECIES; ++s) {
    p->abundances[s] = 1.0;
    p->tau[s] = 1.0;
    p->temperature[s] = 1.0;
    p->mu[s] = 5.5;
    p->theta[s] = 0.3;
    p->charges[s] = 1.0;
  }
  p->incremental_v = 1.0;
  p->deltamu_modifier = -3.0;
  p->mixer = 1;
  p->pulay_scope = 5;
  p->sc_criterion = 1.0e-12;
  p->max_sc_count = 200;
  p->degeneracy = 1.0;
  p->regularization_threshold = 0.375;
  p->taper_off = 1;
  p->coulomb_kernel = MPDPFT_COULOMB_REGULARISED;
  p->gradient_floor = 1.0e-3;
  p->precision = MPDPFT_FP64;
  // mpDPFT.input sample: Mpp 1 1 1e-6, InternalAcc 0.01
  p->gradient_form = MPDPFT_GRADIENT_T0;
  p->airy_threshold = 1.0e-6;
  p->boole_pairs = 1;
  p->boole_max_iter = 1;
  p->internal_acc = 0.01;
}

int mpdpft_abi_version(void) { return MPDPFT_ABI_VERSION; }

size_t mpdpft_struct_size(int which) {
  switch (which) {
    case 0: return sizeof(mpdpft_params);
    case 1: return sizeof(mpdpft_result);
    case 2: return sizeof(mpdpft_iter_log);
    case 3: return sizeof(mpdpft_input);
    case 4: return sizeof(mpdpft_launch_record);
    default: return 0;
  }
}

const char* mpdpft_last_error(void) { return mpdpft::g_last_error.c_str(); }

const char* mpdpft_status_string(int status) {
  switch (status) {
    case MPDPFT_OK: return "ok";
    case MPDPFT_ERR_ARG: return "invalid argument";
    case MPDPFT_ERR_CUDA: return "CUDA error";
    case MPDPFT_ERR_NONFINITE: return "non-finite value";
    case MPDPFT_ERR_MU_BRACKET: return "mu bracket not found";
    case MPDPFT_ERR_PULAY_SINGULAR: return "Pulay matrix rejected";
    case MPDPFT_ERR_TIMEOUT: return "device loop cap reached";
    case MPDPFT_ERR_NOT_CONVERGED: return "not converged";
    case MPDPFT_ERR_NO_DEVICE: return "no usable device";
    case MPDPFT_WARN_MU_TRAPPED: return "mu search trapped (warning)";
    default: return "unknown status";
  }
}

int mpdpft_ctx_create(const mpdpft_params* params, int device, mpdpft_ctx** out) {
  if (!params || !out) return set_error(MPDPFT_ERR_ARG, "null argument");
  *out = nullptr;
  mpdpft_ctx* c = new (std::nothrow) mpdpft_ctx;
  if (!c) return set_error(MPDPFT_ERR_ARG, "out of host memory");
  int st = c->impl.init(*params, device);
  if (!st) st = c->impl.fft_setup();
  if (st) {
    delete c;
    return st;
  }
  *out = c;
  return MPDPFT_OK;
}

int mpdpft_ctx_destroy(mpdpft_ctx* ctx) {
  if (!ctx) return MPDPFT_OK;
  cudaSetDevice(ctx->impl.device);
  cudaStreamSynchronize(ctx->impl.stream);
  ctx->impl.fft_release();
  delete ctx;
  return MPDPFT_OK;
}

int mpdpft_ctx_sync(mpdpft_ctx* ctx) {
  CHECK_CTX(ctx);
  cudaError_t e = cudaStreamSynchronize(ctx->impl.stream);
  if (e != cudaSuccess) return set_error(MPDPFT_ERR_CUDA, cudaGetErrorString(e));
  return MPDPFT_OK;
}

void* mpdpft_ctx_stream(mpdpft_ctx* ctx) { return ctx ? (void*)ctx->impl.stream : nullptr; }

int mpdpft_set_limits(mpdpft_ctx* ctx, int mu_max_passes, long long barrier_spin_limit) {
  CHECK_CTX(ctx);
  return ctx->impl.set_limits(mu_max_passes, barrier_spin_limit);
}

int mpdpft_set_external_potential(mpdpft_ctx* ctx, int s, const double* v_ext, int layout, int mem) {
  CHECK_CTX(ctx);
  Ctx& c = ctx->impl;
  if (s < 0 || s >= c.S) return set_error(MPDPFT_ERR_ARG, "species index out of range");
  cudaSetDevice(c.device);
  return c.import_field(v_ext, (char*)c.d_vext + (size_t)s * c.geom.n * c.rsize, layout, mem);
}

int mpdpft_density(mpdpft_ctx* ctx, int s, const double* v, double mu, double* n_out, double* abundance_out,
                   int layout, int mem) {
  CHECK_CTX(ctx);
  cudaSetDevice(ctx->impl.device);
  return ctx->impl.op_density(s, v, mu, n_out, abundance_out, layout, mem);
}

int mpdpft_vint(mpdpft_ctx* ctx, int type, int s, const double* const* n, double* v_out, int layout, int mem) {
  CHECK_CTX(ctx);
  cudaSetDevice(ctx->impl.device);
  return ctx->impl.op_vint(type, s, n, v_out, layout, mem);
}

int mpdpft_update_v(mpdpft_ctx* ctx, const double* const* n, double incremental, double* const* v_out, int layout,
                    int mem) {
  CHECK_CTX(ctx);
  cudaSetDevice(ctx->impl.device);
  return ctx->impl.op_update_v(n, incremental, v_out, layout, mem);
}

int mpdpft_mu_search(mpdpft_ctx* ctx, int s, const double* v, double n_target, double* mu_io,
                     double* abundance_out, int* trials_out, double* n_out, int layout, int mem) {
  CHECK_CTX(ctx);
  if (!mu_io) return set_error(MPDPFT_ERR_ARG, "null mu");
  cudaSetDevice(ctx->impl.device);
  return ctx->impl.op_mu_search(s, v, n_target, mu_io, abundance_out, trials_out, n_out, layout, mem);
}

int mpdpft_delfield(mpdpft_ctx* ctx, const double* f, double* grad2_out, double* laplacian_out, int layout, int mem) {
  CHECK_CTX(ctx);
  cudaSetDevice(ctx->impl.device);
  return ctx->impl.op_delfield(f, grad2_out, laplacian_out, layout, mem);
}

int mpdpft_fft(mpdpft_ctx* ctx, int sign, const double* in, double* out, int mem) {
  CHECK_CTX(ctx);
  cudaSetDevice(ctx->impl.device);
  return ctx->impl.op_fft(sign, in, out, mem);
}

int mpdpft_integrate(mpdpft_ctx* ctx, const double* f, double* out, int layout, int mem) {
  CHECK_CTX(ctx);
  if (!out) return set_error(MPDPFT_ERR_ARG, "null output");
  cudaSetDevice(ctx->impl.device);
  return ctx->impl.op_integrate(f, out, layout, mem);
}

int mpdpft_pulay_reset(mpdpft_ctx* ctx) {
  CHECK_CTX(ctx);
  cudaSetDevice(ctx->impl.device);
  return ctx->impl.reset_state();
}

int mpdpft_admix(mpdpft_ctx* ctx, const double* const* n_in, const double* const* n_out, const double* theta,
                 double* const* n_mixed, double* coeffs_out, int* n_coeffs_out, int layout, int mem) {
  CHECK_CTX(ctx);
  if (!n_in || !n_out || !n_mixed) return set_error(MPDPFT_ERR_ARG, "null density arrays");
  cudaSetDevice(ctx->impl.device);
  return ctx->impl.op_admix(n_in, n_out, theta, n_mixed, coeffs_out, n_coeffs_out, layout, mem);
}

int mpdpft_sc_init(mpdpft_ctx* ctx, const double* const* v0, int layout, int mem) {
  CHECK_CTX(ctx);
  cudaSetDevice(ctx->impl.device);
  return ctx->impl.sc_init(v0, layout, mem);
}

int mpdpft_sc_step(mpdpft_ctx* ctx, int graph, mpdpft_iter_log* log) {
  CHECK_CTX(ctx);
  cudaSetDevice(ctx->impl.device);
  int st = ctx->impl.sc_step(graph);
  if (st || !log) return st;
  mpdpft::ScState h;
  if ((st = ctx->impl.read_state(&h))) return st;
  int idx = h.sc_count - 1;
  if (idx < 0 || idx >= ctx->impl.log_cap) return MPDPFT_OK;
  cudaError_t e = cudaMemcpy(log, ctx->impl.d_log + idx, sizeof(mpdpft_iter_log), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return set_error(MPDPFT_ERR_CUDA, cudaGetErrorString(e));
  return ctx->impl.status_from_state(h);
}

int mpdpft_sc_run(mpdpft_ctx* ctx, const double* const* v0, int layout, int mem, mpdpft_result* result,
                  mpdpft_iter_log* log, int log_cap) {
  CHECK_CTX(ctx);
  cudaSetDevice(ctx->impl.device);
  // result->seconds: the whole solve, the initial densities (sc_init: V_0
  // import, DelField, the first mu search) included
  const auto t0 = std::chrono::steady_clock::now();
  // (the loop reads the state after the initial densities itself: a device
  // abort there ends the loop before its first iteration and is reported)
  int st = ctx->impl.sc_init(v0, layout, mem, /*check=*/false);
  if (st) return st;
  st = ctx->impl.sc_run(result, log, log_cap, /*use_graph=*/1);
  if (result) result->seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  return st;
}

int mpdpft_get_field(mpdpft_ctx* ctx, int which, int s, double* out, int layout, int mem) {
  CHECK_CTX(ctx);
  cudaSetDevice(ctx->impl.device);
  return ctx->impl.get_field(which, s, out, layout, mem);
}

int mpdpft_write_field_files(mpdpft_ctx* ctx, const char* v_path, const char* den_path) {
  CHECK_CTX(ctx);
  cudaSetDevice(ctx->impl.device);
  return mpdpft::write_field_files(ctx->impl, v_path, den_path);
}

int mpdpft_interpolate_v_file(mpdpft_ctx* ctx, const char* path, double* const* v_out, int layout, int mem,
                              int* n_file) {
  CHECK_CTX(ctx);
  cudaSetDevice(ctx->impl.device);
  return mpdpft::interpolate_v_file(ctx->impl, path, v_out, layout, mem, n_file);
}

int mpdpft_energy(mpdpft_ctx* ctx, mpdpft_result* result) {
  CHECK_CTX(ctx);
  if (!result) return set_error(MPDPFT_ERR_ARG, "null result");
  cudaSetDevice(ctx->impl.device);
  mpdpft::ScState h;
  int st = ctx->impl.read_state(&h);
  if (st) return st;
  std::memset(result, 0, sizeof(*result));
  return ctx->impl.fill_result(result, h);
}

int mpdpft_profile_stage(mpdpft_ctx* ctx, int stage, int reps, double* ms_per_launch, double* bytes_per_launch) {
  CHECK_CTX(ctx);
  if (reps < 1 || !ms_per_launch) return set_error(MPDPFT_ERR_ARG, "bad profile arguments");
  cudaSetDevice(ctx->impl.device);
  return ctx->impl.profile_stage(stage, reps, ms_per_launch, bytes_per_launch);
}

int mpdpft_iteration_launches(mpdpft_ctx* ctx, int* counts, int* total) {
  CHECK_CTX(ctx);
  int t = 0;
  for (int i = 0; i < 6; ++i) {
    if (counts) counts[i] = ctx->impl.iter_cnt[i];
    t += ctx->impl.iter_cnt[i];
  }
  if (total) *total = t;
  return MPDPFT_OK;
}

int mpdpft_fft_config(mpdpft_ctx* ctx, int* path, double* ms_plane, double* ms_pass, int* how) {
  CHECK_CTX(ctx);
  return ctx->impl.fft_config(path, ms_plane, ms_pass, how);
}

int mpdpft_fft_tiles(mpdpft_ctx* ctx, int* axis_lines, int* z_rows) {
  CHECK_CTX(ctx);
  return ctx->impl.fft_tiles(axis_lines, z_rows);
}

int mpdpft_adjoint(mpdpft_ctx* ctx, const double* dl_dn, double* dl_dvext, int layout, int mem, double tol,
                   int max_iter, int* iterations, double* residual) {
  CHECK_CTX(ctx);
  cudaSetDevice(ctx->impl.device);
  return ctx->impl.adjoint(dl_dn, dl_dvext, layout, mem, tol, max_iter, iterations, residual);
}

int mpdpft_adjoint_nuclei(mpdpft_ctx* ctx, const double* dl_dvext, int mem, int n_nuclei, const double* charges,
                          const double* positions, double sigma, double* dl_dpositions) {
  CHECK_CTX(ctx);
  cudaSetDevice(ctx->impl.device);
  return ctx->impl.adjoint_nuclei(dl_dvext, mem, n_nuclei, charges, positions, sigma, dl_dpositions);
}

int mpdpft_iteration_profile(mpdpft_ctx* ctx, int cap, mpdpft_launch_record* records, int* n_out) {
  CHECK_CTX(ctx);
  if (cap < 0) return set_error(MPDPFT_ERR_ARG, "negative capacity");
  cudaSetDevice(ctx->impl.device);
  return ctx->impl.iteration_profile(cap, records, n_out);
}

int mpdpft_step_phase_times(mpdpft_ctx* ctx, double* us, int n) {
  CHECK_CTX(ctx);
  if (!us || n < 1) return set_error(MPDPFT_ERR_ARG, "bad arguments");
  cudaSetDevice(ctx->impl.device);
  mpdpft::ScState h;
  int st = ctx->impl.read_state(&h);
  if (st) return st;
  for (int i = 0; i < n && i < 6; ++i) us[i] = 1e-3 * (double)(h.tphase[i + 1] - h.tphase[i]);
  return MPDPFT_OK;
}

}  // extern "C"
