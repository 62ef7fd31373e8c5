/*
 * mpdpft_gpu.h -- C ABI of the B200 self-consistent DPFT engine.
 *
 * This is the drop-in boundary for mpDPFT's self-consistent (SC) loop.  The
 * reference exposes that loop as free C++ functions over one mutable
 * `datastruct&` (mpDPFT.h:71-93); every entry point below replaces one of
 * them and names it.  All arrays crossing this boundary are IEEE double, the
 * reference's storage type, whatever precision the engine computes in.
 *
 * Grids.  The engine stores every field on the periodic grid of s^D points
 * (s = steps), x-major (index = (i*s + j)*s + k, x = -L/2 + i*dx, dx = L/s).
 * The reference stores (s+1)^D points whose last plane along each axis
 * duplicates plane 0 (mpDPFT.cpp:863, refilled by fftParallel
 * mpDPFT.cpp:8266-8324).  Pass MPDPFT_LAYOUT_REFERENCE to exchange arrays in
 * that layout: inputs drop the duplicate planes, outputs refill them.
 *
 * Memory.  MPDPFT_MEM_HOST pointers are copied through pinned staging
 * buffers on the context stream; MPDPFT_MEM_DEVICE pointers must be device
 * memory on the context's GPU.
 *
 * Errors.  Every call returns an mpdpft_status.  Nothing calls exit(); the
 * text of the last error on the calling host thread is returned by
 * mpdpft_last_error().  A context is not re-entrant; distinct contexts are
 * independent and may be driven from different host threads.
 */
#ifndef MPDPFT_GPU_H
#define MPDPFT_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MPDPFT_ABI_VERSION 2
#define MPDPFT_MAX_SPECIES 4
#define MPDPFT_MAX_INTERACTIONS 8
#define MPDPFT_MAX_PULAY 12
#define MPDPFT_NOALLOC_MAX_POINTS 16777216 /* largest grid of mpdpft_integrate_noalloc (256^3) */

typedef enum {
  MPDPFT_OK = 0,
  MPDPFT_ERR_ARG = 1,           /* invalid argument or unsupported option      */
  MPDPFT_ERR_CUDA = 2,          /* CUDA runtime error                          */
  MPDPFT_ERR_NONFINITE = 3,     /* non-finite value in an input or a result    */
  MPDPFT_ERR_MU_BRACKET = 4,    /* mu bracket not found; mu reset (warning)    */
  MPDPFT_ERR_PULAY_SINGULAR = 5,/* Pulay Gram matrix rejected; linear mixing   */
  MPDPFT_ERR_TIMEOUT = 6,       /* a device loop reached its iteration cap     */
  MPDPFT_ERR_NOT_CONVERGED = 7, /* maxSCcount reached before convergence       */
  MPDPFT_ERR_NO_DEVICE = 8,     /* no usable sm_100 device                     */
  /* warning: the mu search ended inside its bracket without meeting
   * rel_acc (a step of N(mu) at the target), the reference's TrappedQ
   * (mpDPFT.cpp:4690-4703).  Returned by mpdpft_mu_search (mu and N are
   * the search's end point); in an SC iteration a status bit only, and the
   * iteration mixes with theta scaled by min(1, |1 - RelDiff|^30),
   * RelDiff = |N* - N| / |N*| (AdmixDensities, mpDPFT.cpp:4929-4934)     */
  MPDPFT_WARN_MU_TRAPPED = 9
} mpdpft_status;

enum { MPDPFT_FP64 = 0, MPDPFT_MIXED = 1 };
enum { MPDPFT_LAYOUT_PERIODIC = 0, MPDPFT_LAYOUT_REFERENCE = 1 };
enum { MPDPFT_MEM_HOST = 0, MPDPFT_MEM_DEVICE = 1 };

/* Density functionals, numbered as the reference's DensityExpression
 * (mpDPFT.input line 15, dispatcher mpDPFT.cpp:2142-2238). */
enum {
  MPDPFT_DENS_TF_INSPIRED = 1,   /* GetTFinspireddensity T=0   mpDPFT.cpp:3318-3347 */
  MPDPFT_DENS_TF_INSPIRED_T = 2, /* GetTFinspireddensity T>0   mpDPFT.cpp:3340-3345 */
  MPDPFT_DENS_GRADIENT = 5,      /* getDenEnAt small-gradient branch, T->0 form
                                    mpDPFT.cpp:3376-3388; needs DelField        */
  MPDPFT_DENS_TF = 7             /* GetTFdensity               mpDPFT.cpp:4415-4436 */
};

/* Interaction types, numbered as the reference's getVint (mpDPFT.cpp:2240-2318). */
enum {
  MPDPFT_INT_NONE = 0,
  MPDPFT_INT_CONTACT_MUTUAL = 1, /* V_s = beta * sum_{s'!=s} n_s'          :2247-2253 */
  MPDPFT_INT_HARTREE = 8,        /* V_s = gammaH * Coulomb[n_s]           :2677-2715 */
  MPDPFT_INT_CONTACT_SELF = 10,  /* V = 2 beta n_0                        :2261-2264 */
  MPDPFT_INT_DIRAC = 11,         /* V_s = -gammaH (3 n_s/pi)^(1/3)       :2759-2772 */
  MPDPFT_INT_HARTREE_INTER = 21, /* V_s = gammaH * sum_{s'!=s} Coulomb[n_s'] :2273-2285 */
  MPDPFT_INT_COULOMB_CHARGED = 100 /* no reference counterpart: V_s = q_s gammaH
                                      Coulomb[sum_s' q_s' n_s'] (charged species) */
};

/* Coulomb kernels for the Hartree solve. */
enum {
  MPDPFT_COULOMB_REGULARISED = 0, /* reference kernel: (n~ - n~0 e^{-k^2})/k^2 plus
                                     n~0 erf(r/2)/r, mpDPFT.cpp:2677-2715          */
  MPDPFT_COULOMB_TRUNCATED = 1    /* spherical cutoff 4 pi (1 - cos kR)/k^2         */
};

/* Parameters of one SC solve.  Field names follow mpDPFT.input
 * (parser mpDPFT.cpp:633-690); the line number is given for each. */
typedef struct {
  int dim;                  /* line 5  DIM: 2 or 3                                  */
  int steps;                /* line 8  steps s (even; FFT sizes 2^a 3^b)            */
  int species;              /* line 9  S                                            */
  double edge;              /* line 7  box edge L, box [-L/2, L/2]^D                */
  double abundances[MPDPFT_MAX_SPECIES]; /* line 10 target particle numbers N*_s    */
  double rel_acc;           /* line 11 RelAcc of the mu search                      */
  int density_expression;   /* line 15 one of MPDPFT_DENS_*                         */
  double tau[MPDPFT_MAX_SPECIES];   /* line 18 tauVec (TF-inspired densities)       */
  double temperature[MPDPFT_MAX_SPECIES]; /* line 20 TVec                          */
  int n_interactions;       /* line 26 Interactions                                 */
  int interactions[MPDPFT_MAX_INTERACTIONS];
  double incremental_v;     /* line 27 incrementalV ramp per SC iteration (1 = off) */
  double mu[MPDPFT_MAX_SPECIES];    /* line 28 muVec: initial chemical potentials   */
  double deltamu_modifier;  /* line 29 DeltamuModifier                              */
  int mixer;                /* line 30 Mixer[0]: 0 linear, 1 Pulay                  */
  int pulay_scope;          /* line 30 Mixer[1]: Pulay history length (<= MAX)      */
  double theta[MPDPFT_MAX_SPECIES]; /* line 31 thetaVec admixtures                  */
  double sc_criterion;      /* line 32 SCcriterion                                  */
  int max_sc_count;         /* line 33 maxSCcount                                   */
  int schedule;             /* line 37 Schedule: 0 none, 5 adaptive theta, 9 ramp   */
  double beta;              /* line 40 contact strength                             */
  double gamma_h;           /* line 42 gammaH Coulomb prefactor                     */
  double degeneracy;        /* line 43 g                                            */
  double regularization_threshold; /* line 45 RegularizationThreshold (taper radius
                                      fraction of the edge)                         */
  /* hard-coded values of the reference, exposed with the reference defaults */
  int taper_off;            /* TaperOff = 1 (mpDPFT.h:79; DelField :7251-7264)      */
  double smearing_extent;   /* Gaussian smoothing width; <= 0 means 6*dx (:1105)    */
  /* options of this engine */
  double charges[MPDPFT_MAX_SPECIES]; /* species charges for MPDPFT_INT_COULOMB_CHARGED */
  int coulomb_kernel;       /* MPDPFT_COULOMB_*                                     */
  double coulomb_cutoff;    /* truncated kernel radius R; <= 0 means L/2            */
  double gradient_floor;    /* floor on mu - V in the (mu-V)^{-1/2} and ^{-3/2}
                               gradient terms of MPDPFT_DENS_GRADIENT               */
  double gradient_grad2;    /* coefficient of the |grad V|^2 term (0: reference
                               small-gradient branch; 1: second-order
                               Wigner-Kirkwood)                                    */
  double potential_tol;     /* extra exit test: rms(V_new - V_old) <= tol (0: off)  */
  int precision;            /* MPDPFT_FP64 or MPDPFT_MIXED                          */
  /* MPDPFT_DENS_GRADIENT in 3D (ABI version 2) */
  int gradient_form;        /* MPDPFT_GRADIENT_T0 or MPDPFT_GRADIENT_FINITE_T       */
  double airy_threshold;    /* line 17 Mpp[2]: Airy-averaged branch where
                               ar = |grad V|^{2/3}/2 >= |threshold| (finite-T form
                               only; 0: everywhere, 1e300: nowhere)                 */
  int boole_pairs;          /* line 17 Mpp[0]: Boole pairs per half interval       */
  int boole_max_iter;       /* line 17 Mpp[1]: bisection depth of the Airy integral */
  double internal_acc;      /* line 12 InternalAcc: relative accuracy of the Airy
                               integral (RTPNA)                                     */
} mpdpft_params;

/* 3D forms of MPDPFT_DENS_GRADIENT. */
enum {
  MPDPFT_GRADIENT_T0 = 0,       /* closed T -> 0 form (gradient_floor, gradient_grad2) */
  MPDPFT_GRADIENT_FINITE_T = 1  /* the reference's finite-T Fermi-Dirac form with the
                                   Airy-averaged branch, mpDPFT.cpp:3363-3453       */
};

/* Per-iteration record of mpdpft_sc_run (the reference prints SCcount, CC,
 * mu and abundances per iteration, mpDPFT.cpp:4862). */
typedef struct {
  int sc_count;
  int mu_trials;            /* density evaluations spent in the mu search          */
  int pulay_used;           /* 1 if Pulay mixing was applied                       */
  int status_bits;          /* bit k set = status k raised during this iteration    */
  double cc;                /* convergence criterion, CheckConvergence :4759-4782   */
  double v_residual;        /* rms of V between consecutive iterations             */
  double mu[MPDPFT_MAX_SPECIES];
  double abundance[MPDPFT_MAX_SPECIES];
  double theta[MPDPFT_MAX_SPECIES];
  double ms;                /* device time of the iteration                        */
} mpdpft_iter_log;

typedef struct {
  int iterations;           /* SC iterations run                                   */
  int converged;            /* 1 if the exit rule was met                          */
  int total_mu_trials;
  int device_loop;          /* 1 if the SC loop ran as one device-side graph loop
                               (no host round trip per iteration), 0 if the host
                               replayed one iteration at a time                 */
  double cc;
  double v_residual;
  double mu[MPDPFT_MAX_SPECIES];
  double abundance[MPDPFT_MAX_SPECIES];
  double e_total;
  double e_kinetic[MPDPFT_MAX_SPECIES];
  double e_external[MPDPFT_MAX_SPECIES];
  double e_interaction[MPDPFT_MAX_INTERACTIONS];
  double seconds;           /* wall time of the solve (mpdpft_sc_run: from the
                               initial densities to the energies of the result) */
} mpdpft_result;

typedef struct mpdpft_ctx mpdpft_ctx;
typedef struct mpdpft_batch mpdpft_batch;

/* Fill *p with the reference defaults (mpDPFT.input sample values and the
 * hard-coded defaults of InitializeHardCodedParameters, mpDPFT.cpp:858-1115). */
void mpdpft_params_default(mpdpft_params* p);

int mpdpft_abi_version(void);
/* sizeof(mpdpft_params), sizeof(mpdpft_result), sizeof(mpdpft_iter_log),
 * sizeof(mpdpft_input), sizeof(mpdpft_launch_record) for which = 0 .. 4
 * (binding checks); 0 for any other value. */
size_t mpdpft_struct_size(int which);
const char* mpdpft_last_error(void);
const char* mpdpft_status_string(int status);

/* Context: device buffers, FFT plans and the SC state of one solve.
 * Replaces the allocation half of GetData's initialisation
 * (AllocateDensityMemory :6392, InitializeGlobalFFTWplans :6313,
 * AllocateTMPmemory :6337, InitializePulayMixer :7029). */
int mpdpft_ctx_create(const mpdpft_params* params, int device, mpdpft_ctx** out);
int mpdpft_ctx_destroy(mpdpft_ctx* ctx);
int mpdpft_ctx_sync(mpdpft_ctx* ctx);
/* The context's cudaStream_t, as an opaque pointer. */
void* mpdpft_ctx_stream(mpdpft_ctx* ctx);

/* Limits of the device loops of this context (the reference bounds its mu
 * search by 20 bracket steps and DeltamuModifier, mpDPFT.cpp:4584-4711, and
 * has no device waits): mu_max_passes caps the evaluation passes of one mu
 * search (1 .. 24, default 24; reaching it raises MPDPFT_ERR_TIMEOUT with
 * the best mu found), barrier_spin_limit bounds each wait of the mu
 * kernel's grid barriers (polls with a 64 ns back-off, default 2e7; running
 * out aborts the kernel and raises MPDPFT_ERR_TIMEOUT).  Negative values
 * restore the defaults.  The context stays usable after a timeout: the
 * next mpdpft_sc_init, mpdpft_mu_search or mpdpft_pulay_reset clears it. */
int mpdpft_set_limits(mpdpft_ctx* ctx, int mu_max_passes, long long barrier_spin_limit);

/* External potential V_ext of species s.  Replaces GetEnv (mpDPFT.cpp:1385). */
int mpdpft_set_external_potential(mpdpft_ctx* ctx, int s, const double* v_ext,
                                  int layout, int mem);

/* n[V] of species s at chemical potential mu, and N = Integrate(n).
 * Replaces GetDensity (mpDPFT.cpp:2142) followed by Integrate (:7970).
 * For MPDPFT_DENS_GRADIENT the derivatives of V come from DelField. */
int mpdpft_density(mpdpft_ctx* ctx, int s, const double* v, double mu,
                   double* n_out, double* abundance_out, int layout, int mem);

/* V_int[n] of one interaction type for focal species s.  `n` holds the
 * densities of all species, each a pointer to one grid.  Replaces getVint
 * (mpDPFT.cpp:2240), which writes data.TmpField2. */
int mpdpft_vint(mpdpft_ctx* ctx, int type, int s, const double* const* n,
                double* v_out, int layout, int mem);

/* V_s = V_ext,s + incremental * sum_a V_int,a[n] for every species.
 * Replaces UpdateV (mpDPFT.cpp:4815). */
int mpdpft_update_v(mpdpft_ctx* ctx, const double* const* n, double incremental,
                    double* const* v_out, int layout, int mem);

/* Particle-number constraint for species s: find mu with
 * |N(mu) - N*| / (2 N*) <= rel_acc.  Replaces EnforceConstraints
 * (mpDPFT.cpp:4569-4743) for one species.  *mu_io holds the starting mu on
 * entry and the result on exit; the final density is left in n_out when it
 * is not NULL.  Returns MPDPFT_ERR_MU_BRACKET (mu reset to the start value)
 * when no bracket is found, as the reference does, and
 * MPDPFT_WARN_MU_TRAPPED when the bracket closes on a step of N(mu) that
 * the tolerance cannot resolve (the reference's trapped bisection). */
int mpdpft_mu_search(mpdpft_ctx* ctx, int s, const double* v, double n_target,
                     double* mu_io, double* abundance_out, int* trials_out,
                     double* n_out, int layout, int mem);

/* Spectral derivatives of f with Gaussian smoothing (method 5) and the
 * boundary taper.  Writes |grad f|^2 (smoothed, clamped >= 0) and the
 * Laplacian (smoothed).  Replaces DelField(f, s, 5, data) (mpDPFT.cpp:7243-7582). */
int mpdpft_delfield(mpdpft_ctx* ctx, const double* f, double* grad2_out,
                    double* laplacian_out, int layout, int mem);

/* Centred-k complex DFT with the reference's conventions: forward
 * f~(k) = dx^D sum_x f(x) e^{-ikx}, backward f(x) = L^-D sum_k f~(k) e^{ikx},
 * k = -pi/dx + m dk.  Interleaved complex, periodic layout s^D.
 * Replaces fftParallel (mpDPFT.cpp:8173-8335); sign = -1 forward, +1 backward. */
int mpdpft_fft(mpdpft_ctx* ctx, int sign, const double* in, double* out, int mem);

/* Trapezoid integral over the box.  Replaces Integrate(method 1)
 * (Riemann, mpDPFT.cpp:7981-8026).  In the reference layout every stored
 * point counts with Riemann's end weights (1/2 on the first and last plane
 * of each axis); in the periodic layout every point has weight 1. */
int mpdpft_integrate(mpdpft_ctx* ctx, const double* f, double* out, int layout, int mem);

/* The same trapezoid integral without a context and without allocating any
 * device memory.  It has no counterpart in the reference: it exists for
 * callers that cannot call cudaMalloc, e.g. a plug-in whose host application
 * owns all device memory, or a loop that must not pay cudaMalloc's implicit
 * device synchronisation.
 *   f      device pointer, double, periodic s^D or reference (s+1)^D layout
 *          (reference layout: every stored point with the trapezoid end
 *          weights 1/2, as Riemann does; the duplicate planes need not
 *          repeat plane 0);
 *   out    device pointer to one double, written with the integral;
 *   stream cudaStream_t (NULL: the default stream) on the current device.
 * Grids of more than MPDPFT_NOALLOC_MAX_POINTS periodic points (s > 256 in
 * 3D, s > 4096 in 2D) are rejected with MPDPFT_ERR_ARG.  The partial sums
 * live in one fixed array of 33160 bytes that every GPU loading this library
 * holds until the process exits, shared by all calls: calls whose kernels
 * overlap on one GPU (other streams, other host threads) race on it and must
 * be serialised by the caller.  The array's device address belongs to the
 * CUDA context: the first call in each context (and the first after a
 * device reset) looks it up, so make that call before any stream capture.
 * Returns once the work is queued on stream. */
int mpdpft_integrate_noalloc(int dim, int steps, double edge, const double* f, double* out, int layout,
                             void* stream);

/* Density mixing for all species.  mixer 1 runs PulayMixer
 * (mpDPFT.cpp:5005-5167) with its history kept on the device and falls back
 * to linear mixing (AdmixDensities :4921-4992) when the Gram matrix is
 * rejected or on the first call after mpdpft_pulay_reset.  coeffs_out
 * (may be NULL) receives up to MPDPFT_MAX_PULAY coefficients. */
int mpdpft_pulay_reset(mpdpft_ctx* ctx);
int mpdpft_admix(mpdpft_ctx* ctx, const double* const* n_in, const double* const* n_out,
                 const double* theta, double* const* n_mixed, double* coeffs_out,
                 int* n_coeffs_out, int layout, int mem);

/* Full SC solve (GetData's loop, mpDPFT.cpp:210-229).  v0 (may be NULL: start
 * from V_ext) holds the starting potentials of all species.  The per-iteration
 * log is written when log != NULL (at most log_cap records).  The final
 * densities and potentials stay in the context (mpdpft_get_field). */
int mpdpft_sc_run(mpdpft_ctx* ctx, const double* const* v0, int layout, int mem,
                  mpdpft_result* result, mpdpft_iter_log* log, int log_cap);

/* One SC iteration on the current state (captured as a CUDA graph after the
 * first call when graph != 0).  Used by benchmarks and the batch engine. */
int mpdpft_sc_step(mpdpft_ctx* ctx, int graph, mpdpft_iter_log* log);
int mpdpft_sc_init(mpdpft_ctx* ctx, const double* const* v0, int layout, int mem);

enum { MPDPFT_FIELD_DENSITY = 0, MPDPFT_FIELD_POTENTIAL = 1, MPDPFT_FIELD_GRAD2 = 2,
       MPDPFT_FIELD_LAPLACIAN = 3, MPDPFT_FIELD_EXTERNAL = 4 };
int mpdpft_get_field(mpdpft_ctx* ctx, int which, int s, double* out, int layout, int mem);

/* Energies of the current state (GetEnergy, mpDPFT.cpp:5414-5436). */
int mpdpft_energy(mpdpft_ctx* ctx, mpdpft_result* result);

/* Stage timing (the reference's StartTimer/EndTimer per routine,
 * mpDPFT.cpp:11997-12003): launch one stage `reps` times on the context
 * stream, timed with CUDA events; returns the mean device time per launch
 * and the algorithmic bytes one launch must move (its own inputs and
 * outputs, each field counted once).  MPDPFT_STAGE_SC_STEP runs real SC
 * iterations on the current state (after mpdpft_sc_init); the FFT stages
 * transform a zeroed scratch spectrum. */
enum {
  MPDPFT_STAGE_SC_STEP = 0,   /* the SC kernels of one iteration (mu .. mix)  */
  MPDPFT_STAGE_FFT_Z_R2C = 1, /* R2C pass along the contiguous axis           */
  MPDPFT_STAGE_FFT_Y = 2,     /* C2C pass along y (3D)                        */
  MPDPFT_STAGE_FFT_X = 3,     /* x-axis round trip with one k-space multiplier */
  MPDPFT_STAGE_FFT_Z_C2R = 4, /* C2R pass along the contiguous axis           */
  MPDPFT_STAGE_ITERATION = 5, /* one whole SC iteration (graph replay)        */
  MPDPFT_STAGE_SC_MU = 6,     /* mu kernel: V update + mu search              */
  MPDPFT_STAGE_SC_DENSITY = 7,/* density kernel: n_out, residual, sums, scalar step */
  MPDPFT_STAGE_SC_MIX = 8,    /* mixing kernel                                */
  MPDPFT_STAGE_FFT_PLANE_FWD = 9,  /* 3D: z R2C + y C2C by x-planes           */
  MPDPFT_STAGE_FFT_PLANE_INV = 10  /* 3D: y C2C inverse + z C2R by x-planes   */
};
int mpdpft_profile_stage(mpdpft_ctx* ctx, int stage, int reps, double* ms_per_launch,
                         double* bytes_per_launch);

/* Kernel launches in one SC iteration as captured in its CUDA graph:
 * counts[i] for i = MPDPFT_STAGE_SC_STEP .. MPDPFT_STAGE_FFT_Z_C2R (the plane
 * kernels count as Z_R2C / Z_C2R), counts[5] for the remaining (pointwise)
 * kernels; *total = their sum.  Valid after the first graph-mode
 * mpdpft_sc_step. */
int mpdpft_iteration_launches(mpdpft_ctx* ctx, int* counts, int* total);

/* Per-launch device time of one SC iteration as the captured graph runs it
 * (the reference's per-routine timers, mpDPFT.cpp:11997-12003, at kernel
 * granularity).  The nodes of the captured iteration are replayed one at a
 * time, in order, each bracketed by CUDA events on the context stream, so
 * the replay is one real SC iteration on the current state.  Each record
 * names the kernel (or "memset"), its device time and the algorithmic bytes
 * of that launch (its own input and output fields, each counted once).
 * Valid after the first graph-mode mpdpft_sc_step; *n_out = launches. */
typedef struct {
  char name[32];
  double ms;
  double bytes;
} mpdpft_launch_record;
int mpdpft_iteration_profile(mpdpft_ctx* ctx, int cap, mpdpft_launch_record* records, int* n_out);

/* Phase durations (microseconds, block 0 of the grid) of the last SC-step
 * kernel: [0] V update, [1] mu search, [2] densities/residual/Gram row,
 * [3] convergence test and Pulay solve, [4] grid barrier, [5] mix. */
int mpdpft_step_phase_times(mpdpft_ctx* ctx, double* us, int n);

/* FFT path of the context (no counterpart in the reference, which plans
 * FFTW once, mpDPFT.cpp:6313-6335): *path 1 = x-plane kernels, 0 = one pass
 * per axis; the autotuner's best timings of one iteration's transforms on
 * each path over the tile widths it tried (ms; 0 when not measured); *how
 * 0 = nothing to choose, 1 = measured by this context, 2 = taken from an
 * earlier context of the same kind, 3 = path forced by MPDPFT_FFT_PATH. */
int mpdpft_fft_config(mpdpft_ctx* ctx, int* path, double* ms_plane, double* ms_pass, int* how);

/* Tile widths the autotuner chose (3D grids): lines per tile of the Y and X
 * passes (FP32 16 or 8, FP64 8 or 4; fewer where s/2 is not a multiple)
 * and rows per block of the Z passes (16 or 8).  Results do not depend on
 * them; MPDPFT_FFT_TILES=<lines>,<rows> forces them. */
int mpdpft_fft_tiles(mpdpft_ctx* ctx, int* axis_lines, int* z_rows);

/* Adjoint of the converged SC fixed point (no counterpart in the reference,
 * whose optimisation drivers take finite differences of whole solves,
 * mpDPFT.cpp:8448).  After mpdpft_sc_run on a one-species context, dl_dn
 * holds the gradient of a scalar loss L with respect to the converged
 * density at the grid points (periodic layout, host or device doubles);
 * dl_dvext receives dL/dV_ext at the grid points.  The adjoint linear system
 * lambda = dl_dn + J_W^T J_N^T lambda (J_N: density map with the particle-
 * number constraint, DelField and taper; J_W: Hartree, Dirac, contact) is
 * solved by the context's device Pulay mixer until
 * |T(lambda) - lambda| / |T(lambda)| <= tol or max_iter iterations
 * (MPDPFT_ERR_NOT_CONVERGED).  The converged state is kept (its Pulay
 * history restarts).  Functionals: 3D gradient-corrected, 3D TF, 2D
 * gradient-corrected; interactions 8, 10, 11. */
int mpdpft_adjoint(mpdpft_ctx* ctx, const double* dl_dn, double* dl_dvext, int layout, int mem, double tol,
                   int max_iter, int* iterations, double* residual);
/* dL/dR (3 per nucleus) of Gaussian nuclei V_ext = sum_a -Z_a
 * erf(|r - R_a| / (sqrt(2) sigma)) / |r - R_a| from dL/dV_ext (periodic
 * layout, 3D). */
int mpdpft_adjoint_nuclei(mpdpft_ctx* ctx, const double* dl_dvext, int mem, int n_nuclei,
                          const double* charges, const double* positions, double sigma,
                          double* dl_dpositions);

/* ---------------------------------------------------------------------
 * The reference's files.
 *
 * mpDPFT.input: 47 lines, one parameter (or vector) per line in a fixed
 * order, anything after the values ignored (GetInputParameters,
 * mpDPFT.cpp:633-690).  Lines are numbered from 0, as the parser's cases
 * (and the line numbers of mpdpft_params) are.  mpdpft_read_input parses it into mpdpft_input,
 * field by field and in the file's units; mpdpft_params_from_input maps it
 * onto the engine's parameters and rejects (MPDPFT_ERR_ARG, naming the line)
 * options the engine does not implement.  The input's Symmetry is accepted
 * whatever its value: the engine always computes the whole grid.
 */
#define MPDPFT_INPUT_MAX_VEC 16
typedef struct {
  int system;                    /* line 0  System                               */
  int symmetry;                  /* line 1  Symmetry                             */
  int task_type;                 /* line 2  TaskType                             */
  int task_parameter_count;      /* line 3  TaskParameterCount                   */
  int n_task_hyperbox;           /* line 4  TaskHyperBox (values read)           */
  double task_hyperbox[MPDPFT_INPUT_MAX_VEC];
  int dim;                       /* line 5  DIM                                  */
  int units;                     /* line 6  Units: 1 HO / atomic, 2 eV-Angstrom  */
  double edge;                   /* line 7  edge                                 */
  int steps;                     /* line 8  steps                                */
  int species;                   /* line 9 S                                    */
  double abundances[MPDPFT_MAX_SPECIES]; /* line 10                              */
  double rel_acc;                /* line 11 RelAcc                               */
  double internal_acc;           /* line 12 InternalAcc                          */
  int k_resources;               /* line 13 K                                    */
  int density_expression;        /* line 15 DensityExpression                    */
  int n_mpp;                     /* line 16 mpp (environment parameters)         */
  double mpp[MPDPFT_INPUT_MAX_VEC];
  int n_Mpp;                     /* line 17 Mpp (density parameters)             */
  double Mpp[MPDPFT_INPUT_MAX_VEC];
  double tau[MPDPFT_MAX_SPECIES];          /* line 18 tauVec                     */
  double territory[MPDPFT_MAX_SPECIES];    /* line 19 tVec                       */
  double temperature[MPDPFT_MAX_SPECIES];  /* line 20 TVec                       */
  int environments[MPDPFT_MAX_SPECIES];    /* line 21 Environments               */
  double stretchfactor;          /* line 22                                      */
  double wall;                   /* line 23 Wall                                 */
  double noise;                  /* line 24 Noise                                */
  int interpol_vq;               /* line 25 InterpolVQ                           */
  int n_interactions;            /* line 26 Interactions                         */
  int interactions[MPDPFT_INPUT_MAX_VEC];
  double incremental_v;          /* line 27 incrementalV                         */
  double mu[MPDPFT_MAX_SPECIES]; /* line 28 muVec                                */
  double deltamu_modifier;       /* line 29 DeltamuModifier                      */
  double mixer[3];               /* line 30 Mixer: mode, scope, metric weight    */
  double theta[MPDPFT_MAX_SPECIES]; /* line 31 thetaVec                          */
  double sc_criterion;           /* line 32 SCcriterion                          */
  int max_sc_count;              /* line 33 maxSCcount                           */
  int method;                    /* line 34 integration method                   */
  int delfield_method;           /* line 35 DelFieldMethod                       */
  int movie;                     /* line 36 MovieQ                               */
  int n_schedule;                /* line 37 Schedule                             */
  int schedule[MPDPFT_INPUT_MAX_VEC];
  int n_ekin_types;              /* line 38 EkinTypes                            */
  int ekin_types[MPDPFT_INPUT_MAX_VEC];
  double alpha, beta, gamma, gamma_h; /* lines 39-42                             */
  double degeneracy;             /* line 43                                      */
  int n_regularize;              /* line 44 regularize                           */
  int regularize[MPDPFT_INPUT_MAX_VEC];
  double regularization_threshold; /* line 45                                    */
  int print;                     /* line 46 Print                                */
  int lines;                     /* lines read                                   */
} mpdpft_input;

/* Parse an mpDPFT.input file (the reference's line order; lines 0-46
 * above).  MPDPFT_ERR_ARG names the file or the first line that does not
 * parse. */
int mpdpft_read_input(const char* path, mpdpft_input* out);
/* Engine parameters of a parsed input: reference defaults
 * (mpdpft_params_default) overridden by every line the engine uses.
 * Rejected with MPDPFT_ERR_ARG (the message names the line): Units other
 * than 1, DensityExpression other than 1, 2, 5, 7, interaction types the
 * engine lacks, Mixer mode 2, integration method other than 1 (Riemann),
 * DelFieldMethod other than 5 with DensityExpression 5, more than one
 * Schedule entry or one other than 0, 5, 9, and S above
 * MPDPFT_MAX_SPECIES.  DensityExpression 5 in 3D maps to the finite-T form
 * with the Airy branch (Mpp = BoolePairs, maxIter, threshold). */
int mpdpft_params_from_input(const mpdpft_input* in, mpdpft_params* out);

/* Write the context's current potentials and densities in the reference's
 * text formats (ExportData, mpDPFT.cpp:12492-12519): mpDPFT_V.dat has one
 * line per point of the (s+1)^D storage, x-major, with the D coordinates
 * and then V of every species; mpDPFT_Den.dat one line per point with the
 * densities of every species.  16 significant digits.  Either path may be
 * NULL (not written). */
int mpdpft_write_field_files(mpdpft_ctx* ctx, const char* v_path, const char* den_path);

/* Start potentials from an mpDPFT_V.dat of any grid (the InterpolVQ = 1
 * restart, LoadV mpDPFT.cpp:6445-6499): the file's n^D points (x-major,
 * D coordinates then S values per line) are interpolated trilinearly (2D:
 * bilinearly) onto this context's grid on the GPU, the outermost cells
 * continued linearly beyond the file's box, and written to v_out[s] (the
 * caller passes them to mpdpft_sc_run as v0).  *n_file receives n.  The
 * file's species count must equal the context's. */
int mpdpft_interpolate_v_file(mpdpft_ctx* ctx, const char* path, double* const* v_out, int layout, int mem,
                              int* n_file);

/* Batch: many independent SC solves advanced together on one GPU (a
 * parameter sweep, the reference's TaskType 5/6/7 loops of GetData,
 * mpDPFTmain.cpp:110-160, run as one job).  The solves share dimension 2,
 * species count, precision, density functional (MPDPFT_DENS_GRADIENT),
 * Pulay window and the interaction list (pointwise terms only); grid sizes,
 * abundances, couplings, temperatures and potentials may differ.  Each
 * iteration of all unfinished solves is one CUDA graph replay; a solve that
 * has met its exit test does no further work.  Results equal those of
 * mpdpft_sc_run on each solve alone.
 *   params:  count parameter sets
 *   v0:      count * species starting potentials, v0[i * species + s], or NULL
 *   results: count records; status: count per-solve status codes (may be NULL) */
int mpdpft_batch_create(const mpdpft_params* params, int count, int device, mpdpft_batch** out);
int mpdpft_batch_destroy(mpdpft_batch* batch);
int mpdpft_batch_set_external_potential(mpdpft_batch* batch, int i, int s, const double* v_ext,
                                        int layout, int mem);
int mpdpft_batch_sc_init(mpdpft_batch* batch, const double* const* v0, int layout, int mem);
int mpdpft_batch_sc_step(mpdpft_batch* batch, int iterations);
int mpdpft_batch_sc_run(mpdpft_batch* batch, const double* const* v0, int layout, int mem,
                        mpdpft_result* results, int* status);
int mpdpft_batch_get_field(mpdpft_batch* batch, int i, int which, int s, double* out, int layout,
                           int mem);
int mpdpft_batch_get_log(mpdpft_batch* batch, int i, mpdpft_iter_log* log, int log_cap, int* n_out);
int mpdpft_batch_sync(mpdpft_batch* batch);

#ifdef __cplusplus
}
#endif
#endif /* MPDPFT_GPU_H */
