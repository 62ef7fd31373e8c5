"""ctypes mirror of include/mpdpft_gpu.h (ABI version 2).

Only declarations live here: the parameter, result and log structs, the
status codes and the enum values.  ``mpdpft_b200.engine`` binds the CUDA
library against these declarations.
"""
import ctypes as C

ABI_VERSION = 2
MAX_SPECIES = 4
MAX_INTERACTIONS = 8
MAX_PULAY = 12

OK = 0
ERR_ARG = 1
ERR_CUDA = 2
ERR_NONFINITE = 3
ERR_MU_BRACKET = 4
ERR_PULAY_SINGULAR = 5
ERR_TIMEOUT = 6
ERR_NOT_CONVERGED = 7
ERR_NO_DEVICE = 8
WARN_MU_TRAPPED = 9  # status_bits only

FP64 = 0
MIXED = 1
LAYOUT_PERIODIC = 0
LAYOUT_REFERENCE = 1
MEM_HOST = 0
MEM_DEVICE = 1

DENS_TF_INSPIRED = 1
DENS_TF_INSPIRED_T = 2
DENS_GRADIENT = 5
DENS_TF = 7

INT_NONE = 0
INT_CONTACT_MUTUAL = 1
INT_HARTREE = 8
INT_CONTACT_SELF = 10
INT_DIRAC = 11
INT_HARTREE_INTER = 21
INT_COULOMB_CHARGED = 100

COULOMB_REGULARISED = 0
COULOMB_TRUNCATED = 1

GRADIENT_T0 = 0
GRADIENT_FINITE_T = 1

FIELD_DENSITY = 0
FIELD_POTENTIAL = 1
FIELD_GRAD2 = 2
FIELD_LAPLACIAN = 3
FIELD_EXTERNAL = 4

STAGE_SC_STEP = 0
STAGE_FFT_Z_R2C = 1
STAGE_FFT_Y = 2
STAGE_FFT_X = 3
STAGE_FFT_Z_C2R = 4
STAGE_ITERATION = 5
STAGE_SC_MU = 6
STAGE_SC_DENSITY = 7
STAGE_SC_MIX = 8
STAGE_FFT_PLANE_FWD = 9
STAGE_FFT_PLANE_INV = 10

_D4 = C.c_double * MAX_SPECIES


class Params(C.Structure):
    _fields_ = [
        ("dim", C.c_int),
        ("steps", C.c_int),
        ("species", C.c_int),
        ("edge", C.c_double),
        ("abundances", _D4),
        ("rel_acc", C.c_double),
        ("density_expression", C.c_int),
        ("tau", _D4),
        ("temperature", _D4),
        ("n_interactions", C.c_int),
        ("interactions", C.c_int * MAX_INTERACTIONS),
        ("incremental_v", C.c_double),
        ("mu", _D4),
        ("deltamu_modifier", C.c_double),
        ("mixer", C.c_int),
        ("pulay_scope", C.c_int),
        ("theta", _D4),
        ("sc_criterion", C.c_double),
        ("max_sc_count", C.c_int),
        ("schedule", C.c_int),
        ("beta", C.c_double),
        ("gamma_h", C.c_double),
        ("degeneracy", C.c_double),
        ("regularization_threshold", C.c_double),
        ("taper_off", C.c_int),
        ("smearing_extent", C.c_double),
        ("charges", _D4),
        ("coulomb_kernel", C.c_int),
        ("coulomb_cutoff", C.c_double),
        ("gradient_floor", C.c_double),
        ("gradient_grad2", C.c_double),
        ("potential_tol", C.c_double),
        ("precision", C.c_int),
        ("gradient_form", C.c_int),
        ("airy_threshold", C.c_double),
        ("boole_pairs", C.c_int),
        ("boole_max_iter", C.c_int),
        ("internal_acc", C.c_double),
    ]

    def grid_points(self, layout=LAYOUT_PERIODIC):
        n = self.steps + (1 if layout == LAYOUT_REFERENCE else 0)
        return n ** self.dim

    def copy(self):
        other = Params()
        C.memmove(C.byref(other), C.byref(self), C.sizeof(Params))
        return other


class IterLog(C.Structure):
    _fields_ = [
        ("sc_count", C.c_int),
        ("mu_trials", C.c_int),
        ("pulay_used", C.c_int),
        ("status_bits", C.c_int),
        ("cc", C.c_double),
        ("v_residual", C.c_double),
        ("mu", _D4),
        ("abundance", _D4),
        ("theta", _D4),
        ("ms", C.c_double),
    ]


class Result(C.Structure):
    _fields_ = [
        ("iterations", C.c_int),
        ("converged", C.c_int),
        ("total_mu_trials", C.c_int),
        ("device_loop", C.c_int),
        ("cc", C.c_double),
        ("v_residual", C.c_double),
        ("mu", _D4),
        ("abundance", _D4),
        ("e_total", C.c_double),
        ("e_kinetic", _D4),
        ("e_external", _D4),
        ("e_interaction", C.c_double * MAX_INTERACTIONS),
        ("seconds", C.c_double),
    ]


INPUT_MAX_VEC = 16
_DV = C.c_double * INPUT_MAX_VEC
_IV = C.c_int * INPUT_MAX_VEC


class Input(C.Structure):
    """mpdpft_input: the 47 lines of mpDPFT.input (numbered from 0)."""
    _fields_ = [
        ("system", C.c_int), ("symmetry", C.c_int), ("task_type", C.c_int), ("task_parameter_count", C.c_int),
        ("n_task_hyperbox", C.c_int), ("task_hyperbox", _DV),
        ("dim", C.c_int), ("units", C.c_int), ("edge", C.c_double), ("steps", C.c_int), ("species", C.c_int),
        ("abundances", _D4), ("rel_acc", C.c_double), ("internal_acc", C.c_double), ("k_resources", C.c_int),
        ("density_expression", C.c_int),
        ("n_mpp", C.c_int), ("mpp", _DV), ("n_Mpp", C.c_int), ("Mpp", _DV),
        ("tau", _D4), ("territory", _D4), ("temperature", _D4), ("environments", C.c_int * MAX_SPECIES),
        ("stretchfactor", C.c_double), ("wall", C.c_double), ("noise", C.c_double), ("interpol_vq", C.c_int),
        ("n_interactions", C.c_int), ("interactions", _IV),
        ("incremental_v", C.c_double), ("mu", _D4), ("deltamu_modifier", C.c_double), ("mixer", C.c_double * 3),
        ("theta", _D4), ("sc_criterion", C.c_double), ("max_sc_count", C.c_int), ("method", C.c_int),
        ("delfield_method", C.c_int), ("movie", C.c_int),
        ("n_schedule", C.c_int), ("schedule", _IV), ("n_ekin_types", C.c_int), ("ekin_types", _IV),
        ("alpha", C.c_double), ("beta", C.c_double), ("gamma", C.c_double), ("gamma_h", C.c_double),
        ("degeneracy", C.c_double), ("n_regularize", C.c_int), ("regularize", _IV),
        ("regularization_threshold", C.c_double), ("print", C.c_int), ("lines", C.c_int),
    ]


class LaunchRecord(C.Structure):
    _fields_ = [
        ("name", C.c_char * 32),
        ("ms", C.c_double),
        ("bytes", C.c_double),
    ]


def make_params(**kw):
    """Params with the reference defaults, overridden by keyword arguments.

    Defaults follow the sample mpDPFT.input and the hard-coded values of
    InitializeHardCodedParameters (mpDPFT.cpp:858-1115).  Array fields accept
    Python sequences.
    """
    p = Params()
    p.dim = 3
    p.steps = 64
    p.species = 1
    p.edge = 16.0
    p.rel_acc = 1.0e-10
    p.density_expression = DENS_TF
    for s in range(MAX_SPECIES):
        p.abundances[s] = 1.0
        p.tau[s] = 1.0
        p.temperature[s] = 1.0
        p.mu[s] = 5.5
        p.theta[s] = 0.3
        p.charges[s] = 1.0
    p.n_interactions = 0
    p.incremental_v = 1.0
    p.deltamu_modifier = -3.0
    p.mixer = 1
    p.pulay_scope = 5
    p.sc_criterion = 1.0e-12
    p.max_sc_count = 200
    p.schedule = 0
    p.beta = 0.0
    p.gamma_h = 0.0
    p.degeneracy = 1.0
    p.regularization_threshold = 0.375
    p.taper_off = 1
    p.smearing_extent = 0.0
    p.coulomb_kernel = COULOMB_REGULARISED
    p.coulomb_cutoff = 0.0
    p.gradient_floor = 1.0e-3
    p.gradient_grad2 = 0.0
    p.potential_tol = 0.0
    p.precision = FP64
    p.gradient_form = GRADIENT_T0
    p.airy_threshold = 1.0e-6
    p.boole_pairs = 1
    p.boole_max_iter = 1
    p.internal_acc = 0.01
    for key, val in kw.items():
        if key == "interactions":
            p.n_interactions = len(val)
            for i, v in enumerate(val):
                p.interactions[i] = int(v)
            continue
        field = getattr(p, key)
        if isinstance(field, C.Array):
            for i, v in enumerate(val):
                field[i] = v
        else:
            setattr(p, key, val)
    return p
