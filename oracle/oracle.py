"""Python binding of the CPU oracle (test infrastructure only).

The oracle is the checker for the parity tests, the smoke check and the CPU
baseline of bench.py; nothing in the product imports this module.  Inputs
and outputs are periodic s^D numpy arrays; the binding expands them to the
reference's (s+1)^D layout, which the oracle computes on, and drops the
duplicate planes of the results (they are copies of plane 0).
"""
import ctypes as C
import os
import subprocess

import numpy as np

from mpdpft_b200 import abi
from mpdpft_b200.workloads import to_periodic, to_reference

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
_lib = None

_dp = C.POINTER(C.c_double)


def build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        P = C.POINTER(abi.Params)
        L.oracle_fft.argtypes = [P, C.c_int, _dp]
        L.oracle_fft_raw.argtypes = [C.c_int, C.c_int, C.c_int, _dp]
        L.oracle_integrate.argtypes = [P, _dp]
        L.oracle_integrate.restype = C.c_double
        L.oracle_delfield.argtypes = [P, _dp, _dp, _dp]
        L.oracle_density.argtypes = [P, C.c_int, _dp, C.c_double, _dp]
        L.oracle_density.restype = C.c_double
        L.oracle_vint.argtypes = [P, C.c_int, C.c_int, _dp, _dp]
        L.oracle_mu_search.argtypes = [P, _dp, _dp, _dp, _dp, _dp]
        L.oracle_mu_search.restype = C.c_int
        L.oracle_last_status_bits.restype = C.c_int
        L.oracle_sc_run.argtypes = [P, _dp, _dp, C.POINTER(abi.Result), C.POINTER(abi.IterLog),
                                    C.c_int, _dp, _dp]
        L.oracle_sc_run.restype = C.c_int
        L.oracle_energy.argtypes = [P, _dp, _dp, _dp, _dp, C.POINTER(abi.Result)]
        L.oracle_pulay_sequence.argtypes = [P, C.c_int, _dp, _dp, _dp, _dp,
                                            C.POINTER(C.c_int), C.POINTER(C.c_int)]
        L.oracle_num_threads.restype = C.c_int
        L.oracle_set_threads.argtypes = [C.c_int]
        L.oracle_set_threads.restype = None
        L.oracle_polylog.argtypes = [C.c_int, C.c_double]
        L.oracle_polylog.restype = C.c_double
        L.oracle_curly_a.argtypes = [C.c_double]
        L.oracle_curly_a.restype = C.c_double
        L.oracle_i0e.argtypes = [C.c_double]
        L.oracle_i0e.restype = C.c_double
        L.oracle_airy.argtypes = [C.c_double, _dp, _dp]
        L.oracle_airy.restype = None
        L.oracle_finite_t_point.argtypes = [P, C.c_double, C.c_double, C.c_double, C.c_double]
        L.oracle_finite_t_point.restype = C.c_double
        _lib = L
    return _lib


def _ptr(a):
    return a.ctypes.data_as(_dp)


def _ref(p, f):
    return np.ascontiguousarray(to_reference(np.asarray(f, dtype=np.float64).reshape(-1), p.dim))


def _per(p, f):
    return to_periodic(f, p.dim)


def num_threads():
    return lib().oracle_num_threads()


def set_threads(n):
    """OpenMP threads of later oracle calls (0: all host threads)."""
    lib().oracle_set_threads(int(n))


FD_ORDERS = (2.5, 1.5, 0.5, -0.5, -1.5)


def polylog(s, x):
    """Li_s(-e^x) for s in FD_ORDERS (the reference's polylog())."""
    return lib().oracle_polylog(FD_ORDERS.index(s), float(x))


def curly_a(x):
    """int_x^inf Ai(t) dt (the reference's CurlyA)."""
    return lib().oracle_curly_a(float(x))


def airy(x):
    """(Ai(x), Ai'(x)) as the energies of the gradient-corrected density use them."""
    a, b = C.c_double(), C.c_double()
    lib().oracle_airy(float(x), C.byref(a), C.byref(b))
    return a.value, b.value


def i0e(x):
    """e^{-x} I0(x) of the 2D Hartree compensation term."""
    return lib().oracle_i0e(float(x))


def finite_t_point(p, T, u, lap, grad2):
    """The finite-T gradient density of species 0 at one point (u = mu - V)."""
    return lib().oracle_finite_t_point(C.byref(p), T, u, lap, grad2)


def fft(p, field, sign):
    """fftParallel on a periodic complex field (centred k, reference norms)."""
    f = np.asarray(field, dtype=np.complex128).reshape(-1)
    ref = to_reference(f, p.dim)
    buf = np.ascontiguousarray(np.stack([ref.real, ref.imag], axis=-1).reshape(-1))
    lib().oracle_fft(C.byref(p), sign, _ptr(buf))
    out = buf[0::2] + 1j * buf[1::2]
    return to_periodic(out, p.dim)


def fft_raw(dim, s, field, sign):
    f = np.asarray(field, dtype=np.complex128).reshape(-1)
    buf = np.ascontiguousarray(np.stack([f.real, f.imag], axis=-1).reshape(-1))
    lib().oracle_fft_raw(dim, s, sign, _ptr(buf))
    return buf[0::2] + 1j * buf[1::2]


def integrate(p, f):
    r = _ref(p, f)
    return lib().oracle_integrate(C.byref(p), _ptr(r))


def integrate_reference_layout(p, f_ref):
    r = np.ascontiguousarray(np.asarray(f_ref, dtype=np.float64))
    return lib().oracle_integrate(C.byref(p), _ptr(r))


def delfield(p, f):
    r = _ref(p, f)
    g2 = np.empty_like(r)
    lap = np.empty_like(r)
    lib().oracle_delfield(C.byref(p), _ptr(r), _ptr(g2), _ptr(lap))
    return _per(p, g2), _per(p, lap)


def density(p, s, v, mu):
    r = _ref(p, v)
    n = np.empty_like(r)
    N = lib().oracle_density(C.byref(p), s, _ptr(r), mu, _ptr(n))
    return _per(p, n), N


def last_status_bits():
    """Status bits of the last mu_search (1 << abi.WARN_MU_TRAPPED: the
    bisection ended on the reference's trap test)."""
    return lib().oracle_last_status_bits()


def vint(p, type_, s, dens):
    d = np.ascontiguousarray(np.concatenate([_ref(p, x) for x in dens]))
    out = np.empty(p.grid_points(abi.LAYOUT_REFERENCE))
    lib().oracle_vint(C.byref(p), type_, s, _ptr(d), _ptr(out))
    return _per(p, out)


def mu_search(p, v_list, deltamu_modifier=None):
    S = p.species
    v = np.ascontiguousarray(np.concatenate([_ref(p, x) for x in v_list]))
    G = p.grid_points(abi.LAYOUT_REFERENCE)
    mu = np.zeros(S)
    ab = np.zeros(S)
    dens = np.empty(S * G)
    dmm = np.array([p.deltamu_modifier if deltamu_modifier is None else deltamu_modifier])
    trials = lib().oracle_mu_search(C.byref(p), _ptr(v), _ptr(mu), _ptr(ab), _ptr(dens), _ptr(dmm))
    dens_p = [_per(p, dens[q * G:(q + 1) * G]) for q in range(S)]
    return mu, ab, dens_p, trials, float(dmm[0])


def sc_run(p, vext, v0=None, log_cap=2000):
    S = p.species
    G = p.grid_points(abi.LAYOUT_REFERENCE)
    ve = np.ascontiguousarray(np.concatenate([_ref(p, x) for x in vext]))
    v0r = None if v0 is None else np.ascontiguousarray(np.concatenate([_ref(p, x) for x in v0]))
    res = abi.Result()
    log = (abi.IterLog * log_cap)()
    dens = np.empty(S * G)
    vout = np.empty(S * G)
    n = lib().oracle_sc_run(C.byref(p), _ptr(ve), None if v0r is None else _ptr(v0r),
                            C.byref(res), log, log_cap, _ptr(dens), _ptr(vout))
    dens_p = [_per(p, dens[q * G:(q + 1) * G]) for q in range(S)]
    v_p = [_per(p, vout[q * G:(q + 1) * G]) for q in range(S)]
    return res, list(log[:n]), dens_p, v_p


def energy(p, vext, dens, v, mu):
    ve = np.ascontiguousarray(np.concatenate([_ref(p, x) for x in vext]))
    de = np.ascontiguousarray(np.concatenate([_ref(p, x) for x in dens]))
    vv = np.ascontiguousarray(np.concatenate([_ref(p, x) for x in v]))
    m = np.ascontiguousarray(np.asarray(mu, dtype=np.float64))
    res = abi.Result()
    lib().oracle_energy(C.byref(p), _ptr(ve), _ptr(de), _ptr(vv), _ptr(m), C.byref(res))
    return res


def pulay_sequence(p, nin_seq, nout_seq):
    """Feed pairs (n_in[t], n_out[t]) (lists over species) through
    AdmixDensities at SCcount = 0, 1, ...; returns mixed densities per step,
    the final coefficients and the Pulay-used flags."""
    T = len(nin_seq)
    S = p.species
    G = p.grid_points(abi.LAYOUT_REFERENCE)
    nin = np.ascontiguousarray(np.concatenate([_ref(p, x) for step in nin_seq for x in step]))
    nout = np.ascontiguousarray(np.concatenate([_ref(p, x) for step in nout_seq for x in step]))
    mixed = np.empty(T * S * G)
    coeffs = np.zeros(abi.MAX_PULAY + 4)
    nc = C.c_int(0)
    used = (C.c_int * T)()
    lib().oracle_pulay_sequence(C.byref(p), T, _ptr(nin), _ptr(nout), _ptr(mixed), _ptr(coeffs),
                                C.byref(nc), used)
    out = [[_per(p, mixed[(t * S + q) * G:(t * S + q + 1) * G]) for q in range(S)] for t in range(T)]
    return out, coeffs[:nc.value].copy(), list(used)


def block_sums(f, steps, dim, blocks=16):
    """Sums of a periodic s^D field over blocks^D equal coarse blocks
    (steps divisible by blocks), flattened in x-major order."""
    b = steps // blocks
    g = np.asarray(f, dtype=np.float64).reshape((blocks, b) * dim)
    return g.sum(axis=tuple(range(1, 2 * dim, 2))).reshape(-1)
