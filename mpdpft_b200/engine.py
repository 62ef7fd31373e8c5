"""ctypes binding of libmpdpft_b200.so (the C ABI of include/mpdpft_gpu.h).

This is the harness-side host layer: it names the operators after the
reference functions they replace (GetDensity, getVint, EnforceConstraints,
DelField, fftParallel, Integrate, AdmixDensities, GetData loop) and raises
MpdpftError with the library's message when a call returns a non-zero
status.  There is no fallback: if the CUDA library is missing or no sm_100
device is present, construction fails.
"""
import ctypes as C
import os

import numpy as np

from . import abi

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libmpdpft_b200.so")

_dp = C.POINTER(C.c_double)
_dpp = C.POINTER(_dp)
_lib = None

EXPORTS = [
    "mpdpft_params_default", "mpdpft_abi_version", "mpdpft_struct_size", "mpdpft_last_error",
    "mpdpft_status_string",
    "mpdpft_ctx_create", "mpdpft_ctx_destroy", "mpdpft_ctx_sync", "mpdpft_ctx_stream",
    "mpdpft_set_external_potential", "mpdpft_density", "mpdpft_vint", "mpdpft_update_v",
    "mpdpft_mu_search", "mpdpft_delfield", "mpdpft_fft", "mpdpft_integrate", "mpdpft_pulay_reset",
    "mpdpft_admix", "mpdpft_sc_run", "mpdpft_sc_step", "mpdpft_sc_init", "mpdpft_get_field",
    "mpdpft_energy", "mpdpft_profile_stage", "mpdpft_iteration_launches", "mpdpft_step_phase_times",
    "mpdpft_batch_create", "mpdpft_batch_destroy", "mpdpft_batch_set_external_potential", "mpdpft_batch_sc_init",
    "mpdpft_batch_sc_step", "mpdpft_batch_sc_run", "mpdpft_batch_get_field", "mpdpft_batch_get_log",
    "mpdpft_batch_sync", "mpdpft_adjoint", "mpdpft_adjoint_nuclei", "mpdpft_fft_config", "mpdpft_fft_tiles",
    "mpdpft_set_limits", "mpdpft_integrate_noalloc", "mpdpft_iteration_profile",
    "mpdpft_read_input", "mpdpft_params_from_input", "mpdpft_write_field_files", "mpdpft_interpolate_v_file",
]


class MpdpftError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__("%s (status %d): %s" % (_status_name(status), status, msg))
        self.status = status


def _status_name(st):
    names = {v: k for k, v in vars(abi).items() if k.startswith("ERR_") or k == "OK"}
    return names.get(st, "status")


def load(path=LIB_PATH):
    """Load the CUDA library; raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise MpdpftError(abi.ERR_NO_DEVICE, "CUDA library %s not built (python -m mpdpft_b200.build)" % path)
    L = C.CDLL(path)
    P = C.POINTER(abi.Params)
    vp = C.c_void_p
    L.mpdpft_params_default.argtypes = [P]
    L.mpdpft_params_default.restype = None
    L.mpdpft_abi_version.restype = C.c_int
    L.mpdpft_last_error.restype = C.c_char_p
    L.mpdpft_status_string.restype = C.c_char_p
    L.mpdpft_status_string.argtypes = [C.c_int]
    L.mpdpft_ctx_create.argtypes = [P, C.c_int, C.POINTER(vp)]
    L.mpdpft_ctx_destroy.argtypes = [vp]
    L.mpdpft_ctx_sync.argtypes = [vp]
    L.mpdpft_ctx_stream.argtypes = [vp]
    L.mpdpft_ctx_stream.restype = vp
    L.mpdpft_set_limits.argtypes = [vp, C.c_int, C.c_longlong]
    L.mpdpft_iteration_profile.argtypes = [vp, C.c_int, C.POINTER(abi.LaunchRecord), C.POINTER(C.c_int)]
    L.mpdpft_read_input.argtypes = [C.c_char_p, C.POINTER(abi.Input)]
    L.mpdpft_params_from_input.argtypes = [C.POINTER(abi.Input), P]
    L.mpdpft_write_field_files.argtypes = [vp, C.c_char_p, C.c_char_p]
    L.mpdpft_interpolate_v_file.argtypes = [vp, C.c_char_p, _dpp, C.c_int, C.c_int, C.POINTER(C.c_int)]
    L.mpdpft_set_external_potential.argtypes = [vp, C.c_int, _dp, C.c_int, C.c_int]
    L.mpdpft_density.argtypes = [vp, C.c_int, _dp, C.c_double, _dp, _dp, C.c_int, C.c_int]
    L.mpdpft_vint.argtypes = [vp, C.c_int, C.c_int, _dpp, _dp, C.c_int, C.c_int]
    L.mpdpft_update_v.argtypes = [vp, _dpp, C.c_double, _dpp, C.c_int, C.c_int]
    L.mpdpft_mu_search.argtypes = [vp, C.c_int, _dp, C.c_double, _dp, _dp, C.POINTER(C.c_int), _dp,
                                   C.c_int, C.c_int]
    L.mpdpft_delfield.argtypes = [vp, _dp, _dp, _dp, C.c_int, C.c_int]
    L.mpdpft_fft.argtypes = [vp, C.c_int, _dp, _dp, C.c_int]
    L.mpdpft_integrate.argtypes = [vp, _dp, _dp, C.c_int, C.c_int]
    L.mpdpft_pulay_reset.argtypes = [vp]
    L.mpdpft_admix.argtypes = [vp, _dpp, _dpp, _dp, _dpp, _dp, C.POINTER(C.c_int), C.c_int, C.c_int]
    L.mpdpft_sc_run.argtypes = [vp, _dpp, C.c_int, C.c_int, C.POINTER(abi.Result), C.POINTER(abi.IterLog), C.c_int]
    L.mpdpft_sc_step.argtypes = [vp, C.c_int, C.POINTER(abi.IterLog)]
    L.mpdpft_sc_init.argtypes = [vp, _dpp, C.c_int, C.c_int]
    L.mpdpft_get_field.argtypes = [vp, C.c_int, C.c_int, _dp, C.c_int, C.c_int]
    L.mpdpft_energy.argtypes = [vp, C.POINTER(abi.Result)]
    L.mpdpft_profile_stage.argtypes = [vp, C.c_int, C.c_int, _dp, _dp]
    L.mpdpft_iteration_launches.argtypes = [vp, C.POINTER(C.c_int), C.POINTER(C.c_int)]
    L.mpdpft_step_phase_times.argtypes = [vp, _dp, C.c_int]
    L.mpdpft_batch_create.argtypes = [P, C.c_int, C.c_int, C.POINTER(vp)]
    L.mpdpft_batch_destroy.argtypes = [vp]
    L.mpdpft_batch_set_external_potential.argtypes = [vp, C.c_int, C.c_int, _dp, C.c_int, C.c_int]
    L.mpdpft_batch_sc_init.argtypes = [vp, _dpp, C.c_int, C.c_int]
    L.mpdpft_batch_sc_step.argtypes = [vp, C.c_int]
    L.mpdpft_batch_sc_run.argtypes = [vp, _dpp, C.c_int, C.c_int, C.POINTER(abi.Result), C.POINTER(C.c_int)]
    L.mpdpft_batch_get_field.argtypes = [vp, C.c_int, C.c_int, C.c_int, _dp, C.c_int, C.c_int]
    L.mpdpft_batch_get_log.argtypes = [vp, C.c_int, C.POINTER(abi.IterLog), C.c_int, C.POINTER(C.c_int)]
    L.mpdpft_batch_sync.argtypes = [vp]
    L.mpdpft_fft_config.argtypes = [vp, C.POINTER(C.c_int), _dp, _dp, C.POINTER(C.c_int)]
    L.mpdpft_fft_tiles.argtypes = [vp, C.POINTER(C.c_int), C.POINTER(C.c_int)]
    L.mpdpft_adjoint.argtypes = [vp, _dp, _dp, C.c_int, C.c_int, C.c_double, C.c_int, C.POINTER(C.c_int), _dp]
    L.mpdpft_adjoint_nuclei.argtypes = [vp, _dp, C.c_int, C.c_int, _dp, _dp, C.c_double, _dp]
    for name in EXPORTS:
        getattr(L, name)
    _lib = L
    return L


def _arr(x, n=None):
    a = np.ascontiguousarray(np.asarray(x, dtype=np.float64).reshape(-1))
    if n is not None and a.size != n:
        raise ValueError("expected %d values, got %d" % (n, a.size))
    return a


def _ptr(a):
    return a.ctypes.data_as(_dp)


def _ptrs(arrays):
    return (_dp * len(arrays))(*[_ptr(a) for a in arrays])


def _check_lib(L, st):
    if st != abi.OK:
        raise MpdpftError(st, L.mpdpft_last_error().decode())


def read_input(path):
    """Parse an mpDPFT.input file (GetInputParameters): abi.Input.  Host
    code only; needs no GPU."""
    L = load()
    inp = abi.Input()
    _check_lib(L, L.mpdpft_read_input(os.fsencode(path), C.byref(inp)))
    return inp


def params_from_input(inp):
    """Engine parameters of a parsed mpDPFT.input (abi.Params); raises on
    options the engine does not implement."""
    L = load()
    p = abi.Params()
    _check_lib(L, L.mpdpft_params_from_input(C.byref(inp), C.byref(p)))
    return p


class Engine:
    """One SC solve context on one GPU (mpdpft_ctx)."""

    def __init__(self, params, device=0):
        self.lib = load()
        self.params = params.copy()
        h = C.c_void_p()
        self._check(self.lib.mpdpft_ctx_create(C.byref(self.params), device, C.byref(h)))
        self.h = h
        self.S = params.species
        self.n = params.steps ** params.dim

    def _check(self, st):
        if st != abi.OK:
            raise MpdpftError(st, self.lib.mpdpft_last_error().decode())
        return st

    def close(self):
        if getattr(self, "h", None):
            self.lib.mpdpft_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _count(self, layout):
        return self.params.grid_points(layout)

    # --- operators ------------------------------------------------------
    def set_external_potential(self, s, vext, layout=abi.LAYOUT_PERIODIC):
        a = _arr(vext, self._count(layout))
        self._check(self.lib.mpdpft_set_external_potential(self.h, s, _ptr(a), layout, abi.MEM_HOST))

    def GetDensity(self, s, v, mu, layout=abi.LAYOUT_PERIODIC):
        """n[V] at mu and N = Integrate(n)."""
        a = _arr(v, self._count(layout))
        out = np.empty(self._count(layout))
        N = C.c_double()
        self._check(self.lib.mpdpft_density(self.h, s, _ptr(a), mu, _ptr(out), C.byref(N), layout, abi.MEM_HOST))
        return out, N.value

    def getVint(self, type_, s, dens, layout=abi.LAYOUT_PERIODIC):
        arrs = [_arr(d, self._count(layout)) for d in dens]
        out = np.empty(self._count(layout))
        self._check(self.lib.mpdpft_vint(self.h, type_, s, _ptrs(arrs), _ptr(out), layout, abi.MEM_HOST))
        return out

    def UpdateV(self, dens, incremental=1.0, layout=abi.LAYOUT_PERIODIC):
        arrs = [_arr(d, self._count(layout)) for d in dens]
        outs = [np.empty(self._count(layout)) for _ in range(self.S)]
        self._check(self.lib.mpdpft_update_v(self.h, _ptrs(arrs), incremental, _ptrs(outs), layout, abi.MEM_HOST))
        return outs

    def EnforceConstraints(self, s, v, n_target, mu, layout=abi.LAYOUT_PERIODIC, check=True):
        a = _arr(v, self._count(layout))
        mu_io = C.c_double(mu)
        N = C.c_double()
        tr = C.c_int()
        out = np.empty(self._count(layout))
        st = self.lib.mpdpft_mu_search(self.h, s, _ptr(a), n_target, C.byref(mu_io), C.byref(N), C.byref(tr),
                                       _ptr(out), layout, abi.MEM_HOST)
        if check and st != abi.WARN_MU_TRAPPED:  # a trapped search is the reference's result, not an error
            self._check(st)
        return mu_io.value, N.value, tr.value, out, st

    def DelField(self, f, layout=abi.LAYOUT_PERIODIC):
        a = _arr(f, self._count(layout))
        g2 = np.empty(self._count(layout))
        lap = np.empty(self._count(layout))
        self._check(self.lib.mpdpft_delfield(self.h, _ptr(a), _ptr(g2), _ptr(lap), layout, abi.MEM_HOST))
        return g2, lap

    def fftParallel(self, sign, field):
        f = np.asarray(field, dtype=np.complex128).reshape(-1)
        if f.size != self.n:
            raise ValueError("field size")
        buf = np.ascontiguousarray(np.stack([f.real, f.imag], axis=-1).reshape(-1))
        out = np.empty_like(buf)
        self._check(self.lib.mpdpft_fft(self.h, sign, _ptr(buf), _ptr(out), abi.MEM_HOST))
        return out[0::2] + 1j * out[1::2]

    def Integrate(self, f, layout=abi.LAYOUT_PERIODIC):
        a = _arr(f, self._count(layout))
        out = C.c_double()
        self._check(self.lib.mpdpft_integrate(self.h, _ptr(a), C.byref(out), layout, abi.MEM_HOST))
        return out.value

    def PulayReset(self):
        self._check(self.lib.mpdpft_pulay_reset(self.h))

    def AdmixDensities(self, n_in, n_out, theta=None, layout=abi.LAYOUT_PERIODIC, check=True):
        ai = [_arr(x, self._count(layout)) for x in n_in]
        ao = [_arr(x, self._count(layout)) for x in n_out]
        outs = [np.empty(self._count(layout)) for _ in range(self.S)]
        th = None if theta is None else _arr(theta)
        coeffs = np.zeros(abi.MAX_PULAY)
        nc = C.c_int(0)
        st = self.lib.mpdpft_admix(self.h, _ptrs(ai), _ptrs(ao), None if th is None else _ptr(th), _ptrs(outs),
                                   _ptr(coeffs), C.byref(nc), layout, abi.MEM_HOST)
        if check and st not in (abi.OK, abi.ERR_PULAY_SINGULAR):
            self._check(st)
        return outs, coeffs[:nc.value].copy(), st

    # --- SC loop ----------------------------------------------------------
    def sc_run(self, vext, v0=None, layout=abi.LAYOUT_PERIODIC, log_cap=None, check=True, device_v0=None):
        """Full solve.  vext (None: keep the potentials already set);
        device_v0: optional device addresses of float64 start potentials
        (periodic layout) in place of the host arrays v0."""
        if vext is not None:
            for s in range(self.S):
                self.set_external_potential(s, vext[s], layout)
        v0p, mem = None, abi.MEM_HOST
        if device_v0 is not None:
            v0p, mem = (_dp * len(device_v0))(*[C.cast(C.c_void_p(a), _dp) for a in device_v0]), abi.MEM_DEVICE
        elif v0 is not None:
            arrs = [_arr(x, self._count(layout)) for x in v0]
            self._keep = arrs
            v0p = _ptrs(arrs)
        cap = log_cap or (self.params.max_sc_count + 2)
        res = abi.Result()
        log = (abi.IterLog * cap)()
        st = self.lib.mpdpft_sc_run(self.h, v0p, layout, mem, C.byref(res), log, cap)
        if check and st not in (abi.OK, abi.ERR_NOT_CONVERGED):
            self._check(st)
        return res, list(log[:min(res.iterations, cap)]), st

    def sc_init(self, vext, v0=None, layout=abi.LAYOUT_PERIODIC):
        for s in range(self.S):
            self.set_external_potential(s, vext[s], layout)
        v0p = None
        if v0 is not None:
            arrs = [_arr(x, self._count(layout)) for x in v0]
            self._keep = arrs
            v0p = _ptrs(arrs)
        self._check(self.lib.mpdpft_sc_init(self.h, v0p, layout, abi.MEM_HOST))

    def sc_step(self, graph=True, want_log=False):
        log = abi.IterLog()
        self._check(self.lib.mpdpft_sc_step(self.h, 1 if graph else 0, C.byref(log) if want_log else None))
        return log if want_log else None

    def sync(self):
        self._check(self.lib.mpdpft_ctx_sync(self.h))

    def set_limits(self, mu_max_passes=-1, barrier_spin_limit=-1):
        """Device loop limits (negative: defaults)."""
        self._check(self.lib.mpdpft_set_limits(self.h, mu_max_passes, barrier_spin_limit))

    def stream(self):
        return self.lib.mpdpft_ctx_stream(self.h)

    def field(self, which, s, layout=abi.LAYOUT_PERIODIC, out=None):
        """One field of the current state as float64 (into `out`, a
        contiguous float64 array of the grid's size, when given)."""
        if out is None:
            out = np.empty(self._count(layout))
        elif out.dtype != np.float64 or out.size != self._count(layout) or not out.flags["C_CONTIGUOUS"]:
            raise ValueError("out must be a contiguous float64 array of the grid's size")
        self._check(self.lib.mpdpft_get_field(self.h, which, s, _ptr(out), layout, abi.MEM_HOST))
        return out

    def profile_stage(self, stage, reps=20):
        """(ms per launch, algorithmic bytes per launch) of one stage."""
        ms = C.c_double()
        b = C.c_double()
        self._check(self.lib.mpdpft_profile_stage(self.h, stage, reps, C.byref(ms), C.byref(b)))
        return ms.value, b.value

    def _launches(self):
        counts = (C.c_int * 6)()
        total = C.c_int()
        self._check(self.lib.mpdpft_iteration_launches(self.h, counts, C.byref(total)))
        return list(counts), total.value

    def iteration_kernels(self):
        """Kernel launches in one captured SC iteration."""
        return self._launches()[1]

    def stage_launch_counts(self):
        c, _ = self._launches()
        return {"sc_step": c[0], "z_r2c": c[1], "y": c[2], "x": c[3], "z_c2r": c[4], "other": c[5]}

    def write_field_files(self, v_path=None, den_path=None):
        """mpDPFT_V.dat / mpDPFT_Den.dat of the current state (ExportData)."""
        self._check(self.lib.mpdpft_write_field_files(self.h, None if v_path is None else os.fsencode(v_path),
                                                      None if den_path is None else os.fsencode(den_path)))

    def interpolate_v_file(self, path, layout=abi.LAYOUT_PERIODIC):
        """Start potentials interpolated from an mpDPFT_V.dat of any grid
        (InterpolVQ = 1): ([V_s], n of the file)."""
        outs = [np.empty(self._count(layout)) for _ in range(self.S)]
        n = C.c_int()
        self._check(self.lib.mpdpft_interpolate_v_file(self.h, os.fsencode(path), _ptrs(outs), layout, abi.MEM_HOST,
                                                       C.byref(n)))
        return outs, n.value

    def iteration_profile(self, cap=256):
        """One SC iteration replayed launch by launch from its CUDA graph:
        [(kernel name, ms, algorithmic bytes)] in issue order."""
        recs = (abi.LaunchRecord * cap)()
        n = C.c_int()
        self._check(self.lib.mpdpft_iteration_profile(self.h, cap, recs, C.byref(n)))
        return [(r.name.decode(), r.ms, r.bytes) for r in recs[:min(n.value, cap)]]

    def step_phase_times(self):
        """Phase durations (us) of the last SC-step kernel: V update, mu
        search, densities/Gram, solve, barrier, mix."""
        us = np.zeros(6)
        self._check(self.lib.mpdpft_step_phase_times(self.h, _ptr(us), 6))
        return us

    def fft_config(self):
        """(path, ms_plane, ms_pass, how) of the FFT autotuner: path 1 x-plane
        kernels, 0 pass kernels; how 0 one path, 1 measured, 2 cached, 3 forced."""
        path, how = C.c_int(), C.c_int()
        a, b = C.c_double(), C.c_double()
        self._check(self.lib.mpdpft_fft_config(self.h, C.byref(path), C.byref(a), C.byref(b), C.byref(how)))
        return path.value, a.value, b.value, how.value

    def fft_tiles(self):
        """(lines per tile of the Y/X passes, rows per block of the Z passes)
        the FFT autotuner chose."""
        t, z = C.c_int(), C.c_int()
        self._check(self.lib.mpdpft_fft_tiles(self.h, C.byref(t), C.byref(z)))
        return t.value, z.value

    def adjoint(self, dl_dn, tol=1e-10, max_iter=300, check=True):
        """dL/dV_ext of the converged solve for dL/dn (periodic layout):
        (gradient, iterations, residual, status)."""
        g = _arr(dl_dn, self.n)
        out = np.empty(self.n)
        it = C.c_int()
        res = C.c_double()
        st = self.lib.mpdpft_adjoint(self.h, _ptr(g), _ptr(out), abi.LAYOUT_PERIODIC, abi.MEM_HOST, tol, max_iter,
                                     C.byref(it), C.byref(res))
        if check and st != abi.OK:
            self._check(st)
        return out, it.value, res.value, st

    def adjoint_nuclei(self, dl_dvext, z, pos, sigma):
        """dL/dR (n_nuclei x 3) of Gaussian nuclei from dL/dV_ext."""
        g = _arr(dl_dvext, self.n)
        zz = _arr(z)
        pp = _arr(pos)
        out = np.empty(pp.size)
        self._check(self.lib.mpdpft_adjoint_nuclei(self.h, _ptr(g), abi.MEM_HOST, zz.size, _ptr(zz), _ptr(pp),
                                                   sigma, _ptr(out)))
        return out.reshape(-1, 3)

    def energy(self):
        r = abi.Result()
        self._check(self.lib.mpdpft_energy(self.h, C.byref(r)))
        return r


class Batch:
    """Many independent 2D SC solves advanced together (mpdpft_batch).

    problems: list of (params, vext list, v0 list) as the workload builders
    return them.  sc_run() returns (results, statuses)."""

    def __init__(self, problems, device=0):
        self.lib = load()
        self.problems = problems
        self.count = len(problems)
        self.S = problems[0][0].species
        params = (abi.Params * self.count)(*[p for p, _, _ in problems])
        h = C.c_void_p()
        st = self.lib.mpdpft_batch_create(params, self.count, device, C.byref(h))
        if st != abi.OK:
            raise MpdpftError(st, self.lib.mpdpft_last_error().decode())
        self.h = h
        for i, (p, vext, _) in enumerate(problems):
            for s in range(self.S):
                a = _arr(vext[s], p.grid_points(abi.LAYOUT_PERIODIC))
                self._check(self.lib.mpdpft_batch_set_external_potential(self.h, i, s, _ptr(a),
                                                                         abi.LAYOUT_PERIODIC, abi.MEM_HOST))

    def _check(self, st):
        if st != abi.OK:
            raise MpdpftError(st, self.lib.mpdpft_last_error().decode())

    def close(self):
        if getattr(self, "h", None):
            self.lib.mpdpft_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _v0(self):
        arrs = []
        for p, _, v0 in self.problems:
            for s in range(self.S):
                arrs.append(_arr(v0[s], p.grid_points(abi.LAYOUT_PERIODIC)))
        self._keep = arrs
        return _ptrs(arrs)

    def sc_init(self):
        self._check(self.lib.mpdpft_batch_sc_init(self.h, self._v0(), abi.LAYOUT_PERIODIC, abi.MEM_HOST))

    def sc_step(self, iterations=1):
        self._check(self.lib.mpdpft_batch_sc_step(self.h, iterations))

    def sync(self):
        self._check(self.lib.mpdpft_batch_sync(self.h))

    def sc_run(self, check=True, device_v0=None):
        """Initialise and solve all; device_v0: optional count * species
        device addresses of float64 start potentials (periodic layout), in
        place of the host arrays of the problems."""
        res = (abi.Result * self.count)()
        status = (C.c_int * self.count)()
        if device_v0 is None:
            v0, mem = self._v0(), abi.MEM_HOST
        else:
            v0, mem = (_dp * len(device_v0))(*[C.cast(C.c_void_p(a), _dp) for a in device_v0]), abi.MEM_DEVICE
        st = self.lib.mpdpft_batch_sc_run(self.h, v0, abi.LAYOUT_PERIODIC, mem, res, status)
        if check and st not in (abi.OK, abi.ERR_NOT_CONVERGED):
            self._check(st)
        return list(res), list(status)

    def field(self, i, which, s, layout=abi.LAYOUT_PERIODIC):
        p = self.problems[i][0]
        out = np.empty(p.grid_points(layout))
        self._check(self.lib.mpdpft_batch_get_field(self.h, i, which, s, _ptr(out), layout, abi.MEM_HOST))
        return out

    def log(self, i, cap=None):
        cap = cap or (self.problems[i][0].max_sc_count + 2)
        buf = (abi.IterLog * cap)()
        n = C.c_int()
        self._check(self.lib.mpdpft_batch_get_log(self.h, i, buf, cap, C.byref(n)))
        return list(buf[:n.value])
