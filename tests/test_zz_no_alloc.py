"""mpdpft_integrate_noalloc: the trapezoid integral for callers that cannot
allocate device memory (a plug-in whose host application owns every device
allocation, or a loop that must not pay cudaMalloc's implicit device
synchronisation).  It takes device pointers only and keeps its partial sums
in a fixed array inside the library, so the checks here run it through the
C ABI twice in a row on the same buffers and compare each result with the
context-based mpdpft_integrate on the same field and with the oracle's
trapezoid rule (a plain sum in the periodic layout, Riemann's end weights in
the reference layout, whose test fields do not repeat plane 0 in their last
plane).  The 256^3 cases fill the whole scratch array.

This file is collected last on purpose: a failure here leaves every other
test already run.
"""
import ctypes as C

import numpy as np
import pytest

from mpdpft_b200 import abi, engine

REL_TOL = 1e-12  # FP64 sums of the same values in two summation orders


def _bind(lib):
    f = lib.mpdpft_integrate_noalloc
    f.argtypes = [C.c_int, C.c_int, C.c_double, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p]
    f.restype = C.c_int
    return f


def _field(dim, s, layout, seed):
    rng = np.random.default_rng(seed)
    m = s + 1 if layout == abi.LAYOUT_REFERENCE else s
    shape = (m,) * dim
    x = np.linspace(-1.0, 1.0, m)
    grids = np.meshgrid(*([x] * dim), indexing="ij")
    r2 = sum(g * g for g in grids)
    return (np.exp(-3.0 * r2) + 0.1 * rng.standard_normal(shape)).ravel()


def test_noalloc_rejects_grids_beyond_its_scratch():
    lib = engine.load()
    f = _bind(lib)
    fake = C.c_void_p(256)  # never dereferenced: the size check comes first
    st = f(3, 512, 10.0, fake, fake, abi.LAYOUT_PERIODIC, None)
    assert st == abi.ERR_ARG
    assert b"MPDPFT_NOALLOC_MAX_POINTS" in lib.mpdpft_last_error()
    assert f(2, 8192, 10.0, fake, fake, abi.LAYOUT_PERIODIC, None) == abi.ERR_ARG
    assert f(3, 64, 10.0, None, fake, abi.LAYOUT_PERIODIC, None) == abi.ERR_ARG


def _riemann(dim, s, edge, layout, host):
    """Trapezoid rule on the stored values (Riemann, mpDPFT.cpp:7981-8026):
    end weights 1/2 per axis in the reference layout, weight 1 on the
    periodic grid."""
    dvol = (edge / s) ** dim
    if layout != abi.LAYOUT_REFERENCE:
        return float(host.sum()) * dvol
    m = s + 1
    w = np.ones(m)
    w[0] = w[-1] = 0.5
    f = host.reshape((m,) * dim)
    if dim == 3:
        return float(np.einsum("k,ijk->ij", w, f).dot(w).dot(w)) * dvol
    return float(w.dot(f).dot(w)) * dvol


def test_noalloc_riemann_matches_oracle_reference_layout():
    """The test's trapezoid rule equals the oracle's on fields whose last
    planes differ from plane 0 (the case the reference layout must not
    shortcut), and differs from the periodic-only sum there."""
    from oracle import oracle
    for dim, s, edge in ((3, 6, 3.0), (2, 10, 4.0)):
        host = _field(dim, s, abi.LAYOUT_REFERENCE, seed=s)
        p = abi.make_params(dim=dim, steps=s, edge=edge, precision=abi.FP64)
        expect = oracle.integrate_reference_layout(p, host)
        got = _riemann(dim, s, edge, abi.LAYOUT_REFERENCE, host)
        assert abs(got - expect) <= 1e-13 * abs(expect), (got, expect)
        periodic_only = float(host.reshape((s + 1,) * dim)[(slice(0, s),) * dim].sum()) * (edge / s) ** dim
        assert abs(periodic_only - expect) > 1e-6 * abs(expect)


@pytest.mark.gpu
@pytest.mark.parametrize("dim,s,layout", [
    (3, 64, abi.LAYOUT_PERIODIC),
    (3, 48, abi.LAYOUT_REFERENCE),
    (2, 256, abi.LAYOUT_PERIODIC),
    (2, 192, abi.LAYOUT_REFERENCE),
    (3, 256, abi.LAYOUT_PERIODIC),
    (3, 256, abi.LAYOUT_REFERENCE),
])
def test_noalloc_integral_matches_context_integral_twice(dim, s, layout):
    import torch
    lib = engine.load()
    f = _bind(lib)
    edge = 12.0
    host = _field(dim, s, layout, seed=s)
    dev = torch.from_numpy(host).to("cuda:0")
    out = torch.full((1,), float("nan"), dtype=torch.float64, device="cuda:0")

    p = abi.make_params(dim=dim, steps=s, edge=edge, precision=abi.FP64)
    with engine.Engine(p) as e:
        ref = C.c_double()
        fdev = C.cast(C.c_void_p(dev.data_ptr()), C.POINTER(C.c_double))
        e._check(lib.mpdpft_integrate(e.h, fdev, C.pointer(ref), layout, abi.MEM_DEVICE))
        ref = ref.value
    torch.cuda.synchronize()

    results = []
    for _ in range(2):  # the second call reuses the scratch the first one left
        out.fill_(float("nan"))
        torch.cuda.synchronize()
        st = f(dim, s, edge, C.c_void_p(dev.data_ptr()), C.c_void_p(out.data_ptr()), layout, None)
        assert st == abi.OK, lib.mpdpft_last_error()
        torch.cuda.synchronize()
        results.append(float(out.item()))
    expect = _riemann(dim, s, edge, layout, host)
    assert abs(ref - expect) <= REL_TOL * max(1.0, abs(expect)), (ref, expect)
    for v in results:
        assert np.isfinite(v)
        assert abs(v - ref) <= REL_TOL * max(1.0, abs(ref)), (v, ref)
        assert abs(v - expect) <= REL_TOL * max(1.0, abs(expect)), (v, expect)
    assert results[0] == results[1]  # fixed tiling: the same summation order every call
