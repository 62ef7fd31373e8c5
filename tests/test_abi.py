"""CPU tests of the C ABI: the library builds, loads and exports every
function include/mpdpft_gpu.h declares; no compute calls (no GPU here)."""
import ctypes as C
import os
import re

import pytest

from mpdpft_b200 import abi, engine

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    names = []
    for fn in os.listdir(os.path.join(ROOT, "include")):
        if fn.endswith(".h"):
            text = open(os.path.join(ROOT, "include", fn)).read()
            names += re.findall(r"^\s*(?:const\s+)?[a-z_]+\*?\s+\*?(mpdpft_[a-z0-9_]+)\s*\(", text, re.M)
    return sorted(set(names))


@pytest.fixture(scope="module")
def lib():
    from mpdpft_b200 import build
    build.build()
    return engine.load()


def test_every_declared_symbol_is_exported(lib):
    names = header_functions()
    assert len(names) >= 20
    for n in names:
        assert hasattr(lib, n), n
    assert set(names) >= set(engine.EXPORTS)


def test_abi_version_and_struct_sizes(lib):
    assert lib.mpdpft_abi_version() == abi.ABI_VERSION
    lib.mpdpft_struct_size.restype = C.c_size_t
    lib.mpdpft_struct_size.argtypes = [C.c_int]
    assert lib.mpdpft_struct_size(0) == C.sizeof(abi.Params)
    assert lib.mpdpft_struct_size(1) == C.sizeof(abi.Result)
    assert lib.mpdpft_struct_size(2) == C.sizeof(abi.IterLog)
    assert lib.mpdpft_struct_size(3) == C.sizeof(abi.Input)
    assert lib.mpdpft_struct_size(4) == C.sizeof(abi.LaunchRecord)


def test_params_default_matches_python_defaults(lib):
    p = abi.Params()
    lib.mpdpft_params_default(C.byref(p))
    q = abi.make_params()
    for name, _ in abi.Params._fields_:
        a, b = getattr(p, name), getattr(q, name)
        if isinstance(a, C.Array):
            assert list(a) == list(b), name
        else:
            assert a == b, name


def test_status_strings(lib):
    for st in range(9):
        assert lib.mpdpft_status_string(st)


def test_no_device_is_an_error_not_a_fallback(lib):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    h = C.c_void_p()
    st = lib.mpdpft_ctx_create(C.byref(abi.make_params()), 0, C.byref(h))
    assert st in (abi.ERR_NO_DEVICE, abi.ERR_CUDA)
    assert not h.value
