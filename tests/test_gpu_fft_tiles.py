"""GPU tests of the FFT autotuner's tile widths (no counterpart in the
reference, which plans FFTW once, mpDPFT.cpp:6313-6335): lines per tile of
the Y/X passes and rows per block of the Z passes.  A line's arithmetic
does not depend on how many lines a block holds, so DelField
(mpDPFT.cpp:7243-7582) gives the same bits in every configuration of either
path; the Hartree term (mpDPFT.cpp:2677-2715) agrees to round-off (its
zero-mode sum is summed over the Z blocks, whose number the width sets)."""
import numpy as np
import pytest

from mpdpft_b200 import abi
from mpdpft_b200 import workloads as W

pytestmark = pytest.mark.gpu

CONFIGS = {abi.MIXED: [(16, 16), (16, 8), (8, 16), (8, 8)], abi.FP64: [(8, 16), (8, 8), (4, 16), (4, 8)]}


def _problem(prec):
    p = abi.make_params(dim=3, steps=64, edge=12.0, density_expression=abi.DENS_GRADIENT, smearing_extent=0.6,
                        regularization_threshold=0.4, interactions=[abi.INT_HARTREE], gamma_h=1.0, precision=prec)
    r2 = W.radius2(3, 64, 12.0).reshape(-1)
    f = -3.0 / np.sqrt(r2 + 0.5) + 0.1 * np.exp(-0.2 * r2) + W.noise(r2.shape, 1e-3, 11)
    n = np.exp(-0.5 * r2)
    return p, f, n


@pytest.mark.parametrize("prec", [abi.MIXED, abi.FP64])
@pytest.mark.parametrize("path", ["plane", "pass"])
def test_tile_widths_give_the_same_results(eng, monkeypatch, prec, path):
    p, f, n = _problem(prec)
    monkeypatch.setenv("MPDPFT_FFT_PATH", path)
    ref = None
    for tk, zl in CONFIGS[prec]:
        monkeypatch.setenv("MPDPFT_FFT_TILES", "%d,%d" % (tk, zl))
        with eng.Engine(p) as e:
            assert e.fft_config()[0] == (1 if path == "plane" else 0)
            got_tk, got_zl = e.fft_tiles()
            g2, lap = e.DelField(f)
            vh = e.getVint(abi.INT_HARTREE, 0, [n])
        assert got_tk == tk
        if path == "pass":
            assert got_zl == zl
        if ref is None:
            ref = (g2, lap, vh)
            continue
        assert np.array_equal(g2, ref[0]) and np.array_equal(lap, ref[1]), (tk, zl)
        tol = 1e-12 if prec == abi.FP64 else 1e-5
        assert np.abs(vh - ref[2]).max() <= tol * np.abs(ref[2]).max(), (tk, zl)


def test_autotuner_picks_a_tried_configuration(eng, monkeypatch):
    monkeypatch.delenv("MPDPFT_FFT_PATH", raising=False)
    monkeypatch.delenv("MPDPFT_FFT_TILES", raising=False)
    for prec in (abi.MIXED, abi.FP64):
        p, f, n = _problem(prec)
        with eng.Engine(p) as e:
            path, ms_plane, ms_pass, how = e.fft_config()
            tk, zl = e.fft_tiles()
        print("prec %d: path %d plane %.4f ms pass %.4f ms how %d tiles %d,%d" % (prec, path, ms_plane, ms_pass, how,
                                                                               tk, zl))
        assert how in (1, 2)
        assert (tk, zl) in CONFIGS[prec] or (path == 1 and tk in [c[0] for c in CONFIGS[prec]])
        assert ms_pass > 0.0
    with pytest.raises(eng.MpdpftError):
        monkeypatch.setenv("MPDPFT_FFT_TILES", "3,3")
        eng.Engine(_problem(abi.MIXED)[0])
