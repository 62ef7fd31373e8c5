"""GPU tests of the reference's field files: mpDPFT_V.dat / mpDPFT_Den.dat
written from a converged solve (ExportData, mpDPFT.cpp:12492-12519) and the
InterpolVQ restart that reads a V file of another grid and interpolates it
trilinearly onto the context's grid (LoadV, mpDPFT.cpp:6445-6499), checked
against scipy's linear grid interpolation of the same file."""
import numpy as np
import pytest

from mpdpft_b200 import abi
from mpdpft_b200 import workloads as W

pytestmark = pytest.mark.gpu


def test_field_files_match_the_fields(eng, tmp_path):
    p, vext, v0 = W.harmonic_tf(steps=24, precision=abi.FP64)
    vpath, dpath = tmp_path / "mpDPFT_V.dat", tmp_path / "mpDPFT_Den.dat"
    with eng.Engine(p) as e:
        e.sc_run(vext, v0)
        e.write_field_files(str(vpath), str(dpath))
        v = e.field(abi.FIELD_POTENTIAL, 0, layout=abi.LAYOUT_REFERENCE)
        n = e.field(abi.FIELD_DENSITY, 0, layout=abi.LAYOUT_REFERENCE)
    a = np.loadtxt(vpath)
    d = np.loadtxt(dpath)
    el = p.steps + 1
    assert a.shape == (el ** 3, 4) and d.shape == (el ** 3,)
    x = -0.5 * p.edge + p.edge / p.steps * np.arange(el)
    X, Y, Z = np.meshgrid(x, x, x, indexing="ij")
    assert np.array_equal(a[:, 0], X.ravel()) and np.array_equal(a[:, 1], Y.ravel())
    assert np.array_equal(a[:, 2], Z.ravel())
    assert np.abs(a[:, 3] - v).max() <= 1e-15 * np.abs(v).max()  # 16 significant digits
    assert np.abs(d - n).max() <= 1e-15 * np.abs(n).max()


@pytest.mark.parametrize("s_from,s_to", [(24, 32), (32, 24)])
def test_interpolated_restart(eng, tmp_path, s_from, s_to):
    """Solve on one grid, write V, interpolate it onto another grid: the
    GPU interpolation equals scipy's trilinear interpolation of the file
    (linear continuation beyond it), and the restarted solve converges to
    the solve from V_ext on that grid."""
    from scipy.interpolate import RegularGridInterpolator
    p1, vext1, v01 = W.harmonic_tf(steps=s_from, precision=abi.FP64)
    vpath = tmp_path / "mpDPFT_V.dat"
    with eng.Engine(p1) as e:
        e.sc_run(vext1, v01)
        e.write_field_files(str(vpath), None)
    p2, vext2, v02 = W.harmonic_tf(steps=s_to, precision=abi.FP64)
    with eng.Engine(p2) as e:
        vi, n_file = e.interpolate_v_file(str(vpath))
        vi_ref_layout, _ = e.interpolate_v_file(str(vpath), layout=abi.LAYOUT_REFERENCE)
        res_restart, log_r, st = e.sc_run(vext2, vi)
        n_restart = e.field(abi.FIELD_DENSITY, 0)
        res_fresh, log_f, st = e.sc_run(vext2, v02)
        n_fresh = e.field(abi.FIELD_DENSITY, 0)
    assert n_file == s_from + 1
    a = np.loadtxt(vpath)
    el = s_from + 1
    ax = a[::el * el, 0]
    f = RegularGridInterpolator((ax, ax, ax), a[:, 3].reshape(el, el, el), method="linear", bounds_error=False,
                                fill_value=None)
    x = W.axis(s_to, p2.edge)
    X, Y, Z = np.meshgrid(x, x, x, indexing="ij")
    expect = f(np.stack([X.ravel(), Y.ravel(), Z.ravel()], axis=-1))
    assert np.abs(vi[0] - expect).max() <= 1e-12 * np.abs(expect).max()
    assert np.array_equal(W.to_periodic(vi_ref_layout[0], 3), vi[0])
    assert res_restart.converged == 1 and res_fresh.converged == 1
    dvol = (p2.edge / p2.steps) ** 3
    assert np.abs(n_restart - n_fresh).sum() * dvol / 1000.0 < 1e-6
    assert res_restart.iterations <= res_fresh.iterations


def test_interpolate_rejects_bad_files(eng, tmp_path):
    p, vext, v0 = W.harmonic_tf(steps=16)
    bad = tmp_path / "bad.dat"
    bad.write_text("0 0 0 1\n1 0 0 2\n3 4 5\n")
    with eng.Engine(p) as e:
        with pytest.raises(eng.MpdpftError) as ex:
            e.interpolate_v_file(str(bad))
        assert ex.value.status == abi.ERR_ARG
        with pytest.raises(eng.MpdpftError):
            e.interpolate_v_file(str(tmp_path / "absent.dat"))
