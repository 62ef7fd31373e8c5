"""The reference's files (host code of the C ABI; no GPU): mpDPFT.input
parsing (GetInputParameters, mpDPFT.cpp:633-690) and its mapping onto the
engine's parameters, including the options the engine rejects.  The
reference's own sample input is parsed when the reference checkout is
present; the other inputs are written here in its format."""
import os

import numpy as np
import pytest

from mpdpft_b200 import abi, engine

REF_INPUT = "/root/reference/mpDPFT.input"

# mpDPFT.input for config C1 (harmonic trap, TF + contact, 64^3), in the
# reference's line order with its comment style
C1_LINES = [
    "0\t\t\t//System", "0\t\t\t//Symmetry", "0\t\t\t//TaskType", "0\t\t\t//TaskParameterCount",
    "0. 0.\t\t\t//TaskHyperBox", "3\t\t\t//DIM", "1\t\t\t//Units", "24.\t\t\t//edge", "64\t\t\t//steps",
    "1\t\t\t//S", "1000.\t\t\t//Abundances", "1.0e-10\t\t\t//RelAcc", "0.01\t\t\t//InternalAcc",
    "0\t\t\t//K", "0.\t\t\t//Resources", "7\t\t\t//DensityExpression", "0.5 0.5\t\t\t//mpp",
    "1. 1. 1.0e-6\t\t//Mpp", "1.\t\t\t//tauVec", "1.\t\t\t//tVec", "1.\t\t\t//TVec", "1\t\t\t//Environments",
    "1.\t\t\t//stretchfactor", "0.\t\t\t//Wall", "0.\t\t\t//Noise", "0\t\t\t//InterpolVQ",
    "10\t\t\t//Interactions", "1.\t\t\t//incrementalV", "18.17\t\t\t//muVec", "-3.\t\t\t//DeltamuModifier",
    "1. 5. -1.\t\t//Mixer", "0.3\t\t\t//thetaVec", "1.0e-12\t\t\t//SCcriterion", "400\t\t\t//maxSCcount",
    "1\t\t\t//method", "5\t\t\t//DelFieldMethod", "0\t\t\t//MovieQ", "0\t\t\t//Schedule", "0\t\t\t//EkinTypes",
    "0.\t\t\t//alpha", "0.25\t\t\t//beta", "0.\t\t\t//gamma", "0.\t\t\t//gammaH", "1.\t\t\t//degeneracy",
    "0\t\t\t//regularize", "0.375\t\t\t//RegularizationThreshold", "2\t\t\t//Print",
]


@pytest.fixture(scope="module")
def lib():
    from mpdpft_b200 import build
    build.build()
    return engine.load()


def write_input(tmp_path, lines, name="mpDPFT.input"):
    path = tmp_path / name
    path.write_text("\n".join(lines) + "\n")
    return str(path)


def test_c1_input_parses_and_maps(lib, tmp_path):
    inp = engine.read_input(write_input(tmp_path, C1_LINES))
    assert inp.lines == 47
    assert (inp.dim, inp.units, inp.steps, inp.species) == (3, 1, 64, 1)
    assert inp.edge == 24.0 and inp.abundances[0] == 1000.0 and inp.rel_acc == 1e-10
    assert list(inp.Mpp[:inp.n_Mpp]) == [1.0, 1.0, 1e-6]
    assert list(inp.mixer) == [1.0, 5.0, -1.0]
    assert list(inp.interactions[:inp.n_interactions]) == [10]
    p = engine.params_from_input(inp)
    q = abi.make_params(dim=3, steps=64, edge=24.0, abundances=[1000.0], rel_acc=1e-10, density_expression=abi.DENS_TF,
                        interactions=[abi.INT_CONTACT_SELF], beta=0.25, mu=[18.17], mixer=1, pulay_scope=5,
                        theta=[0.3], sc_criterion=1e-12, max_sc_count=400, degeneracy=1.0,
                        regularization_threshold=0.375, internal_acc=0.01)
    for name, _ in abi.Params._fields_:
        a, b = getattr(p, name), getattr(q, name)
        if name in ("abundances", "tau", "temperature", "mu", "theta"):
            assert a[0] == b[0], name
        elif isinstance(a, abi.C.Array):
            assert list(a) == list(b), name
        else:
            assert a == b, name


@pytest.mark.parametrize("line,value,needle", [
    (6, "2", "Units"), (15, "11", "DensityExpression"), (26, "13", "type 13"), (30, "2. 10. -1.", "Pulay2"),
    (34, "2", "Riemann"), (37, "3", "Schedule"),
])
def test_unsupported_options_are_rejected_with_their_line(lib, tmp_path, line, value, needle):
    lines = list(C1_LINES)
    lines[line] = value + "\t\t\t//changed"
    inp = engine.read_input(write_input(tmp_path, lines))
    with pytest.raises(engine.MpdpftError) as ex:
        engine.params_from_input(inp)
    assert ex.value.status == abi.ERR_ARG
    assert ("line %d" % line) in str(ex.value) and needle in str(ex.value)


def test_gradient_input_maps_to_finite_t_form(lib, tmp_path):
    lines = list(C1_LINES)
    lines[15] = "5\t\t\t//DensityExpression"
    lines[17] = "2. 3. 1.0e-4\t\t//Mpp"
    lines[12] = "1.0e-6\t\t\t//InternalAcc"
    p = engine.params_from_input(engine.read_input(write_input(tmp_path, lines)))
    assert p.density_expression == abi.DENS_GRADIENT and p.gradient_form == abi.GRADIENT_FINITE_T
    assert (p.boole_pairs, p.boole_max_iter, p.airy_threshold, p.internal_acc) == (2, 3, 1e-4, 1e-6)
    lines[5] = "2\t\t\t//DIM"
    with pytest.raises(engine.MpdpftError) as ex:
        engine.params_from_input(engine.read_input(write_input(tmp_path, lines)))
    assert "2D Airy" in str(ex.value)
    lines[17] = "2. 3. 1.0e+300\t\t//Mpp"
    p = engine.params_from_input(engine.read_input(write_input(tmp_path, lines)))
    assert p.dim == 2 and p.gradient_form == abi.GRADIENT_T0


def test_short_or_broken_input_is_an_error(lib, tmp_path):
    with pytest.raises(engine.MpdpftError):
        engine.read_input(write_input(tmp_path, C1_LINES[:20]))
    lines = list(C1_LINES)
    lines[10] = "//Abundances missing"
    with pytest.raises(engine.MpdpftError) as ex:
        engine.read_input(write_input(tmp_path, lines))
    assert "line 10" in str(ex.value)
    with pytest.raises(engine.MpdpftError):
        engine.read_input(str(tmp_path / "absent.input"))


@pytest.mark.skipif(not os.path.exists(REF_INPUT), reason="reference checkout not present")
def test_reference_sample_input(lib):
    """The reference's own sample input: a 2D two-species run with
    DensityExpression 11, which the engine does not implement."""
    inp = engine.read_input(REF_INPUT)
    assert (inp.dim, inp.units, inp.steps, inp.species, inp.edge) == (2, 1, 256, 2, 16.0)
    assert list(inp.abundances[:2]) == [15.0, 15.0]
    assert inp.density_expression == 11
    assert list(inp.Mpp[:inp.n_Mpp]) == [1.0, 1.0, 1e-6]
    assert list(inp.mixer) == [0.0, 10.0, -1.0]
    assert list(inp.theta[:2]) == [0.3, 0.3] and inp.sc_criterion == 1e-12
    assert inp.regularization_threshold == 0.375 and inp.print == 2
    with pytest.raises(engine.MpdpftError) as ex:
        engine.params_from_input(inp)
    assert "line 15" in str(ex.value)


@pytest.mark.skipif(not os.path.exists("/root/reference/mpDPFT_V_20250509_104113.dat"),
                    reason="reference checkout not present")
def test_reference_v_file_layout():
    """The reference's own V file (ExportData): (s+1)^D lines, x-major, the
    D lattice coordinates then one V per species -- the layout
    mpdpft_write_field_files writes and mpdpft_interpolate_v_file reads."""
    a = np.loadtxt("/root/reference/mpDPFT_V_20250509_104113.dat")
    n = int(round(np.sqrt(a.shape[0])))
    assert n * n == a.shape[0] and a.shape[1] == 2 + 2
    x = a[::n, 0]
    y = a[:n, 1]
    assert np.allclose(x, y) and np.allclose(np.diff(x), (x[-1] - x[0]) / (n - 1))
    assert abs(x[0] + x[-1]) < 1e-12  # the box [-L/2, L/2] with both end planes stored
