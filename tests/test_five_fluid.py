"""The four-hydrogen-fluid step Setka::Go_5_komponent (Setka.cpp:8269-8950):
the plasma and H1..H4, each with its own HLLC flux, multi-fluid charge
exchange, cylindrical source terms, on the grid moved by Move_surface +
Move_Setka_Calculate.

The oracle is pinned to the reference bit for bit (live when the compiled
reference is present, and against tests/golden/steps_five_fluid_small.npz,
the reference's own output); the device path is compared with the oracle
and with that fixture."""
from pathlib import Path

import numpy as np
import pytest

import gelios_2d_b200 as g
from gelios_2d_b200 import _native as N
from gelios_2d_b200 import workloads as W
from oracle import oracle as O

GOLD = Path(__file__).resolve().parent / "golden"
SMALL = (4, 3, 3, 10, 23, 6, 7, 7)
MEDIUM = (30, 7, 11, 20, 60, 20, 40, 40)


def _oracle(mesh, st0, h0):
    ora = O.Oracle(O.reference_params(), mesh)
    for b in (0, 1):
        ora.set_state(b, st0)
        ora.set_hydrogen(b, h0)
    return ora


def rel_err(a, b):
    out = 0.0
    for k in range(a.shape[0]):
        s = np.max(np.abs(b[k]))
        if s > 0:
            out = max(out, float(np.max(np.abs(a[k] - b[k])) / s))
    return out


def test_oracle_matches_reference_fixture():
    gd = np.load(GOLD / "steps_five_fluid_small.npz")
    m = g.Mesh.setka(*SMALL)
    ora = _oracle(m, gd["state0"], gd["h0"])
    ora.five_komponent(4)
    assert np.array_equal(ora.get_state(0), gd["par0"])
    assert np.array_equal(ora.get_state(1), gd["par1"])
    assert np.array_equal(ora.get_hydrogen(0), gd["h_par0"])
    assert np.array_equal(ora.get_hydrogen(1), gd["h_par1"])
    pts = ora.points()
    assert np.array_equal(pts["x"], gd["x"]) and np.array_equal(pts["y"], gd["y"])


@pytest.mark.parametrize("dims,steps", [(SMALL, 6), (MEDIUM, 2)])
def test_oracle_matches_live_reference(have_ref, dims, steps):
    """Bit for bit against the compiled reference (single thread).  The
    medium grid clamps densities from the first step on in the reference
    too (its initial field is not balanced for this step); the clamps match."""
    from oracle import ref

    ref.set_threads(1)
    S = ref.RefSetka.constructor(*dims)
    S.tvd_prepare()
    S.init_conditions()
    m = g.Mesh.from_arrays(S.export())
    st0 = S.get_state(0)
    h0 = W.hydrogen_fields(m, seed=5)
    for b in (0, 1):
        S.set_hydrogen(b, h0)
    S.set_state(1, st0)
    S.go_5_komponent(steps)
    ora = _oracle(m, st0, h0)
    ora.five_komponent(steps)
    for b in (0, 1):
        assert np.array_equal(ora.get_state(b), S.get_state(b))
        assert np.array_equal(ora.get_hydrogen(b), S.get_hydrogen(b))
    pr, po = S.point_motion(), ora.points()
    assert np.array_equal(pr["x"], po["x"]) and np.array_equal(pr["y"], po["y"])


@pytest.mark.gpu
@pytest.mark.parametrize("steps", [1, 2, 6])
def test_device_matches_oracle_small(steps):
    m = g.Mesh.setka(*SMALL)
    st0 = W.init_conditions_reference(m)
    h0 = W.hydrogen_fields(m, seed=5)
    dev = g.Setka(m, N.reference_params())
    for b in (0, 1):
        dev.set_par(b, st0)
        dev.set_hydrogen(b, h0)
    s = dev.Go_5_komponent(steps)
    ora = _oracle(m, st0, h0)
    ora.five_komponent(steps)
    tol = 1e-12 if steps <= 2 else 1e-10
    for b in (0, 1):
        assert rel_err(dev.par(b), ora.get_state(b)) <= tol
        assert rel_err(dev.hydrogen(b), ora.get_hydrogen(b)) <= tol
    x, y = dev.points()
    pts = ora.points()
    assert np.max(np.abs(x - pts["x"]) / np.maximum(np.abs(pts["x"]), 1e-3)) <= 1e-13
    assert np.max(np.abs(y - pts["y"]) / np.maximum(np.abs(pts["y"]), 1e-3)) <= 1e-13
    assert abs(s.dt - ora.last_dt()) <= 1e-10 * ora.last_dt()


@pytest.mark.gpu
def test_device_matches_oracle_medium_one_step():
    m = g.Mesh.setka(*MEDIUM)
    st0 = W.init_conditions_reference(m)
    h0 = W.hydrogen_fields(m, seed=5)
    dev = g.Setka(m, N.reference_params())
    for b in (0, 1):
        dev.set_par(b, st0)
        dev.set_hydrogen(b, h0)
    s = dev.Go_5_komponent(1)
    ora = _oracle(m, st0, h0)
    ora.five_komponent(1)
    assert rel_err(dev.par(1), ora.get_state(1)) <= 1e-12
    assert rel_err(dev.hydrogen(1), ora.get_hydrogen(1)) <= 1e-12
    st = ora.status()
    assert s.n_ro_clamp == st[1] and s.n_p_clamp == st[2]


@pytest.mark.gpu
def test_device_matches_reference_fixture():
    gd = np.load(GOLD / "steps_five_fluid_small.npz")
    m = g.Mesh.setka(*SMALL)
    dev = g.Setka(m, N.reference_params())
    for b in (0, 1):
        dev.set_par(b, gd["state0"])
        dev.set_hydrogen(b, gd["h0"])
    dev.Go_5_komponent(4)
    for b in (0, 1):
        assert rel_err(dev.par(b), gd[f"par{b}"]) <= 1e-10
        assert rel_err(dev.hydrogen(b), gd[f"h_par{b}"]) <= 1e-10
