"""The C restatement (oracle/gelios_oracle.c) is pinned to the reference.

Against the live compiled reference (oracle/_ref/libgelios_ref.so, the
unmodified reference sources) and against the golden fixtures it produced
(tests/golden/make_golden.py), with the reference's compile-time constants as
parameters, the restatement must agree BIT FOR BIT.
"""
from pathlib import Path

import numpy as np
import pytest

from gelios_2d_b200 import workloads as W
from gelios_2d_b200.mesh import Mesh
from oracle import oracle as O

GOLD = Path(__file__).resolve().parent / "golden"
SMALL = (4, 3, 3, 10, 23, 6, 7, 7)
MEDIUM = (30, 7, 11, 20, 60, 20, 40, 40)


def test_hllc_known_answer_from_main_smoke_check():
    # Gelios_2D.cpp:46-67 evaluated with the compiled reference
    t, P, PQ, _ = O.hllc(O.reference_params(), (2, 1, 2, 1, 0), (1, 1, 1, 0.5, 0), 0.0, 1.0, 0.0, 10.0, 1)
    assert t == 0.43649167310370851
    assert P.tolist() == [2.0169953705134338, 3.9865567562696662, 0.0, 6.0199554761660163]
    assert PQ == 1.0084976852567169


def test_hllc_golden_bitexact():
    d = np.load(GOLD / "kat_hllc.npz")
    P0 = O.reference_params()
    for r, o in zip(d["inputs"], d["outputs"]):
        t, P, PQ, v = O.hllc(P0, r[0:5], r[5:10], r[10], r[11], r[12], r[13], int(r[14]), bool(r[15]))
        assert np.array_equal(np.array([t, *P, PQ, *v]), o, equal_nan=True)


def test_godunov_golden_bitexact():
    d = np.load(GOLD / "kat_godunov.npz")
    P0 = O.reference_params()
    for r, o in zip(d["inputs"], d["outputs"]):
        t, q, ds, st = O.godunov(P0, r[0:5], r[5:10], r[10:13], r[13], r[14])
        assert st == 0
        assert np.array_equal(np.array([t, *q, *ds]), o, equal_nan=True)


def test_hlldq_golden_bitexact():
    """HLLDQ_Korolkov (Solvers.cpp:1642-2185), metods 2 and 3, six axis normals."""
    d = np.load(GOLD / "kat_hlldq.npz")
    P0 = O.reference_params()
    assert set(d["inputs"][:, 22].astype(int)) == {2, 3}
    for r, o in zip(d["inputs"], d["outputs"]):
        t, P, PQ = O.hlldq(P0, r[0:9], r[9:18], r[18:21], r[21], int(r[22]))
        assert np.array_equal(np.array([t, *P, PQ]), o, equal_nan=True)


def test_hlld_golden_bitexact():
    """HLLD_Solver_Alexashov (Solvers.cpp:92-691) with face speed, any normal."""
    d = np.load(GOLD / "kat_hlld.npz")
    P0 = O.reference_params()
    for r, o in zip(d["inputs"], d["outputs"]):
        t, q, ds, st = O.hlld(P0, r[0:8], r[8:16], r[16:19], r[19], r[20])
        assert st == 0
        assert np.array_equal(np.array([t, *q, *ds]), o, equal_nan=True)


def test_hlld_reports_wave_order_instead_of_exiting():
    """Where the reference exits (SR <= SL, Solvers.cpp:244-249) the oracle
    raises the status bit and returns: two equal states without pressure and
    field have no fast speed, so SL == SR (planted on the CPU)."""
    P0 = O.reference_params()
    q = [1.0, 0.0, 0.5, 0.0, 0.0, 0.0, 0.0, 0.0]
    _, _, _, st = O.hlld(P0, q, q, [1.0, 0.0, 0.0], 0.0, 1.0)
    assert st & 32


def _oracle_on_small(mesh_dict, g):
    o = O.Oracle(O.reference_params(), mesh_dict)
    o.set_state(0, g["state0"])
    o.set_state(1, g["state0"])
    o.set_mc(g["Hn"], g["Hu"], g["Hv"], g["HT"], g["ku"], g["kv"], g["kT"])
    return o


@pytest.mark.parametrize("form,steps", [("stationary", 3), ("mk2", 4), ("inner", 3)])
def test_steps_golden_bitexact(form, steps):
    g = np.load(GOLD / "steps_small.npz")
    m = Mesh.setka(*SMALL)
    o = _oracle_on_small(m, g)
    if form == "stationary":
        o.stationary(steps)
    elif form == "mk2":
        o.mk2(steps)
    else:
        o.set_inner_list(g["inner_list"])
        o.inner_mk2(steps)
    for b in (0, 1):
        assert np.array_equal(o.get_state(b), g[f"{form}_par{b}"])
    pts = o.points()
    assert np.array_equal(pts["x"], g[f"{form}_x"]) and np.array_equal(pts["y"], g[f"{form}_y"])


def test_steps_live_reference_medium(have_ref):
    from oracle import ref

    S = ref.RefSetka.constructor(*MEDIUM)
    S.tvd_prepare()
    S.init_conditions()
    m = Mesh.from_arrays(S.export())
    st0 = S.get_state(0)
    mc = W.mc_fields(m, seed=3)
    S.set_mc(*mc)
    o = O.Oracle(O.reference_params(), m)
    o.set_state(0, st0)
    o.set_state(1, st0)
    o.set_mc(*mc)
    S.go_mk2(6)
    o.mk2(6)
    assert np.array_equal(o.get_state(0), S.get_state(0))
    assert np.array_equal(o.get_state(1), S.get_state(1))
    pm = S.point_motion()
    pts = o.points()
    assert np.array_equal(pts["x"], pm["x"]) and np.array_equal(pts["y"], pm["y"])
    S.go_stationary(3)
    o.stationary(3)
    assert np.array_equal(o.get_state(1), S.get_state(1))


def test_source_mk1_bitexact_live_reference(have_ref):
    """The oracle's Get_Sourse_MK1 (Cell.cpp:498-665) against the compiled
    reference's own member function, cell by cell, for every cell the
    moving-grid step updates (centroid radius >= R11), with seeded
    Monte-Carlo moments: bit for bit, inside the radial re-interpolation
    window (bracket search along the Back/Next chains of TVD_prepare) and
    outside it."""
    from oracle import ref

    S = ref.RefSetka.constructor(*MEDIUM)
    S.tvd_prepare()
    S.init_conditions()
    m = Mesh.from_arrays(S.export())
    st0 = S.get_state(0)
    mc = W.mc_fields(m, seed=5)
    S.set_mc(*mc)
    P = O.reference_params()
    o = O.Oracle(P, m)
    o.set_state(0, st0)
    o.set_state(1, st0)
    o.set_mc(*mc)
    x, y = m.centroids()
    rr = np.hypot(x, y)
    upd = np.nonzero(~(rr < P.R11))[0]
    window = (rr > P.src_rmin) & (rr < P.src_rmax) & (x >= 0.0)
    assert window[upd].any() and (~window[upd]).any()
    for c in upd:
        args = (c, st0[2, c], st0[3, c], st0[0, c], st0[1, c])
        assert np.array_equal(o.source_mk1(*args), S.source_mk1(*args)), c


def test_cell_geometry_bitexact_live_reference(have_ref):
    """The oracle's cell geometry against the compiled reference's own
    Cell methods, every cell of the medium rail grid, bit for bit: centre
    and moved centre (Cell.cpp:66-111), area and moved area (146-254),
    rotated volumes (188-206, 256-275)."""
    from oracle import ref

    S = ref.RefSetka.constructor(*MEDIUM)
    S.tvd_prepare()
    S.init_conditions()
    m = Mesh.from_arrays(S.export())
    o = O.Oracle(O.reference_params(), m)
    for c in range(m.n_cells):
        assert np.array_equal(o.cell_geom(c), S.cell_geom(c)), c


def test_polar_grid_through_reference_objects(have_ref):
    """The polar grid of the plain workload, instantiated as reference objects,
    stepped by the reference's own Go_stationary vs the restatement."""
    from oracle import ref

    m = Mesh.polar(24, 16, 1.0, 600.0)
    P = O.reference_params()
    st = W.plain_initial(m, W.plain_params(), seed=1)
    S = ref.RefSetka.from_mesh(m)
    S.set_state(0, st)
    S.set_state(1, st)
    o = O.Oracle(P, m)
    o.set_state(0, st)
    o.set_state(1, st)
    S.go_stationary(5)
    o.stationary(5)
    assert np.array_equal(o.get_state(1), S.get_state(1))
    assert np.array_equal(o.get_state(0), S.get_state(0))


def test_phase_level_motion(have_ref):
    """Move_surface + Move_Setka_Calculate_2 alone (point velocities and x2/y2)."""
    from oracle import ref

    S = ref.RefSetka.constructor(*MEDIUM)
    S.tvd_prepare()
    S.init_conditions()
    m = Mesh.from_arrays(S.export())
    o = O.Oracle(O.reference_params(), m)
    st0 = S.get_state(0)
    o.set_state(0, st0)
    o.set_state(1, st0)
    S.move_surface(0, 1e-3)
    o.move_surface(0, 1e-3)
    S.move_setka2(1e-3)
    o.move_setka2(1e-3)
    a, b = S.point_motion(), o.points()
    for k in ("Vx", "Vy", "x2", "y2", "count"):
        assert np.array_equal(a[k], b[k]), k


@pytest.mark.parametrize("dims", [SMALL, MEDIUM, (15, 5, 7, 15, 30, 10, 20, 20)])
def test_timing_build_constructor_equals_reference(have_ref, dims):
    """The CPU-baseline library's Setka.cpp sorts the tracked-face lines once
    (oracle/hoist_line_sort.py); its constructor and TVD_prepare must export
    exactly the grid of the unmodified reference."""
    from oracle import ref

    a = ref.RefSetka.constructor(*dims)
    b = ref.RefSetka.constructor(*dims, fast=True)
    a.tvd_prepare()
    b.tvd_prepare()
    ea, eb = a.export(), b.export()
    assert ea.keys() == eb.keys()
    for k in ea:
        assert np.array_equal(ea[k], eb[k]), k
    assert len(ea["line_contact"]) > 0 and len(ea["line_outer"]) > 0


def test_hoist_line_sort_touches_only_the_three_sorts():
    """The build-time patch adds one guard in front of each of the three
    sorts and nothing else."""
    from oracle.hoist_line_sort import GUARD, patch

    src = Path("/root/reference/Setka.cpp")
    if not src.exists():
        pytest.skip("reference tree not present")
    a = src.read_bytes()
    b = patch(a)
    assert b.replace(GUARD, b"") == a
    assert b.count(GUARD) == 3


@pytest.mark.parametrize("form", ["mk2", "inner", "k5"])
def test_reference_side_workload_equals_product_inputs(have_ref, form):
    """The reference arm builds its workload from the reference and numpy
    alone; the inputs must equal the product's workload generator (the grid,
    the seeded inputs and the updated-cell count bit for bit)."""
    from oracle import ref_workload as RW

    P = O.reference_params()
    rw = RW.build(MEDIUM, form)
    m = Mesh.setka(*MEDIUM)
    for k in ("x", "y", "contour", "gran", "face_sosed_down", "line_outer"):
        assert np.array_equal(rw.mesh[k], m[k]), k
    # Init_conditions: the reference's pow (glibc) and numpy's may round the
    # pressure of the wind cells differently in the last bit
    st0 = W.init_conditions_reference(m)
    np.testing.assert_allclose(rw.st0, st0, rtol=4e-16, atol=0)
    assert np.array_equal(rw.st0[[0, 2, 3, 4]], st0[[0, 2, 3, 4]])
    assert np.array_equal(rw.S.get_state(1), rw.st0)
    x, y = RW.centroids(rw.mesh)
    assert np.array_equal(np.stack([x, y]), m.centroids())
    if form == "k5":
        assert np.array_equal(rw.extra, W.hydrogen_fields(m, seed=3))
        assert rw.counted == W.counted_cells_mk2(m, P)
    else:
        for a, b in zip(rw.extra, W.mc_fields(m, seed=9)):
            assert np.array_equal(a, b)
        if form == "inner":
            inner = m.inner_cells(P.R111)
            assert rw.counted == int(np.count_nonzero(m["cell_type"][inner] != 5))
        else:
            assert rw.counted == W.counted_cells_mk2(m, P)
