"""The MHD + pickup-proton moving-grid step (GELIOS_FORM_MHD_PUI).

The reference has no such step: it steps gas dynamics only and never calls
its MHD solvers.  The step is this project's assembly of the reference's
parts (grid motion and ion reconstruction of Go_5_komponent__MK2,
Setka.cpp:10121-10482; HLLD of Solvers::HLLDQ_Korolkov, Solvers.cpp:1642-2185,
in the face frame; HLLC of HLLC_2d_Korolkov_b_s, Setka.cpp:10484-10700, for
the pickup protons).  Its flux is pinned to the reference through the HLLDQ
golden vectors (tests/test_oracle_pin.py); the step itself is checked against
the oracle's restatement (oracle/gelios_oracle.c, go_mhd), which evaluates
every face from each side like the reference's cell loops, while the device
evaluates each face once and hands the negated flux to the neighbour.

Tolerances: max-norm relative error per variable <= 1e-12 after one and two
steps, <= 1e-10 after ten; point coordinates <= 1e-13.  Vector components
are measured against the magnitude of their vector: the azimuthal velocity
w (zero at the start, generated by the magnetic tension) against the ion
velocity scale, Bx, By, Bz against max |B|; every other row against itself.
"""
import numpy as np
import pytest

import gelios_2d_b200 as g
from gelios_2d_b200 import _native as N
from gelios_2d_b200 import workloads as W
from oracle import oracle as O

SMALL = (4, 3, 3, 10, 23, 6, 7, 7)
MEDIUM = (30, 7, 11, 20, 60, 20, 40, 40)


def rel_err(a, b):
    out = 0.0
    for k in range(a.shape[0]):
        s = np.max(np.abs(b[k]))
        if s > 0:
            out = max(out, float(np.max(np.abs(a[k] - b[k])) / s))
    return out


def ext_err(xd, xo, ion_o):
    """Error of the extra rows (w, Bx, By, Bz, pickup ro, p, u, v): w against
    the ion velocity scale, the field against max |B|, pickup rows per row."""
    vel = max(np.max(np.abs(ion_o[2])), np.max(np.abs(ion_o[3])))
    bmag = float(np.max(np.sqrt(xo[1] ** 2 + xo[2] ** 2 + xo[3] ** 2)))
    e = float(np.max(np.abs(xd[0] - xo[0]))) / vel
    if bmag > 0:
        e = max(e, max(float(np.max(np.abs(xd[k] - xo[k]))) for k in (1, 2, 3)) / bmag)
    return max(e, rel_err(xd[4:], xo[4:]))


def go_params(p: N.GeliosParams) -> O.GoParams:
    return O.GoParams(**{n: getattr(p, n) for n, _ in O.GoParams._fields_ if n != "pad_"}, pad_=0)


def setup(dims, mp=None, seed=17):
    mesh = g.Mesh.setka(*dims)
    P = N.reference_params()
    mp = mp if mp is not None else W.mhd_params()
    st0 = W.init_conditions_reference(mesh)
    x0 = W.mhd_initial(mesh, st0, mp)
    src = W.mhd_sources(mesh, seed=seed)
    return mesh, P, mp, st0, x0, src


def oracle_run(mesh, P, mp, st0, x0, src, steps):
    ora = O.Oracle(go_params(P), mesh)
    for b in (0, 1):
        ora.set_state(b, st0)
        ora.set_mhd(b, x0)
    ora.set_sources(*src)
    ora.mhd(mp.as_dict(), steps)
    return ora


def device_run(mesh, P, mp, st0, x0, src, steps):
    dev = g.Setka(mesh, P)
    dev.set_mhd_params(mp)
    for b in (0, 1):
        dev.set_par(b, st0)
        dev.set_mhd(b, x0)
    dev.set_sources(*src)
    st = dev.Go_MHD_pickup(steps)
    return dev, st


# ------------------------------------------------------------------ CPU (oracle)
def test_oracle_mhd_step_stays_physical():
    mesh, P, mp, st0, x0, src = setup(SMALL)
    ora = oracle_run(mesh, P, mp, st0, x0, src, 6)
    b = 6 % 2
    s, x = ora.get_state(b), ora.get_mhd(b)
    assert np.all(np.isfinite(s)) and np.all(np.isfinite(x))
    assert np.all(s[0] > 0) and np.all(s[1] > 0) and np.all(x[4] > 0) and np.all(x[5] > 0)
    assert not np.array_equal(s, st0)


def test_oracle_field_free_stays_field_free():
    """With no field anywhere (initial, inflow and wind) and no azimuthal
    velocity, the induction fluxes and the azimuthal terms vanish: B and w
    stay exactly zero."""
    mp = W.mhd_params(b_lism=0.0, inner_bphi=0.0)
    mesh, P, mp, st0, x0, src = setup(SMALL, mp)
    ora = oracle_run(mesh, P, mp, st0, x0, src, 4)
    x = ora.get_mhd(0)
    assert np.all(x[0:4] == 0.0)


def test_oracle_pickup_fluid_decoupled_from_field():
    """The pickup protons see the field only through the common time step:
    two runs with different fields but the same dt history give the same
    pickup fluid.  Checked on one step (dt = dt0 in both runs)."""
    mesh, P, mp1, st0, x0, src = setup(SMALL)
    mp2 = W.mhd_params(b_lism=0.02, b_angle_deg=50.0, inner_bphi=3.0)
    x02 = W.mhd_initial(mesh, st0, mp2)
    o1 = oracle_run(mesh, P, mp1, st0, x0, src, 1)
    o2 = oracle_run(mesh, P, mp2, st0, x02, src, 1)
    assert np.array_equal(o1.get_mhd(1)[4:], o2.get_mhd(1)[4:])
    assert not np.array_equal(o1.get_mhd(1)[1:4], o2.get_mhd(1)[1:4])


def test_mhd_entry_points_declared():
    names = N.header_functions()
    for f in ("gelios_set_mhd_params", "gelios_upload_mhd", "gelios_download_mhd", "gelios_upload_sources"):
        assert f in names
        assert hasattr(N.lib(), f)


# ------------------------------------------------------------------ GPU parity
@pytest.mark.gpu
@pytest.mark.parametrize("dims,steps,tol", [(SMALL, 1, 1e-12), (SMALL, 2, 1e-12), (MEDIUM, 2, 1e-12),
                                            (MEDIUM, 10, 1e-10)])
def test_mhd_device_matches_oracle(dims, steps, tol):
    mesh, P, mp, st0, x0, src = setup(dims)
    ora = oracle_run(mesh, P, mp, st0, x0, src, steps)
    dev, st = device_run(mesh, P, mp, st0, x0, src, steps)
    b = steps % 2
    assert st.result_buf == b
    e_ion = rel_err(dev.par(b), ora.get_state(b))
    e_ext = ext_err(dev.mhd(b), ora.get_mhd(b), ora.get_state(b))
    assert e_ion <= tol, e_ion
    assert e_ext <= tol, e_ext
    x, y = dev.points()
    po = ora.points()
    assert np.max(np.abs(x - po["x"])) <= 1e-13 * np.max(np.abs(po["x"]))
    assert np.max(np.abs(y - po["y"])) <= 1e-13 * np.max(np.abs(po["y"]))
    assert abs(st.dt - ora.last_dt()) <= 1e-12 * ora.last_dt()


@pytest.mark.gpu
def test_mhd_device_field_free_and_deterministic():
    mp = W.mhd_params(b_lism=0.0, inner_bphi=0.0)
    mesh, P, mp, st0, x0, src = setup(MEDIUM, mp)
    d1, _ = device_run(mesh, P, mp, st0, x0, src, 3)
    d2, _ = device_run(mesh, P, mp, st0, x0, src, 3)
    assert np.all(d1.mhd(1)[0:4] == 0.0)
    assert np.array_equal(d1.par(1), d2.par(1)) and np.array_equal(d1.mhd(1), d2.mhd(1))


@pytest.mark.gpu
def test_mhd_fp32_flux_close_to_fp64():
    mesh, P, mp, st0, x0, src = setup(MEDIUM)
    ora = oracle_run(mesh, P, mp, st0, x0, src, 4)
    P32 = P.copy(precision=N.PREC_FP32_FLUX)
    dev, _ = device_run(mesh, P32, mp, st0, x0, src, 4)
    assert rel_err(dev.par(0), ora.get_state(0)) <= 1e-4
    assert ext_err(dev.mhd(0), ora.get_mhd(0), ora.get_state(0)) <= 1e-4


@pytest.mark.gpu
def test_mhd_graph_matches_direct_launches():
    """The captured step graph (default) and direct launches (phase timing
    on) give the same bits."""
    mesh, P, mp, st0, x0, src = setup(MEDIUM)
    d1, _ = device_run(mesh, P, mp, st0, x0, src, 5)
    d2 = g.Setka(mesh, P)
    d2.set_mhd_params(mp)
    for b in (0, 1):
        d2.set_par(b, st0)
        d2.set_mhd(b, x0)
    d2.set_sources(*src)
    d2.set_phase_timing(True)
    d2.Go_MHD_pickup(5)
    assert np.array_equal(d1.par(1), d2.par(1)) and np.array_equal(d1.mhd(1), d2.mhd(1))
    assert np.array_equal(d1.points()[0], d2.points()[0])


def test_variant_counts():
    L = N.lib()
    assert L.gelios_variant_count(N.FORM_MHD_PUI) == 6
    assert L.gelios_variant_count(N.FORM_MK2) == 11
    for f in (N.FORM_STATIONARY, N.FORM_INNER_MK2, N.FORM_5_KOMPONENT):
        assert L.gelios_variant_count(f) == 1


def test_sweep_inflow_draws_in_configured_ranges():
    from gelios_2d_b200 import sweep as sw

    draws = W.splitmix64(7, 5 * 200).reshape(200, 5)
    chi, ro_wind, g_ = 36.1275, 116.667, 5.0 / 3.0
    for d in draws:
        f = sw.inflow_params(d)
        u, ro = -f["in_u"] / chi, f["in_ro"] / ro_wind
        mach = np.sqrt(f["in_ro"] * f["in_u"] ** 2 / (g_ * f["in_p"]))
        assert 0.04 <= u <= 0.08 and 0.002 <= ro <= 0.01 and 1.5 <= mach <= 3.0 + 1e-12
        assert 0.0 <= f["b_lism"] <= 0.02 and 0.0 <= f["b_angle_deg"] <= 60.0
    inst = sw.instance_set_mhd(8, only=[3])
    mesh, P, st0, (mp, x0, src) = inst[0]
    lism = mesh["cell_type"] == 4
    assert np.all(st0[0][lism] == P.in_ro) and np.all(st0[2][lism] == P.in_u)
    assert x0.shape == (8, mesh.n_cells) and len(src) == 3


@pytest.mark.gpu
def test_mhd_launch_shapes_give_same_bits_and_autotune_keeps_state():
    mesh, P, mp, st0, x0, src = setup(MEDIUM)
    ref, _ = device_run(mesh, P, mp, st0, x0, src, 3)
    n = N.lib().gelios_variant_count(N.FORM_MHD_PUI)

    def fresh():
        d = g.Setka(mesh, P)
        d.set_mhd_params(mp)
        for b in (0, 1):
            d.set_par(b, st0)
            d.set_mhd(b, x0)
        d.set_sources(*src)
        return d

    for v in range(1, n):
        d = fresh()
        d.set_variant(N.FORM_MHD_PUI, v)
        d.Go_MHD_pickup(3)
        assert np.array_equal(d.par(1), ref.par(1)) and np.array_equal(d.mhd(1), ref.mhd(1)), v
    d = fresh()
    v, ms = d.autotune(N.FORM_MHD_PUI, reps=2)
    assert 0 <= v < n and ms > 0.0
    d.Go_MHD_pickup(3)
    assert np.array_equal(d.par(1), ref.par(1)) and np.array_equal(d.mhd(1), ref.mhd(1))


@pytest.mark.gpu
def test_batched_instances_match_one_context_steps():
    """gelios_batch (one launch per phase over all instances) against each
    instance stepped on its own: same states, points and dt to rounding (the
    bodies are compiled into other kernels)."""
    from gelios_2d_b200 import sweep as sw

    inst = sw.instance_set_mhd(3, seed=5, scale=(0.12, 0.2))
    alone = sw.Sweep(inst, form=N.FORM_MHD_PUI)
    together = sw.Sweep(inst, form=N.FORM_MHD_PUI, batched=True)
    sa = [S.Go_MHD_pickup(3) for S in alone.items]
    st = together.batch_step(3, statuses=True)
    for i, (mesh, P, st0, extra) in enumerate(inst):
        a, b = alone.items[i], together.items[i]
        assert rel_err(b.par(1), a.par(1)) <= 1e-12
        assert ext_err(b.mhd(1), a.mhd(1), a.par(1)) <= 1e-12
        xa, ya = a.points()
        xb, yb = b.points()
        assert np.max(np.abs(xa - xb)) <= 1e-13 * np.max(np.abs(xa))
        assert np.max(np.abs(ya - yb)) <= 1e-13 * np.max(np.abs(ya))
        assert st[i].result_buf == 1 and st[i].steps_done == 3 and st[i].flags == sa[i].flags
        assert abs(st[i].dt - sa[i].dt) <= 1e-12 * sa[i].dt
    together.close()
    alone.close()


@pytest.mark.gpu
def test_persistent_batch_matches_per_phase_batch():
    """The persistent schedule (every step of a call in one cooperative
    kernel, grid barriers where the per-phase kernels end) against the
    per-phase batch: same states, points, dt and flags to rounding, over two
    calls (odd and even step counts); a block count that cannot be
    co-resident is refused; the autotuner keeps a schedule that fits."""
    from gelios_2d_b200 import sweep as sw

    inst = sw.instance_set_mhd(3, seed=5, scale=(0.12, 0.2))
    per_phase = sw.Sweep(inst, form=N.FORM_MHD_PUI, batched=True)
    persistent = sw.Sweep(inst, form=N.FORM_MHD_PUI, batched=True)
    persistent.set_batch_schedule(2)
    assert persistent.batch_schedules() == [2]
    for n, buf in ((5, 1), (2, 0)):
        sa = per_phase.batch_step(n, statuses=True)
        sp = persistent.batch_step(n, statuses=True)
        for i in range(len(inst)):
            a, b = per_phase.items[i], persistent.items[i]
            assert rel_err(b.par(buf), a.par(buf)) <= 1e-12
            assert ext_err(b.mhd(buf), a.mhd(buf), a.par(buf)) <= 1e-12
            xa, ya = a.points()
            xb, yb = b.points()
            assert np.max(np.abs(xa - xb)) <= 1e-13 * np.max(np.abs(xa))
            assert np.max(np.abs(ya - yb)) <= 1e-13 * np.max(np.abs(ya))
            assert sp[i].result_buf == buf and sp[i].steps_done == n and sp[i].flags == sa[i].flags
            assert abs(sp[i].dt - sa[i].dt) <= 1e-12 * sa[i].dt
    with pytest.raises(N.GeliosError):
        persistent.set_batch_schedule(4096)
    assert persistent.batch_schedules() == [2]
    (sched, ms, each), = persistent.autotune_batch(1)
    assert sched >= 0 and ms > 0.0 and persistent.batch_schedules() == [sched]
    assert len(each) >= 2 and abs(min(each) - ms) <= 1e-9 * ms
    st = persistent.batch_step(1, statuses=True)
    assert all(s.flags == 0 and s.dt > 0.0 for s in st)
    persistent.close()
    per_phase.close()


@pytest.mark.gpu
def test_mk2_launch_shapes_give_same_bits_and_autotune_keeps_state():
    """The moving-grid step's arrangements (face kernel + update kernel, or
    one tile kernel) and launch shapes give the same bits; autotuning writes
    only scratch."""
    mesh = g.Mesh.setka(*MEDIUM)
    P = N.reference_params()
    st0 = W.init_conditions_reference(mesh)
    mc = W.mc_fields(mesh, seed=9)

    def fresh():
        d = g.Setka(mesh, P)
        for b in (0, 1):
            d.set_par(b, st0)
        d.set_mc(*mc)
        return d

    ref = fresh()
    ref.Go_5_komponent__MK2(3)
    n = N.lib().gelios_variant_count(N.FORM_MK2)
    for v in range(1, n):
        d = fresh()
        d.set_variant(N.FORM_MK2, v)
        d.Go_5_komponent__MK2(3)
        assert np.array_equal(d.par(1), ref.par(1)) and np.array_equal(d.points()[0], ref.points()[0]), v
    d = fresh()
    v, ms = d.autotune(N.FORM_MK2, reps=2)
    assert 0 <= v < n and ms > 0.0
    d.Go_5_komponent__MK2(3)
    assert np.array_equal(d.par(1), ref.par(1)) and np.array_equal(d.par(0), ref.par(0))


@pytest.mark.gpu
def test_mhd_operator_residual_is_the_ion_flux_balance_of_a_still_grid():
    """gelios_operator_residual of the MHD + pickup form is the ion density
    change per unit time of a step on a grid that does not move (koef = 0:
    the first step snaps the points onto the rail formulas, the next leaves
    them in place bit for bit; the ion mass update has no source term, so
    |ro' - ro| = dt |sum F.S| / V in each updated cell; relative 1e-6).  The
    call changes no state, point or dt word."""
    mesh, P, mp, st0, x0, src = setup(MEDIUM)
    P = P.copy(koef=0.0)

    def run(with_residual):
        dev, _ = device_run(mesh, P, mp, st0, x0, src, 1)
        s1, h1 = dev.par(1), dev.mhd(1)
        pts1 = dev.points()
        dev.set_par(0, s1)
        dev.set_mhd(0, h1)
        r = None
        if with_residual:
            r = [dev.operator_residual(0, N.FORM_MHD_PUI), dev.operator_residual(0, N.FORM_MHD_PUI)]
        st = dev.Go_MHD_pickup(1)
        return dev, s1, pts1, st, r

    dev, s1, pts1, st, r = run(True)
    assert r[0] == r[1] and np.isfinite(r[0]) and r[0] > 0.0
    pts2 = dev.points()
    assert np.array_equal(pts1[0], pts2[0]) and np.array_equal(pts1[1], pts2[1])
    s2 = dev.par(1)
    ref = float(np.abs(s2[0] - s1[0]).sum() / (P.dt0 * np.abs(s1[0]).sum()))
    assert abs(r[0] - ref) <= 1e-6 * ref, (r[0], ref)
    dev2, _, _, st_b, _ = run(False)
    assert np.array_equal(dev2.par(1), s2) and np.array_equal(dev2.mhd(1), dev.mhd(1)) and st_b.dt == st.dt
    assert np.array_equal(dev2.points()[0], pts2[0])
