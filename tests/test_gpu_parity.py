"""Parity of the sm_100a kernels with the oracle (C restatement pinned to the
reference), called through the C ABI.

Tolerances (FP64 drop-in): max-norm relative error per
primitive variable <= 1e-12 after one/two steps from a common state and
<= 1e-9 after 1000 steps.  Point coordinates after grid motion agree to
1e-13 relative (the rails use cos/sin/pow of libdevice vs glibc: ~1 ulp).
The FP32-flux form is compared to the FP64 oracle with a loose bound and its
L1/Linf errors are reported.
"""
from pathlib import Path

import numpy as np
import pytest

import gelios_2d_b200 as g
from gelios_2d_b200 import _native as N
from gelios_2d_b200 import workloads as W
from oracle import oracle as O

pytestmark = pytest.mark.gpu
GOLD = Path(__file__).resolve().parent / "golden"
MEDIUM = (30, 7, 11, 20, 60, 20, 40, 40)
SMALL = (4, 3, 3, 10, 23, 6, 7, 7)


def rel_err(a: np.ndarray, b: np.ndarray) -> float:
    """max over variables of max|a-b| / max|b| (per row of a (5, n) state)."""
    out = 0.0
    for k in range(a.shape[0]):
        s = np.max(np.abs(b[k]))
        if s > 0:
            out = max(out, float(np.max(np.abs(a[k] - b[k])) / s))
    return out


def go_params(p: N.GeliosParams) -> O.GoParams:
    d = {n: getattr(p, n) for n, _ in O.GoParams._fields_ if n != "pad_"}
    return O.GoParams(**d, pad_=0)


def _pair(mesh, params, st0, mc=None):
    dev = g.Setka(mesh, params)
    dev.set_par(0, st0)
    dev.set_par(1, st0)
    ora = O.Oracle(go_params(params), mesh)
    ora.set_state(0, st0)
    ora.set_state(1, st0)
    if mc is not None:
        dev.set_mc(*mc)
        ora.set_mc(*mc)
    return dev, ora


# ------------------------------------------------------------------ per-face kernels
def test_hllc_device_vs_oracle():
    d = np.load(GOLD / "kat_hllc.npz")
    P = N.reference_params()
    dev = g.hllc_batch(P, d["inputs"])
    ref = d["outputs"]
    # [time, P0..P3, PQ, Vl, Vc, Vp]
    scale = np.maximum(np.abs(ref), 1e-300)
    err = np.abs(dev - ref) / np.maximum(scale, np.max(np.abs(ref), axis=1, keepdims=True) * 1e-3)
    assert np.max(err) <= 1e-13, np.max(err)


def test_hllc_fp32_flux_form():
    d = np.load(GOLD / "kat_hllc.npz")
    P = N.reference_params(precision=N.PREC_FP32_FLUX)
    dev = g.hllc_batch(P, d["inputs"])
    ref = d["outputs"]
    rows = np.max(np.abs(ref[:, 1:6]), axis=1, keepdims=True)
    err = np.abs(dev[:, 1:6] - ref[:, 1:6]) / rows
    assert np.max(err) <= 1e-5, np.max(err)


def test_hllc_fp32_wave_speed_form():
    """FP32 sound speeds and wave-speed estimates, fluxes assembled in FP64:
    against the reference's HLLC / HLL golden vectors the fluxes move by the
    wave speeds' float rounding only, well inside the full FP32 form's
    error."""
    d = np.load(GOLD / "kat_hllc.npz")
    ref = d["outputs"]
    rows = np.max(np.abs(ref[:, 1:6]), axis=1, keepdims=True)
    errs = {}
    for prec in (N.PREC_FP32_WAVES, N.PREC_FP32_FLUX):
        dev = g.hllc_batch(N.reference_params(precision=prec), d["inputs"])
        errs[prec] = float(np.max(np.abs(dev[:, 1:6] - ref[:, 1:6]) / rows))
    assert errs[N.PREC_FP32_WAVES] <= 1e-6, errs
    assert errs[N.PREC_FP32_WAVES] < errs[N.PREC_FP32_FLUX], errs


def test_godunov_device_vs_oracle():
    d = np.load(GOLD / "kat_godunov.npz")
    P = N.reference_params()
    dev = g.godunov_batch(P, d["inputs"])
    ref = d["outputs"]
    assert np.all(dev[:, 9] == 0)
    rows = np.maximum(np.max(np.abs(ref[:, 1:6]), axis=1), 1e-300)
    err = np.max(np.abs(dev[:, 1:6] - ref[:, 1:6]), axis=1) / rows
    assert np.max(err) <= 1e-11, np.max(err)
    assert np.max(np.abs(dev[:, 0] - ref[:, 0]) / np.abs(ref[:, 0])) <= 1e-11


def test_hlldq_device_vs_reference_vectors():
    d = np.load(GOLD / "kat_hlldq.npz")
    P = N.reference_params()
    dev = g.hlldq_batch(P, d["inputs"])
    ref = d["outputs"]
    scale = np.maximum(np.max(np.abs(ref[:, 1:10]), axis=1), 1e-300)
    err = np.max(np.abs(dev[:, 1:10] - ref[:, 1:10]), axis=1) / scale
    assert np.max(err) <= 1e-12, np.max(err)
    assert np.max(np.abs(dev[:, 0] - ref[:, 0]) / np.abs(ref[:, 0])) <= 1e-13


def test_hlld_device_vs_reference_vectors():
    d = np.load(GOLD / "kat_hlld.npz")
    P = N.reference_params()
    dev = g.hlld_batch(P, d["inputs"])
    ref = d["outputs"]
    assert np.all(dev[:, 12] == 0)
    scale = np.maximum(np.max(np.abs(ref[:, 1:9]), axis=1), 1e-300)
    err = np.max(np.abs(dev[:, 1:9] - ref[:, 1:9]), axis=1) / scale
    assert np.max(err) <= 1e-12, np.max(err)
    assert np.max(np.abs(dev[:, 9:12] - ref[:, 9:12]) / np.maximum(np.abs(ref[:, 9:12]), 1e-300)) <= 1e-13
    assert np.max(np.abs(dev[:, 0] - ref[:, 0]) / np.abs(ref[:, 0])) <= 1e-13


# ------------------------------------------------------------------ Go_stationary (plain single fluid)
@pytest.mark.parametrize("steps", [1, 2, 10])
def test_stationary_plain_small(steps):
    mesh = W.plain_mesh(36, 24)
    P = W.plain_params()
    st0 = W.plain_initial(mesh, P, seed=3)
    dev, ora = _pair(mesh, P, st0)
    s = dev.Go_stationary(steps)
    ora.stationary(steps)
    buf = steps % 2
    assert s.result_buf == buf
    e = rel_err(dev.par(buf), ora.get_state(buf))
    assert e <= 1e-12, e
    assert abs(s.dt - ora.last_dt()) <= 1e-12 * ora.last_dt()
    assert s.flags == 0


def test_stationary_plain_full_1000_steps():
    """The plain workload at full size (180 x 120), 1000 steps."""
    mesh = W.plain_mesh()
    P = W.plain_params()
    st0 = W.plain_initial(mesh, P, seed=2024)
    dev, ora = _pair(mesh, P, st0)
    dev.Go_stationary(1000)
    ora.stationary(1000)
    e = rel_err(dev.par(0), ora.get_state(0))
    assert e <= 1e-9, e


# ------------------------------------------------------------------ Go_5_komponent__MK2 (moving grid)
@pytest.mark.parametrize("steps", [1, 2, 12])
def test_mk2_moving_grid(steps):
    mesh = g.Mesh.setka(*MEDIUM)
    P = N.reference_params()
    st0 = W.init_conditions_reference(mesh)
    mc = W.mc_fields(mesh, seed=9)
    dev, ora = _pair(mesh, P, st0, mc)
    s = dev.Go_5_komponent__MK2(steps)
    ora.mk2(steps)
    buf = steps % 2
    e = rel_err(dev.par(buf), ora.get_state(buf))
    e_other = rel_err(dev.par(1 - buf), ora.get_state(1 - buf))
    tol = 1e-12 if steps <= 2 else 1e-10
    assert e <= tol, e
    assert e_other <= tol, e_other
    x, y = dev.points()
    pts = ora.points()
    assert np.max(np.abs(x - pts["x"]) / np.maximum(np.abs(pts["x"]), 1e-3)) <= 1e-13
    assert np.max(np.abs(y - pts["y"]) / np.maximum(np.abs(pts["y"]), 1e-3)) <= 1e-13
    st = ora.status()
    assert (s.flags & 1) == (st[0] & 1)


def test_mk2_source_terms_match_the_oracle():
    """The moving-grid step's charge-exchange source kernel run alone
    (gelios_mk2_source_terms) against the oracle's Get_Sourse_MK1
    (Cell.cpp:498-665) cell by cell on the medium rail grid with seeded
    Monte-Carlo moments: every cell the step updates, inside the radial
    re-interpolation window (bracket search along the cell chains) and
    outside it (the cell's own moments); 0 for the cells it skips.
    Tolerance: 1e-12 of each source row's largest magnitude."""
    mesh = g.Mesh.setka(*MEDIUM)
    P = N.reference_params()
    st0 = W.init_conditions_reference(mesh)
    mc = W.mc_fields(mesh, seed=9)
    dev, ora = _pair(mesh, P, st0, mc)
    n = mesh.n_cells
    q = [np.zeros(n) for _ in range(3)]
    for _ in range(2):  # the second call starts from the brackets the first one cached
        N.check(N.lib().gelios_mk2_source_terms(dev._h, 0, *q), "gelios_mk2_source_terms")
        x, y = mesh.centroids()
        rr = np.hypot(x, y)
        upd = ~(rr < P.R11)
        ref = np.zeros((3, n))
        for c in np.nonzero(upd)[0]:
            ref[:, c] = ora.source_mk1(c, st0[2, c], st0[3, c], st0[0, c], st0[1, c])
        for k in range(3):
            scale = float(np.max(np.abs(ref[k])))
            assert scale > 0.0
            assert float(np.max(np.abs(q[k] - ref[k]))) <= 1e-12 * scale
            assert np.all(q[k][~upd] == 0.0)
    window = upd & (rr > P.src_rmin) & (rr < P.src_rmax) & (x >= 0.0)
    assert window.any() and (upd & ~window).any() and (~upd).any()


def test_inner_mk2():
    mesh = g.Mesh.setka(*MEDIUM)
    P = N.reference_params()
    st0 = W.init_conditions_reference(mesh)
    mc = W.mc_fields(mesh, seed=4)
    dev, ora = _pair(mesh, P, st0, mc)
    dev.build_inner_list()
    assert len(dev.All_Cells_Inner) > 0
    ora.set_inner_list(dev.All_Cells_Inner)
    dev.Go_stationary_5_komponent_inner_MK2(3)
    ora.inner_mk2(3)
    for b in (0, 1):
        e = rel_err(dev.par(b), ora.get_state(b))
        assert e <= 1e-12, e


def test_mk2_golden_fixture():
    """Device vs the reference's own output stored in tests/golden."""
    gd = np.load(GOLD / "steps_small.npz")
    mesh = g.Mesh.setka(*SMALL)
    dev = g.Setka(mesh, N.reference_params())
    dev.set_par(0, gd["state0"])
    dev.set_par(1, gd["state0"])
    dev.set_mc(gd["Hn"], gd["Hu"], gd["Hv"], gd["HT"], gd["ku"], gd["kv"], gd["kT"])
    dev.Go_5_komponent__MK2(4)
    assert rel_err(dev.par(0), gd["mk2_par0"]) <= 1e-12
    assert rel_err(dev.par(1), gd["mk2_par1"]) <= 1e-12


def test_mk2_repeated_single_step_calls():
    """Each call restarts from par[0] on the moved grid (Setka.cpp:10126-10140);
    repeated one-step calls replay the captured step graph."""
    mesh = g.Mesh.setka(*MEDIUM)
    P = N.reference_params()
    st0 = W.init_conditions_reference(mesh)
    mc = W.mc_fields(mesh, seed=9)
    dev, ora = _pair(mesh, P, st0, mc)
    for _ in range(3):
        dev.Go_5_komponent__MK2(1)
        ora.mk2(1)
        assert rel_err(dev.par(1), ora.get_state(1)) <= 1e-12
    x, y = dev.points()
    pts = ora.points()
    assert np.max(np.abs(x - pts["x"]) / np.maximum(np.abs(pts["x"]), 1e-3)) <= 1e-13


def test_mk2_graph_matches_direct_launches():
    """The captured step (graph replay) against the same kernels launched
    directly (phase timing on), bit for bit, across parameter changes and
    odd/even step counts."""
    mesh = g.Mesh.setka(*MEDIUM)
    P = N.reference_params()
    P2 = P.copy(kurant=0.07)
    st0 = W.init_conditions_reference(mesh)
    mc = W.mc_fields(mesh, seed=9)
    runs = []
    for direct in (False, True):
        dev = g.Setka(mesh, P)
        dev.set_par(0, st0)
        dev.set_par(1, st0)
        dev.set_mc(*mc)
        dev.set_phase_timing(direct)
        dev.Go_5_komponent__MK2(1)
        dev.Go_5_komponent__MK2(1)
        dev.set_params(P2)
        dev.Go_5_komponent__MK2(2)
        s = dev.Go_5_komponent__MK2(3)
        runs.append((dev.par(0), dev.par(1), dev.points(), s.dt))
    a, b = runs
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
    assert np.array_equal(a[2][0], b[2][0]) and np.array_equal(a[2][1], b[2][1])
    assert a[3] == b[3]


@pytest.mark.parametrize("variant,precision", [(0, N.PREC_FP64), (8, N.PREC_FP64), (10, N.PREC_FP32_FLUX)])
def test_mk2_pipelined_calls_match_step_by_step(variant, precision):
    """A pipelined call (the next step's surface tracking and rails run while
    the cells they do not read are updated; points double-buffered) leaves
    the bits of one step after the other: states of both buffers, points, dt
    and the clamp / status words, over calls of 1, 2, 3, 7 and 40 steps."""
    mesh = g.Mesh.setka(*MEDIUM)
    P = N.reference_params().copy(precision=precision)
    st0 = W.init_conditions_reference(mesh)
    mc = W.mc_fields(mesh, seed=9)
    runs = []
    for pipelined in (True, False):
        dev = g.Setka(mesh, P)
        dev.set_par(0, st0)
        dev.set_par(1, st0)
        dev.set_mc(*mc)
        dev.set_variant(N.FORM_MK2, variant)
        dev.set_pipelined(pipelined)
        out = []
        for n in (1, 2, 3, 7, 40):
            s = dev.Go_5_komponent__MK2(n)
            out.append((dev.par(0), dev.par(1), dev.points(), s.dt, s.flags, s.n_ro_clamp, s.n_p_clamp))
        runs.append(out)
    for a, b in zip(*runs):
        assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
        assert np.array_equal(a[2][0], b[2][0]) and np.array_equal(a[2][1], b[2][1])
        assert a[3:] == b[3:]


def test_deterministic_runs():
    mesh = g.Mesh.setka(*MEDIUM)
    P = N.reference_params()
    st0 = W.init_conditions_reference(mesh)
    mc = W.mc_fields(mesh, seed=9)
    outs = []
    for _ in range(2):
        dev = g.Setka(mesh, P)
        dev.set_par(0, st0)
        dev.set_par(1, st0)
        dev.set_mc(*mc)
        dev.Go_5_komponent__MK2(6)
        outs.append((dev.par(0), dev.points()))
    assert np.array_equal(outs[0][0], outs[1][0])
    assert np.array_equal(outs[0][1][0], outs[1][1][0])


# ------------------------------------------------------------------ precision form
def test_fp32_flux_errors():
    mesh = W.plain_mesh(36, 24)
    P = W.plain_params()
    st0 = W.plain_initial(mesh, P, seed=3)
    dev32, ora = _pair(mesh, P.copy(precision=N.PREC_FP32_FLUX), st0)
    dev32.Go_stationary(20)
    ora.stationary(20)
    a, b = dev32.par(0), ora.get_state(0)
    for k, name in enumerate(("rho", "p", "u", "v")):
        linf = np.max(np.abs(a[k] - b[k])) / np.max(np.abs(b[k]))
        l1 = np.sum(np.abs(a[k] - b[k])) / np.sum(np.abs(b[k]))
        print(f"FP32-flux {name}: L1 {l1:.3e} Linf {linf:.3e}")
        assert linf <= 1e-4


# ------------------------------------------------------------------ failure detection (no GPU fault)
def test_iteration_cap_reports_status_without_hanging():
    """A Newton/bisection cap of 1 (test-only parameter) must end the solve
    with a status flag; the reference would exit(-1) (Solvers.cpp:1206-1273)."""
    mesh = g.Mesh.setka(*MEDIUM)
    P = N.reference_params(godunov_max_iter=1)
    st0 = W.init_conditions_reference(mesh)
    dev = g.Setka(mesh, P)
    dev.set_par(0, st0)
    dev.set_par(1, st0)
    s = dev.Go_5_komponent__MK2(2)
    assert s.flags & 1
    dev2 = g.Setka(mesh, P, raise_on_status=True)
    dev2.set_par(0, st0)
    dev2.set_par(1, st0)
    with pytest.raises(g.StepError):
        dev2.Go_5_komponent__MK2(2)


def test_launch_count_reported():
    mesh = W.plain_mesh(36, 24)
    P = W.plain_params()
    dev, _ = _pair(mesh, P, W.plain_initial(mesh, P))
    dev.Go_stationary(5)
    # words, centroids, face-centre radii, one cooperative launch for all five steps
    assert dev.launches() == 1 + 1 + 1 + 1
    dev.set_phase_timing(True)
    dev.Go_stationary(5)
    assert dev.launches() == 1 + 3 * 5  # words + (face units, cell update, dt) per step; geometry cached


@pytest.mark.parametrize("precision", [N.PREC_FP64, N.PREC_FP32_FLUX, N.PREC_FP32_WAVES])
def test_stationary_persistent_matches_three_kernel_steps(precision):
    """The cooperative multi-step launch and the three kernels per step
    (phase timing on) agree to rounding (the shared bodies are compiled into
    two kernels, whose multiply-add contraction may differ) with the same
    clamp counts and status."""
    mesh = W.plain_mesh()
    P = W.plain_params(precision=precision)
    st0 = W.plain_initial(mesh, P, seed=9)
    out = []
    for direct in (False, True):
        dev = g.Setka(mesh, P)
        dev.set_par(0, st0)
        dev.set_par(1, st0)
        dev.set_phase_timing(direct)
        st = dev.Go_stationary(25)
        out.append((dev.par(1), st.dt, st.n_ro_clamp, st.n_p_clamp, st.flags))
    # FP64: rounding of the last bits; FP32 fluxes: float rounding (1e-7 per
    # operation) compounds over the 25 steps
    # FP32 wave speeds: a float rounding of a wave speed that flips between
    # the two kernels moves one face's dissipation by ~1e-7 of itself
    tol = {N.PREC_FP64: 1e-13, N.PREC_FP32_FLUX: 1e-4, N.PREC_FP32_WAVES: 1e-6}[precision]
    assert rel_err(out[0][0], out[1][0]) <= tol
    assert abs(out[0][1] - out[1][1]) <= tol * out[1][1]
    assert out[0][2:] == out[1][2:]


def test_residual_matches_host_and_run_to_residual_stops():
    mesh = W.plain_mesh(36, 24)
    P = W.plain_params()
    st0 = W.plain_initial(mesh, P, seed=3)
    dev = g.Setka(mesh, P)
    dev.set_par(0, st0)
    dev.set_par(1, st0)
    st = dev.Go_stationary(10)
    a, b = dev.par(st.result_buf)[0], dev.par(1 - st.result_buf)[0]
    ref = float(np.abs(a - b).sum() / np.abs(a).sum())
    assert abs(dev.residual(st.result_buf) - ref) <= 1e-12 * ref
    n, r, dt = dev.run_to_residual(N.FORM_STATIONARY, 1e300, 1000, 100)
    assert n == 100 and r <= 1e300 and dt > 0
    n, r, dt = dev.run_to_residual(N.FORM_STATIONARY, 0.0, 300, 100)
    assert n == 300 and r > 0.0


def test_operator_residual_is_the_flux_balance_of_a_still_grid():
    """gelios_operator_residual is the density change per unit time of a step
    on a grid that does not move: with the surface speeds scaled by koef = 0
    the first step snaps the points onto the rail formulas and the next step
    leaves them in place bit for bit, so its density change over dt is the
    flux balance the residual evaluates (each updated cell: V2 = V,
    |ro' - ro| = dt |sum F.S| / V; relative 1e-6: ro' - ro is ~1e-8 of ro at
    dt0).  The call changes no state, point or dt word (the following steps
    give the same bits as without it)."""
    mesh = g.Mesh.setka(*MEDIUM)
    P = N.reference_params().copy(koef=0.0)
    st0 = W.init_conditions_reference(mesh)
    mc = W.mc_fields(mesh, seed=9)

    def run(with_residual):
        dev = g.Setka(mesh, P)
        dev.set_par(0, st0)
        dev.set_par(1, st0)
        dev.set_mc(*mc)
        dev.Go_5_komponent__MK2(1)
        s1 = dev.par(1)
        pts1 = dev.points()
        dev.set_par(0, s1)
        r = [dev.operator_residual(0), dev.operator_residual(0)] if with_residual else None
        st = dev.Go_5_komponent__MK2(1)
        return dev, s1, pts1, st, r

    dev, s1, pts1, st, r = run(True)
    assert r[0] == r[1] and np.isfinite(r[0]) and r[0] > 0.0
    pts2 = dev.points()
    assert np.array_equal(pts1[0], pts2[0]) and np.array_equal(pts1[1], pts2[1])
    s2 = dev.par(1)
    dt = N.reference_params().dt0
    ref = float(np.abs(s2[0] - s1[0]).sum() / (dt * np.abs(s1[0]).sum()))
    assert abs(r[0] - ref) <= 1e-6 * ref, (r[0], ref)
    dev2, _, _, st_b, _ = run(False)
    assert np.array_equal(dev2.par(1), s2) and np.array_equal(dev2.points()[0], pts2[0]) and st_b.dt == st.dt
