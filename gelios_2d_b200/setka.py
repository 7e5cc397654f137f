"""Host-side mirror of the reference's operator interface for the plasma step.

The reference drives its time step through member functions of ``Setka``
(Setka.h:21-235).  :class:`Setka` keeps those names and their meaning on top
of the C ABI (include/gelios_b200.h):

==========================================  =====================================
reference (Setka.h)                          here
==========================================  =====================================
``Setka(N1..M4)`` (Setka.cpp:19-1076)        ``Setka.from_constructor(N1..M4)``
``TVD_prepare()`` (Setka.cpp:1294-1492)      ``TVD_prepare()``
``Init_conditions()`` (Setka.cpp:5149-5203)  ``Init_conditions()``
``Cell::par[0/1]``                           ``par(buf)`` / ``set_par(buf, state)``
``Go_stationary(int)``                       ``Go_stationary(step)``
``Go_5_komponent__MK2(int)``                 ``Go_5_komponent__MK2(step)``
``Go_stationary_5_komponent_inner_MK2(int)`` ``Go_stationary_5_komponent_inner_MK2(step)``
``Go_5_komponent(int)``                      ``Go_5_komponent(step)`` (+ ``set_hydrogen``)
(no reference step)                          ``Go_MHD_pickup(step)`` (+ ``set_mhd``, ``set_sources``)
``Save_Setka_ALL_ALPHA(string)``             ``Save_Setka_ALL_ALPHA(name)``
``Download_Setka_ALL_ALPHA_2_0(string)``     ``Setka.Download_Setka_ALL_ALPHA_2_0(name)``
==========================================  =====================================

As in the reference, a step call restarts dt at 1e-8 and the newest state
ends in ``par[step % 2]``; cells a loop skips keep their old values in both
buffers.  Differences in error behaviour: where the reference calls
``exit(-1)`` the step raises :class:`StepError` carrying the device status
flags instead (the kernels never trap).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _native as N
from .mesh import Mesh

STATUS_BITS = {1: "newton/bisection iteration cap", 2: "non-positive TVD state", 4: "negative Newton pressure",
               8: "broken source chain", 16: "non-finite dt", 32: "MHD wave speeds out of order"}


class StepError(RuntimeError):
    def __init__(self, status: N.GeliosStatus):
        names = [v for k, v in STATUS_BITS.items() if status.flags & k]
        super().__init__("device status: " + ", ".join(names))
        self.status = status


class Setka:
    """A grid + state resident on one GPU, stepped by the sm_100a kernels."""

    def __init__(self, mesh: Mesh, params: N.GeliosParams | None = None, device: int = 0,
                 raise_on_status: bool = False):
        self.mesh = mesh
        self.params = params if params is not None else N.reference_params()
        self.raise_on_status = raise_on_status
        L = N.lib()
        h = C.c_void_p()
        N.check(L.gelios_create(C.byref(h), C.byref(self.params), int(device)), "gelios_create")
        self._h = h
        self._L = L
        v, keep = mesh.view()
        N.check(L.gelios_upload_topology(self._h, C.byref(v)), "gelios_upload_topology")
        del keep
        self.last_status = N.GeliosStatus()
        self.All_Cells_Inner = np.zeros(0, np.int32)

    # ------------------------------------------------------------ construction
    @classmethod
    def from_constructor(cls, N1, N2, N3, N4, M1, M2, M3, M4, params=None, device=0) -> "Setka":
        return cls(Mesh.setka(N1, N2, N3, N4, M1, M2, M3, M4, tvd=True), params, device)

    @classmethod
    def Download_Setka_ALL_ALPHA_2_0(cls, name, params=None, device=0) -> "Setka":
        """Setka::Download_Setka_ALL_ALPHA_2_0 (Setka.cpp:2899-3257) followed
        by TVD_prepare: grid, par[0] (copied to par[1], as the loader does)
        and Monte-Carlo moments from the reference's text checkpoint."""
        from . import checkpoint

        c = checkpoint.read_alpha(name)
        S = cls(c.mesh, params, device)
        S.set_par(0, c.par)
        S.set_par(1, c.par)
        S.set_mc(*c.mc)
        S._ckpt_extra = (c.hydrogen, c.I)
        return S

    def Save_Setka_ALL_ALPHA(self, name, buf: int = 0):
        """Setka::Save_Setka_ALL_ALPHA (Setka.cpp:2355-2574): the grid at its
        current point positions and par[buf] (the reference saves par[0]) in
        the reference's text format (6 significant digits)."""
        from . import checkpoint

        m = Mesh.from_arrays(dict(self.mesh))
        m["x"], m["y"] = self.points()
        hyd, I = getattr(self, "_ckpt_extra", (None, None))
        checkpoint.write_alpha(name, m, self.par(buf), getattr(self, "_mc", None), hyd, I)

    def close(self):
        if getattr(self, "_h", None):
            self._L.gelios_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_params(self, params: N.GeliosParams):
        self.params = params
        N.check(self._L.gelios_set_params(self._h, C.byref(params)), "gelios_set_params")

    # ------------------------------------------------------------ reference-named operations
    def TVD_prepare(self):
        """Setka::TVD_prepare: recompute TVD neighbours and source chains from
        the current point positions and re-upload the topology."""
        self.mesh.tvd_prepare()
        v, keep = self.mesh.view()
        st = [self.par(0), self.par(1)]
        N.check(self._L.gelios_upload_topology(self._h, C.byref(v)), "gelios_upload_topology")
        self.set_par(0, st[0])
        self.set_par(1, st[1])

    def Init_conditions(self):
        """Setka::Init_conditions (Setka.cpp:5149-5203) into par[0] and par[1]."""
        from .workloads import init_conditions_reference

        st = init_conditions_reference(self.mesh)
        self.set_par(0, st)
        self.set_par(1, st)

    def build_inner_list(self, r_max: float | None = None):
        """All_Cells_Inner of main (Gelios_2D.cpp:152-231): centroid radius <= R111_."""
        r = self.params.R111 if r_max is None else r_max
        self.All_Cells_Inner = self.mesh.inner_cells(r)
        a = np.ascontiguousarray(self.All_Cells_Inner, np.int32)
        ptr = a.ctypes.data_as(C.POINTER(C.c_int32)) if len(a) else C.cast(None, C.POINTER(C.c_int32))
        N.check(self._L.gelios_set_inner_cells(self._h, ptr, len(a)), "gelios_set_inner_cells")

    def Go_stationary(self, step: int) -> N.GeliosStatus:
        return self._go(N.FORM_STATIONARY, step)

    def Go_5_komponent__MK2(self, step: int) -> N.GeliosStatus:
        return self._go(N.FORM_MK2, step)

    def Go_stationary_5_komponent_inner_MK2(self, step: int) -> N.GeliosStatus:
        return self._go(N.FORM_INNER_MK2, step)

    def Go_5_komponent(self, step: int) -> N.GeliosStatus:
        """Setka::Go_5_komponent (Setka.cpp:8269-8950): the plasma and the
        four hydrogen fluids (set with :meth:`set_hydrogen`) on the grid
        moved by Move_surface + Move_Setka_Calculate."""
        return self._go(N.FORM_5_KOMPONENT, step)

    def Go_MHD_pickup(self, step: int) -> N.GeliosStatus:
        """The moving-grid step for an ion MHD fluid and pickup protons
        (GELIOS_FORM_MHD_PUI; no reference step: same motion as
        Go_5_komponent__MK2, HLLD ion fluxes of Solvers::HLLDQ_Korolkov in
        the face frame, HLLC pickup fluxes).  Extra rows via :meth:`set_mhd`,
        fixed charge-exchange sources via :meth:`set_sources`, boundary data
        via :meth:`set_mhd_params`."""
        return self._go(N.FORM_MHD_PUI, step)

    def set_mhd_params(self, mp: "N.GeliosMhdParams"):
        self.mhd_params = mp
        N.check(self._L.gelios_set_mhd_params(self._h, C.byref(mp)), "gelios_set_mhd_params")

    def set_mhd(self, buf: int, x8: np.ndarray):
        """Extra rows of par[buf] for the MHD form: w, Bx, By, Bz of the ions,
        ro, p, u, v of the pickup protons (shape (8, n_cells))."""
        x8 = np.ascontiguousarray(x8, np.float64)
        if x8.shape != (8, self.mesh.n_cells):
            raise ValueError("MHD extra rows must be (8, n_cells)")
        N.check(self._L.gelios_upload_mhd(self._h, int(buf), x8.ravel()), "gelios_upload_mhd")

    def mhd(self, buf: int) -> np.ndarray:
        out = np.zeros(8 * self.mesh.n_cells)
        N.check(self._L.gelios_download_mhd(self._h, int(buf), out), "gelios_download_mhd")
        return out.reshape(8, self.mesh.n_cells)

    def set_sources(self, q1, q2, q3):
        """Fixed charge-exchange sources of the ion x/y momentum and energy
        (per unit volume, n_cells each) for the MHD form."""
        f = lambda a: np.ascontiguousarray(a, np.float64).ravel()  # noqa: E731
        N.check(self._L.gelios_upload_sources(self._h, f(q1), f(q2), f(q3)), "gelios_upload_sources")

    def residual(self, result_buf: int) -> float:
        """L1 residual of the density over the last step (result_buf newer)."""
        r = C.c_double()
        N.check(self._L.gelios_residual(self._h, int(result_buf), C.byref(r)), "gelios_residual")
        return float(r.value)

    def operator_residual(self, buf: int = 0, form: int = N.FORM_MK2) -> float:
        """Residual per unit time of the moving-grid operator of `form` (MK2
        or MHD + pickup) at par[buf] with the grid held still (face speeds
        0): sum over updated cells of |sum of the mass fluxes F.S| / volume
        over sum |ro|."""
        r = C.c_double()
        N.check(self._L.gelios_operator_residual(self._h, int(form), int(buf), C.byref(r)),
                "gelios_operator_residual")
        return float(r.value)

    def run_to_residual(self, form: int, tol: float, max_steps: int, check_every: int = 20000):
        """Calls of check_every steps until residual / dt <= tol; returns
        (steps run, residual per unit time, dt)."""
        n, r, dt = C.c_int64(), C.c_double(), C.c_double()
        N.check(self._L.gelios_run_to_residual(self._h, int(form), float(tol), int(max_steps), int(check_every),
                                               C.byref(n), C.byref(r), C.byref(dt)), "gelios_run_to_residual")
        return int(n.value), float(r.value), float(dt.value)

    def run_streamed(self, form: int, host_in, host_out):
        """len(host_in) one-step calls of `form` with host I/O overlapped with
        the steps (gelios_run_streamed): call k reads host_in[k] into par[0]
        and writes par[1] into host_out[k].  Blocks are C-contiguous float64
        arrays of shape (gelios_io_rows(form), n_cells), ideally pinned."""
        n = len(host_in)
        if len(host_out) != n:
            raise ValueError("host_in and host_out differ in length")
        rows = int(self._L.gelios_io_rows(int(form)))
        for a in list(host_in) + list(host_out):
            if a.dtype != np.float64 or a.shape != (rows, self.mesh.n_cells) or not a.flags.c_contiguous:
                raise ValueError(f"blocks must be C-contiguous float64 of shape ({rows}, n_cells)")
        pin = (C.c_void_p * max(n, 1))(*[a.ctypes.data for a in host_in])
        pout = (C.c_void_p * max(n, 1))(*[a.ctypes.data for a in host_out])
        N.check(self._L.gelios_run_streamed(self._h, int(form), n, pin, pout), "gelios_run_streamed")

    def autotune(self, form: int = N.FORM_MHD_PUI, reps: int = 5) -> tuple[int, float]:
        """Time every launch shape of the form's dominant kernel on this grid
        and state, keep the fastest; returns (variant, mean ms).  The state
        and the points are not changed."""
        v = C.c_int32()
        ms = C.c_double()
        N.check(self._L.gelios_autotune(self._h, int(form), int(reps), C.byref(v), C.byref(ms)), "gelios_autotune")
        return int(v.value), float(ms.value)

    def set_variant(self, form: int, variant: int):
        N.check(self._L.gelios_set_variant(self._h, int(form), int(variant)), "gelios_set_variant")

    def get_variant(self, form: int) -> int:
        """The variant of the form's dominant kernels this context uses."""
        v = C.c_int32()
        N.check(self._L.gelios_get_variant(self._h, int(form), C.byref(v)), "gelios_get_variant")
        return int(v.value)

    def set_pipelined(self, on: bool):
        """Moving-grid calls with the next step's motion overlapping the
        update (default), or one step after the other (same bits)."""
        N.check(self._L.gelios_set_pipelined(self._h, 1 if on else 0), "gelios_set_pipelined")

    def set_hydrogen(self, buf: int, h16: np.ndarray):
        """ro, p, u, v of the hydrogen fluids H1..H4 of Cell::par[buf]
        (shape (16, n_cells))."""
        h16 = np.ascontiguousarray(h16, np.float64)
        if h16.shape != (16, self.mesh.n_cells):
            raise ValueError("hydrogen state must be (16, n_cells)")
        N.check(self._L.gelios_upload_hydrogen(self._h, int(buf), h16.ravel()), "gelios_upload_hydrogen")

    def hydrogen(self, buf: int) -> np.ndarray:
        out = np.zeros(16 * self.mesh.n_cells)
        N.check(self._L.gelios_download_hydrogen(self._h, int(buf), out), "gelios_download_hydrogen")
        return out.reshape(16, self.mesh.n_cells)

    def _go(self, form: int, step: int) -> N.GeliosStatus:
        st = N.GeliosStatus()
        N.check(self._L.gelios_step(self._h, int(form), int(step), C.byref(st)), "gelios_step")
        self.last_status = st
        if self.raise_on_status and st.flags:
            raise StepError(st)
        return st

    def step(self, form: int, step: int) -> N.GeliosStatus:
        """`step` iterations of the given form (N.FORM_*), synchronously."""
        return self._go(form, step)

    def step_async(self, form: int, step: int):
        """Enqueue `step` iterations without synchronising (timing loops)."""
        N.check(self._L.gelios_step(self._h, int(form), int(step), None), "gelios_step")

    def synchronize(self):
        N.check(self._L.gelios_synchronize(self._h), "gelios_synchronize")

    # ------------------------------------------------------------ state
    def set_par(self, buf: int, st: np.ndarray):
        """Cell::par[buf] = rows (ro, p, u, v, Q) of st (shape (5, n_cells))."""
        st = np.ascontiguousarray(st, np.float64)
        rows = [np.ascontiguousarray(st[k]) for k in range(5)]
        N.check(self._L.gelios_upload_state(self._h, int(buf), *rows), "gelios_upload_state")

    def par(self, buf: int, out: np.ndarray | None = None) -> np.ndarray:
        """Cell::par[buf] as rows (ro, p, u, v, Q); written into `out`
        (shape (5, n_cells), C-contiguous, e.g. pinned host memory) if given."""
        if out is None:
            out = np.zeros((5, self.mesh.n_cells))
        rows = [out[k] for k in range(5)]
        N.check(self._L.gelios_download_state(self._h, int(buf), *rows), "gelios_download_state")
        return out

    def set_mc(self, Hn, Hu, Hv, HT, ku, kv, kT):
        """Monte-Carlo moments of par[0] (H_n/H_u/H_v/H_T[4], k_u/k_v/k_T)."""
        f = lambda a: np.ascontiguousarray(a, np.float64).ravel()  # noqa: E731
        self._mc = (Hn, Hu, Hv, HT, ku, kv, kT)
        N.check(self._L.gelios_upload_mc(self._h, f(Hn), f(Hu), f(Hv), f(HT), f(ku), f(kv), f(kT)),
                "gelios_upload_mc")

    def points(self) -> tuple[np.ndarray, np.ndarray]:
        x = np.zeros(self.mesh.n_points)
        y = np.zeros(self.mesh.n_points)
        N.check(self._L.gelios_download_points(self._h, x, y), "gelios_download_points")
        return x, y

    def set_phase_timing(self, on: bool):
        N.check(self._L.gelios_set_phase_timing(self._h, int(bool(on))), "gelios_set_phase_timing")

    def phase_times(self, reset: bool = True) -> dict:
        """Per-phase device ms and launch counts accumulated while timing was on."""
        ms = np.zeros(5)
        ln = np.zeros(5, np.int64)
        N.check(self._L.gelios_phase_times(self._h, ms, ln, int(bool(reset))), "gelios_phase_times")
        names = ("centroids", "faces", "motion", "cells", "commit_dt")
        return {names[k]: (float(ms[k]), int(ln[k])) for k in range(5)}

    def launches(self) -> int:
        return int(self._L.gelios_last_launch_count(self._h))

    def stream_handle(self) -> int:
        return int(self._L.gelios_stream(self._h) or 0)


def hllc_batch(params: N.GeliosParams, rows: np.ndarray) -> np.ndarray:
    """Device HLLC_2d_Korolkov_b_s over rows of 16 inputs -> rows of 9 outputs."""
    rows = np.ascontiguousarray(rows, np.float64)
    out = np.zeros((len(rows), 9))
    N.check(N.lib().gelios_hllc_batch(C.byref(params), len(rows), rows.ravel(), out.ravel()), "gelios_hllc_batch")
    return out


def godunov_batch(params: N.GeliosParams, rows: np.ndarray) -> np.ndarray:
    """Device Godunov_Solver_Alexashov over rows of 15 inputs -> rows of 10 outputs."""
    rows = np.ascontiguousarray(rows, np.float64)
    out = np.zeros((len(rows), 10))
    N.check(N.lib().gelios_godunov_batch(C.byref(params), len(rows), rows.ravel(), out.ravel()),
            "gelios_godunov_batch")
    return out


def hlldq_batch(params: N.GeliosParams, rows: np.ndarray) -> np.ndarray:
    """Device HLLDQ_Korolkov (Solvers.cpp:1642-2185) over rows of 23 inputs
    (L[9], R[9], n[3], rad, metod) -> rows of 10 outputs (time, P[8], PQ)."""
    rows = np.ascontiguousarray(rows, np.float64)
    out = np.zeros((len(rows), 10))
    N.check(N.lib().gelios_hlldq_batch(C.byref(params), len(rows), rows.ravel(), out.ravel()),
            "gelios_hlldq_batch")
    return out


def hlld_batch(params: N.GeliosParams, rows: np.ndarray) -> np.ndarray:
    """Device HLLD_Solver_Alexashov (Solvers.cpp:92-691) over rows of 21
    inputs (q1[8], q2[8], n[3], w, dist) -> rows of 13 outputs (time, q[8],
    dsl, dsp, dsc, status)."""
    rows = np.ascontiguousarray(rows, np.float64)
    out = np.zeros((len(rows), 13))
    N.check(N.lib().gelios_hlld_batch(C.byref(params), len(rows), rows.ravel(), out.ravel()),
            "gelios_hlld_batch")
    return out
