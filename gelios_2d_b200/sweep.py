"""Batches of independent instances: parameter sweeps over many grids.

An instance is one grid with its own inflow parameters, state and
Monte-Carlo moments; instances never exchange data and each keeps its own
CFL dt (the reference's dt is a minimum over one grid).  A batch therefore
runs every instance on its own context: a step enqueues the captured step
graph of every instance (each on its own streams) before waiting for any, so
the instances' latency-bound kernels fill the GPU together.  Across GPUs the
instances are partitioned by cell count (greedy, largest first) and the
results are gathered on the host: no collective on the step path.
"""
from __future__ import annotations

import numpy as np

from . import _native as N
from .mesh import Mesh
from .setka import Setka


def partition(cell_counts, n_parts: int) -> list[list[int]]:
    """Greedy largest-first assignment of instances to ``n_parts`` GPUs by
    cell count; returns the instance indices of every part (each part in
    increasing index order).  The largest part is at most the mean load plus
    the largest instance."""
    if n_parts < 1:
        raise ValueError("n_parts must be >= 1")
    counts = np.asarray(cell_counts, dtype=np.int64)
    order = sorted(range(len(counts)), key=lambda i: (-int(counts[i]), i))
    load = [0] * n_parts
    parts: list[list[int]] = [[] for _ in range(n_parts)]
    for i in order:
        p = min(range(n_parts), key=lambda q: (load[q], q))
        parts[p].append(i)
        load[p] += int(counts[i])
    return [sorted(p) for p in parts]


class Sweep:
    """Instances stepped together on one GPU.

    ``instances``: sequence of (mesh, params, state (5, n_cells), mc or None).
    """

    def __init__(self, instances, device: int = 0, form: int = N.FORM_MK2, batched: bool = False):
        self.form = form
        self.items: list[Setka] = []
        self._batch = None
        for mesh, params, st0, mc in instances:
            S = Setka(mesh, params, device)
            S.set_par(0, st0)
            S.set_par(1, st0)
            if form == N.FORM_MHD_PUI:
                mp, x0, src = mc  # boundary data, extra rows, fixed sources
                S.set_mhd_params(mp)
                S.set_mhd(0, x0)
                S.set_mhd(1, x0)
                S.set_sources(*src)
            elif mc is not None:
                S.set_mc(*mc)
            self.items.append(S)
        if batched:
            self.enable_batch()

    def enable_batch(self, groups: int = 1):
        """Advance the instances with one launch per phase (gelios_batch, the
        MHD form only), in `groups` batches of about equal cell count, each
        on its own stream so that the batches' phases overlap."""
        import ctypes as C

        if self.form != N.FORM_MHD_PUI:
            raise ValueError("only the MHD form is batched")
        L = N.lib()
        parts = [p for p in partition(self.cells, max(1, min(groups, len(self.items)))) if p]
        self._groups = parts
        self._batch = []
        for p in parts:
            arr = (C.c_void_p * len(p))(*[self.items[i]._h.value for i in p])
            h = C.c_void_p()
            N.check(L.gelios_batch_create(C.byref(h), arr, len(p)), "gelios_batch_create")
            self._batch.append(h)

    def set_batch_schedule(self, schedule: int):
        """0: one launch per phase (a captured graph per step); k > 0: every
        step of a call in one persistent cooperative kernel of k blocks per
        SM (gelios_batch_set_schedule)."""
        import ctypes as C

        L = N.lib()
        for h in self._batch:
            N.check(L.gelios_batch_set_schedule(h, C.c_int32(int(schedule))), "gelios_batch_set_schedule")

    def batch_schedules(self) -> list[int]:
        import ctypes as C

        L = N.lib()
        out = []
        for h in self._batch:
            v = C.c_int32()
            N.check(L.gelios_batch_get_schedule(h, C.byref(v)), "gelios_batch_get_schedule")
            out.append(v.value)
        return out

    def autotune_batch(self, steps: int = 2) -> list[tuple[int, float, list[float]]]:
        """Per batch: time the per-phase schedule and the persistent kernel
        at every co-resident block count on `steps` real steps each (they
        advance the instances) and keep the fastest.  Returns (schedule,
        ms per step, ms per step of every schedule 0..15 that ran) per batch."""
        import ctypes as C

        L = N.lib()
        res = []
        for h in self._batch:
            v, ms = C.c_int32(), C.c_double()
            each = (C.c_double * 16)()
            N.check(L.gelios_batch_autotune(h, int(steps), C.byref(v), C.byref(ms), C.cast(each, C.c_void_p), 16),
                    "gelios_batch_autotune")
            res.append((v.value, ms.value, [x for x in each if x >= 0.0]))
        return res

    def batch_step(self, n: int = 1, statuses: bool = False):
        """n batched steps; with statuses=True waits and returns the
        instances' statuses (in instance order)."""
        L = N.lib()
        out = [None] * len(self.items)
        for h, p in zip(self._batch, self._groups):
            if statuses:
                st = (N.GeliosStatus * len(p))()
                N.check(L.gelios_batch_step(h, self.form, int(n), st), "gelios_batch_step")
                for k, i in enumerate(p):
                    out[i] = st[k]
            else:
                N.check(L.gelios_batch_step(h, self.form, int(n), None), "gelios_batch_step")
        return out if statuses else None

    def __len__(self) -> int:
        return len(self.items)

    @property
    def cells(self) -> list[int]:
        return [S.mesh.n_cells for S in self.items]

    def autotune(self, reps: int = 3) -> list[tuple[int, float]]:
        """Per-instance schedule: every instance gets the launch shape of its
        dominant kernel that is fastest on its own grid (gelios_autotune),
        and the batch enqueues instances in decreasing order of their tuned
        kernel time, so the longest start first and the short ones fill in
        behind them.  Returns (variant, ms) per instance."""
        res = [S.autotune(self.form, reps) for S in self.items]
        self.order = sorted(range(len(self.items)), key=lambda i: (-res[i][1], i))
        return res

    def step_async(self, n: int = 1):
        """Enqueue ``n`` steps on every instance without waiting."""
        if self._batch is not None:
            self.batch_step(n)
            return
        for i in getattr(self, "order", range(len(self.items))):
            self.items[i].step_async(self.form, n)

    def synchronize(self):
        for S in self.items:
            S.synchronize()

    def step(self, n: int = 1):
        """``n`` steps of every instance, then wait for all."""
        self.step_async(n)
        self.synchronize()

    def par(self, i: int, buf: int) -> np.ndarray:
        return self.items[i].par(buf)

    def close(self):
        if self._batch is not None:
            for h in self._batch:
                N.lib().gelios_batch_destroy(h)
            self._batch = None
        for S in self.items:
            S.close()
        self.items = []


BASE_DIMS = (200, 100, 50, 100, 100, 100, 150, 150)  # Setka(N1..M4) of ~200k cells
MIN_DIMS = (8, 4, 3, 6, 23, 6, 7, 7)  # the constructor needs M1 > n_inner = 20


def instance_set(n: int, seed: int = 41, scale=(0.5, 1.4), only=None) -> list[tuple]:
    """``n`` seeded instances of the moving-grid step with uneven grids: the
    rail grid Setka(N1..M4) of ~200k cells with every count scaled by a
    seeded factor in ``scale`` (cells grow with its square: 0.5..1.4 gives
    ~50k..~400k cells, the sweep configuration's range), each with the
    reference's initial field and its own Monte-Carlo moments.  ``only``
    builds just those instance indices (the others' seeds are unchanged)."""
    from . import workloads as W

    u = W.splitmix64(seed, n)
    out = []
    for i in (range(n) if only is None else only):
        f = scale[0] + (scale[1] - scale[0]) * float(u[i])
        dims = tuple(max(lo, int(round(b * f))) for b, lo in zip(BASE_DIMS, MIN_DIMS))
        mesh = Mesh.setka(*dims)
        params = N.reference_params()
        out.append((mesh, params, W.init_conditions_reference(mesh), W.mc_fields(mesh, seed=seed + i)))
    return out


def inflow_params(u: np.ndarray) -> dict:
    """Inflow of one MHD sweep instance from five uniform draws: LISM speed
    U(0.04, 0.08) and density U(0.002, 0.01) in units of the wind at 1 AU,
    Mach U(1.5, 3), |B| U(0, 0.02), field angle to the inflow U(0, 60 deg).
    Speeds and densities map to the grid's units through the inner-sphere
    wind (speed chi, density 116.667 at 1 AU: Setka::Init_conditions,
    Setka.cpp:5149-5203); the inflow runs along -x."""
    chi, ro_wind = 36.1275, 116.667
    g = 5.0 / 3.0
    u_lism = 0.04 + 0.04 * float(u[0])
    ro_lism = 0.002 + 0.008 * float(u[1])
    mach = 1.5 + 1.5 * float(u[2])
    ro = ro_wind * ro_lism
    vel = chi * u_lism
    return {"in_ro": ro, "in_u": -vel, "in_p": ro * vel * vel / (g * mach * mach),
            "b_lism": 0.02 * float(u[3]), "b_angle_deg": 60.0 * float(u[4])}


def instance_set_mhd(n: int, seed: int = 43, scale=(0.5, 1.4), only=None) -> list[tuple]:
    """``n`` seeded instances of the MHD + pickup-proton step: uneven rail
    grids as in :func:`instance_set`, each with its own inflow
    (:func:`inflow_params`): the Input boundary state, the LISM cells of the
    reference's initial field set to it, its LISM field, seeded fixed
    charge-exchange sources.  Returns (mesh, params, state, (mhd params,
    extra rows, sources)) per instance."""
    from . import workloads as W

    u = W.splitmix64(seed, n)
    draws = W.splitmix64(seed + 1, 5 * n).reshape(n, 5)
    out = []
    for i in (range(n) if only is None else only):
        f = scale[0] + (scale[1] - scale[0]) * float(u[i])
        dims = tuple(max(lo, int(round(b * f))) for b, lo in zip(BASE_DIMS, MIN_DIMS))
        mesh = Mesh.setka(*dims)
        inflow = inflow_params(draws[i])
        params = N.reference_params(in_ro=inflow["in_ro"], in_p=inflow["in_p"], in_u=inflow["in_u"])
        st0 = W.init_conditions_reference(mesh)
        lism = mesh["cell_type"] == 4  # C_5, the cells Init_conditions fills with the inflow state
        st0[0][lism], st0[1][lism], st0[2][lism], st0[3][lism] = (inflow["in_ro"], inflow["in_p"],
                                                                  inflow["in_u"], 0.0)
        mp = W.mhd_params(b_lism=inflow["b_lism"], b_angle_deg=inflow["b_angle_deg"])
        out.append((mesh, params, st0, (mp, W.mhd_initial(mesh, st0, mp), W.mhd_sources(mesh, seed=seed + i))))
    return out


def gather_results(local: dict, dist=None) -> dict | None:
    """Merge every rank's {instance index: result} on rank 0 (host-side
    gather; None on the other ranks).  Without a process group the local
    results are returned."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return dict(local)
    parts = [None] * dist.get_world_size() if dist.get_rank() == 0 else None
    dist.gather_object(local, parts, dst=0)
    if dist.get_rank() != 0:
        return None
    merged: dict = {}
    for p in parts:
        dup = set(merged) & set(p)
        if dup:
            raise ValueError(f"instances reported by two ranks: {sorted(dup)}")
        merged.update(p)
    return merged
