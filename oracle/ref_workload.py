"""Test infrastructure: the rail-grid workloads built on the reference side.

The reference arm and the CPU-baseline leg of ``bench.py`` time the
reference's own step on the same workload as the CUDA path.  This module
builds that workload from the compiled reference and numpy alone (it imports
nothing from ``gelios_2d_b200`` and loads no library of the product):

* the grid: the reference's constructor ``Setka::Setka(N1..M4)``
  (Setka.cpp:19-1076) and ``Setka::TVD_prepare`` (Setka.cpp:1294-1492) in
  ``oracle/_ref/libgelios_ref_fast.so`` (the constructor's tracked-line sort
  runs once, see ``hoist_line_sort.py``; the grid is identical);
* the initial field: the reference's ``Setka::Init_conditions``
  (Setka.cpp:5149-5203);
* the seeded inputs the reference does not make itself (Monte-Carlo moments,
  hydrogen fluids, the MHD form's extra rows and sources): the same seeded
  formulas as the product's workload generator, restated here over the
  reference's cell centroids.  ``tests/test_oracle_pin.py`` checks that both
  sides produce identical arrays.
"""
from __future__ import annotations

import numpy as np

from . import ref

RR_ = 390.222


def splitmix64(seed: int, n: int) -> np.ndarray:
    """n uniform doubles in [0, 1) from the splitmix64 sequence of `seed`."""
    with np.errstate(over="ignore"):
        i = np.arange(1, n + 1, dtype=np.uint64)
        z = np.uint64(seed) + i * np.uint64(0x9E3779B97F4A7C15)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        z = z ^ (z >> np.uint64(31))
    return (z >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)


def centroids(m: dict) -> tuple[np.ndarray, np.ndarray]:
    """Cell::Get_Center (Cell.cpp:66-88): polygon centroid, vertex by vertex
    in contour order."""
    x, y = m["x"], m["y"]
    cs, con = m["contour_start"], m["contour"]
    nv = np.diff(cs)
    cx = np.zeros(len(nv))
    cy = np.zeros(len(nv))
    for n in np.unique(nv):
        cells = np.nonzero(nv == n)[0]
        idx = con[cs[cells][:, None] + np.arange(n)[None, :]]
        A = np.zeros(len(cells))
        gx = np.zeros(len(cells))
        gy = np.zeros(len(cells))
        for i in range(n):
            a, b = idx[:, i], idx[:, (i + 1) % n]
            cr = x[a] * y[b] - y[a] * x[b]
            A = A + cr
            gx = gx + (x[a] + x[b]) * cr
            gy = gy + (y[a] + y[b]) * cr
        A = A * 0.5
        cx[cells] = gx / (6.0 * A)
        cy[cells] = gy / (6.0 * A)
    return cx, cy


def mc_fields(x: np.ndarray, y: np.ndarray, seed: int) -> tuple:
    """Seeded smooth Monte-Carlo moments at cell centroids (x, y): density
    A_s exp(-r/R_s)(1 + 0.1 cos(k_s theta)) of four hydrogen sorts, their
    velocities and temperatures, correction factors k_u, k_v, k_T ~ 1."""
    r = np.sqrt(x * x + y * y)
    th = np.arctan2(y, x)
    u = splitmix64(seed, 32)
    n = len(x)
    Hn, Hu, Hv, HT = (np.zeros((n, 4)) for _ in range(4))
    for s in range(4):
        A = 0.05 + 0.15 * u[4 * s]
        R = 1.0 + 3.0 * u[4 * s + 1]
        k = 1 + int(3 * u[4 * s + 2])
        Hn[:, s] = A * np.exp(-r / R) * (1.0 + 0.1 * np.cos(k * th))
        Hu[:, s] = -2.54338 * (0.8 + 0.4 * u[4 * s + 3]) * (1.0 + 0.05 * np.cos(k * th))
        Hv[:, s] = 0.1 * np.sin(k * th) * u[16 + s]
        HT[:, s] = 0.5 + u[20 + s] * (1.0 + 0.1 * np.cos(th))
    ku = 0.9 + 0.2 * u[24] * (1.0 + 0.1 * np.cos(th))
    kv = 0.9 + 0.2 * u[25] * (1.0 + 0.1 * np.cos(2 * th))
    kT = 0.9 + 0.2 * u[26] * (1.0 + 0.1 * np.cos(3 * th))
    return Hn, Hu, Hv, HT, ku, kv, kT


def hydrogen_fields(x: np.ndarray, y: np.ndarray, seed: int) -> np.ndarray:
    """Seeded smooth rows ro, p, u, v of the hydrogen fluids H1..H4, shape
    (16, n_cells), at cell centroids (x, y)."""
    r = np.sqrt(x * x + y * y)
    th = np.arctan2(y, x)
    u = splitmix64(seed, 24)
    h = np.zeros((16, len(x)))
    for k in range(4):
        A = 0.05 + 0.2 * u[4 * k]
        R = 1.0 + 3.0 * u[4 * k + 1]
        mm = 1 + int(3 * u[4 * k + 2])
        ro = A * np.exp(-r / R) * (1.0 + 0.1 * np.cos(mm * th)) + 0.02
        T = 0.4 + 0.2 * u[4 * k + 3]
        h[4 * k + 0] = ro
        h[4 * k + 1] = 0.5 * ro * T * 2.0
        h[4 * k + 2] = -2.54338 * (0.7 + 0.1 * k) * (1.0 + 0.05 * np.cos(th))
        h[4 * k + 3] = 0.1 * np.sin(mm * th) * u[16 + k]
    return h


def counted_cells_mk2(x: np.ndarray, y: np.ndarray) -> int:
    """Cells the moving-grid step updates: centroid radius not below R11_
    (Setka.cpp:10169)."""
    R11 = ref.constants()["R11_"]
    return int(np.count_nonzero(~(np.sqrt(x * x + y * y) < R11)))


class RefWorkload:
    """A rail-grid workload held by the reference: ``S`` (the reference's
    Setka, par[0] = par[1] = Init_conditions), the exported grid ``mesh``,
    the initial state ``st0`` (5, n_cells), the form's seeded extra input
    ``extra`` and the number of cells one step updates."""

    def __init__(self, S, mesh, st0, extra, counted):
        self.S, self.mesh, self.st0, self.extra, self.counted = S, mesh, st0, extra, counted

    @property
    def n_cells(self) -> int:
        return len(self.mesh["cell_type"])

    @property
    def n_faces(self) -> int:
        return len(self.mesh["face_A"])

    @property
    def n_points(self) -> int:
        return len(self.mesh["x"])


def build(dims, form: str = "mk2", seed: int | None = None) -> RefWorkload:
    """The workload of `form` ("mk2", "inner" or "k5") on Setka(*dims): the
    reference's grid, TVD neighbours and initial field, plus the seeded
    Monte-Carlo moments (mk2, inner; seed 9) or hydrogen fluids (k5; seed 3)
    loaded into the reference's cells."""
    S = ref.RefSetka.constructor(*dims, fast=True)
    S.tvd_prepare()
    S.init_conditions()
    m = S.export()
    x, y = centroids(m)
    st0 = S.get_state(0)
    S.set_state(1, st0)
    if form == "k5":
        extra = hydrogen_fields(x, y, 3 if seed is None else seed)
        S.set_hydrogen(0, extra)
        S.set_hydrogen(1, extra)
        counted = counted_cells_mk2(x, y)
    else:
        extra = mc_fields(x, y, 9 if seed is None else seed)
        S.set_mc(*extra)
        counted = counted_cells_mk2(x, y)
        if form == "inner":
            S.build_inner_list()
            inner = S.inner_list()
            counted = int(np.count_nonzero(m["cell_type"][inner] != 5))  # C_centr cells are copied
    return RefWorkload(S, m, st0, extra, counted)
