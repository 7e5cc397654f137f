"""Synthetic workloads of the plasma step (seeded, no external data).

* ``plain_single_fluid``: the axisymmetric half-plane polar grid, 180 rays
  uniform in polar angle x 120 log-spaced radial cells (r = 1..600), gamma
  5/3, inner boundary rho=1, u_r=1, Mach 10, outer inflow along -x rho=0.005,
  u=0.06, Mach 2; initial field = inner solution for r < 150 and the inflow
  state beyond, with seeded +-1% uniform density noise; CFL 0.4; stepped with
  the Go_stationary form.
* ``moving_grid``: the reference's rail grid ``Setka(N1..M4)`` with its own
  initial field (Init_conditions) and seeded smooth Monte-Carlo moments
  (hydrogen densities, velocities, temperatures and correction factors) that
  the charge-exchange source Get_Sourse_MK1 interpolates; stepped with the
  Go_5_komponent__MK2 form (surface tracking + rail motion).
"""
from __future__ import annotations

import numpy as np

from . import _native as N
from .mesh import C_2, C_3, C_4, C_5, Mesh

RR_ = 390.222

# Grid sizes of the moving-grid workloads, N1..M4 of Setka(N1..M4):
# ~200k cells (400 rays x ~500 radial cells) and ~1M cells.
SETKA_200K = (200, 100, 50, 100, 100, 100, 150, 150)
SETKA_1M = (480, 240, 100, 220, 200, 200, 300, 300)
SETKA_SMALL = (30, 7, 11, 20, 60, 20, 40, 40)


def splitmix64(seed: int, n: int) -> np.ndarray:
    """n uniform doubles in [0, 1) from the splitmix64 sequence of `seed`."""
    with np.errstate(over="ignore"):
        i = np.arange(1, n + 1, dtype=np.uint64)
        z = np.uint64(seed) + i * np.uint64(0x9E3779B97F4A7C15)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        z = z ^ (z >> np.uint64(31))
    return (z >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)


# ---------------------------------------------------------------- plain single fluid
def plain_params(**over) -> N.GeliosParams:
    """Parameters of the plain single-fluid workload (Go_stationary form)."""
    g = 5.0 / 3.0
    ro_in, u_in, mach_in = 0.005, 0.06, 2.0
    p = N.reference_params(gamma=g, kurant=0.4, chi=1.0, inner_mach=10.0, in_ro=ro_in,
                           in_p=ro_in * u_in * u_in / (g * mach_in * mach_in), in_u=-u_in, in_v=0.0,
                           in_Q=100.0)
    for k, v in over.items():
        setattr(p, k, v)
    return p


def plain_mesh(n_theta=180, n_r=120, r_in=1.0, r_out=600.0) -> Mesh:
    return Mesh.polar(n_theta, n_r, r_in, r_out)


def plain_initial(mesh: Mesh, params: N.GeliosParams, seed: int = 2024, r_switch: float = 150.0) -> np.ndarray:
    """Inner solution (rho ~ r^-2, u_r = 1, p ~ r^-2gamma) inside r_switch,
    inflow state outside, density times (1 + 0.01 (2U - 1))."""
    c = mesh.centroids()
    x, y = c
    r = np.sqrt(x * x + y * y)
    g = params.gamma
    p0 = 1.0 / (g * params.inner_mach ** 2)
    st = np.zeros((5, mesh.n_cells))
    inner = r < r_switch
    st[0] = np.where(inner, 1.0 / r ** 2, params.in_ro)
    st[1] = np.where(inner, p0 * r ** (-2.0 * g), params.in_p)
    st[2] = np.where(inner, x / r, params.in_u)
    st[3] = np.where(inner, y / r, params.in_v)
    st[4] = np.where(inner, st[0], params.in_Q)
    st[0] *= 1.0 + 0.01 * (2.0 * splitmix64(seed, mesh.n_cells) - 1.0)
    return st


# ---------------------------------------------------------------- moving grid
def init_conditions_reference(mesh: Mesh) -> np.ndarray:
    """Setka::Init_conditions (Setka.cpp:5149-5203): the reference's initial
    field by cell type."""
    x, y = mesh.centroids()
    dist = np.sqrt(x * x + y * y)
    t = mesh["cell_type"]
    g = 5.0 / 3.0
    v_inf, vel_inf = 2.54338, -2.54338
    rr = 1.0 / RR_
    roe, pe, Ve = 116.667, 913.546, 36.1275
    st = np.zeros((5, mesh.n_cells))
    st[4] = 100.0
    c5 = t == C_5
    st[0][c5], st[1][c5], st[2][c5], st[3][c5] = 1.0, 1.0, vel_inf, 0.0
    c4 = t == C_4
    xx = x - 1300.0 / RR_
    yy = y - 0.0
    n = np.sqrt(xx * xx + yy * yy)
    st[0][c4], st[1][c4] = 2.0, 7.0
    st[2][c4] = (0.25 * v_inf * (xx / n))[c4]
    st[3][c4] = (0.25 * v_inf * (yy / n))[c4]
    c23 = (t == C_3) | (t == C_2)
    st[0][c23], st[1][c23] = 1.0 / 20.0, 10.0
    st[2][c23] = (0.1 * Ve * x / dist)[c23]
    st[3][c23] = (0.1 * Ve * y / dist)[c23]
    rest = ~(c5 | c4 | c23)
    st[0][rest] = (roe * (rr / dist) ** 2)[rest]
    st[1][rest] = (pe * (rr / dist) ** (2.0 * g))[rest]
    st[2][rest] = (Ve * x / dist)[rest]
    st[3][rest] = (Ve * y / dist)[rest]
    return st


def mc_fields(mesh: Mesh, seed: int = 7) -> tuple:
    """Seeded smooth Monte-Carlo moments per cell: four hydrogen sorts with
    density A_s exp(-r/R_s)(1 + 0.1 cos(k_s theta)), LISM-like velocity,
    temperature ~ 1, and correction factors k_u, k_v, k_T ~ 1.
    Returns (Hn, Hu, Hv, HT) of shape (n_cells, 4) and (ku, kv, kT)."""
    x, y = mesh.centroids()
    r = np.sqrt(x * x + y * y)
    th = np.arctan2(y, x)
    u = splitmix64(seed, 32)
    Hn = np.zeros((mesh.n_cells, 4))
    Hu = np.zeros((mesh.n_cells, 4))
    Hv = np.zeros((mesh.n_cells, 4))
    HT = np.zeros((mesh.n_cells, 4))
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


def counted_cells_mk2(mesh: Mesh, params: N.GeliosParams) -> int:
    """Cells the MK2 form updates (centroid radius >= R11, Setka.cpp:10169)."""
    x, y = mesh.centroids()
    return int(np.count_nonzero(~(np.sqrt(x * x + y * y) < params.R11)))


def counted_cells_stationary(mesh: Mesh) -> int:
    """Cells Go_stationary updates (all but C_centr, Setka.cpp:5239)."""
    return int(np.count_nonzero(mesh["cell_type"] != 5))


def hydrogen_fields(mesh: Mesh, seed: int = 31) -> np.ndarray:
    """Seeded smooth state of the four hydrogen fluids H1..H4 (rows ro, p, u,
    v of each, shape (16, n_cells)) for the four-fluid step: densities
    A_k exp(-r/R_k)(1 + 0.1 cos(m_k theta)) + 0.02, temperatures ~ 0.5,
    LISM-directed velocities with a small angular modulation."""
    x, y = mesh.centroids()
    r = np.sqrt(x * x + y * y)
    th = np.arctan2(y, x)
    u = splitmix64(seed, 24)
    h = np.zeros((16, mesh.n_cells))
    for k in range(4):
        A = 0.05 + 0.2 * u[4 * k]
        R = 1.0 + 3.0 * u[4 * k + 1]
        m = 1 + int(3 * u[4 * k + 2])
        ro = A * np.exp(-r / R) * (1.0 + 0.1 * np.cos(m * th)) + 0.02
        T = 0.4 + 0.2 * u[4 * k + 3]
        h[4 * k + 0] = ro
        h[4 * k + 1] = 0.5 * ro * T * 2.0
        h[4 * k + 2] = -2.54338 * (0.7 + 0.1 * k) * (1.0 + 0.05 * np.cos(th))
        h[4 * k + 3] = 0.1 * np.sin(m * th) * u[16 + k]
    return h


# ---------------------------------------------------------------- ion MHD + pickup protons
def mhd_params(b_lism: float = 0.01, b_angle_deg: float = 30.0, inner_bphi: float = 1.0) -> N.GeliosMhdParams:
    """Boundary data of the MHD + pickup-proton form: LISM field of magnitude
    b_lism at b_angle_deg to the inflow (the inflow runs along -x), a toroidal
    wind field inner_bphi * R1 sin(theta) / r at the inner sphere, pickup
    protons at 1% of the wind density and 10% of its pressure there and a
    trace population (1e-3) in the inflow."""
    a = np.deg2rad(b_angle_deg)
    mp = N.GeliosMhdParams()
    mp.lism_bx = -b_lism * np.cos(a)
    mp.lism_by = b_lism * np.sin(a)
    mp.lism_bz = 0.0
    mp.inner_bphi = inner_bphi
    mp.pui_in_ro = 1e-3
    mp.pui_in_p = 1e-3
    mp.pui_inner_ro = 0.01
    mp.pui_inner_p = 0.1
    return mp


def mhd_initial(mesh: Mesh, st0: np.ndarray, mp: N.GeliosMhdParams) -> np.ndarray:
    """Extra rows of the MHD form (shape (8, n_cells)) beside the ion state
    st0: no azimuthal velocity; the uniform LISM field everywhere plus the
    wind's toroidal field inner_bphi * R1 sin(theta) / r (both divergence
    free; cells inside R11 keep it as the inner boundary the step does not
    update); pickup protons at 1% of the ion density and 10% of its
    pressure, moving with the ions."""
    x, y = mesh.centroids()
    r2 = x * x + y * y
    x8 = np.zeros((8, mesh.n_cells))
    x8[1] = mp.lism_bx
    x8[2] = mp.lism_by
    x8[3] = mp.lism_bz + mp.inner_bphi * (1.0 / RR_) * y / r2
    x8[4] = 0.01 * st0[0]
    x8[5] = 0.1 * st0[1]
    x8[6] = st0[2]
    x8[7] = st0[3]
    return x8


def mhd_sources(mesh: Mesh, seed: int = 17) -> tuple:
    """Fixed charge-exchange sources of the ion x momentum, y momentum and
    energy: A_i exp(-r/200) (1 + 0.1 cos(k_i theta)) with r in AU (r * 390.222
    in grid units), A_i ~ U(5e-4, 2e-3), k_i in {1, 2, 3}, seeded."""
    x, y = mesh.centroids()
    r = np.sqrt(x * x + y * y) * RR_
    th = np.arctan2(y, x)
    u = splitmix64(seed, 6)
    out = []
    for i in range(3):
        A = 5e-4 + 1.5e-3 * u[2 * i]
        k = 1 + int(3 * u[2 * i + 1])
        out.append(A * np.exp(-r / 200.0) * (1.0 + 0.1 * np.cos(k * th)))
    return tuple(out)
