"""Test infrastructure: ctypes access to the compiled reference (oracle/_ref).

``libgelios_ref.so`` is the unmodified SergeyMSU/Gelios_2D C++ sources plus
``ref_harness.cpp`` (built by ``oracle/Makefile``).  Only the tests, the smoke
check and the CPU-baseline leg of ``bench.py`` use this module; the product
never imports it.

Mesh dictionaries use the unified face numbering of the harness: main faces
(``All_Gran`` order) first, then copies (``All_Gran_copy`` order); cells in
``All_Cells`` order; points in ``All_Points`` order.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REF_DIR = HERE / "_ref"

_i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
_i64p = np.ctypeslib.ndpointer(np.int64, flags="C_CONTIGUOUS")


def _load(name: str) -> C.CDLL:
    path = REF_DIR / name
    if not path.exists():
        raise FileNotFoundError(f"{path} missing: run `make -C oracle` where the reference tree exists")
    return C.CDLL(str(path))


_LIBS: dict[str, C.CDLL] = {}


def lib(fast: bool = False) -> C.CDLL:
    name = "libgelios_ref_fast.so" if fast else "libgelios_ref.so"
    if name in _LIBS:
        return _LIBS[name]
    L = _configure(_load(name))
    _LIBS[name] = L
    return L


def shim_lib() -> C.CDLL:
    """The parity build of the reference plus include/gelios_setka_shim.hpp
    (oracle/shim_harness.cpp), linked against the product library: loads
    gelios_2d_b200/_lib/libgelios_b200.so.  Tests only."""
    name = "libgelios_shim.so"
    if name in _LIBS:
        return _LIBS[name]
    L = _configure(_load(name))
    vp = C.c_void_p
    L.gshim_mirror_check.argtypes = [vp, C.c_char_p, C.c_int]
    L.gshim_new.restype = vp
    L.gshim_free.argtypes = [vp]
    L.gshim_step.argtypes = [vp, vp, C.c_int, C.c_int]
    _LIBS[name] = L
    return L


def _configure(L: C.CDLL) -> C.CDLL:
    vp = C.c_void_p
    L.gref_setka_new.restype = vp
    L.gref_setka_new.argtypes = [C.c_int] * 8
    L.gref_set_hydrogen.argtypes = [vp, C.c_int, _f64p]
    L.gref_get_hydrogen.argtypes = [vp, C.c_int, _f64p]
    L.gref_go_5_komponent.argtypes = [vp, C.c_int]
    L.gref_save_alpha.argtypes = [vp, C.c_char_p]
    L.gref_load_alpha.restype = vp
    L.gref_load_alpha.argtypes = [C.c_char_p]
    L.gref_setka_from_arrays.restype = vp
    L.gref_setka_from_arrays.argtypes = [
        _i32p,
        C.c_int, _f64p, _f64p, _i32p,
        C.c_int, _i32p, _i32p, _i32p, _i32p, _i32p,
        C.c_int, C.c_int, _i32p, _i32p, _i32p, _i32p, _i32p, _i32p, _i32p,
        C.c_int, _i32p, _f64p, _i32p, _i32p, _i32p, _i32p, _i32p,
        C.c_int, _i32p, C.c_int, _i32p, C.c_int, _i32p,
    ]
    L.gref_counts.argtypes = [vp, _i64p]
    L.gref_export_points.argtypes = [vp, _f64p, _f64p, _f64p, _f64p, _i32p]
    L.gref_export_cells.argtypes = [vp, _i32p, _i32p, _i32p, _i32p, _i32p, _i32p, _i32p, _f64p]
    L.gref_export_faces.argtypes = [vp] + [_i32p] * 9
    L.gref_export_rails.argtypes = [vp, _i32p, _f64p, _i32p, _i32p, _i32p, _i32p, _i32p]
    L.gref_export_lines.argtypes = [vp, _i32p, _i32p, _i32p]
    L.gref_export_inner_list.argtypes = [vp, _i32p]
    for f in ("gref_tvd_prepare", "gref_init_conditions", "gref_build_inner_list"):
        getattr(L, f).argtypes = [vp]
    L.gref_set_state.argtypes = [vp, C.c_int] + [_f64p] * 5
    L.gref_get_state.argtypes = [vp, C.c_int] + [_f64p] * 5
    L.gref_set_mc.argtypes = [vp] + [_f64p] * 7
    L.gref_get_point_motion.argtypes = [vp] + [_f64p] * 6 + [_i32p]
    L.gref_set_points.argtypes = [vp, _f64p, _f64p]
    for f in ("gref_go_stationary", "gref_go_mk2", "gref_go_inner_mk2"):
        getattr(L, f).argtypes = [vp, C.c_int]
    L.gref_move_surface.argtypes = [vp, C.c_int, C.c_double]
    L.gref_move_setka2.argtypes = [vp, C.c_double]
    L.gref_face_par.argtypes = [vp, C.c_int, C.c_int, C.c_int, _f64p]
    L.gref_cell_geom.argtypes = [vp, C.c_int, _f64p]
    L.gref_source_mk1.argtypes = [vp, C.c_int] + [C.c_double] * 4 + [_f64p]
    L.gref_hllc.restype = C.c_double
    L.gref_hllc.argtypes = [C.c_double] * 11 + [_f64p, _f64p, C.c_double, C.c_double, C.c_double,
                                                 C.c_int, _f64p, C.c_int]
    L.gref_godunov.restype = C.c_double
    L.gref_godunov.argtypes = [_f64p, _f64p, _f64p, _f64p, _f64p, C.c_double, C.c_double]
    L.gref_hlldq.restype = C.c_double
    L.gref_hlldq.argtypes = [_f64p, _f64p, _f64p, _f64p, _f64p, C.c_double, C.c_int]
    L.gref_hlld.restype = C.c_double
    L.gref_hlld.argtypes = [_f64p, _f64p, _f64p, _f64p, _f64p, C.c_double, C.c_double]
    L.gref_constants.argtypes = [_f64p]
    L.gref_set_threads.argtypes = [C.c_int]
    L.gref_max_threads.restype = C.c_int
    L.gref_set_threads(1)
    return L


def set_threads(n: int, fast: bool = False) -> None:
    """OpenMP threads of the reference loops (1 = parity mode)."""
    lib(fast).gref_set_threads(int(n))


def max_threads() -> int:
    return int(lib().gref_max_threads())


def available() -> bool:
    return (REF_DIR / "libgelios_ref.so").exists()


def constants() -> dict:
    out = np.zeros(18)
    lib().gref_constants(out)
    keys = ["ga", "kurant", "Velosity_inf", "chi_real", "RR_", "R1_", "R11_", "R111_", "R2_", "R3_",
            "R4_", "R5_", "Left_", "Kn_", "a_2", "n_p_LISM_", "n_inner", "n_outer_shock"]
    return dict(zip(keys, out.tolist()))


class RefSetka:
    """A reference ``Setka`` held through the harness."""

    def __init__(self, handle: int, L: C.CDLL, dims=(0,) * 8):
        self.h = C.c_void_p(handle)
        self.L = L
        self.dims = tuple(int(d) for d in dims)

    # ------------------------------------------------------------ construction
    @classmethod
    def constructor(cls, N1, N2, N3, N4, M1, M2, M3, M4, fast=False, L=None) -> "RefSetka":
        L = L or lib(fast)
        return cls(L.gref_setka_new(N1, N2, N3, N4, M1, M2, M3, M4), L, (N1, N2, N3, N4, M1, M2, M3, M4))

    @classmethod
    def load_alpha(cls, path, fast=False) -> "RefSetka":
        """Setka::Download_Setka_ALL_ALPHA_2_0 (Setka.cpp:2899-3257) into a fresh Setka."""
        L = lib(fast)
        with open(path) as f:
            dims = tuple(int(t) for t in f.readline().split()[:8])
        return cls(L.gref_load_alpha(str(path).encode()), L, dims)

    def save_alpha(self, path):
        """Setka::Save_Setka_ALL_ALPHA (Setka.cpp:2355-2574)."""
        self.L.gref_save_alpha(self.h, str(path).encode())

    @classmethod
    def from_mesh(cls, m: dict, fast=False) -> "RefSetka":
        L = lib(fast)
        i32 = lambda a: np.ascontiguousarray(a, dtype=np.int32)  # noqa: E731
        f64 = lambda a: np.ascontiguousarray(a, dtype=np.float64)  # noqa: E731
        dims = i32(m.get("dims", np.zeros(8)))
        nrail = len(m["rail_type"])
        empty_i = np.zeros(1, np.int32)
        h = L.gref_setka_from_arrays(
            dims,
            len(m["x"]), f64(m["x"]), f64(m["y"]), i32(m["point_type"]),
            len(m["cell_type"]), i32(m["cell_type"]), i32(m["contour_start"]), i32(m["contour"]),
            i32(m["gran_start"]), i32(m["gran"]),
            int(m["n_main"]), len(m["face_A"]) - int(m["n_main"]), i32(m["face_A"]), i32(m["face_B"]),
            i32(m["face_type"]), i32(m["face_master"]), i32(m["face_sosed"]), i32(m["face_copy"]),
            i32(m["face_main"] if "face_main" in m else (np.arange(len(m["face_A"])) < int(m["n_main"]))),
            nrail, i32(m["rail_type"]) if nrail else empty_i, f64(m["rail_s"]) if nrail else np.zeros(1),
            i32(m["rail_M"]) if nrail else empty_i, i32(m["rail_pstart"]), i32(m["rail_points"]) if nrail else empty_i,
            i32(m["rail_kstart"]), i32(m["rail_keys"]) if nrail else empty_i,
            len(m["line_contact"]), i32(m["line_contact"]) if len(m["line_contact"]) else empty_i,
            len(m["line_inner"]), i32(m["line_inner"]) if len(m["line_inner"]) else empty_i,
            len(m["line_outer"]), i32(m["line_outer"]) if len(m["line_outer"]) else empty_i,
        )
        return cls(h, L, tuple(int(d) for d in dims))

    # ------------------------------------------------------------ queries
    def counts(self) -> dict:
        out = np.zeros(16, np.int64)
        self.L.gref_counts(self.h, out)
        keys = ["n_points", "n_cells", "n_main", "n_copy", "contour_total", "gran_total", "n_rails",
                "rail_points_total", "rail_keys_total", "n_contact", "n_inner", "n_outer", "n_cells_inner"]
        return {k: int(v) for k, v in zip(keys, out)}

    def export(self) -> dict:
        c = self.counts()
        L, h = self.L, self.h
        npnt, ncell = c["n_points"], c["n_cells"]
        nf = c["n_main"] + c["n_copy"]
        m: dict = {"dims": np.array(self.dims, np.int32), "n_main": c["n_main"]}
        x, y, x2, y2 = (np.zeros(npnt) for _ in range(4))
        pt = np.zeros(npnt, np.int32)
        L.gref_export_points(h, x, y, x2, y2, pt)
        m.update(x=x, y=y, x2=x2, y2=y2, point_type=pt)
        ct = np.zeros(ncell, np.int32)
        cs = np.zeros(ncell + 1, np.int32)
        con = np.zeros(max(c["contour_total"], 1), np.int32)
        gs = np.zeros(ncell + 1, np.int32)
        gr = np.zeros(max(c["gran_total"], 1), np.int32)
        back = np.zeros(ncell, np.int32)
        nxt = np.zeros(ncell, np.int32)
        ri = np.zeros(ncell)
        L.gref_export_cells(h, ct, cs, con, gs, gr, back, nxt, ri)
        m.update(cell_type=ct, contour_start=cs, contour=con[: c["contour_total"]], gran_start=gs,
                 gran=gr[: c["gran_total"]], cell_back=back, cell_next=nxt, r_istoch=ri)
        fa = [np.zeros(max(nf, 1), np.int32) for _ in range(9)]
        L.gref_export_faces(h, *fa)
        names = ["face_A", "face_B", "face_type", "face_master", "face_sosed", "face_copy",
                 "face_sosed_up", "face_sosed_down", "face_main"]
        for k, a in zip(names, fa):
            m[k] = a[:nf]
        nr = c["n_rails"]
        rt = np.zeros(max(nr, 1), np.int32)
        rs = np.zeros(max(nr, 1))
        rM = np.zeros(max(4 * nr, 1), np.int32)
        ps = np.zeros(nr + 1, np.int32)
        pts = np.zeros(max(c["rail_points_total"], 1), np.int32)
        ks = np.zeros(nr + 1, np.int32)
        keys = np.zeros(max(c["rail_keys_total"], 1), np.int32)
        L.gref_export_rails(h, rt, rs, rM, ps, pts, ks, keys)
        m.update(rail_type=rt[:nr], rail_s=rs[:nr], rail_M=rM[: 4 * nr], rail_pstart=ps,
                 rail_points=pts[: c["rail_points_total"]], rail_kstart=ks,
                 rail_keys=keys[: c["rail_keys_total"]])
        lc = np.zeros(max(c["n_contact"], 1), np.int32)
        li = np.zeros(max(c["n_inner"], 1), np.int32)
        lo = np.zeros(max(c["n_outer"], 1), np.int32)
        L.gref_export_lines(h, lc, li, lo)
        m.update(line_contact=lc[: c["n_contact"]], line_inner=li[: c["n_inner"]],
                 line_outer=lo[: c["n_outer"]])
        return m

    def inner_list(self) -> np.ndarray:
        n = self.counts()["n_cells_inner"]
        out = np.zeros(max(n, 1), np.int32)
        self.L.gref_export_inner_list(self.h, out)
        return out[:n]

    # ------------------------------------------------------------ prep / state
    def tvd_prepare(self):
        self.L.gref_tvd_prepare(self.h)

    def init_conditions(self):
        self.L.gref_init_conditions(self.h)

    def build_inner_list(self):
        self.L.gref_build_inner_list(self.h)

    def set_state(self, buf: int, st: np.ndarray):
        """st: (5, ncell) rows ro, p, u, v, Q"""
        st = np.ascontiguousarray(st, dtype=np.float64)
        self.L.gref_set_state(self.h, buf, *[np.ascontiguousarray(st[k]) for k in range(5)])

    def get_state(self, buf: int) -> np.ndarray:
        n = self.counts()["n_cells"]
        out = [np.zeros(n) for _ in range(5)]
        self.L.gref_get_state(self.h, buf, *out)
        return np.stack(out)

    def set_mc(self, Hn, Hu, Hv, HT, ku, kv, kT):
        f = lambda a: np.ascontiguousarray(a, dtype=np.float64).ravel()  # noqa: E731
        self.L.gref_set_mc(self.h, f(Hn), f(Hu), f(Hv), f(HT), f(ku), f(kv), f(kT))

    def point_motion(self) -> dict:
        n = self.counts()["n_points"]
        arrs = [np.zeros(n) for _ in range(6)]
        cnt = np.zeros(n, np.int32)
        self.L.gref_get_point_motion(self.h, *arrs, cnt)
        return dict(zip(["x", "y", "x2", "y2", "Vx", "Vy"], arrs), count=cnt)

    def set_points(self, x, y):
        self.L.gref_set_points(self.h, np.ascontiguousarray(x, np.float64), np.ascontiguousarray(y, np.float64))

    # ------------------------------------------------------------ steps
    def go_stationary(self, steps: int):
        self.L.gref_go_stationary(self.h, int(steps))

    def set_hydrogen(self, buf: int, h16: np.ndarray):
        """ro, p, u, v of H1..H4 in par[buf]; h16 of shape (16, n_cells)."""
        self.L.gref_set_hydrogen(self.h, int(buf), np.ascontiguousarray(h16, np.float64).ravel())

    def get_hydrogen(self, buf: int) -> np.ndarray:
        n = self.counts()["n_cells"]
        out = np.zeros(16 * n)
        self.L.gref_get_hydrogen(self.h, int(buf), out)
        return out.reshape(16, n)

    def go_5_komponent(self, steps: int):
        """Setka::Go_5_komponent (Setka.cpp:8269-8950)."""
        self.L.gref_go_5_komponent(self.h, int(steps))

    def go_mk2(self, steps: int):
        self.L.gref_go_mk2(self.h, int(steps))

    def go_inner_mk2(self, steps: int):
        self.L.gref_go_inner_mk2(self.h, int(steps))

    def move_surface(self, ii: int, dt: float):
        self.L.gref_move_surface(self.h, int(ii), float(dt))

    def move_setka2(self, dt: float):
        self.L.gref_move_setka2(self.h, float(dt))

    def face_par(self, f: int, which: int, ii: int) -> np.ndarray:
        out = np.zeros(5)
        self.L.gref_face_par(self.h, int(f), int(which), int(ii), out)
        return out

    def cell_geom(self, c: int) -> np.ndarray:
        out = np.zeros(8)
        self.L.gref_cell_geom(self.h, int(c), out)
        return out

    def source_mk1(self, c: int, u, v, ro, p) -> np.ndarray:
        out = np.zeros(3)
        self.L.gref_source_mk1(self.h, int(c), float(u), float(v), float(ro), float(p), out)
        return out


def hllc(L_state, R_state, W, n1, n2, rad, metod, nul_potok=False):
    """HLLC_2d_Korolkov_b_s (Setka.cpp:10484-10700). States are (ro, Q, p, v1, v2).
    Returns (time, P[4], PQ, (Vl, Vc, Vp))."""
    P = np.zeros(4)
    PQ = np.zeros(1)
    v = np.zeros(3)
    t = lib().gref_hllc(*[float(a) for a in L_state], *[float(a) for a in R_state], float(W), P, PQ,
                        float(n1), float(n2), float(rad), int(metod), v, int(bool(nul_potok)))
    return t, P, PQ[0], v


def godunov(q1, q2, n, w=0.0, dist=0.0):
    """Godunov_Solver_Alexashov (Solvers.cpp:693-1172); q = (ro, p, u, v, w)."""
    q = np.zeros(5)
    d = np.zeros(3)
    t = lib().gref_godunov(np.asarray(q1, np.float64), np.asarray(q2, np.float64), np.asarray(n, np.float64),
                           q, d, float(w), float(dist))
    return t, q, d


def hlldq(L_state, R_state, n, rad, metod):
    """HLLDQ_Korolkov (Solvers.cpp:1642-2185); states (ro, Q, p, v1, v2, v3, Bx, By, Bz)."""
    P = np.zeros(8)
    PQ = np.zeros(1)
    t = lib().gref_hlldq(np.asarray(L_state, np.float64), np.asarray(R_state, np.float64), P, PQ,
                         np.asarray(n, np.float64), float(rad), int(metod))
    return t, P, PQ[0]


def hlld(q1, q2, n, w=0.0, dist=0.0):
    """HLLD_Solver_Alexashov (Solvers.cpp:92-691); q = (ro, p, u, v, w, bx, by, bz).
    The reference exits the process where its wave speeds are out of order:
    screen inputs with the oracle's status first."""
    q = np.zeros(8)
    d = np.zeros(3)
    t = lib().gref_hlld(np.asarray(q1, np.float64), np.asarray(q2, np.float64), np.asarray(n, np.float64), q, d,
                        float(w), float(dist))
    return t, q, d
