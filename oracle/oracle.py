"""Test infrastructure: ctypes access to the C restatement (oracle/_ref/libgelios_oracle.so).

The restatement (``gelios_oracle.c``) is the checker the CUDA path is compared
against; it is pinned bit-for-bit to the compiled reference in
``tests/test_oracle_pin.py``.  Only tests, the smoke check and bench.py's
CPU-baseline leg use this module.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "_ref" / "libgelios_oracle.so"

RR_ = 390.222


class GoParams(C.Structure):
    """Mirror of ``go_params`` (gelios_oracle.h); same field order as
    ``gelios_params`` in include/gelios_b200.h."""

    _fields_ = [(n, C.c_double) for n in (
        "gamma", "kurant", "chi", "inner_mach", "in_ro", "in_p", "in_u", "in_v", "in_Q",
        "extern_u_par", "extern_u_tvd", "R11", "rad_stat", "R1", "R111", "R5", "Left", "koef",
        "src_rmin", "src_rmax", "src_coef", "a_2", "ro_floor", "p_floor", "dt0")] + [
        ("n_inner", C.c_int32), ("n_outer_shock", C.c_int32), ("godunov_max_iter", C.c_int32),
        ("pad_", C.c_int32)]


def reference_params(**over) -> GoParams:
    """The reference's compile-time constants (Help.h:39-114, Gran.cpp:216-281,
    Setka.cpp:3380, 5256, 10129, 10169, Solvers.cpp:1206)."""
    d = dict(gamma=5.0 / 3.0, kurant=0.1, chi=36.1275, inner_mach=10.0, in_ro=1.0, in_p=1.0,
             in_u=-2.54338, in_v=0.0, in_Q=100.0, extern_u_par=-0.1, extern_u_tvd=-0.01,
             R11=38.0 / RR_, rad_stat=95.0, R1=1.0 / RR_, R111=50.0 / RR_, R5=2200.0 / RR_,
             Left=-1500.0 / RR_, koef=0.1, src_rmin=10.0 / RR_, src_rmax=1500.0 / RR_,
             src_coef=3.0 / 6.0, a_2=0.1307345665, ro_floor=0.00001, p_floor=0.000001, dt0=0.00000001,
             n_inner=20, n_outer_shock=13, godunov_max_iter=1100, pad_=0)
    d.update(over)
    return GoParams(**d)


class GoMesh(C.Structure):
    _fields_ = [
        ("dims", C.c_int32 * 8),
        ("n_points", C.c_int32), ("x", C.c_void_p), ("y", C.c_void_p), ("point_type", C.c_void_p),
        ("n_cells", C.c_int32), ("cell_type", C.c_void_p), ("contour_start", C.c_void_p),
        ("contour", C.c_void_p), ("gran_start", C.c_void_p), ("gran", C.c_void_p),
        ("cell_back", C.c_void_p), ("cell_next", C.c_void_p), ("r_istoch", C.c_void_p),
        ("n_faces", C.c_int32), ("n_main", C.c_int32),
        ("face_A", C.c_void_p), ("face_B", C.c_void_p), ("face_type", C.c_void_p),
        ("face_master", C.c_void_p), ("face_sosed", C.c_void_p), ("face_copy", C.c_void_p),
        ("face_sosed_up", C.c_void_p), ("face_sosed_down", C.c_void_p),
        ("n_rails", C.c_int32), ("rail_type", C.c_void_p), ("rail_s", C.c_void_p),
        ("rail_M", C.c_void_p), ("rail_pstart", C.c_void_p), ("rail_points", C.c_void_p),
        ("rail_kstart", C.c_void_p), ("rail_keys", C.c_void_p),
        ("n_contact", C.c_int32), ("n_inner_line", C.c_int32), ("n_outer_line", C.c_int32),
        ("line_contact", C.c_void_p), ("line_inner", C.c_void_p), ("line_outer", C.c_void_p),
    ]


class GoMhdParams(C.Structure):
    """Mirror of ``go_mhd_params`` (same field order as gelios_mhd_params)."""

    _fields_ = [(n, C.c_double) for n in ("lism_bx", "lism_by", "lism_bz", "inner_bphi", "pui_in_ro", "pui_in_p",
                                          "pui_inner_ro", "pui_inner_p")]


_LIB = None


def lib() -> C.CDLL:
    global _LIB
    if _LIB is not None:
        return _LIB
    if not LIB_PATH.exists():
        raise FileNotFoundError(f"{LIB_PATH} missing: run `make -C oracle`")
    L = C.CDLL(str(LIB_PATH))
    vp = C.c_void_p
    f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
    i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
    L.go_create.restype = vp
    L.go_create.argtypes = [C.POINTER(GoParams), C.POINTER(GoMesh)]
    L.go_destroy.argtypes = [vp]
    L.go_set_state.argtypes = [vp, C.c_int] + [f64p] * 5
    L.go_get_state.argtypes = [vp, C.c_int] + [f64p] * 5
    L.go_set_mc.argtypes = [vp] + [f64p] * 7
    L.go_set_inner_list.argtypes = [vp, i32p, C.c_int32]
    L.go_get_points.argtypes = [vp] + [f64p] * 6 + [i32p]
    L.go_status.argtypes = [vp, np.ctypeslib.ndpointer(np.int64, flags="C_CONTIGUOUS")]
    for f in ("go_stationary", "go_mk2", "go_inner_mk2"):
        getattr(L, f).argtypes = [vp, C.c_int]
    L.go_move_surface.argtypes = [vp, C.c_int, C.c_double]
    L.go_move_setka2.argtypes = [vp, C.c_double]
    L.go_commit_points.argtypes = [vp]
    L.go_last_dt.restype = C.c_double
    L.go_last_dt.argtypes = [vp]
    L.go_hllc.restype = C.c_double
    L.go_hllc.argtypes = [C.POINTER(GoParams), f64p, f64p, C.c_double, f64p, f64p, C.c_double, C.c_double,
                          C.c_double, C.c_int, f64p, C.c_int]
    L.go_godunov.restype = C.c_double
    L.go_godunov.argtypes = [C.POINTER(GoParams), f64p, f64p, f64p, f64p, f64p, C.c_double, C.c_double,
                             C.POINTER(C.c_int)]
    L.go_hlldq.restype = C.c_double
    L.go_hlldq.argtypes = [C.POINTER(GoParams), f64p, f64p, f64p, f64p, f64p, C.c_double, C.c_int]
    L.go_hlld.restype = C.c_double
    L.go_hlld.argtypes = [C.POINTER(GoParams), f64p, f64p, f64p, f64p, f64p, C.c_double, C.c_double,
                          C.POINTER(C.c_int)]
    L.go_set_hydrogen.argtypes = [vp, C.c_int, f64p]
    L.go_get_hydrogen.argtypes = [vp, C.c_int, f64p]
    L.go_5_komponent.argtypes = [vp, C.c_int]
    L.go_move_setka1.argtypes = [vp, C.c_double]
    L.go_face_par.argtypes = [vp, C.c_int, C.c_int, C.c_int, f64p]
    L.go_cell_geom.argtypes = [vp, C.c_int, f64p]
    L.go_source_mk1.argtypes = [vp, C.c_int] + [C.c_double] * 4 + [f64p]
    L.go_set_mhd.argtypes = [vp, C.c_int, f64p]
    L.go_get_mhd.argtypes = [vp, C.c_int, f64p]
    L.go_set_sources.argtypes = [vp, f64p, f64p, f64p]
    L.go_mhd.argtypes = [vp, C.POINTER(GoMhdParams), C.c_int]
    _LIB = L
    return L


def _ptr(a: np.ndarray) -> int:
    return a.ctypes.data


class Oracle:
    """One restatement context over a mesh dict (unified face numbering)."""

    def __init__(self, params: GoParams, mesh: dict):
        self.L = lib()
        self.params = params
        keep = {}

        def arr(name, dtype, default_len=1):
            a = mesh.get(name)
            if a is None or len(a) == 0:
                a = np.zeros(default_len, dtype)
            a = np.ascontiguousarray(a, dtype=dtype)
            keep[name] = a
            return _ptr(a)

        m = GoMesh()
        dims = mesh.get("dims", np.zeros(8, np.int32))
        for i in range(8):
            m.dims[i] = int(dims[i])
        ncell = len(mesh["cell_type"])
        m.n_points = len(mesh["x"])
        m.x, m.y = arr("x", np.float64), arr("y", np.float64)
        m.point_type = arr("point_type", np.int32)
        m.n_cells = ncell
        m.cell_type = arr("cell_type", np.int32)
        m.contour_start, m.contour = arr("contour_start", np.int32), arr("contour", np.int32)
        m.gran_start, m.gran = arr("gran_start", np.int32), arr("gran", np.int32)
        if "cell_back" not in mesh:
            mesh = dict(mesh, cell_back=-np.ones(ncell, np.int32), cell_next=-np.ones(ncell, np.int32),
                        r_istoch=np.zeros(ncell))
        m.cell_back, m.cell_next = arr("cell_back", np.int32), arr("cell_next", np.int32)
        m.r_istoch = arr("r_istoch", np.float64)
        nf = len(mesh["face_A"])
        m.n_faces, m.n_main = nf, int(mesh["n_main"])
        for k in ("face_A", "face_B", "face_type", "face_master", "face_sosed", "face_copy", "face_sosed_up",
                  "face_sosed_down"):
            if k not in mesh:
                mesh = dict(mesh, **{k: -np.ones(nf, np.int32)})
            setattr(m, k, arr(k, np.int32))
        nr = len(mesh.get("rail_type", []))
        m.n_rails = nr
        m.rail_type, m.rail_s, m.rail_M = arr("rail_type", np.int32), arr("rail_s", np.float64), arr("rail_M", np.int32)
        if "rail_pstart" not in mesh:
            mesh = dict(mesh, rail_pstart=np.zeros(1, np.int32), rail_kstart=np.zeros(1, np.int32))
        m.rail_pstart, m.rail_points = arr("rail_pstart", np.int32), arr("rail_points", np.int32)
        m.rail_kstart, m.rail_keys = arr("rail_kstart", np.int32), arr("rail_keys", np.int32)
        m.n_contact = len(mesh.get("line_contact", []))
        m.n_inner_line = len(mesh.get("line_inner", []))
        m.n_outer_line = len(mesh.get("line_outer", []))
        m.line_contact, m.line_inner, m.line_outer = (arr("line_contact", np.int32), arr("line_inner", np.int32),
                                                      arr("line_outer", np.int32))
        self._keep = keep
        self.ncell = ncell
        self.npoint = m.n_points
        self.h = C.c_void_p(self.L.go_create(C.byref(params), C.byref(m)))

    def __del__(self):
        try:
            if self.h:
                self.L.go_destroy(self.h)
                self.h = None
        except Exception:
            pass

    def set_state(self, buf: int, st: np.ndarray):
        st = np.ascontiguousarray(st, dtype=np.float64)
        self.L.go_set_state(self.h, buf, *[np.ascontiguousarray(st[k]) for k in range(5)])

    def get_state(self, buf: int) -> np.ndarray:
        out = [np.zeros(self.ncell) for _ in range(5)]
        self.L.go_get_state(self.h, buf, *out)
        return np.stack(out)

    def set_mc(self, Hn, Hu, Hv, HT, ku, kv, kT):
        f = lambda a: np.ascontiguousarray(a, dtype=np.float64).ravel()  # noqa: E731
        self.L.go_set_mc(self.h, f(Hn), f(Hu), f(Hv), f(HT), f(ku), f(kv), f(kT))

    def set_inner_list(self, cells):
        a = np.ascontiguousarray(cells, dtype=np.int32)
        self.L.go_set_inner_list(self.h, a if len(a) else np.zeros(1, np.int32), len(a))

    def points(self) -> dict:
        arrs = [np.zeros(self.npoint) for _ in range(6)]
        cnt = np.zeros(self.npoint, np.int32)
        self.L.go_get_points(self.h, *arrs, cnt)
        return dict(zip(["x", "y", "x2", "y2", "Vx", "Vy"], arrs), count=cnt)

    def status(self) -> np.ndarray:
        out = np.zeros(4, np.int64)
        self.L.go_status(self.h, out)
        return out

    def stationary(self, steps):
        self.L.go_stationary(self.h, int(steps))

    def mk2(self, steps):
        self.L.go_mk2(self.h, int(steps))

    def set_hydrogen(self, buf, h16):
        """ro, p, u, v of H1..H4 in par[buf]; h16 of shape (16, n_cells)."""
        self.L.go_set_hydrogen(self.h, int(buf), np.ascontiguousarray(h16, np.float64).ravel())

    def get_hydrogen(self, buf) -> np.ndarray:
        out = np.zeros(16 * self.ncell)
        self.L.go_get_hydrogen(self.h, int(buf), out)
        return out.reshape(16, self.ncell)

    def set_mhd(self, buf, x8):
        """Extra rows of the MHD form in par[buf]; x8 of shape (8, n_cells)."""
        self.L.go_set_mhd(self.h, int(buf), np.ascontiguousarray(x8, np.float64).ravel())

    def get_mhd(self, buf) -> np.ndarray:
        out = np.zeros(8 * self.ncell)
        self.L.go_get_mhd(self.h, int(buf), out)
        return out.reshape(8, self.ncell)

    def set_sources(self, q1, q2, q3):
        f = lambda a: np.ascontiguousarray(a, np.float64).ravel()  # noqa: E731
        self.L.go_set_sources(self.h, f(q1), f(q2), f(q3))

    def mhd(self, mp: dict, steps):
        """The MHD + pickup-proton moving-grid step (go_mhd)."""
        self.L.go_mhd(self.h, C.byref(GoMhdParams(**mp)), int(steps))

    def five_komponent(self, steps):
        """Setka::Go_5_komponent (Setka.cpp:8269-8950)."""
        self.L.go_5_komponent(self.h, int(steps))

    def inner_mk2(self, steps):
        self.L.go_inner_mk2(self.h, int(steps))

    def move_surface(self, ii, dt):
        self.L.go_move_surface(self.h, int(ii), float(dt))

    def move_setka2(self, dt):
        self.L.go_move_setka2(self.h, float(dt))

    def commit_points(self):
        self.L.go_commit_points(self.h)

    def last_dt(self) -> float:
        return self.L.go_last_dt(self.h)

    def face_par(self, f, which, buf):
        out = np.zeros(5)
        self.L.go_face_par(self.h, int(f), int(which), int(buf), out)
        return out

    def cell_geom(self, c):
        out = np.zeros(8)
        self.L.go_cell_geom(self.h, int(c), out)
        return out

    def source_mk1(self, c, u, v, ro, p):
        out = np.zeros(3)
        self.L.go_source_mk1(self.h, int(c), float(u), float(v), float(ro), float(p), out)
        return out


def hllc(params: GoParams, Ls, Rs, W, n1, n2, rad, metod, nul_potok=False):
    P = np.zeros(4)
    PQ = np.zeros(1)
    v = np.zeros(3)
    t = lib().go_hllc(C.byref(params), np.asarray(Ls, np.float64), np.asarray(Rs, np.float64), float(W), P, PQ,
                      float(n1), float(n2), float(rad), int(metod), v, int(bool(nul_potok)))
    return t, P, PQ[0], v


def godunov(params: GoParams, q1, q2, n, w=0.0, dist=0.0):
    q = np.zeros(5)
    d = np.zeros(3)
    st = C.c_int(0)
    t = lib().go_godunov(C.byref(params), np.asarray(q1, np.float64), np.asarray(q2, np.float64),
                         np.asarray(n, np.float64), q, d, float(w), float(dist), C.byref(st))
    return t, q, d, st.value


def hlldq(params: GoParams, L_state, R_state, n, rad, metod):
    """HLLDQ_Korolkov (Solvers.cpp:1642-2185); states (ro, Q, p, v1, v2, v3,
    Bx, By, Bz), n a coordinate axis.  Returns (time, P[8], PQ)."""
    P = np.zeros(8)
    PQ = np.zeros(1)
    t = lib().go_hlldq(C.byref(params), np.asarray(L_state, np.float64), np.asarray(R_state, np.float64), P, PQ,
                       np.asarray(n, np.float64), float(rad), int(metod))
    return t, P, PQ[0]


def hlld(params: GoParams, q1, q2, n, w=0.0, dist=0.0):
    """HLLD_Solver_Alexashov (Solvers.cpp:92-691); q = (ro, p, u, v, w, bx,
    by, bz).  Returns (time, q[8], (dsl, dsp, dsc), status)."""
    q = np.zeros(8)
    d = np.zeros(3)
    st = C.c_int(0)
    t = lib().go_hlld(C.byref(params), np.asarray(q1, np.float64), np.asarray(q2, np.float64),
                      np.asarray(n, np.float64), q, d, float(w), float(dist), C.byref(st))
    return t, q, d, st.value
