"""Grids of the plasma step as flat arrays (the gelios_mesh_view layout).

A :class:`Mesh` is a dict-like bundle of numpy arrays with the reference's
numbering: points in ``All_Points`` order, cells in ``All_Cells`` order,
faces = ``All_Gran`` then ``All_Gran_copy``.  The native builders
(``gelios_mesh_build_setka``/``_polar``) and ``TVD_prepare`` run in the C++
part of the library.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _native as N

# Gran_type / Cell_type / Point_type / Rail_type values of the reference
USUALY, INNER_SPHERE, EXTERN, INPUT, AXIS, UPPER_WALL = range(6)
C_1, C_2, C_3, C_4, C_5, C_CENTR = range(6)
P_CONTACT, P_INNER_SHOCK, P_OUTER_SHOCK = 6, 7, 8

_INT_KEYS = ("point_type", "cell_type", "contour_start", "contour", "gran_start", "gran", "cell_back",
             "cell_next", "face_A", "face_B", "face_type", "face_master", "face_sosed", "face_copy",
             "face_sosed_up", "face_sosed_down", "rail_type", "rail_M", "rail_pstart", "rail_points",
             "rail_kstart", "rail_keys", "line_contact", "line_inner", "line_outer", "dims")
_DBL_KEYS = ("x", "y", "r_istoch", "rail_s")


class Mesh(dict):
    """Flat-array grid.  Keys match the harness export of the reference."""

    @property
    def n_cells(self) -> int:
        return len(self["cell_type"])

    @property
    def n_points(self) -> int:
        return len(self["x"])

    @property
    def n_faces(self) -> int:
        return len(self["face_A"])

    # ------------------------------------------------------------ builders
    @classmethod
    def _from_handle(cls, h: int) -> "Mesh":
        L = N.lib()
        v = N.GeliosMeshView()
        N.check(L.gelios_mesh_get_view(h, C.byref(v)), "gelios_mesh_get_view")
        m = cls._from_view(v)
        L.gelios_mesh_free(h)
        return m

    @classmethod
    def _from_view(cls, v: N.GeliosMeshView) -> "Mesh":
        def arr(p, n, dt):
            if n == 0 or not p:
                return np.zeros(0, dt)
            return np.ctypeslib.as_array(p, shape=(n,)).astype(dt, copy=True)

        nc, nf, nr = v.n_cells, v.n_faces, v.n_rails
        m = cls()
        m["dims"] = np.array(list(v.dims), np.int32)
        m["x"] = arr(v.x, v.n_points, np.float64)
        m["y"] = arr(v.y, v.n_points, np.float64)
        m["point_type"] = arr(v.point_type, v.n_points, np.int32)
        m["cell_type"] = arr(v.cell_type, nc, np.int32)
        m["contour_start"] = arr(v.contour_start, nc + 1, np.int32)
        m["contour"] = arr(v.contour, int(m["contour_start"][-1]), np.int32)
        m["gran_start"] = arr(v.gran_start, nc + 1, np.int32)
        m["gran"] = arr(v.gran, int(m["gran_start"][-1]), np.int32)
        m["cell_back"] = arr(v.cell_back, nc, np.int32)
        m["cell_next"] = arr(v.cell_next, nc, np.int32)
        m["r_istoch"] = arr(v.r_istoch, nc, np.float64)
        m["n_main"] = int(v.n_main)
        for k in ("face_A", "face_B", "face_type", "face_master", "face_sosed", "face_copy", "face_sosed_up",
                  "face_sosed_down"):
            m[k] = arr(getattr(v, k), nf, np.int32)
        m["rail_type"] = arr(v.rail_type, nr, np.int32)
        m["rail_s"] = arr(v.rail_s, nr, np.float64)
        m["rail_M"] = arr(v.rail_M, 4 * nr, np.int32)
        m["rail_pstart"] = arr(v.rail_pstart, nr + 1, np.int32) if nr else np.zeros(1, np.int32)
        m["rail_points"] = arr(v.rail_points, int(m["rail_pstart"][-1]), np.int32)
        m["rail_kstart"] = arr(v.rail_kstart, nr + 1, np.int32) if nr else np.zeros(1, np.int32)
        m["rail_keys"] = arr(v.rail_keys, int(m["rail_kstart"][-1]), np.int32)
        m["line_contact"] = arr(v.line_contact, v.n_contact, np.int32)
        m["line_inner"] = arr(v.line_inner, v.n_inner_line, np.int32)
        m["line_outer"] = arr(v.line_outer, v.n_outer_line, np.int32)
        return m

    @classmethod
    def setka(cls, N1, N2, N3, N4, M1, M2, M3, M4, tvd: bool = True) -> "Mesh":
        """Setka::Setka(N1..M4) (Setka.cpp:19-1076), optionally followed by TVD_prepare."""
        L = N.lib()
        h = L.gelios_mesh_build_setka(N1, N2, N3, N4, M1, M2, M3, M4)
        if not h:
            N.check(N.GELIOS_E_ARG, "gelios_mesh_build_setka")
        if tvd:
            N.check(L.gelios_mesh_tvd_prepare(h), "gelios_mesh_tvd_prepare")
        return cls._from_handle(h)

    @classmethod
    def polar(cls, n_theta=180, n_r=120, r_in=1.0, r_out=600.0, tvd: bool = True) -> "Mesh":
        """Axisymmetric half-plane polar grid (n_theta x n_r quads, log-spaced radii)."""
        L = N.lib()
        h = L.gelios_mesh_build_polar(n_theta, n_r, r_in, r_out)
        if not h:
            N.check(N.GELIOS_E_ARG, "gelios_mesh_build_polar")
        if tvd:
            N.check(L.gelios_mesh_tvd_prepare(h), "gelios_mesh_tvd_prepare")
        return cls._from_handle(h)

    @classmethod
    def from_arrays(cls, d: dict) -> "Mesh":
        m = cls()
        for k, v in d.items():
            if k in _INT_KEYS:
                m[k] = np.ascontiguousarray(v, dtype=np.int32)
            elif k in _DBL_KEYS:
                m[k] = np.ascontiguousarray(v, dtype=np.float64)
            else:
                m[k] = v
        m.setdefault("dims", np.zeros(8, np.int32))
        return m

    # ------------------------------------------------------------ views
    def view(self) -> tuple[N.GeliosMeshView, list]:
        """A gelios_mesh_view pointing into this mesh's arrays (keep the
        returned keep-alive list while the view is in use)."""
        keep = []

        def ip(k, required=True):
            a = self.get(k)
            if a is None or (len(a) == 0 and not required):
                return C.cast(None, N._IP)
            a = np.ascontiguousarray(a, dtype=np.int32)
            if len(a) == 0:
                a = np.zeros(1, np.int32)
            keep.append(a)
            return a.ctypes.data_as(N._IP)

        def dp(k, required=True):
            a = self.get(k)
            if a is None or (len(a) == 0 and not required):
                return C.cast(None, N._DP)
            a = np.ascontiguousarray(a, dtype=np.float64)
            if len(a) == 0:
                a = np.zeros(1)
            keep.append(a)
            return a.ctypes.data_as(N._DP)

        v = N.GeliosMeshView()
        dims = self.get("dims", np.zeros(8, np.int32))
        for i in range(8):
            v.dims[i] = int(dims[i])
        v.n_points = self.n_points
        v.x, v.y, v.point_type = dp("x"), dp("y"), ip("point_type")
        v.n_cells = self.n_cells
        v.cell_type = ip("cell_type")
        v.contour_start, v.contour = ip("contour_start"), ip("contour")
        v.gran_start, v.gran = ip("gran_start"), ip("gran")
        v.cell_back, v.cell_next = ip("cell_back", False), ip("cell_next", False)
        v.r_istoch = dp("r_istoch", False)
        v.n_faces, v.n_main = self.n_faces, int(self["n_main"])
        for k in ("face_A", "face_B", "face_type", "face_master", "face_sosed", "face_copy"):
            setattr(v, k, ip(k))
        v.face_sosed_up, v.face_sosed_down = ip("face_sosed_up", False), ip("face_sosed_down", False)
        nr = len(self.get("rail_type", []))
        v.n_rails = nr
        v.rail_type, v.rail_s, v.rail_M = ip("rail_type"), dp("rail_s"), ip("rail_M")
        v.rail_pstart, v.rail_points = ip("rail_pstart"), ip("rail_points")
        v.rail_kstart, v.rail_keys = ip("rail_kstart"), ip("rail_keys")
        v.n_contact = len(self.get("line_contact", []))
        v.n_inner_line = len(self.get("line_inner", []))
        v.n_outer_line = len(self.get("line_outer", []))
        v.line_contact, v.line_inner, v.line_outer = ip("line_contact"), ip("line_inner"), ip("line_outer")
        keep.append(v)
        return v, keep

    def tvd_prepare(self) -> "Mesh":
        """Setka::TVD_prepare (Setka.cpp:1294-1492) on these arrays, in place."""
        v, keep = self.view()
        nf, nc = self.n_faces, self.n_cells
        up = np.zeros(nf, np.int32)
        down = np.zeros(nf, np.int32)
        back = np.zeros(nc, np.int32)
        nxt = np.zeros(nc, np.int32)
        ri = np.zeros(nc)
        # a grid loaded from a checkpoint carries the loader's unique face
        # numbers (see gelios_tvd_prepare_view_numbered)
        uniq = 1 if self.get("face_numbering") == "unique" else 0
        N.check(N.lib().gelios_tvd_prepare_view_numbered(C.byref(v), uniq, up, down, back, nxt, ri),
                "gelios_tvd_prepare_view_numbered")
        self.update(face_sosed_up=up, face_sosed_down=down, cell_back=back, cell_next=nxt, r_istoch=ri)
        return self

    def centroids(self, x=None, y=None) -> np.ndarray:
        """Polygon centroids (Cell::Get_Center, Cell.cpp:66-88) on the host,
        accumulated vertex by vertex in the reference's order."""
        x = self["x"] if x is None else np.asarray(x)
        y = self["y"] if y is None else np.asarray(y)
        cs, con = self["contour_start"], self["contour"]
        nv = np.diff(cs)
        out = np.zeros((2, self.n_cells))
        for n in np.unique(nv):
            cells = np.nonzero(nv == n)[0]
            idx = con[cs[cells][:, None] + np.arange(n)[None, :]]
            A = np.zeros(len(cells))
            Gx = np.zeros(len(cells))
            Gy = np.zeros(len(cells))
            for i in range(n):
                a, b = idx[:, i], idx[:, (i + 1) % n]
                cr = x[a] * y[b] - y[a] * x[b]
                A = A + cr
                Gx = Gx + (x[a] + x[b]) * cr
                Gy = Gy + (y[a] + y[b]) * cr
            A = A * 0.5
            out[0, cells] = Gx / (6.0 * A)
            out[1, cells] = Gy / (6.0 * A)
        return out

    def inner_cells(self, r_max: float) -> np.ndarray:
        """All_Cells_Inner: cells with centroid radius <= r_max (Gelios_2D.cpp:152-231)."""
        c = self.centroids()
        return np.nonzero(np.sqrt(c[0] ** 2 + c[1] ** 2) <= r_max)[0].astype(np.int32)
