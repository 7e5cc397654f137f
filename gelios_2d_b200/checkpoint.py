"""Checkpoints of a grid and its state.

Two formats:

* the reference's text format, written by ``Setka::Save_Setka_ALL_ALPHA``
  (Setka.cpp:2355-2574) and read by ``Setka::Download_Setka_ALL_ALPHA_2_0``
  (Setka.cpp:2899-3257): points, faces (All_Gran, then All_Gran_copy, each
  numbered from 0 in the file), rails A/B/C/D, cells (contour, Grans as
  (number, main_gran) pairs), face links, the cells of every point, the
  tracked lines and 43 numbers of ``par[0]`` per cell.  Floating-point
  numbers are written the way the reference's ``ofstream`` writes them
  (``%g``, 6 significant digits), so this format is lossy; production grids
  in this format load into the device path with :func:`read_alpha`.
* an exact binary snapshot (:func:`save_snapshot` / :func:`load_snapshot`,
  numpy ``.npz``): every mesh array and both state buffers bit for bit, for
  restarts that must not perturb the solution.

A grid read from the text format carries the loader's face numbering (main
faces, then copies, unique: Setka.cpp:3213-3224), which ``TVD_prepare``
sees (Setka.cpp:1328, 1383); :meth:`Mesh.tvd_prepare` honours it through the
mesh key ``face_numbering = "unique"``.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from pathlib import Path

import numpy as np

from .mesh import Mesh

# par[0] fields per cell in the text format, in file order (Setka.cpp:2553-2566)
_PAR_COLS = 43


@dataclass
class Checkpoint:
    """A grid with ``par[0]`` of every cell.

    par      (5, n_cells): ro, p, u, v, Q
    mc       (Hn, Hu, Hv, HT) of shape (n_cells, 4), then ku, kv, kT
    hydrogen (n_cells, 16): ro, p, u, v of the four hydrogen fluids H1..H4
    I        (n_cells, 3): I_u, I_v, I_T
    """

    mesh: Mesh
    par: np.ndarray
    mc: tuple
    hydrogen: np.ndarray
    I: np.ndarray
    point_cells: list = field(default_factory=list)


def _fmt(v: float) -> str:
    # std::ostream with default flags and precision 6 formats like %g
    return "%g" % v


def _read_text(path) -> str:
    path = Path(path)
    if path.suffix == ".gz":
        import gzip

        with gzip.open(path, "rt") as f:
            return f.read()
    return path.read_text()


def point_cells(mesh: Mesh) -> list:
    """Point::my_cell of every point: the cells whose contour holds it, in
    cell order."""
    cs, con = mesh["contour_start"], mesh["contour"]
    out = [[] for _ in range(mesh.n_points)]
    for c in range(mesh.n_cells):
        for p in con[cs[c]:cs[c + 1]]:
            out[int(p)].append(c)
    return out


def read_alpha(path, tvd: bool = True) -> Checkpoint:
    """Setka::Download_Setka_ALL_ALPHA_2_0 (Setka.cpp:2899-3257) into flat
    arrays; with ``tvd`` the TVD neighbours and source chains are prepared
    as the reference does after loading (TVD_prepare)."""
    tok = _read_text(path).split()
    pos = 0

    def take(n: int) -> list:
        nonlocal pos
        a = tok[pos:pos + n]
        if len(a) != n:
            raise ValueError(f"{path}: truncated checkpoint at token {pos}")
        pos += n
        return a

    def one() -> int:
        return int(take(1)[0])

    dims = np.array([int(t) for t in take(8)], np.int32)
    npt = one()
    a = take(3 * npt)
    x = np.array(a[0::3], np.float64)
    y = np.array(a[1::3], np.float64)
    ptype = np.array(a[2::3], np.int32)
    nmain = one()
    a = take(3 * nmain)
    fa_m, fb_m, ft_m = (np.array(a[k::3], np.int32) for k in range(3))
    ncopy = one()
    a = take(3 * ncopy)
    fa_c, fb_c, ft_c = (np.array(a[k::3], np.int32) for k in range(3))
    rtype, rs, rM, rps, rpts, rks, rkeys = [], [], [], [0], [], [0], []
    for _ in range(4):  # A, B, C, D rails
        for _ in range(one()):
            m1, m2, m3, m4, s, t = take(6)
            rM += [int(m1), int(m2), int(m3), int(m4)]
            rs.append(float(s))
            rtype.append(int(t))
            n = one()
            rpts += [int(v) for v in take(n)]
            rps.append(len(rpts))
            n = one()
            rkeys += [int(v) for v in take(n)]
            rks.append(len(rkeys))
    nc = one()
    ctype = np.zeros(nc, np.int32)
    cstart, contour, gstart, gran = [0], [], [0], []
    for c in range(nc):
        ctype[c] = one()
        n = one()
        contour += [int(v) for v in take(n)]
        cstart.append(len(contour))
        n = one()
        a = take(2 * n)
        for k in range(n):
            num, main = int(a[2 * k]), int(a[2 * k + 1])
            gran.append(num if main else nmain + num)
        gstart.append(len(gran))
    one()
    a = take(3 * nmain)
    fm_m, fs_m, fc_m = (np.array(a[k::3], np.int32) for k in range(3))
    one()
    a = take(3 * ncopy)
    fm_c, fs_c, fc_c = (np.array(a[k::3], np.int32) for k in range(3))
    one()
    pc = []
    for _ in range(npt):
        n = one()
        pc.append([int(v) for v in take(n)])
    lines = []
    for _ in range(3):
        n = one()
        lines.append(np.array([int(v) for v in take(n)], np.int32))
    one()
    vals = np.array(take(_PAR_COLS * nc), np.float64).reshape(nc, _PAR_COLS)

    # unified face numbering: main faces [0, nmain), copies [nmain, nmain + ncopy)
    face_copy = np.concatenate([np.where(fc_m >= 0, fc_m + nmain, -1), fc_c]).astype(np.int32)
    m = Mesh.from_arrays(dict(
        dims=dims, x=x, y=y, point_type=ptype, cell_type=ctype,
        contour_start=np.array(cstart), contour=np.array(contour), gran_start=np.array(gstart),
        gran=np.array(gran), n_main=nmain,
        face_A=np.concatenate([fa_m, fa_c]), face_B=np.concatenate([fb_m, fb_c]),
        face_type=np.concatenate([ft_m, ft_c]), face_master=np.concatenate([fm_m, fm_c]),
        face_sosed=np.concatenate([fs_m, fs_c]), face_copy=face_copy,
        face_sosed_up=-np.ones(nmain + ncopy), face_sosed_down=-np.ones(nmain + ncopy),
        cell_back=-np.ones(nc), cell_next=-np.ones(nc), r_istoch=np.zeros(nc),
        rail_type=np.array(rtype), rail_s=np.array(rs), rail_M=np.array(rM), rail_pstart=np.array(rps),
        rail_points=np.array(rpts), rail_kstart=np.array(rks), rail_keys=np.array(rkeys),
        line_contact=lines[0], line_inner=lines[1], line_outer=lines[2]))
    m["face_numbering"] = "unique"
    if tvd:
        m.tvd_prepare()
    par = np.ascontiguousarray(vals[:, 0:5].T)
    hydrogen = np.ascontiguousarray(vals[:, 5:21])
    I = np.ascontiguousarray(vals[:, 21:24])
    h = vals[:, 24:40].reshape(nc, 4, 4)  # [cell, sort, (n, u, v, T)]
    mc = (np.ascontiguousarray(h[:, :, 0]), np.ascontiguousarray(h[:, :, 1]), np.ascontiguousarray(h[:, :, 2]),
          np.ascontiguousarray(h[:, :, 3]), vals[:, 40].copy(), vals[:, 41].copy(), vals[:, 42].copy())
    return Checkpoint(m, par, mc, hydrogen, I, pc)


def write_alpha(path, mesh: Mesh, par: np.ndarray, mc=None, hydrogen=None, I=None, cells_of_points=None) -> None:
    """Setka::Save_Setka_ALL_ALPHA (Setka.cpp:2355-2574): the same records
    in the same order and number format.  ``par`` is (5, n_cells) ro, p, u,
    v, Q; missing Monte-Carlo moments, hydrogen fluids or I are written as 0."""
    nc, npt, nmain = mesh.n_cells, mesh.n_points, int(mesh["n_main"])
    nf = mesh.n_faces
    ncopy = nf - nmain
    par = np.asarray(par, np.float64)
    if par.shape != (5, nc):
        raise ValueError("par must be (5, n_cells)")
    if mc is None:
        mc = (np.zeros((nc, 4)),) * 4 + (np.zeros(nc),) * 3
    hydrogen = np.zeros((nc, 16)) if hydrogen is None else np.asarray(hydrogen, np.float64)
    I = np.zeros((nc, 3)) if I is None else np.asarray(I, np.float64)
    pc = point_cells(mesh) if cells_of_points is None else cells_of_points

    def fnum(f: int) -> int:  # Gran::number at save time: each list from 0
        return f if f < nmain else f - nmain

    out = []
    w = out.append
    w(" ".join(str(int(d)) for d in mesh["dims"]) + " ")
    w(str(npt))
    for i in range(npt):
        w(f"{_fmt(mesh['x'][i])} {_fmt(mesh['y'][i])} {int(mesh['point_type'][i])}")
    A, B, T = mesh["face_A"], mesh["face_B"], mesh["face_type"]
    w(str(nmain))
    for f in range(nmain):
        w(f"{A[f]} {B[f]} {T[f]}")
    w(str(ncopy))
    for f in range(nmain, nf):
        w(f"{A[f]} {B[f]} {T[f]}")
    rt, rps, rks = mesh["rail_type"], mesh["rail_pstart"], mesh["rail_kstart"]
    for kind in range(4):
        idx = [r for r in range(len(rt)) if rt[r] == kind]
        w(str(len(idx)))
        for r in idx:
            M = mesh["rail_M"][4 * r:4 * r + 4]
            w(f"{M[0]} {M[1]} {M[2]} {M[3]} {_fmt(mesh['rail_s'][r])} {rt[r]}")
            pts = mesh["rail_points"][rps[r]:rps[r + 1]]
            w(str(len(pts)))
            out.extend(str(p) for p in pts)
            keys = mesh["rail_keys"][rks[r]:rks[r + 1]]
            w(str(len(keys)))
            out.extend(str(p) for p in keys)
    cs, con, gs, gr = mesh["contour_start"], mesh["contour"], mesh["gran_start"], mesh["gran"]
    w(str(nc))
    for c in range(nc):
        w(str(int(mesh["cell_type"][c])))
        w(str(cs[c + 1] - cs[c]))
        out.extend(str(p) for p in con[cs[c]:cs[c + 1]])
        w(str(gs[c + 1] - gs[c]))
        out.extend(f"{fnum(int(f))} {1 if f < nmain else 0}" for f in gr[gs[c]:gs[c + 1]])
    M, S, Cp = mesh["face_master"], mesh["face_sosed"], mesh["face_copy"]
    w(str(nmain))
    for f in range(nmain):
        w(f"{M[f]} {S[f]} {fnum(int(Cp[f])) if Cp[f] >= 0 else -1}")
    w(str(ncopy))
    for f in range(nmain, nf):
        w(f"{M[f]} {S[f]} {fnum(int(Cp[f]))}")
    w(str(npt))
    for cells in pc:
        w(str(len(cells)))
        out.extend(str(c) for c in cells)
    for key in ("line_contact", "line_inner", "line_outer"):
        lst = mesh[key]
        w(str(len(lst)))
        out.extend(str(int(f)) for f in lst)
    Hn, Hu, Hv, HT, ku, kv, kT = mc
    w(str(nc))
    for c in range(nc):
        w(" ".join(_fmt(v) for v in par[:, c]))
        for s in range(4):
            w(" ".join(_fmt(v) for v in hydrogen[c, 4 * s:4 * s + 4]))
        w(" ".join(_fmt(v) for v in I[c]))
        for s in range(4):
            w(f"{_fmt(Hn[c][s])} {_fmt(Hu[c][s])} {_fmt(Hv[c][s])} {_fmt(HT[c][s])}")
        w(f"{_fmt(ku[c])} {_fmt(kv[c])} {_fmt(kT[c])}")
    Path(path).write_text("\n".join(out) + "\n")


def save_snapshot(path, mesh: Mesh, par0: np.ndarray, par1: np.ndarray | None = None, mc=None) -> None:
    """Exact binary snapshot: every mesh array and both state buffers."""
    arrays = {f"mesh_{k}": np.asarray(v) for k, v in mesh.items() if not isinstance(v, str)}
    meta = {f"meta_{k}": np.array(v) for k, v in mesh.items() if isinstance(v, str)}
    extra = {}
    if mc is not None:
        for name, a in zip(("Hn", "Hu", "Hv", "HT", "ku", "kv", "kT"), mc):
            extra[f"mc_{name}"] = np.asarray(a, np.float64)
    np.savez(path, par0=np.asarray(par0, np.float64),
             par1=np.asarray(par0 if par1 is None else par1, np.float64), **arrays, **meta, **extra)


def load_snapshot(path) -> tuple:
    """(mesh, par0, par1, mc or None) from :func:`save_snapshot`."""
    d = np.load(path, allow_pickle=False)
    m = Mesh.from_arrays({k[5:]: d[k] for k in d.files if k.startswith("mesh_")})
    for k in d.files:
        if k.startswith("meta_"):
            m[k[5:]] = str(d[k])
    if "n_main" in m:
        m["n_main"] = int(m["n_main"])
    mc = None
    if "mc_Hn" in d.files:
        mc = tuple(d[f"mc_{n}"] for n in ("Hn", "Hu", "Hv", "HT", "ku", "kv", "kT"))
    return m, d["par0"], d["par1"], mc
