"""Generates the golden fixtures of tests/golden from the compiled reference.

Run where the reference tree and oracle/_ref/libgelios_ref.so exist:
    python tests/golden/make_golden.py [faces] [steps] [mhd] [checkpoint] [five]
(no argument: all).  The fixtures are the reference's own outputs
(HLLC_2d_Korolkov_b_s, Godunov_Solver_Alexashov, HLLDQ_Korolkov,
HLLD_Solver_Alexashov, and short Go_stationary / Go_5_komponent__MK2 /
Go_stationary_5_komponent_inner_MK2 runs on Setka(4,3,3,10,23,6,7,7)), so the
oracle stays pinned where the reference cannot be built.
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent.parent))

from oracle import ref  # noqa: E402
from gelios_2d_b200 import workloads as W  # noqa: E402
from gelios_2d_b200.mesh import Mesh  # noqa: E402

SMALL = (4, 3, 3, 10, 23, 6, 7, 7)


def hllc_cases(n=96, seed=11):
    u = W.splitmix64(seed, n * 16).reshape(n, 16)
    rows = []
    # the smoke check of main (Gelios_2D.cpp:46-67) first
    rows.append([2.0, 1.0, 2.0, 1.0, 0.0, 1.0, 1.0, 1.0, 0.5, 0.0, 0.0, 1.0, 0.0, 10.0, 1, 0])
    for i in range(1, n):
        a = u[i]
        th = 2 * np.pi * a[11]
        rows.append([0.1 + 2 * a[0], 50 * a[1], 0.05 + 3 * a[2], 4 * (a[3] - 0.5), 4 * (a[4] - 0.5),
                     0.1 + 2 * a[5], 50 * a[6], 0.05 + 3 * a[7], 4 * (a[8] - 0.5), 4 * (a[9] - 0.5),
                     (a[10] - 0.5) * 2.0 if i % 3 else 0.0, np.cos(th), np.sin(th), 0.01 + a[12],
                     i % 2, (i // 2) % 2])
    return np.array(rows)


def godunov_cases(n=96, seed=13):
    u = W.splitmix64(seed, n * 16).reshape(n, 16)
    rows = []
    for i in range(n):
        a = u[i]
        th = 2 * np.pi * a[10]
        scale = 1.0 if i % 4 else 20.0  # strong shocks
        rows.append([0.1 + 2 * a[0], 0.05 + 3 * a[1] * scale, 3 * (a[2] - 0.5), 3 * (a[3] - 0.5), 0.0,
                     0.1 + 2 * a[4], 0.05 + 3 * a[5], 3 * (a[6] - 0.5) - (2.0 if i % 5 == 0 else 0.0),
                     3 * (a[7] - 0.5), 0.0, np.cos(th), np.sin(th), 0.0,
                     (a[8] - 0.5) if i % 2 else 0.0, 0.01 + a[9]])
    return np.array(rows)


AXES = [(1.0, 0.0, 0.0), (0.0, 1.0, 0.0), (0.0, 0.0, 1.0), (-1.0, 0.0, 0.0), (0.0, -1.0, 0.0), (0.0, 0.0, -1.0)]


def mhd_state(a, with_q):
    """(ro, [Q,] p, v1, v2, v3, Bx, By, Bz) from 8 or 9 uniforms."""
    ro = 0.1 + 2 * a[0]
    p = 0.05 + 3 * a[1]
    v = [3 * (a[2] - 0.5), 3 * (a[3] - 0.5), 3 * (a[4] - 0.5)]
    b = [2 * (a[5] - 0.5), 2 * (a[6] - 0.5), 2 * (a[7] - 0.5)]
    return [ro, 100 * a[8], p, *v, *b] if with_q else [ro, p, *v, *b]


def hlldq_cases(n=120, seed=17):
    """Rows of 23: L[9], R[9], n[3] (a coordinate axis), rad, metod (2 or 3)."""
    u = W.splitmix64(seed, n * 20).reshape(n, 20)
    rows = []
    for i in range(n):
        a = u[i]
        L = mhd_state(a[0:9], True)
        R = mhd_state(a[9:18], True)
        if i % 7 == 0:  # weak normal field (the HLLD degenerate branch)
            L[6 + i % 3] = 1e-5
            R[6 + i % 3] = -1e-5
        rows.append([*L, *R, *AXES[i % 6], 0.01 + a[18], 2 + (i // 6) % 2])
    return np.array(rows)


def hlld_cases(n=120, seed=19):
    """Rows of 21: q1[8], q2[8], n[3] (unit), w, dist; only inputs whose wave
    speeds are ordered (the reference exits the process otherwise)."""
    from oracle import oracle as O

    prm = O.reference_params()
    u = W.splitmix64(seed, 4 * n * 22).reshape(4 * n, 22)
    rows = []
    for i in range(4 * n):
        a = u[i]
        q1 = mhd_state(a[0:8], False)
        q2 = mhd_state(a[8:16], False)
        if i % 5 == 0:
            nv = np.array(AXES[i % 6])
        else:
            nv = np.array([a[16] - 0.5, a[17] - 0.5, a[18] - 0.5])
            nv /= np.linalg.norm(nv)
        w = (a[19] - 0.5) * (4.0 if i % 3 == 0 else 0.5)
        if i % 11 == 0:  # field along the normal (the d <= eps frame branch)
            q1[5:8] = list(0.5 * nv)
            q2[5:8] = list(0.5 * nv)
        row = [*q1, *q2, *nv, w, 0.01 + a[20]]
        if O.hlld(prm, row[0:8], row[8:16], row[16:19], row[19], row[20])[3] == 0:
            rows.append(row)
        if len(rows) == n:
            break
    return np.array(rows)


def write_mhd():
    h = hlldq_cases()
    out = np.zeros((len(h), 10))
    for i, r in enumerate(h):
        t, P, PQ = ref.hlldq(r[0:9], r[9:18], r[18:21], r[21], int(r[22]))
        out[i] = [t, *P, PQ]
    np.savez_compressed(HERE / "kat_hlldq.npz", inputs=h, outputs=out)
    g = hlld_cases()
    out = np.zeros((len(g), 12))
    for i, r in enumerate(g):
        t, q, d = ref.hlld(r[0:8], r[8:16], r[16:19], r[19], r[20])
        out[i] = [t, *q, *d]
    np.savez_compressed(HERE / "kat_hlld.npz", inputs=g, outputs=out)


def write_checkpoint():
    """Setka::Save_Setka_ALL_ALPHA of the small rail grid with the reference's
    initial field and seeded moments, and the reference's own state after 3
    Go_5_komponent__MK2 steps on the grid Download_Setka_ALL_ALPHA_2_0 reads
    back from that file."""
    S = ref.RefSetka.constructor(*SMALL)
    S.tvd_prepare()
    S.init_conditions()
    m = Mesh.from_arrays(S.export())
    S.set_mc(*W.mc_fields(m, seed=23))
    import gzip
    import shutil
    import tempfile

    with tempfile.TemporaryDirectory() as tmp:
        path = Path(tmp) / "alpha_small.txt"
        S.save_alpha(path)
        R = ref.RefSetka.load_alpha(path)
        with open(path, "rb") as src, gzip.GzipFile(HERE / "alpha_small.txt.gz", "wb", mtime=0) as dst:
            shutil.copyfileobj(src, dst)
    R.tvd_prepare()
    R.go_mk2(3)
    pm = R.point_motion()
    np.savez_compressed(HERE / "steps_alpha_small.npz", par0=R.get_state(0), par1=R.get_state(1), x=pm["x"],
                        y=pm["y"])


def write_five_fluid():
    """Setka::Go_5_komponent on the small rail grid: the reference's field,
    seeded hydrogen fluids, 4 steps."""
    S = ref.RefSetka.constructor(*SMALL)
    S.tvd_prepare()
    S.init_conditions()
    m = Mesh.from_arrays(S.export())
    st0 = S.get_state(0)
    h0 = W.hydrogen_fields(m, seed=3)
    S.set_hydrogen(0, h0)
    S.set_hydrogen(1, h0)
    S.go_5_komponent(4)
    pm = S.point_motion()
    np.savez_compressed(HERE / "steps_five_fluid_small.npz", state0=st0, h0=h0, par0=S.get_state(0),
                        par1=S.get_state(1), h_par0=S.get_hydrogen(0), h_par1=S.get_hydrogen(1), x=pm["x"],
                        y=pm["y"])


def main(parts):
    ref.set_threads(1)
    if "five" in parts:
        write_five_fluid()
    if "checkpoint" in parts:
        write_checkpoint()
    if "mhd" in parts:
        write_mhd()
    if "faces" in parts:
        write_faces()
    if "steps" in parts:
        write_steps()
    print("golden fixtures written to", HERE)


def write_faces():
    h = hllc_cases()
    out = np.zeros((len(h), 9))
    for i, r in enumerate(h):
        t, P, PQ, v = ref.hllc(r[0:5], r[5:10], r[10], r[11], r[12], r[13], int(r[14]), bool(r[15]))
        out[i] = [t, *P, PQ, *v]
    np.savez_compressed(HERE / "kat_hllc.npz", inputs=h, outputs=out)
    g = godunov_cases()
    out = np.zeros((len(g), 9))
    for i, r in enumerate(g):
        t, q, d = ref.godunov(r[0:5], r[5:10], r[10:13], r[13], r[14])
        out[i] = [t, *q, *d]
    np.savez_compressed(HERE / "kat_godunov.npz", inputs=g, outputs=out)


def write_steps():
    # short runs on the small rail grid
    S = ref.RefSetka.constructor(*SMALL)
    S.tvd_prepare()
    S.init_conditions()
    m = Mesh.from_arrays(S.export())
    st0 = S.get_state(0)
    mc = W.mc_fields(m, seed=5)
    res = {"state0": st0, "Hn": mc[0], "Hu": mc[1], "Hv": mc[2], "HT": mc[3], "ku": mc[4], "kv": mc[5], "kT": mc[6]}
    for name, steps in (("stationary", 3), ("mk2", 4), ("inner", 3)):
        R = ref.RefSetka.constructor(*SMALL)
        R.tvd_prepare()
        R.set_state(0, st0)
        R.set_state(1, st0)
        R.set_mc(*mc)
        if name == "stationary":
            R.go_stationary(steps)
        elif name == "mk2":
            R.go_mk2(steps)
        else:
            R.build_inner_list()
            res["inner_list"] = R.inner_list()
            R.go_inner_mk2(steps)
        res[f"{name}_par0"] = R.get_state(0)
        res[f"{name}_par1"] = R.get_state(1)
        pm = R.point_motion()
        res[f"{name}_x"] = pm["x"]
        res[f"{name}_y"] = pm["y"]
    np.savez_compressed(HERE / "steps_small.npz", **res)


if __name__ == "__main__":
    main(sys.argv[1:] or ["faces", "steps", "mhd", "checkpoint", "five"])
