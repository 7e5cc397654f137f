"""Checkpoints: the reference's text format (Save_Setka_ALL_ALPHA /
Download_Setka_ALL_ALPHA_2_0, Setka.cpp:2355-2574, 2899-3257) and the exact
binary snapshot.

tests/golden/alpha_small.txt.gz was written by the reference's own
Save_Setka_ALL_ALPHA (tests/golden/make_golden.py), so the reader and the
writer are checked against the reference's file without the reference."""
import gzip
from pathlib import Path

import numpy as np
import pytest

import gelios_2d_b200 as g
from gelios_2d_b200 import _native as N
from gelios_2d_b200 import checkpoint as ck
from gelios_2d_b200 import workloads as W

GOLD = Path(__file__).resolve().parent / "golden"
ALPHA = GOLD / "alpha_small.txt.gz"
SMALL = (4, 3, 3, 10, 23, 6, 7, 7)
MESH_KEYS = ("x", "y", "point_type", "cell_type", "contour_start", "contour", "gran_start", "gran", "face_A",
             "face_B", "face_type", "face_master", "face_sosed", "face_copy", "face_sosed_up", "face_sosed_down",
             "cell_back", "cell_next", "r_istoch", "rail_type", "rail_s", "rail_M", "rail_pstart", "rail_points",
             "rail_kstart", "rail_keys", "line_contact", "line_inner", "line_outer")


def test_writer_reproduces_the_reference_file(tmp_path):
    """read -> write gives back the reference's file byte for byte (record
    order, Gran numbering with main_gran flags, Point::my_cell order, %g)."""
    c = ck.read_alpha(ALPHA)
    out = tmp_path / "again.txt"
    ck.write_alpha(out, c.mesh, c.par, c.mc, c.hydrogen, c.I)
    ref_text = gzip.open(ALPHA, "rt").read()
    assert out.read_text() == ref_text
    assert c.point_cells == ck.point_cells(c.mesh)


def test_reader_topology_matches_the_constructor_grid():
    """The file holds the constructor's grid: same points, cells, faces,
    rails and lines as the native constructor (coordinates to 6 digits)."""
    c = ck.read_alpha(ALPHA, tvd=False)
    m = g.Mesh.setka(*SMALL)
    for k in ("point_type", "cell_type", "contour_start", "contour", "gran_start", "gran", "face_A", "face_B",
              "face_type", "face_master", "face_sosed", "face_copy", "rail_type", "rail_M", "rail_pstart",
              "rail_points", "rail_kstart", "rail_keys", "line_contact", "line_inner", "line_outer"):
        assert np.array_equal(c.mesh[k], m[k]), k
    assert int(c.mesh["n_main"]) == int(m["n_main"])
    assert np.array_equal(c.mesh["dims"], np.array(SMALL))
    assert np.allclose(c.mesh["x"], m["x"], rtol=1e-5, atol=0)
    assert np.allclose(c.mesh["y"], m["y"], rtol=1e-5, atol=1e-300)


def test_reader_matches_the_reference_loader(have_ref):
    """Our reader + TVD_prepare with the loader's unique face numbers against
    the reference's Download_Setka_ALL_ALPHA_2_0 + TVD_prepare, bit for bit."""
    from oracle import ref

    c = ck.read_alpha(ALPHA)
    import tempfile

    with tempfile.TemporaryDirectory() as tmp:
        txt = Path(tmp) / "alpha.txt"
        txt.write_text(gzip.open(ALPHA, "rt").read())
        R = ref.RefSetka.load_alpha(txt)
        R.tvd_prepare()
        e = R.export()
        st = R.get_state(0)
    for k in MESH_KEYS:
        assert np.array_equal(np.asarray(c.mesh[k]), np.asarray(e[k]).astype(np.asarray(c.mesh[k]).dtype)), k
    assert np.array_equal(c.par, st)


def test_face_numbering_matters_to_tvd_prepare():
    """TVD_prepare on the same arrays with the constructor's colliding face
    numbers and with the loader's unique ones (Setka.cpp:1328, 1383): the
    TVD neighbours differ (the reference-loader test above shows which one
    the reference takes), the source chains do not."""
    c = ck.read_alpha(ALPHA, tvd=False)
    a = g.Mesh.from_arrays(dict(c.mesh))
    a["face_numbering"] = "unique"
    a.tvd_prepare()
    b = g.Mesh.from_arrays(dict(c.mesh))
    b.pop("face_numbering", None)
    b.tvd_prepare()
    assert np.array_equal(a["cell_back"], b["cell_back"])
    assert np.array_equal(a["r_istoch"], b["r_istoch"])
    assert np.count_nonzero(a["face_sosed_up"] != b["face_sosed_up"]) > 0


def test_snapshot_is_exact(tmp_path):
    m = g.Mesh.setka(*SMALL)
    st = W.init_conditions_reference(m)
    rng = np.random.default_rng(5)
    st1 = st * (1 + 1e-3 * rng.standard_normal(st.shape))
    mc = W.mc_fields(m, seed=3)
    p = tmp_path / "snap.npz"
    ck.save_snapshot(p, m, st, st1, mc)
    m2, a, b, mc2 = ck.load_snapshot(p)
    assert np.array_equal(a, st) and np.array_equal(b, st1)
    for k in MESH_KEYS:
        assert np.array_equal(m2[k], m[k]), k
    assert int(m2["n_main"]) == int(m["n_main"])
    for x, y in zip(mc, mc2):
        assert np.array_equal(x, y)


@pytest.mark.gpu
def test_checkpoint_grid_steps_like_the_reference():
    """The device path on a grid read from the reference's checkpoint: three
    Go_5_komponent__MK2 steps against the reference's own steps on the grid
    its loader read from the same file."""
    c = ck.read_alpha(ALPHA)
    gd = np.load(GOLD / "steps_alpha_small.npz")
    dev = g.Setka(c.mesh, N.reference_params())
    dev.set_par(0, c.par)
    dev.set_par(1, c.par)
    dev.set_mc(*c.mc)
    dev.Go_5_komponent__MK2(3)

    def rel(a, b):
        return max(float(np.max(np.abs(a[k] - b[k])) / np.max(np.abs(b[k]))) for k in range(5))

    assert rel(dev.par(1), gd["par1"]) <= 1e-12
    assert rel(dev.par(0), gd["par0"]) <= 1e-12
    x, y = dev.points()
    assert np.max(np.abs(x - gd["x"]) / np.maximum(np.abs(gd["x"]), 1e-3)) <= 1e-13
    assert np.max(np.abs(y - gd["y"]) / np.maximum(np.abs(gd["y"]), 1e-3)) <= 1e-13


@pytest.mark.gpu
def test_setka_save_and_download_round_trip(tmp_path):
    """Setka.Download_Setka_ALL_ALPHA_2_0 then Save_Setka_ALL_ALPHA gives back
    the reference's file (no step in between)."""
    S = g.Setka.Download_Setka_ALL_ALPHA_2_0(ALPHA)
    out = tmp_path / "saved.txt"
    S.Save_Setka_ALL_ALPHA(out)
    assert out.read_text() == gzip.open(ALPHA, "rt").read()
