"""Native grid builders and TVD_prepare against the reference."""
import numpy as np
import pytest

from gelios_2d_b200.mesh import AXIS, INNER_SPHERE, USUALY, Mesh

DIMS = [(4, 3, 3, 10, 23, 6, 7, 7), (15, 5, 7, 15, 30, 10, 20, 20), (30, 7, 11, 20, 60, 20, 40, 40)]
TOPO_KEYS = ("x", "y", "point_type", "cell_type", "contour_start", "contour", "gran_start", "gran",
             "face_A", "face_B", "face_type", "face_master", "face_sosed", "face_copy", "rail_type", "rail_s",
             "rail_M", "rail_pstart", "rail_points", "rail_kstart", "rail_keys", "line_contact", "line_inner",
             "line_outer")
TVD_KEYS = ("face_sosed_up", "face_sosed_down", "cell_back", "cell_next", "r_istoch")


@pytest.mark.parametrize("dims", DIMS)
def test_setka_constructor_bitexact(dims, have_ref):
    from oracle import ref

    S = ref.RefSetka.constructor(*dims)
    a = S.export()
    b = Mesh.setka(*dims, tvd=False)
    assert a["n_main"] == b["n_main"]
    for k in TOPO_KEYS:
        assert a[k].dtype == b[k].dtype or k in ("x", "y", "rail_s")
        assert np.array_equal(a[k], b[k]), k
    S.tvd_prepare()
    a = S.export()
    b = Mesh.setka(*dims, tvd=True)
    for k in TVD_KEYS:
        assert np.array_equal(a[k], b[k]), k


def test_tvd_prepare_on_view_matches_builder():
    m = Mesh.setka(*DIMS[1])
    v = Mesh.from_arrays({k: val for k, val in m.items() if k not in TVD_KEYS})
    v.tvd_prepare()
    for k in TVD_KEYS:
        assert np.array_equal(v[k], m[k])


def test_polar_grid_consistency():
    """Proverka-style checks (Setka.cpp:2070-2196): quads, normals of interior
    faces point Master -> Sosed, twins reversed, positive areas."""
    m = Mesh.polar(36, 20, 1.0, 600.0)
    assert m.n_cells == 720
    assert np.all(np.diff(m["contour_start"]) == 4)
    assert np.all(np.diff(m["gran_start"]) == 4)
    c = m.centroids()
    x, y = m["x"], m["y"]
    for f in range(m["n_main"]):
        A, B = m["face_A"][f], m["face_B"][f]
        t = np.array([x[B] - x[A], y[B] - y[A]])
        n = np.array([t[1], -t[0]])
        Mc = m["face_master"][f]
        if m["face_type"][f] == USUALY:
            So = m["face_sosed"][f]
            assert np.dot(n, c[:, So] - c[:, Mc]) > 0
            cp = m["face_copy"][f]
            assert m["face_A"][cp] == B and m["face_B"][cp] == A
            assert m["face_master"][cp] == So and m["face_sosed"][cp] == Mc
        fc = np.array([(x[A] + x[B]) / 2, (y[A] + y[B]) / 2])
        assert np.dot(n, fc - c[:, Mc]) > 0  # outward from the master
    types = m["face_type"][: m["n_main"]]
    assert np.count_nonzero(types == AXIS) == 40
    assert np.count_nonzero(types == INNER_SPHERE) == 36
    # every face in a cell's list is mastered by that cell
    for cell in range(m.n_cells):
        for g in range(m["gran_start"][cell], m["gran_start"][cell + 1]):
            assert m["face_master"][m["gran"][g]] == cell


def test_polar_plain_grid_size():
    m = Mesh.polar()
    assert m.n_cells == 21600
    assert m.n_points == 181 * 121
