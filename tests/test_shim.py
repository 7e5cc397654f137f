"""The C++ shim (include/gelios_setka_shim.hpp) that replaces the bodies of
Setka::Go_5_komponent__MK2, Go_stationary and
Go_stationary_5_komponent_inner_MK2 (Setka.h:176-186) in the reference's own
driver, built against the reference sources and the product library
(oracle/shim_harness.cpp, oracle/Makefile -> oracle/_ref/libgelios_shim.so).

* mirror(): the shim's flat view of a reference Setka equals the product's
  native grid builder (Setka(N1..M4) + TVD_prepare) array for array.
* step(): the shim steps a reference Setka in place; par[0], par[1] and the
  points it leaves in the reference's objects equal what the reference's own
  member function leaves there (<= 1e-12 relative per variable after 1-4
  steps; points <= 1e-13).
"""
from pathlib import Path

import ctypes as C
import numpy as np
import pytest

from gelios_2d_b200 import _native as N
from gelios_2d_b200 import workloads as W

SHIM = Path(__file__).resolve().parent.parent / "oracle" / "_ref" / "libgelios_shim.so"
DIMS = [(4, 3, 3, 10, 23, 6, 7, 7), (15, 5, 7, 15, 30, 10, 20, 20), W.SETKA_SMALL]


@pytest.fixture(scope="module")
def shim():
    if not SHIM.exists():
        pytest.skip("oracle/_ref/libgelios_shim.so not built (needs the reference tree at build time)")
    from oracle import ref

    return ref.shim_lib()


@pytest.mark.parametrize("dims", DIMS)
def test_shim_mirror_equals_native_builder(shim, dims):
    from oracle import ref

    S = ref.RefSetka.constructor(*dims, L=shim)
    S.tvd_prepare()
    msg = C.create_string_buffer(64)
    bad = shim.gshim_mirror_check(S.h, msg, 64)
    assert bad == 0, msg.value.decode()


def rel_err(a, b):
    out = 0.0
    for k in range(a.shape[0]):
        s = np.max(np.abs(b[k]))
        if s > 0:
            out = max(out, float(np.max(np.abs(a[k] - b[k])) / s))
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("form,steps", [(N.FORM_MK2, 1), (N.FORM_MK2, 4), (N.FORM_STATIONARY, 3),
                                        (N.FORM_INNER_MK2, 3)])
def test_shim_steps_reference_setka_like_the_reference(shim, form, steps):
    from oracle import ref
    from oracle import ref_workload as RW

    dims = W.SETKA_SMALL

    def setka():
        S = ref.RefSetka.constructor(*dims, L=shim)
        S.tvd_prepare()
        S.init_conditions()
        m = S.export()
        S.set_state(1, S.get_state(0))
        x, y = RW.centroids(m)
        S.set_mc(*RW.mc_fields(x, y, 5))
        if form == N.FORM_INNER_MK2:
            S.build_inner_list()
        return S

    ref.set_threads(1)
    a, b = setka(), setka()
    run = {N.FORM_MK2: a.go_mk2, N.FORM_STATIONARY: a.go_stationary, N.FORM_INNER_MK2: a.go_inner_mk2}[form]
    run(steps)
    h = shim.gshim_new()
    try:
        rc = shim.gshim_step(h, b.h, int(form), int(steps))
    finally:
        shim.gshim_free(h)
    assert rc == 0
    for buf in (0, 1):
        e = rel_err(b.get_state(buf), a.get_state(buf))
        assert e <= 1e-12, (buf, e)
    pa, pb = a.point_motion(), b.point_motion()
    for k in ("x", "y"):
        assert np.max(np.abs(pb[k] - pa[k]) / np.maximum(np.abs(pa[k]), 1e-3)) <= 1e-13
