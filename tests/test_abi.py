"""C ABI of libgelios_b200.so: loads, exports every declared symbol, and the
host side behaves without a GPU (no compute calls here)."""
import ctypes as C
import subprocess

import numpy as np
import pytest

from gelios_2d_b200 import _native as N
from oracle import oracle as O


def test_library_exports_every_header_symbol():
    L = N.lib()
    names = N.header_functions()
    assert len(names) >= 25
    for n in names:
        assert hasattr(L, n), n
    out = subprocess.run(["nm", "-D", "--defined-only", str(N._build.LIB)], capture_output=True, text=True).stdout
    for n in names:
        assert f" T {n}" in out, n


def test_library_is_sm100a_only():
    out = subprocess.run(["cuobjdump", "--list-elf", str(N._build.LIB)], capture_output=True, text=True).stdout
    assert "sm_100a" in out
    for bad in ("sm_80", "sm_90"):
        assert bad not in out


def test_params_layout_matches_oracle():
    assert C.sizeof(N.GeliosParams) == 216
    assert C.sizeof(N.GeliosParams) == C.sizeof(O.GoParams)
    a = N.reference_params()
    b = O.reference_params()
    for name, _ in O.GoParams._fields_:
        if name == "pad_":
            continue
        assert getattr(a, name) == getattr(b, name), name
    assert a.precision == N.PREC_FP64


def test_abi_version_and_errors():
    L = N.lib()
    assert L.gelios_abi_version() == 1
    h = C.c_void_p()
    p = N.reference_params()
    rc = L.gelios_create(C.byref(h), C.byref(p), 0)
    if rc == N.GELIOS_E_NODEVICE:
        assert b"no CUDA device" in L.gelios_last_error()
    else:  # on a GPU machine the context must come up
        assert rc == N.GELIOS_OK
        L.gelios_destroy(h)
    # argument errors are reported, never crash
    assert L.gelios_create(None, C.byref(p), 0) == N.GELIOS_E_ARG
    assert L.gelios_step(None, 0, 1, None) == N.GELIOS_E_ARG
    assert not L.gelios_mesh_build_setka(0, 0, 0, 0, 0, 0, 0, 0)
    assert not L.gelios_mesh_build_polar(1, 1, 1.0, 0.5)


def test_no_cpu_fallback_without_device():
    import gelios_2d_b200 as g

    m = g.Mesh.polar(8, 6)
    h = C.c_void_p()
    if N.lib().gelios_create(C.byref(h), C.byref(N.reference_params()), 0) == N.GELIOS_E_NODEVICE:
        with pytest.raises(N.GeliosError):
            g.Setka(m)
    else:
        N.lib().gelios_destroy(h)


def test_batch_schedule_and_source_entry_points_reject_null_handles():
    """Argument checks that need no GPU: a missing batch or context handle
    is refused before any CUDA call."""
    import numpy as np

    L = N.lib()
    assert L.gelios_batch_set_schedule(None, 1) == N.GELIOS_E_ARG
    assert L.gelios_batch_get_schedule(None, None) == N.GELIOS_E_ARG
    assert L.gelios_batch_autotune(None, 1, None, None, None, 0) == N.GELIOS_E_ARG
    q = np.zeros(1)
    assert L.gelios_mk2_source_terms(None, 0, q, q, q) == N.GELIOS_E_ARG
