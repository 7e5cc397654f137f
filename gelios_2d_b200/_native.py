"""ctypes binding of the gelios_b200 C ABI (include/gelios_b200.h).

The shared library is built in-tree by ``gelios_2d_b200.build``; importing
this module never falls back to anything else: if the library is missing or
does not load, an ImportError-like RuntimeError is raised.
"""
from __future__ import annotations

import ctypes as C
import re
from pathlib import Path

import numpy as np

from . import build as _build

HEADER = Path(__file__).resolve().parent.parent / "include" / "gelios_b200.h"

GELIOS_OK = 0
GELIOS_E_ARG = -1
GELIOS_E_CUDA = -2
GELIOS_E_STATE = -3
GELIOS_E_NODEVICE = -4
GELIOS_E_MESH = -5
GELIOS_E_LIMIT = -6

FORM_STATIONARY = 0
FORM_MK2 = 1
FORM_INNER_MK2 = 2
FORM_5_KOMPONENT = 3
FORM_MHD_PUI = 4
PREC_FP64 = 0
PREC_FP32_FLUX = 1
PREC_FP32_WAVES = 2

_DOUBLE_FIELDS = ("gamma", "kurant", "chi", "inner_mach", "in_ro", "in_p", "in_u", "in_v", "in_Q",
                  "extern_u_par", "extern_u_tvd", "R11", "rad_stat", "R1", "R111", "R5", "Left", "koef",
                  "src_rmin", "src_rmax", "src_coef", "a_2", "ro_floor", "p_floor", "dt0")


class GeliosParams(C.Structure):
    """gelios_params: runtime form of the reference's compile-time constants."""

    _fields_ = [(n, C.c_double) for n in _DOUBLE_FIELDS] + [
        ("n_inner", C.c_int32), ("n_outer_shock", C.c_int32), ("godunov_max_iter", C.c_int32),
        ("precision", C.c_int32)]

    def copy(self, **over) -> "GeliosParams":
        p = GeliosParams()
        C.memmove(C.byref(p), C.byref(self), C.sizeof(self))
        for k, v in over.items():
            setattr(p, k, v)
        return p

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


class GeliosMhdParams(C.Structure):
    """gelios_mhd_params: boundary data of the MHD + pickup-proton form."""

    _fields_ = [(n, C.c_double) for n in ("lism_bx", "lism_by", "lism_bz", "inner_bphi", "pui_in_ro", "pui_in_p",
                                          "pui_inner_ro", "pui_inner_p")]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


_IP = C.POINTER(C.c_int32)
_DP = C.POINTER(C.c_double)


class GeliosMeshView(C.Structure):
    _fields_ = [
        ("dims", C.c_int32 * 8),
        ("n_points", C.c_int32), ("x", _DP), ("y", _DP), ("point_type", _IP),
        ("n_cells", C.c_int32), ("cell_type", _IP), ("contour_start", _IP), ("contour", _IP),
        ("gran_start", _IP), ("gran", _IP), ("cell_back", _IP), ("cell_next", _IP), ("r_istoch", _DP),
        ("n_faces", C.c_int32), ("n_main", C.c_int32),
        ("face_A", _IP), ("face_B", _IP), ("face_type", _IP), ("face_master", _IP), ("face_sosed", _IP),
        ("face_copy", _IP), ("face_sosed_up", _IP), ("face_sosed_down", _IP),
        ("n_rails", C.c_int32), ("rail_type", _IP), ("rail_s", _DP), ("rail_M", _IP), ("rail_pstart", _IP),
        ("rail_points", _IP), ("rail_kstart", _IP), ("rail_keys", _IP),
        ("n_contact", C.c_int32), ("n_inner_line", C.c_int32), ("n_outer_line", C.c_int32),
        ("line_contact", _IP), ("line_inner", _IP), ("line_outer", _IP),
    ]


class GeliosStatus(C.Structure):
    _fields_ = [("flags", C.c_int32), ("steps_done", C.c_int32), ("n_ro_clamp", C.c_int64),
                ("n_p_clamp", C.c_int64), ("dt", C.c_double), ("result_buf", C.c_int32), ("pad_", C.c_int32)]


_UP = C.POINTER(C.c_uint32)


class GeliosDeviceGrid(C.Structure):
    """gelios_device_grid: device pointers of a grid for the allocation-free step."""

    _fields_ = [("n_cells", C.c_int32), ("n_slots", C.c_int32), ("n_units", C.c_int32),
                ("x", C.c_void_p), ("y", C.c_void_p), ("contour_start", C.c_void_p), ("contour", C.c_void_p),
                ("gran_start", C.c_void_p), ("cell_flags", C.c_void_p), ("slot_A", C.c_void_p),
                ("slot_B", C.c_void_p), ("slot_nb", C.c_void_p), ("slot_info", C.c_void_p),
                ("unit_slot", C.c_void_p), ("unit_cell", C.c_void_p), ("unit_twin", C.c_void_p)]


NOALLOC_MAX_CELLS = 32768
NOALLOC_MAX_SLOTS = 131072


class GeliosError(RuntimeError):
    def __init__(self, code: int, where: str, msg: str):
        super().__init__(f"{where} failed with {code}: {msg}")
        self.code = code


_LIB: C.CDLL | None = None


def lib() -> C.CDLL:
    """Load (building first if stale) the native library."""
    global _LIB
    if _LIB is not None:
        return _LIB
    path = _build.build()
    L = C.CDLL(str(path))
    vp = C.c_void_p
    dp = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
    ip = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
    L.gelios_params_reference.argtypes = [C.POINTER(GeliosParams)]
    L.gelios_last_error.restype = C.c_char_p
    L.gelios_abi_version.restype = C.c_int
    L.gelios_mesh_build_setka.restype = vp
    L.gelios_mesh_build_setka.argtypes = [C.c_int] * 8
    L.gelios_mesh_build_polar.restype = vp
    L.gelios_mesh_build_polar.argtypes = [C.c_int, C.c_int, C.c_double, C.c_double]
    L.gelios_mesh_tvd_prepare.argtypes = [vp]
    L.gelios_tvd_prepare_view.argtypes = [C.POINTER(GeliosMeshView), ip, ip, ip, ip, dp]
    L.gelios_tvd_prepare_view_numbered.argtypes = [C.POINTER(GeliosMeshView), C.c_int, ip, ip, ip, ip, dp]
    L.gelios_mesh_inner_cells.argtypes = [vp, C.c_double, C.POINTER(C.c_int32), C.c_int32]
    L.gelios_mesh_get_view.argtypes = [vp, C.POINTER(GeliosMeshView)]
    L.gelios_mesh_free.argtypes = [vp]
    L.gelios_create.argtypes = [C.POINTER(vp), C.POINTER(GeliosParams), C.c_int]
    L.gelios_set_params.argtypes = [vp, C.POINTER(GeliosParams)]
    L.gelios_destroy.argtypes = [vp]
    L.gelios_upload_topology.argtypes = [vp, C.POINTER(GeliosMeshView)]
    L.gelios_upload_state.argtypes = [vp, C.c_int] + [dp] * 5
    L.gelios_download_state.argtypes = [vp, C.c_int] + [dp] * 5
    L.gelios_upload_hydrogen.argtypes = [vp, C.c_int, dp]
    L.gelios_download_hydrogen.argtypes = [vp, C.c_int, dp]
    L.gelios_upload_mc.argtypes = [vp] + [dp] * 7
    L.gelios_set_mhd_params.argtypes = [vp, C.POINTER(GeliosMhdParams)]
    L.gelios_upload_mhd.argtypes = [vp, C.c_int, dp]
    L.gelios_download_mhd.argtypes = [vp, C.c_int, dp]
    L.gelios_upload_sources.argtypes = [vp, dp, dp, dp]
    L.gelios_variant_count.argtypes = [C.c_int]
    L.gelios_io_rows.argtypes = [C.c_int]
    L.gelios_residual.argtypes = [vp, C.c_int, C.POINTER(C.c_double)]
    L.gelios_run_to_residual.argtypes = [vp, C.c_int, C.c_double, C.c_int64, C.c_int32, C.POINTER(C.c_int64),
                                         C.POINTER(C.c_double), C.POINTER(C.c_double)]
    L.gelios_batch_create.argtypes = [C.POINTER(vp), C.POINTER(vp), C.c_int]
    L.gelios_batch_step.argtypes = [vp, C.c_int, C.c_int, C.POINTER(GeliosStatus)]
    L.gelios_batch_destroy.argtypes = [vp]
    L.gelios_batch_set_schedule.argtypes = [vp, C.c_int32]
    L.gelios_batch_get_schedule.argtypes = [vp, C.POINTER(C.c_int32)]
    L.gelios_batch_autotune.argtypes = [vp, C.c_int, C.POINTER(C.c_int32), C.POINTER(C.c_double), C.c_void_p, C.c_int]
    L.gelios_plain_batch_create.argtypes = [C.POINTER(vp), C.POINTER(vp), C.c_int]
    L.gelios_plain_batch_step.argtypes = [vp, C.c_int, C.POINTER(GeliosStatus)]
    L.gelios_plain_batch_run_to_residual.argtypes = [vp, C.c_double, C.c_int64, C.c_int32, C.c_void_p, C.c_void_p,
                                                     C.c_void_p]
    L.gelios_plain_batch_destroy.argtypes = [vp]
    fp = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
    L.gelios_mlp_create.argtypes = [C.POINTER(vp), C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int]
    L.gelios_mlp_destroy.argtypes = [vp]
    L.gelios_mlp_param_count.restype = C.c_int64
    L.gelios_mlp_param_count.argtypes = [vp]
    L.gelios_mlp_set_params.argtypes = [vp, fp, C.c_int64]
    L.gelios_mlp_get_params.argtypes = [vp, fp, C.c_int64]
    L.gelios_mlp_loss_grad.argtypes = [vp, fp, fp, C.c_int, C.POINTER(C.c_double), C.c_void_p]
    L.gelios_mlp_set_data.argtypes = [vp, fp, fp, C.c_int64]
    L.gelios_mlp_train.argtypes = [vp, C.c_int, C.c_int, C.c_float, C.c_float, C.c_int, C.c_uint64, C.c_void_p]
    L.gelios_mlp_predict.argtypes = [vp, fp, C.c_int64, fp]
    L.gelios_mlp_gemm_bf16.argtypes = [C.c_int, C.c_int, C.c_int, vp, C.c_int64, vp, C.c_int64, vp, C.c_int64, vp]
    L.gelios_mlp_time_layer.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.POINTER(C.c_double)]
    L.gelios_run_streamed.argtypes = [vp, C.c_int, C.c_int, C.POINTER(C.c_void_p), C.POINTER(C.c_void_p)]
    L.gelios_autotune.argtypes = [vp, C.c_int, C.c_int, C.POINTER(C.c_int32), C.POINTER(C.c_double)]
    L.gelios_set_variant.argtypes = [vp, C.c_int, C.c_int32]
    L.gelios_get_variant.argtypes = [vp, C.c_int, C.POINTER(C.c_int32)]
    L.gelios_set_pipelined.argtypes = [vp, C.c_int]
    L.gelios_operator_residual.argtypes = [vp, C.c_int, C.c_int, C.POINTER(C.c_double)]
    L.gelios_mk2_source_terms.argtypes = [vp, C.c_int, dp, dp, dp]
    L.gelios_set_inner_cells.argtypes = [vp, C.POINTER(C.c_int32), C.c_int32]
    L.gelios_step.argtypes = [vp, C.c_int, C.c_int, C.POINTER(GeliosStatus)]
    L.gelios_download_points.argtypes = [vp, dp, dp]
    L.gelios_synchronize.argtypes = [vp]
    L.gelios_state_device_ptr.argtypes = [vp, C.c_int, C.POINTER(C.POINTER(C.c_double))]
    L.gelios_stream.restype = vp
    L.gelios_stream.argtypes = [vp]
    L.gelios_last_launch_count.restype = C.c_int64
    L.gelios_last_launch_count.argtypes = [vp]
    L.gelios_set_phase_timing.argtypes = [vp, C.c_int]
    L.gelios_phase_times.argtypes = [vp, dp, np.ctypeslib.ndpointer(np.int64, flags="C_CONTIGUOUS"), C.c_int]
    L.gelios_stationary_step_noalloc.argtypes = [C.POINTER(GeliosParams), C.POINTER(GeliosDeviceGrid),
                                                 C.POINTER(C.c_void_p), C.POINTER(C.c_void_p), C.c_void_p,
                                                 C.c_void_p, C.c_void_p]
    L.gelios_hllc_batch.argtypes = [C.POINTER(GeliosParams), C.c_int, dp, dp]
    L.gelios_godunov_batch.argtypes = [C.POINTER(GeliosParams), C.c_int, dp, dp]
    L.gelios_hlldq_batch.argtypes = [C.POINTER(GeliosParams), C.c_int, dp, dp]
    L.gelios_hlld_batch.argtypes = [C.POINTER(GeliosParams), C.c_int, dp, dp]
    _LIB = L
    return L


def check(rc: int, where: str) -> None:
    if rc != GELIOS_OK:
        msg = lib().gelios_last_error()
        raise GeliosError(rc, where, msg.decode() if msg else "")


def reference_params(**over) -> GeliosParams:
    """The reference's own constants (Help.h:39-114 and literals of Gran.cpp/Setka.cpp)."""
    p = GeliosParams()
    lib().gelios_params_reference(C.byref(p))
    for k, v in over.items():
        setattr(p, k, v)
    return p


def header_functions() -> list[str]:
    """Names of the functions declared in include/gelios_b200.h."""
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = re.findall(r"^[A-Za-z_][\w \*]*?\b(gelios_\w+)\s*\(", text, flags=re.M)
    return sorted(set(names))
