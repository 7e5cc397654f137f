"""gelios_2d_b200: B200-native (sm_100a) plasma time step of Gelios_2D.

The package holds the hot path only: CUDA kernels + host C++ behind a C ABI
(include/gelios_b200.h, built into gelios_2d_b200/_lib/libgelios_b200.so),
and a thin Python mirror of the reference's Setka operator interface.
"""
from . import _native
from ._native import GeliosParams, GeliosStatus, reference_params
from .mesh import Mesh
from .setka import Setka, StepError, godunov_batch, hllc_batch, hlld_batch, hlldq_batch

__all__ = ["GeliosParams", "GeliosStatus", "Mesh", "Setka", "StepError", "godunov_batch", "hllc_batch",
           "hlld_batch", "hlldq_batch", "reference_params", "_native"]
