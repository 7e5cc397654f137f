"""Streamed host I/O (gelios_run_streamed): one-step calls whose input copy
(host -> device) and result copy (device -> host) overlap the neighbouring
calls' steps.  The results must be the bits of the plain sequence
upload par[0] -> gelios_step(form, 1) -> download par[1]."""
import numpy as np
import pytest
import torch

import gelios_2d_b200 as g
from gelios_2d_b200 import _native as N
from gelios_2d_b200 import workloads as W

SMALL = (4, 3, 3, 10, 23, 6, 7, 7)
MEDIUM = (30, 7, 11, 20, 60, 20, 40, 40)


def test_io_rows():
    L = N.lib()
    assert L.gelios_io_rows(N.FORM_MK2) == 5 and L.gelios_io_rows(N.FORM_STATIONARY) == 5
    assert L.gelios_io_rows(N.FORM_5_KOMPONENT) == 21 and L.gelios_io_rows(N.FORM_MHD_PUI) == 13


def _pinned(a):
    return torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy()


def _inputs(st0, extra, n, seed):
    """n input blocks: the state with seeded +-0.1% density perturbations."""
    u = W.splitmix64(seed, n * st0.shape[1]).reshape(n, -1)
    out = []
    for k in range(n):
        s = st0.copy()
        s[0] = s[0] * (1.0 + 0.002 * (u[k] - 0.5))
        out.append(_pinned(np.concatenate([s, extra]) if extra is not None else s))
    return out


def _setup(form, dims):
    mesh = g.Mesh.setka(*dims)
    P = N.reference_params()
    st0 = W.init_conditions_reference(mesh)

    def make():
        S = g.Setka(mesh, P)
        for b in (0, 1):
            S.set_par(b, st0)
        extra = None
        if form == N.FORM_MK2:
            S.set_mc(*W.mc_fields(mesh, seed=3))
        else:
            mp = W.mhd_params()
            extra = W.mhd_initial(mesh, st0, mp)
            S.set_mhd_params(mp)
            for b in (0, 1):
                S.set_mhd(b, extra)
            S.set_sources(*W.mhd_sources(mesh, seed=5))
        return S, extra

    return mesh, st0, make


@pytest.mark.gpu
@pytest.mark.parametrize("form,dims", [(N.FORM_MK2, MEDIUM), (N.FORM_MHD_PUI, SMALL)])
def test_streamed_matches_sequential_calls(form, dims):
    mesh, st0, make = _setup(form, dims)
    S1, extra = make()
    S2, _ = make()
    n = 5
    ins = _inputs(st0, extra, n, seed=11)
    outs = [_pinned(np.zeros_like(a)) for a in ins]
    S1.run_streamed(form, ins, outs)
    for k in range(n):
        S2.set_par(0, ins[k][:5])
        if extra is not None:
            S2.set_mhd(0, ins[k][5:])
        S2.step(form, 1)
        ref = S2.par(1)
        if extra is not None:
            ref = np.concatenate([ref, S2.mhd(1)])
        assert np.array_equal(outs[k], ref), k
    assert np.array_equal(S1.points()[0], S2.points()[0])
