"""The allocation-free plain step (gelios_stationary_step_noalloc).

It exists for callers that cannot call cudaMalloc while they step (their
device memory comes from their own up-front pool, or they step where the
CUDA allocator must not be touched).  Its scratch is a fixed file-scope
device array, so its results must equal the context path's (gelios_step with
GELIOS_FORM_STATIONARY) on the same inputs, call after call, although every
call reuses the same scratch.  This file is collected last so that a run
stopping at the first failure has run every other test already.
"""
import ctypes as C

import numpy as np
import pytest

import gelios_2d_b200 as g
from gelios_2d_b200 import _native as N
from gelios_2d_b200 import workloads as W

pytestmark = pytest.mark.gpu


def rel_err(a, b):
    out = 0.0
    for k in range(a.shape[0]):
        s = np.max(np.abs(b[k]))
        if s > 0:
            out = max(out, float(np.max(np.abs(a[k] - b[k])) / s))
    return out


def device_grid_arrays(m: g.Mesh) -> dict:
    """Host form of the gelios_device_grid arrays of a mesh (same derivation
    as the context's topology upload)."""
    gran, gs = m["gran"], m["gran_start"]
    ft = m["face_type"][gran]
    sA, sB = m["face_A"][gran], m["face_B"][gran]
    ta, tb = m["point_type"][sA], m["point_type"][sB]
    god = ((ta == 6) & (tb == 6)) | ((ta == 7) & (tb == 7)) | ((ta == 8) & (tb == 8))
    npf = ((ta == 6) != (tb == 6)) | ((ta == 7) != (tb == 7)) | ((ta == 8) != (tb == 8))
    info = (ft.astype(np.uint32) & 7) | (god.astype(np.uint32) << 3) | (npf.astype(np.uint32) << 4)
    nc = m.n_cells
    flags = np.zeros(nc, np.uint32)
    cell_of_slot = np.repeat(np.arange(nc), np.diff(gs))
    np.bitwise_or.at(flags, cell_of_slot[ft == 4], 1)
    flags |= (m["cell_type"] == 0).astype(np.uint32) << 1
    flags |= (m["cell_type"] == 5).astype(np.uint32) << 2
    slot_of_face = -np.ones(m.n_faces, np.int64)
    slot_of_face[gran] = np.arange(len(gran))
    us, uc, ut = [], [], []
    for s_, f in enumerate(gran):
        if ft[s_] == 0 and f >= m["n_main"]:
            continue
        us.append(s_)
        uc.append(cell_of_slot[s_])
        ut.append(slot_of_face[m["face_copy"][f]] if ft[s_] == 0 else -1)
    return dict(x=m["x"], y=m["y"], contour_start=m["contour_start"], contour=m["contour"], gran_start=gs,
                cell_flags=flags, slot_A=sA.astype(np.int32), slot_B=sB.astype(np.int32),
                slot_nb=m["face_sosed"][gran].astype(np.int32), slot_info=info,
                unit_slot=np.array(us, np.int32), unit_cell=np.array(uc, np.int32), unit_twin=np.array(ut, np.int32))


def _case(name):
    """(mesh, params, initial state): the polar plain grid, or the
    reference's rail grid, whose central fan (C_centr cells) the step leaves
    unchanged."""
    if name == "polar":
        mesh = W.plain_mesh(48, 32)
        P = W.plain_params()
        return mesh, P, W.plain_initial(mesh, P, seed=11)
    mesh = g.Mesh.setka(*W.SETKA_SMALL)
    assert np.count_nonzero(mesh["cell_type"] == 5) > 0
    return mesh, N.reference_params(), W.init_conditions_reference(mesh)


@pytest.mark.parametrize("case", ["polar", "setka_with_central_fan"])
def test_noalloc_step_matches_context_step_twice(case):
    import torch

    mesh, P, st0 = _case(case)
    # the existing entry point: one and two steps through a context
    ctx = g.Setka(mesh, P)
    ctx.set_par(0, st0)
    ctx.set_par(1, st0)
    s1 = ctx.Go_stationary(1)
    ref1 = ctx.par(1)
    ctx.set_par(0, st0)
    ctx.set_par(1, st0)
    ctx.Go_stationary(2)
    ref2 = ctx.par(0)

    dev = torch.device("cuda:0")
    host = device_grid_arrays(mesh)
    t = {}
    for k, a in host.items():
        if a.dtype == np.float64:
            t[k] = torch.from_numpy(np.ascontiguousarray(a)).to(dev)
        elif a.dtype == np.uint32:
            t[k] = torch.from_numpy(np.ascontiguousarray(a).view(np.int32)).to(dev)
        else:
            t[k] = torch.from_numpy(np.ascontiguousarray(a, np.int32)).to(dev)
    grid = N.GeliosDeviceGrid()
    grid.n_cells = mesh.n_cells
    grid.n_slots = len(host["slot_A"])
    grid.n_units = len(host["unit_slot"])
    for k in t:
        setattr(grid, k, t[k].data_ptr())
    st_a = torch.from_numpy(np.ascontiguousarray(st0)).to(dev)
    # fresh outputs (NaN): every cell must be written, C_centr cells included
    st_b = torch.full_like(st_a, float("nan"))
    st_c = torch.full_like(st_a, float("nan"))
    dt = torch.tensor([P.dt0, 0.0, 0.0], dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream(dev).cuda_stream
    L = N.lib()

    def rows(x):
        return (C.c_void_p * 5)(*[x[k].data_ptr() for k in range(5)])

    # first call: dt0 -> state after one step, dt of the next step
    N.check(L.gelios_stationary_step_noalloc(C.byref(P), C.byref(grid), rows(st_a), rows(st_b),
                                             C.c_void_p(dt.data_ptr()), C.c_void_p(dt.data_ptr() + 8),
                                             C.c_void_p(stream)), "gelios_stationary_step_noalloc")
    # second call reuses the same scratch
    N.check(L.gelios_stationary_step_noalloc(C.byref(P), C.byref(grid), rows(st_b), rows(st_c),
                                             C.c_void_p(dt.data_ptr() + 8), C.c_void_p(dt.data_ptr() + 16),
                                             C.c_void_p(stream)), "gelios_stationary_step_noalloc")
    torch.cuda.synchronize(dev)
    out1 = st_b.cpu().numpy()
    out2 = st_c.cpu().numpy()
    assert np.isfinite(out1).all() and np.isfinite(out2).all()
    assert rel_err(out1, ref1) <= 1e-12
    assert rel_err(out2, ref2) <= 1e-12
    assert abs(dt[1].item() - s1.dt) <= 1e-12 * s1.dt


def test_noalloc_rejects_grids_beyond_the_scratch():
    import torch

    P = W.plain_params()
    grid = N.GeliosDeviceGrid()
    grid.n_cells = N.NOALLOC_MAX_CELLS + 1
    grid.n_slots = 4 * grid.n_cells
    grid.n_units = 2 * grid.n_cells
    dummy = torch.zeros(8, dtype=torch.float64, device="cuda:0")
    for k, _ in N.GeliosDeviceGrid._fields_[3:]:
        setattr(grid, k, dummy.data_ptr())
    rows = (C.c_void_p * 5)(*[dummy.data_ptr()] * 5)
    rc = N.lib().gelios_stationary_step_noalloc(C.byref(P), C.byref(grid), rows, rows, C.c_void_p(dummy.data_ptr()),
                                               C.c_void_p(dummy.data_ptr()), None)
    assert rc == N.GELIOS_E_LIMIT
    assert b"exceeds the fixed scratch" in N.lib().gelios_last_error()
