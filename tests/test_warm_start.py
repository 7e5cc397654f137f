"""The learned warm start: the float64 restatement of the network (oracle/
mlp_oracle.py) pinned by finite differences, the host-side encoding, and on
the GPU the bf16 tensor-core GEMM, the device gradients against the
restatement, the batched plain solver against single contexts, and what
the trained network gains over the cold start."""
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT / "oracle"))

import mlp_oracle as O  # noqa: E402

from gelios_2d_b200 import warmstart as W  # noqa: E402
from gelios_2d_b200.mesh import Mesh  # noqa: E402
from gelios_2d_b200.workloads import plain_initial, plain_params  # noqa: E402


# ---------------------------------------------------------------- CPU
def test_bf16_rounding_is_nearest_even():
    one = 1.0
    assert O.bf16(np.array([one]))[0] == 1.0
    assert O.bf16(np.array([one + 2.0 ** -8]))[0] == 1.0  # tie -> even mantissa
    assert O.bf16(np.array([one + 2.0 ** -8 + 2.0 ** -12]))[0] == one + 2.0 ** -7
    assert O.bf16(np.array([one + 3 * 2.0 ** -8]))[0] == one + 2.0 ** -6  # tie -> even
    assert O.bf16(np.array([-3.0e-20]))[0] < 0


def test_oracle_gradient_matches_central_differences():
    rng = np.random.default_rng(4)
    n_in, nf, width, depth, n_out = 7, 2, 8, 2, 5
    lay = O.layout(n_in, nf, width, depth, n_out)
    p = rng.normal(0, 0.4, lay[4])
    x = rng.uniform(-1, 1, (13, n_in))
    t = rng.normal(size=(13, n_out))
    loss, g = O.loss_grad(p, x, t, nf, lay)
    h = 1e-6
    idx = rng.choice(p.size, 40, replace=False)
    for i in idx:
        e = np.zeros_like(p)
        e[i] = h
        fd = (O.loss_grad(p + e, x, t, nf, lay)[0] - O.loss_grad(p - e, x, t, nf, lay)[0]) / (2 * h)
        assert abs(fd - g[i]) <= 1e-7 * max(1.0, abs(g[i])), (i, fd, g[i])


def test_layout_matches_the_package():
    lay = O.layout(7, 6, 256, 5, 5)
    assert lay[4] == (31 * 256 + 256) + 4 * (256 * 256 + 256) + (256 * 5 + 5)


def test_inflow_sampling_and_parameters():
    a = W.sample_inflows(50, 3)
    assert np.array_equal(a, W.sample_inflows(50, 3))
    assert np.all(a >= W.PARAM_LO) and np.all(a <= W.PARAM_HI)
    p = W.inflow_params([0.005, 0.06, 2.0, 1.0, 10.0])
    ref = plain_params()
    for k in ("in_ro", "in_u", "chi", "inner_mach"):
        assert getattr(p, k) == getattr(ref, k)
    assert abs(p.in_p - ref.in_p) <= 1e-15 * ref.in_p


def test_cold_state_is_the_plain_workload_at_chi_one():
    mesh = Mesh.polar(30, 20, 1.0, 600.0)
    p = W.inflow_params([0.005, 0.06, 2.0, 1.0, 10.0])
    assert np.array_equal(W.cold_state(mesh, p), plain_initial(mesh, p))


def test_inputs_and_encoding():
    mesh = Mesh.polar(30, 20, 1.0, 600.0)
    x = W.cell_inputs(mesh, W.sample_inflows(1, 9)[0])
    assert x.shape == (mesh.n_cells, 7) and x.dtype == np.float32
    assert np.all(np.abs(x) <= 1.0 + 1e-6)
    st = W.cold_state(mesh, W.inflow_params(W.sample_inflows(1, 9)[0]))
    back = W.decode_state(W.encode_state(st))
    assert np.allclose(back, st, rtol=1e-12, atol=0)


def test_nearest_index_picks_the_closest_parameters():
    tr = W.sample_inflows(20, 1)
    assert np.array_equal(W.nearest_index(tr, tr), np.arange(20))


# ---------------------------------------------------------------- GPU
@pytest.mark.gpu
@pytest.mark.parametrize("shape", [(100, 72, 40, 40, 40), (256, 256, 256, 256, 256), (130, 31, 300, 301, 304),
                                   (8192, 5, 31, 31, 32), (333, 200, 1500, 1504, 1500)])
def test_gemm_bf16_against_float64(shape):
    """C = A . B^T for k-contiguous A [M][lda], B [N][ldb]: 16-byte staged
    rows (ld a multiple of 8) and element-wise staged rows, ragged M, N, K
    (K not a multiple of the 32-wide K tile or of the 8-element chunks)."""
    import torch

    from gelios_2d_b200 import _native as N

    M, Nn, K, lda, ldb = shape
    g = torch.Generator().manual_seed(M + Nn + K)
    A = torch.randn(M, lda, generator=g).to(torch.bfloat16)
    B = torch.randn(Nn, ldb, generator=g).to(torch.bfloat16)
    ref = A[:, :K].double() @ B[:, :K].double().t()
    Ad, Bd = A.contiguous().cuda(), B.contiguous().cuda()
    C = torch.full((M, Nn), float("nan"), dtype=torch.float32, device="cuda")
    L = N.lib()
    torch.cuda.synchronize()
    N.check(L.gelios_mlp_gemm_bf16(M, Nn, K, Ad.data_ptr(), lda, Bd.data_ptr(), ldb, C.data_ptr(), Nn, None), "gemm")
    torch.cuda.synchronize()
    err = (C.double().cpu() - ref).abs().max().item()
    assert err <= 1e-5 * ref.abs().max().item() * max(1.0, K / 64), err


@pytest.mark.gpu
def test_hidden_layer_timing_runs():
    """gelios_mlp_time_layer: the TMA-staged GEMM with its bias + GELU
    epilogue on the 8192 x 256 x 256 hidden layer of the warm-start network."""
    import ctypes as C

    from gelios_2d_b200 import _native as N

    for tma in (1, 0):
        ms = C.c_double()
        N.check(N.lib().gelios_mlp_time_layer(8192, 256, 256, 20, tma, C.byref(ms)), "gelios_mlp_time_layer")
        assert ms.value > 0.0
        print(f"hidden layer 8192x256x256 ({'TMA, fused epilogue' if tma else 'cp.async + bias/GELU kernel'}): "
              f"{ms.value * 1e3:.2f} us, {2 * 8192 * 256 * 256 / (ms.value * 1e-3) / 1e12:.1f} TFLOP/s")


@pytest.mark.gpu
def test_device_gradients_match_the_float64_restatement():
    net = W.Mlp(7, 6, 64, 3, 5, 2048)
    try:
        p = net.init_params(3)
        rng = np.random.default_rng(0)
        x = rng.uniform(-1, 1, (1500, 7)).astype(np.float32)  # 1500 rows: the weight gradients are split over K
        t = rng.normal(size=(1500, 5)).astype(np.float32)
        loss, g = net.loss_grad(x, t)
    finally:
        net.close()
    lay = O.layout(7, 6, 64, 3, 5)
    lb, gb = O.loss_grad(p.astype(np.float64), x, t, 6, lay, bf16_mode=True)
    ld, gd = O.loss_grad(p.astype(np.float64), x, t, 6, lay, bf16_mode=False)
    assert abs(loss - lb) <= 1e-5 * lb and abs(loss - ld) <= 1e-3 * ld
    din, dout, w_off, b_off, _ = lay
    for l in range(len(din)):
        for a, n in ((w_off[l], din[l] * dout[l]), (b_off[l], dout[l])):
            # same roundings as the device: fp32 accumulation order only
            assert np.linalg.norm(g[a:a + n] - gb[a:a + n]) <= 2e-3 * np.linalg.norm(gb[a:a + n])
            # exact float64 network: the bf16 roundings
            assert np.linalg.norm(g[a:a + n] - gd[a:a + n]) <= 3e-2 * np.linalg.norm(gd[a:a + n])


@pytest.mark.gpu
def test_training_reduces_the_loss_on_a_smooth_map():
    net = W.Mlp(7, 4, 64, 3, 5, 4096)
    try:
        net.init_params(5)
        rng = np.random.default_rng(2)
        x = rng.uniform(-1, 1, (20000, 7)).astype(np.float32)
        t = np.stack([np.sin(2 * x[:, 5]) * x[:, 0], np.cos(3 * x[:, 6]), x[:, 1] * x[:, 2], x[:, 5] ** 2,
                      np.tanh(x[:, 3] + x[:, 6])], axis=1).astype(np.float32)
        net.set_data(x, t)
        hist = net.train(600, 2048, 3e-3, 1e-4, 50, 1)
    finally:
        net.close()
    assert np.all(np.isfinite(hist))
    assert hist[-20:].mean() < 0.05 * hist[:20].mean()


@pytest.mark.gpu
def test_plain_batch_equals_single_contexts():
    import ctypes as C

    import gelios_2d_b200 as g
    from gelios_2d_b200 import _native as N

    mesh = Mesh.polar(60, 40, 1.0, 600.0)
    th = W.sample_inflows(3, 11)
    sts = [W.cold_state(mesh, W.inflow_params(t)) for t in th]
    single = []
    for t, st in zip(th, sts):
        S = g.Setka(mesh, W.inflow_params(t))
        S.set_par(0, st)
        S.set_par(1, st)
        S.step(N.FORM_STATIONARY, 20)
        single.append((S.par(0), S.par(1)))
        S.close()
    ss = [g.Setka(mesh, W.inflow_params(t)) for t in th]
    try:
        for S, st in zip(ss, sts):
            S.set_par(0, st)
            S.set_par(1, st)
        L = N.lib()
        hs = (C.c_void_p * 3)(*[S._h for S in ss])
        b = C.c_void_p()
        N.check(L.gelios_plain_batch_create(C.byref(b), hs, 3), "gelios_plain_batch_create")
        stt = (N.GeliosStatus * 3)()
        try:
            N.check(L.gelios_plain_batch_step(b, 20, stt), "gelios_plain_batch_step")
        finally:
            L.gelios_plain_batch_destroy(b)
        for S, (s0, s1), st in zip(ss, single, stt):
            assert st.flags == 0 and st.result_buf == 0 and st.dt > 0
            assert np.array_equal(S.par(0), s0) and np.array_equal(S.par(1), s1)
    finally:
        for S in ss:
            S.close()


@pytest.mark.gpu
def test_plain_batch_run_to_residual_equals_single_runs():
    mesh = Mesh.polar(45, 30, 1.0, 600.0)
    th = W.sample_inflows(3, 12)
    sts = [W.cold_state(mesh, W.inflow_params(t)) for t in th]
    bat = W.solve_batched(mesh, th, sts, 1e-4, 200_000, 1000)
    for i in range(3):
        one = W.solve_single(mesh, th[i], sts[i], 1e-4, 200_000, 1000)
        assert one.steps[0] == bat.steps[i]
        assert one.residual[0] == bat.residual[i] and one.residual[0] <= 1e-4
        assert np.array_equal(one.states[0], bat.states[i])


@pytest.mark.gpu
def test_warm_start_needs_fewer_steps_than_the_cold_start():
    mesh = Mesh.polar(45, 30, 1.0, 600.0)
    out, _ = W.experiment(mesh, n_train=48, n_test=6, chunk=64, train=dict(iters=2000), n_serial=0,
                          fp32_max_steps=0)
    cold, warm = out["cold_fp64"], out["warm_fp64"]
    assert cold["reached"] == 6 and warm["reached"] == 6 and out["fallbacks"] == 0
    # the network's start is closer to the converged state than the cold start
    assert out["prediction_vs_converged"]["rho_l1"] < 0.1
    assert warm["steps_mean"] * 4 < cold["steps_mean"]
    assert warm["wall_s"] < cold["wall_s"]
