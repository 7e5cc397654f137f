"""The learned warm start of the plain step (no counterpart in the reference).

A coordinate network maps the inflow parameters of an instance of the plain
single-fluid problem (``workloads.plain_*``: the Go_stationary form on the
axisymmetric polar grid) and a cell position to the converged state of that
cell.  The converged states it learns from are produced by the batched plain
solver (``gelios_plain_batch``: many instances on one mesh marched together
to an L1 residual per unit time); its forward and backward passes are the
library's own kernels (``gelios_mlp_*``: bf16 tensor-core GEMMs with fp32
accumulation).  A prediction only chooses where time marching starts: every
warm-started instance is marched by the same solver to the same residual
tolerance as a cold-started one, and a prediction that is not finite and
positive where it must be falls back to the cold start.

Parameters of an instance (PARAM_NAMES): interstellar inflow density,
speed and Mach number, inner-wind speed chi and inner-wind Mach number.
Network input per cell: the five parameters scaled to [-1, 1], the scaled
log radius and the scaled polar angle (the kernel adds their Fourier
features).  Output: log rho, log p, u, v, log Q, standardised with the
training set's mean and spread.
"""
from __future__ import annotations

import ctypes as C
import time
from dataclasses import dataclass

import numpy as np

from . import _native as N
from .mesh import C_CENTR, Mesh
from .setka import Setka
from .workloads import plain_initial, plain_params, splitmix64

PARAM_NAMES = ("ro_lism", "u_lism", "mach_lism", "chi", "mach_inner")
PARAM_LO = np.array([0.002, 0.04, 1.5, 0.8, 8.0])
PARAM_HI = np.array([0.01, 0.08, 3.0, 1.2, 12.0])


def sample_inflows(n: int, seed: int) -> np.ndarray:
    """n parameter sets, uniform in [PARAM_LO, PARAM_HI] (splitmix64 of seed)."""
    u = splitmix64(seed, n * len(PARAM_NAMES)).reshape(n, len(PARAM_NAMES))
    return PARAM_LO + u * (PARAM_HI - PARAM_LO)


def inflow_params(theta, fp32: int = 0) -> N.GeliosParams:
    """gelios_params of the plain workload with the inflow of `theta`;
    fp32: 0 (or False) FP64 fluxes, 1 (or True) FP32 fluxes, 2 FP32 wave
    speeds with the fluxes assembled in FP64 (N.PREC_*)."""
    ro, u, mach, chi, mach_in = (float(v) for v in theta)
    p = plain_params()
    g = p.gamma
    p.in_ro = ro
    p.in_p = ro * u * u / (g * mach * mach)
    p.in_u = -u
    p.in_v = 0.0
    p.chi = chi
    p.inner_mach = mach_in
    p.precision = int(fp32)
    return p


def cold_state(mesh: Mesh, params: N.GeliosParams, seed: int = 2024) -> np.ndarray:
    """The plain workload's initial field for these parameters: the inner
    solution of wind speed chi (rho = 1/(chi r)^2, u_r = chi, p of Mach
    inner_mach at r = 1 falling as r^-2gamma) inside r = 150, the inflow
    beyond, seeded 1% density noise."""
    st = plain_initial(mesh, params, seed=seed)
    x, y = mesh.centroids()
    inner = np.sqrt(x * x + y * y) < 150.0
    chi = params.chi
    st[0, inner] /= chi * chi
    st[2, inner] *= chi
    st[3, inner] *= chi
    st[4, inner] /= chi * chi
    return st


def cell_inputs(mesh: Mesh, theta) -> np.ndarray:
    """Raw network inputs of every cell (n_cells x 7, float32)."""
    x, y = mesh.centroids()
    r = np.sqrt(x * x + y * y)
    rin, rout = float(r.min()), float(r.max())
    s_r = 2.0 * np.log(r / rin) / np.log(rout / rin) - 1.0
    s_t = 2.0 * np.arctan2(y, x) / np.pi - 1.0
    p = 2.0 * (np.asarray(theta, np.float64) - PARAM_LO) / (PARAM_HI - PARAM_LO) - 1.0
    out = np.empty((mesh.n_cells, 7), np.float32)
    out[:, :5] = p
    out[:, 5] = s_r
    out[:, 6] = s_t
    return out


def encode_state(st: np.ndarray) -> np.ndarray:
    """log rho, log p, u, v, log Q per cell (n_cells x 5)."""
    tiny = 1e-300
    return np.stack([np.log(np.maximum(st[0], tiny)), np.log(np.maximum(st[1], tiny)), st[2], st[3],
                     np.log(np.maximum(st[4], tiny))], axis=1)


def decode_state(y: np.ndarray) -> np.ndarray:
    return np.stack([np.exp(y[:, 0]), np.exp(y[:, 1]), y[:, 2], y[:, 3], np.exp(y[:, 4])], axis=0)


class Mlp:
    """gelios_mlp: the network on one GPU."""

    def __init__(self, n_in=7, n_fourier=6, width=256, depth=5, n_out=5, max_batch=8192, device=0):
        self.shape = (n_in, n_fourier, width, depth, n_out)
        self.max_batch = max_batch
        self._L = N.lib()
        h = C.c_void_p()
        N.check(self._L.gelios_mlp_create(C.byref(h), int(device), n_in, n_fourier, width, depth, n_out, max_batch),
                "gelios_mlp_create")
        self._h = h
        self.n_params = int(self._L.gelios_mlp_param_count(h))

    def close(self):
        if self._h:
            self._L.gelios_mlp_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def layout(self):
        """(din, dout, w_off, b_off) of every layer in the flat parameter vector."""
        n_in, nf, width, depth, n_out = self.shape
        din, dout, w_off, b_off, off = [], [], [], [], 0
        for l in range(depth + 1):
            di = n_in + 4 * nf if l == 0 else width
            do = n_out if l == depth else width
            din.append(di)
            dout.append(do)
            w_off.append(off)
            off += di * do
            b_off.append(off)
            off += do
        assert off == self.n_params
        return din, dout, w_off, b_off

    def init_params(self, seed: int) -> np.ndarray:
        """Weights uniform in +-1/sqrt(fan_in) (splitmix64 of seed), zero
        biases; loaded into the network and returned."""
        din, dout, w_off, b_off = self.layout()
        p = np.zeros(self.n_params, np.float64)
        for l in range(len(din)):
            n = din[l] * dout[l]
            u = splitmix64(seed * 1000 + l + 1, n)
            p[w_off[l]:w_off[l] + n] = (2.0 * u - 1.0) / np.sqrt(din[l])
        p = p.astype(np.float32)
        self.set_params(p)
        return p

    def set_params(self, p: np.ndarray):
        p = np.ascontiguousarray(p, np.float32)
        N.check(self._L.gelios_mlp_set_params(self._h, p, p.size), "gelios_mlp_set_params")

    def params(self) -> np.ndarray:
        p = np.zeros(self.n_params, np.float32)
        N.check(self._L.gelios_mlp_get_params(self._h, p, p.size), "gelios_mlp_get_params")
        return p

    def loss_grad(self, x: np.ndarray, t: np.ndarray) -> tuple[float, np.ndarray]:
        x = np.ascontiguousarray(x, np.float32)
        t = np.ascontiguousarray(t, np.float32)
        g = np.zeros(self.n_params, np.float32)
        loss = C.c_double()
        N.check(self._L.gelios_mlp_loss_grad(self._h, x, t, x.shape[0], C.byref(loss), g.ctypes.data),
                "gelios_mlp_loss_grad")
        return float(loss.value), g

    def set_data(self, x: np.ndarray, t: np.ndarray):
        x = np.ascontiguousarray(x, np.float32)
        t = np.ascontiguousarray(t, np.float32)
        N.check(self._L.gelios_mlp_set_data(self._h, x, t, x.shape[0]), "gelios_mlp_set_data")

    def train(self, iters: int, batch: int, lr_max: float, lr_min: float, warmup: int, seed: int) -> np.ndarray:
        hist = np.zeros(max(iters, 1), np.float32)
        N.check(self._L.gelios_mlp_train(self._h, int(iters), int(batch), float(lr_max), float(lr_min), int(warmup),
                                         int(seed), hist.ctypes.data), "gelios_mlp_train")
        return hist[:iters]

    def predict(self, x: np.ndarray) -> np.ndarray:
        x = np.ascontiguousarray(x, np.float32)
        y = np.zeros((x.shape[0], self.shape[4]), np.float32)
        N.check(self._L.gelios_mlp_predict(self._h, x, x.shape[0], y), "gelios_mlp_predict")
        return y


# ---------------------------------------------------------------- solving
@dataclass
class Solve:
    """Result of marching instances to a residual: per instance the steps
    run, the final residual per unit time and dt, the states reached, and
    the wall time of the whole solve (host clock around the solver calls)."""
    steps: np.ndarray
    residual: np.ndarray
    dt: np.ndarray
    states: np.ndarray
    wall_s: float


def solve_batched(mesh: Mesh, thetas, initial_states, tol: float, max_steps: int, check_every: int = 2000,
                  fp32: bool = False, device: int = 0) -> Solve:
    """All instances in one gelios_plain_batch, marched until each one's
    residual per unit time is at most tol."""
    n = len(thetas)
    ss = [Setka(mesh, inflow_params(thetas[i], fp32), device=device) for i in range(n)]
    try:
        for S, st in zip(ss, initial_states):
            S.set_par(0, st)
            S.set_par(1, st)
        L = N.lib()
        handles = (C.c_void_p * n)(*[S._h for S in ss])
        b = C.c_void_p()
        N.check(L.gelios_plain_batch_create(C.byref(b), handles, n), "gelios_plain_batch_create")
        steps = np.zeros(n, np.int64)
        res = np.zeros(n)
        dts = np.zeros(n)
        try:
            for S in ss:
                S.synchronize()
            t0 = time.perf_counter()
            N.check(L.gelios_plain_batch_run_to_residual(b, float(tol), int(max_steps), int(check_every),
                                                         steps.ctypes.data, res.ctypes.data, dts.ctypes.data),
                    "gelios_plain_batch_run_to_residual")
            wall = time.perf_counter() - t0
        finally:
            L.gelios_plain_batch_destroy(b)
        states = np.stack([S.par(0) for S in ss])
    finally:
        for S in ss:
            S.close()
    return Solve(steps, res, dts, states, wall)


def solve_single(mesh: Mesh, theta, initial_state, tol: float, max_steps: int, check_every: int = 2000,
                 fp32: bool = False, device: int = 0) -> Solve:
    """One instance on its own context (gelios_run_to_residual)."""
    S = Setka(mesh, inflow_params(theta, fp32), device=device)
    try:
        S.set_par(0, initial_state)
        S.set_par(1, initial_state)
        S.synchronize()
        t0 = time.perf_counter()
        steps, r, dt = S.run_to_residual(N.FORM_STATIONARY, tol, max_steps, check_every)
        wall = time.perf_counter() - t0
        st = S.par(0)
    finally:
        S.close()
    return Solve(np.array([steps]), np.array([r]), np.array([dt]), st[None], wall)


# ---------------------------------------------------------------- the network
class WarmStart:
    """The trained map (inflow parameters, cell) -> converged state on one mesh."""

    def __init__(self, mesh: Mesh, n_fourier=6, width=256, depth=5, max_batch=8192, device=0, seed=1):
        self.mesh = mesh
        self.net = Mlp(7, n_fourier, width, depth, 5, max_batch, device)
        self.net.init_params(seed)
        self.mean = np.zeros(5)
        self.std = np.ones(5)
        self.centr = mesh["cell_type"] == C_CENTR  # cells the step does not update

    def close(self):
        self.net.close()

    def fit(self, thetas, states, iters=4000, batch=8192, lr_max=2e-3, lr_min=2e-5, warmup=200, seed=7):
        """Train on converged states (n x 5 x n_cells) of the parameter sets
        thetas (n x 5); returns the loss of every step."""
        X = np.concatenate([cell_inputs(self.mesh, th) for th in thetas])
        Y = np.concatenate([encode_state(st) for st in states])
        self.mean = Y.mean(axis=0)
        self.std = np.maximum(Y.std(axis=0), 1e-12)
        T = ((Y - self.mean) / self.std).astype(np.float32)
        self.net.set_data(X, T)
        return self.net.train(iters, min(batch, self.net.max_batch), lr_max, lr_min, warmup, seed)

    def predict_encoded(self, theta) -> np.ndarray:
        """The prediction as encode_state rows (n_cells x 5)."""
        y = self.net.predict(cell_inputs(self.mesh, theta)).astype(np.float64)
        return y * self.std + self.mean

    def predict(self, theta) -> np.ndarray:
        """The predicted state (5 x n_cells)."""
        return decode_state(self.predict_encoded(theta))

    def delta_state(self, theta, theta_near, state_near) -> np.ndarray:
        """A converged state of nearby parameters moved by the network's
        change between the two parameter sets (in encode_state rows)."""
        y = encode_state(state_near) + self.predict_encoded(theta) - self.predict_encoded(theta_near)
        return decode_state(y)

    def initial_state(self, theta, params: N.GeliosParams | None = None) -> tuple[np.ndarray, bool]:
        """(warm start, True) or, if the prediction is unusable (not finite,
        non-positive density or pressure), (cold start, False)."""
        params = params if params is not None else inflow_params(theta)
        cold = cold_state(self.mesh, params)
        st = self.predict(theta)
        ok = bool(np.all(np.isfinite(st)) and np.all(st[0] > 0) and np.all(st[1] > 0))
        if not ok:
            return cold, False
        st[:, self.centr] = cold[:, self.centr]
        return st, True


def state_difference(a: np.ndarray, b: np.ndarray) -> dict:
    """Relative L1 and max differences of rho, p and |u| between two states."""
    out = {}
    for k, name in ((0, "rho"), (1, "p")):
        d = np.abs(a[k] - b[k])
        out[f"{name}_l1"] = float(d.sum() / np.abs(b[k]).sum())
        out[f"{name}_linf"] = float((d / np.abs(b[k])).max())
    ua = np.hypot(a[2], a[3])
    ub = np.hypot(b[2], b[3])
    out["u_l1"] = float(np.abs(ua - ub).sum() / ub.sum())
    return out


def nearest_index(thetas_train, thetas) -> np.ndarray:
    """Index of the training parameter set nearest (scaled to [-1, 1]) to each of `thetas`."""
    a = 2.0 * (np.asarray(thetas_train) - PARAM_LO) / (PARAM_HI - PARAM_LO)
    b = 2.0 * (np.asarray(thetas) - PARAM_LO) / (PARAM_HI - PARAM_LO)
    return np.argmin(((b[:, None, :] - a[None, :, :]) ** 2).sum(axis=2), axis=1)


def nearest_states(thetas_train, states_train, thetas) -> np.ndarray:
    """The converged training state of the nearest parameters: the warm
    start without a network."""
    return np.asarray(states_train)[nearest_index(thetas_train, thetas)]


def solve_in_chunks(mesh, thetas, states, tol, max_steps, check_every, chunk, fp32=False, device=0) -> Solve:
    """solve_batched over consecutive chunks of at most `chunk` instances."""
    parts = [solve_batched(mesh, thetas[i:i + chunk], states[i:i + chunk], tol, max_steps, check_every, fp32, device)
             for i in range(0, len(thetas), chunk)]
    return Solve(np.concatenate([p.steps for p in parts]), np.concatenate([p.residual for p in parts]),
                 np.concatenate([p.dt for p in parts]), np.concatenate([p.states for p in parts]),
                 sum(p.wall_s for p in parts))


def experiment(mesh: Mesh, n_train=256, n_test=32, tol=1e-6, max_steps=3_000_000, check_every=2000, chunk=64,
               seed_train=101, seed_test=202, train=None, n_serial=2, device=0, net=None, fp32_max_steps=100_000,
               train_states=None) -> dict:
    """The learned warm start end to end on one mesh:

    1. n_train parameter sets marched from the cold start to `tol` by the
       batched solver (FP64 fluxes): the training set;
    2. the network trained on them (GPU kernels);
    3. n_test held-out parameter sets marched to `tol` from the cold start
       (FP64), from the nearest training state (FP64), from the network's
       prediction (FP64 and FP32 fluxes), all batched; the first n_serial
       of them also cold on single contexts one after another (FP64); the
       FP32-flux leg is capped at fp32_max_steps (0: skipped).
    `train_states` (n_train x 5 x n_cells) replaces step 1 when given.
    Returns (summary: steps, wall times and state differences; the
    training states)."""
    train = dict(iters=4000, batch=8192, lr_max=2e-3, lr_min=2e-5, warmup=200, seed=7) | (train or {})
    th_tr = sample_inflows(n_train, seed_train)
    th_te = sample_inflows(n_test, seed_test)
    if train_states is None:
        cold_tr = [cold_state(mesh, inflow_params(t)) for t in th_tr]
        gen = solve_in_chunks(mesh, th_tr, cold_tr, tol, max_steps, check_every, chunk, False, device)
    else:
        gen = Solve(np.zeros(n_train, np.int64), np.zeros(n_train), np.zeros(n_train), np.asarray(train_states), 0.0)
    ws = WarmStart(mesh, device=device, **(net or {}))
    t0 = time.perf_counter()
    hist = ws.fit(th_tr, gen.states, **train)
    fit_s = time.perf_counter() - t0
    cold_te = [cold_state(mesh, inflow_params(t)) for t in th_te]
    t0 = time.perf_counter()
    warm = [ws.initial_state(t) for t in th_te]
    predict_s = time.perf_counter() - t0
    warm_te = [w for w, _ in warm]
    near = nearest_index(th_tr, th_te)
    nn_te = [gen.states[i] for i in near]
    delta_te = [ws.delta_state(th_te[k], th_tr[i], gen.states[i]) for k, i in enumerate(near)]
    delta_te = [d if np.all(np.isfinite(d)) and np.all(d[0] > 0) and np.all(d[1] > 0) else nn_te[k]
                for k, d in enumerate(delta_te)]
    cold = solve_in_chunks(mesh, th_te, cold_te, tol, max_steps, check_every, chunk, False, device)
    nn = solve_in_chunks(mesh, th_te, nn_te, tol, max_steps, check_every, chunk, False, device)
    w64 = solve_in_chunks(mesh, th_te, warm_te, tol, max_steps, check_every, chunk, False, device)
    dl = solve_in_chunks(mesh, th_te, delta_te, tol, max_steps, check_every, chunk, False, device)
    w32 = (solve_in_chunks(mesh, th_te, warm_te, tol, fp32_max_steps, check_every, chunk, True, device)
           if fp32_max_steps > 0 else None)
    w32w = solve_in_chunks(mesh, th_te, warm_te, tol, max_steps, check_every, chunk, N.PREC_FP32_WAVES, device)
    serial = [solve_single(mesh, th_te[i], cold_te[i], tol, max_steps, check_every, False, device)
              for i in range(min(n_serial, n_test))]
    ws.close()

    def stats(s: Solve | None) -> dict | None:
        if s is None:
            return None
        return {"wall_s": s.wall_s, "steps_mean": float(s.steps.mean()), "steps_max": int(s.steps.max()),
                "reached": int(np.sum(s.residual <= tol)), "residual_max": float(s.residual.max()),
                "steps": s.steps.tolist()}

    def diff(a: Solve | None, b: Solve) -> dict | None:
        if a is None:
            return None
        ds = [state_difference(a.states[i], b.states[i]) for i in range(len(a.states))]
        return {k: float(max(d[k] for d in ds)) for k in ds[0]}

    serial_per = float(np.mean([s.wall_s for s in serial])) if serial else None
    out = {
        "mesh_cells": mesh.n_cells, "n_train": n_train, "n_test": n_test, "tol": tol,
        "residual": "sum|ro(n+1)-ro(n)| / (dt sum|ro(n+1)|), checked every %d steps" % check_every,
        "train_set": stats(gen) | {"chunk": chunk},
        "fit": {"s": fit_s, "loss_first": float(hist[:50].mean()), "loss_last": float(hist[-50:].mean()),
                "params": ws.net.n_params, **train},
        "predict_s": predict_s, "fallbacks": int(sum(1 for _, ok in warm if not ok)),
        "cold_fp64": stats(cold), "nearest_fp64": stats(nn), "warm_fp64": stats(w64), "delta_fp64": stats(dl),
        "warm_fp32flux": stats(w32) | {"max_steps": fp32_max_steps} if w32 is not None else None,
        "warm_fp32waves": stats(w32w),
        "serial_cold_fp64": {"instances": len(serial), "wall_s_per_instance": serial_per,
                             "wall_s_projected_all": serial_per * n_test if serial_per else None,
                             "steps": [int(s.steps[0]) for s in serial]},
        "prediction_vs_converged": diff(Solve(None, None, None, np.stack(warm_te), 0.0), cold),
        "nearest_vs_converged": diff(Solve(None, None, None, np.stack(nn_te), 0.0), cold),
        "delta_vs_converged": diff(Solve(None, None, None, np.stack(delta_te), 0.0), cold),
        "converged_warm_vs_cold": diff(w64, cold), "converged_warm32_vs_cold": diff(w32, cold),
        "converged_warm32waves_vs_cold": diff(w32w, cold),
        "converged_nearest_vs_cold": diff(nn, cold), "converged_delta_vs_cold": diff(dl, cold),
    }
    return out, gen.states
