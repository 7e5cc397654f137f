"""Test infrastructure: a float64 numpy restatement of the warm-start network
(gelios_2d_b200/csrc/mlp.cu), the checker for its forward pass, loss and
gradients.  There is no reference counterpart: the reference has no learned
part, so the pins are (1) central finite differences of this restatement's
own loss (tests/test_warm_start.py) and (2) the device gradients compared
with this restatement on the same parameters and rows.

With ``bf16=True`` the restatement rounds where the device rounds (network
inputs, weights, hidden activations and backpropagated pre-activation
gradients to bfloat16, round to nearest even) and computes everything else
in float64; with ``bf16=False`` it is the exact float64 network.

Layout (as gelios_mlp): raw input rows of n_in, network input = raw row +
[sin(2^f pi s), cos(2^f pi s)] for f < n_fourier and s = the last two raw
entries; layers l = 0..depth, weight [out][in] then bias [out] in one flat
vector; GELU on the hidden layers, linear output; loss = mean over rows and
outputs of (y - t)^2.
"""
from __future__ import annotations

import math

import numpy as np

try:
    from scipy.special import erf as _erf
except ImportError:  # pragma: no cover
    _erf = np.vectorize(math.erf)

SQRT1_2 = 1.0 / math.sqrt(2.0)
INV_SQRT_2PI = 1.0 / math.sqrt(2.0 * math.pi)


def bf16(x: np.ndarray) -> np.ndarray:
    """float32 -> bfloat16 (round to nearest even), returned as float64."""
    u = np.ascontiguousarray(x, np.float32).view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def layout(n_in: int, n_fourier: int, width: int, depth: int, n_out: int):
    """(din, dout, w_off, b_off, n_params) per layer, as gelios_mlp_create."""
    in_w = n_in + 4 * n_fourier
    din, dout, w_off, b_off = [], [], [], []
    off = 0
    for l in range(depth + 1):
        di = in_w if l == 0 else width
        do = n_out if l == depth else width
        din.append(di)
        dout.append(do)
        w_off.append(off)
        off += di * do
        b_off.append(off)
        off += do
    return din, dout, w_off, b_off, off


def features(x: np.ndarray, n_fourier: int) -> np.ndarray:
    x = np.asarray(x, np.float64)
    cols = [x]
    for c in (x.shape[1] - 2, x.shape[1] - 1):
        s = x[:, c].astype(np.float32).astype(np.float64)
        w = np.float32(math.pi)
        for _ in range(n_fourier):
            a = (np.float32(w) * s.astype(np.float32)).astype(np.float64)
            cols.append(np.sin(a)[:, None])
            cols.append(np.cos(a)[:, None])
            w = np.float32(w * np.float32(2.0))
    return np.concatenate(cols, axis=1)


def gelu(z):
    return 0.5 * z * (1.0 + _erf(z * SQRT1_2))


def gelu_grad(z):
    return 0.5 * (1.0 + _erf(z * SQRT1_2)) + z * INV_SQRT_2PI * np.exp(-0.5 * z * z)


def _unpack(params, lay):
    din, dout, w_off, b_off, _ = lay
    Ws = [params[w_off[l]:w_off[l] + din[l] * dout[l]].reshape(dout[l], din[l]) for l in range(len(din))]
    bs = [params[b_off[l]:b_off[l] + dout[l]] for l in range(len(din))]
    return Ws, bs


def forward(params, x, n_fourier, lay, bf16_mode=False):
    """Output rows and the per-layer inputs / pre-activations."""
    p = np.asarray(params, np.float64)
    Ws, bs = _unpack(p, lay)
    rnd = bf16 if bf16_mode else (lambda a: np.asarray(a, np.float64))
    h = rnd(features(x, n_fourier))
    hs, zs = [h], []
    L = len(Ws)
    for l in range(L):
        z = h @ rnd(Ws[l]).T + bs[l]
        zs.append(z)
        if l < L - 1:
            h = rnd(gelu(z))
            hs.append(h)
    return zs[-1], hs, zs


def loss_grad(params, x, t, n_fourier, lay, bf16_mode=False):
    """(loss, flat gradient) of the mean squared error."""
    p = np.asarray(params, np.float64)
    Ws, _ = _unpack(p, lay)
    rnd = bf16 if bf16_mode else (lambda a: np.asarray(a, np.float64))
    y, hs, zs = forward(p, x, n_fourier, lay, bf16_mode)
    t = np.asarray(t, np.float64)
    M, No = y.shape
    d = y - t
    loss = float(np.sum(d * d) / (M * No))
    dz = 2.0 * d / (M * No)
    g = np.zeros_like(p)
    din, dout, w_off, b_off, _ = lay
    for l in range(len(Ws) - 1, -1, -1):
        dzr = rnd(dz)
        g[w_off[l]:w_off[l] + din[l] * dout[l]] = (dzr.T @ hs[l]).ravel()
        g[b_off[l]:b_off[l] + dout[l]] = dz.sum(axis=0)
        if l == 0:
            break
        dh = dzr @ rnd(Ws[l])
        dz = dh * gelu_grad(zs[l - 1])
    return loss, g
