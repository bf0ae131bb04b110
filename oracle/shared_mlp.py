"""CPU restatement (numpy) of the shared emission MLP of
gsparc_b200.shared_mlp / csrc/shared_mlp.cu, for one receiver.

TEST / CPU-BASELINE INFRASTRUCTURE ONLY: used by the CPU training step that
bench.py times; never used by the product.

Features per Gaussian (receiver rx): centre mu, sin/cos(2^k pi mu_j) for
k = 0..3, j = 0..2, (mu - rx)/d, 1/d^2, 0; culled Gaussians get zeros.
Hidden layers act(W x + b) (ReLU or erf-GELU), output o = w_o h + b_o,
signal = sigmoid(o).  Parameters flat: per layer W [out, in] then b [out].
"""
from __future__ import annotations

import math

import numpy as np
from scipy.special import erf


def shapes(layers, width, out=1):
    dims = [32] + [width] * layers + [out]
    return [(dims[i + 1], dims[i]) for i in range(len(dims) - 1)]


def unflatten(flat, layers, width, out=1):
    res, off = [], 0
    for o, i in shapes(layers, width, out):
        w = flat[off:off + o * i].reshape(o, i)
        off += o * i
        b = flat[off:off + o]
        off += o
        res.append((w, b))
    return res


def features(means, rx, radii, dtype=np.float32):
    means = means.astype(dtype)
    rx = np.asarray(rx).astype(dtype)
    v = means - rx[None, :]
    d2 = (v * v).sum(1, keepdims=True)
    d = np.sqrt(d2)
    pe = []
    for k in range(4):
        w = (2 ** k) * math.pi
        for j in range(3):
            pe += [np.sin(w * means[:, j]), np.cos(w * means[:, j])]
    with np.errstate(all="ignore"):
        x = np.concatenate([means, np.stack(pe, 1), v / d, 1.0 / d2, np.zeros_like(d)], 1)
    return np.where((radii > 0)[:, None], x, 0.0).astype(dtype)


def _act(act, z):
    return np.maximum(z, 0) if act == "relu" else 0.5 * z * (1 + erf(z / math.sqrt(2)))


def _act_grad(act, z):
    if act == "relu":
        return (z > 0).astype(z.dtype)
    return 0.5 * (1 + erf(z / math.sqrt(2))) + z * np.exp(-0.5 * z * z) / math.sqrt(2 * math.pi)


def forward(params, layers, width, act, means, rx, radii, dtype=np.float32):
    """Returns (signal [P], cache); computed in `dtype` (float64 for the FP64
    oracle render)."""
    lay = [(w.astype(dtype), b.astype(dtype)) for w, b in unflatten(params, layers, width)]
    x = features(means, rx, radii, dtype)
    hs, zs = [x], []
    h = x
    for w, b in lay[:-1]:
        z = h @ w.T + b
        zs.append(z)
        h = _act(act, z).astype(dtype)
        hs.append(h)
    w, b = lay[-1]
    s = (1.0 / (1.0 + np.exp(-(h @ w.T + b)[:, 0]))).astype(dtype)
    return s, (x, hs, zs, s)


def backward(params, layers, width, act, means, rx, radii, cache, dsig):
    """dsig [P] (real channel) -> (dparams flat, dmeans [P,3])."""
    lay = unflatten(params, layers, width)
    x, hs, zs, s = cache
    dz = (dsig * s * (1 - s))[:, None].astype(np.float32)
    grads = []
    for l in range(layers, -1, -1):
        w, _ = lay[l]
        grads.append((dz.T @ hs[l], dz.sum(0)))
        da = dz @ w
        dz = da * _act_grad(act, zs[l - 1]) if l > 0 else da
    dparams = np.concatenate([np.concatenate([gw.reshape(-1), gb]) for gw, gb in reversed(grads)]).astype(np.float32)
    dx = dz
    # features -> centres
    vis = radii > 0
    v = means - rx[None, :]
    d2 = (v * v).sum(1, keepdims=True)
    d = np.sqrt(np.where(vis[:, None], d2, 1.0))
    u = v / d
    dm = dx[:, 0:3].copy()
    for k in range(4):
        w = (2 ** k) * math.pi
        for j in range(3):
            dm[:, j] += w * (np.cos(w * means[:, j]) * dx[:, 3 + 6 * k + 2 * j]
                             - np.sin(w * means[:, j]) * dx[:, 4 + 6 * k + 2 * j])
    gu = (dx[:, 27:30] * u).sum(1, keepdims=True)
    dm += (dx[:, 27:30] - gu * u) / d + dx[:, 30:31] * (-2.0 / (d2 * d2 + (~vis[:, None]))) * v
    dm = np.where(vis[:, None], dm, 0.0)
    return dparams, dm.astype(np.float32)
