"""CPU oracle for fused SSIM (numpy, FP32 or FP64).

TEST INFRASTRUCTURE ONLY: used by the tests and by bench.py's CPU baseline leg
as the checker, never by the product path.

Restates fused-ssim/ssim.cu (forward 187-286, backward 288-366) and the conv2d
SSIM of utils.py:81-124 that the reference tests it against
(fused-ssim/tests/test.py:24-54, :82, :90).  Pinned against golden vectors
produced by importing the reference's own ``utils.ssim``
(tests/golden/make_golden.py).

Padding: "same" = zero padding of 5 pixels (conv2d padding=window//2); the
reference's "valid" mode crops the map to [5:-5, 5:-5] before the mean
(fused_ssim/__init__.py:15-16).
"""
from __future__ import annotations

import math

import numpy as np

# The 11-tap Gaussian window (sigma 1.5) normalised to sum 1, as built by
# utils.py:116-124 (gaussian/create_window).
_g = np.array([math.exp(-((x - 5) ** 2) / (2 * 1.5 ** 2)) for x in range(11)], dtype=np.float64)
WINDOW64 = _g / _g.sum()
WINDOW32 = WINDOW64.astype(np.float32)
C1 = 0.01 ** 2
C2 = 0.03 ** 2


def _conv_same(img, w):
    """Separable 'same' correlation with zero padding over the last two axes:
    first along x (width), then along y, as ssim.cu:100-185 does."""
    dt = img.dtype
    H, W = img.shape[-2:]
    pad = np.zeros(img.shape[:-2] + (H + 10, W + 10), dtype=dt)
    pad[..., 5:5 + H, 5:5 + W] = img
    tmp = np.zeros(img.shape[:-2] + (H + 10, W), dtype=dt)
    for k in range(11):
        tmp = tmp + w[k] * pad[..., :, k:k + W]
    out = np.zeros(img.shape, dtype=dt)
    for k in range(11):
        out = out + w[k] * tmp[..., k:k + H, :]
    return out


def ssim_forward(img1, img2, dtype=np.float64, c1=C1, c2=C2):
    """fusedssimCUDA (ssim.cu:187-286).  Returns (map, dm_dmu1, dm_dsigma1_sq,
    dm_dsigma12), all shaped like the inputs ([B,CH,H,W] or [H,W])."""
    dt = np.dtype(dtype)
    w = WINDOW64.astype(dt)
    x = np.asarray(img1, dtype=dt)
    y = np.asarray(img2, dtype=dt)
    c1, c2 = dt.type(c1), dt.type(c2)
    two = dt.type(2)
    mu1 = _conv_same(x, w)
    mu2 = _conv_same(y, w)
    s11 = _conv_same(x * x, w) - mu1 * mu1
    s22 = _conv_same(y * y, w) - mu2 * mu2
    s12 = _conv_same(x * y, w) - mu1 * mu2
    C = two * mu1 * mu2 + c1
    D = two * s12 + c2
    A = mu1 * mu1 + mu2 * mu2 + c1
    B = s11 + s22 + c2
    m = (C * D) / (A * B)
    dm_dmu1 = ((mu2 * two * D) / (A * B) - (mu2 * two * C) / (A * B)
               - (mu1 * two * C * D) / (A * A * B) + (mu1 * two * C * D) / (A * B * B))
    dm_ds11 = (-C * D) / (A * B * B)
    dm_ds12 = (two * C) / (A * B)
    return m, dm_dmu1, dm_ds11, dm_ds12


def ssim_backward(img1, img2, dL_dmap, dm_dmu1, dm_ds11, dm_ds12, dtype=np.float64):
    """fusedssim_backwardCUDA (ssim.cu:288-366):
    dL/dimg1 = conv(dL*dm_dmu1) + 2*img1*conv(dL*dm_dsigma1_sq) + img2*conv(dL*dm_dsigma12)."""
    dt = np.dtype(dtype)
    w = WINDOW64.astype(dt)
    g = np.asarray(dL_dmap, dtype=dt)
    x = np.asarray(img1, dtype=dt)
    y = np.asarray(img2, dtype=dt)
    return (_conv_same(g * dm_dmu1, w) + x * dt.type(2) * _conv_same(g * dm_ds11, w)
            + y * _conv_same(g * dm_ds12, w))


def fused_ssim(img1, img2, padding="same", dtype=np.float64):
    """fused_ssim() (fused_ssim/__init__.py:34-41): mean of the SSIM map."""
    m = ssim_forward(img1, img2, dtype)[0]
    if padding == "valid":
        m = m[..., 5:-5, 5:-5]
    return m.mean()


def fused_ssim_grad(img1, img2, padding="same", dtype=np.float64):
    """d mean(SSIM map) / d img1, the gradient the autograd path produces."""
    m, a, b, c = ssim_forward(img1, img2, dtype)
    g = np.zeros_like(m)
    if padding == "valid":
        n = m[..., 5:-5, 5:-5].size
        g[..., 5:-5, 5:-5] = 1.0 / n
    else:
        g[...] = 1.0 / m.size
    return ssim_backward(img1, img2, g, a, b, c, dtype)
