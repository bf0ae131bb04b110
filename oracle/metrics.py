"""CPU oracle for the evaluation metrics (numpy, FP64).

TEST INFRASTRUCTURE ONLY: used by the tests as the checker, never by the
product path.

Restates the per-spectrum evaluation of train.py:672-701 with the helpers
it calls: calculate_psnr (train.py:76-83: 20 log10(1 / sqrt(mse)), inf when
mse == 0), calculate_rssi (train.py:86-91: 10 log10(mean x^2) - 30, used as
rssi(pred) - rssi(gt)), calculate_mae (train.py:99-101), utils.ssim (the
11x11 window SSIM, mean of the "same"-padded map, utils.py:81-114), the
renderer's confidence 1 + exp(fc2(relu(fc1(rx)))) (gaussian.py:575-609) and
the evaluation loss (1 - lambda1) l1 + lambda1 (1 - ssim) (train.py:696-697).
"""
from __future__ import annotations

import numpy as np

from .ssim import ssim_forward

NAMES = ("psnr", "rssi_diff", "mae", "ssim", "confidence", "loss")


def confidence(rx, conf_params, hidden):
    """ConfidenceMLP of one receiver; conf_params flat in nn.Module order."""
    p = np.asarray(conf_params, dtype=np.float64)
    w1 = p[:3 * hidden].reshape(hidden, 3)
    b1 = p[3 * hidden:4 * hidden]
    w2 = p[4 * hidden:5 * hidden]
    b2 = p[5 * hidden]
    h = np.maximum(w1 @ np.asarray(rx, dtype=np.float64) + b1, 0.0)
    return 1.0 + np.exp(w2 @ h + b2)


def evaluate(pred, target, rx, conf_params, hidden, lambda1=0.2):
    """[R,H,W] spectra -> [R,6] metrics in the order of NAMES (float64)."""
    pred = np.asarray(pred, dtype=np.float64)
    target = np.asarray(target, dtype=np.float64)
    out = np.zeros((pred.shape[0], len(NAMES)))
    for r in range(pred.shape[0]):
        p, t = pred[r], target[r]
        mse = np.mean((p - t) ** 2)
        psnr = np.inf if mse == 0 else 20.0 * np.log10(1.0 / np.sqrt(mse))
        rssi = lambda x: 10.0 * np.log10(np.mean(x ** 2)) - 30.0
        mae = np.mean(np.abs(p - t))
        ssim = ssim_forward(p, t, dtype=np.float64)[0].mean()
        out[r] = (psnr, rssi(p) - rssi(t), mae, ssim, confidence(rx[r], conf_params, hidden),
                  (1.0 - lambda1) * mae + lambda1 * (1.0 - ssim))
    return out
