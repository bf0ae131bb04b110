"""Generates tests/golden/ssim_golden.npz by importing the reference's own
conv2d SSIM (utils.py:81-124 -- the function fused-ssim/tests/test.py:24-54
checks the fused kernel against) and differentiating it with torch autograd
on the CPU.

Run in a container that has the reference checked out (GSPARC_REFERENCE_ROOT,
default as in oracle/build_ref.py):
    python tests/golden/make_golden.py
The reference's utils.py imports ``plyfile`` (for an unrelated PLY reader);
that package is not installed here, so an empty stand-in module is put in
sys.modules before the import.  Inputs are regenerated from the stored seeds
by ``golden_inputs`` (numpy PCG64), so only outputs are stored.
"""
from __future__ import annotations

import os
import sys
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
from oracle.build_ref import REF_ROOT as REF  # noqa: E402

# (name, shape, kind, seed)
CASES = [
    ("uniform_90x360", (90, 360), "uniform", 10),
    ("blobs_90x360", (90, 360), "blobs", 11),
    ("uniform_b2c3_37x53", (2, 3, 37, 53), "uniform", 12),
]


def golden_inputs(shape, kind, seed):
    """Deterministic image pair for a golden case (float32)."""
    rng = np.random.default_rng(seed)
    if kind == "uniform":
        a = rng.random(shape, dtype=np.float32)
        b = rng.random(shape, dtype=np.float32)
        return a, b
    # smooth spectra-like images: sums of anisotropic Gaussian blobs
    H, W = shape[-2:]
    yy, xx = np.mgrid[0:H, 0:W].astype(np.float64)
    def blobs():
        img = np.zeros((H, W))
        for _ in range(12):
            cy, cx = rng.uniform(0, H), rng.uniform(0, W)
            sy, sx = rng.uniform(2, 10), rng.uniform(3, 30)
            img += rng.uniform(0.1, 1.0) * np.exp(-0.5 * (((yy - cy) / sy) ** 2 + ((xx - cx) / sx) ** 2))
        return img.astype(np.float32)
    return blobs(), blobs()


def main():
    import torch
    sys.modules.setdefault("plyfile", types.SimpleNamespace(PlyData=None, PlyElement=None))
    sys.path.insert(0, REF)
    import utils as ref_utils  # the reference's utils.py
    out = {}
    for name, shape, kind, seed in CASES:
        a, b = golden_inputs(shape, kind, seed)
        x = torch.tensor(a, dtype=torch.float32, requires_grad=True)
        y = torch.tensor(b, dtype=torch.float32)
        if x.dim() == 2:
            val = ref_utils.ssim(x, y)               # utils.py:81-92 (unsqueezes to [1,1,H,W])
        else:
            ch = x.shape[1]
            win = ref_utils.create_window(11, ch)
            val = ref_utils._ssim(x, y, win, 11, ch)  # utils.py:94-114
        val.backward()
        out[name + "/value"] = np.float32(val.item())
        out[name + "/grad"] = x.grad.numpy().astype(np.float32)
    np.savez_compressed(os.path.join(HERE, "ssim_golden.npz"), **out)
    print("wrote", os.path.join(HERE, "ssim_golden.npz"), sorted(out))


if __name__ == "__main__":
    main()
