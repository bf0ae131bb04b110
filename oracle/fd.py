"""FP64 finite-difference oracle for the rasterizer adjoint.

TEST INFRASTRUCTURE ONLY.

The forward of the splatting path has discrete decisions (culling, tile
coverage, alpha < 1/255 skips, early termination).  Central differences across
one of them measure a jump, not a derivative, so this module evaluates the
forward in FP64 with the set of contributing (pixel, list position, Gaussian)
triples frozen at the unperturbed point -- the function whose derivative the
hand-written backward computes (forward.cu:209-236 / backward.cu:544-614).
Everything continuous (projection, conic, opacity, emission MLP, the 0.99
alpha clamp) is re-evaluated under the perturbation.
"""
from __future__ import annotations

import numpy as np

from . import raster


def freeze(means, scales, rots, opac, mlp, view, tx, rx, H, W, tile_h=16, tile_w=16):
    """Run the FP64 forward once and record the contributing triples.

    Returns (pix [N] flat pixel index, gid [N] Gaussian id, order [N]) sorted by
    pixel then front-to-back order."""
    fwd = raster.render(means, scales, rots, opac, mlp, view, tx, rx, H, W,
                        tile_h=tile_h, tile_w=tile_w, dtype=np.float64)
    pre = fwd["pre"]
    _, _, _, rec = raster.blend_forward(fwd["ranges"], fwd["values"], pre["means2D"],
                                        pre["conic_opacity"], pre["signal"], H, W,
                                        tile_h, tile_w, np.float64, record=True)
    pix, gid, order = [], [], []
    for (y, x), trace in rec.items():
        for k, (j, g) in enumerate(trace):
            pix.append(y * W + x)
            gid.append(g)
            order.append(k)
    pix = np.array(pix, dtype=np.int64)
    gid = np.array(gid, dtype=np.int64)
    order = np.array(order, dtype=np.int64)
    idx = np.lexsort((order, pix))
    return pix[idx], gid[idx], order[idx], fwd


def frozen_render(frozen, means, scales, rots, opac, mlp, view, tx, rx, H, W):
    """FP64 render with the contribution set fixed.  Returns out [2,H,W]."""
    pix, gid, order = frozen[:3]
    pre = raster.preprocess(means, scales, rots, opac, mlp, view, tx, rx, H, W, dtype=np.float64)
    xy = pre["means2D"][gid]
    co = pre["conic_opacity"][gid]
    sg = pre["signal"][gid]
    px = (pix % W).astype(np.float64)
    py = (pix // W).astype(np.float64)
    dx = xy[:, 0] - px
    dy = xy[:, 1] - py
    power = -0.5 * (co[:, 0] * dx * dx + co[:, 2] * dy * dy) - co[:, 1] * dx * dy
    alpha = np.minimum(0.99, co[:, 3] * np.exp(power))
    L = np.log1p(-alpha)
    cs = np.cumsum(L)
    # exclusive prefix within each pixel segment
    start = np.ones(pix.size, dtype=bool)
    start[1:] = pix[1:] != pix[:-1]
    seg_first = np.maximum.accumulate(np.where(start, np.arange(pix.size), 0))
    excl = cs - L
    base = excl[seg_first]
    T_before = np.exp(excl - base)
    w = alpha * T_before
    out = np.zeros((2, H * W), dtype=np.float64)
    out[0] = np.bincount(pix, weights=w * sg[:, 0], minlength=H * W)
    out[1] = np.bincount(pix, weights=w * sg[:, 1], minlength=H * W)
    return out.reshape(2, H, W)
