"""Shared helpers for the GPU parity tests (not collected by pytest)."""
from __future__ import annotations

import numpy as np
import torch

from gsparc_b200 import raster, scenes
from oracle import raster as oraster


def make_inputs(P, R=1, seed=0, rx_seed=None, cluster_frac=0.0, device="cuda"):
    sc = scenes.make_scene(P, seed=seed, cluster_frac=cluster_frac)
    m, s, q, o = sc.activated()
    rxs = scenes.make_receivers(R, seed=scenes.SEED_RX if rx_seed is None else rx_seed)
    views = scenes.view_matrices(rxs)
    np_in = dict(means=m, scales=s, rots=q, opac=o, mlp=sc.mlp, views=views, tx=scenes.TX_POS, rxs=rxs)
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(device)
    th_in = dict(means=t(m), scales=t(s), rots=t(q), opac=t(o.reshape(-1)), mlp=t(sc.mlp), views=t(views),
                 tx=t(scenes.TX_POS), rxs=t(rxs))
    return np_in, th_in


def gpu_forward(th, H=90, W=360, tile=(16, 16), capacity=None):
    out_r, out_i, radii, st = raster.forward(th["means"], th["mlp"], th["opac"], th["scales"], th["rots"], H, W,
                                             1.0, th["views"], th["tx"], th["rxs"], tile=tile, capacity=capacity)
    torch.cuda.synchronize()
    return out_r, out_i, radii, st


def to_np(views):
    return {k: v.detach().cpu().numpy() for k, v in views.items()}


def reference_keys(point_list, ranges, depth):
    """Rebuild the reference's sorted 64-bit keys (tile << 32 | depth bits)
    from a per-tile point list and ranges."""
    dbits = depth.astype(np.float32).view(np.uint32).astype(np.uint64)
    keys = np.zeros(point_list.size, dtype=np.uint64)
    for t in range(ranges.shape[0]):
        s, e = int(ranges[t, 0]), int(ranges[t, 1])
        if e > s:
            keys[s:e] = (np.uint64(t) << np.uint64(32)) | dbits[point_list[s:e]]
    return keys


def ambiguous_radius(pre64):
    """Gaussians whose FP64 radius argument 3*sqrt(lambda) lies within 1e-4
    (relative) of an integer, or whose tile rectangle edges lie within 1e-4
    of a tile boundary: FP32 rounding may legitimately move those."""
    # recompute the pre-ceil value in FP64 from the conic inverse
    co = pre64["conic_opacity"]
    a, b, c = co[:, 0], co[:, 1], co[:, 2]
    det_c = a * c - b * b
    with np.errstate(all="ignore"):
        ca, cb, cc = c / det_c, -b / det_c, a / det_c
        det = ca * cc - cb * cb
        mid = 0.5 * (ca + cc)
        lam = mid + np.sqrt(np.maximum(0.1, mid * mid - det))
        v = 3.0 * np.sqrt(lam)
    frac = np.abs(v - np.round(v))
    return ~np.isfinite(v) | (frac < 1e-4 * np.maximum(v, 1.0))
