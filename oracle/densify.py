"""CPU oracle for densification (numpy).

TEST INFRASTRUCTURE ONLY: used by the tests as the checker, never by the
product path.

Restates GaussianModel.densify_and_prune (gaussian.py:515-542) with the
helpers it calls -- densify_and_clone (493-513), densify_and_split
(448-491), prune_points (308-337), densification_postfix (395-443),
cat_tensors_to_optimizer (339-393), _prune_optimizer (266-306) -- on raw
parameter arrays and Adam moments, step by step in the reference's order
(append clones, append the split copies stacked copy by copy, drop the
split originals, prune).  The normal samples of the split come from the
same counter-based generator as the device code (SplitMix64, Box-Muller),
restated here in uint64 / float64; the reference draws them with
torch.normal.
"""
from __future__ import annotations

import numpy as np

M64 = (1 << 64) - 1


def _splitmix64(x):
    x = (x + 0x9E3779B97F4A7C15) & M64
    x = ((x ^ (x >> 30)) * 0xBF58476D1CE4E5B9) & M64
    x = ((x ^ (x >> 27)) * 0x94D049BB133111EB) & M64
    return x ^ (x >> 31)


def normal(seed, g, k, d):
    """Standard normal sample for (seed, Gaussian g, copy k, axis d)."""
    h = _splitmix64(seed ^ _splitmix64(((g << 8) | (k * 4 + d)) & M64))
    u1 = ((h >> 40) + 1) / 16777216.0
    u2 = (((h >> 16) & 0xFFFFFF) + 1) / 16777216.0
    return np.sqrt(-2.0 * np.log(u1)) * np.cos(2.0 * np.pi * u2)


def build_rotation(q):
    """utils.py build_rotation: (w, x, y, z) quaternions -> [N,3,3]."""
    q = q / np.linalg.norm(q, axis=1, keepdims=True)
    r, x, y, z = q[:, 0], q[:, 1], q[:, 2], q[:, 3]
    R = np.zeros((q.shape[0], 3, 3))
    R[:, 0, 0] = 1 - 2 * (y * y + z * z)
    R[:, 0, 1] = 2 * (x * y - r * z)
    R[:, 0, 2] = 2 * (x * z + r * y)
    R[:, 1, 0] = 2 * (x * y + r * z)
    R[:, 1, 1] = 1 - 2 * (x * x + z * z)
    R[:, 1, 2] = 2 * (y * z - r * x)
    R[:, 2, 0] = 2 * (x * z - r * y)
    R[:, 2, 1] = 2 * (y * z + r * x)
    R[:, 2, 2] = 1 - 2 * (x * x + y * y)
    return R


KEYS = ("centre", "log_scale", "rotation", "opacity", "mlp")


def densify_and_prune(state, m1, m2, accum, denom, max_grad, min_opacity, extent, max_screen_size=None,
                      scene_min=None, scene_max=None, percent_dense=0.01, seed=0, split_samples=None):
    """state / m1 / m2: dicts of per-Gaussian arrays (KEYS; "mlp" [P,194] or
    absent); returns the new (state, m1, m2) with float64 values.
    ``split_samples`` [2n, 3], if given, replaces the split's offsets
    stds * z (the draws of torch.normal(0, stds) at gaussian.py:471, in its
    row order: copy-major, then selected Gaussian)."""
    keys = [k for k in KEYS if k in state]
    st = {k: np.asarray(state[k], dtype=np.float64).copy() for k in keys}
    a1 = {k: np.asarray(m1[k], dtype=np.float64).copy() for k in keys}
    a2 = {k: np.asarray(m2[k], dtype=np.float64).copy() for k in keys}
    P = st["centre"].shape[0]
    with np.errstate(invalid="ignore", divide="ignore"):
        grads = np.asarray(accum, dtype=np.float64) / np.asarray(denom, dtype=np.float64)
    grads[np.isnan(grads)] = 0.0
    scaling = lambda: np.exp(st["log_scale"])

    def append(new):
        for k in keys:
            st[k] = np.concatenate([st[k], new[k]])
            a1[k] = np.concatenate([a1[k], np.zeros_like(new[k])])
            a2[k] = np.concatenate([a2[k], np.zeros_like(new[k])])

    def prune(mask):
        keep = ~mask
        for k in keys:
            st[k], a1[k], a2[k] = st[k][keep], a1[k][keep], a2[k][keep]

    # densify_and_clone (|grad| of a [P,1] tensor is its absolute value)
    sel = (np.abs(grads) >= max_grad) & (scaling().max(axis=1) <= percent_dense * extent)
    append({k: st[k][sel] for k in keys})
    # densify_and_split on the grown set, gradients of the clones padded with zero
    n1 = st["centre"].shape[0]
    padded = np.zeros(n1)
    padded[:P] = grads
    sel = (padded >= max_grad) & (scaling().max(axis=1) > percent_dense * extent)
    idx = np.nonzero(sel)[0]
    s = scaling()[idx]
    stds = np.concatenate([s, s])
    if split_samples is None:
        z = np.array([[[normal(seed, int(g), k, d) for d in range(3)] for g in idx]
                      for k in range(2)]).reshape(-1, 3)
        offs = stds * z
    else:
        offs = np.asarray(split_samples, dtype=np.float64).reshape(-1, 3)
        assert offs.shape[0] == 2 * len(idx), (offs.shape, len(idx))
    rots = np.concatenate([build_rotation(st["rotation"][idx])] * 2)
    new = {"centre": np.einsum("nij,nj->ni", rots, offs) + np.concatenate([st["centre"][idx]] * 2),
           "log_scale": np.log(stds / 1.2)}
    for k in keys:
        if k not in new:
            new[k] = np.concatenate([st[k][idx]] * 2)
    append(new)
    prune(np.concatenate([sel, np.zeros(2 * len(idx), dtype=bool)]))
    # prune (the screen-radius statistics were reset by the appends above)
    op = 1.0 / (1.0 + np.exp(-st["opacity"]))
    mask = op < min_opacity
    if max_screen_size:
        mask |= scaling().max(axis=1) > 0.1 * extent
    if scene_min is not None and scene_max is not None:
        c = st["centre"]
        mask |= (c < np.asarray(scene_min)).any(axis=1) | (c > np.asarray(scene_max)).any(axis=1)
    prune(mask)
    return st, a1, a2
