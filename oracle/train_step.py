"""CPU restatement of one GSpaRC training step (numpy, FP32).

TEST / CPU-BASELINE INFRASTRUCTURE ONLY: timed by bench.py's cpu_baseline and
``--impl reference`` legs as the CPU implementation of the path; never used by
the product.

Follows train.py:364-566: render (oracle.raster, the restatement of the
reference rasterizer), L1 + (1 - SSIM) with lambda 0.2 (oracle.ssim),
confidence weighting C*recon - 0.3*log C with C = 1 + exp(MLP(rx))
(gaussian.py:575-609), the reference backward (backward.cu) through
oracle.raster.render_backward, activation adjoints (exp, normalize, sigmoid)
and Adam (eps 1e-15) with the reference's per-group learning rates.
"""
from __future__ import annotations

import numpy as np

from . import raster, ssim
from . import shared_mlp as smlp

LR = dict(centre=0.00016, log_scale=0.005, rotation=0.001, opacity_logit=0.0055, mlp=0.002, conf=0.001)


class OracleTrainer:
    """``shared=(layers, width, act, params)`` selects the shared emission MLP
    (oracle/shared_mlp.py) instead of the scene's per-Gaussian MLPs."""

    def __init__(self, scene, H=90, W=360, seed=0, shared=None):
        self.H, self.W = H, W
        self.shared = shared
        mlp = scene.mlp.copy() if shared is None else np.asarray(shared[3], np.float32).copy()
        self.p = dict(centre=scene.means.copy(), log_scale=scene.log_scales.copy(), rotation=scene.quats.copy(),
                      opacity_logit=scene.opacity_logits.copy(), mlp=mlp)
        rng = np.random.default_rng(seed)
        lim1 = np.sqrt(6.0 / (3 + 32))
        lim2 = np.sqrt(6.0 / (32 + 1))
        self.conf = dict(w1=rng.uniform(-lim1, lim1, (32, 3)).astype(np.float32), b1=np.zeros(32, np.float32),
                         w2=rng.uniform(-lim2, lim2, (1, 32)).astype(np.float32), b2=np.zeros(1, np.float32))
        self.m = {k: np.zeros_like(v) for k, v in list(self.p.items()) + list(self.conf.items())}
        self.v = {k: np.zeros_like(v) for k, v in list(self.p.items()) + list(self.conf.items())}
        self.t = 0

    def step(self, view, rx, tx, target):
        f32 = np.float32
        p = self.p
        scales = np.exp(p["log_scale"]).astype(f32)
        qn = np.linalg.norm(p["rotation"], axis=1, keepdims=True)
        rots = (p["rotation"] / qn).astype(f32)
        opac = (1.0 / (1.0 + np.exp(-p["opacity_logit"]))).astype(f32)
        if self.shared is None:
            fwd = raster.render(p["centre"], scales, rots, opac, p["mlp"], view, tx, rx, self.H, self.W, dtype=f32)
        else:
            layers, width, act = self.shared[:3]
            cache = {}

            def signal_fn(radii):
                s, cache["c"] = smlp.forward(p["mlp"], layers, width, act, p["centre"], rx, radii)
                cache["radii"] = radii
                return np.stack([s * (radii > 0), np.zeros_like(s)], 1)

            fwd = raster.render(p["centre"], scales, rots, opac, None, view, tx, rx, self.H, self.W, dtype=f32,
                                signal_fn=signal_fn)
        pred = fwd["out"][0]
        N = pred.size
        l1 = np.abs(pred - target).mean()
        s_val = ssim.fused_ssim(pred, target, dtype=np.float32)
        recon = 0.8 * l1 + 0.2 * (1.0 - s_val)
        c = self.conf
        h_pre = c["w1"] @ rx + c["b1"]
        h = np.maximum(h_pre, 0)
        raw = float((c["w2"] @ h + c["b2"])[0])
        C = 1.0 + np.exp(raw)
        loss = C * recon - 0.3 * np.log(C)
        # adjoint of the loss
        dpred = C * (0.8 * np.sign(pred - target) / N - 0.2 * ssim.fused_ssim_grad(pred, target, dtype=np.float32))
        dC = recon - 0.3 / C
        draw = dC * np.exp(raw)
        gc = dict(w2=draw * h[None, :], b2=np.array([draw], f32))
        dh = draw * c["w2"][0] * (h_pre > 0)
        gc["w1"] = dh[:, None] * rx[None, :]
        gc["b1"] = dh
        dL = np.stack([dpred, np.zeros_like(dpred)]).astype(f32)
        g = raster.render_backward(fwd, p["centre"], scales, rots, opac, p["mlp"] if self.shared is None else None,
                                   view, tx, rx, dL, self.H, self.W, dtype=f32, ref_compat=True)
        if self.shared is not None:
            layers, width, act = self.shared[:3]
            dmlp, dm = smlp.backward(p["mlp"], layers, width, act, p["centre"], rx, cache["radii"], cache["c"],
                                     g["dL_dsignal"][:, 0])
            g["dL_dmlp"] = dmlp
            g["dL_dmeans3D"] = g["dL_dmeans3D"] + dm
        gp = dict(centre=np.nan_to_num(g["dL_dmeans3D"], nan=0.0), mlp=g["dL_dmlp"],
                  log_scale=g["dL_dscales"] * scales,
                  opacity_logit=g["dL_dopacity"] * opac * (1 - opac))
        dq = g["dL_drotations"]
        gp["rotation"] = (dq - rots * np.sum(dq * rots, axis=1, keepdims=True)) / qn
        self.t += 1
        b1, b2, eps = 0.9, 0.999, 1e-15
        for store, grads, lrs in ((p, gp, LR), (c, gc, None)):
            for k, gk in grads.items():
                key = k
                self.m[key] = b1 * self.m[key] + (1 - b1) * gk
                self.v[key] = b2 * self.v[key] + (1 - b2) * gk * gk
                mh = self.m[key] / (1 - b1 ** self.t)
                vh = self.v[key] / (1 - b2 ** self.t)
                lr = LR[k] if lrs is not None else LR["conf"]
                store[k] = (store[k] - lr * mh / (np.sqrt(vh) + eps)).astype(f32)
        return float(loss)
