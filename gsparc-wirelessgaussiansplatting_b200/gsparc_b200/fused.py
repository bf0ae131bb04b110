"""Training step with flat per-Gaussian state and the fused optimizer.

Same training iteration as ``trainer.SplatTrainer`` (train.py:364-566), with
the per-Gaussian parameters kept the way the kernels consume them:

  * one flat buffer per quantity -- raw parameters, gradients, both Adam
    moments -- in the layout of ``gsparc_gaussian_state_layout`` (centre,
    log-scale, quaternion, opacity logit, emission MLP).  The MLP segment *is*
    the flat ``emission_mlps`` buffer of EmissionMLPs.get_all_params
    (gaussian.py:565-572), so no concatenation or split happens per step;
  * the rasterizer backward writes its gradients straight into the flat
    gradient buffer;
  * ``gsparc_gaussian_adam_step`` applies the activation adjoints
    (exp, normalize, sigmoid), NaN-zeroing of the centre gradient, Adam and
    the centre clamp in one pass;
  * torch autograd only differentiates the loss with respect to the rendered
    spectra and the confidence MLP (gaussian.py:575-609), which keeps its own
    (torch) Adam.

The step is captured in a CUDA graph (``capture`` / ``step``) for R receivers
per step; with a process group the flat gradients (and the confidence MLP's)
are summed over ranks in one bucket before the update.
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch
import torch.nn.functional as F

from . import _lib, raster, scenes
from ._lib import check, ptr, stream_of
from .autograd import RasterPlan
from .trainer import ConfidenceMLP

LR = (0.00016, 0.005, 0.001, 0.0055, 0.002)   # centre, scaling, rotation, opacity, emission MLP (optimizer.py:9-17)
CONF_LR = 0.001


def state_layout(P):
    L = _lib.lib()
    out = (ctypes.c_size_t * 5)()
    check("gaussian state layout", L.gsparc_gaussian_state_layout(int(P), out))
    return [int(v) for v in out], int(L.gsparc_gaussian_state_floats(int(P)))


class FusedTrainer:
    lambda1 = 0.2
    confidence_alpha = 0.3

    def __init__(self, scene: scenes.Scene, H=scenes.H, W=scenes.W, device="cuda", group=None, seed=0,
                 grad_mode="reference", lr=LR, betas=(0.9, 0.999), eps=1e-15):
        self.H, self.W, self.device, self.group = H, W, torch.device(device), group
        self.grad_mode = grad_mode
        self.betas, self.eps = betas, eps
        P = scene.P
        self.P = P
        (oC, oS, oQ, oO, oM), total = state_layout(P)
        dev = self.device
        self.params = torch.zeros(total, dtype=torch.float32, device=dev)
        self.grads = torch.zeros(total, dtype=torch.float32, device=dev)
        self.exp_avg = torch.zeros(total, dtype=torch.float32, device=dev)
        self.exp_avg_sq = torch.zeros(total, dtype=torch.float32, device=dev)

        def seg(buf, off, n, shape):
            return buf[off:off + n].view(*shape)

        self.centre = seg(self.params, oC, 3 * P, (P, 3))
        self.log_scale = seg(self.params, oS, 3 * P, (P, 3))
        self.rotation = seg(self.params, oQ, 4 * P, (P, 4))
        self.opacity_logit = seg(self.params, oO, P, (P,))
        self.mlp = seg(self.params, oM, 194 * P, (194 * P,))
        t = lambda a: torch.tensor(np.ascontiguousarray(a), dtype=torch.float32, device=dev)
        with torch.no_grad():
            self.centre.copy_(t(scene.means))
            self.log_scale.copy_(t(scene.log_scales))
            self.rotation.copy_(t(scene.quats))
            self.opacity_logit.copy_(t(scene.opacity_logits).reshape(-1))
            self.mlp.copy_(t(scene.mlp))
        self.gout = dict(dmeans3D=seg(self.grads, oC, 3 * P, (P, 3)), dscales=seg(self.grads, oS, 3 * P, (P, 3)),
                         drotations=seg(self.grads, oQ, 4 * P, (P, 4)), dopacity=seg(self.grads, oO, P, (P,)),
                         dmlp=seg(self.grads, oM, 194 * P, (194 * P,)))
        self.step_count = torch.zeros(1, dtype=torch.float32, device=dev)
        self.lr5 = torch.tensor(lr, dtype=torch.float32, device=dev)
        self.lo3 = torch.tensor(scenes.ROOM_LO, dtype=torch.float32, device=dev)
        self.hi3 = torch.tensor(scenes.ROOM_HI, dtype=torch.float32, device=dev)
        torch.manual_seed(seed)
        self.confidence = ConfidenceMLP().to(dev)
        self.conf_opt = torch.optim.Adam(self.confidence.parameters(), lr=CONF_LR, eps=eps, fused=True,
                                         capturable=True)
        self.graph = None
        self.plan = None

    # ---- one step -------------------------------------------------------------

    def _activated(self):
        return (torch.exp(self.log_scale), F.normalize(self.rotation), torch.sigmoid(self.opacity_logit))

    def _loss(self, pred, rxs, targets):
        """Per-receiver confidence-weighted L1 + SSIM loss, averaged (train.py:417-439)."""
        from fused_ssim import FusedSSIMMap
        l1 = torch.abs(pred - targets).mean(dim=(1, 2))
        smap = FusedSSIMMap.apply(0.01 ** 2, 0.03 ** 2, pred.unsqueeze(1), targets.unsqueeze(1), "same", True)
        s = smap.mean(dim=(1, 2, 3))
        recon = (1.0 - self.lambda1) * l1 + self.lambda1 * (1.0 - s)
        conf = self.confidence(rxs).reshape(-1)
        return (conf * recon - self.confidence_alpha * torch.log(conf)).mean()

    def _body(self, views, rxs, tx, targets):
        plan = self.plan
        with torch.no_grad():
            scales, rots, opac = self._activated()
            out_r, out_i, radii, st = raster.forward(
                self.centre, self.mlp, opac, scales, rots, self.H, self.W, 1.0, views, tx, rxs, tile=plan.tile,
                capacity=plan.capacity, binning=plan.binning, geom=plan.geom, image=plan.image)
            plan.record_status()
        pred = out_r.detach().requires_grad_(True)
        loss = self._loss(pred, rxs, targets)
        loss.backward()
        with torch.no_grad():
            raster.backward(st, self.centre, self.mlp, scales, rots, 1.0, views, tx, rxs, pred.grad,
                            torch.zeros_like(out_i), grad_mode=self.grad_mode, out=self._bwd_out(plan.R))
            if self.group is not None:
                self._allreduce()
            b1, b2 = self.betas
            check("gaussian_adam_step", _lib.lib().gsparc_gaussian_adam_step(
                self.P, ptr(self.params), ptr(self.grads), ptr(self.exp_avg), ptr(self.exp_avg_sq),
                ptr(self.step_count), ptr(self.lr5), b1, b2, self.eps, ptr(self.lo3), ptr(self.hi3),
                stream_of(self.device)))
        self.conf_opt.step()
        return loss.detach()

    def _bwd_out(self, R):
        if getattr(self, "_bwd_R", None) != R:
            z = lambda *s: torch.empty(s, dtype=torch.float32, device=self.device)
            self._bwd_scratch = dict(dmeans2D=z(R, self.P, 3), dconic=z(R, self.P, 4), dsignal=z(R, self.P, 2),
                                     dcov3D=z(self.P, 6))
            self._bwd_R = R
        return dict(self._bwd_scratch, **self.gout)

    def _allreduce(self):
        import torch.distributed as dist
        cps = [p for p in self.confidence.parameters()]
        flat = torch.cat([self.grads] + [p.grad.reshape(-1) for p in cps])
        dist.all_reduce(flat, op=dist.ReduceOp.SUM, group=self.group)
        self.grads.copy_(flat[:self.grads.numel()])
        off = self.grads.numel()
        for p in cps:
            n = p.numel()
            p.grad.copy_(flat[off:off + n].view_as(p))
            off += n

    # ---- capacity, capture, replay -----------------------------------------------

    def probe_capacity(self, views, rxs, tx, margin=1.25, slack=4096):
        kmax = 0
        with torch.no_grad():
            scales, rots, opac = self._activated()
            for r in range(views.shape[0]):
                _, _, _, st = raster.forward(self.centre, self.mlp, opac, scales, rots, self.H, self.W, 1.0,
                                             views[r], tx, rxs[r])
                kmax = max(kmax, st.num_rendered)
        return int(kmax * margin) + slack

    def capture(self, R, capacity, tx, views=None, rxs=None, targets=None, warmup=3):
        """Capture the step for R receivers per step in a CUDA graph.  Warm-up
        steps (on a side stream, as capture requires) use the given batch;
        parameters and optimizer state are restored afterwards."""
        dev = self.device
        self.plan = RasterPlan(self.P, R, self.H, self.W, capacity, dev, grad_mode=self.grad_mode)
        self._s_views = torch.eye(4, device=dev).repeat(R, 1, 1).contiguous()
        self._s_rxs = torch.zeros((R, 3), device=dev)
        self._s_tx = tx.detach().clone().reshape(3)
        self._s_targets = torch.zeros((R, self.H, self.W), device=dev)
        if views is not None:
            self._s_views.copy_(views.reshape(self._s_views.shape))
            self._s_rxs.copy_(rxs.reshape(self._s_rxs.shape))
            self._s_targets.copy_(targets.reshape(self._s_targets.shape))
        saved = [t.clone() for t in (self.params, self.exp_avg, self.exp_avg_sq, self.step_count)]
        saved_conf = [p.detach().clone() for p in self.confidence.parameters()]
        side = torch.cuda.Stream(dev)
        side.wait_stream(torch.cuda.current_stream(dev))
        with torch.cuda.stream(side):
            for _ in range(warmup):
                self.conf_opt.zero_grad(set_to_none=True)
                self._body(self._s_views, self._s_rxs, self._s_tx, self._s_targets)
        torch.cuda.current_stream(dev).wait_stream(side)
        self.conf_opt.zero_grad(set_to_none=True)
        self.graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(self.graph):
            self._s_loss = self._body(self._s_views, self._s_rxs, self._s_tx, self._s_targets)
        torch.cuda.synchronize(dev)
        with torch.no_grad():
            for t, s in zip((self.params, self.exp_avg, self.exp_avg_sq, self.step_count), saved):
                t.copy_(s)
            for p, s in zip(self.confidence.parameters(), saved_conf):
                p.copy_(s)
            for st in self.conf_opt.state.values():
                for v in st.values():
                    if torch.is_tensor(v):
                        v.zero_()
        torch.cuda.synchronize(dev)

    def step(self, views, rxs, targets):
        """Copy a batch of R receivers (device or pinned host tensors) into the
        graph's inputs and replay the captured step; returns the loss (device)."""
        self._s_views.copy_(views.reshape(self._s_views.shape), non_blocking=True)
        self._s_rxs.copy_(rxs.reshape(self._s_rxs.shape), non_blocking=True)
        self._s_targets.copy_(targets.reshape(self._s_targets.shape), non_blocking=True)
        self.graph.replay()
        return self._s_loss

    def step_eager(self, views, rxs, tx, targets):
        """The same step without a graph (plan must exist)."""
        self.conf_opt.zero_grad(set_to_none=False)
        return self._body(views, rxs, tx, targets)

    # ---- views for comparison with the autograd trainer --------------------------

    def raw_parameters(self):
        P = self.P
        return dict(centre=self.centre, log_scale=self.log_scale, rotation=self.rotation,
                    opacity_logit=self.opacity_logit.view(P, 1), fc1_w=self.mlp[:96 * P].view(P, 32, 3),
                    fc1_b=self.mlp[96 * P:128 * P].view(P, 32), fc2_w=self.mlp[128 * P:192 * P].view(P, 2, 32),
                    fc2_b=self.mlp[192 * P:].view(P, 2))
