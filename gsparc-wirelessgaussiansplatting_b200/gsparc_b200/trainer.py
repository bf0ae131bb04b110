"""One GSpaRC training step over the sm_100a path.

Mirrors the per-receiver training iteration of the reference
(train.py:364-566): activations (gaussian.py:33-38, :82-96), the flat
emission-MLP buffer (gaussian.py:565-572), the rasterizer call of
renderer.py:39-88, L1 + fused SSIM with lambda = 0.2, the DUSt3R-style
confidence weighting with alpha = 0.3 (train.py:417-439, ConfidenceMLP
gaussian.py:575-609), NaN-zeroing of the centre gradient (train.py:443-445),
Adam with eps = 1e-15 and the reference's per-group learning rates
(gaussian.py:176-197, optimizer.py:9-17) and the centre clamp after the step
(train.py:556-562).

Differences: the NaN handling and the clamp are done on the device without
host synchronisation, and with a process group the per-Gaussian gradients
are all-reduced (summed) over ranks -- receivers shard across GPUs, Gaussians
are replicated.  Densification/pruning, LR schedules and logging are out of
scope.
"""
from __future__ import annotations

import numpy as np
import torch
import torch.nn as nn
import torch.nn.functional as F

from . import scenes


class ConfidenceMLP(nn.Module):
    """rx_pos (3) -> confidence 1 + exp(raw) > 1 (gaussian.py:575-609)."""

    def __init__(self, hidden=32):
        super().__init__()
        self.fc1 = nn.Linear(3, hidden)
        self.relu = nn.ReLU()
        self.fc2 = nn.Linear(hidden, 1)
        nn.init.zeros_(self.fc2.bias)
        nn.init.xavier_uniform_(self.fc1.weight)
        nn.init.zeros_(self.fc1.bias)
        nn.init.xavier_uniform_(self.fc2.weight)

    def forward(self, rx_pos):
        if rx_pos.dim() == 1:
            rx_pos = rx_pos.unsqueeze(0)
        return 1.0 + torch.exp(self.fc2(self.relu(self.fc1(rx_pos))))


class SplatTrainer:
    """Gaussian parameters, optimizer and the per-receiver training step."""

    lambda1 = 0.2            # optimizer.py:8
    confidence_alpha = 0.3   # optimizer.py:33

    def __init__(self, scene: scenes.Scene, H=scenes.H, W=scenes.W, device="cuda", group=None, seed=0,
                 capturable=False):
        self.H, self.W, self.device, self.group = H, W, torch.device(device), group
        self.graph = None
        P = scene.P
        t = lambda a: torch.tensor(np.ascontiguousarray(a), dtype=torch.float32, device=self.device)
        self.centre = nn.Parameter(t(scene.means))
        self.log_scale = nn.Parameter(t(scene.log_scales))
        self.rotation = nn.Parameter(t(scene.quats))
        self.opacity_logit = nn.Parameter(t(scene.opacity_logits))
        o1, o2, o3 = P * 96, P * 96 + P * 32, P * 96 + P * 32 + P * 64
        self.fc1_w = nn.Parameter(t(scene.mlp[:o1]).reshape(P, 32, 3))
        self.fc1_b = nn.Parameter(t(scene.mlp[o1:o2]).reshape(P, 32))
        self.fc2_w = nn.Parameter(t(scene.mlp[o2:o3]).reshape(P, 2, 32))
        self.fc2_b = nn.Parameter(t(scene.mlp[o3:]).reshape(P, 2))
        torch.manual_seed(seed)
        self.confidence = ConfidenceMLP().to(self.device)
        groups = [
            {"params": [self.centre], "lr": 0.00016},
            {"params": [self.log_scale], "lr": 0.005},
            {"params": [self.rotation], "lr": 0.001},
            {"params": [self.opacity_logit], "lr": 0.0055},
            {"params": [self.fc1_w, self.fc1_b, self.fc2_w, self.fc2_b], "lr": 0.002},
            {"params": list(self.confidence.parameters()), "lr": 0.001},
        ]
        self.optimizer = torch.optim.Adam(groups, lr=0.0, eps=1e-15, fused=True, capturable=capturable)
        self.scene_lo = torch.tensor(scenes.ROOM_LO, dtype=torch.float32, device=self.device)
        self.scene_hi = torch.tensor(scenes.ROOM_HI, dtype=torch.float32, device=self.device)
        self.eye = torch.eye(4, device=self.device)

    def parameters(self):
        return [self.centre, self.log_scale, self.rotation, self.opacity_logit, self.fc1_w, self.fc1_b,
                self.fc2_w, self.fc2_b] + list(self.confidence.parameters())

    def emission_mlps(self):
        """EmissionMLPs.get_all_params (gaussian.py:565-572)."""
        return torch.cat([self.fc1_w.view(-1), self.fc1_b.view(-1), self.fc2_w.view(-1), self.fc2_b.view(-1)])

    def loss(self, view, rx, tx, target):
        """Forward of one step; returns (loss, rendered real spectrum)."""
        from cuda_kernel_rasterize.cuda_rasterizer import GaussianRasterizer, GaussianRasterizerSetting
        from fused_ssim import fused_ssim
        means2D = torch.zeros_like(self.centre, requires_grad=True)
        settings = GaussianRasterizerSetting(self.H, self.W, 1.0, view, self.eye, tx, rx)
        sig_r, sig_i, radii = GaussianRasterizer(settings)(
            self.centre, means2D, self.emission_mlps(), torch.sigmoid(self.opacity_logit),
            torch.exp(self.log_scale), F.normalize(self.rotation))
        pred = sig_r.squeeze(0)
        l1 = torch.abs(pred - target).mean()
        s = fused_ssim(pred[None, None], target[None, None])
        recon = (1.0 - self.lambda1) * l1 + self.lambda1 * (1.0 - s)
        conf = self.confidence(rx)
        loss = conf * recon - self.confidence_alpha * torch.log(conf)
        return loss.reshape(()), pred

    def step(self, view, rx, tx, target):
        """One optimisation step on device-resident inputs; returns the loss
        as a device scalar (no host synchronisation beyond the rasterizer's
        own instance-count readback)."""
        loss, _ = self.loss(view, rx, tx, target)
        loss.backward()
        with torch.no_grad():
            g = self.centre.grad
            torch.where(torch.isnan(g), torch.zeros_like(g), g, out=g)
            if self.group is not None:
                self._allreduce_grads()
        self.optimizer.step()
        self.optimizer.zero_grad(set_to_none=True)
        with torch.no_grad():
            self.centre.data.clamp_(min=self.scene_lo, max=self.scene_hi)
        return loss.detach()

    # ---- batched, CUDA-graph-capturable step -----------------------------------

    def loss_batched(self, views, rxs, tx, targets, plan):
        """Mean over R receivers of the per-receiver confidence-weighted loss,
        rendered in one launch through a static ``RasterPlan``."""
        from fused_ssim import FusedSSIMMap
        from .autograd import rasterize
        out_r, _, _ = rasterize(self.centre, self.emission_mlps(), torch.sigmoid(self.opacity_logit).reshape(-1),
                                torch.exp(self.log_scale), F.normalize(self.rotation), views, rxs, tx, plan)
        l1 = torch.abs(out_r - targets).mean(dim=(1, 2))
        smap = FusedSSIMMap.apply(0.01 ** 2, 0.03 ** 2, out_r.unsqueeze(1), targets.unsqueeze(1), "same", True)
        s = smap.mean(dim=(1, 2, 3))
        recon = (1.0 - self.lambda1) * l1 + self.lambda1 * (1.0 - s)
        conf = self.confidence(rxs).reshape(-1)
        return (conf * recon - self.confidence_alpha * torch.log(conf)).mean()

    def _batched_body(self):
        loss = self.loss_batched(self._s_views, self._s_rxs, self._s_tx, self._s_targets, self.plan)
        loss.backward()
        with torch.no_grad():
            g = self.centre.grad
            torch.where(torch.isnan(g), torch.zeros_like(g), g, out=g)
            if self.group is not None:
                self._allreduce_grads()
        self.optimizer.step()
        with torch.no_grad():
            self.centre.data.clamp_(min=self.scene_lo, max=self.scene_hi)
        return loss.detach()

    def probe_capacity(self, views, rxs, tx, margin=1.25, slack=4096):
        """Largest instance count over the given receivers, with a margin."""
        from . import raster
        kmax = 0
        with torch.no_grad():
            for r in range(views.shape[0]):
                _, _, _, st = raster.forward(self.centre, self.emission_mlps(),
                                             torch.sigmoid(self.opacity_logit).reshape(-1), torch.exp(self.log_scale),
                                             F.normalize(self.rotation), self.H, self.W, 1.0, views[r], tx, rxs[r])
                kmax = max(kmax, st.num_rendered)
        return int(kmax * margin) + slack

    def capture(self, R, capacity, tx, views=None, rxs=None, targets=None, warmup=3):
        """Build static buffers for R receivers per step and capture the whole
        step (render, loss, adjoint, NaN-zeroing, all-reduce, Adam, clamp) in a
        CUDA graph.  Requires ``capturable=True`` at construction.  The warm-up
        steps that precede capture (on a side stream, as graph capture needs)
        run on the given batch; parameters and optimizer state are restored in
        place afterwards, so the trainer starts from its constructed state."""
        from .autograd import RasterPlan
        dev = self.device
        self.plan = RasterPlan(self.centre.shape[0], R, self.H, self.W, capacity, dev)
        self._s_views = torch.eye(4, device=dev).repeat(R, 1, 1).contiguous()
        self._s_rxs = torch.zeros((R, 3), device=dev)
        self._s_tx = tx.detach().clone().reshape(3)
        self._s_targets = torch.zeros((R, self.H, self.W), device=dev)
        if views is not None:
            self._s_views.copy_(views.reshape(self._s_views.shape))
            self._s_rxs.copy_(rxs.reshape(self._s_rxs.shape))
            self._s_targets.copy_(targets.reshape(self._s_targets.shape))
        backup = [p.detach().clone() for p in self.parameters()]
        side = torch.cuda.Stream(dev)
        side.wait_stream(torch.cuda.current_stream(dev))
        with torch.cuda.stream(side):
            for _ in range(warmup):
                self.optimizer.zero_grad(set_to_none=True)
                self._batched_body()
        torch.cuda.current_stream(dev).wait_stream(side)
        self.optimizer.zero_grad(set_to_none=True)
        self.graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(self.graph):
            self._s_loss = self._batched_body()
        torch.cuda.synchronize(dev)
        with torch.no_grad():   # in place: the graph holds these addresses
            for p, b in zip(self.parameters(), backup):
                p.copy_(b)
            for st in self.optimizer.state.values():
                for v in st.values():
                    if torch.is_tensor(v):
                        v.zero_()
        torch.cuda.synchronize(dev)

    def step_graphed(self, views, rxs, targets):
        """Copy one batch of receivers into the static buffers and replay the
        captured step.  Returns the loss as a device scalar; the rasterizer's
        status (K, error word) is in ``self.plan.status_host`` once the stream
        has been synchronised (``self.plan.check()``)."""
        self._s_views.copy_(views.reshape(self._s_views.shape), non_blocking=True)
        self._s_rxs.copy_(rxs.reshape(self._s_rxs.shape), non_blocking=True)
        self._s_targets.copy_(targets.reshape(self._s_targets.shape), non_blocking=True)
        self.graph.replay()
        return self._s_loss

    def _allreduce_grads(self):
        """Sum every gradient over the process group in one flat bucket (the
        one exchange step of a receiver-sharded step)."""
        from .shard import allreduce_grads
        allreduce_grads(self.parameters(), self.group)
