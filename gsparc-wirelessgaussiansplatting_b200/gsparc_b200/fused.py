"""Training step with flat state, the fused loss and the fused optimizer.

Same training iteration as ``trainer.SplatTrainer`` (train.py:364-566), with
every parameter kept the way the kernels consume it:

  * one flat buffer per quantity -- raw parameters, gradients, both Adam
    moments -- in the layout of ``gsparc_gaussian_state_layout`` (centre,
    log-scale, quaternion, opacity logit, emission MLP, confidence MLP).  The
    MLP segment *is* the flat ``emission_mlps`` buffer of
    EmissionMLPs.get_all_params (gaussian.py:565-572), and the confidence
    MLP's nn.Parameters are views of the last segment, so nothing is
    concatenated or split per step;
  * the activated scales / rotations / opacities the rasterizer reads are
    written by the previous step's optimizer kernel (and by
    ``gsparc_gaussian_activate`` once at start);
  * ``gsparc_splat_loss`` computes L1 + SSIM + confidence loss and its
    gradients (spectra and confidence MLP) in three launches;
  * the rasterizer backward writes its gradients straight into the flat
    gradient buffer;
  * ``gsparc_gaussian_adam_step`` applies the activation adjoints
    (exp, normalize, sigmoid), NaN-zeroing of the centre gradient, Adam for
    all six parameter groups and the centre clamp.

No torch autograd and no torch optimizer run in the step.  It is captured in a
CUDA graph (``capture`` / ``step``) for R receivers per step; with a process
group the flat gradient buffer is summed over ranks in one all-reduce before
the update.
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib, raster, scenes, shard
from ._lib import check, ptr, stream_of
from .autograd import RasterPlan
from .loss import Evaluator, SplatLoss, conf_floats
from .trainer import ConfidenceMLP

# centre, scaling, rotation, opacity, emission MLP (optimizer.py:9-17), confidence MLP (optimizer.py:29)
LR = (0.00016, 0.005, 0.001, 0.0055, 0.002, 0.001)
CONF_HIDDEN = 32   # optimizer.py:35


def state_layout(P, n_mlp, n_conf=0):
    L = _lib.lib()
    out = (ctypes.c_size_t * 6)()
    check("gaussian state layout", L.gsparc_gaussian_state_layout(int(P), int(n_mlp), int(n_conf), out))
    return [int(v) for v in out], int(L.gsparc_gaussian_state_floats(int(P), int(n_mlp), int(n_conf)))


class FusedTrainer:
    lambda1 = 0.2
    confidence_alpha = 0.3

    def __init__(self, scene: scenes.Scene, H=scenes.H, W=scenes.W, device="cuda", group=None, seed=0,
                 grad_mode="reference", lr=LR, betas=(0.9, 0.999), eps=1e-15, conf_hidden=CONF_HIDDEN,
                 shared=None, wrap=False):
        """``shared``: a ``SharedMLP`` to use the benchmark's shared emission
        MLP (initialised from ``seed``) instead of the scene's per-Gaussian
        3-32-2 MLPs.  ``wrap``: continue footprints across the 0/2pi azimuth
        seam (the reference clamps them at the image edges)."""
        self.H, self.W, self.device, self.group = H, W, torch.device(device), group
        self.grad_mode = grad_mode
        self.wrap = bool(wrap)
        self.tile = (16, 16)
        self.betas, self.eps = betas, eps
        self.conf_hidden = int(conf_hidden)
        self.n_conf = conf_floats(self.conf_hidden)
        self.shared = shared
        dev = self.device
        P = scene.P
        n_mlp = 194 * P if shared is None else shared.n_params
        total = state_layout(P, n_mlp, self.n_conf)[1]
        z = lambda: torch.zeros(total, dtype=torch.float32, device=dev)
        torch.manual_seed(seed)
        self.confidence = ConfidenceMLP(self.conf_hidden).to(dev)
        conf0 = torch.cat([q.detach().reshape(-1) for q in self.confidence.parameters()])
        self.densify_stats = False
        self._bind(P, z(), z(), z())
        t = lambda a: torch.tensor(np.ascontiguousarray(a), dtype=torch.float32, device=dev)
        with torch.no_grad():
            self.centre.copy_(t(scene.means))
            self.log_scale.copy_(t(scene.log_scales))
            self.rotation.copy_(t(scene.quats))
            self.opacity_logit.copy_(t(scene.opacity_logits).reshape(-1))
            self.mlp.copy_(t(scene.mlp) if shared is None else shared.init_params(seed, dev))
            self.conf_params.copy_(conf0)
        self.step_count = torch.zeros(2, dtype=torch.float32, device=dev)   # step, arrival counter (0)
        self.lr6 = torch.tensor(lr, dtype=torch.float32, device=dev)
        self.lo3 = torch.tensor(scenes.ROOM_LO, dtype=torch.float32, device=dev)
        self.hi3 = torch.tensor(scenes.ROOM_HI, dtype=torch.float32, device=dev)
        # amplitude channels per spectrum: the shared MLP's outputs (one = the signal path)
        self.channels = 1 if shared is None else int(shared.out)
        self.graph = None
        self.plan = None
        self._R = None
        self.activate()

    def _bind(self, P, params, exp_avg, exp_avg_sq):
        """Views of a flat training state for P Gaussians (raw parameters and
        Adam moments), a zeroed gradient buffer, the activation outputs and
        the densification statistics; step-size buffers are rebuilt on the
        next step and any captured graph is dropped."""
        dev = self.device
        self.P = P
        self.n_mlp = 194 * P if self.shared is None else self.shared.n_params
        (oC, oS, oQ, oO, oM, oG), total = state_layout(P, self.n_mlp, self.n_conf)
        assert params.numel() == total and exp_avg.numel() == total and exp_avg_sq.numel() == total
        self.params, self.exp_avg, self.exp_avg_sq = params, exp_avg, exp_avg_sq
        self.grads = torch.zeros(total, dtype=torch.float32, device=dev)

        def seg(buf, off, n, shape):
            return buf[off:off + n].view(*shape)

        self.centre = seg(self.params, oC, 3 * P, (P, 3))
        self.log_scale = seg(self.params, oS, 3 * P, (P, 3))
        self.rotation = seg(self.params, oQ, 4 * P, (P, 4))
        self.opacity_logit = seg(self.params, oO, P, (P,))
        self.mlp = seg(self.params, oM, self.n_mlp, (self.n_mlp,))
        self.conf_params = seg(self.params, oG, self.n_conf, (self.n_conf,))
        self.conf_grads = seg(self.grads, oG, self.n_conf, (self.n_conf,))
        off = 0
        with torch.no_grad():   # the confidence module's parameters are views of the flat segment
            for prm in self.confidence.parameters():
                n = prm.numel()
                prm.data = self.conf_params[off:off + n].view_as(prm)
                off += n
        self.gout = dict(dmeans3D=seg(self.grads, oC, 3 * P, (P, 3)), dscales=seg(self.grads, oS, 3 * P, (P, 3)),
                         drotations=seg(self.grads, oQ, 4 * P, (P, 4)), dopacity=seg(self.grads, oO, P, (P,)),
                         dmlp=seg(self.grads, oM, self.n_mlp, (self.n_mlp,)))
        self.act_scales = torch.empty((P, 3), dtype=torch.float32, device=dev)
        self.act_rots = torch.empty((P, 4), dtype=torch.float32, device=dev)
        self.act_opac = torch.empty((P,), dtype=torch.float32, device=dev)
        # densification statistics (train.py:508-516), accumulated by the step when densify_stats is set
        self.grad_accum = torch.zeros(P, dtype=torch.float32, device=dev)
        self.grad_denom = torch.zeros(P, dtype=torch.float32, device=dev)
        self.max_radii2D = torch.zeros(P, dtype=torch.float32, device=dev)
        self.graph = None
        self.plan = None
        self._R = None

    def densify_and_prune(self, max_grad, min_opacity, extent, max_screen_size=None, scene_min=None, scene_max=None,
                          percent_dense=0.01, seed=0):
        """densify_and_prune (gaussian.py:515-542) with the statistics the step
        accumulated (``densify_stats = True``; train.py:508-516): clone, split
        into two and prune on the device, in the reference's order.  The flat
        state is rebuilt for the new Gaussian count (one host read of it),
        new Gaussians start with zero Adam moments, the statistics restart at
        zero, and the step has to be captured again.  Returns the new count."""
        lib, dev, P = _lib.lib(), self.device, self.P
        per_g = int(self.shared is None)
        if self.group is not None:
            # receivers are sharded: every rank densifies the same way from the summed statistics
            shard.reduce_densify_stats(self.grad_accum, self.grad_denom, self.max_radii2D, self.group)
        inf = float("inf")
        lo = list(scene_min) if scene_min is not None else [-inf] * 3
        hi = list(scene_max) if scene_max is not None else [inf] * 3
        box = torch.tensor([float(v) for v in lo + hi], dtype=torch.float32)   # host memory
        work = torch.empty(max(int(lib.gsparc_densify_work_ints(P)), 1), dtype=torch.int32, device=dev)
        pn = torch.zeros(1, dtype=torch.int32, device=dev)
        msz = float(max_screen_size) if max_screen_size else 0.0
        args = (float(max_grad), float(percent_dense), float(extent), float(min_opacity), msz, ptr(box), int(seed))
        check("densify_count", lib.gsparc_densify_count(
            P, self.n_mlp, per_g, self.n_conf, ptr(self.params), ptr(self.grad_accum), ptr(self.grad_denom), *args,
            ptr(work), ptr(pn), stream_of(dev)))
        P_new = int(pn.item())
        total = state_layout(P_new, 194 * P_new if per_g else self.n_mlp, self.n_conf)[1]
        new = [torch.empty(total, dtype=torch.float32, device=dev) for _ in range(3)]
        check("densify_apply", lib.gsparc_densify_apply(
            P, P_new, self.n_mlp, per_g, self.n_conf, ptr(self.params), ptr(self.exp_avg), ptr(self.exp_avg_sq), *args,
            ptr(work), ptr(new[0]), ptr(new[1]), ptr(new[2]), stream_of(dev)))
        self._bind(P_new, *new)
        self.activate()
        return P_new

    def reset_opacity(self):
        """reset_opacity (gaussian.py:223-230): opacities capped at 0.01, their
        Adam moments zeroed (in place: a captured step stays valid)."""
        check("reset_opacity", _lib.lib().gsparc_reset_opacity(
            self.P, self.n_mlp, self.n_conf, ptr(self.params), ptr(self.exp_avg), ptr(self.exp_avg_sq),
            stream_of(self.device)))
        self.activate()

    def activate(self):
        """Recompute the activated rasterizer inputs from the raw parameters
        (needed only after the raw parameters were changed from outside)."""
        check("gaussian_activate", _lib.lib().gsparc_gaussian_activate(
            self.P, ptr(self.params), ptr(self.act_scales), ptr(self.act_rots), ptr(self.act_opac),
            stream_of(self.device)))

    # ---- one step -------------------------------------------------------------

    def _buffers(self, R):
        if self._R == R:
            return
        dev, P = self.device, self.P
        z = lambda *s: torch.empty(s, dtype=torch.float32, device=dev)
        self._out_r, self._out_i = z(R, self.H, self.W), z(R, self.H, self.W)
        self._radii = torch.empty((R, P), dtype=torch.int32, device=dev)
        self._zero_imag = torch.zeros((R, self.H, self.W), dtype=torch.float32, device=dev)
        self._scratch = dict(dmeans2D=z(R, P, 3), dconic=z(R, P, 4), dsignal=z(R, P, 2), dcov3D=z(P, 6))
        C = self.channels
        if C > 1:   # R x C spectra; the loss sees R*C spectra, each with its receiver's position
            self._out_mc = z(R, C, self.H, self.W)
            self._scratch = dict(dmeans2D=z(R, P, 3), dconic=z(R, P, 4), dfeatures=z(R, P, C), dcov3D=z(P, 6))
            self._rep_idx = torch.arange(R, device=dev).repeat_interleave(C)
            self._rx_rep = z(R * C, 3)
        self._lossfn = SplatLoss(R * C, self.H, self.W, self.conf_hidden, dev, self.lambda1, self.confidence_alpha)
        self._R = R

    def _body_channels(self, views, rxs, tx, targets):
        plan = self.plan
        R, C, H, W = plan.R, self.channels, self.H, self.W
        out, _, st = raster.forward_channels(
            self.centre, self.act_opac, self.act_scales, self.act_rots, H, W, 1.0, views, tx, rxs, self.shared,
            self.mlp, tile=plan.tile, capacity=plan.capacity, binning=plan.binning, out=self._out_mc,
            radii=self._radii, geom=plan.geom, image=plan.image, wrap=plan.wrap)
        plan.record_status()
        torch.index_select(rxs, 0, self._rep_idx, out=self._rx_rep)
        loss, dpred = self._lossfn(out.view(R * C, H, W), targets.reshape(R * C, H, W), self._rx_rep,
                                   self.conf_params, self.conf_grads)
        bo = dict(self._scratch, dmeans3D=self.gout["dmeans3D"], dscales=self.gout["dscales"],
                  drotations=self.gout["drotations"], dopacity=self.gout["dopacity"], dshared=self.gout["dmlp"])
        raster.backward_channels(st, self.centre, self.act_scales, self.act_rots, 1.0, views, tx, rxs,
                                 dpred.view(R, C, H, W), self.shared, self.mlp, out=bo)
        if self.densify_stats:
            self._accumulate_stats(R)
        return loss

    def _body(self, views, rxs, tx, targets):
        plan = self.plan
        self._buffers(plan.R)
        if self.channels > 1:
            loss = self._body_channels(views, rxs, tx, targets)
            self._reduce_and_adam()
            return loss
        out_r, _, _, st = raster.forward(
            self.centre, self._mlp_arg(), self.act_opac, self.act_scales, self.act_rots, self.H, self.W, 1.0, views, tx,
            rxs, tile=plan.tile, capacity=plan.capacity, binning=plan.binning, geom=plan.geom, image=plan.image,
            wrap=plan.wrap,
            out_real=self._out_r, out_imag=self._out_i, radii=self._radii, **self._shared_kw())
        plan.record_status()
        loss, dpred = self._lossfn(out_r, targets, rxs, self.conf_params, self.conf_grads)
        raster.backward(st, self.centre, self._mlp_arg(), self.act_scales, self.act_rots, 1.0, views, tx, rxs,
                        dpred, self._zero_imag, grad_mode=self.grad_mode, out=self._bwd_out(),
                        **self._shared_kw())
        if self.densify_stats:
            self._accumulate_stats(plan.R)
        self._reduce_and_adam()
        return loss

    def _accumulate_stats(self, R):
        check("densify_stats", _lib.lib().gsparc_densify_stats(
            self.P, R, ptr(self._radii), ptr(self._scratch["dmeans2D"]), ptr(self.grad_accum), ptr(self.grad_denom),
            ptr(self.max_radii2D), stream_of(self.device)))

    def evaluate(self, views, rxs, tx, targets, plan=None):
        """Render R test receivers with the current parameters (forward only)
        and evaluate them as train.py:672-701 does: returns a [R, 6] tensor
        (R*C rows with C channels, receiver-major) of PSNR, RSSI difference,
        MAE, SSIM, confidence and evaluation loss (loss.METRICS).  `plan` is a
        RasterPlan for R receivers (default: the training step's)."""
        plan = self.plan if plan is None else plan
        R, C, H, W, dev = plan.R, self.channels, self.H, self.W, self.device
        with torch.no_grad():
            if C > 1:
                out, _, _ = raster.forward_channels(
                    self.centre, self.act_opac, self.act_scales, self.act_rots, H, W, 1.0, views, tx, rxs,
                    self.shared, self.mlp, tile=plan.tile, capacity=plan.capacity, binning=plan.binning,
                    geom=plan.geom, image=plan.image, wrap=plan.wrap)
                out = out.view(R * C, H, W)
                rxs = rxs.repeat_interleave(C, dim=0).contiguous()
            else:
                out, _, _, _ = raster.forward(
                    self.centre, self._mlp_arg(), self.act_opac, self.act_scales, self.act_rots, H, W, 1.0, views,
                    tx, rxs, tile=plan.tile, capacity=plan.capacity, binning=plan.binning, geom=plan.geom,
                    image=plan.image, wrap=plan.wrap, **self._shared_kw())
            plan.record_status()
            ev = getattr(self, "_evaluator", None)
            if ev is None or ev.R != R * C:
                ev = self._evaluator = Evaluator(R * C, H, W, self.conf_hidden, dev, self.lambda1)
            return ev(out, targets.reshape(R * C, H, W), rxs, self.conf_params)

    def _reduce_and_adam(self):
        if self.group is not None:
            shard.allreduce_flat(self.grads, self.group)
        b1, b2 = self.betas
        check("gaussian_adam_step", _lib.lib().gsparc_gaussian_adam_step(
            self.P, self.n_mlp, self.n_conf, ptr(self.params), ptr(self.grads), ptr(self.exp_avg), ptr(self.exp_avg_sq),
            ptr(self.step_count), ptr(self.lr6), b1, b2, self.eps, ptr(self.lo3), ptr(self.hi3),
            ptr(self.act_scales), ptr(self.act_rots), ptr(self.act_opac), stream_of(self.device)))

    def _mlp_arg(self):
        return self.mlp if self.shared is None else None

    def _shared_kw(self):
        return {} if self.shared is None else dict(shared=self.shared, shared_params=self.mlp)

    def _bwd_out(self):
        out = dict(self._scratch, **self.gout)
        if self.shared is not None:
            out["dshared"] = out.pop("dmlp")
        return out

    def terms(self):
        """Per-receiver (l1, ssim, conf, loss_r) of the last step, [R,4] on the device."""
        return self._lossfn.terms

    # ---- capacity, capture, replay -----------------------------------------------

    def probe_capacity(self, views, rxs, tx, margin=1.25, slack=4096, tile=(16, 16)):
        """Binning capacity per receiver: the largest instance count over the
        given receivers (current parameters, tile shape `tile`) with margin."""
        kmax = 0
        with torch.no_grad():
            for r in range(views.shape[0]):
                if self.channels > 1:
                    _, _, st = raster.forward_channels(self.centre, self.act_opac, self.act_scales, self.act_rots,
                                                       self.H, self.W, 1.0, views[r], tx, rxs[r], self.shared,
                                                       self.mlp, tile=tile, wrap=self.wrap)
                    kmax = max(kmax, st.num_rendered)
                    continue
                _, _, _, st = raster.forward(self.centre, self._mlp_arg(), self.act_opac, self.act_scales,
                                             self.act_rots, self.H, self.W, 1.0, views[r], tx, rxs[r], tile=tile,
                                             wrap=self.wrap, **self._shared_kw())
                kmax = max(kmax, st.num_rendered)
        return int(kmax * margin) + slack

    def _state(self):
        return (self.params, self.exp_avg, self.exp_avg_sq, self.step_count)

    def capture(self, R, capacity, tx, views=None, rxs=None, targets=None, warmup=3, tile=(16, 16)):
        """Capture the step for R receivers per step in a CUDA graph (binning
        capacity `capacity` instances in total, tile shape `tile`).  Warm-up
        steps (on a side stream, as capture requires) use the given batch;
        parameters and optimizer state are restored afterwards."""
        dev = self.device
        self.graph = None
        self.tile = tuple(tile)
        self.plan = RasterPlan(self.P, R, self.H, self.W, capacity, dev, tile=tile, grad_mode=self.grad_mode,
                               wrap=self.wrap)
        self._buffers(R)
        self._s_views = torch.eye(4, device=dev).repeat(R, 1, 1).contiguous()
        self._s_rxs = torch.zeros((R, 3), device=dev)
        self._s_tx = tx.detach().clone().reshape(3)
        self._s_targets = torch.zeros((R, self.H, self.W) if self.channels == 1 else
                                      (R, self.channels, self.H, self.W), device=dev)
        if views is not None:
            self._s_views.copy_(views.reshape(self._s_views.shape))
            self._s_rxs.copy_(rxs.reshape(self._s_rxs.shape))
            self._s_targets.copy_(targets.reshape(self._s_targets.shape))
        state = self._state()
        saved = [t.clone() for t in state]
        side = torch.cuda.Stream(dev)
        side.wait_stream(torch.cuda.current_stream(dev))
        with torch.cuda.stream(side):
            for _ in range(warmup):
                self._body(self._s_views, self._s_rxs, self._s_tx, self._s_targets)
        torch.cuda.current_stream(dev).wait_stream(side)
        self.graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(self.graph):
            self._s_loss = self._body(self._s_views, self._s_rxs, self._s_tx, self._s_targets)
        torch.cuda.synchronize(dev)
        with torch.no_grad():   # in place: the graph holds these addresses
            for t, s in zip(state, saved):
                t.copy_(s)
        self.activate()
        torch.cuda.synchronize(dev)

    def autotune_tile(self, tx, views, rxs, targets, shapes=((16, 16), (8, 32), (32, 8)), steps=5, margin=1.25):
        """Pick the tile shape of the R-receiver step (R = len(views)) by
        measurement: for each shape, probe the binning capacity, capture the
        step and time `steps` graph replays with CUDA events; parameters and
        optimizer state are restored after every trial.  Leaves the fastest
        shape captured and returns {shape: ms per step}."""
        R = views.shape[0]
        dev = self.device
        state = self._state()
        saved = [t.clone() for t in state]
        stream = torch.cuda.current_stream(dev)
        times, caps = {}, {}
        for tile in shapes:
            caps[tile] = self.probe_capacity(views, rxs, tx, margin=margin, tile=tile) * R
            self.capture(R, caps[tile], tx, views, rxs, targets, tile=tile)
            self.step(views, rxs, targets)
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            for _ in range(steps):
                self.step(views, rxs, targets)
            b.record(stream)
            torch.cuda.synchronize(dev)
            self.plan.check()
            times[tile] = a.elapsed_time(b) / steps
            with torch.no_grad():
                for t, s in zip(state, saved):
                    t.copy_(s)
            self.activate()
        best = min(times, key=times.get)
        self.capture(R, caps[best], tx, views, rxs, targets, tile=best)
        return times

    def step(self, views, rxs, targets):
        """Copy a batch of R receivers (device or pinned host tensors) into the
        graph's inputs and replay the captured step; returns the loss (a
        device tensor that the next step overwrites).

        Host inputs are copied on a side stream into one of two staging
        buffers, so the host-to-device transfer of this step overlaps the
        previous step's kernels; a device-to-device copy then moves them into
        the graph's inputs just before the replay.  As with any non-blocking
        copy, the host tensors must stay unchanged until the step has run on
        the device (for example, until its loss has been read)."""
        if views.is_cuda or rxs.is_cuda or targets.is_cuda:
            self._s_views.copy_(views.reshape(self._s_views.shape), non_blocking=True)
            self._s_rxs.copy_(rxs.reshape(self._s_rxs.shape), non_blocking=True)
            self._s_targets.copy_(targets.reshape(self._s_targets.shape), non_blocking=True)
        else:
            self._stage_host_inputs(views, rxs, targets)
        self.graph.replay()
        return self._s_loss

    def _stage_host_inputs(self, views, rxs, targets):
        """Host inputs -> staging buffer (side stream) -> the graph's inputs
        (current stream, after the transfer and the previous step)."""
        if getattr(self, "_stage", None) is None:
            inputs = (self._s_views, self._s_rxs, self._s_targets)
            self._stage = [tuple(torch.empty_like(x) for x in inputs) for _ in range(2)]
            self._stage_ready = [torch.cuda.Event(), torch.cuda.Event()]
            self._stage_free = [torch.cuda.Event(), torch.cuda.Event()]
            self._stage_used = [False, False]
            self._stage_i = 0
            self._copy_stream = torch.cuda.Stream(device=self._s_views.device)
            for b in self._stage:
                for x in b:
                    x.record_stream(self._copy_stream)
        k = self._stage_i
        self._stage_i ^= 1
        buf = self._stage[k]
        cur = torch.cuda.current_stream(self._s_views.device)
        cs = self._copy_stream
        if self._stage_used[k]:
            cs.wait_event(self._stage_free[k])   # the device copy of two steps ago has read it
        with torch.cuda.stream(cs):
            for dst, src in zip(buf, (views, rxs, targets)):
                dst.copy_(src.reshape(dst.shape), non_blocking=True)
            self._stage_ready[k].record(cs)
        cur.wait_event(self._stage_ready[k])
        for dst, src in zip((self._s_views, self._s_rxs, self._s_targets), buf):
            dst.copy_(src, non_blocking=True)
        self._stage_free[k].record(cur)
        self._stage_used[k] = True

    def step_eager(self, views, rxs, tx, targets):
        """The same step without a graph (plan must exist)."""
        return self._body(views.contiguous(), rxs.contiguous(), tx, targets.contiguous())

    # ---- views for comparison with the autograd trainer --------------------------

    def raw_parameters(self):
        P = self.P
        if self.shared is not None:
            return dict(centre=self.centre, log_scale=self.log_scale, rotation=self.rotation,
                        opacity_logit=self.opacity_logit.view(P, 1), shared_mlp=self.mlp)
        return dict(centre=self.centre, log_scale=self.log_scale, rotation=self.rotation,
                    opacity_logit=self.opacity_logit.view(P, 1), fc1_w=self.mlp[:96 * P].view(P, 32, 3),
                    fc1_b=self.mlp[96 * P:128 * P].view(P, 32), fc2_w=self.mlp[128 * P:192 * P].view(P, 2, 32),
                    fc2_b=self.mlp[192 * P:].view(P, 2))
