"""Capture-safe autograd Function over the C ABI (R receivers per call).

The drop-in ``_RasterizeGaussians`` reads the instance count back to size its
binning arena exactly, as the reference does (rasterizer_impl.cu:274).  This
Function instead renders into a ``RasterPlan``: static arenas and a binning
capacity chosen up front, so a whole training step can be captured in a CUDA
graph and replayed.  An overflow of the capacity sets the capacity bit of the
device error word; ``RasterPlan.status_host`` receives that word through a
device-to-host copy recorded in the same stream (and graph), so the host can
check it after any synchronisation without an extra round trip.
"""
from __future__ import annotations

import torch

from . import _lib, raster


class RasterPlan:
    """Static buffers of a fixed-shape render: P Gaussians, R receivers,
    H x W spectra, tile shape, binning capacity, gradient mode and the
    azimuth seam wrap."""

    def __init__(self, P, R, H, W, capacity, device, tile=(16, 16), grad_mode="reference", wrap=False):
        self.P, self.R, self.H, self.W = int(P), int(R), int(H), int(W)
        self.tile = tuple(tile)
        self.wrap = bool(wrap)   # azimuth seam wrap (GSPARC_FLAG_WRAP_AZIMUTH)
        self.capacity = int(capacity)
        self.grad_mode = grad_mode
        dev = torch.device(device)
        self.geom = torch.empty(_lib.geom_state_bytes(self.P, self.R), dtype=torch.uint8, device=dev)
        self.image = torch.empty(_lib.image_state_bytes(self.R, self.H, self.W, *self.tile), dtype=torch.uint8,
                                 device=dev)
        self.binning = torch.empty(max(_lib.binning_state_bytes(self.capacity), 1), dtype=torch.uint8, device=dev)
        self.status_host = torch.zeros(4, dtype=torch.int32).pin_memory()   # K (lo, hi), error word, pad
        self.state = None

    def record_status(self):
        """Queue a copy of (K, error word) into pinned host memory."""
        self.status_host.copy_(self.image[:16].view(torch.int32), non_blocking=True)

    def host_status(self):
        """(K, error word) of the last recorded status; call after a sync."""
        s = self.status_host.tolist()
        return (s[0] & 0xffffffff) | (s[1] << 32), s[2] & 0xffffffff

    def check(self):
        K, err = self.host_status()
        if err & 1:
            raise _lib.GsparcError("rasterize", 3, "binning capacity exceeded",
                                   f"K={K} > capacity={self.capacity}; rebuild the plan with a larger capacity")
        if err:
            raise _lib.GsparcError("rasterize", 4, "device error word set", f"error=0x{err:x}")
        return K


class RasterizeFunction(torch.autograd.Function):
    """(means3D, emission_mlps, opacities[P], scales, rotations, views[R,4,4],
    rx[R,3], tx[3], plan) -> (out_real [R,H,W], out_imag [R,H,W], radii [R,P])."""

    @staticmethod
    def forward(ctx, means3D, mlp, opacities, scales, rotations, views, rxs, tx, plan):
        out_r, out_i, radii, st = raster.forward(
            means3D, mlp, opacities, scales, rotations, plan.H, plan.W, 1.0, views, tx, rxs, tile=plan.tile,
            capacity=plan.capacity, binning=plan.binning, geom=plan.geom, image=plan.image, wrap=plan.wrap)
        plan.record_status()
        ctx.plan, ctx.st = plan, st
        ctx.save_for_backward(means3D, mlp, scales, rotations, views, rxs, tx)
        ctx.mark_non_differentiable(radii)
        return out_r, out_i, radii

    @staticmethod
    def backward(ctx, g_real, g_imag, g_radii):
        means3D, mlp, scales, rotations, views, rxs, tx = ctx.saved_tensors
        if g_real is None:
            g_real = torch.zeros((ctx.plan.R, ctx.plan.H, ctx.plan.W), device=means3D.device)
        if g_imag is None:
            g_imag = torch.zeros((ctx.plan.R, ctx.plan.H, ctx.plan.W), device=means3D.device)
        g = raster.backward(ctx.st, means3D, mlp, scales, rotations, 1.0, views, tx, rxs, g_real.contiguous(),
                            g_imag.contiguous(), grad_mode=ctx.plan.grad_mode)
        return (g["dmeans3D"], g["dmlp"], g["dopacity"], g["dscales"], g["drotations"], None, None, None, None)


def rasterize(means3D, mlp, opacities, scales, rotations, views, rxs, tx, plan):
    return RasterizeFunction.apply(means3D, mlp, opacities, scales, rotations, views, rxs, tx, plan)
