"""Python rasterizer API of the reference (cuda_kernel_rasterize/cuda_rasterizer/__init__.py),
re-implemented over the sm_100a C ABI.

Call surface kept: ``GaussianRasterizerSetting`` (NamedTuple, :93-100),
``GaussianRasterizer`` (nn.Module, :104-131), ``rasterize_gaussians`` (:12-15)
and the autograd Function ``_RasterizeGaussians`` (:17-90).  The backward
returns gradients for (means3D, means2D, emission_mlps, opacities, scales,
rotations, settings) in that order, as the reference does.
"""
from __future__ import annotations

from typing import NamedTuple

import torch
import torch.nn as nn

import wireless_rasterizer as wr


class GaussianRasterizerSetting(NamedTuple):
    image_height: int
    image_width: int
    scale_modifier: float
    viewmatrix: torch.Tensor
    projmatrix: torch.Tensor
    tx_pos: torch.Tensor
    rx_pos: torch.Tensor


def rasterize_gaussians(means3D, means2D, emission_mlps, opacities, scales, rotations, raster_settings):
    return _RasterizeGaussians.apply(means3D, means2D, emission_mlps, opacities, scales, rotations,
                                     raster_settings)


class _RasterizeGaussians(torch.autograd.Function):
    @staticmethod
    def forward(ctx, means3D, means2D, emission_mlps, opacities, scales, rotations, raster_settings):
        s = raster_settings
        (num_rendered, out_real, out_imag, radii, geom, binning, img) = wr.rasterize_gaussians(
            means3D, emission_mlps, opacities, scales, rotations, s.image_height, s.image_width,
            s.scale_modifier, s.viewmatrix, s.projmatrix, s.tx_pos, s.rx_pos)
        ctx.raster_settings = s
        ctx.num_rendered = num_rendered
        ctx.save_for_backward(emission_mlps, out_real, out_imag, means3D, scales, rotations, opacities, radii,
                              geom, binning, img)
        ctx.mark_non_differentiable(radii)
        return out_real, out_imag, radii

    @staticmethod
    def backward(ctx, grad_real, grad_imag, grad_radii):
        s = ctx.raster_settings
        (emission_mlps, out_real, out_imag, means3D, scales, rotations, opacities, radii, geom, binning,
         img) = ctx.saved_tensors
        if grad_real is None:
            grad_real = torch.zeros_like(out_real)
        if grad_imag is None:
            grad_imag = torch.zeros_like(out_imag)
        (g_means2D, g_means3D, g_mlp, g_opac, g_cov3D, g_scales, g_rot) = wr.rasterize_gaussians_backward(
            means3D, emission_mlps, radii, out_real, out_imag, opacities, scales, rotations, s.scale_modifier,
            s.viewmatrix, s.projmatrix, grad_real.contiguous(), grad_imag.contiguous(), s.tx_pos, s.rx_pos,
            geom, ctx.num_rendered, binning, img)
        return (g_means3D, g_means2D, g_mlp, g_opac.reshape(opacities.shape), g_scales, g_rot, None)


class GaussianRasterizer(nn.Module):
    def __init__(self, raster_settings):
        super().__init__()
        self.raster_settings = raster_settings

    def markVisible(self, positions):
        """Range-cull visibility mask.  (The reference calls a misspelled
        ``wr.mark_visisble`` here, cuda_rasterizer/__init__.py:115, which
        raises; this calls the extension's ``mark_visible``.)"""
        with torch.no_grad():
            s = self.raster_settings
            return wr.mark_visible(positions, s.viewmatrix, s.projmatrix)

    def forward(self, means3D, means2D, emission_mlps, opacities, scales=None, rotations=None):
        if scales is None or rotations is None:
            raise ValueError("scales and rotations are required (precomputed covariances are not supported "
                             "by the reference kernel either)")
        return rasterize_gaussians(means3D, means2D, emission_mlps, opacities, scales, rotations,
                                   self.raster_settings)
