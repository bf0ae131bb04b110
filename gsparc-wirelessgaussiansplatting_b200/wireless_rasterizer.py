"""Drop-in for the reference's compiled ``wireless_rasterizer`` module.

Same function names, positional arguments and return tuples as the pybind
module of cuda_kernel_rasterize/ext.cpp:8-10 (rasterize_points.h:8-53); the
work runs in the sm_100a kernels of libgsparc_b200.so through its C ABI.
"""
from __future__ import annotations

import torch

from gsparc_b200 import raster as _r


def rasterize_gaussians(means3D, emission_mlps, opacities, scales, rotations, image_height, image_width,
                        scale_modifier, viewmatrix, projmatrix, tx_pos, rx_pos):
    """RasterizeGaussiansCUDA (rasterize_points.cu:32-102).

    Returns (num_rendered, out_signal_real [1,H,W], out_signal_imag [1,H,W],
    radii int32 [P], geomBuffer, binningBuffer, imgBuffer).  ``projmatrix`` is
    accepted and unused, as in the reference."""
    if means3D.dim() != 2 or means3D.size(1) != 3:
        raise RuntimeError("means3D must have dimensions (num_points, 3)")
    P = means3D.size(0)
    H, W = int(image_height), int(image_width)
    dev = means3D.device
    if P == 0:
        z = torch.zeros((1, H, W), dtype=torch.float32, device=dev)
        e = torch.empty(0, dtype=torch.uint8, device=dev)
        return 0, z, z.clone(), torch.zeros(0, dtype=torch.int32, device=dev), e, e.clone(), e.clone()
    out_r, out_i, radii, st = _r.forward(means3D, emission_mlps, opacities, scales, rotations, H, W,
                                         scale_modifier, viewmatrix, tx_pos, rx_pos)
    return st.num_rendered, out_r, out_i, radii.reshape(P), st.geom, st.binning, st.image


def rasterize_gaussians_backward(means3D, emission_mlps, radii, out_signal_real, out_signal_imag, opacities,
                                 scales, rotations, scale_modifier, viewmatrix, projmatrix,
                                 dL_dout_signal_real, dL_dout_signal_imag, tx_pos, rx_pos, geomBuffer, R,
                                 binningBuffer, imageBuffer):
    """RasterizeGaussiansBackwardCUDA (rasterize_points.cu:106-199).

    Returns (dL_dmeans2D [P,3], dL_dmeans3D [P,3], dL_demission_mlps [M],
    dL_dopacity [P,1], dL_dcov3D [P,6], dL_dscales [P,3], dL_drotations [P,4])."""
    P = means3D.size(0)
    H, W = dL_dout_signal_real.size(1), dL_dout_signal_real.size(2)
    dev = means3D.device
    M = emission_mlps.numel()
    if P == 0:
        z = lambda *s: torch.zeros(s, dtype=torch.float32, device=dev)
        return z(0, 3), z(0, 3), z(M), z(0, 1), z(0, 6), z(0, 3), z(0, 4)
    st = _r.ForwardState(P, 1, H, W, _r.get_tile_shape(), int(R), int(R), geomBuffer, imageBuffer, binningBuffer)
    g = _r.backward(st, means3D, emission_mlps, scales, rotations, scale_modifier, viewmatrix, tx_pos, rx_pos,
                    dL_dout_signal_real, dL_dout_signal_imag)
    return (g["dmeans2D"].reshape(P, 3), g["dmeans3D"], g["dmlp"], g["dopacity"].reshape(P, 1),
            g["dcov3D"], g["dscales"], g["drotations"])


def mark_visible(means3D, viewmatrix, projmatrix):
    """markVisible (rasterize_points.cu:203-221): bool [P], range cull only."""
    return _r.mark_visible(means3D, viewmatrix)
