"""Drop-in for the reference's compiled ``fused_ssim_cuda`` module
(fused-ssim/ext.cpp:4-7, ssim.h:7-26), backed by libgsparc_b200.so."""
from __future__ import annotations

from gsparc_b200 import raster as _r


def fusedssim(C1, C2, img1, img2, train):
    """fusedssim (fused-ssim/ssim.cu:368-404): (map, dm_dmu1, dm_dsigma1_sq, dm_dsigma12)."""
    return _r.ssim_forward(img1, img2, C1, C2, bool(train))


def fusedssim_backward(C1, C2, img1, img2, dL_dmap, dm_dmu1, dm_dsigma1_sq, dm_dsigma12):
    """fusedssim_backward (fused-ssim/ssim.cu:406-444): dL/dimg1."""
    return _r.ssim_backward(img1, img2, dL_dmap, dm_dmu1, dm_dsigma1_sq, dm_dsigma12, C1, C2)
