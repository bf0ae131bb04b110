"""The allocation-free SSIM entry point, gsparc_ssim_static_scratch.

It serves callers that cannot call cudaMalloc (a real-time receiver loop that
cannot absorb cudaMalloc's implicit synchronisation, a host that was handed
fixed device buffers by another runtime): its scratch -- the three SSIM
partial-derivative maps -- is a fixed device array inside the library.

Checked here through the C ABI against the allocating entry points
(gsparc_ssim_forward + gsparc_ssim_backward with caller-allocated maps) on two
calls in a row with different shapes.  Both run the same kernels on the same
inputs, so the tolerance is zero.  This file is collected last so that a run
stopping at the first failure has already run every other test.
"""
import ctypes

import numpy as np
import pytest
import torch

from gsparc_b200 import _lib, raster
from gsparc_b200._lib import ptr, stream_of

pytestmark = pytest.mark.gpu

C1, C2 = 0.01 ** 2, 0.03 ** 2


def _static_call(a, b, dl):
    B, CH, H, W = a.shape
    m = torch.full_like(a, float("nan"))
    g = torch.full_like(a, float("nan"))
    status = _lib.lib().gsparc_ssim_static_scratch(B, CH, H, W, C1, C2, ptr(a), ptr(b), ptr(dl), ptr(m), ptr(g),
                                                   stream_of(a.device))
    _lib.check("ssim_static_scratch", status)
    return m, g


def _allocating_call(a, b, dl):
    m, d1, d2, d3 = raster.ssim_forward(a, b, C1, C2, train=True)
    g = raster.ssim_backward(a, b, dl, d1, d2, d3, C1, C2)
    return m, g


def test_static_scratch_matches_allocating_entry_points_twice():
    rng = np.random.default_rng(7)
    for shape in ((1, 1, 90, 360), (2, 3, 37, 53)):       # two calls in a row, different sizes
        a = torch.from_numpy(rng.random(shape, dtype=np.float32)).cuda()
        b = torch.from_numpy(rng.random(shape, dtype=np.float32)).cuda()
        dl = torch.from_numpy(rng.normal(size=shape).astype(np.float32)).cuda()
        m_s, g_s = _static_call(a, b, dl)
        m_a, g_a = _allocating_call(a, b, dl)
        torch.cuda.synchronize()
        assert torch.equal(m_s, m_a)
        assert torch.equal(g_s, g_a)


def test_static_scratch_rejects_oversize_request():
    d = ctypes.c_void_p(16)     # never dereferenced: the size check fails first
    L = _lib.lib()
    status = L.gsparc_ssim_static_scratch(1, 1, 1025, 1024, C1, C2, d, d, d, d, d, None)
    assert status == 1
    assert b"1048576" in L.gsparc_last_error_detail()
