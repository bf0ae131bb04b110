"""GPU parity of fused SSIM against the oracle, the reference's golden
vectors (utils.ssim) and -- at the reference test's full size
[5,5,1080,1920] -- a conv2d SSIM, as fused-ssim/tests/test.py:59-91 does."""
import math
import os

import numpy as np
import pytest
import torch
import torch.nn.functional as F

from fused_ssim import fused_ssim
from fused_ssim_cuda import fusedssim, fusedssim_backward
from oracle import ssim as ossim
from tests.test_oracle import GOLDEN, _golden_cases

pytestmark = pytest.mark.gpu


def _conv_ssim(img1, img2):
    """conv2d SSIM in torch (the method of utils.py:94-114), FP32 on the GPU."""
    ch = img1.shape[1]
    g = torch.tensor([math.exp(-(x - 5) ** 2 / float(2 * 1.5 ** 2)) for x in range(11)])
    g = (g / g.sum()).unsqueeze(1)
    win = (g @ g.t()).float()[None, None].expand(ch, 1, 11, 11).contiguous().to(img1.device)
    c = lambda x: F.conv2d(x, win, padding=5, groups=ch)
    mu1, mu2 = c(img1), c(img2)
    s11 = c(img1 * img1) - mu1 * mu1
    s22 = c(img2 * img2) - mu2 * mu2
    s12 = c(img1 * img2) - mu1 * mu2
    C1, C2 = 0.01 ** 2, 0.03 ** 2
    m = ((2 * mu1 * mu2 + C1) * (2 * s12 + C2)) / ((mu1 * mu1 + mu2 * mu2 + C1) * (s11 + s22 + C2))
    return m.mean()


@pytest.mark.parametrize("case", ["uniform_90x360", "blobs_90x360", "uniform_b2c3_37x53"])
def test_fused_ssim_matches_reference_golden(case):
    mg = _golden_cases()
    g = np.load(os.path.join(GOLDEN, "ssim_golden.npz"))
    shape, kind, seed = [(s, k, sd) for (n, s, k, sd) in mg.CASES if n == case][0]
    a, b = mg.golden_inputs(shape, kind, seed)
    x = torch.from_numpy(a).cuda()
    y = torch.from_numpy(b).cuda()
    if x.dim() == 2:
        x, y = x[None, None], y[None, None]
    x.requires_grad_(True)
    v = fused_ssim(x, y)
    v.backward()
    assert torch.isclose(v.detach().cpu(), torch.tensor(float(g[case + "/value"])), rtol=1e-5, atol=1e-8)
    gg = g[case + "/grad"].reshape(x.shape)
    np.testing.assert_allclose(x.grad.cpu().numpy(), gg, rtol=1e-4, atol=1e-5 * np.abs(gg).max())


@pytest.mark.parametrize("shape", [(1, 1, 90, 360), (2, 3, 37, 53), (1, 2, 8, 8), (1, 1, 5, 700)])
def test_fusedssim_maps_match_oracle(shape):
    rng = np.random.default_rng(sum(shape))
    a = rng.random(shape, dtype=np.float32)
    b = rng.random(shape, dtype=np.float32)
    m, d1, d2, d3 = fusedssim(0.01 ** 2, 0.03 ** 2, torch.from_numpy(a).cuda(), torch.from_numpy(b).cuda(), True)
    om, o1, o2, o3 = ossim.ssim_forward(a, b)
    np.testing.assert_allclose(m.cpu().numpy(), om, atol=2e-6, rtol=1e-5)
    for gpu, ora in ((d1, o1), (d2, o2), (d3, o3)):
        np.testing.assert_allclose(gpu.cpu().numpy(), ora, rtol=1e-3, atol=1e-4 * np.abs(ora).max())
    dl = rng.normal(size=shape).astype(np.float32)
    g = fusedssim_backward(0.01 ** 2, 0.03 ** 2, torch.from_numpy(a).cuda(), torch.from_numpy(b).cuda(),
                           torch.from_numpy(dl).cuda(), d1, d2, d3)
    og = ossim.ssim_backward(a, b, dl, o1, o2, o3)
    np.testing.assert_allclose(g.cpu().numpy(), og, rtol=1e-3, atol=1e-4 * np.abs(og).max())


def test_valid_padding_and_inference_mode():
    rng = np.random.default_rng(3)
    a = rng.random((1, 1, 90, 360), dtype=np.float32)
    b = rng.random((1, 1, 90, 360), dtype=np.float32)
    x = torch.from_numpy(a).cuda().requires_grad_(True)
    v = fused_ssim(x, torch.from_numpy(b).cuda(), padding="valid")
    v.backward()
    # the valid-region mean of random images is ~4e-3: FP32 summation of ~3e4
    # map entries leaves ~2e-7 absolute error, hence the absolute floor
    assert abs(float(v) - ossim.fused_ssim(a, b, "valid")) <= 1e-4 * abs(ossim.fused_ssim(a, b, "valid")) + 1e-6
    og = ossim.fused_ssim_grad(a, b, "valid")
    np.testing.assert_allclose(x.grad.cpu().numpy(), og, rtol=1e-3, atol=1e-4 * np.abs(og).max())
    m, d1, d2, d3 = fusedssim(0.01 ** 2, 0.03 ** 2, torch.from_numpy(a).cuda(), torch.from_numpy(b).cuda(), False)
    assert d1.numel() == 0 and d2.numel() == 0 and d3.numel() == 0
    with torch.no_grad():
        v2 = fused_ssim(torch.from_numpy(a).cuda(), torch.from_numpy(b).cuda(), train=False)
    assert abs(float(v2) - ossim.fused_ssim(a, b)) <= 1e-5


def test_reference_test_full_size():
    """fused-ssim/tests/test.py:59-91 at its own size: value and gradient
    equal a conv2d SSIM under torch.isclose defaults."""
    torch.manual_seed(0)
    B, CH, H, W = 5, 5, 1080, 1920
    for _ in range(2):
        img1 = torch.rand([B, CH, H, W], device="cuda")
        img2 = torch.rand([B, CH, H, W], device="cuda")
        a = img1.clone().requires_grad_(True)
        b = img1.clone().requires_grad_(True)
        ref = _conv_ssim(a, img2)
        mine = fused_ssim(b, img2)
        assert torch.isclose(ref, mine)
        ref.backward()
        mine.backward()
        assert torch.isclose(a.grad, b.grad).all()
