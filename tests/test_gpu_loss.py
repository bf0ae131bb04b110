"""GPU tests of the fused training loss (gsparc_splat_loss) against the
reference's formulation in plain torch fp32 with autograd (train.py:420-436):
l1_loss, the window-convolution SSIM of utils.py (the non-fused fallback of
the same map), the confidence MLP of gaussian.py:575-609.

Tolerances (fp32 throughout): loss within 2e-6 relative; dL/dpred within
1e-5 of its largest magnitude; confidence-MLP gradients within 1e-5 of their
largest magnitude plus 1e-4 relative."""
import numpy as np
import pytest
import torch
import torch.nn.functional as F

from gsparc_b200.loss import SplatLoss, conf_floats
from gsparc_b200.trainer import ConfidenceMLP

pytestmark = pytest.mark.gpu


def _window(dev):
    g = torch.tensor([np.exp(-(x - 5) ** 2 / (2 * 1.5 ** 2)) for x in range(11)], dtype=torch.float32)
    g = g / g.sum()
    return (g[:, None] @ g[None, :]).to(dev)[None, None]


def _torch_ssim_mean(a, b, win):
    mu1, mu2 = F.conv2d(a, win, padding=5), F.conv2d(b, win, padding=5)
    s11 = F.conv2d(a * a, win, padding=5) - mu1 * mu1
    s22 = F.conv2d(b * b, win, padding=5) - mu2 * mu2
    s12 = F.conv2d(a * b, win, padding=5) - mu1 * mu2
    C1, C2 = 0.01 ** 2, 0.03 ** 2
    m = ((2 * mu1 * mu2 + C1) * (2 * s12 + C2)) / ((mu1 * mu1 + mu2 * mu2 + C1) * (s11 + s22 + C2))
    return m.mean(dim=(1, 2, 3))


def _reference(pred, target, rxs, mlp, lambda1=0.2, alpha=0.3):
    win = _window(pred.device)
    p = pred.detach().clone().requires_grad_(True)
    l1 = (p - target).abs().mean(dim=(1, 2))
    s = _torch_ssim_mean(p.unsqueeze(1), target.unsqueeze(1), win)
    recon = (1.0 - lambda1) * l1 + lambda1 * (1.0 - s)
    conf = mlp(rxs).reshape(-1)
    loss = (conf * recon - alpha * torch.log(conf)).mean()
    mlp.zero_grad(set_to_none=True)
    loss.backward()
    grads = torch.cat([q.grad.reshape(-1) for q in mlp.parameters()])
    return loss.detach(), p.grad.detach(), grads, torch.stack([l1, s, conf], 1).detach()


# R < 16: 32x8 tile blocks; R >= 16: 128-column strips over row bands (one
# band at R = 16 x 90x360 ... several at R = 40, single-strip images below)
@pytest.mark.parametrize("R,H,W,hidden", [(1, 90, 360, 32), (5, 90, 360, 32), (3, 37, 53, 16), (2, 8, 8, 48),
                                          (16, 90, 360, 32), (40, 90, 360, 32), (24, 37, 53, 16), (17, 8, 8, 48),
                                          (16, 45, 300, 8)])
def test_splat_loss_matches_torch_autograd(R, H, W, hidden):
    torch.backends.cudnn.allow_tf32 = False
    dev = torch.device("cuda")
    gen = torch.Generator().manual_seed(R * 1000 + H)
    target = torch.rand((R, H, W), generator=gen).to(dev)
    pred = (target + 0.2 * torch.randn((R, H, W), generator=gen).to(dev)).clamp_min(0.0).contiguous()
    pred[:, : H // 4, : W // 4] = target[:, : H // 4, : W // 4]      # |p - t| = 0: sign 0
    rxs = (torch.rand((R, 3), generator=gen) * 4.0 - 2.0).to(dev)
    torch.manual_seed(R + hidden)
    mlp = ConfidenceMLP(hidden).to(dev)
    with torch.no_grad():
        mlp.fc2.bias.fill_(0.3)
        mlp.fc1.bias.uniform_(-0.5, 0.5)
    flat = torch.cat([q.detach().reshape(-1) for q in mlp.parameters()]).contiguous()
    assert flat.numel() == conf_floats(hidden)
    ref_loss, ref_dpred, ref_dconf, ref_terms = _reference(pred, target, rxs, mlp)
    fn = SplatLoss(R, H, W, hidden, dev)
    dconf = torch.full_like(flat, float("nan"))
    loss, dpred = fn(pred, target, rxs, flat, dconf)
    torch.cuda.synchronize()
    assert abs(loss.item() - ref_loss.item()) <= 2e-6 * abs(ref_loss.item())
    torch.testing.assert_close(fn.terms[:, :3], ref_terms, rtol=2e-6, atol=2e-6)
    scale = ref_dpred.abs().max().item()
    assert (dpred - ref_dpred).abs().max().item() <= 1e-5 * scale
    gs = ref_dconf.abs().max().item()
    assert ((dconf - ref_dconf).abs() <= 1e-5 * gs + 1e-4 * ref_dconf.abs()).all()


@pytest.mark.parametrize("R", [4, 20])
def test_splat_loss_is_deterministic(R):
    dev = torch.device("cuda")
    H, W = 90, 360
    gen = torch.Generator().manual_seed(7)
    target = torch.rand((R, H, W), generator=gen).to(dev)
    pred = torch.rand((R, H, W), generator=gen).to(dev)
    rxs = torch.rand((R, 3), generator=gen).to(dev)
    flat = (0.1 * torch.randn(conf_floats(32), generator=gen)).to(dev)
    fn = SplatLoss(R, H, W, 32, dev)
    outs = []
    for _ in range(3):
        d = torch.empty_like(flat)
        loss, dpred = fn(pred, target, rxs, flat, d)
        outs.append((loss.clone(), dpred.clone(), d))
    for o in outs[1:]:
        for a, b in zip(outs[0], o):
            assert torch.equal(a, b)
