"""GPU tests of the batched evaluation metrics (gsparc_eval_metrics) against
the FP64 oracle restatement of train.py:672-701 (oracle/metrics.py).

Tolerances (FP32 sums over H x W pixels): PSNR and RSSI difference within
1e-4 dB; MAE, SSIM, confidence and loss within 2e-6 relative + 1e-6."""
import numpy as np
import pytest
import torch

from gsparc_b200.loss import METRICS, Evaluator, conf_floats
from oracle import metrics as om

pytestmark = pytest.mark.gpu


def _case(R, H, W, hidden, seed):
    gen = torch.Generator().manual_seed(seed)
    target = torch.rand((R, H, W), generator=gen)
    pred = (target + 0.1 * torch.randn((R, H, W), generator=gen)).clamp_min(0.0)
    rx = torch.rand((R, 3), generator=gen) * 4.0 - 2.0
    cp = 0.3 * torch.randn(conf_floats(hidden), generator=gen)
    return pred, target, rx, cp


# R < 16 runs the 32x8 tile blocks, R >= 16 the 128-column strips
@pytest.mark.parametrize("R,H,W,hidden", [(1, 90, 360, 32), (5, 37, 53, 16), (20, 90, 360, 32), (17, 8, 8, 48)])
def test_eval_metrics_match_oracle(R, H, W, hidden):
    dev = torch.device("cuda")
    pred, target, rx, cp = _case(R, H, W, hidden, R * 100 + H)
    ev = Evaluator(R, H, W, hidden, dev)
    m = ev(pred.to(dev), target.to(dev), rx.to(dev), cp.to(dev)).cpu().numpy().astype(np.float64)
    ref = om.evaluate(pred.numpy(), target.numpy(), rx.numpy(), cp.numpy(), hidden)
    assert METRICS == om.NAMES
    np.testing.assert_allclose(m[:, :2], ref[:, :2], rtol=0, atol=1e-4)
    np.testing.assert_allclose(m[:, 2:], ref[:, 2:], rtol=2e-6, atol=1e-6)


def test_eval_metrics_identical_spectra_and_repeat_calls():
    """mse = 0 gives an infinite PSNR (train.py:79-80), SSIM 1 and a zero RSSI
    difference; the arrival counters are left at zero, so calls repeat exactly."""
    dev = torch.device("cuda")
    pred, target, rx, cp = _case(3, 90, 360, 32, 7)
    t = target.to(dev)
    ev = Evaluator(3, 90, 360, 32, dev)
    m0 = ev(t, t, rx.to(dev), cp.to(dev)).clone()
    assert torch.isinf(m0[:, 0]).all() and (m0[:, 0] > 0).all()
    assert torch.allclose(m0[:, 3], torch.ones(3, device=dev), atol=1e-6)
    assert (m0[:, 1] == 0).all() and (m0[:, 2] == 0).all()
    a = ev(pred.to(dev), t, rx.to(dev), cp.to(dev)).clone()
    b = ev(pred.to(dev), t, rx.to(dev), cp.to(dev)).clone()
    assert torch.equal(a, b)


def test_trainer_evaluate_renders_and_scores_test_receivers():
    """FusedTrainer.evaluate (forward-only render + batched metrics) against
    the oracle metrics of the same render."""
    from gsparc_b200 import raster, scenes
    from gsparc_b200.autograd import RasterPlan
    from gsparc_b200.fused import FusedTrainer
    from gsparc_b200.shared_mlp import SharedMLP
    dev = torch.device("cuda")
    sc = scenes.make_scene(3000, seed=0)
    R = 6
    rxs = scenes.make_receivers(R)
    t = lambda a: torch.tensor(np.ascontiguousarray(a), dtype=torch.float32, device=dev)
    views, rxs_d, tx = t(scenes.view_matrices(rxs)), t(rxs), t(scenes.TX_POS)
    tr = FusedTrainer(sc, device=dev, shared=SharedMLP(2, 64, "relu"))
    cap = tr.probe_capacity(views, rxs_d, tx)
    plan = RasterPlan(tr.P, R, 90, 360, cap * R, dev)
    gen = torch.Generator().manual_seed(3)
    targets = torch.rand((R, 90, 360), generator=gen).to(dev)
    m = tr.evaluate(views, rxs_d, tx, targets, plan=plan).cpu().numpy().astype(np.float64)
    plan.check()
    with torch.no_grad():
        out, _, _, _ = raster.forward(tr.centre, None, tr.act_opac, tr.act_scales, tr.act_rots, 90, 360, 1.0, views,
                                      tx, rxs_d, **tr._shared_kw())
    ref = om.evaluate(out.cpu().numpy(), targets.cpu().numpy(), rxs, tr.conf_params.cpu().numpy(), tr.conf_hidden)
    np.testing.assert_allclose(m[:, :2], ref[:, :2], rtol=0, atol=1e-4)
    np.testing.assert_allclose(m[:, 2:], ref[:, 2:], rtol=2e-6, atol=1e-6)
