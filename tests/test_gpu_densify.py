"""GPU tests of densification (gsparc_densify_*, FusedTrainer.densify_and_prune)
against the numpy restatement of gaussian.py:515-542 (oracle/densify.py),
with the same counter-based normal samples.

Bars: the new Gaussian count and the survivors' order exactly; parameters
within 1e-6 absolute (split centres 2e-5, from the FP32 Box-Muller samples);
Adam moments exactly (copied or zero)."""
import numpy as np
import pytest
import torch

from gsparc_b200 import scenes
from gsparc_b200.fused import FusedTrainer
from gsparc_b200.shared_mlp import SharedMLP
from oracle import densify as od

pytestmark = pytest.mark.gpu


def _trainer(P, shared):
    tr = FusedTrainer(scenes.make_scene(P, seed=1), shared=SharedMLP(2, 64, "relu") if shared else None)
    gen = torch.Generator().manual_seed(5)
    with torch.no_grad():
        tr.log_scale.copy_((torch.rand((P, 3), generator=gen) * 3 - 4.5).cuda())     # scales 0.011 .. 0.22
        tr.opacity_logit.copy_((torch.randn(P, generator=gen) * 3).cuda())
        tr.exp_avg.copy_(torch.randn(tr.exp_avg.numel(), generator=gen).cuda())
        tr.exp_avg_sq.copy_(torch.rand(tr.exp_avg_sq.numel(), generator=gen).cuda())
        tr.grad_accum.copy_((torch.rand(P, generator=gen) * 0.004).cuda())
        d = (torch.rand(P, generator=gen) * 4).floor()                                 # some never visible: 0/0
        tr.grad_denom.copy_(d.cuda())
    tr.activate()
    return tr


def _host_state(tr):
    P = tr.P
    st = dict(centre=tr.centre, log_scale=tr.log_scale, rotation=tr.rotation, opacity=tr.opacity_logit)
    out = {k: v.detach().cpu().numpy().astype(np.float64) for k, v in st.items()}
    moments = []
    from gsparc_b200.fused import state_layout
    (oC, oS, oQ, oO, oM, oG), _ = state_layout(P, tr.n_mlp, tr.n_conf)
    for buf in (tr.exp_avg, tr.exp_avg_sq):
        b = buf.detach().cpu().numpy().astype(np.float64)
        moments.append(dict(centre=b[oC:oC + 3 * P].reshape(P, 3), log_scale=b[oS:oS + 3 * P].reshape(P, 3),
                            rotation=b[oQ:oQ + 4 * P].reshape(P, 4), opacity=b[oO:oO + P]))
    if tr.shared is None:
        def per_g(flat):   # the four per-kind blocks of the flat MLP segment -> [P, 194]
            blocks, o = [], 0
            for w in (96, 32, 64, 2):
                blocks.append(flat[o:o + P * w].reshape(P, w))
                o += P * w
            return np.concatenate(blocks, axis=1)
        out["mlp"] = per_g(tr.mlp.detach().cpu().numpy().astype(np.float64))
        for mom, buf in zip(moments, (tr.exp_avg, tr.exp_avg_sq)):
            mom["mlp"] = per_g(buf.detach().cpu().numpy().astype(np.float64)[oM:oM + 194 * P])
    return out, moments[0], moments[1]


@pytest.mark.parametrize("shared", [True, False])
def test_densify_and_prune_matches_oracle(shared):
    tr = _trainer(3000, shared)
    st, m1, m2 = _host_state(tr)
    accum, denom = tr.grad_accum.cpu().numpy(), tr.grad_denom.cpu().numpy()
    conf_before = tr.conf_params.detach().clone()
    kw = dict(max_grad=0.0004, min_opacity=0.01, extent=5.0, max_screen_size=20,
              scene_min=[-5.5, -4.5, -0.5], scene_max=[5.5, 4.5, 3.5], seed=1234)
    ref_st, ref_m1, ref_m2 = od.densify_and_prune(st, m1, m2, accum, denom, **kw)
    P_new = tr.densify_and_prune(**kw)
    assert P_new == ref_st["centre"].shape[0] and P_new != 3000
    new_st, new_m1, new_m2 = _host_state(tr)
    for k in ref_st:
        tol = 2e-5 if k == "centre" else 1e-6
        np.testing.assert_allclose(new_st[k], ref_st[k], rtol=0, atol=tol, err_msg=k)
        np.testing.assert_array_equal(new_m1[k], ref_m1[k].astype(np.float32), err_msg=k)
        np.testing.assert_array_equal(new_m2[k], ref_m2[k].astype(np.float32), err_msg=k)
    assert torch.equal(tr.conf_params, conf_before)
    assert tr.grad_accum.shape == (P_new,) and float(tr.grad_accum.abs().sum()) == 0.0


def test_densified_trainer_steps_and_accumulates_statistics():
    tr = _trainer(3000, True)
    R = 2
    rxs = scenes.make_receivers(R)
    t = lambda a: torch.tensor(np.ascontiguousarray(a), dtype=torch.float32, device="cuda")
    views, rxs_d, tx = t(scenes.view_matrices(rxs)), t(rxs), t(scenes.TX_POS)
    targets = torch.rand((R, 90, 360), generator=torch.Generator().manual_seed(2)).cuda()
    tr.densify_and_prune(max_grad=0.0004, min_opacity=0.01, extent=5.0, seed=7)
    tr.densify_stats = True
    cap = tr.probe_capacity(views, rxs_d, tx)
    tr.capture(R, R * cap, tx, views, rxs_d, targets)
    losses = [float(tr.step(views, rxs_d, targets)) for _ in range(3)]
    tr.plan.check()
    assert all(np.isfinite(losses))
    assert float(tr.grad_denom.max()) >= 3 and float(tr.grad_accum.sum()) > 0   # three steps x visible receivers
    assert float(tr.max_radii2D.max()) > 0
    tr.reset_opacity()
    assert float(tr.act_opac.max()) <= 0.01 + 1e-6
