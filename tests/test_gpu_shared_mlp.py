"""GPU tests of the shared emission MLP (the benchmark configurations' model)
against a plain PyTorch fp32 reference of the same network with autograd:
features (centre, 4-frequency positional encoding, receiver-relative
direction, 1/d^2), hidden layers, sigmoid of the output.

Tolerances (fp32): signals within 2e-6 absolute (they lie in (0, 1));
parameter and centre gradients within 1e-4 of each tensor's largest
magnitude."""
import math

import numpy as np
import pytest
import torch
import torch.nn.functional as F

from gsparc_b200 import raster, scenes
from gsparc_b200.shared_mlp import SharedMLP

pytestmark = pytest.mark.gpu


def torch_features(means, rxs, radii):
    R, P = radii.shape
    m = means[None].expand(R, P, 3)
    v = m - rxs[:, None, :]
    d2 = (v * v).sum(-1, keepdim=True)
    d = d2.sqrt()
    pe = []
    for k in range(4):
        w = (2 ** k) * math.pi
        for j in range(3):
            pe += [torch.sin(w * m[..., j]), torch.cos(w * m[..., j])]
    x = torch.cat([m, torch.stack(pe, -1), v / d, 1.0 / d2, torch.zeros_like(d)], -1)
    return torch.where((radii > 0)[..., None], x, torch.zeros_like(x))


def torch_signal(mlp, params, means, rxs, radii):
    h = torch_features(means, rxs, radii)
    layers = mlp.unflatten(params)
    act = F.relu if mlp.act == "relu" else F.gelu
    for w, b in layers[:-1]:
        h = act(h @ w.T + b)
    w, b = layers[-1]
    return torch.sigmoid((h @ w.T + b)[..., 0])


def _scene(P, R, seed):
    dev = torch.device("cuda")
    sc = scenes.make_scene(P, seed=seed)
    rx = scenes.make_receivers(R)
    t = lambda a: torch.tensor(np.ascontiguousarray(a), dtype=torch.float32, device=dev)
    m, s, q, o = sc.activated()
    return dict(means=t(m), scales=t(s), rots=t(q), opac=t(o.reshape(-1)), views=t(scenes.view_matrices(rx)),
                rxs=t(rx), tx=t(scenes.TX_POS))


# width 64 with one or two layers runs the fused kernels (R = 7 puts more than
# one 128-row tile on some CTAs; with R = 1 the adjoint also runs the feature
# adjoint); the rest runs the tiled GEMM path
@pytest.mark.parametrize("layers,width,act,R", [(2, 64, "relu", 1), (3, 128, "gelu", 3), (2, 64, "relu", 2),
                                                (2, 64, "relu", 7), (1, 64, "gelu", 2), (2, 64, "gelu", 1),
                                                (3, 64, "relu", 1), (1, 64, "gelu", 1)])
def test_shared_mlp_forward_and_backward_match_torch(layers, width, act, R):
    torch.backends.cuda.matmul.allow_tf32 = False
    P = 3001
    sc = _scene(P, R, seed=4)
    mlp = SharedMLP(layers, width, act)
    params = mlp.init_params(seed=layers * 10 + R)
    out_r, _, radii, st = raster.forward(sc["means"], None, sc["opac"], sc["scales"], sc["rots"], 90, 360, 1.0,
                                         sc["views"], sc["tx"], sc["rxs"], shared=mlp, shared_params=params)
    torch.cuda.synchronize()
    assert st.num_rendered > 0
    sig = raster.state_views(st)["signal"]
    ref = torch_signal(mlp, params, sc["means"], sc["rxs"], radii)
    vis = radii > 0
    assert vis.any()
    assert (sig[..., 0][vis] - ref[vis]).abs().max().item() <= 2e-6
    assert (sig[..., 1][vis] == 0).all()
    # backward of sum(dsig * signal) through the MLP and the features
    gen = torch.Generator().manual_seed(5)
    dsig = torch.randn((R, P, 2), generator=gen).cuda() * vis[..., None]
    dparams = torch.empty_like(params)
    dmeans = torch.zeros_like(sc["means"])
    mlp.backward(P, R, sc["means"], sc["rxs"], params, st.geom, dsig.contiguous(), dparams, dmeans)
    torch.cuda.synchronize()
    p = params.detach().clone().requires_grad_(True)
    mm = sc["means"].detach().clone().requires_grad_(True)
    (dsig[..., 0] * torch_signal(mlp, p, mm, sc["rxs"], radii)).sum().backward()
    for (gw, gb), (rw, rb) in zip(mlp.unflatten(dparams), mlp.unflatten(p.grad)):
        for a, b in ((gw, rw), (gb, rb)):
            assert (a - b).abs().max().item() <= 1e-4 * b.abs().max().item() + 1e-7
    assert (dmeans - mm.grad).abs().max().item() <= 1e-4 * mm.grad.abs().max().item()


def test_shared_mlp_render_rejects_both_models():
    sc = _scene(64, 1, seed=1)
    mlp = SharedMLP()
    with pytest.raises(ValueError, match="either"):
        raster.forward(sc["means"], torch.zeros(194 * 64, device="cuda"), sc["opac"], sc["scales"], sc["rots"],
                       90, 360, 1.0, sc["views"], sc["tx"], sc["rxs"], shared=mlp, shared_params=mlp.init_params())


def _bf(x):
    return x.bfloat16().float()


def torch_bf16_emulation(mlp, params, means, rxs, radii, dsig):
    """The BF16 tensor-core path's arithmetic restated in torch: operands
    rounded to BF16 where the kernels round them (and the hidden layers'
    activation derivatives to FP16, as the adjoint holds them), FP32
    accumulation.
    Returns (signal, dparams, dmeans)."""
    act = (lambda z: F.relu(z)) if mlp.act == "relu" else (lambda z: F.gelu(z))
    layers = mlp.unflatten(params)
    L = len(layers) - 1
    p = params.detach().clone().requires_grad_(True)
    m = means.detach().clone().requires_grad_(True)
    lay = mlp.unflatten(p)
    x = torch_features(m, rxs, radii)
    h = _bf(x)
    zs = []
    for l in range(L):
        w, b = lay[l]
        z = _bf(h @ _bf(w).T + b)
        zs.append(z)
        h = _bf(act(z)) if l + 1 < L else act(z)
    wo, bo = lay[L]
    s = torch.sigmoid(h @ wo.T + bo)[..., 0]
    # adjoint with the kernels' roundings
    with torch.no_grad():
        dO = dsig[..., 0] * s * (1 - s)
        grads = [None] * (2 * L + 2)
        aL = act(zs[-1])
        grads[2 * L] = (dO[..., None] * aL).sum((0, 1))[None]
        grads[2 * L + 1] = dO.sum()[None]
        dz = _bf(dO[..., None] * wo[0] * torch.func.grad(lambda q: act(q).sum())(zs[-1]))
        for l in range(L - 1, -1, -1):
            w, _ = lay[l]
            a_in = _bf(x) if l == 0 else _bf(act(zs[l - 1]))
            grads[2 * l] = torch.einsum("rpo,rpi->oi", dz, a_in)
            grads[2 * l + 1] = dz.sum((0, 1))
            dA = dz @ _bf(w)
            if l == 0:
                dX0 = dA
            else:
                dz = _bf(dA * torch.func.grad(lambda q: act(q).sum())(zs[l - 1]).half().float())
        dparams = torch.cat([g.reshape(-1) for g in grads])
    # centres: through the features only
    mm = means.detach().clone().requires_grad_(True)
    (torch_features(mm, rxs, radii) * dX0).sum().backward()
    return s.detach(), dparams, mm.grad


@pytest.mark.parametrize("layers,act,R", [(3, "gelu", 2), (2, "relu", 1), (1, "gelu", 3)])
def test_shared_mlp_bf16_tensor_cores_match_bf16_emulation(layers, act, R):
    """BF16 operands on tcgen05 with FP32 accumulation, against the same
    roundings restated in torch: signals within 1e-4 absolute, gradients within
    2e-3 of each tensor's largest magnitude (FP32 accumulation order and the
    kernels' atomics differ); against the FP32 network: signals within 1e-2."""
    torch.backends.cuda.matmul.allow_tf32 = False
    P = 2999
    sc = _scene(P, R, seed=7)
    mlp = SharedMLP(layers, 128, act, precision="bf16")
    params = mlp.init_params(seed=11 + layers)
    out_r, _, radii, st = raster.forward(sc["means"], None, sc["opac"], sc["scales"], sc["rots"], 90, 360, 1.0,
                                         sc["views"], sc["tx"], sc["rxs"], shared=mlp, shared_params=params)
    K, err = raster.read_status(st)
    assert err == 0 and K > 0
    sig = raster.state_views(st)["signal"]
    vis = radii > 0
    gen = torch.Generator().manual_seed(8)
    dsig = (torch.randn((R, P, 2), generator=gen).cuda() * vis[..., None]).contiguous()
    ref_s, ref_dp, ref_dm = torch_bf16_emulation(mlp, params, sc["means"], sc["rxs"], radii, dsig)
    # a pre-activation within FP32 rounding of a BF16 rounding boundary may round
    # the other way (accumulation order), which moves a signal by ~1e-5
    assert (sig[..., 0][vis] - ref_s[vis]).abs().max().item() <= 1e-4
    fp32 = torch_signal(SharedMLP(layers, 128, act), params, sc["means"], sc["rxs"], radii)
    assert (sig[..., 0][vis] - fp32[vis]).abs().max().item() <= 1e-2
    dparams = torch.empty_like(params)
    dmeans = torch.zeros_like(sc["means"])
    mlp.backward(P, R, sc["means"], sc["rxs"], params, st.geom, dsig, dparams, dmeans, st.image)
    K, err = raster.read_status(st)
    assert err == 0
    for (gw, gb), (rw, rb) in zip(mlp.unflatten(dparams), mlp.unflatten(ref_dp)):
        for a, b in ((gw, rw), (gb, rb)):
            assert (a - b).abs().max().item() <= 2e-3 * b.abs().max().item() + 1e-6
    assert (dmeans - ref_dm).abs().max().item() <= 2e-3 * ref_dm.abs().max().item()


def test_bf16_and_fp32_renders_against_fp64_oracle():
    """Error of the rendered spectra against the FP64 oracle render (oracle/
    raster + oracle/shared_mlp in float64) for the 3x128 GELU model, FP32 and
    BF16 tensor-core MLPs.  On pixels whose contributor count agrees with the
    oracle's: FP32 within 1e-4 of the peak, BF16 within 2e-2 of the peak; the
    SSIM of either render against the FP64 one is within 1e-3 of 1, and the
    two differ by at most 1e-3.  The measured figures are printed."""
    from fused_ssim import fused_ssim
    from oracle import raster as oraster
    from oracle import shared_mlp as osm
    P, R = 4096, 2
    sc = _scene(P, R, seed=9)
    mlp32 = SharedMLP(3, 128, "gelu")
    params = mlp32.init_params(seed=21)
    outs = {}
    for prec in ("fp32", "bf16"):
        mlp = SharedMLP(3, 128, "gelu", precision=prec)
        out_r, _, radii, st = raster.forward(sc["means"], None, sc["opac"], sc["scales"], sc["rots"], 90, 360, 1.0,
                                             sc["views"], sc["tx"], sc["rxs"], shared=mlp, shared_params=params)
        K, err = raster.read_status(st)
        assert err == 0
        outs[prec] = (out_r.cpu().numpy(), raster.state_views(st)["n_contrib"].cpu().numpy())
    c = lambda a: a.detach().cpu().numpy().astype(np.float64)
    pnp = params.cpu().numpy()
    for r in range(R):
        rx = c(sc["rxs"][r])

        def signal_fn(radii):
            s, _ = osm.forward(pnp, 3, 128, "gelu", c(sc["means"]), rx, radii, dtype=np.float64)
            return np.stack([s * (radii > 0), np.zeros_like(s)], 1)

        ref = oraster.render(c(sc["means"]), c(sc["scales"]), c(sc["rots"]), c(sc["opac"]), None,
                             c(sc["views"][r]), c(sc["tx"]), rx, 90, 360, dtype=np.float64, signal_fn=signal_fn)
        o64, nc64 = ref["out"][0], ref["n_contrib"]
        peak = np.abs(o64).max()
        errs = {}
        for prec, (o, nc) in outs.items():
            same = nc[r] == nc64
            assert same.mean() >= 0.99
            errs[prec] = np.abs(o[r] - o64)[same].max() / peak
        s32, s16 = [float(fused_ssim(torch.tensor(outs[p][0][r])[None, None].cuda(),
                                     torch.tensor(o64, dtype=torch.float32)[None, None].cuda()))
                    for p in ("fp32", "bf16")]
        print(f"receiver {r}: max-abs error / peak vs FP64 oracle: fp32 {errs['fp32']:.3e}, bf16 {errs['bf16']:.3e}; "
              f"SSIM vs FP64 render: fp32 {s32:.6f}, bf16 {s16:.6f}")
        assert errs["fp32"] <= 1e-4
        assert errs["bf16"] <= 2e-2
        assert 1.0 - s32 <= 1e-3 and 1.0 - s16 <= 1e-3 and abs(s32 - s16) <= 1e-3


def torch_bf16_emulation_multi(mlp, params, means, rxs, radii, dfeat):
    """torch_bf16_emulation for an MLP with several outputs, whose output layer
    is one more BF16 MMA: the last hidden activations and dO enter it rounded to
    BF16; db_out sums dO in FP32.  Returns (features [R,P,out], dparams, dmeans)."""
    act = (lambda z: F.relu(z)) if mlp.act == "relu" else (lambda z: F.gelu(z))
    dact = lambda q: torch.func.grad(lambda u: act(u).sum())(q)
    lay = mlp.unflatten(params)
    L = len(lay) - 1
    x = torch_features(means, rxs, radii)
    h = _bf(x)
    zs = []
    for l in range(L):
        w, b = lay[l]
        z = _bf(h @ _bf(w).T + b)
        zs.append(z)
        h = _bf(act(z))
    wo, bo = lay[L]
    s = torch.sigmoid(h @ _bf(wo).T + bo)
    with torch.no_grad():
        dO = dfeat * s * (1 - s)
        dOb = _bf(dO)
        grads = [None] * (2 * L + 2)
        grads[2 * L] = torch.einsum("rpo,rph->oh", dOb, h)
        grads[2 * L + 1] = dO.sum((0, 1))
        dz = _bf((dOb @ _bf(wo)) * dact(zs[-1]).half().float())
        for l in range(L - 1, -1, -1):
            w, _ = lay[l]
            a_in = _bf(x) if l == 0 else _bf(act(zs[l - 1]))
            grads[2 * l] = torch.einsum("rpo,rpi->oi", dz, a_in)
            grads[2 * l + 1] = dz.sum((0, 1))
            dA = dz @ _bf(w)
            if l == 0:
                dX0 = dA
            else:
                dz = _bf(dA * dact(zs[l - 1]).half().float())
        dparams = torch.cat([g.reshape(-1) for g in grads])
    mm = means.detach().clone().requires_grad_(True)
    (torch_features(mm, rxs, radii) * dX0).sum().backward()
    return s, dparams, mm.grad


@pytest.mark.parametrize("layers,act,R", [(3, "gelu", 2), (1, "relu", 1), (2, "gelu", 1)])
def test_shared_mlp_bf16_64_outputs_match_bf16_emulation(layers, act, R):
    """BF16 tensor-core MLP with 64 outputs (the output layer as an MMA, N = 64)
    against the torch restatement of its roundings: >= 99.9 % of amplitudes
    within 1e-5 and all within 2e-3 absolute, gradients within 2e-3 of each
    tensor's largest magnitude; against the FP32 network: amplitudes within
    1e-2."""
    torch.backends.cuda.matmul.allow_tf32 = False
    P = 2999
    sc = _scene(P, R, seed=7)
    mlp = SharedMLP(layers, 128, act, out=64, precision="bf16")
    params = mlp.init_params(seed=11 + layers)
    out, radii, st = raster.forward_channels(sc["means"], sc["opac"], sc["scales"], sc["rots"], 90, 360, 1.0,
                                             sc["views"], sc["tx"], sc["rxs"], mlp, params)
    K, err = raster.read_status(st)
    assert err == 0 and K > 0
    feats = mlp.features(P, R).clone()
    vis = radii > 0
    gen = torch.Generator().manual_seed(8)
    dfeat = (torch.randn((R, P, 64), generator=gen).cuda() * vis[..., None]).contiguous()
    ref_s, ref_dp, ref_dm = torch_bf16_emulation_multi(mlp, params, sc["means"], sc["rxs"], radii, dfeat)
    # a hidden pre-activation within FP32 rounding of a BF16 rounding boundary
    # may round the other way (accumulation order) and moves that pair's 64
    # outputs by up to ~1e-3; all other amplitudes agree to FP32 rounding
    diff = (feats[vis] - ref_s[vis]).abs()
    assert (diff <= 1e-5).float().mean().item() >= 0.999
    assert diff.max().item() <= 2e-3
    fp = SharedMLP(layers, 128, act, out=64)
    h = torch_features(sc["means"], sc["rxs"], radii)
    lay = fp.unflatten(params)
    for w, b in lay[:-1]:
        h = (F.relu if act == "relu" else F.gelu)(h @ w.T + b)
    fp32 = torch.sigmoid(h @ lay[-1][0].T + lay[-1][1])
    assert (feats[vis] - fp32[vis]).abs().max().item() <= 1e-2
    dparams = torch.empty_like(params)
    dmeans = torch.zeros_like(sc["means"])
    mlp.backward(P, R, sc["means"], sc["rxs"], params, st.geom, dfeat, dparams, dmeans, st.image)
    K, err = raster.read_status(st)
    assert err == 0
    for (gw, gb), (rw, rb) in zip(mlp.unflatten(dparams), mlp.unflatten(ref_dp)):
        for a, b in ((gw, rw), (gb, rb)):
            assert (a - b).abs().max().item() <= 2e-3 * b.abs().max().item() + 1e-6
    assert (dmeans - ref_dm).abs().max().item() <= 2e-3 * ref_dm.abs().max().item()
