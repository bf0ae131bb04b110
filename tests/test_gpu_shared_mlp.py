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
from gsparc_b200.shared_mlp import SharedMLP, bf16_act_table

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


# The BF16 path evaluates its activation on BF16 pre-activations in FP32 with
# the hardware tanh (GELU in the tanh form with coefficients fitted to the erf
# GELU), rounding act and act' to BF16; the restatement below takes them from
# the device's own table over all BF16 inputs (checked against the erf GELU in
# test_bf16_activation_table), everything else from torch.
_ACT_TABLES = {}


def bf16_act_and_grad(act, z):
    """act(z) and act'(z) of BF16 pre-activations as the kernels evaluate them."""
    if act not in _ACT_TABLES:
        _ACT_TABLES[act] = bf16_act_table(act)
    _, a, d = _ACT_TABLES[act]
    idx = z.bfloat16().view(torch.int16).to(torch.int64) & 0xFFFF
    return a[idx], d[idx]


def torch_bf16_emulation(mlp, params, means, rxs, radii, dout):
    """The BF16 tensor-core path's arithmetic restated in torch: MMA operands
    rounded to BF16 (features, weights, activations, dO, dZ), FP32
    accumulation, pre-activations z = BF16(acc + b), activations and their
    derivatives in BF16 (bf16_act_and_grad), dZ = BF16(BF16(dA) act'(z)), the
    output layer an MMA like the hidden ones, db_out summed in FP32.
    dout: dL/dsignal [R, P, 2] (one output; its real channel) or
    dL/dfeatures [R, P, out].  Returns (outputs [R, P] or [R, P, out],
    dparams, dmeans)."""
    lay = mlp.unflatten(params)
    L = len(lay) - 1
    x = torch_features(means, rxs, radii)
    h = _bf(x)
    zs, ds = [], []
    for l in range(L):
        w, b = lay[l]
        z = _bf(h @ _bf(w).T + b)
        a, d = bf16_act_and_grad(mlp.act, z)
        zs.append(z)
        ds.append(d)
        h = a
    wo, bo = lay[L]
    s = torch.sigmoid(h @ _bf(wo).T + bo)
    with torch.no_grad():
        g = dout[..., :1] if mlp.out == 1 else dout
        dO = g * s * (1 - s)
        dOb = _bf(dO)
        grads = [None] * (2 * L + 2)
        grads[2 * L] = torch.einsum("rpo,rph->oh", dOb, h)
        grads[2 * L + 1] = dO.sum((0, 1))
        dz = _bf(_bf(dOb @ _bf(wo)) * ds[-1])
        for l in range(L - 1, -1, -1):
            w, _ = lay[l]
            a_in = _bf(x) if l == 0 else bf16_act_and_grad(mlp.act, zs[l - 1])[0]
            grads[2 * l] = torch.einsum("rpo,rpi->oi", dz, a_in)
            grads[2 * l + 1] = dz.sum((0, 1))
            dA = dz @ _bf(w)
            if l == 0:
                dX0 = dA
            else:
                dz = _bf(_bf(dA) * ds[l - 1])
        dparams = torch.cat([q.reshape(-1) for q in grads])
    # centres: through the features only
    mm = means.detach().clone().requires_grad_(True)
    (torch_features(mm, rxs, radii) * dX0).sum().backward()
    return (s[..., 0] if mlp.out == 1 else s).detach(), dparams, mm.grad


def test_bf16_activation_table():
    """The BF16 path's activation over every BF16 input, as its kernels
    evaluate it (both lanes of a packed pair agree -- checked by
    bf16_act_table): the forward's and the adjoint's act are bit for bit the
    same; ReLU is exact (max(z, 0), derivative 1 above 0); GELU against the
    erf GELU in float64 over [-8, 8]: act within 4e-3 max(1, |z|) (one BF16
    step of the result) and act' within 1e-2 (BF16 steps near 1 are 7.8e-3);
    large inputs saturate (act(z) = z, act'(z) = 1 for z >= 8; act = act' = 0
    for z <= -8)."""
    from scipy.special import erf
    v = (np.arange(65536, dtype=np.uint32) << 16).view(np.float32)
    fin = np.isfinite(v)
    for act in ("relu", "gelu"):
        af, a, d = [x.cpu().numpy() for x in bf16_act_table(act)]
        assert np.array_equal(af.view(np.uint32), a.view(np.uint32))
        if act == "relu":
            assert np.array_equal(a[fin], np.maximum(v[fin], 0).astype(np.float32))
            assert np.array_equal(d[fin], (v[fin] > 0).astype(np.float32))
            continue
        m = fin & (np.abs(v) <= 8)
        z = v[m].astype(np.float64)
        phi = 0.5 * (1.0 + erf(z / np.sqrt(2.0)))
        ea = np.abs(a[m] - z * phi) / np.maximum(1.0, np.abs(z))
        ed = np.abs(d[m] - (phi + z * np.exp(-0.5 * z * z) / np.sqrt(2.0 * np.pi)))
        print(f"BF16 GELU vs erf GELU over [-8, 8]: act {ea.max():.3e} (relative to max(1,|z|)), act' {ed.max():.3e}")
        assert ea.max() <= 4e-3 and ed.max() <= 1e-2
        hi = fin & (v >= 8) & (v < 1e18)
        lo = fin & (v <= -8) & (v > -1e18)
        assert np.array_equal(a[hi], v[hi]) and (d[hi] == 1).all()
        assert (a[lo] == 0).all() and (d[lo] == 0).all()


@pytest.mark.parametrize("layers,act,R", [(3, "gelu", 2), (2, "relu", 1), (1, "gelu", 3)])
def test_shared_mlp_bf16_tensor_cores_match_bf16_emulation(layers, act, R):
    """BF16 operands on tcgen05 with FP32 accumulation, against the same
    roundings restated in torch (the activation from the device's own table):
    >= 99.9 % of signals within 1e-4 and all within 2e-3 absolute (a
    pre-activation within FP32 rounding of a BF16 rounding boundary rounds the
    other way under another accumulation order and moves the pair's later
    layers), gradients within 3e-3 of each tensor's largest magnitude (the same
    flips in dA and dZ, and the order of the kernels' FP32 atomics); against
    the FP32 network (erf GELU): signals within 1e-2."""
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
    diff = (sig[..., 0][vis] - ref_s[vis]).abs()
    assert (diff <= 1e-4).float().mean().item() >= 0.999
    assert diff.max().item() <= 2e-3
    fp32 = torch_signal(SharedMLP(layers, 128, act), params, sc["means"], sc["rxs"], radii)
    assert (sig[..., 0][vis] - fp32[vis]).abs().max().item() <= 1e-2
    dparams = torch.empty_like(params)
    dmeans = torch.zeros_like(sc["means"])
    mlp.backward(P, R, sc["means"], sc["rxs"], params, st.geom, dsig, dparams, dmeans, st.image)
    K, err = raster.read_status(st)
    assert err == 0
    for (gw, gb), (rw, rb) in zip(mlp.unflatten(dparams), mlp.unflatten(ref_dp)):
        for a, b in ((gw, rw), (gb, rb)):
            assert (a - b).abs().max().item() <= 3e-3 * b.abs().max().item() + 1e-6
    assert (dmeans - ref_dm).abs().max().item() <= 3e-3 * ref_dm.abs().max().item()


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


@pytest.mark.parametrize("layers,act,R", [(3, "gelu", 2), (1, "relu", 1), (2, "gelu", 1)])
def test_shared_mlp_bf16_64_outputs_match_bf16_emulation(layers, act, R):
    """BF16 tensor-core MLP with 64 outputs (the output layer as an MMA, N = 64)
    against the torch restatement of its roundings: >= 99.9 % of amplitudes
    within 1e-5 and all within 2e-3 absolute, gradients within 3e-3 of each
    tensor's largest magnitude (BF16 rounding flips under another FP32
    accumulation order, as in the one-output test); against the FP32 network:
    amplitudes within 1e-2."""
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
    ref_s, ref_dp, ref_dm = torch_bf16_emulation(mlp, params, sc["means"], sc["rxs"], radii, dfeat)
    # a hidden pre-activation within FP32 rounding of a BF16 rounding boundary
    # (accumulation order), or a hardware tanh one BF16 step from torch's,
    # moves that pair's 64 outputs by up to ~1e-3
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
            assert (a - b).abs().max().item() <= 3e-3 * b.abs().max().item() + 1e-6
    assert (dmeans - ref_dm).abs().max().item() <= 3e-3 * ref_dm.abs().max().item()
