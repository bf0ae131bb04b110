"""GPU parity of the multi-channel render (gsparc_rasterize_render_channels /
_backward_channels) and of the FP32 shared MLP with several outputs.

- Final T and contributor counts equal a single-channel render of the same
  geometry (the decisions do not depend on the amplitudes), bit for bit.
- Spectra against the FP32 oracle (oracle/raster.blend_forward_channels) on
  the GPU's own lists and amplitudes: within 1e-5 of the peak on pixels whose
  contributor count agrees (>= 99.9 %).
- The blend adjoint against oracle/raster.blend_backward_channels on the same
  inputs: relative 2-norm <= 2e-3 and >= 99.5 % of entries within 1e-2, as the
  single-channel adjoint's tests.
- The shared MLP's amplitudes and its parameter / centre gradients against the
  same network in plain torch fp32 with autograd: 2e-6 absolute; 1e-4 of each
  tensor's peak."""
import numpy as np
import pytest
import torch

from gsparc_b200 import raster
from gsparc_b200.shared_mlp import SharedMLP
from oracle import raster as oraster
from tests._helpers import to_np
from tests.test_gpu_backward import _agree
from tests.test_gpu_shared_mlp import _scene, torch_features

pytestmark = pytest.mark.gpu


def _render(sc, mlp, params, tile=(16, 16), wrap=False):
    out, radii, st = raster.forward_channels(sc["means"], sc["opac"], sc["scales"], sc["rots"], 90, 360, 1.0,
                                             sc["views"], sc["tx"], sc["rxs"], mlp, params, tile=tile, wrap=wrap)
    torch.cuda.synchronize()
    return out, radii, st


# 16 channels per CTA: C = 8 and 3 run one group, 64 four, 21 a full and a 5-channel group
@pytest.mark.parametrize("C,R,tile,wrap", [(8, 2, (16, 16), False), (64, 1, (8, 32), True), (3, 1, (32, 8), False),
                                           (21, 2, (16, 16), True)])
def test_channels_forward_and_adjoint_match_oracle(C, R, tile, wrap):
    P = 3000
    sc = _scene(P, R, seed=5)
    mlp = SharedMLP(2, 64, "relu", out=C)
    params = mlp.init_params(seed=3)
    out, radii, st = _render(sc, mlp, params, tile, wrap)
    K, err = raster.read_status(st)
    assert err == 0 and K > 0
    g = to_np(raster.state_views(st))
    feats = mlp.features(P, R).cpu().numpy()
    # the decisions equal a single-channel render of the same geometry
    one = SharedMLP(2, 64, "relu")
    _, _, _, st1 = raster.forward(sc["means"], None, sc["opac"], sc["scales"], sc["rots"], 90, 360, 1.0,
                                  sc["views"], sc["tx"], sc["rxs"], tile=tile, shared=one,
                                  shared_params=one.init_params(seed=3), wrap=wrap)
    torch.cuda.synchronize()
    g1 = to_np(raster.state_views(st1))
    np.testing.assert_array_equal(g["n_contrib"], g1["n_contrib"])
    np.testing.assert_array_equal(g["final_T"], g1["final_T"])
    rng = np.random.default_rng(C)
    dout = rng.normal(size=(R, C, 90, 360)).astype(np.float32)
    grads = raster.backward_channels(st, sc["means"], sc["scales"], sc["rots"], 1.0, sc["views"], sc["tx"],
                                     sc["rxs"], torch.from_numpy(dout).cuda(), mlp, params)
    torch.cuda.synchronize()
    G = {k: v.cpu().numpy() for k, v in grads.items()}
    o_np = out.cpu().numpy()
    pl = g["point_list"].astype(np.uint32)
    dop_sum = 0
    for r in range(R):
        ranges = g["ranges"][r].astype(np.uint32)
        ref, fT, nc = oraster.blend_forward_channels(ranges, pl, g["means2D"][r], g["conic_opacity"][r], feats[r],
                                                     90, 360, tile[0], tile[1], np.float32, wrap=wrap)
        same = g["n_contrib"][r] == nc
        assert same.mean() >= 0.999, same.mean()
        peak = np.abs(ref).max()
        assert np.abs(o_np[r] - ref)[:, same].max() <= 1e-5 * peak
        dm, dc, dop, df = oraster.blend_backward_channels(ranges, pl, g["means2D"][r], g["conic_opacity"][r],
                                                          feats[r], g["final_T"][r], g["n_contrib"][r], dout[r],
                                                          90, 360, tile[0], tile[1], np.float32, wrap=wrap)
        _agree(G["dmeans2D"][r][:, :2], dm[:, :2])
        _agree(G["dconic"][r][:, [0, 1, 3]], dc[:, [0, 1, 3]])
        _agree(G["dfeatures"][r], df)
        dop_sum = dop_sum + dop
    _agree(G["dopacity"], dop_sum)


def test_shared_mlp_with_several_outputs_matches_torch():
    torch.backends.cuda.matmul.allow_tf32 = False
    P, R, C = 2001, 2, 16
    sc = _scene(P, R, seed=6)
    mlp = SharedMLP(3, 32, "gelu", out=C)
    params = mlp.init_params(seed=9)
    out, radii, st = _render(sc, mlp, params)
    feats = mlp.features(P, R)
    vis = radii > 0

    def torch_feats(p, m):
        h = torch_features(m, sc["rxs"], radii)
        lay = mlp.unflatten(p)
        for w, b in lay[:-1]:
            h = torch.nn.functional.gelu(h @ w.T + b)
        w, b = lay[-1]
        return torch.sigmoid(h @ w.T + b)

    ref = torch_feats(params, sc["means"])
    assert (feats[vis] - ref[vis]).abs().max().item() <= 2e-6
    gen = torch.Generator().manual_seed(2)
    dfeat = (torch.randn((R, P, C), generator=gen).cuda() * vis[..., None]).contiguous()
    dparams = torch.empty_like(params)
    dmeans = torch.zeros_like(sc["means"])
    mlp.backward(P, R, sc["means"], sc["rxs"], params, st.geom, dfeat, dparams, dmeans, st.image)
    torch.cuda.synchronize()
    p = params.detach().clone().requires_grad_(True)
    mm = sc["means"].detach().clone().requires_grad_(True)
    (dfeat * torch_feats(p, mm)).sum().backward()
    for (gw, gb), (rw, rb) in zip(mlp.unflatten(dparams), mlp.unflatten(p.grad)):
        for a, b in ((gw, rw), (gb, rb)):
            assert (a - b).abs().max().item() <= 1e-4 * b.abs().max().item() + 1e-7
    assert (dmeans - mm.grad).abs().max().item() <= 1e-4 * mm.grad.abs().max().item()
