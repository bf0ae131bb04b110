"""GPU parity of the azimuth seam wrap (GSPARC_FLAG_WRAP_AZIMUTH) against the
CPU oracle's wrap (oracle/raster.py: get_span, wrap_shift), on a scene with
many footprints across the 0/2pi seam.

Integer work bit-exact (tile ranges and point lists, from the GPU's own
preprocess outputs); spectra within 1e-5 of the peak on pixels whose
contributor count agrees with the FP32 oracle's (>= 99.9% of pixels);
blend gradients agree with the FP32 oracle's adjoint on the GPU's lists as
the clamped adjoint's do (relative 2-norm <= 2e-3, >= 99.5% of entries within
1e-2); the FP64 oracle render's error is stated (<= 1e-4 of the
peak on matching pixels).  With the wrap off the same scene bins exactly as
the reference's clamped rectangles."""
import numpy as np
import pytest
import torch

from gsparc_b200 import raster
from oracle import raster as oraster
from tests._helpers import to_np
from tests.test_gpu_backward import _agree
from tests.test_oracle import _seam_scene

pytestmark = pytest.mark.gpu


def _inputs(H, W, P=900, seed=3):
    means, scales, q, opac, _ = _seam_scene(P, seed)
    rx = np.array([0.3, 1.2, -0.4])
    means = means + rx
    rng = np.random.default_rng(seed + 1)
    mlp = rng.normal(0, 0.3, 194 * P)
    view = np.eye(4)
    view[3, :3] = -rx
    f = lambda a: np.ascontiguousarray(a, dtype=np.float32)
    np_in = dict(means=f(means), scales=f(scales), rots=f(q), opac=f(opac), mlp=f(mlp), view=f(view),
                 tx=f([0.0, 0.5, 3.0]), rx=f(rx))
    t = lambda a: torch.from_numpy(a).cuda()
    th = {k: t(v) for k, v in np_in.items()}
    return np_in, th


def _forward(th, H, W, wrap, tile=(16, 16)):
    out = raster.forward(th["means"], th["mlp"], th["opac"], th["scales"], th["rots"], H, W, 1.0,
                         th["view"][None], th["tx"], th["rx"][None], tile=tile, wrap=wrap)
    torch.cuda.synchronize()
    return out


@pytest.mark.parametrize("H,W,tile", [(90, 360, (16, 16)), (48, 352, (16, 16)), (90, 360, (8, 32))])
def test_wrap_binning_and_blend_match_oracle(H, W, tile):
    np_in, th = _inputs(H, W)
    out_r, out_i, _, st = _forward(th, H, W, True, tile)
    g = to_np(raster.state_views(st))
    keys, vals, ranges = oraster.bin_and_sort(g["means2D"][0], g["depth"][0], g["radii"][0], H, W, *tile, wrap=True)
    keys0, _, _ = oraster.bin_and_sort(g["means2D"][0], g["depth"][0], g["radii"][0], H, W, *tile, wrap=False)
    assert keys.size > keys0.size   # footprints crossed the seam
    assert st.num_rendered == keys.size
    np.testing.assert_array_equal(g["ranges"][0].astype(np.uint32), ranges)
    np.testing.assert_array_equal(g["point_list"].astype(np.uint32), vals)
    out, fT, nc = oraster.blend_forward(g["ranges"][0], g["point_list"], g["means2D"][0], g["conic_opacity"][0],
                                        g["signal"][0], H, W, tile[0], tile[1], np.float32, wrap=True)
    same = g["n_contrib"][0] == nc
    assert same.mean() >= 0.999, same.mean()
    peak = np.abs(out).max()
    gout = np.stack([out_r.cpu().numpy()[0], out_i.cpu().numpy()[0]])
    assert np.abs(gout - out)[:, same].max() <= 1e-5 * peak
    # the seam columns see each other: the wrapped render differs there from the clamped one
    c_r, _, _, _ = _forward(th, H, W, False, tile)
    diff = (out_r - c_r).abs().cpu().numpy()[0]
    assert diff[:, :4].max() > 1e-3 * peak or diff[:, -4:].max() > 1e-3 * peak
    # and the clamped render still bins as the reference
    gc = to_np(raster.state_views(_forward(th, H, W, False, tile)[3]))
    _, vals_c, ranges_c = oraster.bin_and_sort(gc["means2D"][0], gc["depth"][0], gc["radii"][0], H, W, *tile)
    np.testing.assert_array_equal(gc["point_list"].astype(np.uint32), vals_c)


def test_wrap_blend_adjoint_matches_oracle():
    H, W = 90, 360
    np_in, th = _inputs(H, W)
    out_r, out_i, _, st = _forward(th, H, W, True)
    g = to_np(raster.state_views(st))
    rng = np.random.default_rng(7)
    dout = rng.normal(size=(2, H, W)).astype(np.float32)
    gr = raster.backward(st, th["means"], th["mlp"], th["scales"], th["rots"], 1.0, th["view"][None], th["tx"],
                         th["rx"][None], torch.from_numpy(dout[0][None]).cuda(),
                         torch.from_numpy(dout[1][None]).cuda(), grad_mode="exact")
    torch.cuda.synchronize()
    dm, dc, dop, ds = oraster.blend_backward(g["ranges"][0], g["point_list"], g["means2D"][0], g["conic_opacity"][0],
                                             g["signal"][0], g["final_T"][0], g["n_contrib"][0], dout, H, W,
                                             dtype=np.float32, ref_compat=False, wrap=True)
    _agree(gr["dmeans2D"].cpu().numpy()[0][:, :2], dm[:, :2])
    _agree(gr["dconic"].cpu().numpy()[0][:, [0, 1, 3]], dc[:, [0, 1, 3]])
    _agree(gr["dopacity"].cpu().numpy(), dop)
    _agree(gr["dsignal"].cpu().numpy()[0], ds)


def test_wrap_render_error_vs_fp64_oracle():
    H, W = 90, 360
    np_in, th = _inputs(H, W)
    out_r, out_i, _, st = _forward(th, H, W, True)
    f64 = lambda a: a.astype(np.float64)
    ref = oraster.render(f64(np_in["means"]), f64(np_in["scales"]), f64(np_in["rots"]), f64(np_in["opac"]),
                         f64(np_in["mlp"]), f64(np_in["view"]), f64(np_in["tx"]), f64(np_in["rx"]), H, W,
                         dtype=np.float64, wrap=True)
    g = to_np(raster.state_views(st))
    same = g["n_contrib"][0] == ref["n_contrib"]
    assert same.mean() >= 0.99
    gout = np.stack([out_r.cpu().numpy()[0], out_i.cpu().numpy()[0]])
    peak = np.abs(ref["out"]).max()
    err = np.abs(gout - ref["out"])[:, same].max() / peak
    print(f"seam wrap: max-abs error vs FP64 oracle {err:.3e} of peak on {same.mean() * 100:.3f}% of pixels")
    assert err <= 1e-4
