"""CPU tests pinning the densification and evaluation-metric oracles to
outputs of the reference's own Python code (tests/golden/densify_eval_golden.npz,
recorded by tests/golden/make_densify_golden.py from gaussian.py's
GaussianModel.densify_and_prune and train.py's / utils.py's metric functions).

Densification: the oracle, given the same parameters, moments, statistics and
the split offsets the reference drew, must produce the same Gaussian count,
the same order and values (float64 oracle vs the reference's float32: 1e-6
relative), the emission-MLP rows copied from the same input rows, and new
Gaussians' Adam moments at zero exactly where the reference zeroed them.
Metrics: PSNR, RSSI difference, MAE, SSIM, confidence and evaluation loss
within 1e-5 relative + 5e-6 absolute of the reference's float32 values (the
RSSI difference subtracts two values near -30 dBm whose float32 ulp is
1.9e-6)."""
import importlib.util
import os

import numpy as np
import pytest

from oracle import densify as od
from oracle import metrics as om

HERE = os.path.dirname(os.path.abspath(__file__))
FIX = os.path.join(HERE, "golden", "densify_eval_golden.npz")


def _gen():
    spec = importlib.util.spec_from_file_location("mdg", os.path.join(HERE, "golden", "make_densify_golden.py"))
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    return m


def _load(name):
    z = np.load(FIX)
    return {k.split("/", 1)[1]: z[k] for k in z.files if k.startswith(name + "/")}


MLP_PARTS = ("fc1_w", "fc1_b", "fc2_w", "fc2_b")


@pytest.mark.parametrize("case", [c[0] for c in _gen().DENSIFY_CASES])
def test_densify_oracle_matches_reference_densify_and_prune(case):
    gen = _gen()
    name, P, seed, max_grad, min_op, extent, mss, box = [c for c in gen.DENSIFY_CASES if c[0] == case][0]
    st, m1, m2, accum, denom, max_radii, radii = gen.densify_inputs(P, seed)
    g = _load(name)
    cat = lambda d: np.concatenate([d[q].reshape(P, -1) for q in MLP_PARTS], 1)
    mk = lambda d: dict(centre=d["centre"], log_scale=d["log_scale"], rotation=d["rotation"],
                        opacity=d["opacity"].reshape(P), mlp=cat(d))
    kw = dict(max_grad=max_grad, min_opacity=min_op, extent=extent, max_screen_size=mss,
              scene_min=[-4.5, 0.2, -3.5] if box else None, scene_max=[4.5, 2.8, 3.5] if box else None)
    o_st, o_m1, o_m2 = od.densify_and_prune(mk(st), mk(m1), mk(m2), accum.reshape(P), denom.reshape(P),
                                            split_samples=g["split_samples"], **kw)
    n = g["centre"].shape[0]
    assert o_st["centre"].shape[0] == n
    for key in ("centre", "log_scale", "rotation", "opacity"):
        ref = g[key].reshape(n, -1).astype(np.float64)
        for got, r in ((o_st[key], ref), (o_m1[key], g["m1_" + key]), (o_m2[key], g["m2_" + key])):
            r = np.asarray(r, np.float64).reshape(n, -1)
            np.testing.assert_allclose(np.asarray(got).reshape(n, -1), r, rtol=1e-6, atol=1e-7, err_msg=key)
    # emission-MLP rows: copies of the input rows the reference copied, moments zero where it zeroed them
    np.testing.assert_array_equal(o_st["mlp"], cat(st)[g["mlp_src"]].astype(np.float64))
    for o_m, m_in, src in ((o_m1, m1, g["mlp_m1_src"]), (o_m2, m2, g["mlp_m2_src"])):
        exp = np.where((src >= 0)[:, None], cat(m_in)[np.maximum(src, 0)], 0.0)
        np.testing.assert_array_equal(o_m["mlp"], exp)


def test_metrics_oracle_matches_reference_metric_functions():
    gen = _gen()
    for name, R, seed in gen.EVAL_CASES:
        pred, tgt, rx, conf = gen.eval_inputs(R, seed)
        ref = _load(name)["metrics"]
        got = om.evaluate(pred, tgt, rx, conf, gen.CONF_HIDDEN)
        np.testing.assert_allclose(got, ref, rtol=1e-5, atol=5e-6)
