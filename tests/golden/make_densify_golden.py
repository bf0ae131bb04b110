"""Generates tests/golden/densify_eval_golden.npz from the reference's own
Python code, run on the CPU in a container that has the reference checked out
(its location: GSPARC_REFERENCE_ROOT, default as in oracle/build_ref.py):

    python tests/golden/make_densify_golden.py

Densification: GaussianModel.densify_and_prune (gaussian.py:515-542, with
densify_and_clone, densify_and_split, prune_points, densification_postfix,
cat_tensors_to_optimizer and _prune_optimizer) on seeded models whose
parameters, Adam moments and densification statistics are set directly.
The reference hard-codes device="cuda" for a few torch.zeros calls
(gaussian.py:458,464,421-423,486; utils.py:132); while it runs, torch.zeros
is wrapped to drop that argument so everything stays on the CPU.  The split's
torch.normal draws come from a seeded generator and the drawn offsets are
recorded, so the oracle can consume the same samples.

Evaluation metrics: calculate_psnr / calculate_rssi / calculate_mae
(train.py:76-101, taken from train.py's source by its function definitions,
without executing the rest of the module, whose imports -- tensorboard,
matplotlib -- are not installed here), utils.ssim and utils.l1_loss, and the
per-sample assembly of train.py:684-697 on seeded spectra.

The reference's utils.py imports plyfile for an unrelated PLY reader; an empty
stand-in module takes its place (as in make_golden.py).
"""
from __future__ import annotations

import ast
import os
import sys
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

# (name, P, seed, max_grad, min_opacity, extent, max_screen_size, with scene box)
DENSIFY_CASES = [
    ("d64", 64, 1, 0.02, 0.05, 4.0, None, False),
    ("d300_box", 300, 2, 0.03, 0.1, 2.5, 20.0, True),
    ("d500", 500, 3, 0.025, 0.02, 6.0, None, True),
]
EVAL_CASES = [("e4", 4, 11)]   # (name, receivers, seed)
CONF_HIDDEN = 32


def densify_inputs(P, seed):
    """Seeded per-Gaussian state: parameters, Adam moments, statistics."""
    rng = np.random.default_rng(seed)
    f = lambda *s: rng.normal(size=s).astype(np.float32)
    st = dict(centre=rng.uniform([-5, 0, -4], [5, 3, 4], size=(P, 3)).astype(np.float32),
              log_scale=(rng.normal(-2.5, 1.0, size=(P, 3))).astype(np.float32),
              rotation=f(P, 4), opacity=f(P, 1), fc1_w=f(P, 32, 3), fc1_b=f(P, 32), fc2_w=f(P, 2, 32), fc2_b=f(P, 2))
    m1 = {k: (0.01 * f(*v.shape)).astype(np.float32) for k, v in st.items()}
    m2 = {k: np.abs(0.001 * f(*v.shape)).astype(np.float32) for k, v in st.items()}
    accum = np.abs(rng.normal(0, 0.05, size=(P, 1))).astype(np.float32)
    denom = rng.integers(0, 4, size=(P, 1)).astype(np.float32)     # zeros give NaN grads, set to 0
    max_radii = rng.uniform(0, 40, size=P).astype(np.float32)
    radii = rng.integers(0, 30, size=P).astype(np.int32)
    return st, m1, m2, accum, denom, max_radii, radii


def eval_inputs(R, seed):
    rng = np.random.default_rng(seed)
    pred = rng.random((R, 90, 360), dtype=np.float32)
    tgt = np.clip(pred + 0.1 * rng.normal(size=pred.shape), 0, 1).astype(np.float32)
    rx = rng.uniform([-5, 0, -4], [5, 3, 4], size=(R, 3)).astype(np.float32)
    conf = (0.2 * rng.normal(size=5 * CONF_HIDDEN + 1)).astype(np.float32)
    return pred, tgt, rx, conf


def _import_reference(ref):
    sys.modules.setdefault("plyfile", types.SimpleNamespace(PlyData=None, PlyElement=None))
    if ref not in sys.path:
        sys.path.insert(0, ref)
    import initialization  # noqa: F401  (imports gaussian; the reverse order is circular)
    import gaussian
    import utils
    return gaussian, utils


class _CpuZeros:
    """torch.zeros without device="cuda" while the reference runs on the CPU."""

    def __enter__(self):
        import torch
        self._orig = torch.zeros

        def zeros(*a, **k):
            if str(k.get("device", "")).startswith("cuda"):
                k = dict(k, device="cpu")
            return self._orig(*a, **k)
        torch.zeros = zeros
        return self

    def __exit__(self, *exc):
        import torch
        torch.zeros = self._orig


def run_densify(gaussian, case):
    import torch
    import torch.nn as nn
    name, P, seed, max_grad, min_op, extent, mss, box = case
    st, m1, m2, accum, denom, max_radii, radii = densify_inputs(P, seed)
    model = gaussian.GaussianModel()
    model.percent_dense = 0.01
    params = {}
    for key, attr in (("centre", "_centre"), ("log_scale", "_scaling"), ("rotation", "_rotation"),
                      ("opacity", "_opacity")):
        params[key] = nn.Parameter(torch.from_numpy(st[key].copy()))
        setattr(model, attr, params[key])
    mlps = types.SimpleNamespace()
    for key, attr in (("fc1_w", "fc1_weights"), ("fc1_b", "fc1_bias"), ("fc2_w", "fc2_weights"),
                      ("fc2_b", "fc2_bias")):
        params[key] = nn.Parameter(torch.from_numpy(st[key].copy()))
        setattr(mlps, attr, params[key])
    model._emission_mlps = mlps
    groups = [("centre", "centre"), ("scaling", "log_scale"), ("rotation", "rotation"), ("opacity", "opacity"),
              ("emission_fc1_weights", "fc1_w"), ("emission_fc1_bias", "fc1_b"),
              ("emission_fc2_weights", "fc2_w"), ("emission_fc2_bias", "fc2_b")]
    opt = torch.optim.Adam([{"params": [params[k]], "lr": 1e-3, "name": g} for g, k in groups], eps=1e-15)
    for g, k in groups:
        opt.state[params[k]] = {"step": torch.tensor(3.0), "exp_avg": torch.from_numpy(m1[k].copy()),
                                "exp_avg_sq": torch.from_numpy(m2[k].copy())}
    model.optimizer = opt
    model.centre_gradient_accum = torch.from_numpy(accum.copy())
    model.denom = torch.from_numpy(denom.copy())
    model.max_radii2D = torch.from_numpy(max_radii.copy())
    smin = torch.tensor([-4.5, 0.2, -3.5]) if box else None
    smax = torch.tensor([4.5, 2.8, 3.5]) if box else None
    drawn = []
    gen = torch.Generator().manual_seed(1000 + seed)
    orig_normal = torch.normal

    def normal(*a, **k):
        out = orig_normal(*a, **dict(k, generator=gen))
        drawn.append(out.detach().clone())
        return out
    torch.normal = normal
    try:
        with _CpuZeros():
            model.densify_and_prune(max_grad, min_op, extent, mss, torch.from_numpy(radii.copy()),
                                    scene_min=smin, scene_max=smax)
    finally:
        torch.normal = orig_normal
    res = {}
    for g, k in groups:
        p = opt.param_groups[[x["name"] for x in opt.param_groups].index(g)]["params"][0]
        s = opt.state[p]
        res[k] = p.detach().numpy().copy()
        res["m1_" + k] = s["exp_avg"].numpy().copy()
        res["m2_" + k] = s["exp_avg_sq"].numpy().copy()
    # the per-Gaussian groups in full; the emission-MLP rows (copies of input
    # rows) as the input row each output row equals, their moments as that
    # row or -1 for zeros (a new Gaussian)
    out = {k: v for k, v in res.items() if not any(k.endswith(m) for m in ("fc1_w", "fc1_b", "fc2_w", "fc2_b"))}
    def match(new, old, allow_zero):
        idx = np.full(new.shape[0], -2, np.int32)
        lut = {old[i].tobytes(): i for i in range(old.shape[0])}
        for j in range(new.shape[0]):
            if allow_zero and not new[j].any():
                idx[j] = -1
            else:
                idx[j] = lut.get(new[j].tobytes(), -2)
        assert (idx >= -1).all()
        return idx
    cat = lambda d, pre: np.concatenate([d[pre + q].reshape(d[pre + q].shape[0], -1)
                                         for q in ("fc1_w", "fc1_b", "fc2_w", "fc2_b")], 1)
    out["mlp_src"] = match(cat(res, ""), cat(st, ""), False)
    out["mlp_m1_src"] = match(cat(res, "m1_"), cat({("m1_" + k): v for k, v in m1.items()}, "m1_"), True)
    out["mlp_m2_src"] = match(cat(res, "m2_"), cat({("m2_" + k): v for k, v in m2.items()}, "m2_"), True)
    out["split_samples"] = drawn[0].numpy().copy() if drawn else np.zeros((0, 3), np.float32)
    out["accum"] = model.centre_gradient_accum.numpy().copy()
    out["max_radii2D"] = model.max_radii2D.numpy().copy()
    return out


def _train_functions(ref):
    """calculate_psnr / calculate_rssi / calculate_mae from train.py's source."""
    import torch
    src = open(os.path.join(ref, "train.py")).read()
    tree = ast.parse(src)
    keep = [n for n in tree.body if isinstance(n, ast.FunctionDef)
            and n.name in ("calculate_psnr", "calculate_rssi", "calculate_mae")]
    ns = {"torch": torch}
    exec(compile(ast.Module(body=keep, type_ignores=[]), "train.py", "exec"), ns)
    return ns["calculate_psnr"], ns["calculate_rssi"], ns["calculate_mae"]


def run_eval(gaussian, utils, ref, case):
    import torch
    name, R, seed = case
    pred, tgt, rx, conf = eval_inputs(R, seed)
    psnr_f, rssi_f, mae_f = _train_functions(ref)
    orig_to = torch.nn.Module.to
    torch.nn.Module.to = lambda self, *a, **k: self     # ConfidenceMLP.__init__ moves itself to "cuda"
    try:
        cm = gaussian.ConfidenceMLP(CONF_HIDDEN)
    finally:
        torch.nn.Module.to = orig_to
    with torch.no_grad():
        off = 0
        for prm in cm.parameters():
            n = prm.numel()
            prm.copy_(torch.from_numpy(conf[off:off + n]).view_as(prm))
            off += n
    lambda1 = 0.2
    rows = []
    with torch.no_grad():
        for r in range(R):
            p = torch.from_numpy(pred[r])
            t = torch.from_numpy(tgt[r])
            psnr = psnr_f(p, t).item()
            rssi_diff = (rssi_f(p) - rssi_f(t)).item()
            mae = mae_f(p, t).item()
            ssim_val = utils.ssim(p, t).item()
            c = cm(torch.from_numpy(rx[r])).item()
            loss = ((1.0 - lambda1) * utils.l1_loss(p, t) + lambda1 * (1.0 - ssim_val)).item()
            rows.append([psnr, rssi_diff, mae, ssim_val, c, loss])
    return np.array(rows, dtype=np.float64)


def main(out_path):
    from oracle.build_ref import REF_ROOT
    gaussian, utils = _import_reference(REF_ROOT)
    out = {}
    for case in DENSIFY_CASES:
        for k, v in run_densify(gaussian, case).items():
            out[case[0] + "/" + k] = v
        print(case[0], "P", case[1], "->", out[case[0] + "/centre"].shape[0])
    for case in EVAL_CASES:
        out[case[0] + "/metrics"] = run_eval(gaussian, utils, REF_ROOT, case)
    np.savez_compressed(out_path, **out)
    print("wrote", out_path, os.path.getsize(out_path), "bytes")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.path.join(HERE, "densify_eval_golden.npz"))
