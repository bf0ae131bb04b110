"""Records golden vectors from the reference extensions themselves.

Runs on a GPU box with the reference rasterizer and fused-ssim built from
their own sources by oracle/build_ref.py (oracle/_ref/*.so).  For seeded
synthetic scenes it calls the reference's pybind entry points
(rasterize_gaussians / rasterize_gaussians_backward / fusedssim /
fusedssim_backward), decodes the intermediate arrays from the byte arenas
the reference returns, and writes everything to an .npz:

    python tests/golden/make_ref_golden.py OUT.npz           (the small cases, full arrays)
    python tests/golden/make_ref_golden.py --large OUT.npz   (the bench-size cases, digests)

The arena decoding follows the reference's carving: every sub-array starts
at the next 128-byte boundary (rasterizer_impl.h:22-28) in the order of
GeometryState / ImageState / BinningState::fromChunk (rasterizer_impl.cu:60-100).
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "gsparc-wirelessgaussiansplatting_b200"))
sys.path.insert(0, ROOT)

# (name, P, scene seed, receiver seed, cluster fraction, keep MLP grads)
CASES = [
    ("p1", 1, 1, 41, 0.0, True),
    ("p17", 17, 2, 42, 0.0, True),
    ("p512", 512, 3, 33, 0.0, True),
    ("cl2000", 2000, 11, 12, 0.3, False),
    ("cfg0", 4096, 0, 2, 0.0, False),
]
# bench-size cases (name, P, scene seed, receiver seed, cluster fraction): the
# 20,000-Gaussian training scene of the per-receiver workload and one receiver
# of the 50,000-Gaussian clustered scene; recorded as digests and sketches
# into raster_ref_golden_large.npz
LARGE_CASES = [
    ("cfg1", 20000, 0, 2, 0.0),
    ("cfg2r", 50000, 0, 2, 0.3),
]
DIGESTED = ("values", "keys", "radii", "depth", "means2D", "conic_opacity", "signal", "n_contrib", "final_T",
            "out_real", "out_imag")
GRADS = ("dL_dmeans2D", "dL_dmeans3D", "dL_dopacity", "dL_dcov3D", "dL_dscales", "dL_drotations")
SKETCH_BUCKETS, SKETCH_SEED = 4096, 77
DL_SEED = 1234
H, W = 90, 360


def _carve(spec):
    off, out = 0, {}
    for name, dt, n in spec:
        off = (off + 127) // 128 * 128
        out[name] = (off, np.dtype(dt), n)
        off += n * np.dtype(dt).itemsize
    return out


def _take(buf, entry):
    off, dt, n = entry
    return np.frombuffer(buf[off:off + n * dt.itemsize].tobytes(), dtype=dt).copy()


def case_inputs(P, seed, rx_seed, cluster):
    from gsparc_b200 import scenes
    sc = scenes.make_scene(P, seed=seed, cluster_frac=cluster)
    m, s, q, o = sc.activated()
    rx = scenes.make_receivers(1, seed=rx_seed)
    return dict(means=m, scales=s, rots=q, opac=o.reshape(P, 1), mlp=sc.mlp, view=scenes.view_matrix(rx[0]),
                tx=scenes.TX_POS, rx=rx[0])


def case_dL(seed=DL_SEED):
    rng = np.random.default_rng(seed)
    return rng.normal(size=(1, H, W)).astype(np.float32), rng.normal(size=(1, H, W)).astype(np.float32)


def record_case(ref_r, t, P, seed, rx_seed, cluster, keep_mlp, dev="cuda"):
    """Run the reference extension forward and backward on one seeded case;
    returns {name: array} of its outputs and decoded arena contents."""
    import torch
    x = case_inputs(P, seed, rx_seed, cluster)
    args = (t(x["means"]), t(x["mlp"]), t(x["opac"]), t(x["scales"]), t(x["rots"]), H, W, 1.0, t(x["view"]),
            torch.eye(4, device=dev), t(x["tx"]), t(x["rx"]))
    K, o_r, o_i, radii, gb, bb, ib = ref_r.rasterize_gaussians(*args)
    torch.cuda.synchronize()
    gbuf, bbuf, ibuf = gb.cpu().numpy(), bb.cpu().numpy(), ib.cpu().numpy()
    geo = _carve([("depths", "f4", P), ("clamped", "u1", 3 * P), ("radii", "i4", P), ("means2D", "f4", 2 * P),
                  ("cov3D", "f4", 6 * P), ("conic_opacity", "f4", 4 * P), ("sig_r", "f4", P), ("sig_i", "f4", P)])
    img = _carve([("final_T", "f4", H * W), ("n_contrib", "u4", H * W), ("ranges", "u4", 2 * H * W)])
    binc = _carve([("values", "u4", K), ("values_unsorted", "u4", K), ("keys", "u8", K)])
    vis = radii.cpu().numpy() > 0
    out = {}
    out["num_rendered"] = np.int64(K)
    out["radii"] = radii.cpu().numpy()
    out["out_real"] = o_r.cpu().numpy()
    out["out_imag"] = o_i.cpu().numpy()
    out["depth"] = np.where(vis, _take(gbuf, geo["depths"]), 0).astype(np.float32)
    out["means2D"] = np.where(vis[:, None], _take(gbuf, geo["means2D"]).reshape(P, 2), 0).astype(np.float32)
    out["conic_opacity"] = np.where(vis[:, None], _take(gbuf, geo["conic_opacity"]).reshape(P, 4),
                                    0).astype(np.float32)
    out["signal"] = np.where(vis[:, None], np.stack([_take(gbuf, geo["sig_r"]), _take(gbuf, geo["sig_i"])], 1),
                             0).astype(np.float32)
    out["cov3D"] = _take(gbuf, geo["cov3D"]).reshape(P, 6)
    out["final_T"] = _take(ibuf, img["final_T"]).reshape(H, W)
    out["n_contrib"] = _take(ibuf, img["n_contrib"]).reshape(H, W)
    T = ((W + 15) // 16) * ((H + 15) // 16)
    out["ranges"] = _take(ibuf, img["ranges"]).reshape(H * W, 2)[:T]
    out["values"] = _take(bbuf, binc["values"])
    out["keys"] = _take(bbuf, binc["keys"])
    gr, gi = case_dL()
    bargs = (args[0], args[1], radii, o_r, o_i, args[2], args[3], args[4], 1.0, args[8], args[9], t(gr), t(gi),
             args[10], args[11], gb, K, bb, ib)
    g2, g3, gmlp, gop, gcov, gsc, grot = ref_r.rasterize_gaussians_backward(*bargs)
    torch.cuda.synchronize()
    out["dL_dmeans2D"] = g2.cpu().numpy()
    out["dL_dmeans3D"] = g3.cpu().numpy()
    out["dL_dopacity"] = gop.cpu().numpy()
    out["dL_dcov3D"] = gcov.cpu().numpy()
    out["dL_dscales"] = gsc.cpu().numpy()
    out["dL_drotations"] = grot.cpu().numpy()
    if keep_mlp:
        out["dL_dmlp"] = gmlp.cpu().numpy()
    print("P", P, "K", K, "visible", int(vis.sum()))
    return out


def digest(a) -> str:
    """SHA-256 of an array's bytes (C order): the bit-exact fingerprint the
    bench-size fixtures store instead of the arrays themselves."""
    import hashlib
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def sketch(v, m=SKETCH_BUCKETS, seed=SKETCH_SEED):
    """Count-sketch of a flat float vector into m buckets (bucket and sign of
    element i drawn from a seeded generator): a linear map whose output norm
    estimates the input's, so ||sketch(a) - sketch(b)|| estimates ||a - b||
    to a few per cent without storing a or b (float64 sums)."""
    v = np.asarray(v, dtype=np.float64).reshape(-1)
    rng = np.random.default_rng(seed + v.size)
    bucket = rng.integers(0, m, size=v.size)
    sign = rng.integers(0, 2, size=v.size) * 2.0 - 1.0
    return np.bincount(bucket, weights=sign * v, minlength=m)


def main_large(out_path):
    """The bench-size cases: bit-exact arrays as SHA-256 digests, gradients as
    count-sketches with their norms, small arrays (ranges, radii) in full."""
    import torch
    from oracle.build_ref import load_ref
    ref_r, _ = load_ref()
    if ref_r is None:
        raise SystemExit("reference extensions not built (run oracle/build_ref.py where the sources exist)")
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to("cuda")
    out = {}
    for name, P, seed, rx_seed, cluster in LARGE_CASES:
        r = record_case(ref_r, t, P, seed, rx_seed, cluster, False)
        p = name + "/"
        out[p + "num_rendered"] = r["num_rendered"]
        out[p + "radii"] = r["radii"]
        out[p + "ranges"] = r["ranges"]
        for k in DIGESTED:
            out[p + "sha256_" + k] = np.array(digest(r[k]))
        for k in GRADS:
            out[p + "sketch_" + k] = sketch(r[k])
            out[p + "norm_" + k] = np.float64(np.linalg.norm(r[k].astype(np.float64)))
    np.savez_compressed(out_path, **out)
    print("wrote", out_path, os.path.getsize(out_path), "bytes")


def main(out_path):
    import torch
    from oracle.build_ref import load_ref
    ref_r, ref_s = load_ref()
    if ref_r is None or ref_s is None:
        raise SystemExit("reference extensions not built (run oracle/build_ref.py where the sources exist)")
    dev = "cuda"
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    out = {}
    for name, P, seed, rx_seed, cluster, keep_mlp in CASES:
        r = record_case(ref_r, t, P, seed, rx_seed, cluster, keep_mlp, dev)
        for k, v in r.items():
            out[name + "/" + k] = v
    # fused-ssim on the blobs golden pair, train mode, with dL/dmap = 1/N
    sys.path.insert(0, HERE)
    import make_golden as mg
    a, b = mg.golden_inputs((90, 360), "blobs", 11)
    x, y = t(a)[None, None], t(b)[None, None]
    C1, C2 = 0.01 ** 2, 0.03 ** 2
    m, d1, d2, d3 = ref_s.fusedssim(C1, C2, x, y, True)
    dl = torch.full_like(x, 1.0 / x.numel())
    g = ref_s.fusedssim_backward(C1, C2, x, y, dl, d1, d2, d3)
    out["ssim/map"] = m.cpu().numpy()
    out["ssim/dm_dmu1"] = d1.cpu().numpy()
    out["ssim/dm_dsigma1_sq"] = d2.cpu().numpy()
    out["ssim/dm_dsigma12"] = d3.cpu().numpy()
    out["ssim/grad"] = g.cpu().numpy()
    np.savez_compressed(out_path, **out)
    print("wrote", out_path, os.path.getsize(out_path), "bytes")


if __name__ == "__main__":
    if len(sys.argv) > 1 and sys.argv[1] == "--large":
        main_large(sys.argv[2] if len(sys.argv) > 2 else os.path.join(HERE, "raster_ref_golden_large.npz"))
    else:
        main(sys.argv[1] if len(sys.argv) > 1 else os.path.join(HERE, "raster_ref_golden.npz"))
