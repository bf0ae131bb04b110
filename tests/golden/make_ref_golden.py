"""Records golden vectors from the reference extensions themselves.

Runs on a GPU box with the reference rasterizer and fused-ssim built from
their own sources by oracle/build_ref.py (oracle/_ref/*.so).  For seeded
synthetic scenes it calls the reference's pybind entry points
(rasterize_gaussians / rasterize_gaussians_backward / fusedssim /
fusedssim_backward), decodes the intermediate arrays from the byte arenas
the reference returns, and writes everything to an .npz:

    python tests/golden/make_ref_golden.py OUT.npz

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
        p = name + "/"
        out[p + "num_rendered"] = np.int64(K)
        out[p + "radii"] = radii.cpu().numpy()
        out[p + "out_real"] = o_r.cpu().numpy()
        out[p + "out_imag"] = o_i.cpu().numpy()
        out[p + "depth"] = np.where(vis, _take(gbuf, geo["depths"]), 0).astype(np.float32)
        out[p + "means2D"] = np.where(vis[:, None], _take(gbuf, geo["means2D"]).reshape(P, 2), 0).astype(np.float32)
        out[p + "conic_opacity"] = np.where(vis[:, None], _take(gbuf, geo["conic_opacity"]).reshape(P, 4),
                                            0).astype(np.float32)
        out[p + "signal"] = np.where(vis[:, None], np.stack([_take(gbuf, geo["sig_r"]), _take(gbuf, geo["sig_i"])], 1),
                                     0).astype(np.float32)
        out[p + "cov3D"] = _take(gbuf, geo["cov3D"]).reshape(P, 6)
        out[p + "final_T"] = _take(ibuf, img["final_T"]).reshape(H, W)
        out[p + "n_contrib"] = _take(ibuf, img["n_contrib"]).reshape(H, W)
        T = ((W + 15) // 16) * ((H + 15) // 16)
        out[p + "ranges"] = _take(ibuf, img["ranges"]).reshape(H * W, 2)[:T]
        out[p + "values"] = _take(bbuf, binc["values"])
        out[p + "keys"] = _take(bbuf, binc["keys"])
        gr, gi = case_dL()
        bargs = (args[0], args[1], radii, o_r, o_i, args[2], args[3], args[4], 1.0, args[8], args[9], t(gr), t(gi),
                 args[10], args[11], gb, K, bb, ib)
        g2, g3, gmlp, gop, gcov, gsc, grot = ref_r.rasterize_gaussians_backward(*bargs)
        torch.cuda.synchronize()
        out[p + "dL_dmeans2D"] = g2.cpu().numpy()
        out[p + "dL_dmeans3D"] = g3.cpu().numpy()
        out[p + "dL_dopacity"] = gop.cpu().numpy()
        out[p + "dL_dcov3D"] = gcov.cpu().numpy()
        out[p + "dL_dscales"] = gsc.cpu().numpy()
        out[p + "dL_drotations"] = grot.cpu().numpy()
        if keep_mlp:
            out[p + "dL_dmlp"] = gmlp.cpu().numpy()
        print(name, "P", P, "K", K, "visible", int(vis.sum()))
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
    main(sys.argv[1] if len(sys.argv) > 1 else os.path.join(HERE, "raster_ref_golden.npz"))
