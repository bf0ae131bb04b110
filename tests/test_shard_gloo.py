"""Multi-process (gloo, world size 2, CPU) tests of the receiver-sharded
training step's host logic: receiver partitioning and the one-bucket
gradient all-reduce.  Each rank computes the oracle gradients of its own
receivers; after the all-reduce every rank holds the sum over all receivers,
which must equal a single-process sum."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from gsparc_b200.shard import allreduce_grads, shard_receivers


def test_shard_receivers_partitions():
    for R in (1, 5, 16, 17):
        for world in (1, 2, 3, 8):
            parts = [list(shard_receivers(R, r, world)) for r in range(world)]
            assert sum(parts, []) == list(range(R))
            sizes = [len(p) for p in parts]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        shard_receivers(4, 2, 2)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _oracle_grads(ridx):
    from gsparc_b200 import scenes
    from oracle import raster
    sc = scenes.make_scene(60, seed=5)
    m, s, q, o = sc.activated()
    rxs = scenes.make_receivers(4, seed=8)
    H, W = 18, 72
    tot = None
    for r in ridx:
        v = scenes.view_matrix(rxs[r])
        fwd = raster.render(m, s, q, o, sc.mlp, v, scenes.TX_POS, rxs[r], H, W)
        dL = np.random.default_rng(r).normal(size=(2, H, W)).astype(np.float32)
        g = raster.render_backward(fwd, m, s, q, o, sc.mlp, v, scenes.TX_POS, rxs[r], dL, H, W)
        vec = np.concatenate([g["dL_dmeans3D"].ravel(), g["dL_dscales"].ravel(), g["dL_dmlp"].ravel()])
        tot = vec if tot is None else tot + vec
    return tot


def _worker(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        mine = list(shard_receivers(4, rank, world))
        g = torch.from_numpy(_oracle_grads(mine))
        p = torch.nn.Parameter(torch.zeros_like(g))
        p.grad = g.clone()
        q = torch.nn.Parameter(torch.zeros(3))       # a parameter with no gradient on this rank
        n = allreduce_grads([p, q])
        out[rank] = (p.grad.numpy().copy(), q.grad.numpy().copy(), n)
    finally:
        dist.destroy_process_group()


def test_allreduce_grads_gloo_two_ranks():
    world = 2
    port = _free_port()
    manager = mp.Manager()
    out = manager.dict()
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=_worker, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=240)
        assert p.exitcode == 0
    full = _oracle_grads(range(4))
    for r in range(world):
        g, q, n = out[r]
        np.testing.assert_allclose(g, full, rtol=1e-5, atol=1e-6 * np.abs(full).max())
        assert np.all(q == 0) and n == full.size + 3


# ---- the product trainer's exchange steps (gsparc_b200.shard, as FusedTrainer calls them)

def _flat_worker(rank, world, port, out):
    """Each rank lays its receivers' oracle gradients into a flat buffer in
    FusedTrainer's state layout (centre | log-scale | quaternion | opacity |
    emission MLP | confidence MLP) and sums it over the ranks with
    shard.allreduce_flat, the call FusedTrainer's captured step makes."""
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from gsparc_b200.fused import state_layout
        from gsparc_b200.shard import allreduce_flat
        P, n_conf = 60, 5 * 32 + 1
        (oC, oS, oQ, oO, oM, oG), total = state_layout(P, 194 * P, n_conf)
        flat = torch.zeros(total, dtype=torch.float32)
        g = _oracle_grads(list(shard_receivers(4, rank, world)))
        flat[oC:oC + 3 * P] = torch.from_numpy(g[:3 * P])
        flat[oS:oS + 3 * P] = torch.from_numpy(g[3 * P:6 * P])
        flat[oM:oM + 194 * P] = torch.from_numpy(g[6 * P:])
        flat[oG:oG + n_conf] = float(rank + 1)          # confidence-MLP gradient: rank-dependent constant
        allreduce_flat(flat)
        out[rank] = flat.numpy().copy()
    finally:
        dist.destroy_process_group()


def test_fused_trainer_flat_allreduce_gloo_two_ranks():
    world = 2
    port = _free_port()
    out = mp.Manager().dict()
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=_flat_worker, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=240)
        assert p.exitcode == 0
    from gsparc_b200.fused import state_layout
    P, n_conf = 60, 5 * 32 + 1
    (oC, oS, oQ, oO, oM, oG), total = state_layout(P, 194 * P, n_conf)
    full = _oracle_grads(range(4))
    exp = np.zeros(total, np.float32)
    exp[oC:oC + 3 * P] = full[:3 * P]
    exp[oS:oS + 3 * P] = full[3 * P:6 * P]
    exp[oM:oM + 194 * P] = full[6 * P:]
    exp[oG:oG + n_conf] = 3.0
    for r in range(world):
        np.testing.assert_allclose(out[r], exp, rtol=1e-5, atol=1e-6 * np.abs(exp).max())
    np.testing.assert_array_equal(out[0], out[1])


def _densify_worker(rank, world, port, out):
    """Each rank holds the densification statistics of its own receivers;
    after shard.reduce_densify_stats every rank densifies (the oracle
    restatement of gaussian.py:515-542) from the same sums."""
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from gsparc_b200.shard import reduce_densify_stats
        from oracle import densify as od
        st, m1, m2, stats = _densify_case()
        acc, den, rad = (torch.from_numpy(a[rank].copy()) for a in stats)
        reduce_densify_stats(acc, den, rad)
        res = od.densify_and_prune(st, m1, m2, acc.numpy(), den.numpy(), max_grad=0.02, min_opacity=0.05,
                                   extent=4.0, seed=3)
        out[rank] = (res[0]["centre"].copy(), res[0]["mlp"].copy(), acc.numpy().copy(), rad.numpy().copy())
    finally:
        dist.destroy_process_group()


def _densify_case(P=200, world=2):
    rng = np.random.default_rng(21)
    st = dict(centre=rng.uniform(-3, 3, (P, 3)), log_scale=rng.normal(-2.5, 1.0, (P, 3)),
              rotation=rng.normal(size=(P, 4)), opacity=rng.normal(size=P), mlp=rng.normal(size=(P, 194)))
    m1 = {k: 0.01 * rng.normal(size=v.shape) for k, v in st.items()}
    m2 = {k: np.abs(0.001 * rng.normal(size=v.shape)) for k, v in st.items()}
    acc = np.abs(rng.normal(0, 0.03, (world, P))).astype(np.float32)     # per-rank statistics
    den = rng.integers(0, 3, (world, P)).astype(np.float32)
    rad = rng.uniform(0, 30, (world, P)).astype(np.float32)
    return st, m1, m2, (acc, den, rad)


def test_sharded_densify_agrees_across_ranks_gloo():
    world = 2
    port = _free_port()
    out = mp.Manager().dict()
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=_densify_worker, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=240)
        assert p.exitcode == 0
    from oracle import densify as od
    st, m1, m2, (acc, den, rad) = _densify_case()
    single = od.densify_and_prune(st, m1, m2, acc.sum(0), den.sum(0), max_grad=0.02, min_opacity=0.05,
                                  extent=4.0, seed=3)
    for r in range(world):
        c, mlp, a, mr = out[r]
        np.testing.assert_array_equal(a, acc.sum(0))
        np.testing.assert_array_equal(mr, rad.max(0))
        assert c.shape == single[0]["centre"].shape
        np.testing.assert_array_equal(c, single[0]["centre"])
        np.testing.assert_array_equal(mlp, single[0]["mlp"])
    assert out[0][0].shape[0] != st["centre"].shape[0]    # the case does clone / split / prune
