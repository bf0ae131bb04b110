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
