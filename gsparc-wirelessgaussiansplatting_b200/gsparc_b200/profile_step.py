"""Eager training steps of ``FusedTrainer`` for profiler captures.

    python -m gsparc_b200.profile_step [--P 20000] [--R 1] [--steps 3] [--cap 160000]

Builds the seeded synthetic scene of the benchmark (``scenes.make_scene``), a
``FusedTrainer`` with a fixed binning capacity per receiver, and runs
``--steps`` eager steps (no CUDA graph, so a profiler sees every launch on its
own).  Targets are random spectra; the run prints K and the last loss.
"""
from __future__ import annotations

import argparse

import numpy as np
import torch

from . import scenes
from .autograd import RasterPlan
from .fused import FusedTrainer


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--P", type=int, default=20000)
    ap.add_argument("--R", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--cap", type=int, default=160000, help="binning capacity per receiver")
    a = ap.parse_args(argv)
    dev = torch.device("cuda")
    sc = scenes.make_scene(a.P, scenes.SEED_SCENE)
    rxs = scenes.make_receivers(a.R)
    views = scenes.view_matrices(rxs)
    t = lambda x: torch.tensor(np.ascontiguousarray(x), dtype=torch.float32, device=dev)
    gen = torch.Generator().manual_seed(1)
    targets = torch.rand((a.R, scenes.H, scenes.W), generator=gen).to(dev)
    tr = FusedTrainer(sc, device=dev)
    tr.plan = RasterPlan(a.P, a.R, scenes.H, scenes.W, a.cap * a.R, dev)
    tx = t(scenes.TX_POS)
    loss = None
    for _ in range(a.steps):
        loss = tr.step_eager(t(views), t(rxs), tx, targets)
    torch.cuda.synchronize()
    tr.plan.record_status()
    torch.cuda.synchronize()
    print("K", tr.plan.check(), "loss", float(loss))


if __name__ == "__main__":
    main()
