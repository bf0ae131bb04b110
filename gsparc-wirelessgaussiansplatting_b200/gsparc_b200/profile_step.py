"""Eager training steps of ``FusedTrainer`` for profiler captures.

    python -m gsparc_b200.profile_step [--P 20000] [--R 1] [--steps 3] [--cap 160000]
        [--mlp ref|relu64|gelu128|ch64] [--precision fp32|bf16] [--times]

Builds the seeded synthetic scene of the benchmark (``scenes.make_scene``), a
``FusedTrainer`` with a fixed binning capacity per receiver, and runs
``--steps`` eager steps (no CUDA graph, so a profiler sees every launch on its
own).  Targets are random spectra; the run prints K and the last loss, and
with ``--times`` the library's per-kernel device times of the last step.
``--mlp``: the per-Gaussian MLPs (ref), the shared MLP 2x64 ReLU / 3x128
GELU, or 3x128 GELU with 64 outputs for a 64-channel step (ch64).
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
    ap.add_argument("--mlp", choices=["ref", "relu64", "gelu128", "ch64"], default="ref")
    ap.add_argument("--precision", choices=["fp32", "bf16"], default="fp32")
    ap.add_argument("--times", action="store_true")
    a = ap.parse_args(argv)
    dev = torch.device("cuda")
    sc = scenes.make_scene(a.P, scenes.SEED_SCENE)
    rxs = scenes.make_receivers(a.R)
    views = scenes.view_matrices(rxs)
    t = lambda x: torch.tensor(np.ascontiguousarray(x), dtype=torch.float32, device=dev)
    gen = torch.Generator().manual_seed(1)
    from ._lib import KernelTimer
    from .shared_mlp import SharedMLP
    shared = {"ref": None, "relu64": SharedMLP(2, 64, "relu", precision=a.precision),
              "gelu128": SharedMLP(3, 128, "gelu", precision=a.precision),
              "ch64": SharedMLP(3, 128, "gelu", out=64, precision=a.precision)}[a.mlp]
    C = 1 if shared is None else shared.out
    targets = torch.rand((a.R, scenes.H, scenes.W) if C == 1 else (a.R, C, scenes.H, scenes.W), generator=gen).to(dev)
    tr = FusedTrainer(sc, device=dev, shared=shared)
    tr.plan = RasterPlan(a.P, a.R, scenes.H, scenes.W, a.cap * a.R, dev)
    tx = t(scenes.TX_POS)
    loss = None
    for _ in range(a.steps - 1):
        loss = tr.step_eager(t(views), t(rxs), tx, targets)
    torch.cuda.synchronize()
    with KernelTimer() as kt:
        loss = tr.step_eager(t(views), t(rxs), tx, targets)
        torch.cuda.synchronize()
    if a.times:
        for k, (ms, n) in sorted(kt.results().items(), key=lambda x: -x[1][0]):
            if n:
                print(f"  {k:32s} {1000 * ms:9.1f} us  ({n} calls)")
    tr.plan.record_status()
    torch.cuda.synchronize()
    print("K", tr.plan.check(), "loss", float(loss))


if __name__ == "__main__":
    main()
