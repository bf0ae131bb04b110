"""Benchmark of the GSpaRC training step on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload (one "step"): the per-receiver training step of train.py:364-566 on
the 20,000-Gaussian synthetic scene -- forward render of one 90x360
spectrum (preprocess, binning, sort, blend), L1 + fused SSIM + confidence
loss, the full hand-written adjoint, Adam.  Each step uses the next receiver
of a pool; targets are spectra of a second seeded scene at those receivers.
Synthetic data (no dataset in the container).

value: steps/s of the 20,000-Gaussian training workload (shared emission MLP 2x64 ReLU,
FP32, one receiver per step) captured in one CUDA graph (FusedTrainer: flat
training state, fused L1+SSIM+confidence loss, fused activation-adjoint
Adam; every launch one of this library's kernels) with inputs resident in
HBM; per-step CUDA events on the compute stream, L2 flushed (256 MiB write)
between steps outside the events.
e2e: the same step through FusedTrainer.step with the receiver's target
spectrum, view matrix and position copied from pinned host memory and the
loss copied back to pinned host memory every step, inside the step's events;
the host reads each step's loss and the rasterizer status while the next
step runs (the last one after the loop), as a training loop that logs every
loss does.
cfg2_batched_clustered_autotuned: the clustered batched workload (50,000 Gaussians, 30% in five
clusters, 64 receivers per step, shared 2x64 ReLU MLP, FP32): the tile shape
picked by FusedTrainer.autotune_tile from {16x16, 8x32, 32x8} (graph replays
timed per shape), then spectra/s of the captured step at that shape.
cfg3_batched_bf16_vs_plain_fp32: the 200,000-Gaussian workload's model (200,000 Gaussians,
shared MLP 3x128 GELU): the training step with 32 receivers per step and the
MLP in BF16 on the tcgen05 tensor cores, against the plain per-receiver FP32
step, in spectra/s, with the SSIM difference of their renders.
Also reported: the same step with the reference's per-Gaussian emission MLPs,
the eager drop-in path (reference call surface), a 16-receiver batched step,
16-receiver inference with the evaluation metrics of train.py:672-701
(forward-only render + one batched metrics launch), and per-kernel device times (eager runs of the same step; graph replays
bypass the library's event hooks).
N > 1: one process per GPU (torchrun), receivers sharded, Gaussians
replicated, gradients all-reduced over NCCL every step (weak scaling).
cfg4_multichannel: 100,000 Gaussians, 16 receivers x 64 frequency channels per
step: the shared MLP's 64 outputs (BF16 on the tensor cores) are the
amplitudes of a 64-channel FP32 blend,
the loss runs over the 1,024 spectra; spectra/s of the graph-captured step.
--impl reference: the CPU restatement of the same step (oracle/) on the
host, rank 0 only.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "gsparc-wirelessgaussiansplatting_b200")
sys.path.insert(0, PKG)
sys.path.insert(0, ROOT)

METRIC = "train steps/s & spectra/s on 1 B200: batched BF16 vs plain FP32, ΔSSIM≤1e-3"
UNIT = "train steps/s"
P_GAUSS = 20000
POOL = 16
SHARED_CFG1 = dict(layers=2, width=64, act="relu")    # emission MLP of configs 0-1
SHARED_CFG3 = dict(layers=3, width=128, act="gelu")   # emission MLP of config 3
P_CFG2, R_CFG2 = 50000, 64
P_CFG3, R_CFG3 = 200000, 32
P_CFG4, R_CFG4, C_CFG4 = 100000, 16, 64
SHARED_CFG4 = dict(layers=3, width=128, act="gelu", out=C_CFG4, precision="bf16")   # 64 amplitudes, one per bin
WORKLOAD = ("cfg1_train_20k: per-receiver training step (forward + L1/SSIM/confidence loss + hand-written adjoint "
            "+ Adam), P=20000 Gaussians uniform in a 10x8x3 m room, one 90x360 spectrum per step, 16x16 tiles, "
            "shared emission MLP 2x64 ReLU from [position PE, rx-relative direction, 1/d^2] to 1 amplitude, FP32")


def _peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def _traffic_per_launch():
    """DRAM bytes per launch recorded from ncu captures (profiles/traffic_per_launch.txt)."""
    out = {}
    try:
        with open(os.path.join(ROOT, "profiles", "traffic_per_launch.txt")) as f:
            for line in f:
                parts = line.split()
                if parts and not line.startswith("#") and len(parts) >= 2:
                    out[parts[0]] = int(parts[1])
    except OSError:
        pass
    return out


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during a timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.idx = gpu_index
        self.samples = []
        self._stop = threading.Event()
        self._t = None

    def _run(self):
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", f"--id={self.idx}", f"--query-gpu={self.FIELDS}",
                                      "--format=csv,noheader,nounits"], capture_output=True, text=True, timeout=5)
                for line in out.stdout.strip().splitlines():
                    self.samples.append([x.strip() for x in line.split(",")])
            except Exception:
                pass
            self._stop.wait(0.2)

    def __enter__(self):
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        self._t.join(timeout=10)

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for s in self.samples:
            try:
                sm.append(float(s[1]))
                mx = float(s[2])
                for n, v in zip(names, s[5:9]):
                    if v.strip().lower() == "active":
                        reasons.add(n)
            except Exception:
                continue
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def _dist_setup():
    import torch
    import torch.distributed as dist
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    group = None
    if world > 1:
        from datetime import timedelta
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=torch.device("cuda", local))
        group = dist.group.WORLD
    return world, rank, local, group


def _oracle_shared(spec):
    """(layers, width, act, flat params) of the shared MLP as FusedTrainer initialises it (seed 0)."""
    from gsparc_b200.shared_mlp import init_params_host
    return (spec["layers"], spec["width"], spec["act"], init_params_host(spec["layers"], spec["width"], 1, seed=0))


def run_reference(args):
    """CPU restatement of the step (oracle/train_step.py), timed on the host."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    import numpy as np
    from gsparc_b200 import scenes
    from oracle import raster as oraster
    from oracle.train_step import OracleTrainer
    sc = scenes.make_scene(P_GAUSS, scenes.SEED_SCENE)
    tg = scenes.make_scene(P_GAUSS, scenes.SEED_TARGET)
    rxs = scenes.make_receivers(POOL)
    tm, ts, tq, to = tg.activated()
    n_tgt = min(POOL, args.warmup + args.steps)
    targets = [oraster.render(tm, ts, tq, to, tg.mlp, scenes.view_matrix(rxs[i]), scenes.TX_POS, rxs[i], 90,
                              360)["out"][0] for i in range(n_tgt)]
    tr = OracleTrainer(sc, shared=_oracle_shared(SHARED_CFG1))
    # bounded sample: at most ~150 s of timed CPU work
    for i in range(min(args.warmup, 1)):
        tr.step(scenes.view_matrix(rxs[i % n_tgt]), rxs[i % n_tgt], scenes.TX_POS, targets[i % n_tgt])
    times = []
    budget = 150.0
    for i in range(args.steps):
        j = i % n_tgt
        t0 = time.perf_counter()
        tr.step(scenes.view_matrix(rxs[j]), rxs[j], scenes.TX_POS, targets[j])
        times.append(time.perf_counter() - t0)
        if sum(times) > budget:
            break
    v = len(times) / sum(times)
    ncores = int(os.environ.get("OMP_NUM_THREADS", "0")) or 1
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus,
            "steps": len(times), "warmup": min(args.warmup, 1), "ms_per_step": 1000.0 / v,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": WORKLOAD, "gaussians": P_GAUSS, "receivers_per_step": 1, "spectrum": "90x360",
                       "implementation": "CPU restatement of the same step (oracle/train_step.py with "
                                         "oracle/shared_mlp.py, numpy)"},
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": ncores, "kind": "port",
                             "sample": f"{len(times)} of {args.steps} requested steps (capped at {budget:.0f} s)"},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


def _scene_data(P, n_rx, dev, cluster_frac=0.0):
    """Seeded scene, receivers, views and target spectra (a second seeded scene) on the device."""
    import numpy as np
    import torch
    from gsparc_b200 import raster, scenes
    sc = scenes.make_scene(P, scenes.SEED_SCENE, cluster_frac=cluster_frac)
    tg = scenes.make_scene(P, scenes.SEED_TARGET, cluster_frac=cluster_frac)
    rxs = scenes.make_receivers(n_rx)
    views = scenes.view_matrices(rxs)
    t = lambda a: torch.tensor(np.ascontiguousarray(a), dtype=torch.float32, device=dev)
    tm, ts, tq, to = tg.activated()
    with torch.no_grad():
        targets, _, _, _ = raster.forward(t(tm), t(tg.mlp), t(to.reshape(-1)), t(ts), t(tq), 90, 360, 1.0, t(views),
                                          t(scenes.TX_POS), t(rxs))
    return dict(scene=sc, rxs=rxs, views=views, views_d=t(views), rxs_d=t(rxs), tx=t(scenes.TX_POS),
                targets_d=targets.contiguous())


def run_ours(args):
    import numpy as np
    import torch
    import torch.distributed as dist
    from gsparc_b200 import _lib, raster, scenes
    from gsparc_b200.fused import FusedTrainer
    from gsparc_b200.shared_mlp import SharedMLP
    from gsparc_b200.trainer import SplatTrainer

    world, rank, local, group = _dist_setup()
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    # receivers sharded over ranks
    d = _scene_data(P_GAUSS, POOL * world, dev)
    sc = d["scene"]
    sl = slice(rank * POOL, (rank + 1) * POOL)
    views, rxs = d["views"][sl], d["rxs"][sl]
    views_d, rxs_d, tx = d["views_d"][sl].contiguous(), d["rxs_d"][sl].contiguous(), d["tx"]
    targets_d = d["targets_d"][sl].contiguous()
    targets_h = targets_d.cpu().pin_memory()
    views_h = torch.tensor(views).pin_memory()
    rxs_h = torch.tensor(rxs).pin_memory()
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream(dev)

    def timed(fn, steps):
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
        if group is not None:
            dist.barrier()
        torch.cuda.synchronize()
        for i in range(steps):
            flush.zero_()                     # L2 flush outside the timed events
            evs[i][0].record(stream)
            fn(i)
            evs[i][1].record(stream)
        torch.cuda.synchronize()
        if group is not None:
            dist.barrier()
        tot = sum(a.elapsed_time(b) for a, b in evs) / 1000.0
        tt = torch.tensor([tot], dtype=torch.float64, device=dev)
        if group is not None:
            dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        return float(tt)

    # ---- the product path on the 20k workload: shared 2x64 ReLU MLP, FP32, one receiver per step, one CUDA graph
    trainer = FusedTrainer(sc, device=dev, group=group, shared=SharedMLP(**SHARED_CFG1))
    capacity = trainer.probe_capacity(views_d, rxs_d, tx)
    trainer.capture(1, capacity, tx, views_d[0:1], rxs_d[0:1], targets_d[0:1])

    def dev_step(i):
        j = i % POOL
        return trainer.step(views_d[j:j + 1], rxs_d[j:j + 1], targets_d[j:j + 1])

    loss_h = torch.empty(2, dtype=torch.float32).pin_memory()
    loss_done = [torch.cuda.Event(), torch.cuda.Event()]
    losses = []

    def host_step(i):
        # target spectrum, view matrix and receiver position copied from pinned
        # host memory into the graph's inputs, the loss copied back to pinned
        # memory, all on the stream inside the step's events; the host reads
        # step i's loss and the rasterizer status while step i + 1 runs (a
        # training loop that logs every loss), and the last one after the loop
        j = i % POOL
        loss = trainer.step(views_h[j:j + 1], rxs_h[j:j + 1], targets_h[j:j + 1])
        loss_h[i & 1].copy_(loss, non_blocking=True)
        loss_done[i & 1].record(stream)
        if i > 0:
            read_loss(i - 1)

    def read_loss(i):
        loss_done[i & 1].synchronize()
        trainer.plan.check()
        losses.append(float(loss_h[i & 1]))

    for i in range(args.warmup):
        dev_step(i)
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        sec = timed(dev_step, args.steps)
        while len(clk.samples) < 3:          # keep the GPU busy until the sampler has a few readings
            timed(dev_step, max(1, args.steps // 4))
    trainer.plan.check()                      # the capacity held for every timed step
    value = args.steps * world / sec
    n_warm = max(1, min(args.warmup, 3))
    for i in range(n_warm):
        host_step(i)
    read_loss(n_warm - 1)
    losses.clear()
    e2e_sec = timed(host_step, args.steps)
    read_loss(args.steps - 1)
    assert len(losses) == args.steps and all(math.isfinite(v) for v in losses)
    e2e = args.steps * world / e2e_sec
    h2d = (90 * 360 + 16 + 3) * 4
    # per-kernel device times from eager runs of the same step (graph replays
    # bypass the library's event hooks; the kernels and their work are the same)
    n_eager = max(1, min(args.steps, 50))
    for i in range(3):
        trainer.step_eager(views_d[i:i + 1], rxs_d[i:i + 1], tx, targets_d[i:i + 1])
    torch.cuda.synchronize()
    with _lib.KernelTimer() as kt:
        for i in range(n_eager):
            j = i % POOL
            trainer.step_eager(views_d[j:j + 1], rxs_d[j:j + 1], tx, targets_d[j:j + 1])
        torch.cuda.synchronize()
    ktimes = {k: v for k, v in kt.results().items() if v[1] > 0}
    # kernels per timed call (the depth sort is one cooperative launch at this size, the optimizer one)
    # (the one-receiver FP32 MLP adjoint runs the feature adjoint in the same launch)
    per_call = {"splat_loss_kernels": 2, "shared_mlp_forward_kernels": 1, "shared_mlp_backward_kernels": 1}
    launches = sum(c * per_call.get(k, 1) for k, (_, c) in ktimes.items()) // n_eager
    dom = max(ktimes, key=lambda k: ktimes[k][0])
    dom_ms = ktimes[dom][0] / ktimes[dom][1]
    with torch.no_grad():
        _, _, _, st = raster.forward(trainer.centre, None, trainer.act_opac, trainer.act_scales, trainer.act_rots,
                                     90, 360, 1.0, views_d[0], tx, rxs_d[0], shared=trainer.shared,
                                     shared_params=trainer.mlp)
    K = st.num_rendered
    vis = int((raster.state_views(st)["radii"] > 0).sum())
    npix = 90 * 360
    alg = {   # algorithmic bytes per launch (per-unit figures x the launch's units)
        "blend_backward_kernel": K * 36 + npix * 16 + vis * 40,
        "blend_forward_kernel": K * 36 + npix * 24,
        "preprocess_kernel": P_GAUSS * 44 + P_GAUSS * 76,
        "depth_sort_kernels": P_GAUSS * 16 * 4,
        "segment_place_kernel": K * 12 + 138 * 8,
        "scatter_kernel": vis * 24 + K * 4,
        "geometry_backward_kernel": vis * (12 + 40 + 24 + 24 + 24) + P_GAUSS * 64,
        "splat_loss_kernels": npix * (8 + 12) + npix * (8 + 12 + 4),
        "gaussian_adam_kernels": P_GAUSS * (11 * 4 * 7 + 8 * 4) + trainer.n_mlp * 4 * 7,
        # fused width-64 MLP: means, radii in; S, signal and both hidden layers' Z out
        "shared_mlp_forward_kernels": P_GAUSS * (12 + 4 + 4 + 8 + 2 * 64 * 4),
        # means, radii, S, dL/dsignal and Z in, dL/dx out; then dL/dx in, dL/dmeans out
        "shared_mlp_backward_kernels": P_GAUSS * (12 + 4 + 4 + 8 + 2 * 64 * 4 + 32 * 4) + P_GAUSS * (32 * 4 + 12 + 12),
    }
    peak, peak_kind = _peaks()
    achieved = alg.get(dom, 0) / (dom_ms / 1000.0) / 1e9
    traffic = _traffic_per_launch().get(dom)

    # ---- the reference's own emission model (per-Gaussian 3-32-2 MLPs) on the same step
    ref_tr = FusedTrainer(sc, device=dev, group=group)
    ref_tr.capture(1, capacity, tx, views_d[0:1], rxs_d[0:1], targets_d[0:1])
    n_ref = max(1, args.steps // 2)
    ref_sec = timed(lambda i: ref_tr.step(views_d[i % POOL:i % POOL + 1], rxs_d[i % POOL:i % POOL + 1],
                                          targets_d[i % POOL:i % POOL + 1]), n_ref)
    ref_tr.plan.check()
    del ref_tr
    # the eager drop-in path (reference call surface, instance-count readback per step)
    eager = SplatTrainer(sc, device=dev, group=group)

    def eager_step(i):
        j = i % POOL
        return eager.step(views_d[j], rxs_d[j], tx, targets_d[j])

    for i in range(3):
        eager_step(i)
    dropin = n_eager * world / timed(eager_step, n_eager)
    del eager
    # 16 receivers per step, same model
    btr = FusedTrainer(sc, device=dev, group=group, shared=SharedMLP(**SHARED_CFG1))
    btr.capture(POOL, capacity * POOL, tx, views_d, rxs_d, targets_d)
    n_b = max(1, args.steps // 4)
    bsec = timed(lambda i: btr.step(views_d, rxs_d, targets_d), n_b)
    btr.plan.check()
    batched16 = {"receivers_per_step": POOL, "steps_per_s": n_b * world / bsec,
                 "spectra_per_s": n_b * POOL * world / bsec}
    # inference: forward-only render of the 16 receivers and their batched
    # evaluation (PSNR, RSSI difference, MAE, SSIM, confidence, loss per spectrum)
    isec = timed(lambda i: btr.evaluate(views_d, rxs_d, tx, targets_d), n_b)
    btr.plan.check()
    inference16 = {"receivers_per_call": POOL, "spectra_per_s": n_b * POOL * world / isec,
                   "metrics": ["psnr", "rssi_diff", "mae", "ssim", "confidence", "loss"]}
    del btr

    # ---- 50,000 clustered Gaussians, 64 receivers per step, tile shape autotuned
    torch.cuda.empty_cache()
    d2 = _scene_data(P_CFG2, R_CFG2 * world, dev, cluster_frac=0.3)
    s2 = slice(rank * R_CFG2, (rank + 1) * R_CFG2)
    v2, r2, t2 = d2["views_d"][s2].contiguous(), d2["rxs_d"][s2].contiguous(), d2["targets_d"][s2].contiguous()
    tr2 = FusedTrainer(d2["scene"], device=dev, group=group, shared=SharedMLP(**SHARED_CFG1))
    tune = tr2.autotune_tile(tx, v2, r2, t2, steps=3)
    n2 = max(3, args.steps // 20)
    sec2 = timed(lambda i: tr2.step(v2, r2, t2), n2)
    K2, _ = tr2.plan.host_status()
    tr2.plan.check()
    cfg2 = {"workload": f"cfg2: P={P_CFG2} (30% in 5 N(c_k, 0.3 m) clusters), {R_CFG2} receivers per step, shared "
                        "emission MLP 2x64 ReLU, FP32, training step with adjoint, CUDA graph",
            "tile_ms_per_step": {f"{h}x{w}": ms for (h, w), ms in tune.items()},
            "tile": "%dx%d" % tr2.tile, "instances_K": K2,
            "steps_per_s": n2 * world / sec2, "spectra_per_s": n2 * R_CFG2 * world / sec2}
    del tr2, d2

    # ---- 200,000 Gaussians, 3x128 GELU: batched BF16 (tcgen05) vs the plain per-receiver FP32 path on the same GPU
    torch.cuda.empty_cache()
    d3 = _scene_data(P_CFG3, R_CFG3 * world, dev)
    s3 = slice(rank * R_CFG3, (rank + 1) * R_CFG3)
    v3, r3, t3 = d3["views_d"][s3].contiguous(), d3["rxs_d"][s3].contiguous(), d3["targets_d"][s3].contiguous()
    sc3 = d3["scene"]
    # SSIM of BF16 and FP32 renders of the same parameters against the targets
    from fused_ssim import fused_ssim
    with torch.no_grad():
        m3 = FusedTrainer(sc3, device=dev, shared=SharedMLP(**SHARED_CFG3, precision="fp32"))
        ssim_d = []
        for prec in ("fp32", "bf16"):
            out, _, _, _ = raster.forward(m3.centre, None, m3.act_opac, m3.act_scales, m3.act_rots, 90, 360, 1.0,
                                          v3[:4], tx, r3[:4], shared=SharedMLP(**SHARED_CFG3, precision=prec),
                                          shared_params=m3.mlp)
            ssim_d.append([float(fused_ssim(out[i][None, None], t3[i][None, None])) for i in range(4)])
        dssim = max(abs(a - b) for a, b in zip(*ssim_d))
        cap3 = m3.probe_capacity(v3, r3, tx)
        del m3
    plain = FusedTrainer(sc3, device=dev, group=group, shared=SharedMLP(**SHARED_CFG3, precision="fp32"))
    plain.capture(1, cap3, tx, v3[0:1], r3[0:1], t3[0:1])
    n_p = max(3, args.steps // 10)
    psec = timed(lambda i: plain.step(v3[i % R_CFG3:i % R_CFG3 + 1], r3[i % R_CFG3:i % R_CFG3 + 1],
                                      t3[i % R_CFG3:i % R_CFG3 + 1]), n_p)
    plain.plan.check()
    del plain
    torch.cuda.empty_cache()
    bf = FusedTrainer(sc3, device=dev, group=group, shared=SharedMLP(**SHARED_CFG3, precision="bf16"))
    bf.capture(R_CFG3, cap3 * R_CFG3, tx, v3, r3, t3)
    n_bf = max(3, args.steps // 20)
    bfsec = timed(lambda i: bf.step(v3, r3, t3), n_bf)
    bf.plan.check()
    del bf
    plain_sps = n_p * world / psec
    bf_sps = n_bf * R_CFG3 * world / bfsec
    cfg3 = {"workload": f"cfg3: P={P_CFG3}, shared emission MLP 3x128 GELU, 90x360, training step with adjoint",
            "plain_fp32": {"receivers_per_step": 1, "steps_per_s": plain_sps, "spectra_per_s": plain_sps},
            "batched_bf16": {"receivers_per_step": R_CFG3, "steps_per_s": n_bf * world / bfsec,
                             "spectra_per_s": bf_sps},
            "speedup_spectra_per_s": bf_sps / plain_sps,
            "delta_ssim_bf16_vs_fp32": dssim}

    # ---- 100,000 Gaussians, 16 receivers x 64 frequency bins per step (multi-channel render)
    del d3, sc3
    torch.cuda.empty_cache()
    sc4 = scenes.make_scene(P_CFG4, scenes.SEED_SCENE)
    tg4 = scenes.make_scene(P_CFG4, scenes.SEED_TARGET)
    rx4 = scenes.make_receivers(R_CFG4 * world)[rank * R_CFG4:(rank + 1) * R_CFG4]
    t = lambda a: torch.tensor(np.ascontiguousarray(a), dtype=torch.float32, device=dev)
    v4, r4 = t(scenes.view_matrices(rx4)), t(rx4)
    with torch.no_grad():   # targets: the second scene rendered through a seeded 64-output MLP
        tm, ts, tq, to = tg4.activated()
        tmlp = SharedMLP(**SHARED_CFG4)
        t4, _, _ = raster.forward_channels(t(tm), t(to.reshape(-1)), t(ts), t(tq), 90, 360, 1.0, v4, tx, r4, tmlp,
                                           tmlp.init_params(seed=7, device=dev))
        t4 = t4.clone()
        del tmlp
    tr4 = FusedTrainer(sc4, device=dev, group=group, shared=SharedMLP(**SHARED_CFG4))
    cap4 = tr4.probe_capacity(v4, r4, tx) * R_CFG4
    tr4.capture(R_CFG4, cap4, tx, v4, r4, t4)
    n4 = max(3, args.steps // 40)
    sec4 = timed(lambda i: tr4.step(v4, r4, t4), n4)
    K4, _ = tr4.plan.host_status()
    tr4.plan.check()
    cfg4 = {"workload": f"cfg4: P={P_CFG4}, {R_CFG4} receivers x {C_CFG4} frequency channels per step, shared "
                        "emission MLP 3x128 GELU -> 64 amplitudes (BF16 on tcgen05), multi-channel FP32 blend, loss over "
                        "R*C spectra, training step with adjoint, CUDA graph",
            "instances_K": K4, "steps_per_s": n4 * world / sec4,
            "spectra_per_s": n4 * R_CFG4 * C_CFG4 * world / sec4}
    del tr4
    torch.cuda.empty_cache()

    cpu_base = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        from oracle.train_step import OracleTrainer
        otr = OracleTrainer(sc, shared=_oracle_shared(SHARED_CFG1))
        tgt0 = targets_d[0].cpu().numpy()
        t0 = time.perf_counter()
        otr.step(views[0], rxs[0], scenes.TX_POS, tgt0)
        dt = time.perf_counter() - t0
        cpu_base = {"value": 1.0 / dt, "unit": UNIT, "cores": 1, "kind": "port",
                    "sample": "1 full training step of the same workload (numpy restatement, single thread)"}
    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": 1000.0 * sec / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": {"workload": WORKLOAD, "gaussians": P_GAUSS, "receivers_per_step": 1,
                           "spectrum": "90x360", "tiles": "16x16", "instances_K": K,
                           "l2": "flushed between steps (256 MiB write, outside the timed events)",
                           "parallelism": f"dp{world} (receivers sharded, gradients all-reduced)"},
                "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": 4},
                "gpu_launches": launches * args.steps,
                "clocks": clk.summary(),
                "roofline": {"kernel": dom, "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                             "frac": achieved / peak, "traffic": traffic, "peak_kind": peak_kind,
                             "avg_launch_ms": dom_ms, "algorithmic_bytes": alg.get(dom)},
                "kernel_ms_per_step": {k: v[0] / n_eager for k, v in sorted(ktimes.items())},
                "cfg2_batched_clustered_autotuned": cfg2,
                "cfg3_batched_bf16_vs_plain_fp32": cfg3,
                "cfg4_multichannel": cfg4,
                "reference_mlp_steps_per_s": n_ref * world / ref_sec,
                "dropin_eager_steps_per_s": dropin,
                "batched": batched16,
                "inference_eval": inference16,
                "path": "CUDA-graph-captured step (gsparc_b200.fused.FusedTrainer): flat training state, shared "
                        "emission MLP, fused L1+SSIM+confidence loss, fused activation-adjoint Adam; binning "
                        f"capacity {capacity}",
                "cpu_baseline": cpu_base}
        print(json.dumps(line))
    if group is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
