"""Benchmark of the GSpaRC training step on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
    python bench.py --eager-steps S [--P P] [--R R] [--cap C] [--mlp ...] [--precision ...]

Headline workload (one "step"): the batched mixed-precision training step of
train.py:364-566 on 200,000 synthetic Gaussians (means uniform in a 10x3x8 m
room, log-scales N(-2, 0.5), quaternions normalise(N(0, I4)), opacity logits
N(0, 1)) with 32 receivers per step: forward render of 32 90x360 spectra
(preprocess, binning, depth order, blend), the shared emission MLP 3x128 GELU
in BF16 on the tcgen05 tensor cores with FP32 accumulation, L1 + fused SSIM +
confidence loss over the 32 spectra, the full hand-written adjoint, fused Adam;
blend, transmittance, sort keys and SSIM in FP32.  The step is captured in one
CUDA graph (FusedTrainer).  Targets are spectra of a second seeded scene;
steps alternate between two batches of 32 receivers.  Synthetic data (no
dataset in the container).

value: spectra/s of that step with inputs resident in HBM (per-step CUDA
events on the compute stream; L2 flushed by a 256 MiB write between steps,
outside the events; the step's own state is several GB, above L2).
e2e: the same step through FusedTrainer.step with each step's 32 target
spectra, view matrices and receiver positions copied from pinned host memory
and the loss copied back to pinned host memory, inside the step's events; the
host reads each step's loss and the rasterizer status while the next step runs.
plain_fp32: the same model and scene trained the plain way -- one receiver
per step, the emission MLP in FP32 -- on the same GPU; ``speedup_vs_plain_fp32``
is value / its spectra/s, ``delta_ssim_bf16_vs_fp32`` the largest SSIM
difference of BF16 and FP32 renders of the same parameters against the targets.
roofline: the dominant kernel of the step (the BF16 MLP adjoint): its
algorithmic FLOPs per launch / its CUDA-event time in eager runs of the same
step, against the measured sustained BF16 tensor peak.
Side lines (N = 1): the 20,000-Gaussian per-receiver FP32 step (cfg1), the
50,000-Gaussian clustered 64-receiver step with the autotuned tile (cfg2), the
64-channel step (cfg4), 16-receiver inference with the evaluation metrics,
and the reference CUDA extension (built from its own sources into oracle/_ref)
timed beside this library's drop-in modules on the reference's per-Gaussian
MLP model (forward, forward + backward, fused SSIM).
cpu_baseline / --impl reference: a multi-threaded CPU PyTorch rendition of the
same training step (oracle/torch_cpu.py), one receiver per step on the full
200,000-Gaussian scene, timed on the host cores (rank 0 only).
N > 1: one process per GPU (torchrun; started by bench.py itself when
WORLD_SIZE is unset), 32 receivers per rank, Gaussians replicated, the flat
gradient all-reduced over NCCL inside the captured step (weak scaling).
--eager-steps: eager steps of one FusedTrainer configuration (no graph, every
launch on its own) for profiler captures; prints K, the loss and with --times
the library's per-kernel device times.
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
UNIT = "spectra/s"
H, W = 90, 360
P_CFG1, POOL1 = 20000, 16
P_CFG2, R_CFG2 = 50000, 64
P_CFG3, R_CFG3, BATCHES3 = 200000, 32, 2
P_CFG4, R_CFG4, C_CFG4 = 100000, 16, 64
P_CFG0 = 4096
SHARED_CFG1 = dict(layers=2, width=64, act="relu")    # emission MLP of configs 0-2
SHARED_CFG3 = dict(layers=3, width=128, act="gelu")   # emission MLP of config 3
SHARED_CFG4 = dict(layers=3, width=128, act="gelu", out=C_CFG4, precision="bf16")   # 64 amplitudes, one per bin
WORKLOAD = ("cfg3_batched_bf16_200k: training step (forward + L1/SSIM/confidence loss + hand-written adjoint + "
            "Adam) with 32 receivers per step, P=200000 Gaussians uniform in a 10x3x8 m room, 32 90x360 spectra per "
            "step, 16x16 tiles, shared emission MLP 3x128 GELU from [position PE, rx-relative direction, 1/d^2] to 1 "
            "amplitude in BF16 on tcgen05 (FP32 accumulation), FP32 blend/transmittance/sort keys/SSIM, one CUDA graph")
# algorithmic FLOPs per (Gaussian, receiver) row of the 3x128 GELU MLP: 2 * (32*128 + 128*128 + 128*128 + 128)
MLP3_FWD_FLOP = 2 * (32 * 128 + 128 * 128 + 128 * 128 + 128)
MLP3_BWD_FLOP = 2 * MLP3_FWD_FLOP      # a weight-gradient and an input-gradient product per layer


def _peaks():
    """Roofline denominators: measured on this pool (MEASURED_PEAKS.json) or the fallback."""
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        hbm = float(d["hbm_gbs"])
        bf = float(d.get("bf16_tflops_sustained") or d["bf16_tflops"])
        return dict(hbm=hbm, bf16=bf, bf16_burst=float(d.get("bf16_tflops", bf)), kind="measured")
    except Exception:
        return dict(hbm=6650.0, bf16=1400.0, bf16_burst=1590.0, kind="fallback")


def _traffic_per_launch():
    """DRAM bytes per launch recorded from ncu captures (profiles/traffic_per_launch.txt)."""
    out = {}
    try:
        with open(os.path.join(ROOT, "profiles", "traffic_per_launch.txt")) as f:
            for line in f:
                parts = line.split()
                if parts and not line.startswith("#") and len(parts) >= 2:
                    out[parts[0]] = float(parts[1])
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


def _launch_ranks(args):
    """--gpus N > 1 without a launcher: start N ranks of this script with
    torch.distributed.run on 127.0.0.1 and return their exit status."""
    import socket
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={args.gpus}",
           "--master-addr", "127.0.0.1", "--master-port", str(port), os.path.abspath(__file__)] + sys.argv[1:]
    env = dict(os.environ, NCCL_DEBUG=os.environ.get("NCCL_DEBUG", "INFO"), NCCL_DEBUG_SUBSYS="INIT")
    return subprocess.call(cmd, env=env)


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


def _torch_cpu_trainer(threads):
    """The CPU PyTorch rendition of the headline step (oracle/torch_cpu.py) on
    the 200,000-Gaussian scene with the shared 3x128 GELU MLP (FP32), and the
    receivers / targets of the first batch.  Targets are FP32 renders of the
    second seeded scene by the same rendition."""
    import numpy as np
    import torch
    from gsparc_b200 import scenes
    from gsparc_b200.shared_mlp import init_params_host
    from oracle.torch_cpu import TorchCPUTrainer
    torch.set_num_threads(threads)
    sc = scenes.make_scene(P_CFG3, scenes.SEED_SCENE)
    tg = scenes.make_scene(P_CFG3, scenes.SEED_TARGET)
    rxs = scenes.make_receivers(R_CFG3)
    room = (torch.tensor(scenes.ROOM_LO, dtype=torch.float32), torch.tensor(scenes.ROOM_HI, dtype=torch.float32))
    spec = SHARED_CFG3
    tr = TorchCPUTrainer(sc, spec["layers"], spec["width"], spec["act"],
                         init_params_host(spec["layers"], spec["width"], 1, seed=0), room=room)
    ttr = TorchCPUTrainer(tg, spec["layers"], spec["width"], spec["act"],
                          init_params_host(spec["layers"], spec["width"], 1, seed=7))
    return tr, ttr, rxs, scenes.view_matrices(rxs)


def _cpu_steps(steps, budget_s, threads, warmup=1):
    """Time up to `steps` CPU training steps (one receiver each) within
    budget_s seconds of timed work; returns (spectra/s, steps timed, threads)."""
    import torch
    tr, ttr, rxs, views = _torch_cpu_trainer(threads)
    n = 4                  # steps cycle over the first four receivers of the batch
    targets = {}

    def target(j):
        if j not in targets:
            with torch.no_grad():
                targets[j] = ttr.render(torch.tensor(views[j]), torch.tensor(rxs[j])).clone()
        return targets[j]

    for i in range(warmup):
        tr.step(views[i % n], rxs[i % n], target(i % n))
    times = []
    for i in range(steps):
        j = (warmup + i) % n
        tg = target(j)
        t0 = time.perf_counter()
        tr.step(views[j], rxs[j], tg)
        times.append(time.perf_counter() - t0)
        if sum(times) > budget_s:
            break
    return len(times) / sum(times), len(times), torch.get_num_threads()


def run_reference(args):
    """The CPU PyTorch rendition of the same training step, timed on the host
    cores (rank 0 only; the other ranks exit without work)."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    threads = os.cpu_count() or 1
    budget = 150.0
    v, n, threads = _cpu_steps(args.steps, budget, threads, warmup=min(max(args.warmup, 1), 2))
    sample = (f"{n} of {args.steps} requested steps (capped at {budget:.0f} s of timed work); each step is one "
              f"receiver's training step on the full {P_CFG3}-Gaussian scene (a 1/{R_CFG3} share of the batched step "
              "plus a full Adam update)")
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus,
            "steps": n, "warmup": min(max(args.warmup, 1), 2), "ms_per_step": 1000.0 / v,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": WORKLOAD, "gaussians": P_CFG3, "receivers_per_step": 1,
                       "spectrum": "90x360", "same_config": True,
                       "implementation": "CPU PyTorch rendition of the same step (oracle/torch_cpu.py: vectorised "
                                         "preprocess, shared MLP in FP32, pair-wise blend with one stable sort, "
                                         "conv2d SSIM, autograd adjoint, torch.optim.Adam)"},
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": threads, "kind": "port", "port": "torch-cpu",
                             "sample": sample},
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
    targets = []
    with torch.no_grad():
        for s in range(0, n_rx, 32):
            e = min(n_rx, s + 32)
            out, _, _, _ = raster.forward(t(tm), t(tg.mlp), t(to.reshape(-1)), t(ts), t(tq), H, W, 1.0,
                                          t(views[s:e]), t(scenes.TX_POS), t(rxs[s:e]))
            targets.append(out.clone())
    return dict(scene=sc, rxs=rxs, views=views, views_d=t(views), rxs_d=t(rxs), tx=t(scenes.TX_POS),
                targets_d=torch.cat(targets).contiguous())


class _Timer:
    """Per-step CUDA events on the compute stream, an L2 flush between steps
    outside the events, barrier + synchronize on both sides, max over ranks."""

    def __init__(self, dev, group):
        import torch
        self.dev, self.group = dev, group
        self.flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
        self.stream = torch.cuda.current_stream(dev)

    def __call__(self, fn, steps):
        import torch
        import torch.distributed as dist
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
        if self.group is not None:
            dist.barrier()
        torch.cuda.synchronize()
        for i in range(steps):
            self.flush.zero_()
            evs[i][0].record(self.stream)
            fn(i)
            evs[i][1].record(self.stream)
        torch.cuda.synchronize()
        if self.group is not None:
            dist.barrier()
        tot = sum(a.elapsed_time(b) for a, b in evs) / 1000.0
        tt = torch.tensor([tot], dtype=torch.float64, device=self.dev)
        if self.group is not None:
            dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        return float(tt)


def _launches_per_step(kt_results, n_steps, P, R, capacity, tiles=138, sms=148):
    """Kernel launches per step from the library's per-call timing counts:
    the loss is two launches per call, the depth sort 1 or 4 (the library
    says which), the blend adjoint two when a one-CTA scan first numbers its
    multi-chunk work items (capacity / 64 + R x tiles >= 2 x 64 x SMs), every
    other timed call one launch."""
    from gsparc_b200 import _lib
    sort_n = int(_lib.lib().gsparc_depth_sort_launches(int(P), int(R)))
    per_call = {"splat_loss_kernels": 2, "depth_sort_kernels": sort_n,
                "blend_backward_kernel": 2 if capacity // 64 + R * tiles >= 2 * 64 * sms else 1}
    tot = sum(c * per_call.get(k, 1) for k, (_, c) in kt_results.items())
    return tot // max(n_steps, 1)


def _reference_extension_leg(dev, iters=200, warmup=20):
    """The reference CUDA extension (rasterize_gaussians / _backward, fusedssim /
    _backward, built from the reference's own sources into oracle/_ref) and
    this library's drop-in modules on the same inputs: the reference's
    per-Gaussian 3-32-2 MLP model, one receiver, cfg0 (4,096) and cfg1 (20,000
    Gaussians).  Median ms over `iters` CUDA-event-timed calls."""
    import numpy as np
    import torch
    import fused_ssim_cuda as ours_ssim
    import wireless_rasterizer as ours
    from gsparc_b200 import _lib, scenes
    from oracle.build_ref import load_ref
    ref_r, ref_s = load_ref()
    if ref_r is None or ref_s is None:
        return {"unavailable": "oracle/_ref not built (the reference sources were absent where build() ran)"}
    t = lambda a: torch.tensor(np.ascontiguousarray(a), dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream(dev)

    def med(fn):
        for _ in range(warmup):
            fn()
        torch.cuda.synchronize()
        ts = []
        for _ in range(iters):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            fn()
            b.record(stream)
            ts.append((a, b))
        torch.cuda.synchronize()
        return statistics.median(x.elapsed_time(y) for x, y in ts)

    res = {"timing": f"median of {iters} CUDA-event-timed calls after {warmup} warm-up calls, one receiver per call",
           "model": "the reference's per-Gaussian emission MLPs (3-32-2 leaky ReLU), FP32"}
    C1, C2 = 0.01 ** 2, 0.03 ** 2
    for name, P in (("cfg0", P_CFG0), ("cfg1", P_CFG1)):
        sc = scenes.make_scene(P, scenes.SEED_SCENE)
        m, s, q, o = sc.activated()
        rx = scenes.make_receivers(1)[0]
        args = (t(m), t(sc.mlp), t(o.reshape(P, 1)), t(s), t(q), H, W, 1.0, t(scenes.view_matrix(rx)),
                torch.eye(4, device=dev), t(scenes.TX_POS), t(rx))
        g = torch.Generator().manual_seed(3)
        dr = torch.randn((1, H, W), generator=g).to(dev)
        di = torch.zeros_like(dr)
        row = {}
        for label, mod in (("reference", ref_r), ("ours", ours)):
            def fwd():
                return mod.rasterize_gaussians(*args)

            def fwd_bwd():
                K, o_r, o_i, radii, gb, bb, ib = mod.rasterize_gaussians(*args)
                return mod.rasterize_gaussians_backward(args[0], args[1], radii, o_r, o_i, args[2], args[3], args[4],
                                                        1.0, args[8], args[9], dr, di, args[10], args[11], gb, K,
                                                        bb, ib)
            row[label] = {"forward_ms": med(fwd), "forward_backward_ms": med(fwd_bwd)}
        # this library's blend kernels inside the same calls (per-launch events)
        with _lib.KernelTimer() as kt:
            for _ in range(20):
                K, o_r, o_i, radii, gb, bb, ib = ours.rasterize_gaussians(*args)
            torch.cuda.synchronize()
        kr = kt.results()
        row["ours"]["blend_forward_kernel_ms"] = kr["blend_forward_kernel"][0] / max(kr["blend_forward_kernel"][1], 1)
        row["forward_speedup"] = row["reference"]["forward_ms"] / row["ours"]["forward_ms"]
        row["forward_backward_speedup"] = row["reference"]["forward_backward_ms"] / row["ours"]["forward_backward_ms"]
        res[name] = row
    img1 = torch.rand((1, 1, H, W), generator=torch.Generator().manual_seed(4)).to(dev)
    img2 = torch.rand((1, 1, H, W), generator=torch.Generator().manual_seed(5)).to(dev)
    dl = torch.full_like(img1, 1.0 / img1.numel())
    row = {}
    for label, mod in (("reference", ref_s), ("ours", ours_ssim)):
        def ss():
            mp, d1, d2, d3 = mod.fusedssim(C1, C2, img1, img2, True)
            return mod.fusedssim_backward(C1, C2, img1, img2, dl, d1, d2, d3)
        row[label] = {"ssim_forward_backward_ms": med(ss)}
    row["speedup"] = row["reference"]["ssim_forward_backward_ms"] / row["ours"]["ssim_forward_backward_ms"]
    res["fused_ssim_90x360"] = row
    return res


def run_ours(args):
    import numpy as np
    import torch
    from gsparc_b200 import _lib, raster, scenes
    from gsparc_b200.fused import FusedTrainer
    from gsparc_b200.shared_mlp import SharedMLP

    world, rank, local, group = _dist_setup()
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    timed = _Timer(dev, group)
    stream = timed.stream

    # ---- headline: 200,000 Gaussians, 32 receivers per step, BF16 MLP on tcgen05, one CUDA graph
    nb = R_CFG3 * BATCHES3
    d3 = _scene_data(P_CFG3, nb * world, dev)
    s3 = slice(rank * nb, (rank + 1) * nb)
    v3, r3, t3 = d3["views_d"][s3].contiguous(), d3["rxs_d"][s3].contiguous(), d3["targets_d"][s3].contiguous()
    tx, sc3 = d3["tx"], d3["scene"]
    batches = [(v3[b * R_CFG3:(b + 1) * R_CFG3], r3[b * R_CFG3:(b + 1) * R_CFG3], t3[b * R_CFG3:(b + 1) * R_CFG3])
               for b in range(BATCHES3)]
    # SSIM of BF16 and FP32 renders of the same parameters against the targets (first 4 receivers)
    from fused_ssim import fused_ssim
    with torch.no_grad():
        m3 = FusedTrainer(sc3, device=dev, shared=SharedMLP(**SHARED_CFG3, precision="fp32"))
        ssim_d = []
        for prec in ("fp32", "bf16"):
            out, _, _, _ = raster.forward(m3.centre, None, m3.act_opac, m3.act_scales, m3.act_rots, H, W, 1.0,
                                          v3[:4], tx, r3[:4], shared=SharedMLP(**SHARED_CFG3, precision=prec),
                                          shared_params=m3.mlp)
            ssim_d.append([float(fused_ssim(out[i][None, None], t3[i][None, None])) for i in range(4)])
        dssim = max(abs(a - b) for a, b in zip(*ssim_d))
        cap3 = m3.probe_capacity(v3, r3, tx)
        del m3
    torch.cuda.empty_cache()
    bf = FusedTrainer(sc3, device=dev, group=group, shared=SharedMLP(**SHARED_CFG3, precision="bf16"))
    bf.capture(R_CFG3, cap3 * R_CFG3, tx, *batches[0])

    def dev_step(i):
        return bf.step(*batches[i % BATCHES3])

    for i in range(max(args.warmup, 3)):
        dev_step(i)
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        sec = timed(dev_step, args.steps)
        while len(clk.samples) < 3:          # keep the GPU busy until the sampler has a few readings
            timed(dev_step, max(1, args.steps // 4))
    K3, _ = bf.plan.host_status()
    bf.plan.check()                           # the capacity held for every timed step
    value = args.steps * R_CFG3 * world / sec

    # e2e: the same step fed from pinned host memory, the loss read back every step
    host = [tuple(x.cpu().pin_memory() for x in b) for b in batches]
    loss_h = torch.empty(2, dtype=torch.float32).pin_memory()
    loss_done = [torch.cuda.Event(), torch.cuda.Event()]
    losses = []

    def read_loss(i):
        loss_done[i & 1].synchronize()
        bf.plan.check()
        losses.append(float(loss_h[i & 1]))

    def host_step(i):
        loss = bf.step(*host[i % BATCHES3])
        loss_h[i & 1].copy_(loss, non_blocking=True)
        loss_done[i & 1].record(stream)
        if i > 0:
            read_loss(i - 1)

    for i in range(3):
        host_step(i)
    read_loss(2)
    losses.clear()
    e2e_sec = timed(host_step, args.steps)
    read_loss(args.steps - 1)
    assert len(losses) == args.steps and all(math.isfinite(v) for v in losses)
    e2e = args.steps * R_CFG3 * world / e2e_sec
    h2d = R_CFG3 * (H * W + 16 + 3) * 4

    # per-kernel device times of the same step (eager: graph replays bypass the library's event hooks)
    n_eager = max(3, min(args.steps, 20))
    for i in range(2):
        bf.step_eager(*batches[i % BATCHES3][:2], tx, batches[i % BATCHES3][2])
    torch.cuda.synchronize()
    with _lib.KernelTimer() as kt:
        for i in range(n_eager):
            b = batches[i % BATCHES3]
            bf.step_eager(b[0], b[1], tx, b[2])
        torch.cuda.synchronize()
    ktimes = {k: v for k, v in kt.results().items() if v[1] > 0}
    launches = _launches_per_step(ktimes, n_eager, P_CFG3, R_CFG3, cap3 * R_CFG3,
                                  sms=torch.cuda.get_device_properties(dev).multi_processor_count)
    kms = {k: v[0] / n_eager for k, v in sorted(ktimes.items())}
    dom = max(ktimes, key=lambda k: ktimes[k][0])
    rows3 = P_CFG3 * R_CFG3
    flops = {"shared_mlp_backward_kernels": rows3 * MLP3_BWD_FLOP, "shared_mlp_forward_kernels": rows3 * MLP3_FWD_FLOP}
    peaks = _peaks()
    traffic = _traffic_per_launch()
    roof = {"kernel": dom}
    if dom in flops:
        dom_ms = ktimes[dom][0] / ktimes[dom][1]
        ach = flops[dom] / (dom_ms / 1000.0) / 1e12
        roof.update({"bound": "tensor", "achieved": ach, "peak": peaks["bf16"], "unit": "TFLOP/s",
                     "frac": ach / peaks["bf16"], "traffic": traffic.get(dom), "peak_kind": peaks["kind"],
                     "peak_figure": "bf16_tflops_sustained", "avg_launch_ms": dom_ms, "algorithmic_flops": flops[dom]})
    else:
        roof.update({"bound": "unknown", "achieved": None, "peak": None, "unit": None, "frac": None,
                     "traffic": traffic.get(dom), "peak_kind": peaks["kind"]})
    mlp_rates = {k: {"ms": ktimes[k][0] / ktimes[k][1], "tflops": flops[k] / (ktimes[k][0] / ktimes[k][1]) / 1e9,
                     "frac_of_sustained_bf16": flops[k] / (ktimes[k][0] / ktimes[k][1]) / 1e9 / peaks["bf16"]}
                 for k in flops if k in ktimes}
    del bf
    torch.cuda.empty_cache()

    # ---- the plain way: one receiver per step, FP32 MLP, same scene and model
    plain = FusedTrainer(sc3, device=dev, group=group, shared=SharedMLP(**SHARED_CFG3, precision="fp32"))
    plain.capture(1, cap3, tx, v3[0:1], r3[0:1], t3[0:1])
    n_p = max(3, args.steps)

    def plain_step(i):
        j = i % nb
        return plain.step(v3[j:j + 1], r3[j:j + 1], t3[j:j + 1])

    for i in range(3):
        plain_step(i)
    psec = timed(plain_step, n_p)
    plain.plan.check()
    del plain
    torch.cuda.empty_cache()
    plain_sps = n_p * world / psec
    cfg3 = {"receivers_per_step": R_CFG3, "steps_per_s": args.steps * world / sec, "spectra_per_s": value,
            "instances_K": K3,
            "plain_fp32": {"receivers_per_step": 1, "steps_per_s": plain_sps, "spectra_per_s": plain_sps,
                           "timed_steps": n_p},
            "speedup_vs_plain_fp32": value / plain_sps, "delta_ssim_bf16_vs_fp32": dssim}

    side = {}
    if world == 1 and not args.headline_only:
        side = _side_lines(args, dev, timed)

    cpu_base = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        v, n, threads = _cpu_steps(3, 60.0, threads, warmup=1)
        cpu_base = {"value": v, "unit": UNIT, "cores": threads, "kind": "port", "port": "torch-cpu",
                    "sample": f"{n} timed training steps (after 1 warm-up) of one receiver each on the full "
                              f"{P_CFG3}-Gaussian scene, CPU PyTorch rendition (oracle/torch_cpu.py), "
                              f"{threads} threads"}
    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": max(args.warmup, 3), "ms_per_step": 1000.0 * sec / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "bf16 MLP (tcgen05, fp32 accumulate) + f32 blend/SSIM",
                "data": "synthetic",
                "config": {"workload": WORKLOAD, "gaussians": P_CFG3, "receivers_per_step": R_CFG3,
                           "receivers_per_rank": R_CFG3, "spectrum": "90x360", "tiles": "16x16",
                           "instances_K": K3,
                           "l2": "flushed between steps (256 MiB write, outside the timed events); the step's state "
                                 "is several GB",
                           "parallelism": f"dp{world} (receivers sharded, gradients all-reduced)"},
                "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": 4},
                "gpu_launches": launches * args.steps,
                "gpu_launches_per_step": launches,
                "clocks": clk.summary(),
                "roofline": roof,
                "mlp_tensor_rates": mlp_rates,
                "kernel_ms_per_step": kms,
                "kernel_ms_note": "eager steps with per-launch events; their sum exceeds the graph step's time",
                "cfg3_batched_bf16_vs_plain_fp32": cfg3,
                "path": "CUDA-graph-captured step (gsparc_b200.fused.FusedTrainer): flat training state, shared "
                        "emission MLP in BF16 on tcgen05, fused L1+SSIM+confidence loss, fused activation-adjoint "
                        f"Adam; binning capacity {cap3 * R_CFG3}",
                "cpu_baseline": cpu_base}
        line.update(side)
        print(json.dumps(line))
    if group is not None:
        dist_barrier_and_destroy(group)
    return 0


def dist_barrier_and_destroy(group):
    import torch.distributed as dist
    dist.barrier()
    dist.destroy_process_group()


def _side_lines(args, dev, timed):
    """Further workloads on one GPU (not the headline)."""
    import numpy as np
    import torch
    from gsparc_b200 import scenes
    from gsparc_b200.fused import FusedTrainer
    from gsparc_b200.shared_mlp import SharedMLP
    out = {}
    # ---- cfg1: 20,000 Gaussians, shared 2x64 ReLU FP32, one receiver per step
    d = _scene_data(P_CFG1, POOL1, dev)
    tx = d["tx"]
    tr = FusedTrainer(d["scene"], device=dev, shared=SharedMLP(**SHARED_CFG1))
    cap = tr.probe_capacity(d["views_d"], d["rxs_d"], tx)
    tr.capture(1, cap, tx, d["views_d"][0:1], d["rxs_d"][0:1], d["targets_d"][0:1])

    def st1(i):
        j = i % POOL1
        return tr.step(d["views_d"][j:j + 1], d["rxs_d"][j:j + 1], d["targets_d"][j:j + 1])

    for i in range(3):
        st1(i)
    n1 = max(3, args.steps)
    sec1 = timed(st1, n1)
    tr.plan.check()
    del tr
    # 16 receivers per step and 16-receiver inference with the evaluation metrics, same model
    btr = FusedTrainer(d["scene"], device=dev, shared=SharedMLP(**SHARED_CFG1))
    btr.capture(POOL1, cap * POOL1, tx, d["views_d"], d["rxs_d"], d["targets_d"])
    n_b = max(3, args.steps // 4)
    bsec = timed(lambda i: btr.step(d["views_d"], d["rxs_d"], d["targets_d"]), n_b)
    isec = timed(lambda i: btr.evaluate(d["views_d"], d["rxs_d"], tx, d["targets_d"]), n_b)
    btr.plan.check()
    del btr
    out["cfg1_per_receiver_fp32"] = {
        "workload": f"cfg1: P={P_CFG1}, one receiver per step, shared emission MLP 2x64 ReLU, FP32, CUDA graph",
        "steps_per_s": n1 / sec1, "spectra_per_s": n1 / sec1,
        "batched16": {"steps_per_s": n_b / bsec, "spectra_per_s": n_b * POOL1 / bsec},
        "inference16_eval": {"spectra_per_s": n_b * POOL1 / isec,
                             "metrics": ["psnr", "rssi_diff", "mae", "ssim", "confidence", "loss"]}}
    del d
    torch.cuda.empty_cache()
    # ---- cfg2: 50,000 clustered Gaussians, 64 receivers per step, tile shape autotuned
    d2 = _scene_data(P_CFG2, R_CFG2, dev, cluster_frac=0.3)
    v2, r2, t2 = d2["views_d"], d2["rxs_d"], d2["targets_d"]
    tr2 = FusedTrainer(d2["scene"], device=dev, shared=SharedMLP(**SHARED_CFG1))
    tune = tr2.autotune_tile(tx, v2, r2, t2, steps=3)
    n2 = max(3, args.steps // 10)
    sec2 = timed(lambda i: tr2.step(v2, r2, t2), n2)
    K2, _ = tr2.plan.host_status()
    tr2.plan.check()
    out["cfg2_batched_clustered_autotuned"] = {
        "workload": f"cfg2: P={P_CFG2} (30% in 5 N(c_k, 0.3 m) clusters), {R_CFG2} receivers per step, shared "
                    "emission MLP 2x64 ReLU, FP32, training step with adjoint, CUDA graph",
        "tile_ms_per_step": {f"{h}x{w}": ms for (h, w), ms in tune.items()}, "tile": "%dx%d" % tr2.tile,
        "instances_K": K2, "steps_per_s": n2 / sec2, "spectra_per_s": n2 * R_CFG2 / sec2}
    del tr2, d2
    torch.cuda.empty_cache()
    # ---- cfg4: 100,000 Gaussians, 16 receivers x 64 frequency channels per step
    from gsparc_b200 import raster
    sc4 = scenes.make_scene(P_CFG4, scenes.SEED_SCENE)
    tg4 = scenes.make_scene(P_CFG4, scenes.SEED_TARGET)
    rx4 = scenes.make_receivers(R_CFG4)
    t = lambda a: torch.tensor(np.ascontiguousarray(a), dtype=torch.float32, device=dev)
    v4, r4 = t(scenes.view_matrices(rx4)), t(rx4)
    with torch.no_grad():   # targets: the second scene rendered through a seeded 64-output MLP
        tm, ts, tq, to = tg4.activated()
        tmlp = SharedMLP(**SHARED_CFG4)
        t4, _, _ = raster.forward_channels(t(tm), t(to.reshape(-1)), t(ts), t(tq), H, W, 1.0, v4, tx, r4, tmlp,
                                           tmlp.init_params(seed=7, device=dev))
        t4 = t4.clone()
    tr4 = FusedTrainer(sc4, device=dev, shared=SharedMLP(**SHARED_CFG4))
    cap4 = tr4.probe_capacity(v4, r4, tx) * R_CFG4
    tr4.capture(R_CFG4, cap4, tx, v4, r4, t4)
    n4 = max(3, args.steps // 10)
    sec4 = timed(lambda i: tr4.step(v4, r4, t4), n4)
    K4, _ = tr4.plan.host_status()
    tr4.plan.check()
    out["cfg4_multichannel"] = {
        "workload": f"cfg4: P={P_CFG4}, {R_CFG4} receivers x {C_CFG4} frequency channels per step, shared emission "
                    "MLP 3x128 GELU -> 64 amplitudes (BF16 on tcgen05), multi-channel FP32 blend, loss over R*C "
                    "spectra, training step with adjoint, CUDA graph",
        "instances_K": K4, "steps_per_s": n4 / sec4, "spectra_per_s": n4 * R_CFG4 * C_CFG4 / sec4}
    del tr4
    torch.cuda.empty_cache()
    # ---- the reference CUDA extension beside the drop-in modules
    try:
        out["reference_extension"] = _reference_extension_leg(dev)
    except Exception as exc:   # report, never hide: the headline above does not depend on it
        out["reference_extension"] = {"error": f"{type(exc).__name__}: {exc}"}
    return out


def run_check_ranks():
    """Launcher check without GPUs: join a gloo process group on 127.0.0.1;
    rank 0 prints every rank's place in it (one line per rank, gathered, so
    the ranks' output never interleaves), then all leave."""
    import torch.distributed as dist
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if world > 1:
        dist.init_process_group("gloo")
        places = [None] * dist.get_world_size()
        dist.all_gather_object(places, {"rank": dist.get_rank(), "world": dist.get_world_size()})
        if dist.get_rank() == 0:
            for p in places:
                print(json.dumps(p), flush=True)
        dist.barrier()
        dist.destroy_process_group()
    else:
        print(json.dumps({"rank": 0, "world": 1}), flush=True)
    return 0


def run_eager(args):
    """Eager steps of one FusedTrainer configuration for profiler captures."""
    import numpy as np
    import torch
    from gsparc_b200 import scenes
    from gsparc_b200._lib import KernelTimer
    from gsparc_b200.autograd import RasterPlan
    from gsparc_b200.fused import FusedTrainer
    from gsparc_b200.shared_mlp import SharedMLP
    dev = torch.device("cuda")
    sc = scenes.make_scene(args.P, scenes.SEED_SCENE)
    rxs = scenes.make_receivers(args.R)
    views = scenes.view_matrices(rxs)
    t = lambda x: torch.tensor(np.ascontiguousarray(x), dtype=torch.float32, device=dev)
    gen = torch.Generator().manual_seed(1)
    shared = {"ref": None, "relu64": SharedMLP(2, 64, "relu", precision=args.precision),
              "gelu128": SharedMLP(3, 128, "gelu", precision=args.precision),
              "ch64": SharedMLP(3, 128, "gelu", out=64, precision=args.precision)}[args.mlp]
    C = 1 if shared is None else shared.out
    targets = torch.rand((args.R, H, W) if C == 1 else (args.R, C, H, W), generator=gen).to(dev)
    tr = FusedTrainer(sc, device=dev, shared=shared)
    tr.plan = RasterPlan(args.P, args.R, H, W, args.cap * args.R, dev)
    tx = t(scenes.TX_POS)
    for _ in range(args.eager_steps - 1):
        tr.step_eager(t(views), t(rxs), tx, targets)
    torch.cuda.synchronize()
    with KernelTimer() as kt:
        loss = tr.step_eager(t(views), t(rxs), tx, targets)
        torch.cuda.synchronize()
    if args.times:
        for k, (ms, n) in sorted(kt.results().items(), key=lambda x: -x[1][0]):
            if n:
                print(f"  {k:32s} {1000 * ms:9.1f} us  ({n} calls)")
    tr.plan.record_status()
    torch.cuda.synchronize()
    print("K", tr.plan.check(), "loss", float(loss))
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--headline-only", action="store_true", help="skip the side lines")
    ap.add_argument("--eager-steps", type=int, default=0, help="profiling mode: eager steps of one configuration")
    ap.add_argument("--P", type=int, default=20000)
    ap.add_argument("--R", type=int, default=1)
    ap.add_argument("--cap", type=int, default=160000, help="binning capacity per receiver (--eager-steps)")
    ap.add_argument("--mlp", choices=["ref", "relu64", "gelu128", "ch64"], default="ref")
    ap.add_argument("--precision", choices=["fp32", "bf16"], default="fp32")
    ap.add_argument("--times", action="store_true")
    ap.add_argument("--check-ranks", action="store_true",
                    help="start the ranks as for --gpus N, have each join a gloo group and print its rank, and exit")
    args = ap.parse_args()
    if args.eager_steps > 0:
        return run_eager(args)
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        return _launch_ranks(args)
    if args.check_ranks:
        return run_check_ranks()
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
