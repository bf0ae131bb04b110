"""Multi-GPU layout of the training step: receivers are independent given
the Gaussians, so they are partitioned across ranks (one process per GPU)
with every Gaussian and MLP weight replicated; the one exchange per step is
a sum all-reduce of the per-Gaussian gradients, done over one flat bucket.
(The reference is single-GPU, train.py:182; this is the B200 scale-out of
the same step.)"""
from __future__ import annotations

import torch
import torch.distributed as dist


def shard_receivers(R: int, rank: int, world: int):
    """Contiguous block of receiver indices owned by ``rank`` (sizes differ by
    at most one)."""
    if not (0 <= rank < world):
        raise ValueError("rank out of range")
    base, extra = divmod(R, world)
    start = rank * base + min(rank, extra)
    return range(start, start + base + (1 if rank < extra else 0))


def allreduce_grads(params, group=None) -> int:
    """Sum the gradients of ``params`` over ``group`` in one bucket.
    Parameters without a gradient contribute zeros so every rank issues the
    same collective with the same size.  Returns the bucket size in floats."""
    ps = list(params)
    sizes = [p.numel() for p in ps]
    dev = ps[0].device
    flat = torch.empty(sum(sizes), dtype=torch.float32, device=dev)
    off = 0
    for p, n in zip(ps, sizes):
        if p.grad is None:
            flat[off:off + n].zero_()
        else:
            flat[off:off + n].copy_(p.grad.reshape(-1))
        off += n
    dist.all_reduce(flat, op=dist.ReduceOp.SUM, group=group)
    off = 0
    for p, n in zip(ps, sizes):
        g = flat[off:off + n].view_as(p)
        if p.grad is None:
            p.grad = g.clone()
        else:
            p.grad.copy_(g)
        off += n
    return int(flat.numel())


def allreduce_flat(flat: torch.Tensor, group=None) -> None:
    """The exchange step of the receiver-sharded training step: sum the flat
    gradient buffer (every parameter group, the MLPs included, in one
    contiguous tensor) over the ranks in one collective, in place.
    FusedTrainer issues it inside its captured step, between the adjoint and
    the optimizer kernel, on the step's stream."""
    dist.all_reduce(flat, op=dist.ReduceOp.SUM, group=group)


def reduce_densify_stats(accum: torch.Tensor, denom: torch.Tensor, max_radii2D: torch.Tensor, group=None) -> None:
    """Densification statistics of the receivers of every rank (train.py:508-516
    accumulates them per rendered receiver): the gradient-norm sums and
    counts add up, the screen radii take the maximum; in place, so that every
    rank then densifies the same Gaussians the same way."""
    dist.all_reduce(accum, op=dist.ReduceOp.SUM, group=group)
    dist.all_reduce(denom, op=dist.ReduceOp.SUM, group=group)
    dist.all_reduce(max_radii2D, op=dist.ReduceOp.MAX, group=group)
