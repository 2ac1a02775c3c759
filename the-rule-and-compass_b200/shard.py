"""Candidate sharding across ranks (one process per GPU).

The device path shards by candidate: programs are independent given the
resident rows, so each rank keeps its own copy of the dataset, evaluates or
fits a contiguous slice of the candidate batch, and the per-candidate
outputs (a few words each) are gathered once at the end. There is no
collective on the data path; the only collectives are the final gather and
the max-over-ranks of the device time that the benchmark reports.

The functions take a `torch.distributed` process group (NCCL on GPUs, gloo on
CPU); with `group=None` and no initialised process group they act as a
single rank.
"""
from __future__ import annotations

import numpy as np


def _dist():
    import torch.distributed as dist
    return dist if dist.is_available() and dist.is_initialized() else None


def shard_bounds(n_items: int, rank: int, world: int) -> tuple[int, int]:
    """[start, end) of rank's contiguous slice; sizes differ by at most one,
    the first `n_items % world` ranks taking the extra item."""
    if world <= 0 or not 0 <= rank < world:
        raise ValueError("rank must be in [0, world)")
    base, extra = divmod(int(n_items), world)
    start = rank * base + min(rank, extra)
    return start, start + base + (1 if rank < extra else 0)


def gather_candidates(local, n_items: int, group=None, device=None):
    """Concatenate every rank's slice (a [slice, ...] array) in rank order,
    on every rank. Slices are padded to the largest slice for the
    collective and trimmed afterwards."""
    import torch
    dist = _dist()
    local = np.ascontiguousarray(local)
    if dist is None:
        return local.copy()
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    counts = [shard_bounds(n_items, r, world) for r in range(world)]
    counts = [e - s for s, e in counts]
    if local.shape[0] != counts[rank]:
        raise ValueError("local slice does not match this rank's shard")
    width = max(counts)
    tail = local.shape[1:]
    pad = np.zeros((width,) + tail, local.dtype)
    pad[: local.shape[0]] = local
    t = torch.from_numpy(pad.view(np.uint8).copy())
    if device is not None:
        t = t.to(device)
    parts = [torch.empty_like(t) for _ in range(world)]
    dist.all_gather(parts, t, group=group)
    out = []
    for r, p in enumerate(parts):
        a = p.cpu().numpy().view(local.dtype).reshape((width,) + tail)
        out.append(a[: counts[r]])
    return np.concatenate(out, axis=0)


def max_over_ranks(value: float, group=None, device=None) -> float:
    """The maximum of a per-rank scalar (the device time of a step)."""
    import torch
    dist = _dist()
    if dist is None:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.item())
