"""Splitting a WoS job across ranks and combining the results.

Walks and points are independent, so a job shards two ways: by points (each
rank evaluates a disjoint range of points with all walks), or by walks (every
rank evaluates all points with its share of the walks and its own walk
stream).  Per-point statistics are sums (FP64 sum, sum of squares, counts,
steps), so combining walk shards is one element-wise all-reduce; point shards
only need gathering.  torch.distributed is the transport (NCCL on GPUs, gloo
on CPU); nothing here touches the device kernels.
"""
from __future__ import annotations

import numpy as np

STAT_FIELDS = ("sum", "sum_sq", "count", "steps", "forced")


def point_range(n: int, rank: int, world: int) -> tuple[int, int]:
    """Contiguous, balanced share [start, start + count) of n points."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("need 0 <= rank < world")
    base, extra = divmod(n, world)
    start = rank * base + min(rank, extra)
    return start, base + (1 if rank < extra else 0)


def walk_share(walks: int, rank: int, world: int) -> int:
    """Walks per point for this rank when walks are split (shares sum to walks)."""
    return point_range(walks, rank, world)[1]


def rank_seed(seed: int, rank: int) -> int:
    """Independent Philox key per rank (keys differ in every bit pattern)."""
    return (int(seed) + 0x9E3779B97F4A7C15 * (rank + 1)) & 0xFFFFFFFFFFFFFFFF


def allreduce_point_stats(stats: dict, group=None) -> dict:
    """Element-wise sum of per-point statistics over ranks (walk shards).

    `stats` maps STAT_FIELDS to numpy arrays (as PointStatsBuffers.download
    returns them, or raw sums); returns the combined arrays and the derived
    mean / sample_variance / stderr.  Runs on the process group's backend."""
    import torch
    import torch.distributed as dist

    backend = dist.get_backend(group)
    dev = torch.device("cuda", torch.cuda.current_device()) if backend == "nccl" else torch.device("cpu")
    out = {}
    for f in STAT_FIELDS:
        t = torch.from_numpy(np.ascontiguousarray(stats[f], np.float64)).to(dev)
        dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
        out[f] = t.cpu().numpy()
    return finish_stats(out)


def finish_stats(s: dict) -> dict:
    """mean, unbiased sample variance and standard error from summed statistics."""
    cnt = s["count"].astype(np.float64)
    mean = s["sum"] / np.maximum(cnt, 1)
    var = np.where(cnt > 1, (s["sum_sq"] - cnt * mean * mean) / np.maximum(cnt - 1, 1), 0.0)
    var = np.maximum(var, 0.0)
    out = dict(s)
    out.update(mean=mean, sample_variance=var, stderr=np.sqrt(var / np.maximum(cnt, 1)),
               mean_steps=s["steps"] / np.maximum(cnt, 1))
    return out


def gather_point_ranges(values: np.ndarray, n: int, group=None) -> np.ndarray:
    """Concatenates each rank's point_range share of a per-point array (point shards)."""
    import torch
    import torch.distributed as dist

    world = dist.get_world_size(group)
    parts = [None] * world
    dist.all_gather_object(parts, np.asarray(values), group=group)
    out = np.concatenate(parts)
    if len(out) != n:
        raise ValueError(f"gathered {len(out)} values for {n} points")
    return out
