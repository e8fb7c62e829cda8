"""Splitting a WoS job across ranks and combining the results.

Walks and points are independent, so a job shards two ways: by points (each
rank evaluates a disjoint range of points with all walks), or by walks (every
rank evaluates all points with its share of the walks and its own walk
stream).  Per-point statistics are sums (FP64 sum, sum of squares, counts,
steps), so combining walk shards is one element-wise all-reduce; point shards
are combined the same way from zero-padded full-length arrays.

The transport is a communicator object with `rank`, `world`,
`allreduce_host(arrays, op)` (host numpy arrays in, reduced copies out) and
`barrier()`.  On GPUs it is NcclComm: the library's NCCL communicator
(n2w_comm_*, one process per GPU); nothing here touches the walker kernels.
"""
from __future__ import annotations

import ctypes as C
import os
import tempfile
import time
from pathlib import Path

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


def allreduce_point_stats(stats: dict, comm) -> dict:
    """Element-wise sum of per-point statistics over ranks (walk shards).

    `stats` maps STAT_FIELDS to numpy arrays (as PointStatsBuffers.download
    returns them, or raw sums); returns the combined arrays and the derived
    mean / sample_variance / stderr."""
    summed = comm.allreduce_host([np.ascontiguousarray(stats[f], np.float64) for f in STAT_FIELDS], "sum")
    return finish_stats(dict(zip(STAT_FIELDS, summed)))


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


def gather_point_ranges(values: np.ndarray, n: int, comm) -> np.ndarray:
    """Every rank's point_range share of a per-point array, in point order
    (point shards): each rank contributes its range of a zero-padded array."""
    start, count = point_range(n, comm.rank, comm.world)
    values = np.asarray(values, np.float64)
    if len(values) != count:
        raise ValueError(f"rank {comm.rank} holds {len(values)} values for its {count} points")
    full = np.zeros(n, np.float64)
    full[start:start + count] = values
    return comm.allreduce_host([full], "sum")[0]


class NcclComm:
    """This process's NCCL communicator (n2w_comm_*) on its current device.

    Rank 0 creates the NCCL id and hands it to the other ranks of the node
    through a file in `directory` (default: the temp directory) named by `key`,
    which must be unique per job launch; every rank then joins the
    communicator (which waits until all `world` ranks have joined)."""

    def __init__(self, rank: int, world: int, key: str, directory: str | None = None, timeout: float = 120.0):
        from ._lib import call

        self.rank, self.world = rank, world
        self._call = call
        self.h = C.c_void_p()
        uid = (C.c_uint8 * 128)()
        path = Path(directory or tempfile.gettempdir()) / f"n2w_nccl_{key}.id"
        if rank == 0:
            call("n2w_comm_unique_id", uid)
            tmp = path.with_suffix(".tmp")
            tmp.write_bytes(bytes(uid))
            os.replace(tmp, path)
        else:
            deadline = time.monotonic() + timeout
            while not (path.exists() and path.stat().st_size == 128):
                if time.monotonic() > deadline:
                    raise TimeoutError(f"rank {rank}: no NCCL id at {path} after {timeout} s")
                time.sleep(0.02)
            C.memmove(uid, path.read_bytes(), 128)
        call("n2w_comm_create", uid, world, rank, C.byref(self.h))
        if rank == 0:
            path.unlink(missing_ok=True)  # every rank has joined, so every rank has read it

    def allreduce_host(self, arrays, op: str = "sum"):
        """All-reduce of host float64 arrays through one device buffer."""
        from . import DeviceBuffer
        from ._lib import N2W_DTYPE_F64, N2W_OP_MAX, N2W_OP_MIN, N2W_OP_SUM

        code = {"sum": N2W_OP_SUM, "max": N2W_OP_MAX, "min": N2W_OP_MIN}[op]
        flat = np.concatenate([np.ascontiguousarray(a, np.float64).ravel() for a in arrays])
        if len(flat) == 0:
            return [np.asarray(a, np.float64).copy() for a in arrays]
        buf = DeviceBuffer.from_array(flat)
        self._call("n2w_comm_allreduce", self.h, buf.ptr, buf.ptr, len(flat), N2W_DTYPE_F64, code, None)
        out = buf.download(np.float64, len(flat))
        res, off = [], 0
        for a in arrays:
            a = np.asarray(a)
            res.append(out[off:off + a.size].reshape(a.shape))
            off += a.size
        return res

    def allreduce_point_stats_device(self, stats, n: int, stream=None):
        """In-place device all-reduce of a PointStatsBuffers (walk shards)."""
        self._call("n2w_comm_allreduce_point_stats", self.h, stats.struct(), n, stream.handle if stream else None)

    def barrier(self):
        self._call("n2w_comm_barrier", self.h, None)

    def close(self):
        from ._lib import lib

        if self.h:
            lib.n2w_comm_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
