"""Multi-rank host logic (n2w.shard) with 2-rank gloo groups on CPU: point
ranges partition the job, walk shares sum to the walk count, rank seeds are
distinct, and combining walk shards by all-reduce equals one process holding
every sample; point shards gather back in order; data-parallel cache training
(the convention of n2w_nc_train_dp: every rank's mean gradient over its own
batch, summed over ranks, Adam on the sum / world) equals one process training
on the union batch, checked with the FP64 cache oracle.

The product's transport is NcclComm (NCCL through the C ABI, one process per
GPU); these CPU tests drive the same shard functions through GlooComm, a
test-only communicator over torch.distributed's gloo backend."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from n2w import shard


class GlooComm:
    """Test communicator with NcclComm's host interface over gloo."""

    def __init__(self):
        self.rank, self.world = dist.get_rank(), dist.get_world_size()

    def allreduce_host(self, arrays, op="sum"):
        red = {"sum": dist.ReduceOp.SUM, "max": dist.ReduceOp.MAX, "min": dist.ReduceOp.MIN}[op]
        out = []
        for a in arrays:
            t = torch.from_numpy(np.ascontiguousarray(a, np.float64).copy())
            dist.all_reduce(t, op=red)
            out.append(t.numpy())
        return out

    def barrier(self):
        dist.barrier()


def test_point_ranges_partition():
    for n in (0, 1, 7, 1000, 170364):
        for world in (1, 2, 3, 8):
            ranges = [shard.point_range(n, r, world) for r in range(world)]
            assert ranges[0][0] == 0
            assert sum(c for _, c in ranges) == n
            for (s0, c0), (s1, _) in zip(ranges, ranges[1:]):
                assert s0 + c0 == s1
            assert max(c for _, c in ranges) - min(c for _, c in ranges) <= 1
    assert sum(shard.walk_share(1024, r, 3) for r in range(3)) == 1024
    assert len({shard.rank_seed(12345, r) for r in range(64)}) == 64
    with pytest.raises(ValueError):
        shard.point_range(10, 2, 2)


def samples(rank, world, n_points=97, walks=40):
    """Synthetic per-walk values of every point: rank r draws its share of walks."""
    w = shard.walk_share(walks, rank, world)
    rng = np.random.default_rng(shard.rank_seed(7, rank) % (2**63))
    return rng.normal(1.0 + np.arange(n_points)[:, None] * 0.01, 0.3, (n_points, w))


def stats_of(v):
    return {"sum": v.sum(1), "sum_sq": (v * v).sum(1), "count": np.full(len(v), v.shape[1], np.float64),
            "steps": np.full(len(v), 20.0 * v.shape[1]), "forced": np.zeros(len(v))}


def _worker(rank, world, port, out_dir):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        comm = GlooComm()
        v = samples(rank, world)
        comb = shard.allreduce_point_stats(stats_of(v), comm)
        n = 53
        s, c = shard.point_range(n, rank, world)
        gathered = shard.gather_point_ranges(np.arange(s, s + c, dtype=np.float64) * 2.0, n, comm)
        np.savez(os.path.join(out_dir, f"r{rank}.npz"), mean=comb["mean"], var=comb["sample_variance"],
                 count=comb["count"], gathered=gathered)
    finally:
        dist.destroy_process_group()


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_rank_gloo_combination(tmp_path):
    world = 2
    mp.spawn(_worker, args=(world, free_port(), str(tmp_path)), nprocs=world, join=True)
    allv = np.concatenate([samples(r, world) for r in range(world)], axis=1)
    ref = shard.finish_stats(stats_of(allv))
    for r in range(world):
        d = np.load(tmp_path / f"r{r}.npz")
        np.testing.assert_allclose(d["mean"], ref["mean"], rtol=1e-12)
        np.testing.assert_allclose(d["var"], ref["sample_variance"], rtol=1e-9)
        assert np.all(d["count"] == 40)
        np.testing.assert_array_equal(d["gathered"], np.arange(53) * 2.0)


# ---- data-parallel training algebra ------------------------------------------------

def dp_problem(seed=5):
    from oracle import cache_oracle as co

    lay = co.layout(4, 10, 4.0, 32.0, 0.0, 16, 1)
    rng = np.random.default_rng(seed)
    params = np.concatenate([rng.uniform(-1e-2, 1e-2, lay["grid_params"]),
                             rng.uniform(-0.3, 0.3, lay["mlp"]["total"])])
    B = 64  # per rank
    u = rng.uniform(0, 1, (2 * B, 3))
    t = np.sin(3 * u[:, 0]) * np.cos(2 * u[:, 1]) + u[:, 2]
    return lay, params, u, t, B


def adam(p, g, m, v, step, lr=1e-2, b1=0.9, b2=0.99, eps=1e-15):
    """The product's Adam update (FP32 kernel restated in FP64)."""
    m = b1 * m + (1 - b1) * g
    v = b2 * v + (1 - b2) * g * g
    p = p - lr * (m / (1 - b1 ** step)) / (np.sqrt(v / (1 - b2 ** step)) + eps)
    return p, m, v


def _dp_worker(rank, world, port, out_dir):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from oracle import cache_oracle as co

        comm = GlooComm()
        lay, p, u, t, B = dp_problem()
        m, v = np.zeros_like(p), np.zeros_like(p)
        for step in (1, 2, 3):
            lo = rank * B
            _, g = co.gradients(lay, p, u[lo:lo + B], t[lo:lo + B])  # mean over this rank's batch
            g = comm.allreduce_host([g], "sum")[0] / world
            p, m, v = adam(p, g, m, v, step)
        np.save(os.path.join(out_dir, f"p{rank}.npy"), p)
    finally:
        dist.destroy_process_group()


def test_data_parallel_gradients_equal_union_batch(tmp_path):
    from oracle import cache_oracle as co

    world = 2
    mp.spawn(_dp_worker, args=(world, free_port(), str(tmp_path)), nprocs=world, join=True)
    lay, p, u, t, B = dp_problem()
    m, v = np.zeros_like(p), np.zeros_like(p)
    for step in (1, 2, 3):
        _, g = co.gradients(lay, p, u, t)  # one process, the union batch of 2B points
        p, m, v = adam(p, g, m, v, step)
    p0, p1 = np.load(tmp_path / "p0.npy"), np.load(tmp_path / "p1.npy")
    np.testing.assert_array_equal(p0, p1)  # ranks stay identical
    np.testing.assert_allclose(p0, p, rtol=1e-10, atol=1e-13)


def test_nccl_comm_id_handover(monkeypatch, tmp_path):
    """NcclComm's host side for N > 1 ranks, with the library's NCCL calls
    replaced by a stand-in (no GPU): rank 0's id reaches rank 1 through the
    launch's file even when rank 1 starts first, both join with the same id,
    the world size and their rank, the file is gone afterwards, and a rank
    whose rank 0 never writes the id fails with a clear timeout."""
    import ctypes as C
    import threading

    from n2w import _lib, shard

    uid_bytes = bytes((7 * i + 3) & 0xFF for i in range(128))
    joined = threading.Barrier(2, timeout=30)
    seen = {}

    def fake_call(name, *args):
        if name == "n2w_comm_unique_id":
            for i, b in enumerate(uid_bytes):
                args[0][i] = b
        elif name == "n2w_comm_create":
            uid, world, rank, handle = args
            seen[rank] = (bytes(uid), world)
            joined.wait()  # like ncclCommInitRank: returns once every rank has joined
            handle._obj.value = 1000 + rank
        else:
            raise AssertionError(f"unexpected call {name}")
        return 0

    monkeypatch.setattr(_lib, "call", fake_call)
    comms, errors = {}, []

    def join(rank):
        try:
            comms[rank] = shard.NcclComm(rank, 2, key="launch1", directory=str(tmp_path), timeout=30)
        except Exception as e:  # pragma: no cover - reported below
            errors.append(e)

    threads = [threading.Thread(target=join, args=(r,)) for r in (1, 0)]  # rank 1 waits for the file
    for th in threads:
        th.start()
    for th in threads:
        th.join(60)
    try:
        assert not errors, errors
        assert seen[0] == seen[1] == (uid_bytes, 2)
        assert (comms[0].rank, comms[1].rank, comms[0].world) == (0, 1, 2)
        assert not (tmp_path / "n2w_nccl_launch1.id").exists()
    finally:
        for c in comms.values():
            c.h = C.c_void_p()  # stand-in handles: nothing to destroy
    with pytest.raises(TimeoutError, match="no NCCL id"):
        shard.NcclComm(1, 2, key="no_rank0", directory=str(tmp_path), timeout=0.2)
