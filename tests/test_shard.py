"""Multi-rank host logic (n2w.shard) with 2-rank gloo groups on CPU: point
ranges partition the job, walk shares sum to the walk count, rank seeds are
distinct, and combining walk shards by all-reduce equals one process holding
every sample; point shards gather back in order."""
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from n2w import shard


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
        v = samples(rank, world)
        comb = shard.allreduce_point_stats(stats_of(v))
        n = 53
        s, c = shard.point_range(n, rank, world)
        gathered = shard.gather_point_ranges(np.arange(s, s + c, dtype=np.float64) * 2.0, n)
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
