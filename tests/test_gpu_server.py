"""Serving loop (n2w_server_*): continuous batching on one GPU.

Checks that a request gives the same answer alone and in a mix (same walk
counts, FP64 sums equal to rounding of the addition order), that results meet
their target standard error against the FP64 analytic solution, that admission
respects the device pool (oversized requests refused, the rest queued until
memory frees), that concurrent requests share launches, and the walk cap;
NC+2LMC requests (a trained cache, and the analytic cache) are unbiased and
also the same alone and in a mix of plain and NC+2LMC requests.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def meshes(gpu):
    from n2w import workloads

    out = []
    for st, sl in ((24, 48), (40, 80)):
        m = workloads.bumpy_sphere(gpu, st, sl)
        out.append((m, gpu.Bvh(m, 4, "sah")))
    return out


def problems(gpu):
    return [gpu.problem_charges_seeded(8, 1.6, 2.0, seed=5), gpu.problem_from_name("harmonic_zebra_k4")]


def points(meshes, k, n, seed):
    from n2w import workloads

    return workloads.interior_ball_points(meshes[k][1], n, np.random.default_rng(seed))


def check_accuracy(gpu, prob, pts, mean, se, info, target):
    exact = gpu.problem_exact(prob, pts.astype(np.float64))
    assert info["state"] == 2  # N2W_REQUEST_DONE
    assert info["max_stderr"] <= target
    assert np.all(se <= target * (1 + 1e-6))
    z = (mean - exact) / np.maximum(se, 1e-12)
    assert np.mean(np.abs(z) < 4) >= 0.97 if len(z) >= 30 else np.all(np.abs(z) < 5)


def test_alone_equals_mix_and_accuracy(gpu, meshes):
    probs = problems(gpu)
    bvhs = [b for _, b in meshes]
    pa = points(meshes, 0, 300, seed=1)
    srv = gpu.Server(bvhs, probs, pool_bytes=64 << 20, tick_walks=1 << 16, epsilon=1e-3)
    ra = srv.submit(0, 0, pa, 2e-2, seed=77)
    mean_a, se_a, info_a = srv.wait(ra, timeout=120)
    check_accuracy(gpu, probs[0], pa, mean_a, se_a, info_a, 2e-2)
    # the same request in a mix of uneven requests on both meshes and problems
    others = []
    for k, (mesh, prob, n, tgt) in enumerate([(1, 1, 5000, 3e-2), (0, 1, 1, 1e-2), (1, 0, 40, 1e-2),
                                               (0, 0, 2000, 3e-2), (1, 1, 7, 5e-3)]):
        p = points(meshes, mesh, n, seed=10 + k)
        others.append((srv.submit(mesh, prob, p, tgt, seed=100 + k), mesh, prob, p, tgt))
    rb = srv.submit(0, 0, pa, 2e-2, seed=77)
    mean_b, se_b, info_b = srv.wait(rb, timeout=300)
    assert info_b["walks_per_point"] == info_a["walks_per_point"]
    assert info_b["sweeps"] == info_a["sweeps"]
    np.testing.assert_allclose(mean_b, mean_a, rtol=1e-12, atol=1e-14)
    np.testing.assert_allclose(se_b, se_a, rtol=1e-9, atol=1e-14)
    for rid, mesh, prob, p, tgt in others:
        m, s, info = srv.wait(rid, timeout=300)
        check_accuracy(gpu, probs[prob], p, m, s, info, tgt)
    st = srv.stats()
    assert st["completed"] == 7 and st["overflow"] == 0 and st["peak_inflight"] >= 2
    srv.close()


def test_pool_admission_and_oversized_requests(gpu, meshes):
    probs = problems(gpu)
    bvhs = [b for _, b in meshes]
    srv = gpu.Server(bvhs, probs, pool_bytes=1 << 20, tick_walks=1 << 16, epsilon=1e-3)
    big = points(meshes, 0, 30000, seed=3)
    with pytest.raises(gpu.N2wError, match="whole serving pool"):
        srv.submit(0, 0, big, 1e-2)
    # ~9000 points hold ~400 KB: at most two fit in the 1 MiB pool at once
    ids = [srv.submit(0, k % 2, big[3000 * k:3000 * k + 9000], 5e-2, seed=k) for k in range(6)]
    for rid in ids:
        _, _, info = srv.wait(rid, timeout=300)
        assert info["state"] == 2
    st = srv.stats()
    assert st["peak_inflight"] <= 2
    assert st["peak_pool_bytes"] <= st["pool_bytes"] and st["pool_used"] == 0
    srv.close()


def test_small_requests_share_launches_and_walk_cap(gpu, meshes):
    probs = problems(gpu)
    bvhs = [b for _, b in meshes]
    srv = gpu.Server(bvhs, probs, pool_bytes=64 << 20, tick_walks=1 << 18, epsilon=1e-3)
    p = points(meshes, 1, 64, seed=9)
    ids = [srv.submit(1, k % 2, p[k:k + 1 + (k % 7)], 1e-2, seed=k) for k in range(40)]
    infos = [srv.wait(rid, timeout=300)[2] for rid in ids]
    st = srv.stats()
    assert all(i["state"] == 2 for i in infos)
    # forty requests, each needing several launches, completed in far fewer launches in total
    assert st["ticks"] < sum(i["ticks"] for i in infos) / 3
    assert st["peak_inflight"] >= 10
    rid = srv.submit(1, 0, p[:5], 1e-6, seed=3, min_walks=32, max_walks=96)
    _, se, info = srv.wait(rid, timeout=120)
    assert info["state"] == 3 and info["walks_per_point"] == 96  # N2W_REQUEST_CAPPED
    srv.close()


def test_nc2lmc_requests_alone_equal_mix_and_unbiased(gpu, meshes):
    from n2w import nc

    probs = problems(gpu)
    bvhs = [b for _, b in meshes]
    m0, m1 = meshes[0][0], meshes[1][0]
    cache = gpu.Cache(gpu.cache_config(log2_hashmap_size=16, max_resolution=256.0))
    nc.train(cache, bvhs[0], probs[0], m0, steps=60, batch=8192, walks_per_label=32, epsilon=1e-3)
    srv = gpu.Server(bvhs, probs, pool_bytes=64 << 20, tick_walks=1 << 17, epsilon=1e-3)
    srv.set_nc(0, 0, cache, *nc.input_box(m0), depth_m=4, residual_fraction=0.25)
    srv.set_nc(1, 1, None, *nc.input_box(m1), depth_m=2, residual_fraction=0.5)
    with pytest.raises(gpu.N2wError, match="no cache registered"):
        srv.submit(1, 0, points(meshes, 1, 4, seed=2), 1e-2, mode="nc2lmc")
    pa = points(meshes, 0, 5000, seed=21)  # chunks of at most 1,024 points: five or more per sweep
    ra = srv.submit(0, 0, pa, 3e-2, seed=5, mode="nc2lmc")
    mean_a, se_a, info_a = srv.wait(ra, timeout=300)
    check_accuracy(gpu, probs[0], pa, mean_a, se_a, info_a, 3e-2)
    assert info_a["residual_walks_per_point"] >= max(2, info_a["walks_per_point"] // 4)
    assert info_a["ticks"] >= 5 * info_a["sweeps"]
    mix = []
    for k, (mesh, prob, n, tgt, mode) in enumerate([(1, 1, 3000, 2e-2, "nc2lmc"), (0, 0, 800, 2e-2, "plain"),
                                                    (1, 1, 50, 1e-2, "plain"), (0, 0, 9, 1e-2, "nc2lmc")]):
        p = points(meshes, mesh, n, seed=40 + k)
        mix.append((srv.submit(mesh, prob, p, tgt, seed=60 + k, mode=mode), prob, p, tgt))
    rb = srv.submit(0, 0, pa, 3e-2, seed=5, mode="nc2lmc")
    mean_b, se_b, info_b = srv.wait(rb, timeout=300)
    assert info_b["walks_per_point"] == info_a["walks_per_point"]
    assert info_b["residual_walks_per_point"] == info_a["residual_walks_per_point"]
    assert info_b["ticks"] == info_a["ticks"]  # the same chunking alone and in the mix
    np.testing.assert_allclose(mean_b, mean_a, rtol=1e-12, atol=1e-14)
    np.testing.assert_allclose(se_b, se_a, rtol=1e-9, atol=1e-14)
    for rid, prob, p, tgt in mix:
        m, s, info = srv.wait(rid, timeout=300)
        check_accuracy(gpu, probs[prob], p, m, s, info, tgt)
    st = srv.stats()
    assert st["completed"] == 6 and st["nc_chunks"] >= 6 and st["nc_walks"] > 0 and st["pool_used"] == 0
    srv.close()
