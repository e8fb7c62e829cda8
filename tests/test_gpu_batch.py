"""Batched instances in one persistent launch (through the C ABI).

An instance's estimates must not depend on the rest of the batch: every
instance is compared with a single-problem n2w_wos_estimate on the same points
and seed (walk counts and step totals exactly, FP64 sums to rounding of the
addition order).  Graph replay, autotuning (which changes the launch shape and
queue layout) and accumulation across launches must leave results unchanged;
per-instance means must match the FP64 analytic solution.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def interior_points(gpu, bvh, n, seed, radius=0.6):
    rng = np.random.default_rng(seed)
    pts = rng.uniform(-radius, radius, (4 * n + 64, 3)).astype(np.float32)
    inside = bvh.inside(pts)
    pts = pts[inside.astype(bool)]
    assert len(pts) >= n
    return pts[:n]


@pytest.fixture(scope="module")
def scene3(gpu):
    meshes, bvhs = [], []
    for (st, sl, amp, leaf) in [(16, 32, 0.08, 4), (32, 64, 0.10, 8), (48, 96, 0.06, 4)]:
        m = gpu.Mesh.bumpy_sphere_trig(st, sl, amp, 6, 8)
        m.normalize()
        meshes.append(m)
        bvhs.append(gpu.Bvh(m, leaf, "sah"))
    scene = gpu.Scene(bvhs)
    return meshes, bvhs, scene


def make_instances(gpu, bvhs):
    # (mesh, problem, points, walks per point); one instance has no points
    spec = [(0, 0, 37, 64), (1, 1, 200, 16), (2, 2, 5, 128), (1, 0, 0, 32), (0, 3, 90, 8), (2, 1, 64, 40)]
    inst = []
    for k, (mesh, prob, n, wpp) in enumerate(spec):
        pts = interior_points(gpu, bvhs[mesh], n, seed=100 + k) if n else np.zeros((0, 3), np.float32)
        inst.append({"mesh": mesh, "problem": prob, "points": pts, "walks_per_point": wpp, "seed": 1000 + 17 * k})
    return inst


def problems(gpu):
    return [gpu.problem_charges_seeded(8, 1.6, 2.0, seed=11), gpu.problem_charges_seeded(8, 1.6, 2.0, seed=22),
            gpu.problem_from_name("harmonic_zebra_k4"),
            gpu.problem_sinprod(omega=2 * np.pi * 0.5, source_sampling=gpu.N2W_SOURCE_BALL)]


def single(gpu, bvh, problem, inst, opts):
    o = gpu.walk_options(walks_per_point=inst["walks_per_point"], seed=inst["seed"], epsilon=opts.epsilon,
                         max_steps=opts.max_steps)
    r, _ = gpu.wos_estimate(bvh, problem, inst["points"], options=o)
    return r


def assert_same(batch_r, single_r):
    np.testing.assert_array_equal(batch_r["count"], single_r["count"])
    np.testing.assert_array_equal(batch_r["mean_steps"], single_r["mean_steps"])
    np.testing.assert_array_equal(batch_r["forced"], single_r["forced"])
    np.testing.assert_allclose(batch_r["sum"], single_r["sum"], rtol=1e-12, atol=1e-12)
    np.testing.assert_allclose(batch_r["sum_sq"], single_r["sum_sq"], rtol=1e-12, atol=1e-12)


def test_batch_equals_single_instance_runs(gpu, scene3):
    meshes, bvhs, scene = scene3
    probs = problems(gpu)
    inst = make_instances(gpu, bvhs)
    opts = gpu.walk_options(epsilon=1e-3)
    b = gpu.Batch(scene, probs, inst, opts)
    info = b.info()
    assert info["total_points"] == sum(len(i["points"]) for i in inst)
    b.launch()
    res = b.results()
    cnt = b.run_counters()
    assert cnt["walks"] == info["total_walks"] and cnt["overflow"] == 0
    for k, i in enumerate(inst):
        if not len(i["points"]):
            assert res[k] is None
            continue
        assert_same(res[k], single(gpu, bvhs[i["mesh"]], probs[i["problem"]], i, opts))


def test_graph_replay_autotune_and_accumulate(gpu, scene3):
    meshes, bvhs, scene = scene3
    probs = problems(gpu)
    inst = make_instances(gpu, bvhs)
    b = gpu.Batch(scene, probs, inst, gpu.walk_options(epsilon=1e-3))
    b.launch()
    ref = b.results()
    tune = b.autotune(sample_fraction=0.5)
    best = tune["best"]
    assert best["block_size"] in (64, 128, 256) and best["reg_variant"] in (0, 1)
    assert best["chunk"] in (2, 4, 8, 16) and 1 <= best["regen_threshold"] <= 32
    assert len(tune["trials"]) >= 10 and all(t["ms"] > 0 for t in tune["trials"])
    info = b.info()
    assert (info["block_size"], info["chunk"], info["regen_threshold"]) == (
        best["block_size"], best["chunk"], best["regen_threshold"])
    s = gpu.Stream()
    b.capture_graph(s)
    for _ in range(2):
        b.graph_launch(s)
    s.sync()
    got = b.results(s)
    for r0, r1 in zip(ref, got):
        if r0 is not None:
            assert_same(r1, r0)  # new launch shape, same walks
    # accumulate: two launches with different seeds = sum of both single runs
    b2 = gpu.Batch(scene, probs, inst, gpu.walk_options(epsilon=1e-3, accumulate=1))
    b2.launch()
    seeds2 = [i["seed"] + 5 for i in inst]
    b2.set_seeds(seeds2)
    b2.launch()
    acc = b2.results()
    for k, i in enumerate(inst):
        if not len(i["points"]):
            continue
        a = single(gpu, bvhs[i["mesh"]], probs[i["problem"]], i, gpu.walk_options(epsilon=1e-3))
        c = single(gpu, bvhs[i["mesh"]], probs[i["problem"]], dict(i, seed=seeds2[k]), gpu.walk_options(epsilon=1e-3))
        np.testing.assert_array_equal(acc[k]["count"], a["count"] + c["count"])
        np.testing.assert_allclose(acc[k]["sum"], a["sum"] + c["sum"], rtol=1e-12, atol=1e-12)


def test_batch_instances_match_analytic(gpu, scene3):
    meshes, bvhs, scene = scene3
    probs = problems(gpu)
    inst = [{"mesh": k % 3, "problem": k % 2, "points": interior_points(gpu, bvhs[k % 3], 48, seed=7 + k),
             "walks_per_point": 512, "seed": 99 + k} for k in range(6)]
    b = gpu.Batch(scene, probs, inst, gpu.walk_options(epsilon=1e-4))
    b.launch()
    for i, r in zip(inst, b.results()):
        exact = gpu.problem_exact(probs[i["problem"]], i["points"].astype(np.float64))
        z = (r["mean"] - exact) / np.maximum(r["stderr"], 1e-9)
        # unbiased up to the O(eps) shell bias: pooled z within a few sigma
        assert abs(z.mean()) < 4.0 / np.sqrt(len(z)) + 0.5
        assert np.mean(np.abs(z) < 4) > 0.97


def test_batch_errors(gpu, scene3):
    meshes, bvhs, scene = scene3
    probs = problems(gpu)
    bad = [{"mesh": 7, "problem": 0, "points": np.zeros((1, 3), np.float32), "walks_per_point": 4}]
    with pytest.raises(gpu.N2wError, match="mesh index out of range"):
        gpu.Batch(scene, probs, bad)
    bad = [{"mesh": 0, "problem": 9, "points": np.zeros((1, 3), np.float32), "walks_per_point": 4}]
    with pytest.raises(gpu.N2wError, match="problem index out of range"):
        gpu.Batch(scene, probs, bad)
    ok = [{"mesh": 0, "problem": 0, "points": np.zeros((1, 3), np.float32), "walks_per_point": 4}]
    b = gpu.Batch(scene, probs, ok)
    with pytest.raises(gpu.N2wError, match="no captured graph"):
        b.graph_launch(gpu.Stream())
