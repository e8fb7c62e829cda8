"""GPU walkers (through the C ABI): statistical parity with the oracle's scalar
WoS over 8 seeds, agreement with FP64 analytic solutions, per-sample vs
per-point reduction identity, prefix/residual semantics, deadline and errors,
and size-independent properties of the config-1 slice at its full size."""
import ctypes as C

import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def small_scene(gpu):
    m = gpu.Mesh.bumpy_sphere_trig(32, 64, 0.08, 6, 8)
    m.normalize()
    bvh = gpu.Bvh(m, 4, "sah")
    nodes, tris = bvh.layout()
    pts = np.array([[0.0, 0.0, 0.0], [0.3, -0.2, 0.1], [-0.5, 0.2, -0.3], [0.1, 0.6, 0.2],
                    [0.7, 0.1, -0.1], [-0.2, -0.7, 0.05], [0.05, 0.05, 0.75], [-0.6, -0.4, 0.2]], np.float32)
    return m, bvh, nodes, tris, pts


def run(gpu, bvh, problem, pts, **kw):
    o = gpu.walk_options(**kw)
    return gpu.wos_estimate(bvh, problem, pts, options=o)


def key_words(seed, tag=0):
    k0 = (seed & 0xFFFFFFFF) ^ ((tag * 0x85EBCA6B) & 0xFFFFFFFF)
    k1 = (seed >> 32) ^ ((tag * 0xC2B2AE35) & 0xFFFFFFFF)
    return k0, k1


@pytest.mark.parametrize("problem_name", ["charges_seeded", "harmonic_zebra_k8"])
def test_statistical_parity_with_oracle_8_seeds(gpu, small_scene, problem_name):
    m, bvh, nodes, tris, pts = small_scene
    p = gpu.problem_from_name(problem_name)
    W = 512
    gm, gv, om, ov = [], [], [], []
    for seed in range(1, 9):
        r, cnt = run(gpu, bvh, p, pts, walks_per_point=W, epsilon=1e-3, seed=seed)
        assert cnt["walks"] == W * len(pts) and cnt["overflow"] == 0
        o = oracle.wos(nodes, tris, bytes(p), pts, W, 256, 1e-3, 0.999, *key_words(seed))
        gm.append(r["mean"]); gv.append(r["stderr"] ** 2)
        om.append(o["mean"]); ov.append(o["stderr"] ** 2)
    gm, gv, om, ov = map(np.array, (gm, gv, om, ov))
    # pooled over 8 seeds: |GPU - oracle| within 3 sigma of the combined MC error
    diff = gm.mean(0) - om.mean(0)
    sigma = np.sqrt(gv.mean(0) / 8 + ov.mean(0) / 8)
    assert np.all(np.abs(diff) <= 3 * sigma), (diff, sigma)
    # and against the FP64 analytic solution (plus the O(eps) shell bias)
    from n2w import problem_exact
    exact = problem_exact(p, pts.astype(np.float64))
    assert np.all(np.abs(gm.mean(0) - exact) <= 3 * np.sqrt(gv.mean(0) / 8) + 5e-3)


def test_samples_and_stats_paths_agree(gpu, small_scene):
    """Per-sample outputs reduced on the device equal the fused per-point reduction
    (same Philox streams -> same walks; sums differ only by FP64 addition order)."""
    from n2w._lib import call
    m, bvh, nodes, tris, pts = small_scene
    p = gpu.problem_charges_seeded()
    W = 300
    o = gpu.walk_options(walks_per_point=W, epsilon=1e-3, seed=77, chunk=7)
    r, _ = gpu.wos_estimate(bvh, p, pts, options=o)
    n = len(pts)
    dp = gpu.DeviceBuffer.from_array(pts)
    val, st, fo, ov = (gpu.DeviceBuffer(4 * n * W) for _ in range(4))
    call("n2w_wos_pure_samples", bvh.handle, C.byref(p), dp.ptr, n, C.byref(o), val.ptr, st.ptr, fo.ptr, ov.ptr,
         None)
    call("n2w_device_sync")
    values = val.download(np.float32).reshape(n, W).astype(np.float64)
    steps = st.download(np.int32).reshape(n, W)
    assert np.allclose(values.sum(1), r["sum"], rtol=1e-12, atol=1e-9)
    assert np.allclose((values ** 2).sum(1), r["sum_sq"], rtol=1e-12, atol=1e-9)
    assert np.array_equal(steps.sum(1) / W, r["mean_steps"])
    from n2w import PointStatsBuffers
    stats = PointStatsBuffers.allocate(n)
    call("n2w_reduce_samples", val.ptr, st.ptr, fo.ptr, n, W, stats.struct(), 0, None)
    red = stats.download()
    assert np.allclose(red["sum"], r["sum"], rtol=1e-12, atol=1e-9)
    assert np.array_equal(red["count"], r["count"])


def test_poisson_ball_sampling_unbiased_center_rule_biased(gpu):
    """Non-harmonic source (sin-product, omega = 3 pi): the in-ball Green's
    function sample is unbiased; the reference's centre rule r^2/6 f(x) is not."""
    m = gpu.Mesh.icosphere_displaced(5, 0.12, 3.0, 4, 0.5, 12345)
    m.normalize()
    bvh = gpu.Bvh(m, 4, "sah")
    pts = np.array([[0.0, 0.0, 0.12], [0.2, -0.1, 0.12], [-0.3, 0.25, 0.12], [0.1, 0.4, -0.2]], np.float32)
    from n2w import problem_exact
    ball = gpu.problem_sinprod(3 * np.pi, gpu.N2W_SOURCE_BALL)
    center = gpu.problem_sinprod(3 * np.pi, gpu.N2W_SOURCE_CENTER)
    exact = problem_exact(ball, pts.astype(np.float64))
    rb, _ = run(gpu, bvh, ball, pts, walks_per_point=65536, epsilon=5e-4, seed=3)
    rc, _ = run(gpu, bvh, center, pts, walks_per_point=65536, epsilon=5e-4, seed=3)
    err_b = np.abs(rb["mean"] - exact)
    err_c = np.abs(rc["mean"] - exact)
    assert np.all(err_b <= 4 * rb["stderr"] + 3e-3), (err_b, rb["stderr"])
    assert np.sqrt(np.mean(err_c ** 2)) > 3 * np.sqrt(np.mean(err_b ** 2))


def test_poisson_multi_sample_source_parity_and_variance(gpu, small_scene):
    """K in-ball source samples per ball: GPU vs oracle over 8 seeds (3 sigma), and
    the per-walk variance drops relative to one sample per ball."""
    m, bvh, nodes, tris, pts = small_scene
    W = 512
    p1 = gpu.problem_sinprod(3 * np.pi, gpu.N2W_SOURCE_BALL)
    p4 = gpu.problem_sinprod(3 * np.pi, gpu.N2W_SOURCE_BALL)
    p4.source_samples = 4
    gm, gv, om, ov = [], [], [], []
    for seed in range(1, 9):
        r, _ = run(gpu, bvh, p4, pts, walks_per_point=W, epsilon=1e-3, seed=seed)
        o = oracle.wos(nodes, tris, bytes(p4), pts, W, 256, 1e-3, 0.999, *key_words(seed))
        gm.append(r["mean"]); gv.append(r["stderr"] ** 2)
        om.append(o["mean"]); ov.append(o["stderr"] ** 2)
    gm, gv, om, ov = map(np.array, (gm, gv, om, ov))
    sigma = np.sqrt(gv.mean(0) / 8 + ov.mean(0) / 8)
    assert np.all(np.abs(gm.mean(0) - om.mean(0)) <= 3 * sigma)
    r1, _ = run(gpu, bvh, p1, pts, walks_per_point=8192, epsilon=1e-3, seed=11)
    r4, _ = run(gpu, bvh, p4, pts, walks_per_point=8192, epsilon=1e-3, seed=11)
    assert r4["sample_variance"].mean() < 0.6 * r1["sample_variance"].mean()


def test_reference_poisson_modes_both_rules_unbiased(gpu, small_scene):
    """Harmonic sources (reference modes 30/31): the centre rule is exact and the
    ball sample agrees with it."""
    m, bvh, nodes, tris, pts = small_scene
    from n2w import problem_exact
    for name in ("poisson_multiscale", "poisson_figlike_hf"):
        pc = gpu.problem_from_name(name, gpu.N2W_SOURCE_CENTER)
        pb = gpu.problem_from_name(name, gpu.N2W_SOURCE_BALL)
        ex = problem_exact(pc, pts.astype(np.float64))
        rc, _ = run(gpu, bvh, pc, pts, walks_per_point=16384, epsilon=1e-3, seed=5)
        rb, _ = run(gpu, bvh, pb, pts, walks_per_point=16384, epsilon=1e-3, seed=6)
        for r in (rc, rb):
            assert np.all(np.abs(r["mean"] - ex) <= 4 * r["stderr"] + 3e-3)


def prefix(gpu, bvh, p, pts, mode, **kw):
    from n2w._lib import call
    o = gpu.walk_options(**kw)
    n, W = len(pts), o.walks_per_point
    S = n * W
    dp = gpu.DeviceBuffer.from_array(pts)
    inp, bnd, cont = gpu.DeviceBuffer(12 * S), gpu.DeviceBuffer(4 * S), gpu.DeviceBuffer(4 * S)
    needs, st, fo, ov = gpu.DeviceBuffer(S), gpu.DeviceBuffer(4 * S), gpu.DeviceBuffer(4 * S), gpu.DeviceBuffer(4 * S)
    lo = np.array([-1.05, -1.05, -1.05], np.float32)
    ext = np.array([2.1, 2.1, 2.1], np.float32)
    call("n2w_wos_prefix_samples", bvh.handle, C.byref(p), dp.ptr, n, C.byref(o), mode, lo.ctypes.data,
         ext.ctypes.data, inp.ptr, bnd.ptr, cont.ptr, needs.ptr, st.ptr, fo.ptr, ov.ptr, None)
    call("n2w_device_sync")
    return {"inputs": inp.download(np.float32).reshape(n, W, 3), "boundary": bnd.download(np.float32).reshape(n, W),
            "cont": cont.download(np.float32).reshape(n, W), "needs": needs.download(np.uint8).reshape(n, W),
            "steps": st.download(np.int32).reshape(n, W), "lo": lo, "ext": ext}


def test_prefix_and_residual_semantics(gpu, small_scene):
    m, bvh, nodes, tris, pts = small_scene
    p = gpu.problem_charges_seeded()
    from n2w import problem_exact
    exact = problem_exact(p, pts.astype(np.float64))
    W = 4096
    # depth 0 coarse: every walk needs the cache at its start point, A_0 = 0
    r0 = prefix(gpu, bvh, p, pts, gpu.N2W_WALK_PREFIX, walks_per_point=64, depth_m=0, epsilon=1e-3)
    assert r0["needs"].all() and np.all(r0["boundary"] == 0) and np.all(r0["steps"] == 0)
    want = np.clip((pts - r0["lo"]) / r0["ext"], 0, 1)
    assert np.allclose(r0["inputs"], want[:, None, :], atol=1e-6)
    # depth 8 coarse with the exact cache C = u is unbiased: A_m + u(X_m)
    r8 = prefix(gpu, bvh, p, pts, gpu.N2W_WALK_PREFIX, walks_per_point=W, depth_m=8, epsilon=1e-3, seed=9)
    xm = r8["lo"] + r8["inputs"] * r8["ext"]
    cache = problem_exact(p, xm.reshape(-1, 3).astype(np.float64)).reshape(len(pts), W)
    est = r8["boundary"] + np.where(r8["needs"], cache, 0.0)
    se = est.std(1) / np.sqrt(W)
    assert np.all(np.abs(est.mean(1) - exact) <= 4 * se + 3e-3)
    assert np.all(r8["steps"][r8["needs"] == 1] == 8) and np.all(r8["steps"][r8["needs"] == 0] <= 8)
    # residual with the exact cache has mean ~0; continuation + prefix is a full walk
    rr = prefix(gpu, bvh, p, pts, gpu.N2W_WALK_RESIDUAL, walks_per_point=W, depth_m=8, epsilon=1e-3, seed=10)
    xm = rr["lo"] + rr["inputs"] * rr["ext"]
    cache = problem_exact(p, xm.reshape(-1, 3).astype(np.float64)).reshape(len(pts), W)
    resid = np.where(rr["needs"], rr["cont"] - cache, 0.0)
    assert np.all(np.abs(resid.mean(1)) <= 4 * resid.std(1) / np.sqrt(W) + 3e-3)
    full = np.where(rr["needs"], rr["boundary"] + rr["cont"], rr["boundary"])
    assert np.all(np.abs(full.mean(1) - exact) <= 4 * full.std(1) / np.sqrt(W) + 3e-3)
    assert np.all(rr["boundary"][rr["needs"] == 0] == rr["cont"][rr["needs"] == 0])


def test_combine_kernel(gpu):
    from n2w._lib import call
    rng = np.random.default_rng(0)
    n = 10007
    cache, bnd, cont = (rng.normal(size=n).astype(np.float32) for _ in range(3))
    needs = (rng.random(n) < 0.6).astype(np.uint8)
    bufs = [gpu.DeviceBuffer.from_array(a) for a in (cache, bnd, cont, needs)]
    nc, res = gpu.DeviceBuffer(4 * n), gpu.DeviceBuffer(4 * n)
    call("n2w_wos_combine", *[b.ptr for b in bufs], n, nc.ptr, res.ptr, 128, None)
    assert np.array_equal(nc.download(np.float32), np.where(needs == 1, bnd + cache, bnd))
    assert np.array_equal(res.download(np.float32), np.where(needs == 1, cont - cache, np.float32(0)))


def test_deadline_stops_walkers(gpu, small_scene):
    m, bvh, nodes, tris, pts = small_scene
    p = gpu.problem_charges_seeded()
    big = np.repeat(pts, 512, axis=0)
    r, cnt = run(gpu, bvh, p, big, walks_per_point=4096, epsilon=1e-4, deadline_ns=200_000)
    assert cnt["walks"] < 4096 * len(big)
    assert cnt["timed_out"] > 0
    assert r["count"].sum() == cnt["walks"]


def test_walks_from_outside_points_stay_bounded(gpu, small_scene):
    """A start point outside the closed mesh (e.g. a misclassified sample) must not
    send walks into the unbounded exterior: they stop at the domain box as forced,
    with finite values, in bounded time."""
    m, bvh, nodes, tris, pts = small_scene
    p = gpu.problem_sinprod(3 * np.pi, gpu.N2W_SOURCE_BALL)
    outside = np.array([[1.3, 0.0, 0.0], [0.0, -1.25, 0.3], [0.9, 0.9, 0.9]], np.float32)
    r, cnt = run(gpu, bvh, p, outside, walks_per_point=4096, epsilon=1e-3)
    assert np.all(np.isfinite(r["mean"])) and np.all(np.isfinite(r["sample_variance"]))
    assert cnt["walks"] == 3 * 4096 and cnt["forced"] > 0


def test_invalid_options(gpu, small_scene):
    m, bvh, nodes, tris, pts = small_scene
    p = gpu.problem_charges_seeded()
    for kw in ({"walks_per_point": 0}, {"max_steps": 0}, {"epsilon": 0.0}, {"step_scale": 1.5},
               {"block_size": 48}, {"block_size": 512}):
        with pytest.raises(gpu.N2wError):
            run(gpu, bvh, p, pts, **kw)
    for mode in (17, 29, 33, 99, 102):  # outside the modes 0-16, 30-32, 100-101
        bad = gpu.problem_charges_seeded()
        bad.mode = mode
        with pytest.raises(gpu.N2wError):
            run(gpu, bvh, bad, pts)
    r, cnt = run(gpu, bvh, p, pts[:0])
    assert len(r["mean"]) == 0


@pytest.mark.parametrize("name", ["harmonic_mixture_figlike", "harmonic_mixture_figlike_hf", "poisson_figlike_hf_x5"])
def test_reference_analytic_modes_walk_to_exact(gpu, small_scene, name):
    """The reference's analytic mixtures (13-16) and the x5 Poisson field (32):
    plain WoS (in-ball source sampling) converges to the FP64 solution."""
    m, bvh, nodes, tris, pts = small_scene
    p = gpu.problem_reference(gpu.N2W_BC[name], gpu.N2W_SOURCE_BALL)
    r, cnt = run(gpu, bvh, p, pts, walks_per_point=4096, epsilon=1e-4, seed=3)
    assert cnt["overflow"] == 0
    exact = gpu.problem_exact(p, pts.astype(np.float64))
    assert np.all(np.abs(r["mean"] - exact) <= 4 * r["stderr"] + 2e-3), (r["mean"] - exact, r["stderr"])


def test_config1_full_slice_properties(gpu):
    """The config-1 workload at its full size: displaced icosphere L6 (81,920
    triangles), the z = 0.12 slice of 512 x 512 masked to the interior, the
    manufactured Poisson problem (sin product, omega = 3 pi), eps = 5e-4; 32
    walks per point keep it to a fraction of a second.  Size-independent
    properties over every point: standardized errors (mean - u) / stderr have
    mean ~0 and variance ~1 (32-walk stderr: variance 31/29), the slice MSE
    equals the mean estimator variance (no bias at the statistical scale), the
    same seed reproduces every walk and step count and the means to FP64
    rounding, and a second seed gives uncorrelated errors."""
    m = gpu.Mesh.icosphere_displaced(6, 0.12, 3.0, 4, 0.5, 12345)
    m.normalize()
    bvh = gpu.Bvh(m, 4, "sah")
    lo, hi = m.bounds()
    grid, _ = gpu.slice_points(lo, hi, "xy", 0.12, 512, 512, 0.02, True)
    pts = np.ascontiguousarray(grid[bvh.inside(grid).astype(bool)])
    assert len(pts) > 150000
    p = gpu.problem_sinprod(3.0 * np.pi, gpu.N2W_SOURCE_BALL)
    exact = gpu.problem_exact(p, pts.astype(np.float64))
    kw = dict(walks_per_point=32, epsilon=5e-4, max_steps=256)
    a, ca = run(gpu, bvh, p, pts, seed=101, **kw)
    b, cb = run(gpu, bvh, p, pts, seed=101, **kw)
    c, _ = run(gpu, bvh, p, pts, seed=202, **kw)
    assert ca["walks"] == len(pts) * 32 and ca["overflow"] == 0
    assert np.all(a["count"] == 32)
    assert ca["steps"] == cb["steps"] and np.array_equal(a["mean_steps"], b["mean_steps"])
    np.testing.assert_allclose(b["mean"], a["mean"], rtol=1e-12, atol=1e-12)
    # slice MSE over every point equals the mean estimator variance (the
    # eps-shell bias of points next to the boundary is far below it)
    mse = np.mean((a["mean"] - exact) ** 2)
    ev = np.mean(a["stderr"] ** 2)
    assert abs(mse / ev - 1.0) < 0.05, (mse, ev)
    # standardized errors where the statistical error dominates the shell bias:
    # points whose walks all stop at once next to the boundary have ~0 stderr
    sel = (a["stderr"] > 0.05) & (c["stderr"] > 0.05)
    assert sel.mean() > 0.8, sel.mean()
    za = (a["mean"][sel] - exact[sel]) / a["stderr"][sel]
    zc = (c["mean"][sel] - exact[sel]) / c["stderr"][sel]
    n = int(sel.sum())
    assert abs(za.mean()) < 5.0 / np.sqrt(n) + 0.01, za.mean()
    assert 0.9 < za.var() < 1.3, za.var()
    assert 0.90 < np.mean(np.abs(za) < 1.96) < 0.975, np.mean(np.abs(za) < 1.96)
    assert abs(np.corrcoef(za, zc)[0, 1]) < 5.0 / np.sqrt(n), np.corrcoef(za, zc)[0, 1]


def config0_points(gpu, bvh, n=4096, radius=0.9, seed=2024):
    """Points uniform in the ball of radius `radius`, rejected when the mesh's
    ray-parity test puts them outside, until n are kept."""
    rng = np.random.default_rng(seed)
    kept = []
    while sum(len(k) for k in kept) < n:
        c = rng.uniform(-radius, radius, (4 * n, 3)).astype(np.float32)
        c = c[np.einsum("ij,ij->i", c, c) < radius * radius]
        kept.append(c[bvh.inside(c).astype(bool)])
    return np.ascontiguousarray(np.concatenate(kept)[:n])


def test_config0_wos_at_spec(gpu):
    """Config 0 at its stated size: the 128 x 256 bumpy sphere r = 1 + 0.08 sin(6t)
    cos(8p) (65,024 triangles), normalised; seeded 8-charge shell boundary
    (r in [1.6, 2.0]); 4,096 interior points uniform in r < 0.9; 256 walks,
    eps = 1e-3, 256-step cap.  The slice MSE against the FP64 solution equals
    the estimator variance and the mean error is zero within its Monte Carlo
    error.  (Per-point standardised errors err / stderr are not the test:
    near the boundary a walk's value is strongly skewed -- most walks stop next
    to the start, a few wander far -- so with 256 walks the sample mean and the
    sample spread are correlated and err / stderr has a small positive mean
    even though err has none; the oracle's exact-arithmetic walk shows the same.)"""
    m = gpu.Mesh.bumpy_sphere_trig(128, 256, 0.08, 6, 8)
    m.normalize()
    assert m.counts[1] == 65024
    bvh = gpu.Bvh(m, 4, "sah")
    pts = config0_points(gpu, bvh)
    p = gpu.problem_charges_seeded(8, 1.6, 2.0, 12345)
    r, cnt = gpu.wos_estimate(bvh, p, pts, options=gpu.walk_options(walks_per_point=256, epsilon=1e-3,
                                                                     max_steps=256, seed=7))
    assert cnt["walks"] == 4096 * 256 and cnt["overflow"] == 0 and cnt["forced"] == 0
    exact = gpu.problem_exact(p, pts.astype(np.float64))
    err = r["mean"] - exact
    var = r["stderr"] ** 2
    mse = float(np.mean(err ** 2))
    # points already inside the epsilon shell: every walk stops at once at the
    # same closest point, so there is no variance and the error is O(eps)
    shell = r["stderr"] == 0
    assert shell.sum() < 0.01 * len(pts) and np.all(np.abs(err[shell]) < 0.05)
    # unbiased: the mean error is within 4 sigma of its Monte Carlo error
    assert abs(float(np.mean(err))) <= 4 * np.sqrt(np.sum(var)) / len(err), (np.mean(err), np.mean(var))
    # the slice MSE is the estimator variance (the epsilon-shell bias is far below it)
    assert 0.9 * np.mean(var) < mse < 1.15 * np.mean(var), (mse, np.mean(var))
