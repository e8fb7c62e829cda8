"""Neural-cache estimators on the GPU: interior sampling, online training,
NC+2LMC unbiasedness and variance behaviour (the cache's gain over plain WoS)."""
import ctypes as C

import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def scene(gpu):
    m = gpu.Mesh.bumpy_sphere_trig(48, 96, 0.08, 6, 8)
    m.normalize()
    return m, gpu.Bvh(m, 4, "sah")


def test_sample_interior(gpu, scene):
    from n2w._lib import call
    m, bvh = scene
    lo, hi = m.bounds()
    n = 20000
    d = gpu.DeviceBuffer(12 * n)
    acc = C.c_int64()
    call("n2w_sample_interior", bvh.handle, lo.ctypes.data, hi.ctypes.data, n, 5, d.ptr, C.byref(acc), None)
    assert acc.value == n
    pts = d.download(np.float32).reshape(n, 3)
    v, t = m.arrays()
    assert oracle.inside_bruteforce(v, t, pts[:3000]).all()
    assert np.all(pts >= lo - 1e-6) and np.all(pts <= hi + 1e-6)
    # roughly uniform: octant counts within 10 % of each other
    oct_ = ((pts > 0).astype(int) * [1, 2, 4]).sum(1)
    counts = np.bincount(oct_, minlength=8)
    assert counts.min() > 0.85 * counts.max()


def test_online_training_reduces_loss(gpu, scene):
    from n2w import nc
    m, bvh = scene
    cache = gpu.Cache(gpu.cache_config(log2_hashmap_size=16, max_resolution=256.0))
    p = gpu.problem_charges_seeded()
    losses = nc.train(cache, bvh, p, m, steps=60, batch=8192, walks_per_label=32, epsilon=1e-3)
    assert losses[-10:].mean() < 0.3 * losses[:5].mean()
    # the trained cache approximates the exact solution in the interior
    lo, hi = m.bounds()
    x = np.random.default_rng(0).uniform(-0.5, 0.5, (2000, 3)).astype(np.float32)
    imin, iext = nc.input_box(m)
    y = cache.infer((x - imin) / iext)
    from n2w import problem_exact
    exact = problem_exact(p, x.astype(np.float64))
    # after 60 short steps the cache is far closer to u than a zero predictor
    assert np.sqrt(np.mean((y - exact) ** 2)) < 0.1 * np.sqrt(np.mean(exact ** 2))


def test_nc2lmc_is_unbiased_and_cache_cuts_residual_variance(gpu, scene):
    from n2w import nc, problem_exact
    m, bvh = scene
    p = gpu.problem_charges_seeded()
    pts = np.random.default_rng(1).uniform(-0.45, 0.45, (64, 3)).astype(np.float32)
    exact = problem_exact(p, pts.astype(np.float64))
    # an untrained cache (~0 output) still gives an unbiased 2LMC estimate
    raw = gpu.Cache(gpu.cache_config(log2_hashmap_size=16, max_resolution=256.0))
    o = nc.nc2lmc_options(m, coarse_walks=2048, residual_walks=2048, depth_m=4, epsilon=1e-3)
    r0 = nc.nc2lmc(bvh, p, raw, pts, o)
    z = (r0["mean"] - exact) / r0["stderr"]
    assert np.all(np.abs(z) < 4.5), z
    # after training, the residual variance drops well below the untrained one
    trained = gpu.Cache(gpu.cache_config(log2_hashmap_size=16, max_resolution=256.0))
    nc.train(trained, bvh, p, m, steps=80, batch=8192, walks_per_label=32, epsilon=1e-3)
    r1 = nc.nc2lmc(bvh, p, trained, pts, o)
    z1 = (r1["mean"] - exact) / r1["stderr"]
    assert np.all(np.abs(z1) < 4.5), z1
    v0 = r0["residual"]["sample_variance"].mean()
    v1 = r1["residual"]["sample_variance"].mean()
    assert v1 < 0.5 * v0, (v0, v1)


def test_nc_wos_only_is_biased_without_cache(gpu, scene):
    """Coarse level alone (NC-WoS) inherits the cache's bias: with an untrained
    cache it misses u(X_m) and is far from the exact value."""
    from n2w import nc, problem_exact
    m, bvh = scene
    p = gpu.problem_charges_seeded()
    pts = np.array([[0.1, 0.0, 0.0], [-0.2, 0.1, 0.2]], np.float32)
    raw = gpu.Cache(gpu.cache_config(log2_hashmap_size=16, max_resolution=256.0))
    o = nc.nc2lmc_options(m, coarse_walks=4096, residual_walks=0, depth_m=2, epsilon=1e-3)
    r = nc.nc2lmc(bvh, p, raw, pts, o)
    exact = problem_exact(p, pts.astype(np.float64))
    assert np.any(np.abs(r["mean"] - exact) > 10 * r["stderr"])


def test_progressive_snapshots(gpu, scene):
    """n2w_nc_progressive: blocks estimated with frozen snapshots while the
    training cache advances.  Without training, overlapped and serial runs give
    the same pooled estimate; with training, the pooled estimate is unbiased,
    holds every block's samples, and theta_infer ends on theta_train's final
    parameters (the last block does not train)."""
    from n2w import nc, problem_exact
    m, bvh = scene
    p = gpu.problem_charges_seeded()
    pts = np.random.default_rng(3).uniform(-0.45, 0.45, (48, 3)).astype(np.float32)
    exact = problem_exact(p, pts.astype(np.float64))
    cfg = gpu.cache_config(log2_hashmap_size=16, max_resolution=256.0)
    to = nc.train_options(m, batch=8192, walks_per_label=16, epsilon=1e-3, seed=11)
    eo = nc.nc2lmc_options(m, coarse_walks=512, residual_walks=256, depth_m=2, epsilon=1e-3, seed=5)
    frozen = [nc.progressive(gpu.Cache(cfg), gpu.Cache(cfg), bvh, p, pts, to, eo, blocks=3,
                             train_steps_per_block=0, overlap=ov) for ov in (True, False)]
    np.testing.assert_allclose(frozen[0]["mean"], frozen[1]["mean"], rtol=1e-12, atol=1e-14)
    np.testing.assert_allclose(frozen[0]["stderr"], frozen[1]["stderr"], rtol=1e-9, atol=1e-14)
    fresh = gpu.Cache(cfg).params()[0]
    for overlap in (True, False):
        theta_train, theta_infer = gpu.Cache(cfg), gpu.Cache(cfg)
        r = nc.progressive(theta_train, theta_infer, bvh, p, pts, to, eo, blocks=3, train_steps_per_block=10,
                           overlap=overlap)
        assert np.all(r["coarse"]["count"] == 3 * 512) and np.all(r["residual"]["count"] == 3 * 256)
        z = (r["mean"] - exact) / r["stderr"]
        assert np.all(np.abs(z) < 4.5), z
        final_train, final_infer = theta_train.params()[0], theta_infer.params()[0]
        assert np.array_equal(final_train, final_infer)
        assert not np.array_equal(final_train, fresh)
        b = r["blocks"]
        assert len(b) == 3 and b[0]["train_ms"] > 0 and b[1]["train_ms"] > 0 and b[2]["train_ms"] == 0
        assert all(x["eval_ms"] > 0 and x["wall_ms"] >= max(x["eval_ms"], x["train_ms"]) * 0.999 for x in b)
    with pytest.raises(gpu.N2wError):
        same = gpu.Cache(cfg)
        nc.progressive(same, same, bvh, p, pts, to, eo, blocks=2)
