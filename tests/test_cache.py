"""Neural cache: layout on the CPU; on the GPU, forward and gradients against
the FP64 oracle (oracle/cache_oracle.py), training, checkpoints."""
import numpy as np
import pytest

from oracle import cache_oracle as co


def small_cfg(n2w, **kw):
    base = dict(n_levels=16, log2_hashmap_size=14, base_resolution=16.0, max_resolution=512.0, n_neurons=64,
                n_hidden_layers=2)
    base.update(kw)
    return n2w.cache_config(**base)


def oracle_layout(n2w, cfg):
    d = n2w.cache_describe(cfg)
    lay = co.layout(cfg.n_levels, cfg.log2_hashmap_size, cfg.base_resolution, cfg.max_resolution, 0.0,
                    cfg.n_neurons, cfg.n_hidden_layers, resolutions=d["resolution"])
    return d, lay


def test_default_config_matches_spec(n2w):
    cfg = n2w.cache_config()
    assert (cfg.n_levels, cfg.n_features_per_level, cfg.log2_hashmap_size) == (16, 2, 19)
    assert (cfg.base_resolution, cfg.max_resolution, cfg.n_neurons, cfg.n_hidden_layers) == (16.0, 2048.0, 64, 2)
    assert abs(cfg.learning_rate - 1e-2) < 1e-9
    d = n2w.cache_describe(cfg)
    assert d["resolution"][0] == 16 and d["resolution"][-1] == 2048
    assert np.all(np.diff(d["resolution"]) > 0)
    assert np.all(d["table_size"] <= 1 << 19)
    assert d["mlp_params"] == 64 * 32 + 64 * 64 + 64


@pytest.mark.parametrize("kw", [{}, {"n_levels": 6, "log2_hashmap_size": 13, "n_neurons": 16, "n_hidden_layers": 1},
                                {"n_levels": 12, "n_neurons": 32, "n_hidden_layers": 3}])
def test_layout_matches_oracle(n2w, kw):
    cfg = small_cfg(n2w, **kw)
    d, lay = oracle_layout(n2w, cfg)
    assert d["grid_params"] == lay["grid_params"]
    assert d["mlp_params"] == lay["mlp"]["total"]
    assert list(d["table_size"]) == [lv["size"] for lv in lay["levels"]]


def test_oracle_gradients_match_finite_differences():
    """Pins the FP64 oracle's backward pass by central differences."""
    rng = np.random.default_rng(0)
    lay = co.layout(4, 10, 4.0, 16.0, 0.0, 16, 2)
    n_params = lay["grid_params"] + lay["mlp"]["total"]
    p = rng.normal(scale=0.5, size=n_params)
    u = rng.random((24, 3))
    t = rng.normal(size=24)
    _, g = co.gradients(lay, p, u, t)

    def loss(q):
        y, _ = co.forward(lay, q, u)
        return np.mean((y - t) ** 2)

    used_grid = np.flatnonzero(g[:lay["grid_params"]])
    picks = np.concatenate([rng.choice(used_grid, 20, replace=False),
                            lay["grid_params"] + rng.choice(lay["mlp"]["total"] - 8, 20, replace=False)])
    h = 1e-6
    for i in picks:
        e = np.zeros(n_params)
        e[i] = h
        fd = (loss(p + e) - loss(p - e)) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 + 1e-5 * abs(fd), (i, fd, g[i])


def test_invalid_configs_rejected(n2w):
    for kw in ({"n_neurons": 48}, {"n_hidden_layers": 0}, {"n_levels": 17}, {"n_features_per_level": 4}):
        with pytest.raises(n2w.N2wError):
            n2w.cache_describe(small_cfg(n2w, **kw))


def random_params(cache, rng, grid_scale=0.5):
    p32, _, _ = cache.params()
    info = cache.info()
    G = info["grid_params"]
    p = p32.copy()
    p[:G] = rng.uniform(-grid_scale, grid_scale, G)
    return p


@pytest.mark.gpu
@pytest.mark.parametrize("kw", [{}, {"n_neurons": 32, "n_hidden_layers": 1}, {"n_neurons": 16, "n_hidden_layers": 3},
                                {"n_levels": 8, "n_neurons": 64, "n_hidden_layers": 2}])
def test_forward_matches_oracle(gpu, kw):
    rng = np.random.default_rng(1)
    cfg = small_cfg(gpu, **kw)
    cache = gpu.Cache(cfg)
    cache.set_params(random_params(cache, rng))
    _, p16, _ = cache.params()
    d, lay = oracle_layout(gpu, cfg)
    u = rng.random((3000, 3)).astype(np.float32)
    y = cache.infer(u)
    yo, _ = co.forward(lay, p16.astype(np.float64), u)
    err = np.linalg.norm(y - yo) / (np.linalg.norm(yo) + 1e-12)
    assert err < 2e-2, err


@pytest.mark.gpu
@pytest.mark.parametrize("kw", [{}, {"n_neurons": 32, "n_hidden_layers": 3}])
def test_gradients_match_oracle(gpu, kw):
    """FP16 MMA backward vs the FP64 oracle, evaluated at the FP16 parameters."""
    rng = np.random.default_rng(2)
    cfg = small_cfg(gpu, **kw)
    cache = gpu.Cache(cfg)
    cache.set_params(random_params(cache, rng))
    _, p16, _ = cache.params()
    d, lay = oracle_layout(gpu, cfg)
    u = rng.random((4096, 3)).astype(np.float32)
    t = rng.normal(size=4096).astype(np.float32)
    y, g = cache.gradients(u, t)
    yo, go = co.gradients(lay, p16.astype(np.float64), u, t.astype(np.float64))
    G = lay["grid_params"]
    assert np.linalg.norm(y - yo) / np.linalg.norm(yo) < 2e-2
    for name, sl in (("grid", slice(0, G)), ("mlp", slice(G, None))):
        e = np.linalg.norm(g[sl] - go[sl]) / (np.linalg.norm(go[sl]) + 1e-30)
        assert e < 5e-2, (name, e)


@pytest.mark.gpu
def test_training_fits_a_smooth_field(gpu):
    cfg = small_cfg(gpu)
    cache = gpu.Cache(cfg)
    rng = np.random.default_rng(3)
    n = 16384

    def field(u):
        return np.sin(3 * u[:, 0]) * np.cos(2 * u[:, 1]) + u[:, 2] ** 2

    losses = []
    for step in range(300):
        u = rng.random((n, 3)).astype(np.float32)
        du, dt = gpu.DeviceBuffer.from_array(u), gpu.DeviceBuffer.from_array(field(u).astype(np.float32))
        losses.append(cache.train_step(du.ptr, dt.ptr, n))
    assert losses[-1] < losses[0] / 50, (losses[0], losses[-1])
    u = rng.random((5000, 3)).astype(np.float32)
    assert np.sqrt(np.mean((cache.infer(u) - field(u)) ** 2)) < 0.05


@pytest.mark.gpu
def test_checkpoint_roundtrip(gpu, tmp_path):
    cache = gpu.Cache(small_cfg(gpu))
    rng = np.random.default_rng(4)
    cache.set_params(random_params(cache, rng))
    u = rng.random((1000, 3)).astype(np.float32)
    y = cache.infer(u)
    path = tmp_path / "cache.bin"
    cache.save(str(path))
    other = gpu.Cache.load(str(path))
    assert np.array_equal(other.infer(u), y)
