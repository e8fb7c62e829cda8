"""Pins the oracle's reference-path pieces on the CPU.

* The displaced icosphere and slice grids the oracle generates equal the
  product's bit for bit, so the reference arm of the bench walks the same
  workload without loading the product library.
* The restated closest_point_bvh_kernel traversal (src/cuda/bvh_query.cu:75-160)
  over the reference's own median-split host BVH (bvh_build_host.cpp) returns
  the brute-force distance bit for bit; triangle ids differ only on exact ties.
* The BVH-culled ray-parity mask equals the reference's brute-force mask.
* The per-sample walk modes (pure, prefix, 2LMC prefix+continuation;
  cubql_bvh.cu:1422-1606), the combine kernel (1608-1627) and the label update
  (1372-1420) obey their defining identities.
"""
import numpy as np
import pytest

import oracle

needs_ref = pytest.mark.skipif(not oracle.ref_available(), reason="oracle/_ref not built (reference sources absent)")


@pytest.fixture(scope="module")
def ico5(n2w):
    v, t = oracle.icosphere_displaced(5, 0.12, 3.0, 4, 0.5, 12345)
    return v, t


def test_icosphere_matches_product(n2w, ico5):
    v, t = ico5
    m = n2w.Mesh.icosphere_displaced(5, 0.12, 3.0, 4, 0.5, 12345)
    v2, t2 = m.arrays()
    assert np.array_equal(v.view(np.uint32), v2.view(np.uint32))
    assert np.array_equal(t, t2)
    assert len(t) == 20 * 4 ** 5


@pytest.mark.parametrize("rule", [oracle.SLICE_RULE_RENDER, oracle.SLICE_RULE_EVAL])
@pytest.mark.parametrize("view,plane", [("xy", 0.12), ("xz", -0.3), ("yz", 0.0)])
def test_slice_points_match_product(n2w, rule, view, plane):
    from n2w._lib import call
    import ctypes as C

    b = np.array([-0.93, -0.81, -1.02, 0.97, 0.88, 0.99], np.float32)
    W, H = 61, 47
    got, fr = oracle.slice_points(b, view, plane, W, H, 0.02, True, rule)
    want = np.empty((H * W, 3), np.float32)
    fw = np.empty(4, np.float32)
    call("n2w_slice_points_ex", b.ctypes.data_as(C.c_void_p), None, view.encode(), C.c_float(plane), W, H,
         C.c_float(0.02), 1, rule, want.ctypes.data_as(C.c_void_p), fw.ctypes.data_as(C.c_void_p))
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
    assert np.array_equal(fr, fw)


@needs_ref
def test_reference_bvh_query_matches_bruteforce(ico5):
    v, t = ico5
    rm = oracle.RefMesh.from_arrays(v, t)
    rm.normalize()
    v, t = rm.arrays()
    bvh = rm.host_bvh(8)
    assert bvh.nodes["count"].max() <= 8 and len(bvh.idx) == len(t)
    rng = np.random.default_rng(11)
    pts = np.concatenate([rng.uniform(-1.2, 1.2, (1500, 3)), v[rng.integers(0, len(v), 100)]]).astype(np.float32)
    q = oracle.ref_bvh_query(bvh, pts)
    bf = oracle.bruteforce(v, t, pts)
    assert np.array_equal(q["distance2"].view(np.uint32), bf["distance2"].view(np.uint32))
    diff = q["triangle_id"] != bf["triangle_id"]
    assert np.all(bf["ties"][diff] > 1)  # a BVH keeps the first visited triangle of an exact tie
    assert (q["node_visits"] > 0).all() and (q["tri_tests"] > 0).all()


@needs_ref
def test_reference_bvh_mask_matches_bruteforce(ico5):
    v, t = ico5
    rm = oracle.RefMesh.from_arrays(v, t)
    rm.normalize()
    v, t = rm.arrays()
    bvh = rm.host_bvh(8)
    b6 = np.concatenate([v.min(0), v.max(0)])
    grid, _ = oracle.slice_points(b6, "xy", 0.12, 96, 96, 0.02, True)
    fast = oracle.inside_ref_bvh(bvh, grid)
    slow = oracle.inside_bruteforce(v, t, grid)
    assert np.array_equal(fast, slow)
    assert 0 < fast.sum() < len(grid)


@needs_ref
def test_reference_bvh_walk_equals_product_layout_walk(n2w, ico5):
    """The same walks (key, walk ids) over two BVHs of one mesh: the closest
    distances are identical, so the walks and their sums are identical."""
    v, t = ico5
    rm = oracle.RefMesh.from_arrays(v, t)
    rm.normalize()
    v, t = rm.arrays()
    rbvh = rm.host_bvh(8)
    h = n2w.HostBvh(n2w.Mesh.from_arrays(v, t), 4, "sah")
    nodes, tris = h.layout()
    p = n2w.problem_sinprod(3.0 * np.pi, n2w.N2W_SOURCE_BALL)
    pts = np.array([[0.1, 0.2, 0.12], [-0.3, 0.1, 0.12], [0.0, -0.5, 0.12]], np.float32)
    a = oracle.wos_ref_bvh(rbvh, bytes(p), pts, 64, 256, 5e-4, 0.999, 5, 9)
    b = oracle.wos(nodes, tris, bytes(p), pts, 64, 256, 5e-4, 0.999, 5, 9)
    assert np.array_equal(a["steps"], b["steps"])
    assert np.allclose(a["sum"], b["sum"], rtol=0, atol=1e-9)


@pytest.fixture(scope="module")
def walk_scene(n2w):
    m = n2w.Mesh.bumpy_sphere_trig(24, 48, 0.08, 6, 8)
    m.normalize()
    h = n2w.HostBvh(m, 4, "sah")
    nodes, tris = h.layout()
    pts = np.array([[0.0, 0.0, 0.0], [0.3, -0.2, 0.1], [-0.5, 0.2, -0.3], [0.1, 0.6, 0.2]], np.float32)
    return nodes, tris, pts


def test_pure_samples_equal_per_point_sums(n2w, walk_scene):
    nodes, tris, pts = walk_scene
    p = n2w.problem_sinprod(3.0 * np.pi, n2w.N2W_SOURCE_BALL)
    W = 32
    s = oracle.walk_samples(nodes, tris, bytes(p), pts, W, oracle.MODE_PURE, 0, 256, 1e-3, 0.999, 3, 4)
    r = oracle.wos(nodes, tris, bytes(p), pts, W, 256, 1e-3, 0.999, 3, 4)
    vals = s["value"].reshape(len(pts), W).astype(np.float64)
    assert np.allclose(vals.sum(1), r["sum"], rtol=0, atol=1e-9)
    assert np.array_equal(s["steps"].reshape(len(pts), W).sum(1), r["steps"])
    assert (s["needs_cache"] == 0).all()


def test_prefix_and_residual_modes(n2w, walk_scene):
    nodes, tris, pts = walk_scene
    p = n2w.problem_sinprod(3.0 * np.pi, n2w.N2W_SOURCE_CENTER)
    W, m = 16, 3
    lo, ext = np.full(3, -1.1, np.float32), np.full(3, 2.2, np.float32)
    pure = oracle.walk_samples(nodes, tris, bytes(p), pts, W, oracle.MODE_PURE, 0, 256, 1e-3, 0.999, 7, 8, lo, ext)
    pre = oracle.walk_samples(nodes, tris, bytes(p), pts, W, oracle.MODE_PREFIX, m, 256, 1e-3, 0.999, 7, 8, lo, ext)
    res = oracle.walk_samples(nodes, tris, bytes(p), pts, W, oracle.MODE_RESIDUAL, m, 256, 1e-3, 0.999, 7, 8, lo,
                              ext)
    # same key and walk ids: the three modes share their first m steps
    needs = pre["needs_cache"].astype(bool)
    assert np.array_equal(needs, res["needs_cache"].astype(bool))
    assert np.array_equal(pre["inputs"], res["inputs"])
    assert (pre["steps"][needs] == m).all() and (res["steps"][needs] >= m).all()
    # walks that stopped before depth m are whole walks in all three modes
    assert np.array_equal(pre["value"][~needs], pure["value"][~needs])
    assert np.array_equal(res["value"][~needs], pure["value"][~needs])
    assert np.array_equal(res["continuation"][~needs], res["value"][~needs])
    # the residual's prefix value is the coarse walk's A_m
    assert np.array_equal(res["value"][needs], pre["value"][needs])
    # prefix + continuation is a whole walk from the same start: identical
    # directions for the first m steps, so the step counts of the residual walk
    # equal the pure walk's
    assert np.array_equal(res["steps"], pure["steps"])
    assert np.allclose(res["value"] + np.where(needs, res["continuation"], 0.0), pure["value"], atol=2e-5)
    assert ((res["inputs"] >= 0) & (res["inputs"] <= 1)).all()


def test_combine_matches_definition():
    rng = np.random.default_rng(3)
    n = 1000
    c, b, w = (rng.normal(size=n).astype(np.float32) for _ in range(3))
    needs = (rng.random(n) < 0.6).astype(np.uint8)
    nc, res = oracle.nc_combine(c, b, w, needs)
    m = needs.astype(bool)
    assert np.array_equal(nc[m], b[m] + c[m]) and np.array_equal(nc[~m], b[~m])
    assert np.array_equal(res[m], w[m] - c[m]) and (res[~m] == 0).all()


def test_label_update_running_average(n2w, walk_scene):
    nodes, tris, pts = walk_scene
    p = n2w.problem_charges_seeded(8, 1.6, 2.0, 12345)
    lo, ext = np.full(3, -1.1, np.float32), np.full(3, 2.2, np.float32)
    n = len(pts)
    tg, cnt = np.zeros(n, np.float32), np.zeros(n, np.int32)
    labels = []
    for refresh, key in enumerate([(1, 2), (3, 4)]):
        inp = oracle.nc_update_labels(nodes, tris, bytes(p), pts, 40, 256, 1e-3, 0.999, *key, 1, lo, ext, tg, cnt)
        labels.append(oracle.wos(nodes, tris, bytes(p), pts, 40, 256, 1e-3, 0.999, *key)["mean"])
    assert (cnt == 80).all()
    np.testing.assert_allclose(tg, (labels[0] + labels[1]) / 2, rtol=0, atol=2e-6)
    np.testing.assert_allclose(inp, (pts - lo) / ext, rtol=0, atol=1e-6)
    tg2, cnt2 = np.zeros(n, np.float32), np.zeros(n, np.int32)
    oracle.nc_update_labels(nodes, tris, bytes(p), pts, 40, 256, 1e-3, 0.999, 1, 2, 0, lo, ext, tg2, cnt2)
    from n2w import problem_eval_f32
    assert (cnt2 == 1).all()
    assert np.array_equal(tg2, problem_eval_f32(p, pts)[0])
