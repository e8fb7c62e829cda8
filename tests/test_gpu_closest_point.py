"""GPU closest-point parity (through the C ABI) against the oracle and the
reference's own brute-force outputs: distance2, closest point and triangle id
bit-exact (lowest id on exact ties, like the reference brute force)."""
import ctypes as C
import time

import numpy as np
import pytest

import oracle
from conftest import uniform_box

pytestmark = pytest.mark.gpu


def assert_bitexact(got, want):
    assert np.array_equal(got["distance2"].view(np.uint32), want["distance2"].view(np.uint32))
    assert np.array_equal(got["closest"].view(np.uint32), want["closest"].view(np.uint32))
    assert np.array_equal(got["triangle_id"], want["triangle_id"])


@pytest.fixture(scope="module")
def ref_bvh(gpu, bumpy_ref_mesh):
    return gpu.Bvh(bumpy_ref_mesh, 4, "sah")


def test_golden_reference_vectors(gpu, ref_bvh, golden_closest):
    r = ref_bvh.query(golden_closest["points"])
    assert_bitexact(r, golden_closest)
    assert not r["overflow"].any()


@pytest.mark.parametrize("method,leaf", [("sah", 4), ("sah", 1), ("sah", 8), ("spatial_median", 8)])
def test_config0_queries_vs_oracle(gpu, method, leaf):
    """BASELINE config-0 geometry: trig bumpy sphere 128x256, 262,144 uniform
    queries in [-1.2,1.2]^3; all compared with the CPU restatement over the same
    layout, and 2,048 with the brute force."""
    m = gpu.Mesh.bumpy_sphere_trig(128, 256, 0.08, 6, 8)
    m.normalize()
    v, t = m.arrays()
    bvh = gpu.Bvh(m, leaf, method)
    pts = uniform_box(262144, 1.2, 12345)
    r = bvh.query(pts, counted=True)
    nodes, tris = bvh.layout()
    tr = oracle.traverse4(nodes, tris, pts, seed=bvh.seed_grid())
    assert_bitexact(r, tr)
    assert np.array_equal(r["node_visits"], tr["node_visits"])
    assert np.array_equal(r["tri_tests"], tr["tri_tests"])
    # the uncounted launch (long queries finished by whole warps) gives the same answers
    plain = bvh.query(pts)
    assert_bitexact(plain, r)
    assert (plain["overflow"] == 0).all()
    bf = oracle.bruteforce(v, t, pts[:2048])
    sub = {k: r[k][:2048] for k in ("distance2", "closest", "triangle_id")}
    assert_bitexact(sub, bf)
    print(f"ties among 2048 validation points: {(bf['ties'] > 1).sum()}")


def test_seed_grid_holds_nearest_triangles(gpu, ref_bvh, bumpy_ref_mesh):
    slots, lo, h, n = ref_bvh.seed_grid()
    assert n == 128 and len(slots) == 129 ** 3
    nodes, tris = ref_bvh.layout()
    v, t = bumpy_ref_mesh.arrays()
    idx = np.random.default_rng(3).integers(0, len(slots), 3000)
    s = n + 1
    g = np.stack([idx % s, (idx // s) % s, idx // (s * s)], 1).astype(np.float32)
    pts = (lo + np.float32(h) * g).astype(np.float32)
    bf = oracle.bruteforce(v, t, pts)
    assert np.array_equal(tris["id"][slots[idx]], bf["triangle_id"])


def test_query_modes_surface_and_shell(gpu):
    m = gpu.Mesh.icosphere_displaced(5, 0.12, 3.0, 4, 0.5, 7)
    m.normalize()
    v, t = m.arrays()
    bvh = gpu.Bvh(m, 4, "sah")
    rng = np.random.default_rng(9)
    tri = t[rng.integers(0, len(t), 3000)]
    w = rng.dirichlet([1, 1, 1], 3000)
    surf = (v[tri[:, 0]] * w[:, :1] + v[tri[:, 1]] * w[:, 1:2] + v[tri[:, 2]] * w[:, 2:]).astype(np.float32)
    shell = surf * (1 + rng.uniform(-1e-3, 1e-3, (3000, 1))).astype(np.float32)
    pts = np.concatenate([surf, shell, v[:1000]])
    assert_bitexact(bvh.query(pts), oracle.bruteforce(v, t, pts))


def test_masked_query(gpu, ref_bvh, golden_closest):
    pts = golden_closest["points"]
    active = (np.arange(len(pts)) % 3 != 0).astype(np.uint8)
    r = ref_bvh.query(pts, active=active)
    off = active == 0
    assert np.all(r["distance2"][off] == 0) and np.all(r["triangle_id"][off] == -1)
    assert np.array_equal(r["closest"][off], pts[off]) and np.all(r["overflow"][off] == 0)
    on = ~off
    assert np.array_equal(r["distance2"][on], golden_closest["distance2"][on])
    assert np.array_equal(r["triangle_id"][on], golden_closest["triangle_id"][on])


def test_argument_errors(gpu, ref_bvh):
    from n2w._lib import lib

    d = gpu.DeviceBuffer(4096)
    h = ref_bvh.handle
    assert lib.n2w_bvh_query_device(h, d.ptr, 0, d.ptr, d.ptr, d.ptr, d.ptr, 128, None) == 0
    assert lib.n2w_bvh_query_device(h, d.ptr, -1, d.ptr, d.ptr, d.ptr, d.ptr, 128, None) == 1
    assert lib.n2w_bvh_query_device(h, None, 4, d.ptr, d.ptr, d.ptr, d.ptr, 128, None) == 1
    assert lib.n2w_bvh_query_device(h, d.ptr, 4, d.ptr, d.ptr, d.ptr, d.ptr, 0, None) == 1
    assert lib.n2w_bvh_query_device(h, d.ptr, 4, d.ptr, d.ptr, d.ptr, d.ptr, 1025, None) == 1
    assert lib.n2w_bvh_query_device(None, d.ptr, 4, d.ptr, d.ptr, d.ptr, d.ptr, 128, None) == 1


@pytest.mark.parametrize("block", [1, 32, 96, 1024])
def test_block_sizes(gpu, ref_bvh, golden_closest, block):
    assert_bitexact(ref_bvh.query(golden_closest["points"], block_size=block), golden_closest)


def test_inside_classification_matches_reference_rule(gpu):
    m = gpu.Mesh.bumpy_sphere_trig(48, 96, 0.08, 6, 8)
    m.normalize()
    v, t = m.arrays()
    bvh = gpu.Bvh(m, 4, "sah")
    pts = uniform_box(20000, 1.1, 4)
    lo, hi = m.bounds()
    grid, _ = gpu.slice_points(lo, hi, "xy", 0.12, 64, 64)
    pts = np.concatenate([pts, grid])
    got = bvh.inside(pts)
    want = oracle.inside_bruteforce(v, t, pts)
    assert np.array_equal(got, want)
    r = np.linalg.norm(pts, axis=1)
    assert got[r < 0.8].all() and not got[r > 1.0001].any()


@pytest.mark.skipif(not oracle.ref_gpu_available(), reason="reference GPU kernel not built")
def test_reference_gpu_kernel_agrees(gpu, bumpy_ref_mesh, golden_closest):
    """The reference's own GPU kernel (bvh_query.cu, compiled for sm_100a) on the
    same device: distances within its own 2e-4 acceptance of ours."""
    v, t = bumpy_ref_mesh.arrays()
    R = oracle.ref_gpu()
    h = R.ref_gpu_bvh_create(v.ctypes.data, len(v), t.ctypes.data, len(t), 8)
    assert h, R.ref_gpu_last_error()
    try:
        pts = golden_closest["points"]
        n = len(pts)
        dp = gpu.DeviceBuffer.from_array(pts)
        dd, dc, di, do = gpu.DeviceBuffer(4 * n), gpu.DeviceBuffer(12 * n), gpu.DeviceBuffer(4 * n), gpu.DeviceBuffer(4 * n)
        assert R.ref_gpu_query_device(h, dp.ptr, n, dd.ptr, dc.ptr, di.ptr, do.ptr, 128, None) == 0
        d2 = dd.download(np.float32)
        assert np.max(np.abs(np.sqrt(d2) - np.sqrt(golden_closest["distance2"]))) <= 2e-4
    finally:
        R.ref_gpu_bvh_destroy(C.c_void_p(h))


@pytest.mark.parametrize("masked", [False, True])
def test_long_queries_handed_to_warp_finisher_stay_exact(gpu, masked):
    """Points near the centre of a closed mesh are far from the surface in every
    direction, so their traversals run past the per-lane budget and are
    finished by a whole warp from the lane's best so far.  The answers stay
    the brute force's bit for bit (lowest id on ties), no overflow slot is left
    marked, and queries on the surface or far outside (short traversals) in
    the same launch are unaffected."""
    m = gpu.Mesh.bumpy_sphere_trig(128, 256, 0.08, 6, 8)
    m.normalize()
    bvh = gpu.Bvh(m, 4, "sah")
    v, t = m.arrays()
    rng = np.random.default_rng(77)
    centre = rng.uniform(-0.25, 0.25, (3000, 3)).astype(np.float32)
    others = rng.uniform(-1.2, 1.2, (3000, 3)).astype(np.float32)
    pts = np.concatenate([centre, others, v[:200]]).astype(np.float32)
    active = None
    if masked:
        active = (rng.random(len(pts)) < 0.8).astype(np.uint8)
    got = bvh.query(pts, active=active)
    want = oracle.bruteforce(v, t, pts)
    sel = np.ones(len(pts), bool) if active is None else active.astype(bool)
    assert np.array_equal(got["distance2"][sel].view(np.uint32), want["distance2"][sel].view(np.uint32))
    assert np.array_equal(got["triangle_id"][sel], want["triangle_id"][sel])
    assert np.array_equal(got["closest"][sel].view(np.uint32), want["closest"][sel].view(np.uint32))
    assert (got["overflow"] == 0).all()
    if active is not None:
        assert (got["triangle_id"][~sel] == -1).all() and (got["distance2"][~sel] == 0).all()
    # the centre queries really are the long ones: many exceed the per-lane budget
    counted = bvh.query(centre[:1024], counted=True)
    work = counted["node_visits"] + counted["tri_tests"]
    assert np.mean(work > 320) > 0.1


def test_degenerate_duplicate_and_single_triangle_meshes(gpu):
    """A tetrahedron with a duplicated face and a zero-area sliver (ties on the
    duplicate resolve to the lower id), and a one-triangle mesh; queries include
    the vertices themselves.  Plain and counted launches equal the brute force."""
    v = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1], [0.5, 0, 0]], np.float32)
    t = np.array([[0, 2, 1], [0, 1, 3], [1, 2, 3], [0, 3, 2], [1, 2, 3], [0, 4, 1]], np.uint32)
    pts = uniform_box(4000, 1.5, 11)
    pts[:5] = v
    for verts, tri in ((v, t), (v[:3], np.array([[0, 1, 2]], np.uint32))):
        m = gpu.Mesh.from_arrays(verts, tri)
        bf = oracle.bruteforce(verts, tri, pts)
        for leaf in (1, 8):
            bvh = gpu.Bvh(m, leaf, "sah")
            for counted in (False, True):
                r = bvh.query(pts, counted=counted)
                assert_bitexact(r, bf)
                assert not r["overflow"].any()


@pytest.mark.parametrize("n", [1, 31, 33, 257, 4099])
def test_ragged_query_counts(gpu, ref_bvh, golden_closest, n):
    """Counts that fill no whole warp or block: every query still answered
    exactly, and nothing past the end is written."""
    from n2w._lib import call

    pts = uniform_box(n, 1.2, 700 + n)
    nodes, tris = ref_bvh.layout()
    want = oracle.traverse4(nodes, tris, pts, seed=ref_bvh.seed_grid())
    assert_bitexact(ref_bvh.query(pts), want)
    # guard words after each output array stay untouched
    dp = gpu.DeviceBuffer.from_array(pts)
    guard = 0x7F7F7F7F
    d2, cp, ids, ov = (gpu.DeviceBuffer.from_array(np.full(k * (n + 8), guard, np.uint32)) for k in (1, 3, 1, 1))
    call("n2w_bvh_query_device", ref_bvh.handle, dp.ptr, n, d2.ptr, cp.ptr, ids.ptr, ov.ptr, 128, None)
    for buf, k in ((d2, 1), (cp, 3), (ids, 1), (ov, 1)):
        tail = buf.download(np.uint32)[k * n:]
        assert (tail == guard).all()
    assert np.array_equal(d2.download(np.float32)[:n].view(np.uint32), want["distance2"].view(np.uint32))
    assert np.array_equal(ids.download(np.int32)[:n], want["triangle_id"])


def test_bunny_mesh_queries_exact(gpu):
    """The reference's bundled bunny (a scanned mesh, 69,663 triangles after
    loading): uniform, surface (triangle centroids) and far-away queries, plain
    and counted launches, against the brute force and the CPU restatement."""
    from conftest import REFERENCE_BUNNY

    if not REFERENCE_BUNNY.exists():
        pytest.fail(f"{REFERENCE_BUNNY} is missing: oracle/build.py stages it from the reference checkout")
    m = gpu.Mesh.load(str(REFERENCE_BUNNY))
    m.normalize()
    v, t = m.arrays()
    rng = np.random.default_rng(77)
    cent = v[t[rng.integers(0, len(t), 600)]].mean(axis=1).astype(np.float32)
    far = (rng.normal(size=(200, 3)) * 1e3).astype(np.float32)
    pts = np.concatenate([uniform_box(1248, 1.3, 78), cent, far]).astype(np.float32)
    bvh = gpu.Bvh(m, 4, "sah")
    plain = bvh.query(pts)
    counted = bvh.query(pts, counted=True)
    bf = oracle.bruteforce(v, t, pts)
    assert_bitexact(plain, bf)
    assert_bitexact(counted, bf)
    nodes, tris = bvh.layout()
    tr = oracle.traverse4(nodes, tris, pts, seed=bvh.seed_grid())
    assert np.array_equal(counted["node_visits"], tr["node_visits"])
    assert np.array_equal(counted["tri_tests"], tr["tri_tests"])
    assert not plain["overflow"].any()
    assert (plain["distance2"][1248:1848] < 1e-8).all()  # the centroids lie on the surface
