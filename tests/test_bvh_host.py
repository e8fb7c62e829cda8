"""Host-built 4-wide BVH layout: structural invariants, and the traversal over
it (restated on the CPU) reproduces the reference brute force bit for bit."""
import numpy as np
import pytest

import oracle
from conftest import uniform_box

EMPTY = np.iinfo(np.int32).min


def check_layout(nodes, tris, nt):
    assert sorted(tris["id"].tolist()) == list(range(nt))
    seen = np.zeros(len(tris), bool)
    for ni, nd in enumerate(nodes):
        for k in range(4):
            r = int(nd["child"][k])
            if r == EMPTY:
                assert nd["lo_x"][k] == np.inf and nd["hi_x"][k] == -np.inf
                continue
            lo = np.array([nd["lo_x"][k], nd["lo_y"][k], nd["lo_z"][k]])
            hi = np.array([nd["hi_x"][k], nd["hi_y"][k], nd["hi_z"][k]])
            if r >= 0:
                assert r > ni  # pre-order layout
                continue
            first, count = (~r) >> 3, ((~r) & 7) + 1
            for i in range(first, first + count):
                assert not seen[i]
                seen[i] = True
                for vk in ("v0", "v1", "v2"):
                    assert np.all(tris[vk][i] >= lo) and np.all(tris[vk][i] <= hi)
    assert seen.all()


@pytest.mark.parametrize("method", ["sah", "spatial_median"])
@pytest.mark.parametrize("leaf", [1, 4, 8])
def test_layout_invariants(n2w, method, leaf):
    m = n2w.Mesh.bumpy_sphere_trig(24, 48, 0.08, 6, 8)
    h = n2w.HostBvh(m, leaf, method)
    nodes, tris = h.layout()
    check_layout(nodes, tris, m.counts[1])
    assert h.stats["triangles"] == m.counts[1]


def shell_points(v, t, n, seed, width):
    rng = np.random.default_rng(seed)
    tri = t[rng.integers(0, len(t), n)]
    a, b, c = v[tri[:, 0]], v[tri[:, 1]], v[tri[:, 2]]
    nrm = np.cross(b - a, c - a)
    nrm /= np.linalg.norm(nrm, axis=1, keepdims=True) + 1e-30
    r1, r2 = rng.random((n, 1)), rng.random((n, 1))
    su = np.sqrt(r1)
    q = a * (1 - su) + b * su * (1 - r2) + c * su * r2
    return (q + nrm * rng.uniform(-width, width, (n, 1))).astype(np.float32)


@pytest.mark.parametrize("method,leaf", [("sah", 4), ("sah", 1), ("spatial_median", 8)])
def test_traversal_equals_bruteforce(n2w, bumpy_ref_mesh, golden_closest, method, leaf):
    v, t = bumpy_ref_mesh.arrays()
    h = n2w.HostBvh(bumpy_ref_mesh, leaf, method)
    nodes, tris = h.layout()
    pts = np.concatenate([golden_closest["points"], shell_points(v, t, 500, 3, 1e-3), v[::97]])
    bf = oracle.bruteforce(v, t, pts)
    tr = oracle.traverse4(nodes, tris, pts)
    assert np.array_equal(tr["distance2"].view(np.uint32), bf["distance2"].view(np.uint32))
    assert np.array_equal(tr["closest"].view(np.uint32), bf["closest"].view(np.uint32))
    assert np.array_equal(tr["triangle_id"], bf["triangle_id"])


def test_seeded_traversal_is_exact_for_any_seed(n2w, bumpy_ref_mesh, golden_closest):
    """Seeds are real candidate triangles: whatever they are, the answer is the
    brute-force (d2, lowest id) minimum."""
    v, t = bumpy_ref_mesh.arrays()
    nodes, tris = n2w.HostBvh(bumpy_ref_mesh, 4, "sah").layout()
    n = 16
    slots = np.random.default_rng(5).integers(0, len(tris), (n + 1) ** 3).astype(np.int32)
    seed = (slots, np.array([-1.3, -1.3, -1.3], np.float32), 2.6 / n, n)
    pts = golden_closest["points"]
    tr = oracle.traverse4(nodes, tris, pts, seed=seed)
    bf = oracle.bruteforce(v, t, pts)
    assert np.array_equal(tr["distance2"].view(np.uint32), bf["distance2"].view(np.uint32))
    assert np.array_equal(tr["triangle_id"], bf["triangle_id"])


def test_degenerate_and_duplicate_triangles(n2w):
    # A tetrahedron plus a duplicated face and a zero-area sliver.
    v = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1], [0.5, 0, 0]], np.float32)
    t = np.array([[0, 2, 1], [0, 1, 3], [1, 2, 3], [0, 3, 2], [1, 2, 3], [0, 4, 1]], np.uint32)
    m = n2w.Mesh.from_arrays(v, t)
    assert m.degenerate_count() == 1
    pts = uniform_box(400, 1.5, 11)
    pts[:5] = v
    bf = oracle.bruteforce(v, t, pts)
    for leaf in (1, 2, 8):
        nodes, tris = n2w.HostBvh(m, leaf, "sah").layout()
        tr = oracle.traverse4(nodes, tris, pts)
        assert np.array_equal(tr["distance2"], bf["distance2"])
        assert np.array_equal(tr["triangle_id"], bf["triangle_id"])  # duplicate face -> lowest id


def test_single_triangle_mesh(n2w):
    v = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0]], np.float32)
    m = n2w.Mesh.from_arrays(v, np.array([[0, 1, 2]], np.uint32))
    nodes, tris = n2w.HostBvh(m, 4, "sah").layout()
    assert len(nodes) == 1 and len(tris) == 1
    pts = uniform_box(64, 2.0, 5)
    tr = oracle.traverse4(nodes, tris, pts)
    bf = oracle.bruteforce(v, np.array([[0, 1, 2]], np.uint32), pts)
    assert np.array_equal(tr["distance2"], bf["distance2"]) and np.all(tr["triangle_id"] == 0)


def test_invalid_build_arguments(n2w, bumpy_ref_mesh):
    for leaf in (0, 9):
        with pytest.raises(n2w.N2wError):
            n2w.HostBvh(bumpy_ref_mesh, leaf, "sah")
    with pytest.raises(n2w.N2wError):
        n2w.HostBvh(bumpy_ref_mesh, 4, "rebin_radix")
