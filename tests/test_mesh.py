"""Mesh generators, loaders and normalisation against the reference's own outputs."""
import hashlib
import json

import numpy as np
import pytest

import oracle
from conftest import GOLDEN, REFERENCE_BUNNY


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def test_bumpy_ref_small_matches_reference_golden(n2w):
    g = np.load(GOLDEN / "bumpy_ref_16x32.npz")
    m = n2w.Mesh.bumpy_sphere_ref(16, 32, 0.15)
    v, t = m.arrays()
    assert np.array_equal(v.view(np.uint32), g["vertices_raw"].view(np.uint32))
    assert np.array_equal(t, g["triangles"])
    c, s = m.normalize()
    v2, _ = m.arrays()
    assert np.array_equal(v2.view(np.uint32), g["vertices_normalized"].view(np.uint32))
    assert np.array_equal(c, g["center"]) and np.float32(s) == g["scale"]


def test_bumpy_ref_config_mesh_hash(n2w, bumpy_ref_mesh):
    h = json.loads((GOLDEN / "mesh_hashes.json").read_text())["bumpy_ref_128x256_a0.15_normalized"]
    v, t = bumpy_ref_mesh.arrays()
    assert len(t) == h["triangles"] == 2 * 256 * 127
    assert sha(v) == h["vertices_sha256"]
    assert sha(t) == h["triangles_sha256"]
    assert bumpy_ref_mesh.degenerate_count() == h["degenerate_triangles"]


def test_uv_topology_counts(n2w):
    for stacks, slices in [(32, 64), (128, 256), (256, 512)]:
        m = n2w.Mesh.bumpy_sphere_trig(stacks, slices, 0.08, 6, 8)
        nv, nt = m.counts
        assert nt == 2 * slices * (stacks - 1)
        assert nv == 2 + (stacks - 1) * slices


def test_trig_bumpy_radius_formula(n2w):
    m = n2w.Mesh.bumpy_sphere_trig(16, 32, 0.08, 6, 8)
    v, _ = m.arrays()
    r = np.linalg.norm(v.astype(np.float64), axis=1)
    theta = np.arccos(np.clip(v[:, 2] / r, -1, 1))
    phi = np.arctan2(v[:, 1], v[:, 0])
    expect = 1 + 0.08 * np.sin(6 * theta) * np.cos(8 * phi)
    assert np.allclose(r, expect, atol=2e-5)


def edge_use_counts(t):
    e = np.concatenate([t[:, [0, 1]], t[:, [1, 2]], t[:, [2, 0]]])
    e = np.sort(e, axis=1)
    _, counts = np.unique(e, axis=0, return_counts=True)
    return counts


def test_icosphere_displaced_watertight_and_counts(n2w):
    m = n2w.Mesh.icosphere_displaced(6, 0.12, 3.0, 4, 0.5, 12345)
    nv, nt = m.counts
    assert nt == 20 * 4 ** 6 == 81920
    assert nv == 10 * 4 ** 6 + 2
    _, t = m.arrays()
    assert np.all(edge_use_counts(t) == 2)  # closed 2-manifold
    v, _ = m.arrays()
    r = np.linalg.norm(v, axis=1)
    assert r.min() >= 1 - 0.12 - 1e-6 and r.max() <= 1 + 0.12 + 1e-6
    m.normalize()
    v2, _ = m.arrays()
    assert abs(np.linalg.norm(v2, axis=1).max() - 1.0) < 1e-6


def test_icosphere_seed_changes_surface(n2w):
    a, _ = n2w.Mesh.icosphere_displaced(3, 0.12, 3.0, 4, 0.5, 1).arrays()
    b, _ = n2w.Mesh.icosphere_displaced(3, 0.12, 3.0, 4, 0.5, 2).arrays()
    c, _ = n2w.Mesh.icosphere_displaced(3, 0.12, 3.0, 4, 0.5, 1).arrays()
    assert not np.array_equal(a, b)
    assert np.array_equal(a, c)


def test_uv_sphere_closed(n2w):
    _, t = n2w.Mesh.bumpy_sphere_trig(32, 64, 0.08, 6, 8).arrays()
    assert np.all(edge_use_counts(t) == 2)


def test_invalid_generators_rejected(n2w):
    with pytest.raises(n2w.N2wError):
        n2w.Mesh.bumpy_sphere_ref(3, 32, 0.1)
    with pytest.raises(n2w.N2wError):
        n2w.Mesh.bumpy_sphere_ref(16, 4, 0.1)
    with pytest.raises(n2w.N2wError):
        n2w.Mesh.bumpy_sphere_ref(16, 32, 0.6)
    with pytest.raises(n2w.N2wError):
        n2w.Mesh.from_arrays(np.zeros((3, 3)), np.array([[0, 1, 5]]))


def test_ply_and_obj_roundtrip(n2w, tmp_path):
    v = np.array([[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0], [0.5, 0.5, 1]], np.float32)
    quads = [[0, 1, 2, 3]]
    tris = [[0, 1, 4], [1, 2, 4], [2, 3, 4], [3, 0, 4]]
    obj = tmp_path / "m.obj"
    obj.write_text("# test\n" + "".join(f"v {a} {b} {c}\n" for a, b, c in v) +
                   "f 1/1 2/2 3/3 4/4\n" + "".join(f"f {a+1} {b+1} -1\n" for a, b, _ in tris))
    m = n2w.Mesh.load(str(obj))
    _, t = m.arrays()
    assert t.tolist() == [[0, 1, 2], [0, 2, 3]] + [[a, b, 4] for a, b, _ in tris]
    ply = tmp_path / "m.ply"
    body = "".join(f"{a} {b} {c}\n" for a, b, c in v)
    faces = "".join(f"{len(f)} " + " ".join(map(str, f)) + "\n" for f in quads + tris)
    ply.write_text("ply\nformat ascii 1.0\nelement vertex 5\nproperty float x\nproperty float y\n"
                   "property float z\nelement face 5\nproperty list uchar int vertex_indices\nend_header\n" +
                   body + faces)
    mp = n2w.Mesh.load(str(ply))
    vp, tp = mp.arrays()
    assert np.array_equal(vp, v)
    assert tp.tolist() == [[0, 1, 2], [0, 2, 3]] + tris
    if oracle.ref_available():
        rv, rt = oracle.RefMesh.load_ply(ply).arrays()
        assert np.array_equal(rv, vp) and np.array_equal(rt, tp)
        ov, ot = oracle.RefMesh.load_obj(obj).arrays()
        assert np.array_equal(ot, t)


def test_bad_files_fail_cleanly(n2w, tmp_path):
    p = tmp_path / "bad.ply"
    p.write_text("not a ply\n")
    with pytest.raises(n2w.N2wError):
        n2w.Mesh.load(str(p))
    with pytest.raises(n2w.N2wError):
        n2w.Mesh.load(str(tmp_path / "missing.obj"))


@pytest.mark.skipif(not REFERENCE_BUNNY.exists(), reason="reference bunny mesh not present on this machine")
def test_bunny_ply_matches_reference_loader(n2w):
    h = json.loads((GOLDEN / "mesh_hashes.json").read_text())["bunny_ply"]
    m = n2w.Mesh.load(str(REFERENCE_BUNNY))
    v, t = m.arrays()
    assert len(t) == h["triangles"] and len(v) == h["vertices"]
    assert sha(v) == h["vertices_sha256"] and sha(t) == h["triangles_sha256"]
    c, s = m.normalize()
    v2, _ = m.arrays()
    assert sha(v2) == h["normalized_vertices_sha256"]
    assert np.allclose(c, h["center"]) and abs(s - h["scale"]) < 1e-5
