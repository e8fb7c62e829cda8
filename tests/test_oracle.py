"""Pins the oracle: its closest-point restatement against the reference's own
outputs (golden vectors from tests/golden/make_golden.py and, when built, the
reference library itself), and its Philox against published known answers."""
import numpy as np
import pytest

import oracle


def test_oracle_bruteforce_matches_reference_golden(bumpy_ref_mesh, golden_closest):
    v, t = bumpy_ref_mesh.arrays()
    r = oracle.bruteforce(v, t, golden_closest["points"])
    assert np.array_equal(r["distance2"].view(np.uint32), golden_closest["distance2"].view(np.uint32))
    assert np.array_equal(r["closest"].view(np.uint32), golden_closest["closest"].view(np.uint32))
    assert np.array_equal(r["triangle_id"], golden_closest["triangle_id"])
    # ties are common on this mesh (shared vertices/edges): the reference keeps the lowest id
    assert (r["ties"] > 1).sum() > 100


@pytest.mark.skipif(not oracle.ref_available(), reason="oracle/_ref not built (reference sources absent)")
def test_oracle_bruteforce_matches_reference_library_live():
    rm = oracle.RefMesh.bumpy_sphere(48, 96, 0.15)
    rm.normalize()
    v, t = rm.arrays()
    pts = np.random.default_rng(7).uniform(-1.3, 1.3, (600, 3)).astype(np.float32)
    pts[:50] = v[:50]  # queries exactly on vertices
    d2, cp, ids = rm.bruteforce(pts)
    r = oracle.bruteforce(v, t, pts)
    assert np.array_equal(d2.view(np.uint32), r["distance2"].view(np.uint32))
    assert np.array_equal(cp.view(np.uint32), r["closest"].view(np.uint32))
    assert np.array_equal(ids, r["triangle_id"])


def test_closest_point_on_triangle_regions():
    a, b, c = np.array([0, 0, 0.]), np.array([1, 0, 0.]), np.array([0, 1, 0.])
    cases = {(-1, -1, 0): a, (2, -0.5, 0): b, (-0.5, 2, 0): c, (0.5, -1, 0): (0.5, 0, 0),
             (-1, 0.5, 0): (0, 0.5, 0), (1, 1, 0): (0.5, 0.5, 0), (0.2, 0.3, 5): (0.2, 0.3, 0)}
    for p, want in cases.items():
        got = oracle.closest_point_on_triangle(p, a, b, c)
        assert np.allclose(got, want, atol=1e-7), (p, got, want)


# Known-answer vectors of Philox4x32-10 from the Random123 distribution
# (counter words, key words -> output words).
PHILOX_KAT = [
    ((0, 0, 0, 0), (0, 0), (0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8)),
    ((0xFFFFFFFF,) * 4, (0xFFFFFFFF, 0xFFFFFFFF), (0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD)),
    ((0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344), (0xA4093822, 0x299F31D0),
     (0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1)),
]


@pytest.mark.parametrize("ctr,key,want", PHILOX_KAT)
def test_oracle_philox_known_answers(ctr, key, want):
    assert tuple(int(x) for x in oracle.philox(ctr, *key)) == want


@pytest.mark.parametrize("ctr,key,want", PHILOX_KAT)
def test_product_philox_known_answers(n2w, ctr, key, want):
    """The walkers' generator (tag 0 keys with the seed words) gives the same answers."""
    from n2w._lib import lib

    c = np.array(ctr, np.uint32)
    out = np.zeros(4, np.uint32)
    seed = key[0] | (key[1] << 32)
    assert lib.n2w_rng_philox4x32_10(c.ctypes.data, seed, 0, out.ctypes.data) == 0
    assert tuple(int(x) for x in out) == want


def test_oracle_wos_unit_ball_harmonic(n2w):
    """Oracle WoS on an icosphere of radius ~1 with harmonic data converges to u."""
    m = n2w.Mesh.icosphere_displaced(4, 0.0, 3.0, 1, 0.5, 1)
    h = n2w.HostBvh(m, 4, "sah")
    nodes, tris = h.layout()
    p = n2w.problem_reference(n2w.N2W_BC["harmonic_x2_minus_y2"])
    pts = np.array([[0.1, 0.2, -0.1], [0.4, -0.3, 0.2], [-0.5, 0.1, 0.3]], np.float32)
    r = oracle.wos(nodes, tris, bytes(p), pts, 4000, 256, 1e-3, 0.999, 1, 2)
    exact = pts[:, 0] ** 2 - pts[:, 1] ** 2
    z = np.abs(r["mean"] - exact) / r["stderr"]
    # tolerance: 4 sigma plus the O(eps) shell bias
    assert np.all(np.abs(r["mean"] - exact) <= 4 * r["stderr"] + 5e-3), (r["mean"], exact, z)
