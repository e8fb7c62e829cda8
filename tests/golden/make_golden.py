"""Generates the golden fixtures in tests/golden/ from the reference's OWN code.

Runs only where the reference checkout is present and oracle/_ref is built
(``python oracle/build.py``).  The outputs are small .npz/.json files that the
tests (CPU and GPU) read without the reference.

Fixtures:
* bumpy_ref_16x32.npz — the reference generator's bumpy sphere (stacks 16,
  slices 32, amplitude 0.15), raw and normalised, with the normalisation.
* analytic_modes.npz — u and f of the reference's analytic modes 13-16 and
  30-32 (its header functions) at 256 seeded points;
* mesh_hashes.json — SHA-256 of the reference generator's normalised
  128x256 bumpy sphere (vertices float32 bytes, triangles uint32 bytes) and of
  the reference PLY loader's output for the bundled bunny mesh.
* closest_golden.npz — 1,536 query points on the normalised 128x256 sphere
  (512 uniform in [-1.2,1.2]^3, 512 on triangles, 512 within 0.05 of the
  surface; numpy seed 20240601) and the reference brute force's
  distance2 / closest / triangle_id for each (src/geometry/closest_point.cpp:50-68).
"""
from __future__ import annotations

import hashlib
import json
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT))

import oracle  # noqa: E402
from oracle import build as ob  # noqa: E402

BUNNY = ob.reference_root() / "meshes" / "bunny_zipper_wataertight.ply"


def sha(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def query_points(v: np.ndarray, t: np.ndarray) -> np.ndarray:
    rng = np.random.default_rng(20240601)
    box = rng.uniform(-1.2, 1.2, (512, 3))
    tri = t[rng.integers(0, len(t), 512)]
    r1, r2 = rng.random(512), rng.random(512)
    su = np.sqrt(r1)
    w = np.stack([1 - su, su * (1 - r2), su * r2], 1)
    surf = (v[tri[:, 0]] * w[:, :1] + v[tri[:, 1]] * w[:, 1:2] + v[tri[:, 2]] * w[:, 2:])
    tri2 = t[rng.integers(0, len(t), 512)]
    cen = (v[tri2[:, 0]] + v[tri2[:, 1]] + v[tri2[:, 2]]) / 3.0
    n = np.cross(v[tri2[:, 1]] - v[tri2[:, 0]], v[tri2[:, 2]] - v[tri2[:, 0]])
    n /= np.linalg.norm(n, axis=1, keepdims=True)
    shell = cen + n * rng.uniform(-0.05, 0.05, (512, 1))
    return np.concatenate([box, surf, shell]).astype(np.float32)


def main() -> None:
    if not oracle.ref_available():
        raise SystemExit("oracle/_ref is not built; run python oracle/build.py with the reference present")
    small = oracle.RefMesh.bumpy_sphere(16, 32, 0.15)
    v_raw, t_small = small.arrays()
    c, s = small.normalize()
    v_norm, _ = small.arrays()
    np.savez_compressed(HERE / "bumpy_ref_16x32.npz", vertices_raw=v_raw, vertices_normalized=v_norm,
                        triangles=t_small, center=c, scale=np.float32(s))

    big = oracle.RefMesh.bumpy_sphere(128, 256, 0.15)
    big.normalize()
    v, t = big.arrays()
    hashes = {"bumpy_ref_128x256_a0.15_normalized": {"vertices_sha256": sha(v), "triangles_sha256": sha(t),
                                                     "vertices": len(v), "triangles": len(t),
                                                     "degenerate_triangles": big.degenerate_count()}}
    if BUNNY.exists():
        bunny = oracle.RefMesh.load_ply(BUNNY)
        bv, bt = bunny.arrays()
        bc, bs = bunny.normalize()
        bvn, _ = bunny.arrays()
        hashes["bunny_ply"] = {"vertices_sha256": sha(bv), "triangles_sha256": sha(bt), "vertices": len(bv),
                               "triangles": len(bt), "normalized_vertices_sha256": sha(bvn),
                               "center": [float(x) for x in bc], "scale": bs}
    nodes, depth = big.host_bvh_stats(8)
    hashes["bumpy_ref_128x256_median_bvh_leaf8"] = {"nodes": nodes, "max_depth": depth}
    (HERE / "mesh_hashes.json").write_text(json.dumps(hashes, indent=2) + "\n")

    pts = query_points(v.astype(np.float64), t)
    d2, cp, ids = big.bruteforce(pts)
    np.savez_compressed(HERE / "closest_golden.npz", points=pts, distance2=d2, closest=cp, triangle_id=ids)
    ap = np.random.default_rng(2024).uniform(-1.1, 1.1, (256, 3)).astype(np.float32)
    modes = {}
    for mode in (13, 14, 15, 16, 30, 31, 32):
        u, f = oracle.ref_analytic(mode, ap)
        modes[f"u_{mode}"], modes[f"f_{mode}"] = u, f
    np.savez_compressed(HERE / "analytic_modes.npz", points=ap, **modes)
    print("wrote golden fixtures to", HERE)


if __name__ == "__main__":
    main()
