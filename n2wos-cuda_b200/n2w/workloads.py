"""Seeded synthetic workloads shared by the benchmark, the tests and the
serving loop: the batched-instance set (64 Laplace instances over 4 bumpy
spheres) and its helpers.

Every random choice is drawn from numpy's PCG64 with a recorded seed, so a
workload is reproducible from its parameters alone.
"""
from __future__ import annotations

import numpy as np

# Bumpy spheres r = 1 + 0.08 sin(6 theta) cos(8 phi), normalised to unit radius,
# from coarse to fine (2 * slices * (stacks - 1) triangles each).
BATCH_MESHES = ((32, 64), (64, 128), (128, 256), (256, 512))


def bumpy_sphere(n2w, stacks: int, slices: int):
    m = n2w.Mesh.bumpy_sphere_trig(stacks, slices, 0.08, 6, 8)
    m.normalize()
    return m


def interior_ball_points(bvh, n: int, rng: np.random.Generator, radius: float = 0.9) -> np.ndarray:
    """n points uniform in the ball of the given radius, kept if inside the mesh
    (GPU ray parity); draws in rounds until n are accepted."""
    out = []
    have = 0
    while have < n:
        m = max(2 * (n - have), 256)
        d = rng.normal(size=(m, 3))
        d /= np.linalg.norm(d, axis=1, keepdims=True)
        r = radius * np.cbrt(rng.uniform(size=(m, 1)))
        p = (d * r).astype(np.float32)
        keep = p[bvh.inside(p).astype(bool)]
        out.append(keep)
        have += len(keep)
    return np.ascontiguousarray(np.concatenate(out)[:n])


def log_uniform_int(rng: np.random.Generator, lo: int, hi: int) -> int:
    return int(round(float(np.exp(rng.uniform(np.log(lo), np.log(hi))))))


def batch_workload(n2w, instances: int = 64, points=(256, 65536), walks=(64, 1024), meshes=BATCH_MESHES,
                   seed: int = 2024, problem_pool: int | None = None):
    """64 Laplace instances spread over the meshes, each with its own seeded
    8-charge harmonic boundary (charges on the shell r in [1.6, 2.0],
    amplitudes U[-1, 1]); point counts log-uniform in `points`, walks per
    point log-uniform in `walks`, points uniform in the ball r = 0.9 and
    inside the mesh.  Returns a dict with the meshes, BVHs, scene, problems
    and instance list (Batch input)."""
    rng = np.random.default_rng(seed)
    ms = [bumpy_sphere(n2w, st, sl) for st, sl in meshes]
    bvhs = [n2w.Bvh(m, 4, "sah") for m in ms]
    scene = n2w.Scene(bvhs)
    npb = problem_pool or instances
    problems = [n2w.problem_charges_seeded(8, 1.6, 2.0, seed=int(rng.integers(1, 2**62))) for _ in range(npb)]
    inst = []
    for k in range(instances):
        mesh = k % len(ms)
        n = log_uniform_int(rng, *points)
        w = log_uniform_int(rng, *walks)
        pts = interior_ball_points(bvhs[mesh], n, rng)
        inst.append({"mesh": mesh, "problem": k % npb, "points": pts, "walks_per_point": w,
                     "seed": int(rng.integers(1, 2**62))})
    return {"meshes": ms, "bvhs": bvhs, "scene": scene, "problems": problems, "instances": inst,
            "triangles": [m.counts[1] for m in ms]}


def instance_mse(n2w, problems, instances, results):
    """Per-instance MSE of the estimates against the FP64 analytic solution."""
    out = []
    for inst, r in zip(instances, results):
        if r is None:
            out.append(None)
            continue
        exact = n2w.problem_exact(problems[inst["problem"]], inst["points"].astype(np.float64))
        out.append(float(np.mean((r["mean"] - exact) ** 2)))
    return out
