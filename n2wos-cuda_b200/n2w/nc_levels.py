"""Cost of the NC+2LMC levels, one call each (one JSON line).

Workload: the headline slice (displaced icosphere L6, z = 0.12 slice 512 x 512
masked to the interior), --points evenly spaced slice points, the manufactured
Poisson problem (sin product, omega = 3 pi) with 16 Green's-function source
samples per ball, eps = 5e-4.  The default cache (16 levels x 2 features, 2^19
entries, 64 x 2 MLP) is trained for --train-steps steps of 65,536 points x
32-walk labels; then the coarse level alone (walks truncated at --depth and
closed by the cache) and the residual level alone (walks continued to the
boundary) each run once untimed and --repeat times timed with CUDA events.

Reported per level: milliseconds per call (best of the timed calls), seconds
per walk, and the per-walk sample variance.  Under a launch-list profiler the
kernels of each call show how a level's time splits between walks and cache
inference.

    python -m n2w.nc_levels [--points N] [--walks W] [--depth M] [--repeat R]
"""
from __future__ import annotations

import argparse
import json
import sys

import numpy as np


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--points", type=int, default=16384)
    ap.add_argument("--walks", type=int, default=256)
    ap.add_argument("--depth", type=int, default=1)
    ap.add_argument("--train-steps", type=int, default=5)
    ap.add_argument("--repeat", type=int, default=1)
    args = ap.parse_args(argv)

    import n2w
    from n2w import nc

    mesh = n2w.Mesh.icosphere_displaced(6, 0.12, 3.0, 4, 0.5, 12345)
    mesh.normalize()
    bvh = n2w.Bvh(mesh, 4, "sah")
    lo, hi = mesh.bounds()
    grid, _ = n2w.slice_points(lo, hi, "xy", 0.12, 512, 512, 0.02, True)
    pts = np.ascontiguousarray(grid[bvh.inside(grid).astype(bool)])
    x = np.ascontiguousarray(pts[np.linspace(0, len(pts) - 1, min(args.points, len(pts))).astype(np.int64)])
    n = len(x)
    problem = n2w.problem_sinprod(3.0 * np.pi, n2w.N2W_SOURCE_BALL)
    problem.source_samples = 16
    cache = n2w.Cache(n2w.cache_config())
    nc.train(cache, bvh, problem, mesh, steps=args.train_steps, batch=65536, walks_per_label=32, epsilon=5e-4)
    dp = n2w.DeviceBuffer.from_array(x)
    timer = n2w.Timer()
    out = {"points": n, "walks_per_point": args.walks, "depth_m": args.depth, "train_steps": args.train_steps,
           "samples_per_call": n * args.walks}
    for name, coarse, resid in (("coarse", args.walks, 0), ("residual", 0, args.walks)):
        o = nc.nc2lmc_options(mesh, coarse_walks=coarse, residual_walks=resid, depth_m=args.depth, epsilon=5e-4,
                              seed=7)
        nc.nc2lmc(bvh, problem, cache, x, o, d_points=dp)  # untimed: one-time scratch mapping
        ms, r = [], None
        for _ in range(max(args.repeat, 1)):
            timer.start()
            r = nc.nc2lmc(bvh, problem, cache, x, o, d_points=dp)
            timer.stop()
            ms.append(timer.ms())
        level = r["coarse"] if coarse else r["residual"]
        out[name] = {"ms_per_call": min(ms), "s_per_walk": min(ms) / 1e3 / (n * args.walks),
                     "var_per_walk": float(np.mean(level["sample_variance"]))}
    print(json.dumps(out))
    return 0


if __name__ == "__main__":
    sys.exit(main())
