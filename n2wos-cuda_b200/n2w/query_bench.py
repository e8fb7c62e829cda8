"""Closest-point query throughput against its roofline (one JSON line).

Workload: the bumpy sphere r = 1 + 0.08 sin(6 theta) cos(8 phi), 128 stacks x
256 slices (65,280 triangles), normalised to unit radius, 4-wide SAH BVH with
leaves of up to 4 triangles; 262,144 query points uniform in [-1.2, 1.2]^3
(PCG64 seed 12345).  Node visits and triangle tests per query are counted by
the counting variant of the query kernel; the timed launches are the plain
n2w_bvh_query_device kernel (CUDA events, median of --repeat launches).

achieved = (12 B in + 28 B out + node visits x 128 B + triangle tests x 48 B)
           / median kernel time, against the measured HBM copy bandwidth.
Every result is checked against the host brute force on --validate points.

    python -m n2w.query_bench [--queries N] [--repeat R] [--block B] [--leaf L]
"""
from __future__ import annotations

import argparse
import json
import sys
from pathlib import Path

import numpy as np


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--queries", type=int, default=262144)
    ap.add_argument("--repeat", type=int, default=20)
    ap.add_argument("--block", type=int, default=128)
    ap.add_argument("--leaf", type=int, default=4)
    ap.add_argument("--method", default="sah")
    ap.add_argument("--extent", type=float, default=1.2)
    ap.add_argument("--validate", type=int, default=2048)
    args = ap.parse_args(argv)

    import n2w
    from n2w._lib import call

    mesh = n2w.Mesh.bumpy_sphere_trig(128, 256, 0.08, 6, 8)
    mesh.normalize()
    bvh = n2w.Bvh(mesh, args.leaf, args.method)
    pts = np.random.default_rng(12345).uniform(-args.extent, args.extent, (args.queries, 3)).astype(np.float32)
    n = len(pts)
    counted = bvh.query(pts, block_size=args.block, counted=True)
    visits = int(counted["node_visits"].astype(np.int64).sum())
    tests = int(counted["tri_tests"].astype(np.int64).sum())

    dp = n2w.DeviceBuffer.from_array(pts)
    dd, dc, di, do = (n2w.DeviceBuffer(4 * n), n2w.DeviceBuffer(12 * n), n2w.DeviceBuffer(4 * n),
                      n2w.DeviceBuffer(4 * n))
    stream = n2w.Stream()
    timer = n2w.Timer()
    for _ in range(3):
        bvh.query_device(dp.ptr, n, dd.ptr, dc.ptr, di.ptr, do.ptr, args.block, stream)
    stream.sync()
    ms = []
    for _ in range(args.repeat):
        timer.start(stream)
        bvh.query_device(dp.ptr, n, dd.ptr, dc.ptr, di.ptr, do.ptr, args.block, stream)
        timer.stop(stream)
        ms.append(timer.ms())
    med = float(np.median(ms))
    d2 = dd.download(np.float32, n, stream)
    ids = di.download(np.int32, n, stream)
    ov = int(do.download(np.int32, n, stream).sum())
    m = min(args.validate, n)
    ref = mesh.closest_point_host(pts[:m])
    bytes_alg = n * (12 + 28) + visits * 128.0 + tests * 48.0
    achieved = bytes_alg / (med / 1e3) / 1e9
    peaks = Path(__file__).resolve().parents[2] / "MEASURED_PEAKS.json"
    if peaks.exists():
        peak, kind = float(json.loads(peaks.read_text())["hbm_gbs"]), "measured"
    else:
        peak, kind = 6650.0, "fallback"
    line = {
        "metric": "closest-point queries/s (262,144 uniform points, bumpy sphere 65,280 tris)",
        "value": n / (med / 1e3), "unit": "queries/s", "kernel_ms_median": med, "kernel_ms": ms,
        "config": {"mesh": "bumpy_sphere_trig(128, 256, 0.08, 6, 8), normalised", "triangles": mesh.counts[1],
                   "queries": n, "extent": args.extent, "leaf_size": args.leaf, "build": args.method,
                   "block_size": args.block, "seed": 12345, "bvh_nodes": bvh.stats["nodes"]},
        "per_query": {"node_visits": visits / n, "tri_tests": tests / n,
                      "algorithmic_bytes": bytes_alg / n},
        "roofline": {"bound": "hbm (working set L2-resident)", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_source": kind},
        "validation": {"checked": m, "triangle_id_mismatch": int(np.sum(ids[:m] != ref["triangle_id"])),
                       "distance2_mismatch": int(np.sum(d2[:m] != ref["distance2"])), "overflow": ov},
    }
    print(json.dumps(line))
    return 0


if __name__ == "__main__":
    sys.exit(main())
