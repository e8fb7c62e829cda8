#!/usr/bin/env python3
"""Benchmark of the B200 Walk-on-Spheres hot path (one JSON line on rank 0).

Workload (one "step"): plain WoS, Poisson -Lap u = f with the manufactured
solution u = sin(w x) sin(w y) sin(w z), w = 2 pi * 1.5, f = 3 w^2 u, Dirichlet
g = u, on the seeded displaced icosphere (subdivision 6, 81,920 triangles,
4-octave value noise, amplitude 0.12, base frequency 3, persistence 0.5,
normalised to unit radius).  Evaluation points: the z = 0.12 slice, 512 x 512
grid masked to the interior (GPU ray parity), 1,024 walks per point,
epsilon = 5e-4, 256-step cap, FP32 walkers, FP64 per-point sums, in-ball
Green's-function source sampling.  MSE is against the FP64 analytic u.

value      = walk-steps (ball moves) of all ranks / max-over-ranks device time
e2e        = same metric through the C ABI with host buffers: pinned H2D of the
             points and D2H of the per-point FP64 sums inside the timed region
roofline   = walker kernel: algorithmic bytes (node fetches x 128 B + triangle
             tests x 48 B + point I/O) / kernel time, against the measured HBM
             copy bandwidth (the BVH working set is L2-resident; see traffic)
cpu_baseline = the oracle's scalar WoS port (same walk, CPU BVH) on the host
             cores, bounded sample of the same workload

--impl reference runs the reference path's CPU implementation (the oracle port
of nc_wos_from_point over a CPU BVH; the reference's own walker exists only as
GPU code built on cuBQL, which is not vendored) on rank 0 and prints its line.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import subprocess
import sys
import tempfile
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT / "n2wos-cuda_b200"))
sys.path.insert(0, str(ROOT))

METRIC = "walk-steps/s (plain WoS, Poisson sin-product, icosphere L6, z=0.12 slice 512x512 x 1024 walks)"
UNIT = "walk-steps/s"
CONFIG = {
    "workload": "plain WoS Poisson manufactured solution on displaced icosphere L6 (81,920 tris), "
                "z=0.12 slice 512x512 masked to interior, 1024 walks/point, eps=5e-4, max_steps=256",
    "mesh": "icosphere_displaced(level=6, amp=0.12, freq=3, octaves=4, persistence=0.5, seed=12345)",
    "slice": {"view": "xy", "plane": 0.12, "width": 512, "height": 512, "padding": 0.02},
    "walks_per_point": 1024, "epsilon": 5e-4, "max_steps": 256, "omega": "3*pi",
    "source_sampling": "ball", "l2": "flushed between timed steps (256 MiB memset)",
}
MEASURED_PEAKS = ROOT / "MEASURED_PEAKS.json"


def peaks():
    if MEASURED_PEAKS.exists():
        d = json.loads(MEASURED_PEAKS.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def traffic_per_walk_step():
    """DRAM bytes per walk-step of walker_kernel from the committed ncu summary
    (dram__bytes_read.sum + dram__bytes_write.sum of a small capture divided by
    its walk-steps; traffic grows in proportion to walk-steps)."""
    p = ROOT / "profiles" / "walker_kernel_icosphere_slice_4096pts.md"
    if p.exists():
        for line in p.read_text().splitlines():
            if line.startswith("traffic_bytes_per_walk_step:"):
                return float(line.split(":")[1])
    return None


class ClockSampler:
    """nvidia-smi sampling of SM clocks and throttle reasons during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.dev = device_index
        self.proc = None
        self.path = Path(tempfile.mkstemp(prefix="n2w_clocks_", suffix=".csv")[1])

    def __enter__(self):
        try:
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.dev}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.fh,
                                         stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            self.fh.close()

    def summary(self) -> dict:
        rows = []
        if self.path.exists():
            for line in self.path.read_text().splitlines():
                parts = [p.strip() for p in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def build_scene(n2w, lib, call):
    mesh = n2w.Mesh.icosphere_displaced(6, 0.12, 3.0, 4, 0.5, 12345)
    mesh.normalize()
    bvh = n2w.Bvh(mesh, 4, "sah")
    lo, hi = mesh.bounds()
    grid, frame = n2w.slice_points(lo, hi, "xy", 0.12, 512, 512, 0.02, True)
    inside = bvh.inside(grid).astype(bool)
    pts = np.ascontiguousarray(grid[inside])
    problem = n2w.problem_sinprod(3.0 * np.pi, n2w.N2W_SOURCE_BALL)
    exact = n2w.problem_exact(problem, pts.astype(np.float64))
    return mesh, bvh, pts, problem, exact, frame


REF_SAMPLE_STRIDE = 256  # the CPU legs walk every 256th interior slice point


def loaded_libraries() -> list[str]:
    """Shared objects of this repository mapped into the process (/proc/self/maps)."""
    found = set()
    try:
        for line in Path("/proc/self/maps").read_text().splitlines():
            path = line.split()[-1] if line.split() else ""
            if path.endswith(".so") and path.startswith(str(ROOT)):
                found.add(str(Path(path).relative_to(ROOT)))
    except OSError:
        pass
    return sorted(found)


def reference_cpu_scene():
    """The headline workload rebuilt without the product library: the oracle's
    displaced icosphere, normalised by the reference's own normalize_to_unit_radius
    and indexed by the reference's own median-split host BVH (leaf 8), both from
    its sources compiled into oracle/_ref; the slice grid and the reference's
    ray-parity mask from the oracle; the sin-product problem record."""
    import oracle

    if not oracle.ref_available():
        raise RuntimeError("oracle/_ref (the reference's CPU sources) is not built")
    v, t = oracle.icosphere_displaced(6, 0.12, 3.0, 4, 0.5, 12345)
    rm = oracle.RefMesh.from_arrays(v, t)
    rm.normalize()
    v, t = rm.arrays()
    bvh = rm.host_bvh(8)
    b6 = np.concatenate([v.min(0), v.max(0)]).astype(np.float32)
    grid, _ = oracle.slice_points(b6, "xy", 0.12, 512, 512, 0.02, True, oracle.SLICE_RULE_RENDER)
    pts = np.ascontiguousarray(grid[oracle.inside_ref_bvh(bvh, grid).astype(bool)])
    problem = oracle.problem_record(101, 0, np.float32(3.0 * np.pi), 0)
    return bvh, pts, problem


def reference_cpu_sample(scene, walks, seed=12345, threads=None):
    """The reference path's CPU form on a fixed sample of the workload: every
    REF_SAMPLE_STRIDE-th interior slice point x `walks` walks, the oracle's port
    of nc_wos_from_point (src/cuda/cubql_bvh.cu:1323-1357) whose closest points
    come from its port of closest_point_bvh_kernel (src/cuda/bvh_query.cu:75-160)
    over the reference's host BVH, on all host threads."""
    import oracle

    bvh, pts, problem = scene
    sel = np.ascontiguousarray(pts[::REF_SAMPLE_STRIDE])
    threads = threads or os.cpu_count() or 1
    t0 = time.perf_counter()
    r = oracle.wos_ref_bvh(bvh, problem, sel, walks, 256, 5e-4, 0.999, seed & 0xFFFFFFFF, seed >> 32, threads)
    dt = time.perf_counter() - t0
    steps = float(r["steps"].sum())
    return {"value": steps / dt, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": (f"every {REF_SAMPLE_STRIDE}th of the {len(pts)} interior slice points ({len(sel)} points) x "
                       f"{walks} walks = {steps:.4g} walk-steps in {dt:.2f} s; reference median-split host BVH "
                       "(leaf 8, bvh_build_host.cpp built from its sources) walked by the oracle's ports of "
                       "closest_point_bvh_kernel and nc_wos_from_point")}


def cache_level_peaks(call):
    """L1 and L2 read bandwidth measured live by the library's own probe kernels
    (n2w_probe_read_bandwidth): the denominators for the traversal's bytes,
    which are L1 / L2 hits, beside the HBM copy peak."""
    out = {}
    for level, key, nbytes, iters in ((1, "l1_gbs", 0, 4096), (2, "l2_gbs", 32 << 20, 64)):
        g = C.c_double()
        try:
            call("n2w_probe_read_bandwidth", level, nbytes, iters, C.byref(g))
            out[key] = g.value
        except Exception as e:  # a probe failure must not break the bench line
            out[key] = None
            out[key + "_error"] = str(e)
    return out


def fractions(achieved_gbs, hbm_peak, cache_peaks):
    fr = {"hbm": achieved_gbs / hbm_peak}
    for key, lvl in (("l2_gbs", "l2"), ("l1_gbs", "l1")):
        if cache_peaks.get(key):
            fr[lvl] = achieved_gbs / cache_peaks[key]
    return fr


def closest_point_segment(n2w, call, stream, timer, flush, cache_peaks, repeat=20, validate=2048,
                          reference_kernel=True, n=262144):
    """Config-0 closest-point queries: 262,144 points uniform in [-1.2, 1.2]^3
    (PCG64 seed 12345) on the bumpy sphere r = 1 + 0.08 sin(6 theta) cos(8 phi),
    128 x 256 (65,024 triangles), normalised; 4-wide SAH BVH, leaves of <= 4.
    Each timed launch of n2w_bvh_query_device follows a 256 MiB L2 flush and is
    timed with CUDA events on its stream.  Algorithmic bytes per query:
    12 in + 28 out + node visits x 128 + triangle tests x 48 (counts from the
    counting variant of the same traversal).  Beside it, as a baseline, the
    reference's own closest_point_bvh_kernel (src/cuda/bvh_query.cu:75-160,
    median-split BVH, leaf 8, block 128), compiled from its sources for sm_100a,
    on the same points with the same flush."""
    mesh = n2w.Mesh.bumpy_sphere_trig(128, 256, 0.08, 6, 8)
    mesh.normalize()
    bvh = n2w.Bvh(mesh, 4, "sah")
    pts = np.random.default_rng(12345).uniform(-1.2, 1.2, (n, 3)).astype(np.float32)
    counted = bvh.query(pts, counted=True)
    visits = float(counted["node_visits"].astype(np.int64).sum())
    tests = float(counted["tri_tests"].astype(np.int64).sum())
    dp = n2w.DeviceBuffer.from_array(pts, stream)
    dd, dc, di, do = (n2w.DeviceBuffer(4 * n), n2w.DeviceBuffer(12 * n), n2w.DeviceBuffer(4 * n),
                      n2w.DeviceBuffer(4 * n))

    def timed(launch):
        for _ in range(3):
            launch()
        stream.sync()
        ms = []
        for _ in range(repeat):
            flush.zero(stream)
            timer.start(stream)
            launch()
            timer.stop(stream)
            ms.append(timer.ms())
        return ms

    ms = timed(lambda: bvh.query_device(dp.ptr, n, dd.ptr, dc.ptr, di.ptr, do.ptr, 128, stream))
    d2 = dd.download(np.float32, n, stream)
    ids = di.download(np.int32, n, stream)
    ref = mesh.closest_point_host(pts[:validate])
    bytes_q = n * (12 + 28) + visits * 128.0 + tests * 48.0
    med = float(np.median(ms))
    achieved = bytes_q / (med / 1e3) / 1e9
    hbm, hbm_kind = peaks()
    seg = {"workload": f"{n:,} queries uniform in [-1.2,1.2]^3 (PCG64 seed 12345), bumpy sphere "
                       "r=1+0.08 sin6t cos8p 128x256 normalised (65,024 triangles), 4-wide SAH BVH leaf<=4, "
                       "L2 flushed before every timed launch",
           "queries_per_s": n / (med / 1e3), "kernel_ms_median": med, "kernel_ms_min": float(np.min(ms)),
           "per_query": {"node_visits": visits / n, "tri_tests": tests / n, "algorithmic_bytes": bytes_q / n},
           "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
                        "peak_source": hbm_kind, "fractions": fractions(achieved, hbm, cache_peaks),
                        "kernel": "closest_point_kernel"},
           "validation": {"checked": validate,
                          "triangle_id_mismatch": int(np.sum(ids[:validate] != ref["triangle_id"])),
                          "distance2_mismatch": int(np.sum(d2[:validate] != ref["distance2"]))},
           "gpu_launches": repeat}
    if reference_kernel:
        seg["reference_kernel"] = reference_kernel_leg(mesh, pts, dp, d2, stream, timed)
        rk = seg["reference_kernel"]
        if rk.get("queries_per_s"):
            seg["speedup_vs_reference_kernel"] = seg["queries_per_s"] / rk["queries_per_s"]
    return seg


def reference_kernel_leg(mesh, pts, dp, d2_ours, stream, timed):
    """Baseline leg: the reference's closest_point_bvh_kernel through its own
    CudaBvh::query_device (oracle/_ref/libn2wos_ref_gpu.so, built from
    src/cuda/bvh_query.cu + bvh_build_host.cpp), same device points."""
    import oracle

    if not oracle.ref_gpu_available():
        return {"unavailable": "oracle/_ref/libn2wos_ref_gpu.so not built"}
    import n2w

    R = oracle.ref_gpu()
    v, t = mesh.arrays()
    h = R.ref_gpu_bvh_create(v.ctypes.data, len(v), t.ctypes.data, len(t), 8)
    if not h:
        return {"unavailable": R.ref_gpu_last_error().decode()}
    n = len(pts)
    dd, dc, di, do = (n2w.DeviceBuffer(4 * n), n2w.DeviceBuffer(12 * n), n2w.DeviceBuffer(4 * n),
                      n2w.DeviceBuffer(4 * n))
    try:
        def launch():
            if R.ref_gpu_query_device(h, dp.ptr, n, dd.ptr, dc.ptr, di.ptr, do.ptr, 128, stream.handle) != 0:
                raise RuntimeError(R.ref_gpu_last_error().decode())
        ms = timed(launch)
        d2 = dd.download(np.float32, n, stream)
        ov = int(do.download(np.int32, n, stream).sum())
    finally:
        R.ref_gpu_bvh_destroy(h)
    med = float(np.median(ms))
    return {"kernel": "closest_point_bvh_kernel (reference src/cuda/bvh_query.cu:75-160), median-split BVH leaf 8, "
                      "block 128, compiled from its sources for sm_100a",
            "queries_per_s": n / (med / 1e3), "kernel_ms_median": med, "overflow": ov,
            "distance2_equal_to_ours": int(np.sum(d2 == d2_ours)), "queries": n}


def time_to_mse(n2w, lib, call, mesh, bvh, pts, exact, problem, target=1e-4, sub=16384, train_steps=200,
                real_stride=4, real_cap_s=60.0):
    """Time for the slice MSE against the FP64 analytic u to reach `target`:
    this project's plain GPU WoS against NC+2LMC (cache trained online from WoS
    labels; coarse walks truncated at depth m and closed by the cache; the
    unbiased residual level continues fewer walks to the boundary).

    (1) Per-walk cost (CUDA events) and variance on an evenly spaced subsample
        of the slice, for plain WoS with 1 and with 16 Green's-function source
        samples per ball, and for NC+2LMC (16 samples) at depths 1, 2, 4, 8
        with the trained cache and with the exact solution in place of the
        cache.  With cost c and variance V per walk at each level, the best
        allocation reaches MSE e in (sqrt(Vc cc) + sqrt(Vr cr))^2 / e per point.
        The exact-solution column is the bound for any cache: the residual
        level then carries E[Var(W | X_m)] at full-walk cost.
    (2) Measured: on every `real_stride`-th slice point, walk blocks are added
        until the measured MSE against the FP64 solution is below `target`:
        plain WoS with 16 source samples, and NC+2LMC at the trained cache's
        best depth with its optimal residual fraction (training time
        included).  Times are CUDA-event sums over the blocks, scaled by
        `real_stride` to the full slice (the cost is linear in the points; the
        MSE is a mean over points, which the subsample estimates)."""
    from n2w import nc

    P = len(pts)
    sel = np.linspace(0, P - 1, min(sub, P)).astype(np.int64)
    x = np.ascontiguousarray(pts[sel])
    n = len(x)
    dp = n2w.DeviceBuffer.from_array(x)
    t = n2w.Timer()
    st = n2w.PointStatsBuffers.allocate(n)
    ws = n2w.DeviceBuffer(lib.n2w_wos_workspace_bytes(n))
    W = 256
    out = {"target_mse": target, "subsample_points": n, "slice_points": P, "walks_measured_per_point": W}

    def plain(pb):
        o = n2w.walk_options(walks_per_point=W, epsilon=5e-4, seed=1)
        ms = None
        for _ in range(2):
            t.start()
            call("n2w_wos_estimate", bvh.handle, C.byref(pb), dp.ptr, n, C.byref(o), st.struct(), None, ws.ptr, None)
            t.stop()
            ms = t.ms()
        r = st.download()
        tw, var = ms / 1e3 / (n * W), float(np.mean(r["sample_variance"]))
        # per-point (Neyman) allocation of walks: N_i proportional to sqrt(V_i)
        neyman = P * tw * float(np.mean(np.sqrt(r["sample_variance"]))) ** 2 / target
        return {"s_per_walk": tw, "var_per_walk": var, "seconds_extrapolated": nc.time_to_mse(target, P * tw, var, 0.0),
                "seconds_per_point_allocation": neyman}

    out["plain_wos"] = plain(problem)
    p16 = n2w.problem_sinprod(3.0 * np.pi, n2w.N2W_SOURCE_BALL)
    p16.source_samples = 16
    out["plain_wos_16_source_samples"] = plain(p16)
    var16 = out["plain_wos_16_source_samples"]["var_per_walk"]
    t16 = out["plain_wos_16_source_samples"]["s_per_walk"]

    cache = n2w.Cache(n2w.cache_config())
    t.start()
    losses = nc.train(cache, bvh, p16, mesh, steps=train_steps, batch=65536, walks_per_label=32, epsilon=5e-4)
    t.stop()
    train_s = t.ms() / 1e3

    def level(c, m, coarse, resid):
        o = nc.nc2lmc_options(mesh, coarse_walks=coarse, residual_walks=resid, depth_m=m, epsilon=5e-4, seed=7)
        ms, r = [], None
        for _ in range(3):  # best of three (the first includes one-time scratch mapping)
            t.start()
            r = nc.nc2lmc(bvh, p16, c, x, o, d_points=dp)
            t.stop()
            ms.append(t.ms())
        return min(ms) / 1e3 / (n * max(coarse, resid)), r

    levels = {}
    for cache_kind, c in (("trained", cache), ("exact_solution", None)):
        for m in (1, 2, 4, 8):
            tc, rc = level(c, m, W, 0)
            tr, rr = level(c, m, 0, W)
            vc = float(np.mean(rc["coarse"]["sample_variance"]))
            vr = float(np.mean(rr["residual"]["sample_variance"]))
            fixed = train_s if c is not None else 0.0
            opt = fixed + P * (np.sqrt(vc * tc) + np.sqrt(vr * tr)) ** 2 / target
            # per-point allocation of both levels' walks (sqrt(V_c,i t_c) + sqrt(V_r,i t_r) per point)
            opt_pp = fixed + P * float(np.mean(np.sqrt(rc["coarse"]["sample_variance"] * tc) +
                                               np.sqrt(rr["residual"]["sample_variance"] * tr))) ** 2 / target
            levels[f"{cache_kind}_m{m}"] = {
                "cache": cache_kind, "depth_m": m, "s_per_coarse_walk": tc, "s_per_residual_walk": tr,
                "var_coarse": vc, "var_residual": vr, "seconds_optimal_allocation": opt,
                "seconds_per_point_allocation": opt_pp,
                "seconds_residual_1_16": nc.time_to_mse(target, P * (tc + tr / 16), vc + 16 * vr, 0.0, fixed),
                "optimal_residual_fraction": float(np.sqrt((vr / tr) / (vc / tc))),
                "explained_variance_R2": max(0.0, 1.0 - vr / var16),
                "speedup_vs_plain_16_same_walks": (P * var16 * t16 / target) / opt}
    out["nc2lmc_levels"] = levels
    trained = {k: v for k, v in levels.items() if v["cache"] == "trained"}
    bound = {k: v for k, v in levels.items() if v["cache"] == "exact_solution"}
    best = min(trained.values(), key=lambda v: v["seconds_optimal_allocation"])
    best_bound = min(bound.values(), key=lambda v: v["seconds_optimal_allocation"])
    out["nc2lmc_training"] = {"train_s": train_s, "train_steps": train_steps, "train_batch": 65536,
                              "walks_per_label": 32, "source_samples": 16,
                              "loss_first_last": [float(losses[0]), float(losses[-1])]}
    out["extrapolated"] = {
        "speedup_nc2lmc_vs_plain_16_source_samples": out["plain_wos_16_source_samples"]["seconds_extrapolated"] /
        best["seconds_optimal_allocation"],
        "best_trained_depth": best["depth_m"],
        "bound_exact_solution_cache_speedup": best_bound["speedup_vs_plain_16_same_walks"],
        "per_point_allocation_both": out["plain_wos_16_source_samples"]["seconds_per_point_allocation"] /
        min(v["seconds_per_point_allocation"] for v in trained.values()),
        "per_point_allocation_bound_exact_cache": out["plain_wos_16_source_samples"]["seconds_per_point_allocation"] /
        min(v["seconds_per_point_allocation"] for v in bound.values()),
        "bound_depth": best_bound["depth_m"],
        "config2_m8_residual_1_16_speedup_vs_plain_16": out["plain_wos_16_source_samples"]["seconds_extrapolated"] /
        levels["trained_m8"]["seconds_residual_1_16"],
        "one_sample_plain_vs_nc2lmc_16_samples_not_like_for_like": out["plain_wos"]["seconds_extrapolated"] /
        best["seconds_optimal_allocation"]}
    out["measured"] = measured_time_to_mse(n2w, call, bvh, mesh, pts, exact, p16, cache, best, train_s, target,
                                           real_stride, real_cap_s)
    m = out["measured"]
    if m["plain_16"].get("reached") and m["nc2lmc"].get("reached"):
        out["speedup_nc2lmc_vs_plain_16_source_samples"] = m["plain_16"]["seconds_full_slice"] / \
            m["nc2lmc"]["seconds_full_slice"]
    out["progressive_snapshots"] = progressive_overlap(n2w, mesh, bvh, pts, p16)
    return out


def measured_time_to_mse(n2w, call, bvh, mesh, pts, exact, problem, cache, best, train_s, target, stride, cap_s):
    """Adds walk blocks until the slice MSE against the FP64 solution is below
    `target` on every `stride`-th slice point (see time_to_mse)."""
    from n2w import nc

    x = np.ascontiguousarray(pts[::stride])
    ex = exact[::stride]
    n = len(x)
    dp = n2w.DeviceBuffer.from_array(x)
    t = n2w.Timer()
    res = {"points": n, "stride": stride, "target_mse": target, "cap_seconds_subsample": cap_s}

    # plain WoS, 16 source samples, blocks of 1,024 walks per point accumulated on the device
    st = n2w.PointStatsBuffers.allocate(n)
    ws = n2w.DeviceBuffer(n2w._lib.lib.n2w_wos_workspace_bytes(n))
    total_ms, blocks, mse = 0.0, 0, None
    while total_ms / 1e3 < cap_s:
        o = n2w.walk_options(walks_per_point=1024, epsilon=5e-4, seed=1000 + blocks, accumulate=1 if blocks else 0)
        t.start()
        call("n2w_wos_estimate", bvh.handle, C.byref(problem), dp.ptr, n, C.byref(o), st.struct(), None, ws.ptr, None)
        t.stop()
        total_ms += t.ms()
        blocks += 1
        r = st.download()
        mse = float(np.mean((r["mean"] - ex) ** 2))
        if mse < target:
            break
    res["plain_16"] = {"reached": bool(mse is not None and mse < target), "mse": mse, "blocks": blocks,
                       "walks_per_point": 1024 * blocks, "seconds_subsample": total_ms / 1e3,
                       "seconds_full_slice": total_ms / 1e3 * stride}

    # NC+2LMC at the trained cache's best depth with its optimal residual fraction
    m = best["depth_m"]
    frac = min(1.0, max(best["optimal_residual_fraction"], 1.0 / 64))
    wc = 1024
    wr = max(1, int(round(wc * frac)))
    acc = {k: [np.zeros(n), np.zeros(n), np.zeros(n)] for k in ("c", "r")}
    total_ms, blocks, mse = 0.0, 0, None
    while total_ms / 1e3 + train_s / stride < cap_s:
        o = nc.nc2lmc_options(mesh, coarse_walks=wc, residual_walks=wr, depth_m=m, epsilon=5e-4, seed=5000 + blocks)
        t.start()
        r = nc.nc2lmc(bvh, problem, cache, x, o, d_points=dp)
        t.stop()
        total_ms += t.ms()
        blocks += 1
        for k, lv in (("c", r["coarse"]), ("r", r["residual"])):
            acc[k][0] += lv["sum"]
            acc[k][1] += lv["sum_sq"]
            acc[k][2] += lv["count"]
        est = acc["c"][0] / acc["c"][2] + acc["r"][0] / acc["r"][2]
        mse = float(np.mean((est - ex) ** 2))
        if mse < target:
            break
    res["nc2lmc"] = {"reached": bool(mse is not None and mse < target), "mse": mse, "blocks": blocks,
                     "depth_m": m, "coarse_walks_per_point": wc * blocks, "residual_walks_per_point": wr * blocks,
                     "seconds_subsample_walks": total_ms / 1e3, "train_seconds": train_s,
                     "seconds_full_slice": total_ms / 1e3 * stride + train_s}
    return res


def progressive_overlap(n2w, mesh, bvh, pts, problem, blocks=4, train_steps=12):
    """Progressive NC+2LMC over the full slice (n2w_nc_progressive): block k
    estimates with snapshot theta_k (depth 1, 256 coarse + 128 residual walks
    per point) while theta_train takes `train_steps` steps toward theta_{k+1};
    the same work with overlap on two streams and serially.  Reports the wall
    times and the reference's accounting model sum_k max(eval_k, train_{k+1})."""
    from n2w import nc

    cfg = n2w.cache_config()
    to = nc.train_options(mesh, batch=65536, walks_per_label=32, epsilon=5e-4, seed=2024)
    eo = nc.nc2lmc_options(mesh, coarse_walks=256, residual_walks=128, depth_m=1, epsilon=5e-4, seed=7)
    d_pts = n2w.DeviceBuffer.from_array(np.ascontiguousarray(pts, np.float32))
    res = {}
    for overlap in (False, True, False, True):  # second pair timed
        r = nc.progressive(n2w.Cache(cfg), n2w.Cache(cfg), bvh, problem, pts, to, eo, blocks=blocks,
                           train_steps_per_block=train_steps, overlap=overlap, d_points=d_pts)
        res["overlap" if overlap else "serial"] = r["blocks"]
    ser, ovl = res["serial"], res["overlap"]
    # block k evaluates theta_k and trains toward theta_{k+1}: the reference's model time is max of the two
    model = sum(max(b["eval_ms"], b["train_ms"]) for b in ser)
    return {"blocks": blocks, "train_steps_per_block": train_steps, "points": len(pts),
            "walks_per_block": {"coarse": 256, "residual": 128, "depth_m": 1},
            "serial_wall_s": sum(b["wall_ms"] for b in ser) / 1e3,
            "overlap_wall_s": sum(b["wall_ms"] for b in ovl) / 1e3,
            "eval_s": sum(b["eval_ms"] for b in ser) / 1e3, "train_s": sum(b["train_ms"] for b in ser) / 1e3,
            "reference_overlap_model_s": model / 1e3,
            "per_block_overlap": ovl}


def run_reference(args):
    """The reference path's CPU implementation on this arm's workload (rank 0
    only): the headline slice rebuilt by the oracle and the reference's own
    sources (no product code), each step a fixed sample of it (every
    REF_SAMPLE_STRIDE-th interior point x 1,024 walks, a new walk stream per step)."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    try:
        scene = reference_cpu_scene()
    except RuntimeError as e:
        print(json.dumps({"impl": "reference", "unavailable": str(e)}))
        return 0
    vals = []
    for i in range(args.warmup + args.steps):
        s = reference_cpu_sample(scene, 1024, seed=12345 + i)
        if i >= args.warmup:
            vals.append(s)
    steps_per_s = [s["value"] for s in vals]
    value = float(np.mean(steps_per_s))
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": None, "higher_is_better": True,
            "dtype": "f32", "data": "synthetic", "config": dict(CONFIG, points=int(len(scene[1]))),
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": vals[-1]["cores"], "kind": "port",
                             "sample": vals[-1]["sample"]},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "step_values": steps_per_s,
            "libraries_loaded": loaded_libraries(),
            "note": "the reference's walker exists only as GPU code on cuBQL (not vendored); its CPU form here is "
                    "the oracle's port of nc_wos_from_point over the reference's own median-split host BVH "
                    "(oracle/_ref, built from its sources), on every host thread; no product code is loaded"}
    print(json.dumps(line))
    return 0


def run_figure(args):
    """The reference's two published evaluation runs (figures/zebra_k8_m2.json,
    figures/bunny_zebra_k8_m2.json: RTX 3070, cuBQL, tiny-cuda-nn), re-run with
    their exact command lines through this project's n2wos_eval_tcnn_nc_wos
    (output paths redirected; the bunny PLY from the copy staged under
    oracle/_ref).  Reported per run: pure-WoS walk-steps/s (samples x mean steps
    / CUDA-event time) against the published figure, and the published vs
    measured mesh, mask and estimator statistics."""
    import shutil

    golden = json.loads((ROOT / "tests" / "golden" / "figure_runs.json").read_text())
    tool = ROOT / "n2wos-cuda_b200" / "bin" / "n2wos_eval_tcnn_nc_wos"
    bunny = ROOT / "oracle" / "_ref" / "meshes" / "bunny_zipper_wataertight.ply"
    out_dir = Path(tempfile.mkdtemp(prefix="n2w_figure_"))
    runs = {}
    try:
        for name, fig in sorted(golden.items()):
            argv = fig["command_line"].split()[1:]
            fixed, i = [], 0
            while i < len(argv):
                a = argv[i]
                if a in ("--mesh-path", "--save-estimates-prefix", "--output"):
                    val = {"--mesh-path": str(bunny), "--save-estimates-prefix": str(out_dir / name),
                           "--output": str(out_dir / f"{name}.json")}[a]
                    fixed += [a, val]
                    i += 2
                else:
                    fixed.append(a)
                    i += 1
            r = subprocess.run([str(tool), *fixed], capture_output=True, text=True, timeout=1200)
            if r.returncode != 0:
                runs[name] = {"error": r.stderr[-2000:]}
                continue
            js = json.loads((out_dir / f"{name}.json").read_text())
            got, want = js["runs"]["pure_wos"], fig["runs"]["pure_wos"]
            ws = got["samples"] * got["mean_steps"] / (got["elapsed_ms"] / 1e3)
            ws_pub = want["samples"] * want["mean_steps"] / (want["elapsed_ms"] / 1e3)
            runs[name] = {
                "walk_steps_per_s": ws, "published_walk_steps_per_s": ws_pub, "published_device": fig["device"],
                "speedup_vs_published": ws / ws_pub,
                "eval_points": [got["eval_points"], want["eval_points"]],
                "mean_steps": [got["mean_steps"], want["mean_steps"]],
                "mean_sample_variance": [got["mean_sample_variance"], want["mean_sample_variance"]],
                "rmse": [got["rmse"], want["rmse"]], "elapsed_ms": [got["elapsed_ms"], want["elapsed_ms"]],
                "mesh_triangles": [js["mesh_stats"]["triangles"], fig["mesh_stats"]["triangles"]],
                "normalization": [js["mesh_stats"]["normalization"], fig["mesh_stats"]["normalization"]],
                "nc_wos_rmse": [js["runs"]["nc_wos"]["rmse"], fig["runs"]["nc_wos"]["rmse"]],
                "nc_2lmc_rmse": [js["runs"]["nc_2lmc"]["rmse"], fig["runs"]["nc_2lmc"]["rmse"]],
                "training_ms": [js["training"]["total_training_ms"], fig["training"]["total_training_ms"]],
                "pairs": "[this run, published]"}
    finally:
        shutil.rmtree(out_dir, ignore_errors=True)
    head = runs.get("zebra_k8_m2", {})
    line = {"metric": "walk-steps/s (pure WoS, reference figure run zebra_k8_m2: bumpy sphere 65,024 tris, "
                      "harmonic_zebra_k8, z=0 slice 512x512 = 162,215 px x 64 walks, eps=1e-4)",
            "value": head.get("walk_steps_per_s"), "unit": UNIT, "n_gpus": 1, "steps": 1, "warmup": 0,
            "higher_is_better": True, "dtype": "f32", "data": "synthetic (the reference's own procedural mesh and "
            "bundled bunny, its published command lines)",
            "vs_baseline": head.get("speedup_vs_published"),
            "config": {"workload": "reference figure runs zebra_k8_m2 and bunny_zebra_k8_m2, exact command lines"},
            "runs": runs}
    print(json.dumps(line))
    return 0


def run_nc_levels(args):
    """Cost of the NC+2LMC levels, one call each: the headline slice's points
    (--nc-points of them, evenly spaced), the sin-product
    problem with 16 Green's-function source samples per ball, eps = 5e-4; the
    default cache trained for --nc-train-steps steps of 65,536 points x 32-walk
    labels; then the coarse level alone (walks truncated at --nc-depth and closed
    by the cache) and the residual level alone, each once untimed and once timed
    with CUDA events.  Under a launch-list profiler the kernels of each call show
    how a level's time splits between walks and cache inference."""
    import n2w
    from n2w import nc
    from n2w._lib import call, lib

    call("n2w_set_device", int(os.environ.get("LOCAL_RANK", "0")))
    mesh, bvh, pts, _, _, _ = build_scene(n2w, lib, call)
    x = np.ascontiguousarray(pts[np.linspace(0, len(pts) - 1, min(args.nc_points, len(pts))).astype(np.int64)])
    n = len(x)
    problem = n2w.problem_sinprod(3.0 * np.pi, n2w.N2W_SOURCE_BALL)
    problem.source_samples = 16
    cache = n2w.Cache(n2w.cache_config())
    nc.train(cache, bvh, problem, mesh, steps=args.nc_train_steps, batch=65536, walks_per_label=32, epsilon=5e-4)
    dp = n2w.DeviceBuffer.from_array(x)
    timer = n2w.Timer()
    W = args.walks if args.walks != 1024 else 256
    out = {"workload": "nc-levels", "points": n, "walks_per_point": W, "depth_m": args.nc_depth,
           "train_steps": args.nc_train_steps, "samples_per_call": n * W}
    for name, coarse, resid in (("coarse", W, 0), ("residual", 0, W)):
        o = nc.nc2lmc_options(mesh, coarse_walks=coarse, residual_walks=resid, depth_m=args.nc_depth, epsilon=5e-4,
                              seed=7)
        nc.nc2lmc(bvh, problem, cache, x, o, d_points=dp)  # untimed: one-time scratch mapping
        timer.start()
        r = nc.nc2lmc(bvh, problem, cache, x, o, d_points=dp)
        timer.stop()
        level = r["coarse"] if coarse else r["residual"]
        out[name] = {"ms_per_call": timer.ms(), "s_per_walk": timer.ms() / 1e3 / (n * W),
                     "var_per_walk": float(np.mean(level["sample_variance"]))}
    print(json.dumps(out))
    return 0


def run_query(args):
    """The config-0 closest-point segment of the default line on its own, with
    --queries points (the default 262,144 is config 0)."""
    import n2w
    from n2w._lib import call

    call("n2w_set_device", int(os.environ.get("LOCAL_RANK", "0")))
    stream = n2w.Stream()
    seg = closest_point_segment(n2w, call, stream, n2w.Timer(), n2w.DeviceBuffer(256 << 20), cache_level_peaks(call),
                                reference_kernel=not args.no_reference_kernel, n=args.queries)
    print(json.dumps(dict(metric="closest-point queries/s", value=seg["queries_per_s"], unit="queries/s", **seg)))
    return 0


BATCH_METRIC = ("walk-steps/s (64 batched Laplace instances over 4 bumpy spheres, 8-charge harmonic boundaries, "
                "one persistent launch under a CUDA graph)")


def run_batch(args):
    """Batched uneven instances in one persistent launch: 64 Laplace instances
    over 4 bumpy spheres (32/64 .. 256/512 stacks/slices), seeded 8-charge
    boundaries, points log-uniform in 256..65,536, walks per point log-uniform
    in 64..1,024, eps = 1e-3, 256-step cap.  The launch shape comes from the
    batch autotuner; timed launches replay a captured CUDA graph.  Reported
    beside the batched rate: the same instances run one launch each
    (n2w_wos_estimate), and per-instance MSE against the FP64 solution."""
    import n2w
    from n2w import workloads
    from n2w._lib import call, lib

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    call("n2w_set_device", local)
    t0 = time.time()
    wl = workloads.batch_workload(n2w, seed=2024)
    build_s = time.time() - t0
    inst = wl["instances"]
    for k, i in enumerate(inst):  # replicas on several GPUs walk distinct streams
        i["seed"] = i["seed"] + 1000003 * rank
    opts = n2w.walk_options(max_steps=256, epsilon=1e-3, step_scale=0.999)
    b = n2w.Batch(wl["scene"], wl["problems"], inst, opts)
    stream = n2w.Stream()
    t0 = time.time()
    tune = b.autotune(sample_fraction=1.0 / 16, stream=stream)
    tune_s = time.time() - t0
    b.capture_graph(stream)
    flush = n2w.DeviceBuffer(256 << 20)
    timer = n2w.Timer()
    for _ in range(args.warmup):
        b.graph_launch(stream)
        stream.sync()
    times, counters = [], []
    with ClockSampler(local) as clocks:
        call("n2w_device_sync")
        for _ in range(args.steps):
            flush.zero(stream)
            timer.start(stream)
            b.graph_launch(stream)
            timer.stop(stream)
            times.append(timer.ms())
            counters.append(b.run_counters())
        call("n2w_device_sync")
    total_ms = float(np.sum(times))
    c_last = counters[-1]
    steps_done = float(sum(c["steps"] for c in counters))
    value = steps_done / (total_ms / 1e3)
    res = b.results(stream)
    mses = workloads.instance_mse(n2w, wl["problems"], inst, res)

    # the same instances, one launch each (n2w_wos_estimate), for the batching gain
    seq_ms, seq_steps = 0.0, 0
    d_cnt = n2w.DeviceBuffer(C.sizeof(n2w._lib.WalkCounters))
    for i, dp, st in zip(inst, b.points, b.stats):
        if not len(i["points"]):
            continue
        o = n2w.walk_options(walks_per_point=i["walks_per_point"], max_steps=256, epsilon=1e-3, seed=i["seed"])
        timer.start(stream)
        call("n2w_wos_estimate", wl["bvhs"][i["mesh"]].handle, C.byref(wl["problems"][i["problem"]]), dp.ptr,
             len(i["points"]), C.byref(o), st.struct(), d_cnt.ptr, None, stream.handle)
        timer.stop(stream)
        seq_ms += timer.ms()
        seq_steps += int(d_cnt.download(np.uint64, 8, stream)[1])

    # end to end: pinned host points in, per-point FP64 sums out, every step
    total_pts = sum(len(i["points"]) for i in inst)
    hp = C.c_void_p()
    call("n2w_malloc_host", C.byref(hp), max(12 * total_pts, 1))
    off = 0
    for i in inst:
        C.memmove(hp.value + off, i["points"].ctypes.data, i["points"].nbytes)
        off += i["points"].nbytes
    out_bytes = 20 * total_pts
    hout = C.c_void_p()
    call("n2w_malloc_host", C.byref(hout), max(out_bytes, 1))
    e2e_ms, e2e_steps = 0.0, 0.0
    for _ in range(max(1, args.steps)):
        flush.zero(stream)
        timer.start(stream)
        off = 0
        for i, dp in zip(inst, b.points):
            if i["points"].nbytes:
                call("n2w_memcpy_h2d", dp.ptr, C.c_void_p(hp.value + off), i["points"].nbytes, stream.handle)
            off += i["points"].nbytes
        b.graph_launch(stream)
        o8 = 0
        for i, st in zip(inst, b.stats):
            n = len(i["points"])
            if n:
                call("n2w_memcpy_d2h", C.c_void_p(hout.value + o8), st.sum.ptr, 8 * n, stream.handle)
                call("n2w_memcpy_d2h", C.c_void_p(hout.value + o8 + 8 * n), st.sum_sq.ptr, 8 * n, stream.handle)
                call("n2w_memcpy_d2h", C.c_void_p(hout.value + o8 + 16 * n), st.count.ptr, 4 * n, stream.handle)
            o8 += 20 * n
        timer.stop(stream)
        e2e_ms += timer.ms()
        e2e_steps += b.run_counters()["steps"]
    lib.n2w_free_host(hp)
    lib.n2w_free_host(hout)

    kernel_ms = float(np.mean(times))
    alg_bytes = c_last["node_visits"] * 128.0 + c_last["tri_tests"] * 48.0 + total_pts * (12 + 8 + 8 + 4 + 8 + 4)
    achieved = alg_bytes / (kernel_ms / 1e3) / 1e9
    peak, peak_kind = peaks()
    valid = [m for m in mses if m is not None]
    if rank == 0:
        line = {
            "metric": BATCH_METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": "64 Laplace instances, 4 bumpy spheres r=1+0.08 sin6t cos8p "
                                   "(stacks/slices 32/64..256/512), 8-charge shells seeded per instance, "
                                   "points log-uniform 256..65536 in ball r=0.9, walks log-uniform 64..1024, "
                                   "eps=1e-3, max_steps=256",
                       "triangles": wl["triangles"], "points": total_pts,
                       "walks": int(sum(len(i["points"]) * i["walks_per_point"] for i in inst)),
                       "parallelism": f"replicas x{world} (distinct seeds)",
                       "l2": "flushed between timed steps (256 MiB memset)", "seed": 2024},
            "e2e": {"value": e2e_steps / (e2e_ms / 1e3), "unit": UNIT, "h2d_bytes_per_step": 12 * total_pts,
                    "d2h_bytes_per_step": out_bytes},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "traffic": None, "peak_source": peak_kind, "kernel": "walker_kernel<batch>",
                         "bytes_per_launch": alg_bytes, "kernel_ms": kernel_ms},
            "gpu_launches": 3 * args.steps,  # per graph replay: stats zeroing, first queries, walker
            "clocks": clocks.summary(),
            "autotune": {"best": tune["best"], "trials": len(tune["trials"]), "seconds": tune_s,
                         "sample_fraction": 1.0 / 16},
            "sequential_launches": {"walk_steps_per_s": seq_steps / (seq_ms / 1e3), "ms": seq_ms,
                                    "batched_speedup": value / (seq_steps / (seq_ms / 1e3))},
            "accuracy": {"instance_mse_median": float(np.median(valid)), "instance_mse_max": float(np.max(valid)),
                         "instances": len(valid)},
            "setup_seconds": build_s,
            "counters_last_step": c_last,
        }
        print(json.dumps(line))
    return 0


def run_serve(args):
    if not args.serve_rates:
        print(json.dumps(serve_line(args)))
        return 0
    # offered-load sweep: each rate runs --serve-sweep-seconds of Poisson arrivals
    sweep = []
    for rate in [float(r) for r in args.serve_rates.split(",")]:
        a = argparse.Namespace(**vars(args))
        a.serve_rate = rate
        a.serve_requests = max(20, int(rate * args.serve_sweep_seconds))
        a.serve_time_limit = args.serve_sweep_seconds + args.serve_sweep_drain
        line = serve_line(a)
        sweep.append({"offered_req_per_s": rate, "requests": a.serve_requests, "complete": line["complete"],
                      "finished": line["finished_requests"], "latency_s": line["latency_s"],
                      "throughput": line["throughput"], "accuracy": line["accuracy"],
                      "nc2lmc": line["modes"]["nc2lmc"], "server": line["server"], "clocks": line["clocks"]})
        print(f"[serve sweep] rate {rate}: p50 {line['latency_s']['p50']:.3f}s p99<=4096 "
              f"{line['latency_s']['p99_le4096']:.3f}s done {line['finished_requests']}/{a.serve_requests}",
              file=sys.stderr, flush=True)
    sat = [r for r in sweep if not r["complete"] or r["latency_s"]["p99_le4096"] > 10 * sweep[0]["latency_s"]["p99_le4096"]]
    print(json.dumps({"metric": "serving loop p50/p99 latency vs offered load", "value": None, "unit": "s",
                      "n_gpus": 1, "higher_is_better": False, "data": "synthetic",
                      "config": {"workload": "serving sweep (see --workload serve)", "rates": args.serve_rates,
                                 "seconds_of_arrivals_per_rate": args.serve_sweep_seconds},
                      "sweep": sweep,
                      "first_saturated_rate": sat[0]["offered_req_per_s"] if sat else None}))
    return 0


def serve_line(args):
    """Serving loop under mixed load: Poisson arrivals of requests on 4
    device-resident meshes (the config-0 bumpy sphere, the config-1 icosphere,
    the smallest and largest config-3 spheres) with either an 8-charge harmonic
    boundary or the config-1 manufactured Poisson problem; points uniform in
    the interior (ball r = 0.9 masked by the mesh); a fraction of large
    requests.  Each request stops when the root mean square of its per-point
    standard errors meets its target.  A fraction (--serve-nc-fraction) of the
    requests are NC+2LMC requests on the icosphere with the Poisson problem,
    served with a cache trained online before the timed region (depth 1,
    residual walks = 1/2 of the coarse walks).  Latency is measured natively
    (submission -> result ready).  The run stops at --serve-time-limit and
    then reports how many requests had not finished."""
    import threading as th

    import n2w
    from n2w import workloads
    from n2w._lib import N2W_REQUEST_DONE, call

    local = int(os.environ.get("LOCAL_RANK", "0"))
    call("n2w_set_device", local)
    rng = np.random.default_rng(args.serve_seed)
    meshes = [workloads.bumpy_sphere(n2w, 128, 256), n2w.Mesh.icosphere_displaced(6, 0.12, 3.0, 4, 0.5, 12345),
              workloads.bumpy_sphere(n2w, 32, 64), workloads.bumpy_sphere(n2w, 256, 512)]
    meshes[1].normalize()
    bvhs = [n2w.Bvh(m, 4, "sah") for m in meshes]
    pool_pts = [workloads.interior_ball_points(b, 65536, rng) for b in bvhs]
    problems = [n2w.problem_charges_seeded(8, 1.6, 2.0, seed=2024), n2w.problem_sinprod(3.0 * np.pi, n2w.N2W_SOURCE_BALL)]
    problems[1].source_samples = args.serve_source_samples  # variance reduction of the Poisson source term
    srv = n2w.Server(bvhs, problems, tick_walks=args.serve_tick_walks, epsilon=1e-3, chunk=args.serve_chunk,
                     tick_walks_max=max(args.serve_tick_walks_max, args.serve_tick_walks))
    nc_train = None
    if args.serve_nc_fraction > 0:
        from n2w import nc

        cache = n2w.Cache(n2w.cache_config())
        tt = time.perf_counter()
        losses = nc.train(cache, bvhs[1], problems[1], meshes[1], steps=args.serve_nc_train_steps, batch=65536,
                          walks_per_label=32, epsilon=1e-3)
        nc_train = {"seconds": time.perf_counter() - tt, "steps": args.serve_nc_train_steps, "batch": 65536,
                    "walks_per_label": 32, "loss_first_last": [float(losses[0]), float(losses[-1])]}
        srv.set_nc(1, 1, cache, *nc.input_box(meshes[1]), depth_m=1, residual_fraction=0.5)
    N = args.serve_requests
    arrivals = np.cumsum(rng.exponential(1.0 / args.serve_rate, N))
    reqs = []
    for k in range(N):
        large = rng.uniform() < args.serve_large_fraction
        lo, hi = (4096, args.serve_large_max) if large else (1, 4096)
        n = min(workloads.log_uniform_int(rng, lo, hi), 65536)
        mesh = int(rng.integers(0, 4))
        prob = int(rng.uniform() < args.serve_poisson_fraction)
        mode = "nc2lmc" if rng.uniform() < args.serve_nc_fraction else "plain"
        if mode == "nc2lmc":
            mesh, prob = 1, 1
        tgt = 1e-3 if (prob == 0 and n <= 256 and rng.uniform() < 0.5) else 1e-2
        off = int(rng.integers(0, 65536 - n + 1))
        reqs.append({"t": float(arrivals[k]), "n": n, "mesh": mesh, "problem": prob, "target": tgt, "off": off,
                     "seed": int(rng.integers(1, 2**62)), "mode": mode})
    ids = [None] * N
    stop = th.Event()
    errors = []
    t0 = time.perf_counter()

    def submitter():
        try:
            for k, r in enumerate(reqs):
                while not stop.is_set():
                    dt = r["t"] - (time.perf_counter() - t0)
                    if dt <= 0:
                        break
                    time.sleep(min(dt, 0.05))
                if stop.is_set():
                    return
                pts = pool_pts[r["mesh"]][r["off"]:r["off"] + r["n"]]
                ids[k] = srv.submit(r["mesh"], r["problem"], pts, r["target"], seed=r["seed"],
                                    max_walks=args.serve_max_walks, rms=True, mode=r["mode"])
        except Exception as e:  # surfaced by the collector below
            errors.append(e)
            stop.set()

    sub = th.Thread(target=submitter, daemon=True)
    deadline = t0 + args.serve_time_limit
    results = []
    last = t0
    outstanding = {}  # request index -> id, submitted and not yet collected
    next_k = 0
    with ClockSampler(local) as clocks:
        sub.start()
        while len(results) < N and not errors:
            now = time.perf_counter()
            if now > deadline:
                break
            if now - last > 5.0:
                st = srv.stats()
                print(f"[serve] t={now - t0:.0f}s done={len(results)}/{N} submitted={st['submitted']} "
                      f"inflight={st['inflight']} pending={st['pending']} ticks={st['ticks']} "
                      f"nc_chunks={st['nc_chunks']} walk_steps={st['walk_steps']:.3g}", file=sys.stderr, flush=True)
                last = now
            while next_k < N and ids[next_k] is not None:
                outstanding[next_k] = ids[next_k]
                next_k += 1
            collected = False
            # requests finish out of order; latency is the server's own timestamp, so
            # collecting order does not affect it
            for k, rid in list(outstanding.items()):
                if srv.poll(rid) < N2W_REQUEST_DONE:
                    continue
                mean, se, info = srv.wait(rid, timeout=0.0)
                del outstanding[k]
                collected = True
                r = reqs[k]
                pts = pool_pts[r["mesh"]][r["off"]:r["off"] + r["n"]]
                exact = n2w.problem_exact(problems[r["problem"]], pts.astype(np.float64))
                results.append({"n": r["n"], "latency": info["latency_seconds"], "queue": info["queue_seconds"],
                                "mse": float(np.mean((mean - exact) ** 2)), "target": r["target"],
                                "state": info["state"], "walks": info["walks_per_point"], "mode": r["mode"]})
            if not collected:
                time.sleep(0.002)
        stop.set()
        makespan = time.perf_counter() - t0
    if errors:
        raise errors[0]
    st = srv.stats()
    srv.close()
    sub.join(timeout=5)
    done = len(results)
    lat = np.array([r["latency"] for r in results]) if results else np.array([np.nan])
    small = np.array([r["latency"] for r in results if r["n"] <= 4096]) if results else np.array([np.nan])
    mse_ratio = np.array([r["mse"] / r["target"] ** 2 for r in results]) if results else np.array([np.nan])
    complete = done == N

    def by_mode(mode):
        rs = [r for r in results if r["mode"] == mode]
        if not rs:
            return {"finished": 0}
        lat_m = np.array([r["latency"] for r in rs])
        ratio = np.array([r["mse"] / r["target"] ** 2 for r in rs])
        return {"finished": len(rs), "p50_s": float(np.percentile(lat_m, 50)), "p99_s": float(np.percentile(lat_m, 99)),
                "median_mse_over_target2": float(np.median(ratio)), "points": int(sum(r["n"] for r in rs))}
    line = {
        "metric": "p99 latency of <=4096-point requests, serving loop under mixed load (s)",
        "value": float(np.percentile(small, 99)) if complete else None, "unit": "s", "n_gpus": 1, "steps": N,
        "warmup": 0, "ms_per_step": 1e3 * makespan / max(done, 1), "higher_is_better": False, "scaling": "none",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": f"{N} requests, Poisson arrivals at {args.serve_rate}/s, 4 meshes (bumpy sphere "
                               "128x256, icosphere L6, bumpy spheres 32x64 and 256x512), problems: 8-charge "
                               f"harmonic / sin-product Poisson ({100 * args.serve_poisson_fraction:.0f}%, "
                               f"{args.serve_source_samples} source samples per ball), points "
                               f"log-uniform 1..4096 ({100 * args.serve_large_fraction:.0f}% log-uniform "
                               f"4096..{args.serve_large_max}), RMS stderr target 1e-2 (1e-3 for half of the "
                               f"<=256-point harmonic requests); {100 * args.serve_nc_fraction:.0f}% NC+2LMC "
                               "requests (icosphere, Poisson problem, pre-trained cache, m = 1, residual 1/2)",
                   "tick_walks": args.serve_tick_walks, "tick_walks_max": args.serve_tick_walks_max,
                   "chunk": args.serve_chunk or 1,
                   "max_walks_per_point": args.serve_max_walks,
                   "seed": args.serve_seed, "time_limit_s": args.serve_time_limit},
        "complete": complete, "finished_requests": done,
        "latency_s": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99)),
                      "p50_le4096": float(np.percentile(small, 50)), "p99_le4096": float(np.percentile(small, 99)),
                      "max": float(np.max(lat))},
        "throughput": {"requests_per_s": done / makespan, "points_per_s": sum(r["n"] for r in results) / makespan,
                       "walk_steps_per_s": st["walk_steps"] / makespan,
                       "walks_per_s_incl_nc2lmc": (st["walks"] + st["nc_walks"]) / makespan,
                       "makespan_s": makespan, "note": "walk_steps_per_s counts the plain ticks' walks; "
                       "walks_per_s_incl_nc2lmc adds the NC+2LMC chunks' coarse and residual walks"},
        "accuracy": {"median_mse_over_target2": float(np.median(mse_ratio)),
                     "p99_mse_over_target2": float(np.percentile(mse_ratio, 99)),
                     "done": int(sum(r["state"] == 2 for r in results)),
                     "capped": int(sum(r["state"] == 3 for r in results))},
        "modes": {"plain": by_mode("plain"), "nc2lmc": by_mode("nc2lmc")}, "nc_cache_training": nc_train,
        "server": st, "clocks": clocks.summary(),
        # plain ticks: first query + walker; NC+2LMC chunks: per level first query, walker, cache
        # inference, combine and reduction, plus the chunk's add (more when a chunk splits into batches)
        "gpu_launches": int(st["ticks"]) * 2 + int(st["nc_chunks"]) * 11,
    }
    return line


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="n2w", choices=["n2w", "reference"])
    ap.add_argument("--walks", type=int, default=1024)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-ttm", action="store_true", help="skip the time-to-MSE comparison (NC+2LMC vs plain)")
    ap.add_argument("--points", type=int, default=0,
                    help="use only the first N slice points (smaller workload for profiler captures; "
                         "the default 0 runs the full slice)")
    ap.add_argument("--workload", default="slice", choices=["slice", "batch", "serve", "figure", "nc-levels", "query"],
                    help="slice: the headline Poisson slice (default); batch: 64 batched Laplace instances; "
                         "serve: the serving loop under Poisson arrivals; figure: the reference's published "
                         "figure runs; nc-levels: one call of each NC+2LMC level (for launch-list profiles)")
    ap.add_argument("--serve-requests", type=int, default=300)
    ap.add_argument("--serve-rate", type=float, default=10.0, help="mean arrivals per second")
    ap.add_argument("--serve-large-fraction", type=float, default=0.05)
    ap.add_argument("--serve-large-max", type=int, default=16384)
    ap.add_argument("--serve-poisson-fraction", type=float, default=0.25)
    ap.add_argument("--serve-max-walks", type=int, default=1 << 16)
    ap.add_argument("--serve-time-limit", type=float, default=150.0)
    ap.add_argument("--serve-source-samples", type=int, default=16,
                    help="Green's-function source samples per ball of the Poisson problem")
    ap.add_argument("--serve-tick-walks", type=int, default=1 << 21)
    ap.add_argument("--serve-chunk", type=int, default=0, help="walks per queue pop in a tick (0 = server default 1)")
    ap.add_argument("--serve-tick-walks-max", type=int, default=1 << 23,
                    help="tick budget when every request in flight has a sweep larger than --serve-tick-walks")
    ap.add_argument("--serve-seed", type=int, default=4242)
    ap.add_argument("--serve-nc-fraction", type=float, default=0.1,
                    help="fraction of requests served as NC+2LMC with a pre-trained cache")
    ap.add_argument("--serve-nc-train-steps", type=int, default=200)
    ap.add_argument("--serve-rates", default="", help="serve: comma-separated offered rates to sweep (req/s)")
    ap.add_argument("--serve-sweep-seconds", type=float, default=30.0, help="serve sweep: seconds of arrivals per rate")
    ap.add_argument("--serve-sweep-drain", type=float, default=30.0, help="serve sweep: extra seconds to drain")
    ap.add_argument("--e2e-steps", type=int, default=5, help="end-to-end steps (host buffers) timed after the "
                    "device-resident ones (at most --steps)")
    ap.add_argument("--no-closest-point", action="store_true", help="skip the config-0 closest-point segment")
    ap.add_argument("--no-serve", action="store_true", help="skip the short serving segment of the default line")
    ap.add_argument("--line-serve-requests", type=int, default=200,
                    help="requests of the default line's serving segment (Poisson arrivals at --serve-rate)")
    ap.add_argument("--line-serve-time-limit", type=float, default=45.0)
    ap.add_argument("--nc-points", type=int, default=16384, help="nc-levels: evenly spaced slice points")
    ap.add_argument("--nc-depth", type=int, default=1, help="nc-levels: truncation depth m")
    ap.add_argument("--nc-train-steps", type=int, default=5, help="nc-levels: training steps before the calls")
    ap.add_argument("--queries", type=int, default=262144, help="query: number of uniform query points")
    ap.add_argument("--no-reference-kernel", action="store_true",
                    help="query / default line: skip the reference closest-point kernel baseline leg")
    ap.add_argument("--ttm-stride", type=int, default=4,
                    help="the measured time-to-MSE runs use every N-th slice point, scaled to the full slice")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)
    if args.workload == "batch":
        return run_batch(args)
    if args.workload == "serve":
        return run_serve(args)
    if args.workload == "figure":
        return run_figure(args)
    if args.workload == "nc-levels":
        return run_nc_levels(args)
    if args.workload == "query":
        return run_query(args)

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    import n2w
    from n2w._lib import call, lib

    call("n2w_set_device", local)
    comm = None
    if world > 1:
        # one process per GPU; NCCL through the library's C ABI, the id handed
        # over by a file keyed by this launch (the ranks share their parent)
        from n2w.shard import NcclComm

        comm = NcclComm(rank, world, key=f"{os.environ.get('MASTER_PORT', '0')}_{os.getppid()}")
    mesh, bvh, pts, problem, exact, frame = build_scene(n2w, lib, call)
    if args.points > 0:
        sel = np.linspace(0, len(pts) - 1, min(args.points, len(pts))).astype(np.int64)
        pts, exact = np.ascontiguousarray(pts[sel]), exact[sel]
    n = len(pts)
    W = args.walks
    stream = n2w.Stream()
    d_pts = n2w.DeviceBuffer.from_array(pts)
    stats = n2w.PointStatsBuffers.allocate(n)
    d_cnt = n2w.DeviceBuffer(C.sizeof(n2w._lib.WalkCounters))
    d_ws = n2w.DeviceBuffer(lib.n2w_wos_workspace_bytes(n))
    flush = n2w.DeviceBuffer(256 << 20)
    from n2w import shard

    # every rank walks the whole slice with its own walk stream (weak scaling);
    # the per-point sums of all ranks are combined after the timed region
    opts = n2w.walk_options(walks_per_point=W, max_steps=256, epsilon=5e-4, step_scale=0.999,
                            seed=shard.rank_seed(12345, rank) if world > 1 else 12345)
    timer = n2w.Timer()

    def barrier():
        if comm is not None:
            comm.barrier()

    def step(o):
        call("n2w_wos_estimate", bvh.handle, C.byref(problem), d_pts.ptr, n, C.byref(o), stats.struct(),
             d_cnt.ptr, d_ws.ptr, stream.handle)

    for i in range(args.warmup):
        step(opts)
        stream.sync()

    times, counters = [], []
    with ClockSampler(local) as clocks:
        barrier()
        call("n2w_device_sync")
        for i in range(args.steps):
            flush.zero(stream)
            timer.start(stream)
            step(opts)
            timer.stop(stream)
            times.append(timer.ms())
            raw = d_cnt.download(np.uint64, 8, stream)
            counters.append(dict(zip([f for f, _ in n2w._lib.WalkCounters._fields_], map(int, raw))))
        call("n2w_device_sync")
        barrier()
    total_ms = float(np.sum(times))
    steps_done = float(sum(c["steps"] for c in counters))
    if comm is not None:
        total_ms = float(comm.allreduce_host([np.array([total_ms])], "max")[0][0])
        steps_done = float(comm.allreduce_host([np.array([steps_done])], "sum")[0][0])
    value = steps_done / (total_ms / 1e3)

    # accuracy of the last step (per-point FP64 sums -> MSE vs FP64 analytic);
    # with several ranks, the combined estimate of all ranks' walks (summed on
    # the device over NCCL)
    if comm is not None:
        comm.allreduce_point_stats_device(stats, n, stream)
    res = stats.download(stream)
    err = res["mean"] - exact
    mse = float(np.mean(err ** 2))
    var_part = float(np.mean(res["stderr"] ** 2))
    bias2 = max(mse - var_part, 0.0)

    # end to end: pinned host points in, per-point sums out, every step
    hp = C.c_void_p()
    call("n2w_malloc_host", C.byref(hp), pts.nbytes)
    C.memmove(hp, pts.ctypes.data, pts.nbytes)
    hout = C.c_void_p()
    out_bytes = n * (8 + 8 + 4)
    call("n2w_malloc_host", C.byref(hout), out_bytes)
    e2e_times = []
    barrier()
    for i in range(max(1, min(args.steps, args.e2e_steps))):
        flush.zero(stream)
        timer.start(stream)
        call("n2w_memcpy_h2d", d_pts.ptr, hp, pts.nbytes, stream.handle)
        step(opts)
        call("n2w_memcpy_d2h", hout, stats.sum.ptr, 8 * n, stream.handle)
        call("n2w_memcpy_d2h", C.c_void_p(hout.value + 8 * n), stats.sum_sq.ptr, 8 * n, stream.handle)
        call("n2w_memcpy_d2h", C.c_void_p(hout.value + 16 * n), stats.count.ptr, 4 * n, stream.handle)
        timer.stop(stream)
        e2e_times.append(timer.ms())
    barrier()
    e2e_ms = float(np.sum(e2e_times))
    e2e_steps = float(np.mean([c["steps"] for c in counters])) * len(e2e_times)
    if comm is not None:
        e2e_ms = float(comm.allreduce_host([np.array([e2e_ms])], "max")[0][0])
        e2e_steps = float(comm.allreduce_host([np.array([e2e_steps])], "sum")[0][0])
    lib.n2w_free_host(hp)
    lib.n2w_free_host(hout)

    c_last = counters[-1]
    kernel_ms = float(np.mean(times))
    alg_bytes = c_last["node_visits"] * 128.0 + c_last["tri_tests"] * 48.0 + n * (12 + 8 + 8 + 4 + 8 + 4)
    achieved = alg_bytes / (kernel_ms / 1e3) / 1e9
    peak, peak_kind = peaks()
    cache_peaks = cache_level_peaks(call)

    if rank == 0:
        cpu = None
        if not args.no_cpu_baseline and world == 1:
            try:
                ref_scene = reference_cpu_scene()
                cpu = reference_cpu_sample(ref_scene, W)
                cpu["same_points_as_gpu_workload"] = bool(args.points == 0 and np.array_equal(ref_scene[1], pts))
            except Exception as e:  # the baseline must never break the bench line
                cpu = {"value": None, "unit": UNIT, "cores": os.cpu_count(), "kind": "port",
                       "sample": f"failed: {e}"}
        wsteps_per_walk = c_last["steps"] / max(c_last["walks"], 1)
        cp_seg = None
        if not args.no_closest_point and world == 1:
            cp_seg = closest_point_segment(n2w, call, stream, timer, flush, cache_peaks,
                                           reference_kernel=not args.no_reference_kernel)
        ttm = None
        if not args.no_ttm and world == 1 and args.points == 0:
            ttm = time_to_mse(n2w, lib, call, mesh, bvh, pts, exact, problem, real_stride=args.ttm_stride)
        serving = None
        if not args.no_serve and world == 1 and args.points == 0:
            sargs = argparse.Namespace(**vars(args))
            sargs.serve_requests, sargs.serve_time_limit = args.line_serve_requests, args.line_serve_time_limit
            sargs.serve_nc_train_steps = 50
            serving = serve_line(sargs)
            serving = {k: serving[k] for k in ("metric", "value", "unit", "config", "complete", "finished_requests",
                                                "latency_s", "throughput", "accuracy", "modes", "clocks",
                                                "gpu_launches") if k in serving}
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": dict(CONFIG, points=n, parallelism=(f"walk shards x{world}: every rank walks the slice "
                                                          "with its own stream, per-point sums all-reduced")
                                                         if world > 1 else "1 GPU"),
            "e2e": {"value": e2e_steps / (e2e_ms / 1e3), "unit": UNIT, "h2d_bytes_per_step": int(pts.nbytes),
                    "d2h_bytes_per_step": int(out_bytes)},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak,
                         "traffic": (traffic_per_walk_step() * c_last["steps"]) if traffic_per_walk_step() else None,
                         "traffic_source": "profiles/walker_kernel_icosphere_slice_4096pts.md (scaled by walk-steps)",
                         "peak_source": peak_kind,
                         "kernel": "walker_kernel", "bytes_per_launch": alg_bytes,
                         "kernel_ms": kernel_ms, "fractions": fractions(achieved, peak, cache_peaks),
                         "cache_level_peaks_gbs": cache_peaks,
                         "note": "algorithmic bytes are L1/L2 hits (BVH + triangles L2-resident); frac is the "
                                 "HBM-copy scale, fractions.l1 / fractions.l2 divide by this box's measured L1 / L2 "
                                 "read bandwidth"},
            "cpu_baseline": cpu,
            "gpu_launches": 2 * args.steps,  # per step: first-query pre-pass + persistent walker
            "clocks": clocks.summary(),
            "accuracy": {"mse_vs_fp64_exact": mse, "mean_estimator_variance": var_part, "bias2_estimate": bias2,
                         "walks_per_point": W * world, "mean_steps_per_walk": wsteps_per_walk},
            "time_to_mse_1e-4": ttm,
            "closest_point": cp_seg,
            "serving": serving,
            "counters_last_step": c_last,
            "walks_per_s": c_last["walks"] / (kernel_ms / 1e3),
        }
        print(json.dumps(line))
    if comm is not None:
        comm.barrier()
        comm.close()
    return 0


if __name__ == "__main__":
    sys.exit(main())
