"""Neural-cache estimator orchestration over the C ABI (training + NC+2LMC).

Mirrors the flow of the reference's NC evaluator (src/tools/eval_tcnn_nc_wos.cu:
714-856): build the geometry, train the cache on WoS labels, then estimate with
coarse walks closed by the cache plus a residual level continued to the
boundary.  Every step runs on the device; Python only sequences calls.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import DeviceBuffer, PointStatsBuffers
from ._lib import Nc2lmcOptions, NcProgressiveBlock, NcProgressiveOptions, NcTrainOptions, call


def input_box(mesh, pad_fraction: float = 0.05):
    """Unit-cube map of the cache inputs: mesh bounds grown by pad_fraction of the
    extent on each side (reference eval_tcnn_nc_wos.cu:522-523)."""
    lo, hi = mesh.bounds()
    ext = hi - lo
    return (lo - pad_fraction * ext).astype(np.float32), (ext * (1 + 2 * pad_fraction)).astype(np.float32)


def train_options(mesh, steps=200, batch=65536, walks_per_label=32, max_steps=256, epsilon=1e-3, step_scale=0.999,
                  seed=2024):
    o = NcTrainOptions()
    o.steps, o.batch, o.walks_per_label, o.max_steps = steps, batch, walks_per_label, max_steps
    o.epsilon, o.step_scale, o.seed = epsilon, step_scale, seed
    imin, iext = input_box(mesh)
    lo, hi = mesh.bounds()
    for k in range(3):
        o.input_min[k], o.input_extent[k] = float(imin[k]), float(iext[k])
        o.sample_lo[k], o.sample_hi[k] = float(lo[k]), float(hi[k])
    return o


def train(cache, bvh, problem, mesh, steps=200, batch=65536, walks_per_label=32, max_steps=256, epsilon=1e-3,
          step_scale=0.999, seed=2024, stream=None):
    """Online training; returns the per-step batch losses."""
    o = train_options(mesh, steps, batch, walks_per_label, max_steps, epsilon, step_scale, seed)
    losses = np.zeros(max(steps, 1), np.float32)
    call("n2w_nc_train", cache.handle, bvh.handle, C.byref(problem), C.byref(o), C.c_void_p(losses.ctypes.data),
         stream.handle if stream else None)
    return losses[:steps]


def nc2lmc_options(mesh, coarse_walks=256, residual_walks=16, depth_m=8, max_steps=256, epsilon=1e-3,
                   step_scale=0.999, seed=99, point_batch=0):
    o = Nc2lmcOptions()
    o.coarse_walks, o.residual_walks, o.depth_m, o.max_steps = coarse_walks, residual_walks, depth_m, max_steps
    o.epsilon, o.step_scale, o.seed, o.point_batch = epsilon, step_scale, seed, point_batch
    imin, iext = input_box(mesh)
    for k in range(3):
        o.input_min[k], o.input_extent[k] = float(imin[k]), float(iext[k])
    return o


def nc2lmc(bvh, problem, cache, points, options, stream=None, d_points=None):
    """Runs coarse + residual levels; returns per-point combined estimate,
    estimator variance and the per-level statistics.  cache=None closes the
    coarse walks with the exact solution instead of a network (the analytic
    stand-in: the best any cache can do, used for bounds)."""
    if d_points is None:
        pts = np.ascontiguousarray(points, np.float32).reshape(-1, 3)
        n = len(pts)
        d_points = DeviceBuffer.from_array(pts)
    else:
        n = len(points)
    cs, rs = PointStatsBuffers.allocate(n), PointStatsBuffers.allocate(n)
    s = stream.handle if stream else None
    if cache is None:
        call("n2w_nc2lmc_estimate_ex", bvh.handle, C.byref(problem), None, d_points.ptr, n, C.byref(options),
             cs.struct(), rs.struct(), None, s)
    else:
        call("n2w_nc2lmc_estimate", bvh.handle, C.byref(problem), cache.handle, d_points.ptr, n, C.byref(options),
             cs.struct(), rs.struct(), s)
    call("n2w_stream_sync", s)
    c = cs.download(stream) if options.coarse_walks > 0 else None
    r = rs.download(stream) if options.residual_walks > 0 else None
    return combine(c, r, options.coarse_walks, options.residual_walks)


def progressive(theta_train, theta_infer, bvh, problem, points, train_opts, estimate_opts, blocks=4,
                train_steps_per_block=50, overlap=True, d_points=None):
    """Progressive NC+2LMC (n2w_nc_progressive): block k estimates with the
    frozen snapshot theta_k while theta_train trains toward theta_{k+1} on a
    second stream (overlap=True) or after the block (overlap=False).  Returns
    the pooled estimate (mean, stderr), the per-level statistics and the
    per-block times (eval_ms, train_ms, wall_ms)."""
    from . import Stream

    if d_points is None:
        pts = np.ascontiguousarray(points, np.float32).reshape(-1, 3)
        n = len(pts)
        d_points = DeviceBuffer.from_array(pts)
    else:
        n = len(points)
    o = NcProgressiveOptions()
    o.blocks, o.train_steps_per_block, o.overlap = blocks, train_steps_per_block, 1 if overlap else 0
    o.train, o.estimate = train_opts, estimate_opts
    cs, rs = PointStatsBuffers.allocate(n), PointStatsBuffers.allocate(n)
    es, ts = Stream(), Stream()
    out = (NcProgressiveBlock * blocks)()
    call("n2w_nc_progressive", theta_train.handle, theta_infer.handle, bvh.handle, C.byref(problem), d_points.ptr, n,
         C.byref(o), cs.struct(), rs.struct(), C.cast(out, C.c_void_p), es.handle, ts.handle)
    es.sync()
    c = cs.download(es) if estimate_opts.coarse_walks > 0 else None
    r = rs.download(es) if estimate_opts.residual_walks > 0 else None
    mean = (c["mean"] if c is not None else 0.0) + (r["mean"] if r is not None else 0.0)
    var = ((c["sample_variance"] / np.maximum(c["count"], 1) if c is not None else 0.0) +
           (r["sample_variance"] / np.maximum(r["count"], 1) if r is not None else 0.0))
    return {"mean": mean, "estimator_variance": var, "stderr": np.sqrt(var), "coarse": c, "residual": r,
            "blocks": [{"eval_ms": b.eval_ms, "train_ms": b.train_ms, "wall_ms": b.wall_ms} for b in out]}


def combine(c, r, Nc, Nr):
    mean = (c["mean"] if c is not None else 0.0) + (r["mean"] if r is not None else 0.0)
    var = (c["sample_variance"] / Nc if c is not None else 0.0) + (r["sample_variance"] / Nr if r is not None else 0.0)
    return {"mean": mean, "estimator_variance": var, "stderr": np.sqrt(var), "coarse": c, "residual": r}


def time_to_mse(target, seconds_per_unit, var_per_unit, bias2=0.0, fixed_seconds=0.0):
    """Seconds to reach slice MSE `target` when MSE(k units) = bias2 + var_per_unit / k
    and each unit of work costs seconds_per_unit (plus fixed_seconds once).
    Returns None when the bias alone exceeds the target."""
    if bias2 >= target:
        return None
    k = var_per_unit / (target - bias2)
    return fixed_seconds + k * seconds_per_unit
