"""Python orchestration layer over libn2w.so (ctypes; no PyTorch on the path).

Mirrors the reference's host objects: ``Mesh`` (include/n2wos/mesh.hpp),
``Bvh`` with ``query_device`` (include/n2wos/cuda_bvh.hpp:50-57), the boundary
problems of include/n2wos/tcnn_nc_wos.hpp:14-35, and the walker entry points.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from ._lib import (EXPORTED, LIB_PATH, N2W_BC, N2W_SOURCE_BALL, N2W_SOURCE_CENTER, N2W_WALK_PREFIX,
                   N2W_WALK_PURE, N2W_WALK_RESIDUAL, BvhStats, N2wError, PointStats, Problem,
                   WalkCounters, WalkOptions, call, check, lib)

__all__ = [
    "Mesh", "HostBvh", "Bvh", "DeviceBuffer", "Stream", "Timer", "problem_charges_seeded",
    "problem_sinprod", "problem_reference", "problem_from_name", "walk_options", "wos_estimate",
    "N2wError", "LIB_PATH", "EXPORTED", "N2W_BC", "device_count", "device_summary", "runtime_version",
    "N2W_SOURCE_BALL", "N2W_SOURCE_CENTER", "N2W_WALK_PURE", "N2W_WALK_PREFIX", "N2W_WALK_RESIDUAL",
    "Scene", "Batch", "Server",
]


def _ptr(a: np.ndarray) -> C.c_void_p:
    return C.c_void_p(a.ctypes.data)


class Mesh:
    """Host triangle mesh (vertices float32 [nv,3], triangles uint32 [nt,3])."""

    def __init__(self, handle: C.c_void_p):
        self._h = handle

    @classmethod
    def from_arrays(cls, vertices, triangles, name: str = "mesh") -> "Mesh":
        v = np.ascontiguousarray(vertices, dtype=np.float32).reshape(-1, 3)
        t = np.ascontiguousarray(triangles, dtype=np.uint32).reshape(-1, 3)
        h = C.c_void_p()
        call("n2w_mesh_create", _ptr(v), len(v), _ptr(t), len(t), name.encode(), C.byref(h))
        return cls(h)

    @classmethod
    def bumpy_sphere_ref(cls, stacks=128, slices=256, amplitude=0.15) -> "Mesh":
        h = C.c_void_p()
        call("n2w_mesh_bumpy_sphere_ref", stacks, slices, C.c_float(amplitude), C.byref(h))
        return cls(h)

    @classmethod
    def bumpy_sphere_trig(cls, stacks=128, slices=256, amplitude=0.08, k_theta=6, k_phi=8) -> "Mesh":
        h = C.c_void_p()
        call("n2w_mesh_bumpy_sphere_trig", stacks, slices, C.c_float(amplitude), k_theta, k_phi, C.byref(h))
        return cls(h)

    @classmethod
    def icosphere_displaced(cls, level=6, amplitude=0.12, base_frequency=3.0, octaves=4,
                            persistence=0.5, seed=12345) -> "Mesh":
        h = C.c_void_p()
        call("n2w_mesh_icosphere_displaced", level, C.c_float(amplitude), C.c_float(base_frequency),
             octaves, C.c_float(persistence), C.c_uint64(seed), C.byref(h))
        return cls(h)

    @classmethod
    def load(cls, path: str) -> "Mesh":
        h = C.c_void_p()
        fn = "n2w_mesh_load_obj" if str(path).lower().endswith(".obj") else "n2w_mesh_load_ply"
        call(fn, str(path).encode(), C.byref(h))
        return cls(h)

    def normalize(self):
        c = np.zeros(3, np.float32)
        s = C.c_float()
        call("n2w_mesh_normalize", self._h, _ptr(c), C.byref(s))
        return c, float(s.value)

    @property
    def counts(self):
        nv, nt = C.c_int64(), C.c_int64()
        call("n2w_mesh_counts", self._h, C.byref(nv), C.byref(nt))
        return nv.value, nt.value

    def arrays(self):
        nv, nt = self.counts
        v = np.empty((nv, 3), np.float32)
        t = np.empty((nt, 3), np.uint32)
        call("n2w_mesh_copy_out", self._h, _ptr(v), _ptr(t))
        return v, t

    def bounds(self):
        b = np.empty(6, np.float32)
        call("n2w_mesh_bounds", self._h, _ptr(b))
        return b[:3].copy(), b[3:].copy()

    def closest_point_host(self, points: np.ndarray, threads: int = 0) -> dict:
        """Host brute force over every triangle (the probes' validator)."""
        pts = np.ascontiguousarray(points, np.float32).reshape(-1, 3)
        n = len(pts)
        d2 = np.empty(n, np.float32)
        cp = np.empty((n, 3), np.float32)
        ids = np.empty(n, np.int32)
        call("n2w_mesh_closest_point_host", self._h, _ptr(pts), n, _ptr(d2), _ptr(cp), _ptr(ids), threads)
        return {"distance2": d2, "closest": cp, "triangle_id": ids}

    @property
    def name(self) -> str:
        return lib.n2w_mesh_name(self._h).decode()

    def degenerate_count(self, eps: float = 1e-20) -> int:
        out = C.c_int64()
        call("n2w_mesh_count_degenerate", self._h, C.c_float(eps), C.byref(out))
        return out.value

    def __del__(self):
        if getattr(self, "_h", None):
            lib.n2w_mesh_free(self._h)
            self._h = None


NODE_DTYPE = np.dtype([("lo_x", "<f4", 4), ("hi_x", "<f4", 4), ("lo_y", "<f4", 4), ("hi_y", "<f4", 4),
                       ("lo_z", "<f4", 4), ("hi_z", "<f4", 4), ("child", "<i4", 4), ("pad", "<i4", 4)])
TRI_DTYPE = np.dtype([("v0", "<f4", 3), ("id", "<i4"), ("v1", "<f4", 3), ("pad1", "<i4"),
                      ("v2", "<f4", 3), ("pad2", "<i4")])
assert NODE_DTYPE.itemsize == 128 and TRI_DTYPE.itemsize == 48


def _stats_dict(s: BvhStats) -> dict:
    return {f: getattr(s, f) for f, _ in BvhStats._fields_}


class HostBvh:
    """Host-only build of the device layout (no GPU needed)."""

    def __init__(self, mesh: Mesh, leaf_size: int = 4, method: str = "sah"):
        self._h = C.c_void_p()
        call("n2w_bvh_host_build", mesh._h, leaf_size, method.encode(), C.byref(self._h))

    @property
    def stats(self) -> dict:
        s = BvhStats()
        call("n2w_bvh_host_stats", self._h, C.byref(s))
        return _stats_dict(s)

    def layout(self):
        st = self.stats
        nodes = np.empty(st["nodes"], NODE_DTYPE)
        tris = np.empty(st["triangles"], TRI_DTYPE)
        call("n2w_bvh_host_copy", self._h, _ptr(nodes), _ptr(tris))
        return nodes, tris

    def __del__(self):
        if getattr(self, "_h", None):
            lib.n2w_bvh_host_free(self._h)
            self._h = None


class Stream:
    def __init__(self):
        self.handle = C.c_void_p()
        call("n2w_stream_create", C.byref(self.handle))

    def sync(self):
        call("n2w_stream_sync", self.handle)

    def __del__(self):
        if getattr(self, "handle", None):
            lib.n2w_stream_destroy(self.handle)
            self.handle = None


class DeviceBuffer:
    """Raw device allocation with numpy upload/download helpers."""

    def __init__(self, nbytes: int):
        self.nbytes = int(nbytes)
        self.ptr = C.c_void_p()
        call("n2w_malloc", C.byref(self.ptr), max(self.nbytes, 1))

    @classmethod
    def from_array(cls, a: np.ndarray, stream=None) -> "DeviceBuffer":
        a = np.ascontiguousarray(a)
        b = cls(a.nbytes)
        b.upload(a, stream)
        return b

    def upload(self, a: np.ndarray, stream=None):
        a = np.ascontiguousarray(a)
        assert a.nbytes <= self.nbytes
        call("n2w_memcpy_h2d", self.ptr, _ptr(a), a.nbytes, stream.handle if stream else None)
        if stream is None:
            call("n2w_stream_sync", None)

    def download(self, dtype, count: int | None = None, stream=None) -> np.ndarray:
        dtype = np.dtype(dtype)
        n = self.nbytes // dtype.itemsize if count is None else int(count)
        out = np.empty(n, dtype)
        call("n2w_memcpy_d2h", _ptr(out), self.ptr, out.nbytes, stream.handle if stream else None)
        call("n2w_stream_sync", stream.handle if stream else None)
        return out

    def zero(self, stream=None):
        call("n2w_memset", self.ptr, 0, self.nbytes, stream.handle if stream else None)

    def __del__(self):
        if getattr(self, "ptr", None) and self.ptr.value:
            lib.n2w_free(self.ptr)
            self.ptr = None


class Timer:
    def __init__(self):
        self._h = C.c_void_p()
        call("n2w_timer_create", C.byref(self._h))

    def start(self, stream=None):
        call("n2w_timer_start", self._h, stream.handle if stream else None)

    def stop(self, stream=None):
        call("n2w_timer_stop", self._h, stream.handle if stream else None)

    def ms(self) -> float:
        v = C.c_float()
        call("n2w_timer_elapsed_ms", self._h, C.byref(v))
        return float(v.value)

    def __del__(self):
        if getattr(self, "_h", None):
            lib.n2w_timer_destroy(self._h)
            self._h = None


class Bvh:
    """Device-resident BVH (reference CudaBvh / CuBqlBvh)."""

    def __init__(self, mesh: Mesh, leaf_size: int = 4, method: str = "sah"):
        self._h = C.c_void_p()
        call("n2w_bvh_create", mesh._h, leaf_size, method.encode(), C.byref(self._h))

    @property
    def handle(self):
        return self._h

    @property
    def stats(self) -> dict:
        s = BvhStats()
        call("n2w_bvh_stats_get", self._h, C.byref(s))
        return _stats_dict(s)

    def query_device(self, d_points, n, d_d2, d_cp, d_id, d_ov, block_size=128, stream=None, d_active=None):
        s = stream.handle if stream else None
        if d_active is None:
            call("n2w_bvh_query_device", self._h, d_points, n, d_d2, d_cp, d_id, d_ov, block_size, s)
        else:
            call("n2w_bvh_query_device_masked", self._h, d_points, d_active, n, d_d2, d_cp, d_id, d_ov,
                 block_size, s)

    def query(self, points: np.ndarray, block_size: int = 128, counted: bool = False, active=None):
        """Host convenience wrapper: upload, query, download (reference CudaBvh::query)."""
        pts = np.ascontiguousarray(points, np.float32).reshape(-1, 3)
        n = len(pts)
        dp = DeviceBuffer.from_array(pts)
        dd = DeviceBuffer(4 * n)
        dc = DeviceBuffer(12 * n)
        di = DeviceBuffer(4 * n)
        do = DeviceBuffer(4 * n)
        out = {}
        if counted:
            dn = DeviceBuffer(4 * n)
            dt = DeviceBuffer(4 * n)
            call("n2w_bvh_query_device_counted", self._h, dp.ptr, n, dd.ptr, dc.ptr, di.ptr, do.ptr, dn.ptr,
                 dt.ptr, block_size, None)
            out["node_visits"] = dn.download(np.int32)
            out["tri_tests"] = dt.download(np.int32)
        elif active is not None:
            da = DeviceBuffer.from_array(np.ascontiguousarray(active, np.uint8))
            self.query_device(dp.ptr, n, dd.ptr, dc.ptr, di.ptr, do.ptr, block_size, None, da.ptr)
        else:
            self.query_device(dp.ptr, n, dd.ptr, dc.ptr, di.ptr, do.ptr, block_size)
        call("n2w_device_sync")
        out["distance2"] = dd.download(np.float32)
        out["closest"] = dc.download(np.float32).reshape(n, 3)
        out["triangle_id"] = di.download(np.int32)
        out["overflow"] = do.download(np.int32)
        return out

    def layout(self):
        st = self.stats
        nodes = np.empty(st["nodes"], NODE_DTYPE)
        tris = np.empty(st["triangles"], TRI_DTYPE)
        call("n2w_bvh_copy_layout", self._h, _ptr(nodes), _ptr(tris))
        return nodes, tris

    def seed_grid(self):
        """(slots int32[(n+1)^3], lo float32[3], h, n) of the BVH's seed grid."""
        lo = np.empty(3, np.float32)
        h = C.c_float()
        n = C.c_int()
        call("n2w_bvh_seed_grid", self._h, _ptr(lo), C.byref(h), C.byref(n), None)
        slots = np.empty((n.value + 1) ** 3, np.int32)
        call("n2w_bvh_seed_grid", self._h, None, None, None, _ptr(slots))
        return slots, lo, float(h.value), n.value

    def inside(self, points: np.ndarray, block_size: int = 128) -> np.ndarray:
        """Ray-parity inside/outside of each point (uint8 0/1) on the device."""
        pts = np.ascontiguousarray(points, np.float32).reshape(-1, 3)
        n = len(pts)
        if n == 0:
            return np.zeros(0, np.uint8)
        dp = DeviceBuffer.from_array(pts)
        di = DeviceBuffer(n)
        dov = DeviceBuffer(4)
        dov.zero()
        call("n2w_bvh_inside_device", self._h, dp.ptr, n, di.ptr, dov.ptr, block_size, None)
        out = di.download(np.uint8, n)
        if dov.download(np.int32, 1)[0]:
            raise N2wError(6, "ray-parity traversal stack overflow")
        return out

    def __del__(self):
        if getattr(self, "_h", None):
            lib.n2w_bvh_destroy(self._h)
            self._h = None


def slice_points(bounds_min, bounds_max, view="xy", plane=0.0, width=512, height=512, padding=0.02,
                 preserve_aspect=True):
    """Pixel-centre grid of the reference slice renderer; returns (points[H*W,3], frame[4])."""
    b = np.ascontiguousarray(np.concatenate([bounds_min, bounds_max]), np.float32)
    pts = np.empty((width * height, 3), np.float32)
    frame = np.empty(4, np.float32)
    call("n2w_slice_points", _ptr(b), view.encode(), C.c_float(plane), width, height, C.c_float(padding),
         int(preserve_aspect), _ptr(pts), _ptr(frame))
    return pts, frame


def problem_charges_seeded(count=8, r_min=1.6, r_max=2.0, seed=12345) -> Problem:
    p = Problem()
    call("n2w_problem_charges_seeded", count, C.c_float(r_min), C.c_float(r_max), C.c_uint64(seed), C.byref(p))
    return p


def problem_sinprod(omega=2 * np.pi * 1.5, source_sampling=N2W_SOURCE_BALL) -> Problem:
    p = Problem()
    call("n2w_problem_sinprod", C.c_float(omega), source_sampling, C.byref(p))
    return p


def problem_reference(mode: int, source_sampling=N2W_SOURCE_CENTER) -> Problem:
    p = Problem()
    call("n2w_problem_reference_mode", mode, source_sampling, C.byref(p))
    return p


def problem_from_name(name: str, source_sampling=N2W_SOURCE_BALL, seed=12345) -> Problem:
    m = C.c_int()
    call("n2w_problem_mode_from_name", name.encode(), C.byref(m))
    if m.value == N2W_BC["charges_seeded"]:
        return problem_charges_seeded(seed=seed)
    if m.value == N2W_BC["poisson_sinprod"]:
        return problem_sinprod(source_sampling=source_sampling)
    return problem_reference(m.value, source_sampling)


def problem_exact(p: Problem, xyz: np.ndarray) -> np.ndarray:
    x = np.ascontiguousarray(xyz, np.float64).reshape(-1, 3)
    out = np.empty(len(x), np.float64)
    call("n2w_problem_exact", C.byref(p), _ptr(x), len(x), _ptr(out))
    return out


def problem_eval_f32(p: Problem, xyz: np.ndarray):
    x = np.ascontiguousarray(xyz, np.float32).reshape(-1, 3)
    g = np.empty(len(x), np.float32)
    f = np.empty(len(x), np.float32)
    call("n2w_problem_eval_f32", C.byref(p), _ptr(x), len(x), _ptr(g), _ptr(f))
    return g, f


def walk_options(walks_per_point=256, max_steps=256, depth_m=8, epsilon=1e-3, step_scale=0.999,
                 seed=12345, block_size=0, blocks_per_sm=0, chunk=0, accumulate=0, deadline_ns=0,
                 regen_threshold=0):
    o = WalkOptions()
    o.walks_per_point, o.max_steps, o.depth_m = walks_per_point, max_steps, depth_m
    o.epsilon, o.step_scale, o.seed = epsilon, step_scale, seed
    o.block_size, o.blocks_per_sm, o.chunk = block_size, blocks_per_sm, chunk
    o.accumulate, o.deadline_ns, o.regen_threshold = accumulate, deadline_ns, regen_threshold
    return o


def label_options(walks_per_point=32, max_steps=256, epsilon=1e-3, step_scale=0.999, seed=12345, refresh_index=0,
                  label_source=1, input_min=(0.0, 0.0, 0.0), input_extent=(1.0, 1.0, 1.0), block_size=0):
    """n2w_nc_label_options: one refresh of n2w_nc_update_labels (label_source
    1 = WoS walks, 0 = the exact solution)."""
    from ._lib import NcLabelOptions

    o = NcLabelOptions()
    o.walks_per_point, o.max_steps, o.epsilon, o.step_scale = walks_per_point, max_steps, epsilon, step_scale
    o.seed, o.refresh_index, o.label_source, o.block_size = seed, refresh_index, label_source, block_size
    for k in range(3):
        o.input_min[k] = float(input_min[k])
        o.input_extent[k] = float(input_extent[k])
    return o


@dataclass
class PointStatsBuffers:
    n: int
    sum: DeviceBuffer
    sum_sq: DeviceBuffer
    count: DeviceBuffer
    steps: DeviceBuffer
    forced: DeviceBuffer

    @classmethod
    def allocate(cls, n: int) -> "PointStatsBuffers":
        return cls(n, DeviceBuffer(8 * n), DeviceBuffer(8 * n), DeviceBuffer(4 * n), DeviceBuffer(8 * n),
                   DeviceBuffer(4 * n))

    def struct(self) -> PointStats:
        return PointStats(self.sum.ptr, self.sum_sq.ptr, self.count.ptr, self.steps.ptr, self.forced.ptr)

    def zero(self, stream=None):
        """Clears every accumulator (device allocations start uninitialised)."""
        for b in (self.sum, self.sum_sq, self.count, self.steps, self.forced):
            b.zero(stream)

    def download(self, stream=None) -> dict:
        s = self.sum.download(np.float64, self.n, stream)
        s2 = self.sum_sq.download(np.float64, self.n, stream)
        cnt = self.count.download(np.uint32, self.n, stream).astype(np.float64)
        steps = self.steps.download(np.uint64, self.n, stream).astype(np.float64)
        forced = self.forced.download(np.uint32, self.n, stream)
        mean = s / np.maximum(cnt, 1)
        var = np.where(cnt > 1, (s2 - cnt * mean * mean) / np.maximum(cnt - 1, 1), 0.0)
        var = np.maximum(var, 0.0)
        return {"mean": mean, "sample_variance": var, "stderr": np.sqrt(var / np.maximum(cnt, 1)),
                "count": cnt, "mean_steps": steps / np.maximum(cnt, 1), "forced": forced,
                "sum": s, "sum_sq": s2}


def wos_estimate(bvh: Bvh, problem: Problem, points: np.ndarray | DeviceBuffer, n: int | None = None,
                 options: WalkOptions | None = None, stats: PointStatsBuffers | None = None,
                 stream: Stream | None = None, counters: bool = True):
    """Plain WoS per-point estimates; returns (per-point dict, counters dict)."""
    options = options or walk_options()
    if isinstance(points, DeviceBuffer):
        dp = points
        assert n is not None
    else:
        pts = np.ascontiguousarray(points, np.float32).reshape(-1, 3)
        n = len(pts)
        dp = DeviceBuffer.from_array(pts)
    stats = stats or PointStatsBuffers.allocate(n)
    dcount = DeviceBuffer(C.sizeof(WalkCounters)) if counters else None
    s = stream.handle if stream else None
    call("n2w_wos_estimate", bvh.handle, C.byref(problem), dp.ptr, n, C.byref(options), stats.struct(),
         dcount.ptr if dcount else None, None, s)
    call("n2w_stream_sync", s)
    res = stats.download(stream)
    cnt = {}
    if dcount:
        raw = dcount.download(np.uint64, 8)
        cnt = dict(zip([f for f, _ in WalkCounters._fields_], (int(v) for v in raw)))
    return res, cnt


class Scene:
    """Several BVHs merged into one device layout for batched launches."""

    def __init__(self, bvhs):
        arr = (C.c_void_p * len(bvhs))(*[b.handle for b in bvhs])
        h = C.c_void_p()
        call("n2w_scene_create", arr, len(bvhs), C.byref(h))
        self._h = h

    @property
    def handle(self):
        return self._h

    def info(self) -> dict:
        m, nodes, tris, by = C.c_int(), C.c_int64(), C.c_int64(), C.c_int64()
        call("n2w_scene_info", self._h, C.byref(m), C.byref(nodes), C.byref(tris), C.byref(by))
        return {"meshes": m.value, "nodes": nodes.value, "triangles": tris.value, "device_bytes": by.value}

    def __del__(self):
        if getattr(self, "_h", None):
            lib.n2w_scene_destroy(self._h)
            self._h = None


class Batch:
    """Many plain-WoS instances in one persistent launch (optionally a CUDA graph).

    ``instances`` is a list of dicts with keys mesh, problem (index), points
    (N x 3 array), walks_per_point and seed.  Per-instance statistics are kept
    in device buffers owned by the batch."""

    def __init__(self, scene: Scene, problems, instances, options: WalkOptions | None = None):
        from ._lib import BatchItem

        self.scene = scene
        self.options = options or walk_options()
        self.points = []
        self.stats = []
        items = (BatchItem * len(instances))()
        for k, inst in enumerate(instances):
            pts = np.ascontiguousarray(inst["points"], np.float32).reshape(-1, 3)
            dp = DeviceBuffer.from_array(pts) if len(pts) else DeviceBuffer(12)
            st = PointStatsBuffers.allocate(max(len(pts), 1))
            for buf in (st.sum, st.sum_sq, st.count, st.steps, st.forced):
                buf.zero()  # launches with accumulate=1 add to these
            st.n = len(pts)
            self.points.append(dp)
            self.stats.append(st)
            items[k].mesh = inst["mesh"]
            items[k].problem = inst["problem"]
            items[k].d_points = dp.ptr
            items[k].point_count = len(pts)
            items[k].walks_per_point = inst["walks_per_point"]
            items[k].seed = inst.get("seed", 12345 + k)
            items[k].stats = st.struct()
        self._problems = (Problem * len(problems))(*problems)
        h = C.c_void_p()
        call("n2w_batch_create", scene.handle, self._problems, len(problems), items, len(instances),
             C.byref(self.options), C.byref(h))
        self._h = h
        self.counters = DeviceBuffer(C.sizeof(WalkCounters))

    @property
    def handle(self):
        return self._h

    def launch(self, stream: Stream | None = None, counters: bool = True):
        call("n2w_batch_launch", self._h, self.counters.ptr if counters else None,
             stream.handle if stream else None)

    def capture_graph(self, stream: Stream):
        call("n2w_batch_capture_graph", self._h, self.counters.ptr, stream.handle)

    def graph_launch(self, stream: Stream):
        call("n2w_batch_graph_launch", self._h, stream.handle)

    def set_seeds(self, seeds, stream: Stream | None = None):
        arr = (C.c_uint64 * len(seeds))(*[int(s) for s in seeds])
        call("n2w_batch_set_seeds", self._h, arr, stream.handle if stream else None)

    def autotune(self, sample_fraction: float = 0.0625, stream: Stream | None = None) -> dict:
        from ._lib import BatchTuning

        best = BatchTuning()
        trials = (BatchTuning * 64)()
        n = C.c_int()
        call("n2w_batch_autotune", self._h, C.c_double(sample_fraction), C.byref(best), trials, 64, C.byref(n),
             stream.handle if stream else None)
        fields = [f for f, _ in BatchTuning._fields_]

        def as_dict(t):
            return {f: getattr(t, f) for f in fields}

        return {"best": as_dict(best), "trials": [as_dict(trials[i]) for i in range(n.value)]}

    def set_tuning(self, tuning: dict, stream: Stream | None = None):
        from ._lib import BatchTuning

        t = BatchTuning()
        for k, v in tuning.items():
            if k != "ms":
                setattr(t, k, int(v))
        call("n2w_batch_set_tuning", self._h, C.byref(t), stream.handle if stream else None)

    def info(self) -> dict:
        tp, tw, rv = C.c_int64(), C.c_int64(), C.c_int()
        o = WalkOptions()
        call("n2w_batch_info", self._h, C.byref(tp), C.byref(tw), C.byref(o), C.byref(rv))
        return {"total_points": tp.value, "total_walks": tw.value, "block_size": o.block_size, "chunk": o.chunk,
                "regen_threshold": o.regen_threshold, "reg_variant": rv.value}

    def results(self, stream: Stream | None = None):
        call("n2w_stream_sync", stream.handle if stream else None)
        return [st.download(stream) if st.n else None for st in self.stats]

    def run_counters(self) -> dict:
        raw = self.counters.download(np.uint64, 8)
        return dict(zip([f for f, _ in WalkCounters._fields_], (int(v) for v in raw)))

    def __del__(self):
        if getattr(self, "_h", None):
            lib.n2w_batch_destroy(self._h)
            self._h = None


class Server:
    """Continuous-batching WoS server (native worker thread; see n2w_server_*).

    meshes: list of Bvh; problems: list of Problem.  submit() returns a request
    id; wait() returns (mean, stderr, info dict).  set_nc() registers a
    pre-trained Cache for NC+2LMC requests (submit(..., mode="nc2lmc")); the
    server keeps references to the BVHs and caches it walks."""

    def __init__(self, bvhs, problems, **options):
        from ._lib import ServerOptions

        o = ServerOptions()
        call("n2w_server_options_default", C.byref(o))
        for k, v in options.items():
            setattr(o, k, v)
        self.options = o
        arr = (C.c_void_p * len(bvhs))(*[b.handle for b in bvhs])
        self._problems = (Problem * len(problems))(*problems)
        h = C.c_void_p()
        call("n2w_server_create", arr, len(bvhs), self._problems, len(problems), C.byref(o), C.byref(h))
        self._h = h
        self._sizes = {}
        self._bvhs = list(bvhs)
        self._caches = {}

    def set_nc(self, mesh: int, problem: int, cache, input_min, input_extent, depth_m: int = 8,
               residual_fraction: float = 1.0 / 16):
        """Cache for NC+2LMC requests on (mesh, problem); cache=None selects the
        analytic cache C(x) = u(x) (a check of the estimator)."""
        from ._lib import ServerNc

        c = ServerNc()
        c.cache = cache.handle if cache is not None else None
        c.input_min[:] = [float(v) for v in input_min]
        c.input_extent[:] = [float(v) for v in input_extent]
        c.depth_m = depth_m
        c.residual_fraction = residual_fraction
        call("n2w_server_set_nc", self._h, mesh, problem, C.byref(c))
        self._caches[(mesh, problem)] = cache

    def submit(self, mesh: int, problem: int, points: np.ndarray, target_stderr: float, seed: int = 1,
               min_walks: int = 32, max_walks: int = 1 << 16, rms: bool = False, mode: str = "plain") -> int:
        """rms=False: every point meets the target; rms=True: the root mean
        square of the per-point standard errors does.  mode: "plain" WoS or
        "nc2lmc" with the cache set_nc registered (max/min walks count the
        coarse walks)."""
        from ._lib import N2W_REQUEST_MODE_NC2LMC, N2W_REQUEST_MODE_PLAIN, Request

        modes = {"plain": N2W_REQUEST_MODE_PLAIN, "nc2lmc": N2W_REQUEST_MODE_NC2LMC}
        if mode not in modes:
            raise ValueError(f"mode must be one of {sorted(modes)}")
        pts = np.ascontiguousarray(points, np.float32).reshape(-1, 3)
        r = Request(mesh, problem, len(pts), target_stderr, min_walks, max_walks, seed, 1 if rms else 0, modes[mode])
        rid = C.c_int64()
        call("n2w_server_submit", self._h, C.byref(r), _ptr(pts), C.byref(rid))
        self._sizes[rid.value] = len(pts)
        return rid.value

    def poll(self, rid: int) -> int:
        st = C.c_int()
        call("n2w_server_poll", self._h, rid, C.byref(st))
        return st.value

    def wait(self, rid: int, timeout: float = -1.0):
        from ._lib import RequestInfo

        n = self._sizes[rid]
        mean = np.empty(n, np.float64)
        se = np.empty(n, np.float64)
        info = RequestInfo()
        call("n2w_server_wait", self._h, rid, C.c_double(timeout), _ptr(mean), _ptr(se), C.byref(info))
        del self._sizes[rid]  # collected (a timeout leaves the request pending)
        return mean, se, {f: getattr(info, f) for f, _ in RequestInfo._fields_}

    def stats(self) -> dict:
        from ._lib import ServerStats

        s = ServerStats()
        call("n2w_server_get_stats", self._h, C.byref(s))
        return {f: getattr(s, f) for f, _ in ServerStats._fields_}

    def close(self):
        if getattr(self, "_h", None):
            lib.n2w_server_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()


def cache_config(**overrides):
    """Default cache config (16 levels x 2, 2^19, res 16..2048, 64x2 hidden, Adam 1e-2)."""
    from ._lib import CacheConfig

    cfg = CacheConfig()
    call("n2w_cache_config_default", C.byref(cfg))
    for k, v in overrides.items():
        setattr(cfg, k, v)
    return cfg


def cache_describe(cfg):
    g, m = C.c_int64(), C.c_int64()
    res = np.zeros(16, np.int32)
    tab = np.zeros(16, np.int32)
    call("n2w_cache_describe", C.byref(cfg), C.byref(g), C.byref(m), _ptr(res), _ptr(tab))
    L = cfg.n_levels
    return {"grid_params": g.value, "mlp_params": m.value, "resolution": res[:L].copy(), "table_size": tab[:L].copy()}


class Cache:
    """Hash-grid + MLP neural cache on the device (replaces tiny-cuda-nn)."""

    def __init__(self, cfg=None, handle=None):
        if handle is not None:
            self._h = handle
        else:
            cfg = cfg or cache_config()
            self._h = C.c_void_p()
            call("n2w_cache_create", C.byref(cfg), C.byref(self._h))

    @classmethod
    def load(cls, path: str) -> "Cache":
        h = C.c_void_p()
        call("n2w_cache_load", str(path).encode(), C.byref(h))
        return cls(handle=h)

    @property
    def handle(self):
        return self._h

    def info(self):
        from ._lib import CacheConfig

        cfg = CacheConfig()
        g, m = C.c_int64(), C.c_int64()
        res = np.zeros(16, np.int32)
        tab = np.zeros(16, np.int32)
        call("n2w_cache_info", self._h, C.byref(cfg), C.byref(g), C.byref(m), _ptr(res), _ptr(tab))
        L = cfg.n_levels
        return {"config": cfg, "grid_params": g.value, "mlp_params": m.value, "resolution": res[:L].copy(),
                "table_size": tab[:L].copy()}

    def n_params(self) -> int:
        i = self.info()
        return i["grid_params"] + i["mlp_params"]

    def params(self):
        n = self.n_params()
        p32 = np.empty(n, np.float32)
        p16 = np.empty(n, np.uint16)
        g = np.empty(n, np.float32)
        call("n2w_cache_get_params", self._h, _ptr(p32), _ptr(p16), _ptr(g))
        return p32, p16.view(np.float16), g

    def set_params(self, p: np.ndarray):
        p = np.ascontiguousarray(p, np.float32)
        assert len(p) == self.n_params()
        call("n2w_cache_set_params", self._h, _ptr(p))

    def infer(self, inputs: np.ndarray) -> np.ndarray:
        x = np.ascontiguousarray(inputs, np.float32).reshape(-1, 3)
        n = len(x)
        dx = DeviceBuffer.from_array(x)
        dy = DeviceBuffer(4 * max(n, 1))
        call("n2w_cache_infer", self._h, dx.ptr, n, dy.ptr, None)
        return dy.download(np.float32, n)

    def gradients(self, inputs, targets):
        x = np.ascontiguousarray(inputs, np.float32).reshape(-1, 3)
        t = np.ascontiguousarray(targets, np.float32)
        dx, dt = DeviceBuffer.from_array(x), DeviceBuffer.from_array(t)
        dy = DeviceBuffer(4 * len(x))
        call("n2w_cache_zero_grad", self._h, None)
        call("n2w_cache_gradients", self._h, dx.ptr, dt.ptr, len(x), dy.ptr, None)
        call("n2w_device_sync")
        return dy.download(np.float32, len(x)), self.params()[2]

    def train_step(self, d_inputs, d_targets, n, stream=None) -> float:
        loss = C.c_float()
        call("n2w_cache_train_step", self._h, d_inputs, d_targets, n, C.byref(loss),
             stream.handle if stream else None)
        return float(loss.value)

    def save(self, path: str):
        call("n2w_cache_save", self._h, str(path).encode())

    def __del__(self):
        if getattr(self, "_h", None):
            lib.n2w_cache_destroy(self._h)
            self._h = None


def device_count() -> int:
    n = C.c_int()
    st = lib.n2w_device_count(C.byref(n))
    return n.value if st == 0 else 0


def device_summary() -> str:
    buf = C.create_string_buffer(256)
    call("n2w_cuda_device_summary", buf, 256)
    return buf.value.decode()


def runtime_version() -> str:
    buf = C.create_string_buffer(128)
    call("n2w_cuda_runtime_version_string", buf, 128)
    return buf.value.decode()
