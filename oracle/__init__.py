"""ORACLE — test infrastructure only (the checker, never the product).

numpy wrappers over liboracle.so (CPU restatement of the reference's hot path,
oracle.cpp) and, when built, oracle/_ref/libn2wos_ref.so (the reference's own CPU
sources) and oracle/_ref/libn2wos_ref_gpu.so (the reference's GPU kernel).
Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import it.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
_lib = None
_ref = None
_ref_gpu = None


def _p(a):
    return C.c_void_p(a.ctypes.data) if a is not None else None


def lib():
    global _lib
    if _lib is None:
        path = HERE / "liboracle.so"
        if not path.exists():
            from . import build as _b
            _b.build_oracle()
        _lib = C.CDLL(str(path))
    return _lib


def ref_available() -> bool:
    return (HERE / "_ref" / "libn2wos_ref.so").exists()


def ref():
    global _ref
    if _ref is None:
        _ref = C.CDLL(str(HERE / "_ref" / "libn2wos_ref.so"))
        _ref.ref_bumpy_sphere.restype = C.c_void_p
        _ref.ref_bumpy_sphere.argtypes = [C.c_int, C.c_int, C.c_float]
        _ref.ref_load_ply.restype = C.c_void_p
        _ref.ref_load_ply.argtypes = [C.c_char_p]
        _ref.ref_load_obj.restype = C.c_void_p
        _ref.ref_load_obj.argtypes = [C.c_char_p]
        _ref.ref_mesh_from_arrays.restype = C.c_void_p
        _ref.ref_mesh_from_arrays.argtypes = [C.c_void_p, C.c_int64, C.c_void_p, C.c_int64]
        _ref.ref_mesh_free.argtypes = [C.c_void_p]
        _ref.ref_mesh_counts.argtypes = [C.c_void_p, C.POINTER(C.c_int64), C.POINTER(C.c_int64)]
        _ref.ref_mesh_copy.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
        _ref.ref_normalize.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
        _ref.ref_bruteforce.argtypes = [C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p]
        _ref.ref_count_degenerate.restype = C.c_int64
        _ref.ref_count_degenerate.argtypes = [C.c_void_p]
        _ref.ref_host_bvh_stats.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_int64), C.POINTER(C.c_int32)]
        _ref.ref_last_error.restype = C.c_char_p
        _ref.ref_analytic_mode.argtypes = [C.c_int, C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p]
    return _ref


def ref_analytic(mode: int, points):
    """u and f of the reference's header-only analytic modes (13-16, 30-32)."""
    pts = np.ascontiguousarray(points, np.float32).reshape(-1, 3)
    u = np.empty(len(pts), np.float32)
    f = np.empty(len(pts), np.float32)
    if ref().ref_analytic_mode(mode, _p(pts), len(pts), _p(u), _p(f)) != 0:
        raise ValueError(f"mode {mode} is not an analytic reference mode")
    return u, f


class RefMesh:
    """A mesh owned by the reference library (n2wos::Mesh)."""

    def __init__(self, handle):
        if not handle:
            raise RuntimeError(ref().ref_last_error().decode())
        self.h = C.c_void_p(handle)

    @classmethod
    def bumpy_sphere(cls, stacks, slices, amplitude=0.15):
        return cls(ref().ref_bumpy_sphere(stacks, slices, amplitude))

    @classmethod
    def load_ply(cls, path):
        return cls(ref().ref_load_ply(str(path).encode()))

    @classmethod
    def load_obj(cls, path):
        return cls(ref().ref_load_obj(str(path).encode()))

    @classmethod
    def from_arrays(cls, v, t):
        v = np.ascontiguousarray(v, np.float32)
        t = np.ascontiguousarray(t, np.uint32)
        return cls(ref().ref_mesh_from_arrays(_p(v), len(v), _p(t), len(t)))

    def normalize(self):
        c = np.zeros(3, np.float32)
        s = np.zeros(1, np.float32)
        if ref().ref_normalize(self.h, _p(c), _p(s)) != 0:
            raise RuntimeError(ref().ref_last_error().decode())
        return c, float(s[0])

    def arrays(self):
        nv, nt = C.c_int64(), C.c_int64()
        ref().ref_mesh_counts(self.h, C.byref(nv), C.byref(nt))
        v = np.empty((nv.value, 3), np.float32)
        t = np.empty((nt.value, 3), np.uint32)
        ref().ref_mesh_copy(self.h, _p(v), _p(t))
        return v, t

    def bruteforce(self, points):
        pts = np.ascontiguousarray(points, np.float32).reshape(-1, 3)
        n = len(pts)
        d2 = np.empty(n, np.float32)
        cp = np.empty((n, 3), np.float32)
        ids = np.empty(n, np.int32)
        ref().ref_bruteforce(self.h, _p(pts), n, _p(d2), _p(cp), _p(ids))
        return d2, cp, ids

    def degenerate_count(self):
        return int(ref().ref_count_degenerate(self.h))

    def host_bvh(self, leaf_size=8):
        """The reference's own host BVH (build_host_bvh, median split)."""
        return RefHostBvh(self, leaf_size)

    def host_bvh_stats(self, leaf_size=8):
        n, d = C.c_int64(), C.c_int32()
        if ref().ref_host_bvh_stats(self.h, leaf_size, C.byref(n), C.byref(d)) != 0:
            raise RuntimeError(ref().ref_last_error().decode())
        return n.value, d.value

    def __del__(self):
        if getattr(self, "h", None) and _ref is not None:
            _ref.ref_mesh_free(self.h)
            self.h = None


class RefHostBvh:
    """Arrays of the reference's host BVH (src/cuda/bvh_build_host.cpp): 36-byte
    triangles, 40-byte nodes (box, left, right, first, count), leaf index list."""

    TRI = np.dtype([("v", np.float32, (3, 3))])
    NODE = np.dtype([("lo", np.float32, 3), ("hi", np.float32, 3), ("left", np.int32), ("right", np.int32),
                     ("first", np.int32), ("count", np.int32)])

    def __init__(self, mesh: "RefMesh", leaf_size: int = 8):
        R = ref()
        R.ref_host_bvh_build.restype = C.c_void_p
        R.ref_host_bvh_build.argtypes = [C.c_void_p, C.c_int]
        R.ref_host_bvh_counts.argtypes = [C.c_void_p] + [C.POINTER(C.c_int64)] * 3 + [C.POINTER(C.c_int32)]
        R.ref_host_bvh_copy.argtypes = [C.c_void_p] * 4
        R.ref_host_bvh_free.argtypes = [C.c_void_p]
        h = R.ref_host_bvh_build(mesh.h, leaf_size)
        if not h:
            raise RuntimeError(R.ref_last_error().decode())
        nt, nn, ni, dep = C.c_int64(), C.c_int64(), C.c_int64(), C.c_int32()
        R.ref_host_bvh_counts(h, C.byref(nt), C.byref(nn), C.byref(ni), C.byref(dep))
        self.tris = np.empty(nt.value, self.TRI)
        self.nodes = np.empty(nn.value, self.NODE)
        self.idx = np.empty(ni.value, np.int32)
        R.ref_host_bvh_copy(h, _p(self.tris), _p(self.nodes), _p(self.idx))
        R.ref_host_bvh_free(h)
        self.leaf_size = leaf_size
        self.depth = dep.value

    def args(self):
        return _p(self.nodes), _p(self.tris), _p(self.idx)


def ref_gpu_available() -> bool:
    return (HERE / "_ref" / "libn2wos_ref_gpu.so").exists()


def ref_gpu():
    global _ref_gpu
    if _ref_gpu is None:
        _ref_gpu = C.CDLL(str(HERE / "_ref" / "libn2wos_ref_gpu.so"))
        _ref_gpu.ref_gpu_bvh_create.restype = C.c_void_p
        _ref_gpu.ref_gpu_bvh_create.argtypes = [C.c_void_p, C.c_int64, C.c_void_p, C.c_int64, C.c_int]
        _ref_gpu.ref_gpu_query_device.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p,
                                                  C.c_void_p, C.c_void_p, C.c_int, C.c_void_p]
        _ref_gpu.ref_gpu_bvh_destroy.argtypes = [C.c_void_p]
        _ref_gpu.ref_gpu_last_error.restype = C.c_char_p
    return _ref_gpu


# ---- the CPU restatement ---------------------------------------------------------

def _setup():
    L = lib()
    L.oracle_bruteforce.argtypes = [C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p, C.c_int64, C.c_void_p,
                                    C.c_void_p, C.c_void_p, C.c_void_p, C.c_int]
    L.oracle_traverse4.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p,
                                   C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p,
                                   C.c_float, C.c_int]
    L.oracle_philox4x32_10.argtypes = [C.c_void_p, C.c_uint32, C.c_uint32, C.c_void_p]
    L.oracle_closest_point_on_triangle.argtypes = [C.c_void_p] * 5
    L.oracle_wos.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64, C.c_int, C.c_int,
                             C.c_float, C.c_float, C.c_uint32, C.c_uint32, C.c_void_p, C.c_void_p, C.c_void_p,
                             C.c_int]
    L.oracle_wos_ref_bvh.argtypes = [C.c_void_p] * 5 + [C.c_int64, C.c_int, C.c_int, C.c_float, C.c_float,
                                                        C.c_uint32, C.c_uint32, C.c_void_p, C.c_void_p, C.c_void_p,
                                                        C.c_int]
    L.oracle_ref_bvh_query.argtypes = [C.c_void_p] * 4 + [C.c_int64] + [C.c_void_p] * 5 + [C.c_int]
    L.oracle_inside_ref_bvh.argtypes = [C.c_void_p] * 4 + [C.c_int64, C.c_void_p, C.c_int]
    L.oracle_walk_samples.argtypes = [C.c_void_p] * 4 + [C.c_int64, C.c_int, C.c_int, C.c_int, C.c_int, C.c_float,
                                                        C.c_float, C.c_uint32, C.c_uint32] + [C.c_void_p] * 8 + [C.c_int]
    L.oracle_nc_combine.argtypes = [C.c_void_p] * 4 + [C.c_int64, C.c_void_p, C.c_void_p]
    L.oracle_nc_update_labels.argtypes = [C.c_void_p] * 4 + [C.c_int64, C.c_int, C.c_int, C.c_float, C.c_float,
                                                            C.c_uint32, C.c_uint32, C.c_int] + [C.c_void_p] * 5 + [C.c_int]
    L.oracle_icosphere_displaced.argtypes = [C.c_int, C.c_float, C.c_float, C.c_int, C.c_float, C.c_uint64,
                                             C.POINTER(C.c_int64), C.POINTER(C.c_int64), C.c_void_p, C.c_void_p]
    L.oracle_slice_points.argtypes = [C.c_void_p, C.c_int, C.c_float, C.c_int, C.c_int, C.c_float, C.c_int, C.c_int,
                                      C.c_void_p, C.c_void_p]
    return L


def bruteforce(vertices, triangles, points, threads=8):
    """Brute-force closest point with tie counts (reference closest_point.cpp:50-68)."""
    L = _setup()
    v = np.ascontiguousarray(vertices, np.float32)
    t = np.ascontiguousarray(triangles, np.uint32)
    pts = np.ascontiguousarray(points, np.float32).reshape(-1, 3)
    n = len(pts)
    d2 = np.empty(n, np.float32)
    cp = np.empty((n, 3), np.float32)
    ids = np.empty(n, np.int32)
    ties = np.empty(n, np.int32)
    L.oracle_bruteforce(_p(v), _p(t), len(t), _p(pts), n, _p(d2), _p(cp), _p(ids), _p(ties), threads)
    return {"distance2": d2, "closest": cp, "triangle_id": ids, "ties": ties}


def traverse4(nodes, tris, points, threads=8, seed=None):
    """The product's 4-wide traversal restated on the CPU (visit counts).

    seed: optional (slots int32[(n+1)^3], lo float32[3], h, n) seed grid."""
    L = _setup()
    pts = np.ascontiguousarray(points, np.float32).reshape(-1, 3)
    n = len(pts)
    d2 = np.empty(n, np.float32)
    cp = np.empty((n, 3), np.float32)
    ids = np.empty(n, np.int32)
    nv = np.empty(n, np.int32)
    nt = np.empty(n, np.int32)
    if seed is not None:
        slots, lo, h, sn = seed
        slots = np.ascontiguousarray(slots, np.int32)
        lo = np.ascontiguousarray(lo, np.float32)
        inv_h = float(np.float32(1.0) / np.float32(h))
        sargs = (_p(slots), _p(lo), inv_h, int(sn))
    else:
        sargs = (None, None, 0.0, 0)
    L.oracle_traverse4(_p(np.ascontiguousarray(nodes)), _p(np.ascontiguousarray(tris)), _p(pts), n, _p(d2),
                       _p(cp), _p(ids), _p(nv), _p(nt), threads, *sargs)
    return {"distance2": d2, "closest": cp, "triangle_id": ids, "node_visits": nv, "tri_tests": nt}


def inside_bruteforce(vertices, triangles, points, threads=8):
    """Reference +x ray-parity mask over all triangles (cubql_bvh.cu:407-455)."""
    L = lib()
    L.oracle_inside_bruteforce.argtypes = [C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p, C.c_int64,
                                           C.c_void_p, C.c_int]
    v = np.ascontiguousarray(vertices, np.float32)
    t = np.ascontiguousarray(triangles, np.uint32)
    pts = np.ascontiguousarray(points, np.float32).reshape(-1, 3)
    out = np.empty(len(pts), np.uint8)
    L.oracle_inside_bruteforce(_p(v), _p(t), len(t), _p(pts), len(pts), _p(out), threads)
    return out


def philox(ctr, k0, k1):
    L = _setup()
    c = np.ascontiguousarray(ctr, np.uint32)
    out = np.empty(4, np.uint32)
    L.oracle_philox4x32_10(_p(c), k0, k1, _p(out))
    return out


def closest_point_on_triangle(p, a, b, c):
    L = _setup()
    arrs = [np.ascontiguousarray(x, np.float32) for x in (p, a, b, c)]
    out = np.empty(3, np.float32)
    L.oracle_closest_point_on_triangle(*[_p(x) for x in arrs], _p(out))
    return out


def wos(nodes, tris, problem_bytes, points, walks_per_point, max_steps, eps, step_scale, k0, k1, threads=8):
    """Scalar CPU WoS (reference nc_wos_from_point semantics); per-point FP64 sums."""
    L = _setup()
    pts = np.ascontiguousarray(points, np.float32).reshape(-1, 3)
    n = len(pts)
    s = np.empty(n, np.float64)
    s2 = np.empty(n, np.float64)
    st = np.empty(n, np.float64)
    pb = np.frombuffer(problem_bytes, dtype=np.uint8).copy()
    L.oracle_wos(_p(np.ascontiguousarray(nodes)), _p(np.ascontiguousarray(tris)), _p(pb), _p(pts), n,
                 walks_per_point, max_steps, eps, step_scale, k0, k1, _p(s), _p(s2), _p(st), threads)
    W = float(walks_per_point)
    mean = s / W
    var = np.maximum((s2 - W * mean * mean) / max(W - 1, 1), 0.0)
    return {"mean": mean, "sample_variance": var, "stderr": np.sqrt(var / W), "mean_steps": st / W,
            "sum": s, "sum_sq": s2, "steps": st}


# ---- the reference path on the CPU: its host BVH, the walk, the slice mask -----

def _moments(s, s2, st, W):
    W = float(W)
    mean = s / W
    var = np.maximum((s2 - W * mean * mean) / max(W - 1, 1), 0.0)
    return {"mean": mean, "sample_variance": var, "stderr": np.sqrt(var / W), "mean_steps": st / W,
            "sum": s, "sum_sq": s2, "steps": st}


def wos_ref_bvh(bvh: RefHostBvh, problem_bytes, points, walks_per_point, max_steps, eps, step_scale, k0, k1,
                threads=8):
    """Scalar CPU WoS over the reference's own host BVH (reference
    nc_wos_from_point semantics, closest points by the restated
    closest_point_bvh_kernel traversal); per-point FP64 sums."""
    L = _setup()
    pts = np.ascontiguousarray(points, np.float32).reshape(-1, 3)
    n = len(pts)
    s, s2, st = (np.empty(n, np.float64) for _ in range(3))
    pb = np.frombuffer(problem_bytes, dtype=np.uint8).copy()
    L.oracle_wos_ref_bvh(*bvh.args(), _p(pb), _p(pts), n, walks_per_point, max_steps, eps, step_scale, k0, k1,
                         _p(s), _p(s2), _p(st), threads)
    return _moments(s, s2, st, walks_per_point)


def ref_bvh_query(bvh: RefHostBvh, points, threads=8):
    """Closest point over the reference's host BVH (restated bvh_query.cu:75-160)."""
    L = _setup()
    pts = np.ascontiguousarray(points, np.float32).reshape(-1, 3)
    n = len(pts)
    d2 = np.empty(n, np.float32)
    cp = np.empty((n, 3), np.float32)
    ids, nv, nt = (np.empty(n, np.int32) for _ in range(3))
    L.oracle_ref_bvh_query(*bvh.args(), _p(pts), n, _p(d2), _p(cp), _p(ids), _p(nv), _p(nt), threads)
    return {"distance2": d2, "closest": cp, "triangle_id": ids, "node_visits": nv, "tri_tests": nt}


def inside_ref_bvh(bvh: RefHostBvh, points, threads=8):
    """Reference +x ray-parity mask (cubql_bvh.cu:446-455), culled by the
    reference BVH's boxes (same hit count as the brute force)."""
    L = _setup()
    pts = np.ascontiguousarray(points, np.float32).reshape(-1, 3)
    out = np.empty(len(pts), np.uint8)
    L.oracle_inside_ref_bvh(*bvh.args(), _p(pts), len(pts), _p(out), threads)
    return out


MODE_PURE, MODE_PREFIX, MODE_RESIDUAL = 0, 1, 2


def walk_samples(nodes, tris, problem_bytes, points, walks_per_point, mode, depth_m, max_steps, eps, step_scale,
                 k0, k1, input_min=None, input_extent=None, threads=8):
    """Per-sample walks (sample i*W + j) restating nc_pure_wos_samples_kernel
    (mode 0), nc_hybrid_prefix_kernel (1) and nc_2lmc_prefix_continue_kernel (2)
    of cubql_bvh.cu:1422-1606."""
    L = _setup()
    pts = np.ascontiguousarray(points, np.float32).reshape(-1, 3)
    S = len(pts) * walks_per_point
    value, cont = np.empty(S, np.float32), np.empty(S, np.float32)
    inputs = np.empty((S, 3), np.float32)
    needs = np.empty(S, np.uint8)
    steps, forced = np.empty(S, np.int32), np.empty(S, np.int32)
    lo = np.ascontiguousarray(input_min if input_min is not None else np.zeros(3), np.float32)
    ext = np.ascontiguousarray(input_extent if input_extent is not None else np.ones(3), np.float32)
    pb = np.frombuffer(problem_bytes, dtype=np.uint8).copy()
    L.oracle_walk_samples(_p(np.ascontiguousarray(nodes)), _p(np.ascontiguousarray(tris)), _p(pb), _p(pts), len(pts),
                          walks_per_point, mode, depth_m, max_steps, eps, step_scale, k0, k1, _p(lo), _p(ext),
                          _p(value), _p(cont), _p(inputs), _p(needs), _p(steps), _p(forced), threads)
    return {"value": value, "continuation": cont, "inputs": inputs, "needs_cache": needs, "steps": steps,
            "forced": forced}


def nc_combine(cache_out, boundary, cont, needs):
    """nc_combine_cache_and_residual_kernel (cubql_bvh.cu:1608-1627)."""
    L = _setup()
    c = np.ascontiguousarray(cache_out, np.float32)
    b = np.ascontiguousarray(boundary, np.float32)
    w = np.ascontiguousarray(cont, np.float32)
    nd = np.ascontiguousarray(needs, np.uint8)
    nc, res = np.empty(len(c), np.float32), np.empty(len(c), np.float32)
    L.oracle_nc_combine(_p(c), _p(b), _p(w), _p(nd), len(c), _p(nc), _p(res))
    return nc, res


def nc_update_labels(nodes, tris, problem_bytes, points, walks_per_point, max_steps, eps, step_scale, k0, k1,
                     label_source, input_min, input_extent, targets, counts, threads=8):
    """One refresh of nc_update_labels_kernel (cubql_bvh.cu:1372-1420); updates
    `targets` (float32) and `counts` (int32) in place, returns the inputs."""
    L = _setup()
    pts = np.ascontiguousarray(points, np.float32).reshape(-1, 3)
    assert targets.dtype == np.float32 and counts.dtype == np.int32 and targets.flags.c_contiguous
    inputs = np.empty((len(pts), 3), np.float32)
    pb = np.frombuffer(problem_bytes, dtype=np.uint8).copy()
    lo = np.ascontiguousarray(input_min, np.float32)
    ext = np.ascontiguousarray(input_extent, np.float32)
    L.oracle_nc_update_labels(_p(np.ascontiguousarray(nodes)), _p(np.ascontiguousarray(tris)), _p(pb), _p(pts),
                              len(pts), walks_per_point, max_steps, eps, step_scale, k0, k1, label_source, _p(lo),
                              _p(ext), _p(inputs), _p(targets), _p(counts), threads)
    return inputs


def icosphere_displaced(level=6, amplitude=0.12, base_frequency=3.0, octaves=4, persistence=0.5, seed=12345):
    """The displaced icosphere of the Poisson slice workload (unnormalised)."""
    L = _setup()
    nv, nt = C.c_int64(), C.c_int64()
    L.oracle_icosphere_displaced(level, amplitude, base_frequency, octaves, persistence, seed, C.byref(nv),
                                 C.byref(nt), None, None)
    v = np.empty((nv.value, 3), np.float32)
    t = np.empty((nt.value, 3), np.uint32)
    L.oracle_icosphere_displaced(level, amplitude, base_frequency, octaves, persistence, seed, C.byref(nv),
                                 C.byref(nt), _p(v), _p(t))
    return v, t


SLICE_RULE_RENDER, SLICE_RULE_EVAL = 0, 1


def slice_points(bounds6, view="xy", plane=0.0, width=512, height=512, padding=0.02, preserve_aspect=True,
                 rule=SLICE_RULE_RENDER):
    """Slice pixel grid of the reference's render / evaluation tools."""
    L = _setup()
    b = np.ascontiguousarray(bounds6, np.float32)
    pts = np.empty((height * width, 3), np.float32)
    frame = np.empty(4, np.float32)
    if L.oracle_slice_points(_p(b), {"xy": 0, "xz": 1, "yz": 2}[view], plane, width, height, padding,
                             int(preserve_aspect), rule, _p(pts), _p(frame)) != 0:
        raise ValueError("bad slice view")
    return pts, frame


def problem_record(mode, source_sampling=0, omega=0.0, source_samples=0, charges=None) -> bytes:
    """A boundary-problem record with the byte layout the walkers read (mode,
    source rule, charge count, omega, 16 x (x, y, z, amplitude) charges, source
    samples per ball, reserved).  Modes the oracle evaluates: 0 (x^2 - y^2),
    4 (Re((x + i y)^8)), 12 (constant 1), 100 (charges), 101 (sin product with
    f = 3 omega^2 u)."""
    import struct

    ch = np.zeros((16, 4), np.float32)
    count = 0
    if charges is not None:
        c = np.asarray(charges, np.float32).reshape(-1, 4)
        count = len(c)
        ch[:count] = c
    return (struct.pack("<iiif", mode, source_sampling, count, np.float32(omega)) + ch.tobytes() +
            struct.pack("<ii", source_samples, 0))
