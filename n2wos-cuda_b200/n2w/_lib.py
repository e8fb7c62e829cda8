"""ctypes binding of libn2w.so (the C ABI declared in include/n2w.h).

The library is loaded from ``n2wos-cuda_b200/lib/libn2w.so``.  There is no
fallback: if the shared library is missing the import raises, so a caller can
never silently run a CPU path in its place.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

PKG_ROOT = Path(__file__).resolve().parent.parent
LIB_PATH = Path(os.environ.get("N2W_LIB", PKG_ROOT / "lib" / "libn2w.so"))

if not LIB_PATH.exists():
    raise ImportError(f"libn2w.so not found at {LIB_PATH}; build it with "
                      f"'python n2wos-cuda_b200/build.py' (no CPU fallback exists)")

lib = C.CDLL(str(LIB_PATH))

N2W_OK, N2W_EINVAL, N2W_ECUDA, N2W_ENOMEM, N2W_ETIMEOUT, N2W_EIO, N2W_EINTERNAL = range(7)

N2W_BC = {
    "harmonic_x2_minus_y2": 0, "external_charges_medium": 1, "external_charges_high": 2,
    "harmonic_zebra_k4": 3, "harmonic_zebra_k8": 4, "harmonic_zebra_k12": 5,
    "external_charges_shell_k8": 6, "external_charges_shell_k16": 7,
    "boundary_texture_stripes_k8": 8, "boundary_texture_stripes_k16": 9,
    "boundary_texture_checker_k8": 10, "boundary_texture_checker_k16": 11,
    "constant_one": 12, "harmonic_mixture_smooth": 13, "harmonic_mixture_figlike": 14,
    "harmonic_mixture_multiscale": 15, "harmonic_mixture_figlike_hf": 16,
    "poisson_multiscale": 30, "poisson_figlike_hf": 31, "poisson_figlike_hf_x5": 32,
    "charges_seeded": 100, "poisson_sinprod": 101,
}
N2W_SOURCE_BALL, N2W_SOURCE_CENTER = 0, 1
N2W_WALK_PURE, N2W_WALK_PREFIX, N2W_WALK_RESIDUAL = 0, 1, 2
N2W_MAX_CHARGES = 16


class N2wError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"[n2w error {code}] {msg}")
        self.code = code


class Vec3(C.Structure):
    _fields_ = [("x", C.c_float), ("y", C.c_float), ("z", C.c_float)]


class BvhStats(C.Structure):
    _fields_ = [("triangles", C.c_int64), ("nodes", C.c_int64), ("binary_nodes", C.c_int64),
                ("leaves", C.c_int64), ("leaf_size", C.c_int32), ("max_depth", C.c_int32),
                ("build_milliseconds", C.c_double), ("sah_cost", C.c_double),
                ("device_bytes", C.c_int64)]


class Problem(C.Structure):
    _fields_ = [("mode", C.c_int32), ("source_sampling", C.c_int32), ("charge_count", C.c_int32),
                ("omega", C.c_float), ("charges", (C.c_float * 4) * N2W_MAX_CHARGES), ("source_samples", C.c_int32),
                ("reserved", C.c_int32)]


class WalkOptions(C.Structure):
    _fields_ = [("walks_per_point", C.c_int32), ("max_steps", C.c_int32), ("depth_m", C.c_int32),
                ("epsilon", C.c_float), ("step_scale", C.c_float), ("seed", C.c_uint64),
                ("block_size", C.c_int32), ("blocks_per_sm", C.c_int32), ("chunk", C.c_int32),
                ("accumulate", C.c_int32), ("deadline_ns", C.c_int64), ("regen_threshold", C.c_int32)]


class PointStats(C.Structure):
    _fields_ = [("d_sum", C.c_void_p), ("d_sum_sq", C.c_void_p), ("d_count", C.c_void_p),
                ("d_steps", C.c_void_p), ("d_forced", C.c_void_p)]


class WalkCounters(C.Structure):
    _fields_ = [(n, C.c_ulonglong) for n in
                ("walks", "steps", "queries", "node_visits", "tri_tests", "overflow", "forced",
                 "timed_out")]


class CacheConfig(C.Structure):
    _fields_ = [("n_levels", C.c_int32), ("n_features_per_level", C.c_int32), ("log2_hashmap_size", C.c_int32),
                ("base_resolution", C.c_float), ("per_level_scale", C.c_float), ("max_resolution", C.c_float),
                ("n_neurons", C.c_int32), ("n_hidden_layers", C.c_int32), ("learning_rate", C.c_float),
                ("beta1", C.c_float), ("beta2", C.c_float), ("epsilon", C.c_float), ("seed", C.c_uint64)]


class NcTrainOptions(C.Structure):
    _fields_ = [("steps", C.c_int32), ("batch", C.c_int32), ("walks_per_label", C.c_int32),
                ("max_steps", C.c_int32), ("epsilon", C.c_float), ("step_scale", C.c_float), ("seed", C.c_uint64),
                ("input_min", C.c_float * 3), ("input_extent", C.c_float * 3), ("sample_lo", C.c_float * 3),
                ("sample_hi", C.c_float * 3)]


class Nc2lmcOptions(C.Structure):
    _fields_ = [("coarse_walks", C.c_int32), ("residual_walks", C.c_int32), ("depth_m", C.c_int32),
                ("max_steps", C.c_int32), ("epsilon", C.c_float), ("step_scale", C.c_float), ("seed", C.c_uint64),
                ("input_min", C.c_float * 3), ("input_extent", C.c_float * 3), ("point_batch", C.c_int32)]


class NcProgressiveOptions(C.Structure):
    _fields_ = [("blocks", C.c_int32), ("train_steps_per_block", C.c_int32), ("overlap", C.c_int32),
                ("reserved", C.c_int32), ("train", NcTrainOptions), ("estimate", Nc2lmcOptions)]


class NcProgressiveBlock(C.Structure):
    _fields_ = [("eval_ms", C.c_float), ("train_ms", C.c_float), ("wall_ms", C.c_float), ("reserved", C.c_float)]


class Nc2lmcCounters(C.Structure):
    _fields_ = [(n, C.c_ulonglong) for n in
                ("coarse_cache_queries", "coarse_forced", "coarse_overflow", "residual_cache_queries",
                 "residual_forced", "residual_overflow")]


class NcLabelOptions(C.Structure):
    _fields_ = [("walks_per_point", C.c_int32), ("max_steps", C.c_int32), ("epsilon", C.c_float),
                ("step_scale", C.c_float), ("seed", C.c_uint64), ("refresh_index", C.c_int32),
                ("label_source", C.c_int32), ("input_min", C.c_float * 3), ("input_extent", C.c_float * 3),
                ("block_size", C.c_int32), ("reserved", C.c_int32)]


class BatchItem(C.Structure):
    _fields_ = [("mesh", C.c_int32), ("problem", C.c_int32), ("d_points", C.c_void_p), ("point_count", C.c_int64),
                ("walks_per_point", C.c_int32), ("reserved", C.c_int32), ("seed", C.c_uint64),
                ("stats", PointStats)]


class BatchTuning(C.Structure):
    _fields_ = [("block_size", C.c_int32), ("blocks_per_sm", C.c_int32), ("chunk", C.c_int32),
                ("regen_threshold", C.c_int32), ("reg_variant", C.c_int32), ("ms", C.c_float)]


class ServerOptions(C.Structure):
    _fields_ = [("pool_bytes", C.c_int64), ("pool_fraction", C.c_float), ("max_inflight", C.c_int32),
                ("tick_walks", C.c_int64), ("max_steps", C.c_int32), ("epsilon", C.c_float),
                ("step_scale", C.c_float), ("block_size", C.c_int32), ("regen_threshold", C.c_int32),
                ("chunk", C.c_int32), ("tick_walks_max", C.c_int64)]


class Request(C.Structure):
    _fields_ = [("mesh", C.c_int32), ("problem", C.c_int32), ("point_count", C.c_int64),
                ("target_stderr", C.c_float), ("min_walks_per_point", C.c_int32),
                ("max_walks_per_point", C.c_int32), ("seed", C.c_uint64), ("stderr_norm", C.c_int32),
                ("mode", C.c_int32)]


class ServerNc(C.Structure):
    _fields_ = [("cache", C.c_void_p), ("input_min", C.c_float * 3), ("input_extent", C.c_float * 3),
                ("depth_m", C.c_int32), ("residual_fraction", C.c_float)]


class RequestInfo(C.Structure):
    _fields_ = [("state", C.c_int32), ("sweeps", C.c_int32), ("walks_per_point", C.c_int64), ("ticks", C.c_int64),
                ("max_stderr", C.c_float), ("rms_stderr", C.c_float), ("queue_seconds", C.c_double),
                ("latency_seconds", C.c_double), ("residual_walks_per_point", C.c_int64)]


class ServerStats(C.Structure):
    _fields_ = [(n, C.c_int64) for n in
                ("submitted", "completed", "inflight", "pending", "peak_inflight", "ticks", "walks", "walk_steps",
                 "overflow", "pool_bytes", "pool_used", "peak_pool_bytes", "nc_chunks", "nc_walks",
                 "tick_us", "nc_us", "tick_gpu_us")]


N2W_REQUEST_PENDING, N2W_REQUEST_ACTIVE, N2W_REQUEST_DONE, N2W_REQUEST_CAPPED, N2W_REQUEST_FAILED = range(5)
N2W_REQUEST_MODE_PLAIN, N2W_REQUEST_MODE_NC2LMC = 0, 1
N2W_LABEL_EXACT, N2W_LABEL_WOS = 0, 1
N2W_SLICE_RULE_RENDER, N2W_SLICE_RULE_EVAL = 0, 1
N2W_DTYPE_F32, N2W_DTYPE_F64, N2W_DTYPE_U32, N2W_DTYPE_U64, N2W_DTYPE_I32 = range(5)
N2W_OP_SUM, N2W_OP_MAX, N2W_OP_MIN = range(3)

P = C.c_void_p
I = C.c_int
I64 = C.c_int64
PP = C.POINTER(C.c_void_p)

_SIGS = {
    "n2w_last_error": (C.c_char_p, []),
    "n2w_abi_version": (I, []),
    "n2w_cuda_runtime_version_string": (I, [C.c_char_p, C.c_size_t]),
    "n2w_cuda_device_summary": (I, [C.c_char_p, C.c_size_t]),
    "n2w_mesh_create": (I, [P, I64, P, I64, C.c_char_p, PP]),
    "n2w_mesh_bumpy_sphere_ref": (I, [I, I, C.c_float, PP]),
    "n2w_mesh_bumpy_sphere_trig": (I, [I, I, C.c_float, I, I, PP]),
    "n2w_mesh_icosphere_displaced": (I, [I, C.c_float, C.c_float, I, C.c_float, C.c_uint64, PP]),
    "n2w_mesh_load_ply": (I, [C.c_char_p, PP]),
    "n2w_mesh_load_obj": (I, [C.c_char_p, PP]),
    "n2w_mesh_normalize": (I, [P, P, P]),
    "n2w_mesh_counts": (I, [P, C.POINTER(I64), C.POINTER(I64)]),
    "n2w_mesh_copy_out": (I, [P, P, P]),
    "n2w_mesh_bounds": (I, [P, P]),
    "n2w_mesh_count_degenerate": (I, [P, C.c_float, C.POINTER(I64)]),
    "n2w_mesh_closest_point_host": (I, [P, P, I64, P, P, P, I]),
    "n2w_mesh_name": (C.c_char_p, [P]),
    "n2w_mesh_free": (None, [P]),
    "n2w_bvh_host_build": (I, [P, I, C.c_char_p, PP]),
    "n2w_bvh_host_stats": (I, [P, C.POINTER(BvhStats)]),
    "n2w_bvh_host_copy": (I, [P, P, P]),
    "n2w_bvh_host_free": (None, [P]),
    "n2w_bvh_create": (I, [P, I, C.c_char_p, PP]),
    "n2w_bvh_stats_get": (I, [P, C.POINTER(BvhStats)]),
    "n2w_bvh_destroy": (None, [P]),
    "n2w_bvh_query_device": (I, [P, P, I, P, P, P, P, I, P]),
    "n2w_bvh_query_device_masked": (I, [P, P, P, I, P, P, P, P, I, P]),
    "n2w_bvh_query_device_counted": (I, [P, P, I, P, P, P, P, P, P, I, P]),
    "n2w_bvh_copy_layout": (I, [P, P, P]),
    "n2w_bvh_inside_device": (I, [P, P, I, P, P, I, P]),
    "n2w_slice_points": (I, [P, C.c_char_p, C.c_float, I, I, C.c_float, I, P, P]),
    "n2w_slice_points_ex": (I, [P, P, C.c_char_p, C.c_float, I, I, C.c_float, I, I, P, P]),
    "n2w_problem_charges_seeded": (I, [I, C.c_float, C.c_float, C.c_uint64, C.POINTER(Problem)]),
    "n2w_problem_sinprod": (I, [C.c_float, I, C.POINTER(Problem)]),
    "n2w_problem_reference_mode": (I, [I, I, C.POINTER(Problem)]),
    "n2w_problem_exact": (I, [C.POINTER(Problem), P, I64, P]),
    "n2w_problem_eval_f32": (I, [C.POINTER(Problem), P, I64, P, P]),
    "n2w_problem_mode_from_name": (I, [C.c_char_p, C.POINTER(I)]),
    "n2w_problem_mode_name": (C.c_char_p, [I]),
    "n2w_rng_philox4x32_10": (I, [P, C.c_uint64, C.c_uint32, P]),
    "n2w_wos_workspace_bytes": (C.c_size_t, [I64]),
    "n2w_bvh_seed_grid": (I, [P, P, P, P, P]),
    "n2w_wos_estimate": (I, [P, C.POINTER(Problem), P, I64, C.POINTER(WalkOptions), PointStats, P, P, P]),
    "n2w_wos_estimate_noalloc": (I, [P, C.POINTER(Problem), P, I64, C.POINTER(WalkOptions), PointStats, P, P]),
    "n2w_wos_pure_samples": (I, [P, C.POINTER(Problem), P, I64, C.POINTER(WalkOptions), P, P, P, P, P]),
    "n2w_wos_prefix_samples": (I, [P, C.POINTER(Problem), P, I64, C.POINTER(WalkOptions), I, P, P,
                                   P, P, P, P, P, P, P, P]),
    "n2w_wos_combine": (I, [P, P, P, P, I64, P, P, I, P]),
    "n2w_reduce_samples": (I, [P, P, P, I64, I, PointStats, I, P]),
    "n2w_cache_config_default": (I, [C.POINTER(CacheConfig)]),
    "n2w_cache_describe": (I, [C.POINTER(CacheConfig), C.POINTER(I64), C.POINTER(I64), P, P]),
    "n2w_cache_create": (I, [C.POINTER(CacheConfig), PP]),
    "n2w_cache_destroy": (None, [P]),
    "n2w_cache_info": (I, [P, C.POINTER(CacheConfig), C.POINTER(I64), C.POINTER(I64), P, P]),
    "n2w_cache_infer": (I, [P, P, I64, P, P]),
    "n2w_cache_gradients": (I, [P, P, P, I64, P, P]),
    "n2w_cache_train_step": (I, [P, P, P, I64, C.POINTER(C.c_float), P]),
    "n2w_cache_zero_grad": (I, [P, P]),
    "n2w_cache_gradient_buffer": (I, [P, C.POINTER(P), C.POINTER(C.c_int64), C.POINTER(P)]),
    "n2w_cache_apply_gradients": (I, [P, C.c_float, P]),
    "n2w_cache_copy_params": (I, [P, P, P]),
    "n2w_cache_get_params": (I, [P, P, P, P]),
    "n2w_cache_set_params": (I, [P, P]),
    "n2w_cache_save": (I, [P, C.c_char_p]),
    "n2w_cache_load": (I, [C.c_char_p, PP]),
    "n2w_sample_interior": (I, [P, P, P, I64, C.c_uint64, P, C.POINTER(I64), P]),
    "n2w_sample_interior_ex": (I, [P, P, P, I64, C.c_uint64, P, C.POINTER(I64), C.POINTER(I64), P]),
    "n2w_map_to_unit": (I, [P, I64, P, P, P, P]),
    "n2w_nc_train": (I, [P, P, C.POINTER(Problem), C.POINTER(NcTrainOptions), P, P]),
    "n2w_nc_train_dp": (I, [P, P, C.POINTER(Problem), C.POINTER(NcTrainOptions), P, P, P]),
    "n2w_nc_progressive": (I, [P, P, P, C.POINTER(Problem), P, I64, C.POINTER(NcProgressiveOptions), PointStats,
                               PointStats, P, P, P]),
    "n2w_nc2lmc_estimate": (I, [P, C.POINTER(Problem), P, P, I64, C.POINTER(Nc2lmcOptions), PointStats,
                                PointStats, P]),
    "n2w_nc2lmc_estimate_ex": (I, [P, C.POINTER(Problem), P, P, I64, C.POINTER(Nc2lmcOptions), PointStats,
                                   PointStats, P, P]),
    "n2w_nc_update_labels": (I, [P, C.POINTER(Problem), P, I64, C.POINTER(NcLabelOptions), PointStats, P, P, P,
                                 P]),
    "n2w_problem_exact_device": (I, [C.POINTER(Problem), P, I64, P, P]),
    "n2w_oracle_cache_infer": (I, [C.POINTER(Problem), P, I64, P, P, P, P]),
    "n2w_fill_unit_samples": (I, [C.POINTER(Problem), I64, C.c_uint64, C.c_uint32, P, P, P, P, P]),
    "n2w_compare_accumulate": (I, [P, P, I64, P, P]),
    "n2w_count_samples": (I, [P, P, P, I64, P, P]),
    "n2w_scene_create": (I, [C.POINTER(C.c_void_p), I, PP]),
    "n2w_scene_info": (I, [P, C.POINTER(I), C.POINTER(I64), C.POINTER(I64), C.POINTER(I64)]),
    "n2w_scene_destroy": (None, [P]),
    "n2w_batch_create": (I, [P, C.POINTER(Problem), I, C.POINTER(BatchItem), I, C.POINTER(WalkOptions), PP]),
    "n2w_batch_info": (I, [P, C.POINTER(I64), C.POINTER(I64), C.POINTER(WalkOptions), C.POINTER(I)]),
    "n2w_batch_set_seeds": (I, [P, C.POINTER(C.c_uint64), P]),
    "n2w_batch_launch": (I, [P, P, P]),
    "n2w_batch_capture_graph": (I, [P, P, P]),
    "n2w_batch_graph_launch": (I, [P, P]),
    "n2w_batch_autotune": (I, [P, C.c_double, C.POINTER(BatchTuning), C.POINTER(BatchTuning), I, C.POINTER(I), P]),
    "n2w_batch_set_tuning": (I, [P, C.POINTER(BatchTuning), P]),
    "n2w_batch_destroy": (None, [P]),
    "n2w_server_options_default": (I, [C.POINTER(ServerOptions)]),
    "n2w_server_create": (I, [C.POINTER(C.c_void_p), I, C.POINTER(Problem), I, C.POINTER(ServerOptions), PP]),
    "n2w_server_set_nc": (I, [P, I, I, C.POINTER(ServerNc)]),
    "n2w_server_submit": (I, [P, C.POINTER(Request), P, C.POINTER(I64)]),
    "n2w_server_poll": (I, [P, I64, C.POINTER(I)]),
    "n2w_server_wait": (I, [P, I64, C.c_double, P, P, C.POINTER(RequestInfo)]),
    "n2w_server_get_stats": (I, [P, C.POINTER(ServerStats)]),
    "n2w_server_destroy": (None, [P]),
    "n2w_device_count": (I, [C.POINTER(I)]),
    "n2w_set_device": (I, [I]),
    "n2w_malloc": (I, [PP, C.c_size_t]),
    "n2w_free": (I, [P]),
    "n2w_malloc_host": (I, [PP, C.c_size_t]),
    "n2w_free_host": (I, [P]),
    "n2w_memcpy_h2d": (I, [P, P, C.c_size_t, P]),
    "n2w_memcpy_d2h": (I, [P, P, C.c_size_t, P]),
    "n2w_memset": (I, [P, I, C.c_size_t, P]),
    "n2w_stream_create": (I, [PP]),
    "n2w_stream_destroy": (I, [P]),
    "n2w_stream_sync": (I, [P]),
    "n2w_comm_unique_id": (I, [P]),
    "n2w_comm_create": (I, [P, I, I, C.POINTER(P)]),
    "n2w_comm_info": (I, [P, C.POINTER(I), C.POINTER(I)]),
    "n2w_comm_allreduce": (I, [P, P, P, C.c_int64, I, I, P]),
    "n2w_comm_allreduce_point_stats": (I, [P, PointStats, C.c_int64, P]),
    "n2w_comm_barrier": (I, [P, P]),
    "n2w_comm_destroy": (None, [P]),
    "n2w_device_sync": (I, []),
    "n2w_timer_create": (I, [PP]),
    "n2w_timer_start": (I, [P, P]),
    "n2w_timer_stop": (I, [P, P]),
    "n2w_timer_elapsed_ms": (I, [P, C.POINTER(C.c_float)]),
    "n2w_timer_destroy": (None, [P]),
    "n2w_sm_count": (I, [C.POINTER(I)]),
    "n2w_mem_info": (I, [C.POINTER(C.c_size_t), C.POINTER(C.c_size_t)]),
    "n2w_probe_read_bandwidth": (I, [I, C.c_size_t, I, C.POINTER(C.c_double)]),
}

EXPORTED = tuple(_SIGS)

for _name, (_res, _args) in _SIGS.items():
    _fn = getattr(lib, _name)
    _fn.restype = _res
    _fn.argtypes = _args


def check(status: int) -> None:
    if status != N2W_OK:
        raise N2wError(status, lib.n2w_last_error().decode(errors="replace"))


def call(name: str, *args) -> None:
    check(getattr(lib, name)(*args))
