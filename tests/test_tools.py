"""Command-line tools: flags, exit codes and JSON schemas of the reference
tools (src/tools/*.cpp|cu), plus the host pieces they rely on.

CPU tests cover --help, option validation (exit 1 with "error: ..."), the host
brute-force closest point against the oracle, and the slice-grid rounding
rules.  GPU tests run each tool on a small case and check the keys the
reference's JSON carries, the honest implementation labels, and the numbers.
"""
from __future__ import annotations

import json
import subprocess
from pathlib import Path

import numpy as np
import pytest

from conftest import PKG, uniform_box

BIN = PKG / "bin"
TOOLS = ["n2wos_probe_cuda_bvh", "n2wos_probe_geometry_backends", "n2wos_eval_wavefront_wos",
         "n2wos_eval_tcnn_nc_wos", "n2wos_probe_tcnn_cache", "n2wos_render_harmonic_slice"]
SMALL_MESH = ["--bumpy-stacks", "32", "--bumpy-slices", "64"]


def run(tool, *args, timeout=600):
    return subprocess.run([str(BIN / tool), *map(str, args)], capture_output=True, text=True, timeout=timeout)


# ---- CPU ------------------------------------------------------------------------

@pytest.mark.parametrize("tool", TOOLS)
def test_help_exits_zero(tool):
    r = run(tool, "--help")
    assert r.returncode == 0
    assert "--" in (r.stdout + r.stderr)


@pytest.mark.parametrize("tool", TOOLS)
def test_unknown_option_is_an_error(tool):
    r = run(tool, "--no-such-flag", "1")
    assert r.returncode == 1
    assert r.stderr.startswith("error: ")


@pytest.mark.parametrize("tool,args,msg", [
    ("n2wos_probe_cuda_bvh", ["--queries", "0"], "--queries must be positive"),
    ("n2wos_probe_cuda_bvh", ["--mesh", "obj"], "--mesh-path is required"),
    ("n2wos_probe_cuda_bvh", ["--repeat", "x"], "failed to parse integer"),
    ("n2wos_probe_geometry_backends", ["--query-mode", "nope"], "--query-mode must be"),
    ("n2wos_probe_geometry_backends", ["--shell-min", "0.5", "--shell-max", "0.1"], "--shell-min"),
    ("n2wos_probe_geometry_backends", ["--cubql-build-methods", "rebin_radix"], "rebin_radix is disabled"),
    ("n2wos_eval_wavefront_wos", ["--method", "bogus"], "--method must be"),
    ("n2wos_eval_wavefront_wos", ["--x0", "1,2"], "--x0 expects 3"),
    ("n2wos_eval_tcnn_nc_wos", ["--cache-preset", "huge"], "unknown cache preset"),
    ("n2wos_eval_tcnn_nc_wos", ["--bc", "no_such_bc"], "unknown boundary mode"),
    ("n2wos_eval_tcnn_nc_wos", ["--label-refreshes", "0"], "invalid training schedule"),
    ("n2wos_eval_tcnn_nc_wos", ["--eval-mode", "cube"], "--eval-mode must be"),
    ("n2wos_probe_tcnn_cache", ["--network", "Transformer"], "--network must be"),
    ("n2wos_probe_tcnn_cache", ["--repeat", "0"], "repeat must be positive"),
    ("n2wos_render_harmonic_slice", ["--view", "zz"], "--view must be one of"),
    ("n2wos_render_harmonic_slice", ["--frame", "0,1,2"], "--frame expects 4"),
])
def test_validation_messages(tool, args, msg):
    r = run(tool, *args)
    assert r.returncode == 1
    assert msg in r.stderr


def test_bc_names_normalised_like_reference():
    # Hyphens / upper case are folded before the lookup (eval_tcnn_nc_wos.cu:147-162),
    # so a bad-but-normalisable name fails only later, not in option parsing.
    r = run("n2wos_eval_tcnn_nc_wos", "--bc", "Harmonic-Zebra-K8", "--train-points", "0")
    assert "invalid sample counts" in r.stderr


def test_host_bruteforce_matches_oracle(n2w):
    from oracle import bruteforce

    m = n2w.Mesh.bumpy_sphere_ref(24, 48, 0.15)
    m.normalize()
    v, t = m.arrays()
    pts = uniform_box(512, 1.35, seed=3)
    got = m.closest_point_host(pts, threads=4)
    ref = bruteforce(v, t, pts)
    np.testing.assert_array_equal(got["triangle_id"], ref["triangle_id"])
    np.testing.assert_array_equal(got["distance2"], ref["distance2"])
    np.testing.assert_array_equal(got["closest"], ref["closest"])


def test_host_bruteforce_surface_points_and_ties(n2w):
    from oracle import bruteforce

    m = n2w.Mesh.bumpy_sphere_ref(16, 32, 0.0)
    m.normalize()
    v, t = m.arrays()
    # Vertices are shared by up to six triangles: every query is an exact tie.
    got = m.closest_point_host(v[:200], threads=2)
    ref = bruteforce(v, t, v[:200])
    assert (ref["ties"] > 1).all()
    np.testing.assert_array_equal(got["triangle_id"], ref["triangle_id"])
    assert (got["distance2"] == 0).all()


def test_slice_rules_follow_reference_rounding(n2w):
    from n2w._lib import N2W_SLICE_RULE_EVAL, N2W_SLICE_RULE_RENDER, call
    import ctypes as C

    b = np.array([-1.0, -0.9, -1.1, 1.0, 0.95, 1.2], np.float32)
    W, H = 37, 23
    out = {}
    frames = {}
    for rule in (N2W_SLICE_RULE_RENDER, N2W_SLICE_RULE_EVAL):
        pts = np.empty((H * W, 3), np.float32)
        fr = np.empty(4, np.float32)
        call("n2w_slice_points_ex", b.ctypes.data_as(C.c_void_p), None, b"xz", C.c_float(0.25), W, H,
             C.c_float(0.02), 1, rule, pts.ctypes.data_as(C.c_void_p), fr.ctypes.data_as(C.c_void_p))
        out[rule], frames[rule] = pts, fr
    np.testing.assert_array_equal(frames[0], frames[1])
    u0, u1, v0, v1 = frames[0]
    f32 = np.float32
    for ix in (0, 5, W - 1):
        du = f32(u1) - f32(u0)
        render = f32(u0) + du * (f32(ix) / f32(W - 1))
        evalr = f32(u0) + (du * f32(ix)) / f32(W - 1)
        assert out[0][ix, 0] == render
        assert out[1][ix, 0] == evalr
    assert (out[0][:, 1] == f32(0.25)).all()  # y is the fixed axis of the xz view
    # An explicit frame replaces the bounds.
    pts = np.empty((4, 3), np.float32)
    frame = np.array([-2, 2, -1, 1], np.float32)
    fr = np.empty(4, np.float32)
    call("n2w_slice_points_ex", None, frame.ctypes.data_as(C.c_void_p), b"xy", C.c_float(0.0), 2, 2,
         C.c_float(0.0), 0, N2W_SLICE_RULE_EVAL, pts.ctypes.data_as(C.c_void_p), fr.ctypes.data_as(C.c_void_p))
    np.testing.assert_array_equal(fr, frame)
    np.testing.assert_array_equal(pts[:, :2], [[-2, -1], [2, -1], [-2, 1], [2, 1]])


# ---- GPU ------------------------------------------------------------------------

def load(path: Path) -> dict:
    return json.loads(path.read_text())


CUDA_KEYS = {"runtime", "device"}


@pytest.mark.gpu
def test_probe_cuda_bvh_schema_and_validation(gpu, tmp_path):
    out = tmp_path / "probe.json"
    r = run("n2wos_probe_cuda_bvh", *SMALL_MESH, "--queries", 20000, "--validate", 256, "--repeat", 3,
            "--output", out)
    assert r.returncode == 0, r.stderr
    j = load(out)
    assert j["schema"] == "n2wos_cuda_probe_bvh_v1"
    assert {"schema", "patch", "generated_at_utc", "command_line", "cuda", "implementation_mode", "options",
            "mesh_stats", "bvh_stats", "timing", "validation"} <= set(j)
    assert set(j["cuda"]) == CUDA_KEYS
    assert j["implementation_mode"]["geometry_query"] == "n2w_sm100a_bvh"
    assert {"kernel_ms", "kernel_ms_median", "kernel_ms_mean", "median_us_per_query", "mean_us_per_query",
            "median_mqueries_per_second"} <= set(j["timing"])
    v = j["validation"]
    assert v["checked"] == 256
    assert v["bad_distance_count_threshold_2e_4"] == 0
    assert v["triangle_id_mismatch_count"] == 0
    assert v["max_abs_distance_error"] == 0.0
    assert v["cuda_stack_overflow_count"] == 0
    assert {"nodes", "triangle_indices", "leaf_size", "max_depth"} <= set(j["bvh_stats"])
    assert {"normalization", "bounds_min", "bounds_max", "degenerate_triangles"} <= set(j["mesh_stats"])


@pytest.mark.gpu
@pytest.mark.parametrize("mode", ["uniform_box", "interior_slice", "surface_exact", "near_boundary_shell",
                                  "wos_like_prefix"])
def test_probe_geometry_backends_modes(gpu, tmp_path, mode):
    out = tmp_path / "geo.json"
    r = run("n2wos_probe_geometry_backends", *SMALL_MESH, "--queries", 8192, "--validate", 256, "--repeat", 2,
            "--query-mode", mode, "--cubql-leaf-sizes", "4,8", "--output", out)
    assert r.returncode == 0, r.stderr
    j = load(out)
    assert j["schema"] == "n2wos_geometry_backend_probe_v2"
    assert {"backend_policy", "options", "mesh_stats", "build_features", "recommendation", "backends"} <= set(j)
    b = j["backends"]
    built = {k: v for k, v in b.items() if v["built"]}
    # median-split comparison + {sah, spatial_median} x {4, 8}; radix / elh do not build here
    assert len(built) == 5
    for k, v in b.items():
        if "radix" in k or "elh" in k:
            assert not v["built"] and "cuBQL builder" in v["error"]
    for v in built.values():
        assert v["validation_passed"]
        assert v["validation"]["bad_distance_count_threshold_2e_4"] == 0
        assert v["validation"]["triangle_id_disagreement_count"] == 0
        assert v["validation"]["max_backend_distance_delta"] == 0.0
        assert v["overflow_count"] == 0
    assert j["recommendation"]["selected_production_candidate"].startswith("n2w_sm100a_bvh_")


@pytest.mark.gpu
def test_eval_wavefront_oracle_2lmc_unbiased(gpu, tmp_path):
    out = tmp_path / "wf.json"
    r = run("n2wos_eval_wavefront_wos", *SMALL_MESH, "--method", "oracle_2lmc", "--samples", 65536,
            "--depth-m", 4, "--epsilon", "1e-3", "--output", out)
    assert r.returncode == 0, r.stderr
    j = load(out)
    assert j["schema"] == "n2wos_wavefront_wos_eval_v1"
    assert set(j["runs"]) == {"coarse", "residual"}
    assert j["implementation_mode"]["cache_backend"] == "analytic_oracle_debug_only"
    run_keys = {"samples", "mean", "exact_target", "error", "abs_error", "sample_variance", "estimator_variance",
                "stderr", "mean_steps", "elapsed_ms", "us_per_sample", "launched_query_slots",
                "mean_launched_query_slots_per_sample", "scheduled_query_rounds", "forced_max_steps",
                "overflow_count"}
    assert run_keys <= set(j["runs"]["coarse"])
    e = j["estimator"]
    # Exact cache: the coarse level alone is unbiased, the residual has mean 0.
    assert abs(e["error"]) < 5 * e["stderr"] + 1e-4
    assert abs(j["runs"]["residual"]["mean"]) < 5 * j["runs"]["residual"]["stderr"] + 1e-4
    assert j["runs"]["residual"]["samples"] == 65536 // 8
    assert j["runs"]["coarse"]["mean_steps"] <= 4.0


@pytest.mark.gpu
@pytest.mark.parametrize("method", ["pure_wos", "oracle_coarse", "oracle_residual"])
def test_eval_wavefront_methods(gpu, tmp_path, method):
    out = tmp_path / "wf.json"
    r = run("n2wos_eval_wavefront_wos", *SMALL_MESH, "--method", method, "--samples", 32768, "--epsilon", "1e-3",
            "--engine", "persistent", "--output", out)
    assert r.returncode == 0, r.stderr
    j = load(out)
    e = j["estimator"]
    target = 0.0 if method == "oracle_residual" else e["exact"]
    assert abs(e["mean"] - target) < 5 * e["stderr"] + 1e-4
    assert list(j["runs"]) == [method]


@pytest.mark.gpu
def test_eval_tcnn_nc_wos_small(gpu, tmp_path):
    out = tmp_path / "nc.json"
    est = tmp_path / "est"
    r = run("n2wos_eval_tcnn_nc_wos", *SMALL_MESH, "--bc", "harmonic_x2_minus_y2", "--cache-preset", "light",
            "--train-points", 3000, "--eval-points", 512, "--label-refreshes", 2, "--walks-per-label-refresh", 16,
            "--train-steps-per-refresh", 150, "--pure-walks-per-point", 32, "--hybrid-walks-per-point", 8,
            "--coarse-walks-per-point", 32, "--residual-walks-per-point", 4, "--depth-m", 2, "--epsilon", "1e-3",
            "--save-estimates-prefix", est, "--save-train-points-prefix", est, "--output", out)
    assert r.returncode == 0, r.stderr
    j = load(out)
    assert j["schema"] == "n2wos_tcnn_nc_wos_eval_v4"
    assert j["implementation_mode"]["cache_backend"] == "n2w_hashgrid_mlp_native"
    assert j["implementation_mode"]["geometry_backend"] == "n2w_sm100a_bvh"
    assert {"pure_wos", "nc_wos", "nc_2lmc", "nc_2lmc_m2"} == set(j["runs"])
    assert j["options"]["train_points_padded"] == 3072
    tps = j["training_point_sampler"]
    assert tps["accepted_points"] == 3000 and tps["padding_reuses_accepted_points"]
    assert 0.2 < tps["acceptance_rate"] <= 1.0
    pure, nc, tl = j["runs"]["pure_wos"], j["runs"]["nc_wos"], j["runs"]["nc_2lmc"]
    # Plain WoS is unbiased: |mean bias| within a few standard errors of the point average.
    assert abs(pure["mean_bias"]) < 5 * np.sqrt(pure["mean_sample_variance"] / (32 * 512)) + 1e-3
    assert pure["rmse"] < 0.2
    assert 0.0 < nc["cache_query_fraction"] <= 1.0
    assert tl["coarse_samples"] == 512 * 32 and tl["residual_samples"] == 512 * 4
    assert tl["mean_coarse_steps"] <= 2.0
    assert {"coarse_cache_query_fraction", "residual_cache_query_fraction", "us_per_effective_sample"} <= set(tl)
    assert "nc_2lmc_rmse_div_pure_wos_rmse" in j["comparison"]
    csv = (tmp_path / "est_estimates.csv").read_text().splitlines()
    assert csv[0].startswith("point_id,x,y,z,analytic_value,pure_mean")
    assert len(csv) == 513
    assert len((tmp_path / "est_train_points.csv").read_text().splitlines()) == 3073


@pytest.mark.gpu
def test_eval_tcnn_nc_wos_slice_exact_labels(gpu, tmp_path):
    out = tmp_path / "nc_slice.json"
    r = run("n2wos_eval_tcnn_nc_wos", *SMALL_MESH, "--bc", "zebra4", "--label-source", "exact",
            "--cache-preset", "nano", "--train-points", 2048, "--label-refreshes", 1,
            "--train-steps-per-refresh", 100, "--eval-mode", "slice", "--slice-width", 48, "--slice-height", 32,
            "--pure-walks-per-point", 8, "--hybrid-walks-per-point", 4, "--coarse-walks-per-point", 8,
            "--residual-walks-per-point", 2, "--epsilon", "1e-3", "--enable-2lmc", 0, "--output", out)
    assert r.returncode == 0, r.stderr
    j = load(out)
    s = j["slice_eval"]
    assert s["candidate_pixels"] == 48 * 32 and 0 < s["inside_pixels"] < 48 * 32
    assert j["options"]["eval_points"] == s["inside_pixels"]
    assert set(j["runs"]) == {"pure_wos", "nc_wos"}
    assert Path(s["mask_ppm"]).read_bytes().startswith(b"P6\n48 32\n255\n")


@pytest.mark.gpu
def test_probe_tcnn_cache_learns_target(gpu, tmp_path):
    out = tmp_path / "cache.json"
    r = run("n2wos_probe_tcnn_cache", "--samples", 65536, "--batch-size", 16384, "--train-steps", 300,
            "--repeat", 3, "--n-levels", 8, "--log2-hashmap-size", 15, "--output", out)
    assert r.returncode == 0, r.stderr
    j = load(out)
    assert j["schema"] == "n2wos_tcnn_cache_probe_v1"
    assert j["implementation_mode"]["cache_backend"] == "n2w_hashgrid_mlp_native"
    assert {"training", "inference", "inference_plus_downstream_consumer", "validation"} <= set(j)
    v = j["validation"]
    assert v["checked_repeated_samples"] == 65536 * 3
    # x^2 - y^2 over [-1,1]^3 has RMS 0.73; a trained cache is far below that.
    assert v["rmse"] < 0.1
    assert abs(v["mean_exact"]) < 0.02


@pytest.mark.gpu
def test_render_harmonic_slice_outputs(gpu, tmp_path):
    prefix = tmp_path / "slice"
    r = run("n2wos_render_harmonic_slice", *SMALL_MESH, "--width", 40, "--height", 30, "--samples-per-pixel", 64,
            "--epsilon", "1e-3", "--output-prefix", prefix)
    assert r.returncode == 0, r.stderr
    j = load(Path(str(prefix) + ".json"))
    assert j["schema"] == "n2wos_harmonic_slice_render_v2"
    s = j["summary"]
    assert 0 < s["inside_pixels"] < 1200
    assert s["rmse_inside"] < 0.05
    rows = Path(str(prefix) + ".csv").read_text().splitlines()
    assert rows[0].startswith("ix,iy,x,y,z,inside,samples,mean,exact")
    assert len(rows) == 1201
    inside = [r for r in rows[1:] if r.split(",")[5] == "1"]
    assert len(inside) == s["inside_pixels"]
    for name in ("mask", "exact", "estimate", "error", "stderr"):
        data = Path(f"{prefix}_{name}.ppm").read_bytes()
        assert data.startswith(b"P6\n40 30\n255\n") and len(data) == len(b"P6\n40 30\n255\n") + 40 * 30 * 3
