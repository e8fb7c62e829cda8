"""Walker parity against the reference's own published runs.

The reference commits two runs of its n2wos_eval_tcnn_nc_wos (RTX 3070, cuBQL
SAH, tiny-cuda-nn): figures/zebra_k8_m2.json (its bumpy sphere, boundary
harmonic_zebra_k8 = Re((x + i y)^8), z = 0 slice) and
figures/bunny_zebra_k8_m2.json (the bundled bunny, z = 0.12 slice), both
512 x 512 pixels, eps = 1e-4, 64 pure walks per interior pixel.  Their JSON
fields and slice masks are fixtures (tests/golden/make_figure_golden.py).

Each test runs this project's n2wos_eval_tcnn_nc_wos with the published
command line (output paths replaced) and checks:
* the mesh: vertex / triangle counts, bounds and the normalisation centre and
  scale, bit-equal as float32;
* the slice: frame bit-equal, the interior mask pixel for pixel, hence the
  number of evaluation points;
* runs.pure_wos: mean steps per walk within 4 sigma of the published value
  (sigma from the per-walk step spread, both runs' Monte Carlo error), mean
  per-pixel sample variance within 2 %, and the slice MSE against the exact
  solution within 4 sigma of the published RMSE^2 (sigma of the MSE from the
  per-pixel variances, both runs), with no forced or overflowed walks.
The reference's RNG (PCG32) differs from this walker's (Philox), so walk
statistics agree in distribution, never bit for bit.
"""
from __future__ import annotations

import csv
import ctypes as C
import json
import subprocess

import numpy as np
import pytest

from conftest import GOLDEN, PKG, REFERENCE_BUNNY

pytestmark = pytest.mark.gpu

FIG = json.loads((GOLDEN / "figure_runs.json").read_text())
MASKS = np.load(GOLDEN / "figure_masks.npz")
TOOL = PKG / "bin" / "n2wos_eval_tcnn_nc_wos"


def published_args(name: str, out_dir) -> list[str]:
    """The published command line with its file paths redirected."""
    argv = FIG[name]["command_line"].split()[1:]
    out, i = [], 0
    while i < len(argv):
        a = argv[i]
        if a == "--mesh-path":
            out += [a, str(REFERENCE_BUNNY)]
        elif a == "--save-estimates-prefix":
            out += [a, str(out_dir / name)]
        elif a == "--output":
            out += [a, str(out_dir / f"{name}.json")]
        else:
            out.append(a)
            i += 1
            continue
        i += 2
    return out


def read_ppm_mask(path) -> np.ndarray:
    raw = open(path, "rb").read()
    _, dims, _, body = raw.split(b"\n", 3)
    w, h = map(int, dims.split())
    return np.frombuffer(body, np.uint8).reshape(h, w, 3)[..., 0] == 235


@pytest.fixture(scope="module", params=sorted(FIG))
def figure_run(request, gpu, tmp_path_factory):
    name = request.param
    if "--mesh-path" in FIG[name]["command_line"] and not REFERENCE_BUNNY.exists():
        pytest.fail(f"{REFERENCE_BUNNY} is missing: oracle/build.py stages it from the reference checkout")
    out_dir = tmp_path_factory.mktemp(name)
    r = subprocess.run([str(TOOL), *published_args(name, out_dir)], capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stderr
    js = json.loads((out_dir / f"{name}.json").read_text())
    with open(out_dir / f"{name}_estimates.csv") as f:
        rows = list(csv.DictReader(f))
    est = {k: np.array([float(row[k]) for row in rows]) for k in ("pure_mean", "pure_sample_variance",
                                                                  "analytic_value", "x", "y", "z")}
    return name, js, out_dir, est


def f32(x):
    return np.float32(np.float64(x))


def test_mesh_and_normalisation_bit_equal(figure_run):
    name, js, _, _ = figure_run
    want, got = FIG[name]["mesh_stats"], js["mesh_stats"]
    assert got["triangles"] == want["triangles"] and got["vertices"] == want["vertices"]
    assert got["degenerate_triangles"] == want["degenerate_triangles"]
    for k in ("bounds_min", "bounds_max"):
        assert [f32(a) for a in got[k]] == [f32(b) for b in want[k]], k
    assert [f32(a) for a in got["normalization"]["center"]] == [f32(b) for b in want["normalization"]["center"]]
    assert f32(got["normalization"]["scale"]) == f32(want["normalization"]["scale"])


def test_slice_frame_and_mask_pixel_exact(figure_run):
    name, js, _, _ = figure_run
    want, got = FIG[name]["slice_eval"], js["slice_eval"]
    for k in ("frame_u_min", "frame_u_max", "frame_v_min", "frame_v_max"):
        assert f32(got[k]) == f32(want[k]), k
    mask = read_ppm_mask(got["mask_ppm"])
    h, w = MASKS[name + "_shape"]
    published = np.unpackbits(MASKS[name])[: h * w].reshape(h, w).astype(bool)
    assert np.array_equal(mask, published), f"{int((mask != published).sum())} pixels differ"
    assert got["inside_pixels"] == want["inside_pixels"] == js["options"]["eval_points"]


def test_pure_wos_statistics_match_published(figure_run, gpu):
    name, js, out_dir, est = figure_run
    want, got = FIG[name]["runs"]["pure_wos"], js["runs"]["pure_wos"]
    W = want["walks_per_point"]
    assert got["eval_points"] == want["eval_points"] and got["walks_per_point"] == W
    assert got["forced_max_steps"] == 0 and got["overflow_count"] == 0

    # spread of steps per walk, from per-sample walks on every 16th evaluation point
    pts = np.stack([est["x"], est["y"], est["z"]], 1).astype(np.float32)[::16]
    mesh = gpu.Mesh.bumpy_sphere_ref(128, 256, 0.15) if "--mesh-path" not in FIG[name]["command_line"] \
        else gpu.Mesh.load(str(REFERENCE_BUNNY))
    mesh.normalize()
    bvh = gpu.Bvh(mesh, 4, "sah")
    p = gpu.problem_from_name("harmonic_zebra_k8")
    o = gpu.walk_options(walks_per_point=W, epsilon=float(FIG[name]["options"]["epsilon"]), seed=99)
    from n2w._lib import call
    n = len(pts)
    dp = gpu.DeviceBuffer.from_array(pts)
    val, st, fo, ov = (gpu.DeviceBuffer(4 * n * W) for _ in range(4))
    call("n2w_wos_pure_samples", bvh.handle, C.byref(p), dp.ptr, n, C.byref(o), val.ptr, st.ptr, fo.ptr, ov.ptr,
         None)
    steps = st.download(np.int32).astype(np.float64)
    samples = want["eval_points"] * W
    sigma_steps = np.sqrt(2.0) * steps.std() / np.sqrt(samples)  # both runs' Monte Carlo error
    assert abs(got["mean_steps"] - want["mean_steps"]) <= 4 * sigma_steps, \
        (got["mean_steps"], want["mean_steps"], sigma_steps)

    assert abs(got["mean_sample_variance"] / want["mean_sample_variance"] - 1) <= 0.02, \
        (got["mean_sample_variance"], want["mean_sample_variance"])

    mse = got["rmse"] ** 2
    mse_pub = want["rmse"] ** 2
    var_mean = est["pure_sample_variance"] / W
    sigma_mse = np.sqrt(2.0) * np.sqrt(2.0 * np.sum(var_mean ** 2)) / len(var_mean)
    assert abs(mse - mse_pub) <= 4 * sigma_mse, (got["rmse"], want["rmse"], sigma_mse)
    # this run's own MSE is its estimator variance (no measurable bias)
    assert abs(mse - var_mean.mean()) <= 4 * np.sqrt(2.0 * np.sum(var_mean ** 2)) / len(var_mean) + 1e-6
