"""The reference-based slice time-to-MSE runner
(n2w.slice_reference_time_to_mse, the reference's
run_nc_slice_reference_time_to_mse.py form): the chunked reference merged by
Chan's pairwise update equals the statistics of all its walks pooled, errors
and thresholds against a stand-in executable on the CPU, and one small run
through the real n2wos_eval_tcnn_nc_wos on the GPU."""
from __future__ import annotations

import csv
import json
import math
import stat
import sys
import textwrap

import numpy as np
import pytest

from n2w import slice_reference_time_to_mse as srt

# per-walk values of the stand-in executable's pure runs (pixels x walks);
# shared verbatim by the stand-in and the test
SAMPLES_SRC = textwrap.dedent("""\
    PIXELS = 50


    def samples(seed, walks):
        rng = np.random.default_rng(seed)
        mu = np.linspace(-1.0, 1.0, PIXELS)[:, None]
        return mu + rng.normal(0.0, 0.5, (PIXELS, walks))
    """)
exec(SAMPLES_SRC)


FAKE = textwrap.dedent(f"""\
    #!{sys.executable}
    import argparse, json
    import numpy as np
    {{SAMPLES}}
    ap = argparse.ArgumentParser()
    ap.add_argument("--output"); ap.add_argument("--save-estimates-prefix")
    for f in ("--pure-walks-per-point", "--hybrid-walks-per-point", "--enable-2lmc", "--coarse-walks-per-point",
              "--residual-walks-per-point", "--seed", "--train-steps-per-refresh", "--skip-training"):
        ap.add_argument(f, type=int, default=0)
    a, _ = ap.parse_known_args()
    s = samples(a.seed, a.pure_walks_per_point)
    mu = np.linspace(-1.0, 1.0, PIXELS)
    pure_var = s.var(1, ddof=1) if s.shape[1] > 1 else np.zeros(PIXELS)
    nc = mu + 0.2 + 0.0 * a.hybrid_walks_per_point  # a biased NC-only estimate
    lmc = mu + 0.2 / (a.coarse_walks_per_point * a.residual_walks_per_point)
    with open(a.save_estimates_prefix + "_estimates.csv", "w") as f:
        f.write("point_id,x,y,z,analytic_value,pure_mean,pure_sample_variance,nc_wos_mean,nc_2lmc_mean\\n")
        for i in range(PIXELS):
            f.write(f"{{i}},{{i}},0,0,{{float(mu[i])!r}},{{float(s[i].mean())!r}},{{float(pure_var[i])!r}},{{float(nc[i])!r}},{{float(lmc[i])!r}}\\n")
    train = 0.0 if a.skip_training else 500.0
    runs = {{"pure_wos": {{"elapsed_ms": 0.1 * a.pure_walks_per_point}},
            "nc_wos": {{"elapsed_ms": 1.0 * a.hybrid_walks_per_point}},
            "nc_2lmc": {{"elapsed_ms": 0.2 * a.coarse_walks_per_point + 1.0 * a.residual_walks_per_point}}}}
    open(a.output, "w").write(json.dumps({{"runs": runs, "training": {{"total_training_ms": train}}}}))
    """)
FAKE = FAKE.replace("{SAMPLES}", SAMPLES_SRC)


@pytest.fixture()
def fake_exe(tmp_path):
    exe = tmp_path / "fake_eval"
    exe.write_text(FAKE)
    exe.chmod(exe.stat().st_mode | stat.S_IXUSR)
    return exe


def read_csv(path):
    with open(path, newline="") as f:
        return list(csv.DictReader(f))


def test_chunked_reference_equals_pooled_walks(fake_exe, tmp_path):
    out = tmp_path / "ref"
    assert srt.main(["--executable", str(fake_exe), "--output-dir", str(out), "--reference-wpp", "1000",
                     "--reference-chunk-wpp", "300", "--pure-wpp-list", "4,64", "--nc-hybrid-wpp-list", "2",
                     "--lmc-allocations", "1:1,4:4", "--threshold-rmse-list", "0.15,0.5"]) == 0
    summary = json.loads((out / "summary_reference.json").read_text())
    chunks = summary["reference"]["reference_chunks"]
    assert [c.rsplit("_wpp", 1)[1] for c in chunks] == ["300_estimates.csv"] * 3 + ["100_estimates.csv"]
    # the same walks, pooled
    seeds = [987654321 + 100003 * k for k in range(4)]
    pooled = np.concatenate([samples(sd, w) for sd, w in zip(seeds, (300, 300, 300, 100))], axis=1)
    ref = read_csv(out / "estimates" / "reference_pure_estimates.csv")
    got_mean = np.array([float(r["pure_mean"]) for r in ref])
    got_var = np.array([float(r["pure_sample_variance"]) for r in ref])
    np.testing.assert_allclose(got_mean, pooled.mean(1), rtol=0, atol=1e-12)
    np.testing.assert_allclose(got_var, pooled.var(1, ddof=1), rtol=1e-10)
    assert all(r["reference_wpp"] == "1000" for r in ref)
    assert summary["reference"]["reference_rmse_floor_estimate"] == pytest.approx(
        math.sqrt(pooled.var(1, ddof=1).mean() / 1000))

    pts = {p["label"]: p for p in read_csv(out / "time_mse_points_reference.csv")}
    assert list(pts) == ["pure_wpp4", "pure_wpp64", "nc_wpp2", "nc2lmc_c1_r1", "nc2lmc_c4_r4"]
    s4 = samples(12345 + 1000 + 4, 4).mean(1)
    e = s4 - pooled.mean(1)
    assert float(pts["pure_wpp4"]["mse_vs_reference"]) == pytest.approx(np.mean(e * e))
    assert float(pts["pure_wpp4"]["mean_error_vs_reference"]) == pytest.approx(e.mean())
    assert float(pts["pure_wpp4"]["default_time_ms"]) == pytest.approx(0.4)  # solve only
    assert float(pts["nc_wpp2"]["default_time_ms"]) == pytest.approx(502.0)  # training included
    assert float(pts["nc_wpp2"]["training_plus_solve_ms"]) == pytest.approx(502.0)
    thr = {(float(r["threshold_rmse"]), r["method"], r["time_mode"]): r
           for r in read_csv(out / "time_to_threshold_reference.csv")}
    assert len(thr) == 2 * 3 * 2
    assert thr[(0.15, "nc_2lmc", "solve_only_ms")]["best_label"] == "nc2lmc_c4_r4"
    assert thr[(0.15, "nc_wos", "solve_only_ms")]["hit"] == "False"  # its bias is 0.2
    assert thr[(0.5, "pure_wos", "solve_only_ms")]["best_label"] == "pure_wpp4"


def test_merge_rejects_bad_chunks(tmp_path):
    p = tmp_path / "c_estimates.csv"
    p.write_text("point_id,pure_mean,pure_sample_variance\n0,1.0,-0.5\n")
    with pytest.raises(RuntimeError, match="negative reference chunk variance"):
        srt.merge_chunks([p], [10], tmp_path / "out.csv")
    q = tmp_path / "d_estimates.csv"
    q.write_text("point_id,pure_mean,pure_sample_variance\n0,1.0,0.5\n1,2.0,0.5\n")
    with pytest.raises(RuntimeError, match="row count mismatch"):
        srt.merge_chunks([q, p], [10, 10], tmp_path / "out.csv")
    with pytest.raises(RuntimeError, match="count mismatch"):
        srt.merge_chunks([q], [10, 10], tmp_path / "out.csv")


def test_dry_run_manifest(fake_exe, tmp_path):
    out = tmp_path / "dry"
    assert srt.main(["--executable", str(fake_exe), "--output-dir", str(out), "--dry-run",
                     "--reference-wpp", "1024", "--reference-chunk-wpp", "512"]) == 0
    man = json.loads((out / "manifest.json").read_text())
    assert man["dry_run"] and len(man["reference_commands"]) == 2 and len(man["commands"]) == 5 + 5 + 4
    cmd = man["reference_commands"][1]["command"]
    assert cmd[cmd.index("--seed") + 1] == str(987654321 + 100003)
    assert cmd[cmd.index("--skip-training") + 1] == "1"
    nc = man["commands"][7]["command"]  # nc_wpp4
    assert nc[nc.index("--seed") + 1] == str(12345 + 2000 + 4)
    assert nc[nc.index("--train-sampler") + 1] == "rejection"


@pytest.mark.gpu
def test_small_run_with_the_real_executable(gpu, tmp_path):
    out = tmp_path / "real"
    assert srt.main(["--output-dir", str(out), "--slice-width", "40", "--slice-height", "40",
                     "--bumpy-stacks", "32", "--bumpy-slices", "64", "--epsilon", "1e-3",
                     "--boundary", "harmonic_x2_minus_y2", "--reference-wpp", "1024", "--reference-chunk-wpp", "256",
                     "--pure-wpp-list", "4,64", "--nc-hybrid-wpp-list", "2", "--lmc-allocations", "8:4",
                     "--train-points", "2048", "--label-refreshes", "1", "--walks-per-label-refresh", "4",
                     "--train-steps-per-refresh", "20", "--threshold-rmse-list", "10,1e-7"]) == 0
    ref = read_csv(out / "estimates" / "reference_pure_estimates.csv")
    assert len(ref) > 0 and all(r["reference_wpp"] == "1024" for r in ref)
    # the merged Monte Carlo reference agrees with the analytic solution
    err = np.array([float(r["pure_mean"]) - float(r["analytic_value"]) for r in ref])
    se = np.sqrt(np.array([float(r["pure_sample_variance"]) for r in ref]) / 1024)
    assert abs(err.mean()) < 4 * np.sqrt(np.sum(se ** 2)) / len(se) + 1e-6
    pts = {p["label"]: p for p in read_csv(out / "time_mse_points_reference.csv")}
    assert float(pts["pure_wpp64"]["rmse_vs_reference"]) < 0.5 * float(pts["pure_wpp4"]["rmse_vs_reference"])
    summary = json.loads((out / "summary_reference.json").read_text())
    floor = summary["reference"]["reference_rmse_floor_estimate"]
    assert 0 < floor < float(pts["pure_wpp64"]["rmse_vs_reference"])
