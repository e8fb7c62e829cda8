"""The oracle_2lmc sweep and its multi-seed aggregation
(n2w.wavefront_oracle_sweep, the reference's run_wavefront_oracle_sweep.py /
run_wavefront_oracle_multiseed.py form): statistics against hand-computed
values with a stand-in executable on the CPU, and a small multi-seed sweep
through the real n2wos_eval_wavefront_wos on the GPU whose bias z-scores
stay within the reference's 3-sigma band."""
from __future__ import annotations

import csv
import json
import math
import stat
import sys
import textwrap

import pytest

from n2w import wavefront_oracle_sweep as ws

FAKE = textwrap.dedent(f"""\
    #!{sys.executable}
    # Stand-in for n2wos_eval_wavefront_wos: numbers are simple functions of
    # the flags (method, samples, depth, seed).
    import argparse, json
    ap = argparse.ArgumentParser()
    ap.add_argument("--method"); ap.add_argument("--output"); ap.add_argument("--engine")
    for f in ("--samples", "--coarse-samples", "--residual-samples", "--depth-m", "--seed"):
        ap.add_argument(f, type=int, default=0)
    a, _ = ap.parse_known_args()
    exact = 0.25
    shift = 0.001 * ((a.seed % 3) - 1)
    if a.method == "pure_wos":
        v = 1.0 / a.samples
        est = dict(method="pure_wos", engine=a.engine, mean=exact + shift, exact=exact, abs_error=abs(shift),
                   stderr=v ** 0.5, estimator_variance=v, elapsed_ms_total=0.01 * a.samples)
        runs = {{"pure_wos": dict(samples=a.samples, mean=exact + shift, forced_max_steps=1, overflow_count=0)}}
    else:
        vc, vr = 0.5 / a.depth_m, 0.1 * a.depth_m
        cc, cr = 1.0 * a.depth_m, 10.0  # us per sample
        c = dict(samples=a.coarse_samples, mean=exact + shift, sample_variance=vc, estimator_variance=vc / a.coarse_samples,
                 stderr=(vc / a.coarse_samples) ** 0.5, elapsed_ms=cc * a.coarse_samples / 1000, us_per_sample=cc,
                 mean_steps=a.depth_m, forced_max_steps=0, overflow_count=2)
        r = dict(samples=a.residual_samples, mean=-0.5 * shift, sample_variance=vr,
                 estimator_variance=vr / a.residual_samples, stderr=(vr / a.residual_samples) ** 0.5,
                 elapsed_ms=cr * a.residual_samples / 1000, us_per_sample=cr, mean_steps=20, forced_max_steps=3,
                 overflow_count=0)
        var = c["estimator_variance"] + r["estimator_variance"]
        m = c["mean"] + r["mean"]
        est = dict(method="oracle_2lmc", engine=a.engine, mean=m, exact=exact, abs_error=abs(m - exact),
                   stderr=var ** 0.5, estimator_variance=var, elapsed_ms_total=c["elapsed_ms"] + r["elapsed_ms"])
        runs = {{"coarse": c, "residual": r}}
    doc = dict(estimator=est, runs=runs, options=dict(method=a.method, engine=a.engine, depth_m=a.depth_m,
               samples=a.samples, coarse_samples=a.coarse_samples, residual_samples=a.residual_samples))
    open(a.output, "w").write(json.dumps(doc))
    """)


@pytest.fixture()
def fake_exe(tmp_path):
    exe = tmp_path / "fake_wavefront"
    exe.write_text(FAKE)
    exe.chmod(exe.stat().st_mode | stat.S_IXUSR)
    return exe


def read_csv(path):
    with open(path, newline="") as f:
        return list(csv.DictReader(f))


def test_sweep_statistics(fake_exe, tmp_path):
    out = tmp_path / "sweep"
    assert ws.main(["--executable", str(fake_exe), "--output-dir", str(out), "--pure-samples", "10000",
                    "--residual-samples", "1000", "--coarse-ratios", "1,4", "--depths", "2", "--seed", "12346"]) == 0
    rows = {r["label"]: r for r in read_csv(out / "summary.csv")}
    assert list(rows) == ["pure_wos", "oracle_2lmc_m2_r1", "oracle_2lmc_m2_r4"]
    pure_vt = (1.0 / 10000) * (0.01 * 10000)
    assert float(rows["pure_wos"]["variance_time_product_ms"]) == pytest.approx(pure_vt)
    assert float(rows["pure_wos"]["score_speedup_vs_pure"]) == pytest.approx(1.0)
    assert int(rows["pure_wos"]["forced_max_steps_total"]) == 1
    r = rows["oracle_2lmc_m2_r4"]
    nc, nr, vc, vr, cc, cr = 4000, 1000, 0.25, 0.2, 2.0, 10.0
    var = vc / nc + vr / nr
    vt = var * (cc * nc + cr * nr) / 1000
    assert float(r["variance_time_product_ms"]) == pytest.approx(vt)
    assert float(r["score_speedup_vs_pure"]) == pytest.approx(pure_vt / vt)
    assert float(r["optimal_coarse_to_residual_sample_ratio"]) == pytest.approx(math.sqrt(vc * cr / (vr * cc)))
    best = (math.sqrt(vc * cc * 1e-3) + math.sqrt(vr * cr * 1e-3)) ** 2
    assert float(r["optimal_variance_time_product_ms_predicted"]) == pytest.approx(best)
    assert float(r["measured_coarse_to_residual_sample_ratio"]) == pytest.approx(4.0)
    assert float(r["residual_variance_ratio_vs_coarse"]) == pytest.approx(vr / vc)
    # seed 12346: shift = 0 -> exact estimate
    assert float(r["z_abs_error"]) == 0.0 and r["diagnostic_flag_large_estimator_z"] == "False"
    assert int(r["forced_max_steps_total"]) == 3 and int(r["overflow_count_total"]) == 2
    lab = read_csv(out / "summary_by_label.csv")
    assert [x["label"] for x in lab] == list(rows) and all(x["seed_count"] == "1" for x in lab)
    doc = json.loads((out / "summary.json").read_text())
    assert doc["schema"] == "n2wos_wavefront_oracle_sweep_v1" and doc["seeds"] == [12346]
    assert len(doc["records"]) == 3


def test_sweep_commands_and_seeds(fake_exe, tmp_path, capsys):
    ws.main(["--executable", str(fake_exe), "--output-dir", str(tmp_path / "d"), "--dry-run", "--seed-count", "2",
             "--depths", "1,4", "--coarse-ratios", "2", "--residual-samples", "333"])
    lines = [ln for ln in capsys.readouterr().out.splitlines() if ln.startswith("+ ")]
    assert len(lines) == 2 * (1 + 2)
    first = lines[0].split()
    assert first[2:4] == ["--method", "pure_wos"] and "--seed" in first and first[first.index("--seed") + 1] == "12345"
    assert lines[3].split()[lines[3].split().index("--seed") + 1] == str(12345 + 1000003)
    lmc = lines[1].split()
    assert lmc[lmc.index("--coarse-samples") + 1] == "666" and lmc[lmc.index("--depth-m") + 1] == "1"
    assert lmc[lmc.index("--bumpy-stacks") + 1] == "128" and lmc[lmc.index("--engine") + 1] == "wavefront"


def test_multiseed_aggregate(fake_exe, tmp_path):
    out = tmp_path / "multi"
    seeds = [3, 4, 5]  # shifts +0.001, -0.001... (seed % 3 - 1): -1, 0, +1 thousandths
    assert ws.multiseed_main(["--executable", str(fake_exe), "--output-dir", str(out), "--seeds", "3,4,5",
                              "--pure-samples", "10000", "--residual-samples", "1000", "--coarse-ratios", "2",
                              "--depths", "1"]) == 0
    agg = {r["label"]: r for r in read_csv(out / "summary_aggregate.csv")}
    assert set(agg) == {"pure_wos", "oracle_2lmc_m1_r2"}
    p = agg["pure_wos"]
    assert int(p["num_seeds"]) == 3
    assert float(p["mean_estimate_across_seeds"]) == pytest.approx(0.25)
    assert float(p["pooled_stderr_of_seed_mean"]) == pytest.approx(math.sqrt(3 * 1e-4) / 3)
    assert float(p["rmse_of_seed_estimates"]) == pytest.approx(math.sqrt(2e-6 / 3))
    assert int(p["forced_max_steps_total_sum"]) == 3
    by_seed = read_csv(out / "summary_by_seed.csv")
    assert sorted({int(r["seed"]) for r in by_seed}) == seeds
    man = json.loads((out / "summary_aggregate.json").read_text())
    assert man["schema"] == "n2wos_wavefront_oracle_multiseed_v1"
    assert man["best_actual_oracle_2lmc"]["label"] == "oracle_2lmc_m1_r2"
    assert len(man["seed_runs"]) == 3


@pytest.mark.gpu
def test_multiseed_with_the_real_executable(gpu, tmp_path):
    """Five seeds, pure WoS and the exact-cache 2LMC at two depths, at x0 on
    the bumpy sphere (u = x^2 - y^2): every label's seed-mean bias stays within
    4 pooled standard errors, and the residual level is centred on zero."""
    out = tmp_path / "real"
    assert ws.multiseed_main(["--output-dir", str(out), "--pure-samples", "65536", "--residual-samples", "8192",
                              "--coarse-ratios", "2", "--depths", "1,4", "--bumpy-stacks", "64",
                              "--bumpy-slices", "128", "--epsilon", "1e-3"]) == 0
    agg = {r["label"]: r for r in read_csv(out / "summary_aggregate.csv")}
    assert set(agg) == {"pure_wos", "oracle_2lmc_m1_r2", "oracle_2lmc_m4_r2"}
    for label, r in agg.items():
        assert int(r["num_seeds"]) == 5
        assert abs(float(r["bias_z_score"])) < 4.0, (label, r["bias_z_score"])
        assert int(r["overflow_count_total_sum"]) == 0
    rows = read_csv(out / "summary_by_seed.csv")
    lmc = [r for r in rows if r["label"].startswith("oracle_2lmc")]
    assert len(lmc) == 10
    # |z| of the residual mean above 3 in at most one of ten runs
    assert sum(float(r["residual_z_abs_mean"]) > 3 for r in lmc) <= 1
    assert all(float(r["optimal_coarse_to_residual_sample_ratio"]) > 0 for r in lmc)
