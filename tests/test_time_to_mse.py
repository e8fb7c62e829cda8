"""The time-to-MSE runner (n2w.time_to_mse, the reference's
scripts/run_nc_slice_time_to_mse.py form): command lines, accounting and
thresholds against a stand-in executable on the CPU, and one small sweep
through the real n2wos_eval_tcnn_nc_wos on the GPU."""
from __future__ import annotations

import csv
import json
import math
import stat
import sys
import textwrap

import pytest

from n2w import time_to_mse as ttm

FAKE = textwrap.dedent(f"""\
    #!{sys.executable}
    # Stand-in for n2wos_eval_tcnn_nc_wos: reads the flags the runner passes
    # and writes a result JSON whose numbers are simple functions of them.
    import argparse, json, sys
    ap = argparse.ArgumentParser()
    for f in ("--output", "--boundary", "--cache-preset"):
        ap.add_argument(f)
    for f in ("--pure-walks-per-point", "--hybrid-walks-per-point", "--enable-2lmc", "--coarse-walks-per-point",
              "--residual-walks-per-point", "--train-points", "--label-refreshes", "--train-steps-per-refresh",
              "--walks-per-label-refresh"):
        ap.add_argument(f, type=int)
    a, _ = ap.parse_known_args()
    if a.hybrid_walks_per_point == 3:
        sys.exit(7)  # a failing run
    train = 100.0 * a.label_refreshes * a.train_steps_per_refresh + a.train_points / 100.0
    p, h, c, r = a.pure_walks_per_point, a.hybrid_walks_per_point, a.coarse_walks_per_point, a.residual_walks_per_point
    runs = {{"pure_wos": {{"rmse": 0.8 / p ** 0.5, "elapsed_ms": 2.0 * p, "mean_sample_variance": 0.64,
                          "mean_bias": 0.0, "eval_points": 1000, "training_plus_elapsed_ms": train + 2.0 * p}},
            "nc_wos": {{"rmse": 0.12 + 0.3 / h ** 0.5, "elapsed_ms": 0.5 * h, "mean_sample_variance": 0.09,
                        "eval_points": 1000, "training_plus_elapsed_ms": train + 0.5 * h}}}}
    if a.enable_2lmc:
        runs["nc_2lmc_m4"] = {{"rmse": (0.04 / c + 0.16 / r) ** 0.5, "elapsed_ms": 0.5 * c + 2.0 * r,
                              "mean_coarse_sample_variance": 0.04, "mean_residual_sample_variance": 0.16,
                              "eval_points": 1000, "training_plus_elapsed_ms": train + 0.5 * c + 2.0 * r}}
    out = {{"options": {{"train_points_padded": a.train_points}}, "runs": runs,
            "training": {{"total_training_ms": train, "label_update_ms": train / 4, "tcnn_training_ms": train * 3 / 4}},
            "slice_eval": {{"inside_pixels": 1000}}}}
    open(a.output, "w").write(json.dumps(out))
    """)


@pytest.fixture()
def fake_exe(tmp_path):
    exe = tmp_path / "fake_eval"
    exe.write_text(FAKE)
    exe.chmod(exe.stat().st_mode | stat.S_IXUSR)
    return exe


def read_csv(path):
    with open(path, newline="") as f:
        return list(csv.DictReader(f))


def test_commands_accounting_and_thresholds(fake_exe, tmp_path):
    out = tmp_path / "ttm"
    rc = ttm.main(["--executable", str(fake_exe), "--output-dir", str(out), "--pure-wpp-list", "4,16,64",
                   "--nc-hybrid-wpp-list", "1,4", "--lmc-allocations", "16:8,64:32", "--train-points", "3000",
                   "--label-refreshes", "2", "--train-steps-per-refresh", "10",
                   "--threshold-rmse-list", "0.25,0.15,0.01"])
    assert rc == 0
    man = json.loads((out / "manifest.json").read_text())
    cmds = {c["label"]: c["command"] for c in man["commands"]}
    assert list(cmds) == ["pure_wpp4", "pure_wpp16", "pure_wpp64", "nc_wpp1", "nc_wpp4", "nc2lmc_c16_r8",
                          "nc2lmc_c64_r32"]

    def flag(cmd, name):
        return cmd[cmd.index(name) + 1]

    # pure runs train a throw-away cache; NC runs the requested schedule
    assert flag(cmds["pure_wpp16"], "--train-points") == "512"
    assert flag(cmds["pure_wpp16"], "--label-refreshes") == "1"
    assert flag(cmds["pure_wpp16"], "--train-steps-per-refresh") == "0"
    assert flag(cmds["nc_wpp4"], "--train-points") == "3000"
    assert flag(cmds["nc_wpp4"], "--pure-walks-per-point") == "64"  # the largest pure budget
    assert flag(cmds["nc2lmc_c64_r32"], "--hybrid-walks-per-point") == "1"  # the smallest hybrid budget
    assert flag(cmds["nc2lmc_c64_r32"], "--enable-2lmc") == "1"
    assert flag(cmds["nc_wpp1"], "--eval-mode") == "slice"
    assert flag(cmds["nc_wpp1"], "--bumpy-stacks") == "128"

    rows = read_csv(out / "time_mse_points.csv")
    assert [r["label"] for r in rows] == list(cmds)
    assert list(rows[0]) == ttm.POINT_COLUMNS
    by = {r["label"]: r for r in rows}
    train = 100.0 * 2 * 10 + 3000 / 100.0
    # pure: every time mode is the solve alone
    p = by["pure_wpp16"]
    assert float(p["solve_only_ms"]) == float(p["end_to_end_ms"]) == float(p["single_snapshot_total_ms"]) == 32.0
    assert float(p["training_ms"]) == 0.0 and p["cache_preset"] == "" and p["depth_m"] == ""
    # NC: end to end from the run, single snapshot = median NC training + solve
    n = by["nc_wpp4"]
    assert float(n["training_ms"]) == train and float(n["end_to_end_ms"]) == train + 2.0
    assert float(n["single_snapshot_total_ms"]) == train + 2.0
    summary = json.loads((out / "summary.json").read_text())
    assert summary["representative_training_ms_for_single_snapshot_total"] == train
    # 2LMC: residual variance over the largest pure run's variance
    assert math.isclose(float(by["nc2lmc_c16_r8"]["residual_variance_ratio_vs_pure"]), 0.16 / 0.64)
    assert float(by["nc2lmc_c16_r8"]["mse"]) == pytest.approx(0.04 / 16 + 0.16 / 8)

    thr = read_csv(out / "time_to_threshold.csv")
    assert len(thr) == 3 * 3 * 3

    def pick(t, m, mode):
        return next(r for r in thr if float(r["threshold_rmse"]) == t and r["method"] == m and r["time_mode"] == mode)

    # pure: rmse 0.4 / 0.2 / 0.1 -> fastest under 0.25 is wpp16
    assert pick(0.25, "pure_wos", "solve_only_ms")["best_label"] == "pure_wpp16"
    assert pick(0.15, "pure_wos", "end_to_end_ms")["best_label"] == "pure_wpp64"
    # NC-only: 0.12 + 0.3 / sqrt(h), never under 0.25 for h <= 4
    assert pick(0.25, "nc_wos", "solve_only_ms")["hit"] == "False"
    assert pick(0.25, "nc_2lmc", "solve_only_ms")["best_label"] == "nc2lmc_c16_r8"
    assert all(r["hit"] == "False" for r in thr if float(r["threshold_rmse"]) == 0.01)


def test_dry_run_and_failed_runs(fake_exe, tmp_path):
    out = tmp_path / "dry"
    assert ttm.main(["--executable", str(fake_exe), "--output-dir", str(out), "--dry-run"]) == 0
    man = json.loads((out / "manifest.json").read_text())
    assert len(man["commands"]) == 5 + 5 + 4 and not (out / "runs" / "pure_wpp8.json").exists()
    assert read_csv(out / "time_mse_points.csv") == []
    # a run that fails stops the sweep, unless --continue-on-error records it
    args = ["--executable", str(fake_exe), "--pure-wpp-list", "4", "--nc-hybrid-wpp-list", "2,3",
            "--lmc-allocations", "4:2"]
    with pytest.raises(SystemExit) as e:
        ttm.main(args + ["--output-dir", str(tmp_path / "stop")])
    assert e.value.code == 7
    assert ttm.main(args + ["--output-dir", str(tmp_path / "go"), "--continue-on-error"]) == 0
    man = json.loads((tmp_path / "go" / "manifest.json").read_text())
    assert man["errors"] == [{"label": "nc_wpp3", "returncode": 7}]
    assert [r["label"] for r in read_csv(tmp_path / "go" / "time_mse_points.csv")] == \
        ["pure_wpp4", "nc_wpp2", "nc2lmc_c4_r2"]
    # --skip-existing reuses the JSON of earlier runs
    assert ttm.main(args + ["--output-dir", str(tmp_path / "go"), "--continue-on-error", "--skip-existing"]) == 0


def test_allocation_parsing():
    assert ttm._allocations("16:8, 32:16,") == [(16, 8), (32, 16)]
    with pytest.raises(ValueError):
        ttm._allocations("16")


@pytest.mark.gpu
def test_small_sweep_with_the_real_executable(gpu, tmp_path):
    out = tmp_path / "real"
    rc = ttm.main(["--output-dir", str(out), "--slice-width", "48", "--slice-height", "48",
                   "--bumpy-stacks", "32", "--bumpy-slices", "64", "--epsilon", "1e-3",
                   "--pure-wpp-list", "4,64", "--nc-hybrid-wpp-list", "2", "--lmc-allocations", "8:4",
                   "--train-points", "2048", "--label-refreshes", "1", "--walks-per-label-refresh", "4",
                   "--train-steps-per-refresh", "20", "--threshold-rmse-list", "10.0,1e-7"])
    assert rc == 0
    rows = {r["label"]: r for r in read_csv(out / "time_mse_points.csv")}
    assert set(rows) == {"pure_wpp4", "pure_wpp64", "nc_wpp2", "nc2lmc_c8_r4"}
    for r in rows.values():
        assert math.isfinite(float(r["rmse"])) and float(r["solve_only_ms"]) > 0
        assert int(r["eval_points"]) > 0
    # sixteen times the walks: about a quarter of the RMSE
    assert float(rows["pure_wpp64"]["rmse"]) < 0.5 * float(rows["pure_wpp4"]["rmse"])
    assert float(rows["nc_wpp2"]["training_ms"]) > 0
    thr = read_csv(out / "time_to_threshold.csv")
    assert all(r["hit"] == "True" for r in thr if float(r["threshold_rmse"]) == 10.0 and r["method"] == "pure_wos")
    assert all(r["hit"] == "False" for r in thr if float(r["threshold_rmse"]) == 1e-7)
