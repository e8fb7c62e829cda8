"""Fixed-slice time-to-MSE sweep: pure WoS, NC-only and NC+2LMC budget curves
around the ``n2wos_eval_tcnn_nc_wos`` executable.

Drop-in for the reference's runner ``scripts/run_nc_slice_time_to_mse.py``:
the same command-line flags and defaults (213-300), the same per-run command
lines handed to the executable (add_common_args, 100-138), the same output
files (``time_mse_points.csv``, ``time_to_threshold.csv``, ``summary.json``,
``manifest.json``) with the same columns, and the same accounting rules:

* ``solve_only_ms``  -- the run's ``elapsed_ms`` (evaluation with a trained
  snapshot);
* ``end_to_end_ms``  -- ``training_plus_elapsed_ms`` of that run (its own
  training + solve); for pure WoS the solve alone;
* ``single_snapshot_total_ms`` -- the median training time of the NC runs plus
  this run's solve (training once, reusing the snapshot for every budget);
* time to a threshold RMSE r, per method and time mode: the fastest run with
  MSE <= r^2 (compute_thresholds, 213-247).

Pure-WoS budget points are run with a throw-away cache (the executable always
trains one): 512 training points, one refresh of one walk, no training steps
(flags ``--pure-probe-train-points``), as the reference does.

    python -m n2w.time_to_mse --output-dir out/ttm [--executable BIN] [reference flags ...]
"""
from __future__ import annotations

import argparse
import csv
import json
import math
import statistics
import subprocess
import sys
from dataclasses import dataclass, field
from pathlib import Path
from typing import Any, Dict, List, Optional, Sequence

DEFAULT_EXECUTABLE = Path(__file__).resolve().parent.parent / "bin" / "n2wos_eval_tcnn_nc_wos"

POINT_COLUMNS = [
    "method", "label", "json_path", "cache_preset", "boundary_condition", "depth_m",
    "train_points_requested", "train_points_padded", "total_train_steps",
    "pure_walks_per_point", "hybrid_walks_per_point", "coarse_walks_per_point", "residual_walks_per_point",
    "slice_width", "slice_height", "slice_view", "slice_plane", "eval_points", "inside_pixels",
    "rmse", "mse", "mean_bias", "mean_sample_variance", "mean_coarse_sample_variance",
    "mean_residual_sample_variance", "residual_variance_ratio_vs_pure",
    "solve_only_ms", "training_ms", "single_snapshot_total_ms", "end_to_end_ms",
    "label_update_ms", "tcnn_training_ms",
]
THRESHOLD_COLUMNS = ["threshold_rmse", "threshold_mse", "method", "time_mode", "hit", "best_time_ms",
                     "best_label", "best_rmse"]
TIME_MODES = ("solve_only_ms", "single_snapshot_total_ms", "end_to_end_ms")
NAN = float("nan")


def _ints(text: str) -> List[int]:
    return [int(t) for t in str(text).split(",") if t.strip()]


def _floats(text: str) -> List[float]:
    return [float(t) for t in str(text).split(",") if t.strip()]


def _allocations(text: str) -> List[tuple]:
    out = []
    for t in str(text).split(","):
        t = t.strip()
        if not t:
            continue
        c, sep, r = t.partition(":")
        if not sep:
            raise ValueError(f"allocation must be coarse:residual, got {t!r}")
        out.append((int(c), int(r)))
    return out


def _num(v: Any, default: float = NAN) -> float:
    """Float of a JSON field; `default` when absent, null or not numeric."""
    if v is None or v == "":
        return default
    try:
        return float(v)
    except (TypeError, ValueError):
        return default


def parser() -> argparse.ArgumentParser:
    """The reference runner's flags, names and defaults unchanged."""
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0],
                                 formatter_class=argparse.ArgumentDefaultsHelpFormatter)
    ap.add_argument("--executable", default=str(DEFAULT_EXECUTABLE))
    ap.add_argument("--output-dir", required=True)
    ap.add_argument("--mesh", default="procedural_bumpy_sphere")
    ap.add_argument("--mesh-path", default="")
    ap.add_argument("--normalize", type=int, default=1)
    ap.add_argument("--bumpy-stacks", type=int, default=128)
    ap.add_argument("--bumpy-slices", type=int, default=256)
    ap.add_argument("--bumpy-amplitude", type=float, default=0.15)
    ap.add_argument("--boundary", default="external_charges_medium")
    ap.add_argument("--label-source", default="wos_supervision")
    ap.add_argument("--cache-preset", default="nano")
    ap.add_argument("--train-points", type=int, default=20000)
    ap.add_argument("--label-refreshes", type=int, default=4)
    ap.add_argument("--walks-per-label-refresh", type=int, default=50)
    ap.add_argument("--train-steps-per-refresh", type=int, default=5000)
    ap.add_argument("--depth-m", type=int, default=4)
    ap.add_argument("--slice-width", type=int, default=512)
    ap.add_argument("--slice-height", type=int, default=512)
    ap.add_argument("--slice-view", default="xy", choices=["xy", "xz", "yz"])
    ap.add_argument("--slice-plane", type=float, default=0.0)
    ap.add_argument("--slice-frame", default="")
    ap.add_argument("--slice-padding-fraction", type=float, default=0.02)
    ap.add_argument("--slice-preserve-world-aspect", type=int, default=1)
    ap.add_argument("--pure-wpp-list", default="8,16,32,64,128")
    ap.add_argument("--nc-hybrid-wpp-list", default="1,2,4,8,16")
    ap.add_argument("--lmc-allocations", default="16:8,32:16,32:32,64:32")
    ap.add_argument("--pure-probe-train-points", type=int, default=512,
                    help="training points of the throw-away cache of pure-WoS runs")
    ap.add_argument("--max-steps", type=int, default=256)
    ap.add_argument("--epsilon", default="1e-4")
    ap.add_argument("--seed", type=int, default=12345)
    ap.add_argument("--cubql-build-method", default="sah")
    ap.add_argument("--cubql-leaf-size", type=int, default=8)
    ap.add_argument("--jit", type=int, default=0)
    ap.add_argument("--threshold-rmse-list", default="0.05,0.06,0.075,0.1")
    ap.add_argument("--run-pure", type=int, default=1)
    ap.add_argument("--run-nc", type=int, default=1)
    ap.add_argument("--run-2lmc", type=int, default=1)
    ap.add_argument("--dry-run", action="store_true")
    ap.add_argument("--skip-existing", action="store_true")
    ap.add_argument("--continue-on-error", action="store_true")
    return ap


@dataclass
class RunPlan:
    """One invocation of the executable: its label, method, walk budget flags
    and the training settings it runs with."""
    label: str
    method: str  # pure_wos | nc_wos | nc_2lmc
    budget: Dict[str, int]
    training: Dict[str, int]
    walks: Dict[str, Optional[int]] = field(default_factory=dict)


def plan_runs(a: argparse.Namespace) -> List[RunPlan]:
    pure, hybrid, allocs = _ints(a.pure_wpp_list), _ints(a.nc_hybrid_wpp_list), _allocations(a.lmc_allocations)
    trained = {"train_points": a.train_points, "label_refreshes": a.label_refreshes,
               "walks_per_label_refresh": a.walks_per_label_refresh,
               "train_steps_per_refresh": a.train_steps_per_refresh}
    probe = {"train_points": a.pure_probe_train_points, "label_refreshes": 1, "walks_per_label_refresh": 1,
             "train_steps_per_refresh": 0}
    widest_pure = max(pure) if pure else 64
    plans: List[RunPlan] = []
    if a.run_pure:
        for w in pure:
            plans.append(RunPlan(f"pure_wpp{w}", "pure_wos",
                                 {"pure": w, "hybrid": 1, "lmc": 0, "coarse": 1, "residual": 1}, probe,
                                 {"pure": w}))
    if a.run_nc:
        for w in hybrid:
            plans.append(RunPlan(f"nc_wpp{w}", "nc_wos",
                                 {"pure": widest_pure, "hybrid": w, "lmc": 0, "coarse": 1, "residual": 1}, trained,
                                 {"hybrid": w}))
    if a.run_2lmc:
        for c, r in allocs:
            plans.append(RunPlan(f"nc2lmc_c{c}_r{r}", "nc_2lmc",
                                 {"pure": widest_pure, "hybrid": min(hybrid) if hybrid else 4, "lmc": 1,
                                  "coarse": c, "residual": r}, trained,
                                 {"coarse": c, "residual": r}))
    return plans


def command(a: argparse.Namespace, plan: RunPlan, output: Path) -> List[str]:
    """Command line of one run (the reference's flag order)."""
    t = plan.training
    cmd = [a.executable, "--mesh", a.mesh]
    if a.mesh_path:
        cmd += ["--mesh-path", a.mesh_path]
    cmd += ["--boundary", a.boundary, "--label-source", a.label_source, "--cache-preset", a.cache_preset,
            "--train-points", str(t["train_points"]), "--eval-mode", "slice",
            "--slice-width", str(a.slice_width), "--slice-height", str(a.slice_height),
            "--slice-view", a.slice_view, "--slice-plane", str(a.slice_plane),
            "--slice-preserve-world-aspect", "1" if a.slice_preserve_world_aspect else "0",
            "--slice-padding-fraction", str(a.slice_padding_fraction)]
    if a.slice_frame:
        cmd += ["--slice-frame", a.slice_frame]
    cmd += ["--label-refreshes", str(t["label_refreshes"]),
            "--walks-per-label-refresh", str(t["walks_per_label_refresh"]),
            "--train-steps-per-refresh", str(t["train_steps_per_refresh"]),
            "--depth-m", str(a.depth_m), "--max-steps", str(a.max_steps), "--epsilon", str(a.epsilon),
            "--seed", str(a.seed), "--cubql-build-method", a.cubql_build_method,
            "--cubql-leaf-size", str(a.cubql_leaf_size), "--output", str(output),
            "--normalize", "1" if a.normalize else "0", "--jit", "1" if a.jit else "0"]
    if a.mesh == "procedural_bumpy_sphere":
        cmd += ["--bumpy-stacks", str(a.bumpy_stacks), "--bumpy-slices", str(a.bumpy_slices),
                "--bumpy-amplitude", str(a.bumpy_amplitude)]
    b = plan.budget
    cmd += ["--pure-walks-per-point", str(b["pure"]), "--hybrid-walks-per-point", str(b["hybrid"]),
            "--enable-2lmc", str(b["lmc"]), "--coarse-walks-per-point", str(b["coarse"]),
            "--residual-walks-per-point", str(b["residual"])]
    return cmd


def method_run(data: Dict[str, Any], method: str) -> Optional[Dict[str, Any]]:
    """The run record of `method` in a result JSON (an ``nc_2lmc*`` key for NC+2LMC)."""
    runs = data.get("runs") or {}
    if method in runs:
        return runs[method]
    if method == "nc_2lmc":
        return next((v for k, v in runs.items() if k.startswith("nc_2lmc")), None)
    return None


def point_row(a: argparse.Namespace, plan: RunPlan, path: Path, data: Dict[str, Any],
              run: Dict[str, Any]) -> Dict[str, Any]:
    """One row of time_mse_points.csv."""
    pure = plan.method == "pure_wos"
    tr, opts = data.get("training") or {}, data.get("options") or {}
    rmse = _num(run.get("rmse"))
    solve = _num(run.get("elapsed_ms"))
    train = 0.0 if pure else _num(tr.get("total_training_ms"), 0.0)
    w = plan.walks
    return {
        "method": plan.method, "label": plan.label, "json_path": str(path),
        "cache_preset": "" if pure else a.cache_preset, "boundary_condition": a.boundary,
        "depth_m": "" if pure else a.depth_m, "train_points_requested": "" if pure else a.train_points,
        "train_points_padded": opts.get("train_points_padded", ""),
        "total_train_steps": int(a.label_refreshes) * int(a.train_steps_per_refresh),
        "pure_walks_per_point": w.get("pure", ""), "hybrid_walks_per_point": w.get("hybrid", ""),
        "coarse_walks_per_point": w.get("coarse", ""), "residual_walks_per_point": w.get("residual", ""),
        "slice_width": a.slice_width, "slice_height": a.slice_height, "slice_view": a.slice_view,
        "slice_plane": a.slice_plane,
        "eval_points": run.get("eval_points", opts.get("eval_points", "")),
        "inside_pixels": (data.get("slice") or {}).get("inside_pixels", run.get("eval_points", "")),
        "rmse": rmse, "mse": rmse * rmse if math.isfinite(rmse) else NAN,
        "mean_bias": _num(run.get("mean_bias")), "mean_sample_variance": _num(run.get("mean_sample_variance")),
        "mean_coarse_sample_variance": _num(run.get("mean_coarse_sample_variance")),
        "mean_residual_sample_variance": _num(run.get("mean_residual_sample_variance")),
        "residual_variance_ratio_vs_pure": NAN,
        "solve_only_ms": solve, "training_ms": train,
        "end_to_end_ms": _num(run.get("training_plus_elapsed_ms"), train + solve),
        "single_snapshot_total_ms": NAN,
        "label_update_ms": 0.0 if pure else _num(tr.get("label_update_ms"), 0.0),
        "tcnn_training_ms": 0.0 if pure else _num(tr.get("tcnn_training_ms"), 0.0),
    }


def account(rows: List[Dict[str, Any]]) -> float:
    """Single-snapshot accounting and residual-variance ratios, in place.
    Returns the representative (median) training time of the NC runs."""
    trained = [r["training_ms"] for r in rows if r["method"] != "pure_wos" and _num(r["training_ms"]) > 0]
    rep = statistics.median(trained) if trained else 0.0
    for r in rows:
        if r["method"] == "pure_wos":
            r["single_snapshot_total_ms"] = r["end_to_end_ms"] = r["solve_only_ms"]
        else:
            r["single_snapshot_total_ms"] = rep + _num(r["solve_only_ms"])
    pure_var = [_num(r["mean_sample_variance"]) for r in rows if r["method"] == "pure_wos"]
    pure_var = [v for v in pure_var if math.isfinite(v)]
    ref = pure_var[-1] if pure_var else NAN  # the last (largest-budget) pure run
    if math.isfinite(ref) and ref > 0:
        for r in rows:
            rv = _num(r["mean_residual_sample_variance"])
            if r["method"] == "nc_2lmc" and math.isfinite(rv):
                r["residual_variance_ratio_vs_pure"] = rv / ref
    return rep


def time_to_thresholds(rows: List[Dict[str, Any]], rmse_list: Sequence[float]) -> List[Dict[str, Any]]:
    """Per threshold RMSE, method and time mode: the fastest run whose MSE is
    at most the threshold squared (hit = False when none is)."""
    out = []
    methods = sorted({str(r["method"]) for r in rows})
    for thr in rmse_list:
        mse_max = thr * thr
        for m in methods:
            for mode in TIME_MODES:
                ok = [r for r in rows if r["method"] == m and _num(r["mse"]) <= mse_max
                      and math.isfinite(_num(r[mode]))]
                rec = {"threshold_rmse": thr, "threshold_mse": mse_max, "method": m, "time_mode": mode}
                if ok:
                    best = min(ok, key=lambda r: _num(r[mode]))
                    rec.update(hit=True, best_time_ms=best[mode], best_label=best["label"], best_rmse=best["rmse"])
                else:
                    rec.update(hit=False, best_time_ms="", best_label="", best_rmse="")
                out.append(rec)
    return out


def _write_csv(path: Path, rows: List[Dict[str, Any]], columns: List[str]) -> None:
    path.parent.mkdir(parents=True, exist_ok=True)
    with path.open("w", newline="", encoding="utf-8") as f:
        w = csv.DictWriter(f, fieldnames=columns, extrasaction="ignore")
        w.writeheader()
        w.writerows(rows)


def main(argv: Optional[Sequence[str]] = None) -> int:
    a = parser().parse_args(argv)
    out_dir = Path(a.output_dir)
    runs_dir = out_dir / "runs"
    runs_dir.mkdir(parents=True, exist_ok=True)
    thresholds = _floats(a.threshold_rmse_list)
    manifest: Dict[str, Any] = {
        "script": "run_nc_slice_time_to_mse.py",
        "purpose": "Build MSE-vs-time points for pure WoS, NC-only, and NC+2LMC on a fixed slice.",
        "limitations": {
            "underlying_solver": "n2wos_eval_tcnn_nc_wos fixed-snapshot executable",
            "actual_progressive_online_training": False,
            "single_snapshot_total_ms_is_accounting": True,
            "pure_probe_uses_dummy_cache_training": True,
            "reference": "Current executable RMSE is used as reported. High-sample pure-WoS numerical "
                         "reference is not created by this runner.",
        },
        "arguments": vars(a), "commands": [], "errors": [],
    }
    rows: List[Dict[str, Any]] = []
    for plan in plan_runs(a):
        output = runs_dir / f"{plan.label}.json"
        cmd = command(a, plan, output)
        manifest["commands"].append({"label": plan.label, "output": str(output), "command": cmd})
        if a.skip_existing and output.exists():
            print(f"[skip] {output}", flush=True)
        else:
            print(" ".join(cmd), flush=True)
            if a.dry_run:
                continue
            rc = subprocess.run(cmd).returncode
            if rc != 0:
                if not a.continue_on_error:
                    raise SystemExit(rc)
                manifest["errors"].append({"label": plan.label, "returncode": rc})
                continue
        if a.dry_run:
            continue
        if not output.exists():
            manifest["errors"].append({"label": plan.label, "error": "output_missing"})
            continue
        data = json.loads(output.read_text(encoding="utf-8"))
        run = method_run(data, plan.method)
        if run:
            rows.append(point_row(a, plan, output, data, run))
    rep = account(rows)
    thr_rows = time_to_thresholds(rows, thresholds)
    _write_csv(out_dir / "time_mse_points.csv", rows, POINT_COLUMNS)
    _write_csv(out_dir / "time_to_threshold.csv", thr_rows, THRESHOLD_COLUMNS)
    summary = {"manifest": manifest, "representative_training_ms_for_single_snapshot_total": rep,
               "rows": rows, "thresholds": thr_rows}
    (out_dir / "summary.json").write_text(json.dumps(summary, indent=2), encoding="utf-8")
    (out_dir / "manifest.json").write_text(json.dumps(manifest, indent=2), encoding="utf-8")
    for name in ("time_mse_points.csv", "time_to_threshold.csv", "summary.json"):
        print(f"Wrote {out_dir / name}")
    return 0


if __name__ == "__main__":
    sys.exit(main())
