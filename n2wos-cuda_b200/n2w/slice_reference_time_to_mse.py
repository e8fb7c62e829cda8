"""Slice time-to-MSE against a Monte Carlo reference (no analytic solution
needed), around the ``n2wos_eval_tcnn_nc_wos`` executable.

Drop-in for the reference's ``scripts/run_nc_slice_reference_time_to_mse.py``:
the same flags and defaults (170-212), the same command lines (common flags
216-241, reference chunks 252-270, pure / NC / NC+2LMC budget curves
327-404), the same output files (``estimates/reference_pure_estimates.csv``,
``time_mse_points_reference.csv``, ``time_to_threshold_reference.csv``,
``summary_reference.json``, ``manifest.json`` for a dry run) and columns:

1. a high-budget pure-WoS reference is run in chunks of at most
   ``--reference-chunk-wpp`` walks per pixel (so no run's sample counters
   overflow), each chunk with its own seed, and the chunks' per-pixel means
   and sample variances are merged with the pairwise update of Chan, Golub &
   LeVeque (1979): n = n_a + n_b, d = m_b - m_a, m = m_a + d n_b / n,
   M2 = M2_a + M2_b + d^2 n_a n_b / n, with M2 = (n - 1) s^2;
2. every low-budget run's per-pixel estimates are compared with the merged
   reference: MSE, RMSE, MAE and mean error; the reference's own RMSE floor is
   sqrt(mean reference variance / reference walks);
3. per threshold RMSE, method and time mode (solve only; training + solve)
   the fastest run under the threshold.

    python -m n2w.slice_reference_time_to_mse --output-dir out/ref [--executable BIN] [reference flags ...]
"""
from __future__ import annotations

import argparse
import csv
import json
import math
import subprocess
import sys
from pathlib import Path
from typing import Any, Dict, List, Optional, Sequence, Tuple

import numpy as np

from .time_to_mse import method_run

DEFAULT_EXECUTABLE = Path(__file__).resolve().parent.parent / "bin" / "n2wos_eval_tcnn_nc_wos"
REFERENCE_COLUMNS = ["point_id", "x", "y", "z", "analytic_value", "pure_mean", "pure_sample_variance",
                     "reference_wpp"]
POINT_COLUMNS = ["method", "label", "rmse_vs_reference", "mse_vs_reference", "mae_vs_reference",
                 "mean_error_vs_reference", "solve_only_ms", "training_ms", "training_plus_solve_ms",
                 "default_time_ms", "reference_wpp", "reference_rmse_floor_estimate", "json_path", "estimates_csv"]
THRESHOLD_COLUMNS = ["threshold_rmse", "method", "time_mode", "hit", "best_time_ms", "best_label",
                     "best_rmse_vs_reference"]
SCHEMA = "n2wos_reference_slice_time_to_mse_v1"


def parser() -> argparse.ArgumentParser:
    ap = argparse.ArgumentParser(description="Reference-based slice time-to-MSE runner.")
    ap.add_argument("--executable", default=str(DEFAULT_EXECUTABLE))
    ap.add_argument("--output-dir", required=True)
    ap.add_argument("--mesh", default="procedural_bumpy_sphere")
    ap.add_argument("--mesh-path", default="")
    ap.add_argument("--normalize", type=int, default=1)
    ap.add_argument("--bumpy-stacks", type=int, default=128)
    ap.add_argument("--bumpy-slices", type=int, default=256)
    ap.add_argument("--bumpy-amplitude", type=float, default=0.15)
    ap.add_argument("--boundary", default="boundary_texture_stripes_k16")
    ap.add_argument("--label-source", default="wos_supervision")
    ap.add_argument("--cache-preset", default="nano")
    ap.add_argument("--train-points", type=int, default=20000)
    ap.add_argument("--train-sampler", default="rejection")
    ap.add_argument("--label-refreshes", type=int, default=4)
    ap.add_argument("--walks-per-label-refresh", type=int, default=50)
    ap.add_argument("--train-steps-per-refresh", type=int, default=5000)
    ap.add_argument("--depth-m", type=int, default=4)
    ap.add_argument("--slice-width", type=int, default=512)
    ap.add_argument("--slice-height", type=int, default=512)
    ap.add_argument("--slice-view", default="xy")
    ap.add_argument("--slice-plane", default="0")
    ap.add_argument("--slice-padding-fraction", default="0.02")
    ap.add_argument("--slice-preserve-world-aspect", type=int, default=1)
    ap.add_argument("--reference-wpp", type=int, default=16384,
                    help="total pure-WoS walks per point of the numerical reference")
    ap.add_argument("--reference-chunk-wpp", type=int, default=512,
                    help="walks per point of one reference chunk (keeps each run's sample counts small)")
    ap.add_argument("--reference-seed", type=int, default=987654321)
    ap.add_argument("--pure-wpp-list", default="8,16,32,64,128")
    ap.add_argument("--nc-hybrid-wpp-list", default="1,2,4,8,16")
    ap.add_argument("--lmc-allocations", default="16:8,32:16,32:32,64:32")
    ap.add_argument("--threshold-rmse-list", default="0.03,0.05,0.075,0.1")
    ap.add_argument("--max-steps", type=int, default=256)
    ap.add_argument("--epsilon", default="1e-4")
    ap.add_argument("--seed", type=int, default=12345)
    ap.add_argument("--cubql-build-method", default="sah")
    ap.add_argument("--cubql-leaf-size", type=int, default=8)
    ap.add_argument("--jit", type=int, default=0)
    ap.add_argument("--dry-run", action="store_true")
    ap.add_argument("--skip-existing", action="store_true")
    return ap


def _ints(text: str) -> List[int]:
    return [int(t) for t in text.split(",") if t.strip()]


def _floats(text: str) -> List[float]:
    return [float(t) for t in text.split(",") if t.strip()]


def _allocations(text: str) -> List[Tuple[int, int]]:
    out = []
    for t in text.split(","):
        if t.strip():
            c, r = t.split(":")
            out.append((int(c), int(r)))
    return out


def read_estimates(path: Path) -> List[Dict[str, str]]:
    with Path(path).open(newline="", encoding="utf-8") as f:
        return list(csv.DictReader(f))


def _write(path: Path, rows: List[Dict[str, Any]], columns: List[str]) -> None:
    path.parent.mkdir(parents=True, exist_ok=True)
    with path.open("w", newline="", encoding="utf-8") as f:
        w = csv.DictWriter(f, fieldnames=columns, extrasaction="ignore")
        w.writeheader()
        w.writerows(rows)


def merge_chunks(paths: Sequence[Path], wpps: Sequence[int], out_path: Path) -> Tuple[np.ndarray, np.ndarray, int]:
    """Per-pixel mean and sample variance of the union of the reference
    chunks (pairwise Chan update, one chunk at a time); writes the merged
    estimates CSV and returns (means, variances, total walks per pixel)."""
    if not paths:
        raise RuntimeError("no reference chunks to combine")
    if len(paths) != len(wpps):
        raise RuntimeError("chunk path/wpp count mismatch")
    first = read_estimates(paths[0])
    if not first:
        raise RuntimeError("empty reference estimates")
    n = np.zeros(len(first))
    mean = np.zeros(len(first))
    m2 = np.zeros(len(first))
    for path, wpp in zip(paths, wpps):
        rows = first if path == paths[0] else read_estimates(path)
        if len(rows) != len(first):
            raise RuntimeError(f"reference chunk row count mismatch in {path}: {len(rows)} vs {len(first)}")
        if wpp <= 0:
            raise RuntimeError(f"invalid reference chunk wpp {wpp} in {path}")
        mb = np.array([float(r["pure_mean"]) for r in rows])
        vb = np.array([float(r.get("pure_sample_variance", 0.0)) for r in rows])
        vb[(vb < 0) & (vb > -1e-12)] = 0.0  # rounding of an exact zero
        if (vb < 0).any():
            i = int(np.argmax(vb < 0))
            raise RuntimeError(f"negative reference chunk variance at point {i} in {path}: {vb[i]}")
        nb = float(wpp)
        m2b = (nb - 1.0) * vb if wpp > 1 else np.zeros_like(vb)
        tot = n + nb
        d = mb - mean
        mean = np.where(n > 0, mean + d * (nb / tot), mb)
        m2 = np.where(n > 0, m2 + m2b + d * d * (n * nb / tot), m2b)
        n = tot
    var = m2 / np.maximum(1.0, n - 1.0)
    var[(var < 0) & (var > -1e-12)] = 0.0
    total = int(sum(wpps))
    _write(out_path, [{"point_id": r.get("point_id", i), "x": r.get("x", ""), "y": r.get("y", ""),
                       "z": r.get("z", ""), "analytic_value": r.get("analytic_value", ""), "pure_mean": float(mean[i]),
                       "pure_sample_variance": float(var[i]), "reference_wpp": total}
                      for i, r in enumerate(first)], REFERENCE_COLUMNS)
    return mean, var, total


def errors_vs(rows: List[Dict[str, str]], ref: np.ndarray, column: str) -> Tuple[float, float, float, float]:
    """(MSE, RMSE, MAE, mean error) of a run's per-pixel column against the reference."""
    if len(rows) != len(ref):
        raise RuntimeError(f"row count mismatch for {column}: {len(rows)} vs reference {len(ref)}")
    e = np.array([float(r[column]) for r in rows]) - ref
    mse = float(np.mean(e * e))
    return mse, math.sqrt(max(0.0, mse)), float(np.mean(np.abs(e))), float(np.mean(e))


def main(argv: Optional[Sequence[str]] = None) -> int:
    a = parser().parse_args(argv)
    out_dir = Path(a.output_dir)
    runs_dir, est_dir = out_dir / "runs", out_dir / "estimates"
    for d in (out_dir, runs_dir, est_dir):
        d.mkdir(parents=True, exist_ok=True)
    common = [a.executable, "--mesh", a.mesh, "--boundary", a.boundary, "--label-source", a.label_source,
              "--cache-preset", a.cache_preset, "--train-sampler", a.train_sampler, "--eval-mode", "slice",
              "--slice-width", str(a.slice_width), "--slice-height", str(a.slice_height), "--slice-view", a.slice_view,
              "--slice-plane", str(a.slice_plane), "--slice-preserve-world-aspect", str(a.slice_preserve_world_aspect),
              "--slice-padding-fraction", str(a.slice_padding_fraction), "--depth-m", str(a.depth_m),
              "--max-steps", str(a.max_steps), "--epsilon", str(a.epsilon),
              "--cubql-build-method", a.cubql_build_method, "--cubql-leaf-size", str(a.cubql_leaf_size),
              "--normalize", str(a.normalize), "--jit", str(a.jit), "--bumpy-stacks", str(a.bumpy_stacks),
              "--bumpy-slices", str(a.bumpy_slices), "--bumpy-amplitude", str(a.bumpy_amplitude)]
    if a.mesh_path:
        common += ["--mesh-path", a.mesh_path]
    no_training = ["--train-points", "128", "--label-refreshes", "1", "--walks-per-label-refresh", "1",
                   "--train-steps-per-refresh", "0", "--skip-training", "1"]
    training = ["--train-points", str(a.train_points), "--label-refreshes", str(a.label_refreshes),
                "--walks-per-label-refresh", str(a.walks_per_label_refresh),
                "--train-steps-per-refresh", str(a.train_steps_per_refresh)]

    def budget(pure: int, hybrid: int, lmc: int, coarse: int, residual: int) -> List[str]:
        return ["--pure-walks-per-point", str(pure), "--hybrid-walks-per-point", str(hybrid), "--enable-2lmc",
                str(lmc), "--coarse-walks-per-point", str(coarse), "--residual-walks-per-point", str(residual)]

    def outputs(seed: int, prefix: Path, json_path: Path) -> List[str]:
        return ["--seed", str(seed), "--slice-output-prefix", str(out_dir / "slice"),
                "--save-estimates-prefix", str(prefix), "--output", str(json_path)]

    def run(cmd: List[str], json_path: Path, prefix: Path) -> None:
        if a.skip_existing and json_path.exists() and Path(f"{prefix}_estimates.csv").exists():
            return
        print("+", " ".join(cmd), flush=True)
        if not a.dry_run:
            subprocess.run(cmd, check=True)

    # 1. the chunked pure-WoS reference
    if a.reference_chunk_wpp <= 0 and a.reference_wpp > 0:
        raise RuntimeError("--reference-chunk-wpp must be positive")
    ref_cmds: List[Dict[str, Any]] = []
    chunk_csvs: List[Path] = []
    chunk_wpps: List[int] = []
    left, k = a.reference_wpp, 0
    while left > 0:
        w = min(a.reference_chunk_wpp, left)
        label = f"reference_pure_chunk{k:03d}_wpp{w}"
        json_path, prefix = runs_dir / f"{label}.json", est_dir / label
        cmd = common + no_training + budget(w, 1, 0, 1, 1) + outputs(a.reference_seed + 100003 * k, prefix, json_path)
        ref_cmds.append({"method": "reference_pure", "label": label, "wpp": w, "command": cmd})
        run(cmd, json_path, prefix)
        chunk_csvs.append(Path(f"{prefix}_estimates.csv"))
        chunk_wpps.append(w)
        left -= w
        k += 1
    ref_csv = est_dir / "reference_pure_estimates.csv"
    if a.dry_run:
        ref, ref_var, ref_wpp = np.zeros(0), np.zeros(0), a.reference_wpp
    else:
        ref, ref_var, ref_wpp = merge_chunks(chunk_csvs, chunk_wpps, ref_csv)
    mean_ref_var = float(np.mean(ref_var)) if len(ref_var) else 0.0
    floor = math.sqrt(max(0.0, mean_ref_var / max(1, ref_wpp))) if len(ref_var) else 0.0

    # 2-4. the budget curves
    plans = [("pure_wos", f"pure_wpp{w}", no_training + budget(w, 1, 0, 1, 1), a.seed + 1000 + w, "pure_mean", False)
             for w in _ints(a.pure_wpp_list)]
    plans += [("nc_wos", f"nc_wpp{w}", training + budget(1, w, 0, 1, 1), a.seed + 2000 + w, "nc_wos_mean", True)
              for w in _ints(a.nc_hybrid_wpp_list)]
    plans += [("nc_2lmc", f"nc2lmc_c{c}_r{r}", training + budget(1, 1, 1, c, r), a.seed + 3000 + 17 * c + r,
               "nc_2lmc_mean", True) for c, r in _allocations(a.lmc_allocations)]
    commands: List[Dict[str, Any]] = []
    points: List[Dict[str, Any]] = []
    for method, label, flags, seed, column, with_training in plans:
        json_path, prefix = runs_dir / f"{label}.json", est_dir / label
        cmd = common + flags + outputs(seed, prefix, json_path)
        commands.append({"method": method, "label": label, "command": cmd})
        run(cmd, json_path, prefix)
        if a.dry_run:
            continue
        doc = json.loads(json_path.read_text(encoding="utf-8"))
        est_csv = f"{prefix}_estimates.csv"
        mse, rmse, mae, mean_err = errors_vs(read_estimates(Path(est_csv)), ref, column)
        solve = float((method_run(doc, method) or {}).get("elapsed_ms", 0.0))
        train = float((doc.get("training") or {}).get("total_training_ms", 0.0))
        points.append({"method": method, "label": label, "rmse_vs_reference": rmse, "mse_vs_reference": mse,
                       "mae_vs_reference": mae, "mean_error_vs_reference": mean_err, "solve_only_ms": solve,
                       "training_ms": train, "training_plus_solve_ms": solve + train,
                       "default_time_ms": solve + train if with_training else solve, "reference_wpp": ref_wpp,
                       "reference_rmse_floor_estimate": floor, "json_path": str(json_path),
                       "estimates_csv": est_csv})
    if a.dry_run:
        (out_dir / "manifest.json").write_text(json.dumps(
            {"arguments": vars(a), "reference_commands": ref_cmds, "commands": commands, "dry_run": True},
            indent=2), encoding="utf-8")
        return 0
    _write(out_dir / "time_mse_points_reference.csv", points, POINT_COLUMNS)
    thr_rows: List[Dict[str, Any]] = []
    for thr in _floats(a.threshold_rmse_list):
        for method in ("pure_wos", "nc_wos", "nc_2lmc"):
            ok = [p for p in points if p["method"] == method and p["rmse_vs_reference"] <= thr]
            for mode in ("solve_only_ms", "training_plus_solve_ms"):
                rec = {"threshold_rmse": thr, "method": method, "time_mode": mode}
                if ok:
                    b = min(ok, key=lambda p: float(p[mode]))
                    rec.update(hit=True, best_time_ms=b[mode], best_label=b["label"],
                               best_rmse_vs_reference=b["rmse_vs_reference"])
                else:
                    rec.update(hit=False, best_time_ms="", best_label="", best_rmse_vs_reference="")
                thr_rows.append(rec)
    _write(out_dir / "time_to_threshold_reference.csv", thr_rows, THRESHOLD_COLUMNS)
    summary = {
        "schema": SCHEMA, "arguments": vars(a),
        "reference": {"estimates_csv": str(ref_csv), "reference_chunk_wpp": a.reference_chunk_wpp,
                      "reference_chunks": [str(p) for p in chunk_csvs], "reference_wpp": ref_wpp,
                      "reference_rmse_floor_estimate": floor, "mean_reference_sample_variance": mean_ref_var},
        "points": points, "thresholds": thr_rows, "reference_commands": ref_cmds, "commands": commands,
        "limitations": {"reference_is_monte_carlo": True, "reference_seed_independent_from_method_seeds": True,
                        "method_runs_retrain_cache_independently": True, "not_true_online_progressive_runner": True},
    }
    (out_dir / "summary_reference.json").write_text(json.dumps(summary, indent=2), encoding="utf-8")
    print("wrote", out_dir / "time_mse_points_reference.csv")
    print("wrote", out_dir / "time_to_threshold_reference.csv")
    return 0


if __name__ == "__main__":
    sys.exit(main())
