"""Pure WoS vs analytic-cache 2LMC ("oracle_2lmc") sweeps around the
``n2wos_eval_wavefront_wos`` executable, per seed and aggregated over seeds.

Drop-in for the reference's ``scripts/run_wavefront_oracle_sweep.py`` and
``scripts/run_wavefront_oracle_multiseed.py``: the same flags and defaults
(sweep 308-345, multi-seed 207-231), the same per-run command lines
(add_common_solver_args, sweep 60-83), the same output files and columns, and
the same statistics:

* variance-time product of a run = estimator variance x total elapsed ms, and
  its speedup against the pure-WoS run of the same seed (sweep 105-106);
* |error| / stderr of the 2LMC estimate against the exact value, and of the
  residual level's mean against zero (the exact cache makes the residual a
  zero-mean quantity), flagged above 3 (sweep 112-160);
* the variance-optimal coarse : residual sample ratio sqrt(v_c c_r / (v_r c_c))
  and its predicted variance-time product (sqrt(v_c c_c) + sqrt(v_r c_r))^2,
  c = ms per sample (sweep 162-176);
* over seeds: the bias of the seed-mean estimate with the pooled standard
  error sqrt(sum_i var_i) / n, its z-score, and the RMSE of the seed estimates
  (multi-seed 166-185).

    python -m n2w.wavefront_oracle_sweep [--executable BIN] [reference flags ...]
    python -m n2w.wavefront_oracle_sweep multiseed [--seeds 12345,23456,...] [flags ...]
"""
from __future__ import annotations

import argparse
import csv
import json
import math
import shlex
import subprocess
import sys
import time
from pathlib import Path
from typing import Any, Dict, Iterable, List, Optional

DEFAULT_EXECUTABLE = Path(__file__).resolve().parent.parent / "bin" / "n2wos_eval_wavefront_wos"
NAN = math.nan
SWEEP_SCHEMA = "n2wos_wavefront_oracle_sweep_v1"
MULTISEED_SCHEMA = "n2wos_wavefront_oracle_multiseed_v1"
# columns summarised per label (mean / std / min / max) in <summary>_by_label.csv
LABEL_STAT_COLUMNS = (
    "score_speedup_vs_pure", "optimal_speedup_vs_pure_predicted", "variance_time_product_ms",
    "actual_variance_time_product_ms", "estimator_variance", "elapsed_ms_total", "abs_error", "stderr",
    "z_abs_error", "estimator_z_abs_error", "residual_z_abs_mean", "residual_variance_ratio_vs_coarse",
    "coarse_us_per_sample", "residual_us_per_sample", "coarse_mean_steps", "residual_mean_steps",
)


def _list(text: str, conv, what: str) -> list:
    vals = [conv(t.strip()) for t in str(text).split(",") if t.strip()]
    if not vals:
        raise argparse.ArgumentTypeError(f"expected at least one {what}")
    return vals


def _ints(text: str) -> List[int]:
    return _list(text, int, "integer")


def _floats(text: str) -> List[float]:
    return _list(text, float, "number")


def _seeds(text: str) -> List[int]:
    vals = _list(text, lambda t: int(t, 0), "seed")
    if any(v < 0 for v in vals):
        raise argparse.ArgumentTypeError("seeds must be non-negative")
    return vals


def _f(v: Any) -> float:
    """Finite float of a field, NaN otherwise."""
    try:
        x = float(v)
    except (TypeError, ValueError):
        return NAN
    return x if math.isfinite(x) else NAN


def _finite(vals: Iterable[Any]) -> List[float]:
    return [x for x in (_f(v) for v in vals) if math.isfinite(x)]


def _mean(vals: Iterable[Any]) -> float:
    xs = _finite(vals)
    return sum(xs) / len(xs) if xs else NAN


def _z(err: float, se: float) -> float:
    return abs(err) / se if math.isfinite(err) and math.isfinite(se) and se > 0 else NAN


def _ratio(num: Optional[float], den: float) -> float:
    return num / den if num and math.isfinite(den) and den > 0 else NAN


def vt_product(estimator: Dict[str, Any]) -> float:
    """Variance-time product (ms) of a run's estimator."""
    return _f(estimator.get("estimator_variance")) * _f(estimator.get("elapsed_ms_total"))


# ---- one sweep ----------------------------------------------------------------

def sweep_parser() -> argparse.ArgumentParser:
    ap = argparse.ArgumentParser(description="pure WoS vs oracle_2lmc sweep over n2wos_eval_wavefront_wos")
    ap.add_argument("--executable", default=str(DEFAULT_EXECUTABLE))
    ap.add_argument("--output-dir", default="results/wavefront_oracle_sweep")
    ap.add_argument("--summary-name", default="summary")
    _solver_flags(ap, engine="wavefront")
    ap.add_argument("--seed", type=int, default=12345)
    ap.add_argument("--seeds", type=_seeds, default=None, help="repeat the sweep for each of these seeds")
    ap.add_argument("--seed-count", type=int, default=1, help="without --seeds: this many seeds from --seed")
    ap.add_argument("--seed-stride", type=int, default=1000003, help="seed increment with --seed-count")
    ap.add_argument("--skip-pure", action="store_true")
    ap.add_argument("--dry-run", action="store_true")
    return ap


def _solver_flags(ap: argparse.ArgumentParser, engine: str, list_type=None) -> None:
    ap.add_argument("--mesh", default="procedural_bumpy_sphere", choices=["procedural_bumpy_sphere", "obj", "ply"])
    ap.add_argument("--engine", default=engine, choices=["wavefront", "persistent"])
    ap.add_argument("--mesh-path", default="")
    ap.add_argument("--normalize", type=int, choices=[0, 1], default=1)
    ap.add_argument("--bumpy-stacks", type=int, default=128)
    ap.add_argument("--bumpy-slices", type=int, default=256)
    ap.add_argument("--bumpy-amplitude", type=float, default=0.15)
    ap.add_argument("--pure-samples", type=int, default=262144)
    ap.add_argument("--residual-samples", type=int, default=65536)
    ap.add_argument("--coarse-ratios", type=list_type or _floats, default=(list_type or _floats)("1,2,4,8"))
    ap.add_argument("--depths", type=list_type or _ints, default=(list_type or _ints)("1,2,4,8,16"))
    ap.add_argument("--max-steps", type=int, default=256)
    ap.add_argument("--epsilon", type=float, default=1e-4)
    ap.add_argument("--step-scale", type=float, default=0.999)
    ap.add_argument("--x0", default="0.1,0.05,0")
    ap.add_argument("--block-size", type=int, default=128)
    ap.add_argument("--cubql-build-method", default="sah")
    ap.add_argument("--cubql-leaf-size", type=int, default=8)


def solver_flags(a: argparse.Namespace, seed: int) -> List[str]:
    f = ["--mesh", a.mesh, "--engine", a.engine, "--max-steps", str(a.max_steps), "--epsilon", str(a.epsilon),
         "--step-scale", str(a.step_scale), "--x0", a.x0, "--seed", str(seed), "--block-size", str(a.block_size),
         "--cubql-build-method", a.cubql_build_method, "--cubql-leaf-size", str(a.cubql_leaf_size)]
    if a.mesh_path:
        f += ["--mesh-path", a.mesh_path]
    f += ["--normalize", "1" if a.normalize else "0"]
    if a.mesh == "procedural_bumpy_sphere":
        f += ["--bumpy-stacks", str(a.bumpy_stacks), "--bumpy-slices", str(a.bumpy_slices),
              "--bumpy-amplitude", str(a.bumpy_amplitude)]
    return f


def _run(cmd: List[str], dry_run: bool) -> None:
    print("+ " + " ".join(shlex.quote(c) for c in cmd), flush=True)
    if not dry_run:
        subprocess.run(cmd, check=True)


def lmc_metrics(doc: Dict[str, Any], pure_vt: Optional[float]) -> Dict[str, Any]:
    """Per-run statistics of an oracle_2lmc result."""
    est, runs = doc.get("estimator") or {}, doc.get("runs") or {}
    c, r = runs.get("coarse") or {}, runs.get("residual") or {}
    exact = _f(est.get("exact"))
    vt = vt_product(est)
    out: Dict[str, Any] = {
        "actual_variance_time_product_ms": vt,
        "actual_speedup_vs_pure": _ratio(pure_vt, vt),
        "estimator_z_abs_error": _z(_f(est.get("mean")) - exact, _f(est.get("stderr"))),
    }
    for name, run, target in (("coarse", c, exact), ("residual", r, 0.0)):
        for k in ("mean", "sample_variance", "estimator_variance", "stderr", "elapsed_ms", "us_per_sample",
                  "mean_steps"):
            out[f"{name}_{k}"] = run.get(k)
        z = _z(_f(run.get("mean")) - target, _f(run.get("stderr")))
        out["coarse_z_abs_error" if name == "coarse" else "residual_z_abs_mean"] = z
    # a persistent |z| > 3 across seeds points at a coupling or stopping-rule bug
    out["diagnostic_flag_large_estimator_z"] = bool(out["estimator_z_abs_error"] > 3.0)
    out["diagnostic_flag_large_residual_z"] = bool(out["residual_z_abs_mean"] > 3.0)
    vc, vr = _f(c.get("sample_variance")), _f(r.get("sample_variance"))
    cc, cr = 1e-3 * _f(c.get("us_per_sample")), 1e-3 * _f(r.get("us_per_sample"))
    if all(x > 0 for x in (vc, vr, cc, cr)):  # NaN compares false
        best = (math.sqrt(vc * cc) + math.sqrt(vr * cr)) ** 2
        out.update({
            "measured_coarse_to_residual_sample_ratio": _f(c.get("samples")) / _f(r.get("samples")),
            "optimal_coarse_to_residual_sample_ratio": math.sqrt((vc * cr) / (vr * cc)),
            "optimal_variance_time_product_ms_predicted": best,
            "optimal_speedup_vs_pure_predicted": _ratio(pure_vt, best),
            "residual_variance_ratio_vs_coarse": vr / vc,
        })
    return out


def summary_row(label: str, doc: Dict[str, Any], extra: Dict[str, Any], pure_vt: Optional[float]) -> Dict[str, Any]:
    est, opts = doc.get("estimator") or {}, doc.get("options") or {}
    vt = vt_product(est)
    runs = list((doc.get("runs") or {}).values())
    row: Dict[str, Any] = {
        "label": label, "method": est.get("method", opts.get("method")),
        "engine": est.get("engine", opts.get("engine")), "depth_m": opts.get("depth_m"),
        "samples": opts.get("samples"), "coarse_samples": opts.get("coarse_samples"),
        "residual_samples": opts.get("residual_samples"), "mean": est.get("mean"), "exact": est.get("exact"),
        "abs_error": est.get("abs_error"), "stderr": est.get("stderr"),
        "z_abs_error": _z(_f(est.get("mean")) - _f(est.get("exact")), _f(est.get("stderr"))),
        "elapsed_ms_total": est.get("elapsed_ms_total"), "estimator_variance": est.get("estimator_variance"),
        "variance_time_product_ms": vt, "score_speedup_vs_pure": _ratio(pure_vt, vt),
        "forced_max_steps_total": sum(int(x.get("forced_max_steps", 0)) for x in runs),
        "overflow_count_total": sum(int(x.get("overflow_count", 0)) for x in runs),
        "json_path": extra.get("json_path", ""),
    }
    row.update(extra)
    return row


def _std(xs: List[float]) -> float:
    if len(xs) < 2:
        return 0.0 if xs else NAN
    m = sum(xs) / len(xs)
    return math.sqrt(sum((x - m) ** 2 for x in xs) / (len(xs) - 1))


def rows_by_label(rows: List[Dict[str, Any]]) -> List[Dict[str, Any]]:
    """Per label (in first-seen order): mean / std / min / max of the
    summarised columns over its seeds and the count of large-z flags."""
    groups: Dict[str, List[Dict[str, Any]]] = {}
    for r in rows:
        groups.setdefault(str(r.get("label", "")), []).append(r)
    out = []
    for label, g in groups.items():
        rec: Dict[str, Any] = {"label": label, "method": g[0].get("method"), "engine": g[0].get("engine"),
                               "depth_m": g[0].get("depth_m"),
                               "coarse_ratio_requested": g[0].get("coarse_ratio_requested"), "seed_count": len(g)}
        for col in LABEL_STAT_COLUMNS:
            xs = _finite(r.get(col) for r in g)
            rec[f"{col}_mean"] = sum(xs) / len(xs) if xs else NAN
            rec[f"{col}_std"] = _std(xs)
            rec[f"{col}_min"] = min(xs) if xs else NAN
            rec[f"{col}_max"] = max(xs) if xs else NAN
        rec["large_estimator_z_count"] = sum(bool(r.get("diagnostic_flag_large_estimator_z")) for r in g)
        rec["large_residual_z_count"] = sum(bool(r.get("diagnostic_flag_large_residual_z")) for r in g)
        out.append(rec)
    return out


def write_rows(path: Path, rows: List[Dict[str, Any]]) -> None:
    """CSV with the union of the rows' keys, in first-seen order (nothing for no rows)."""
    if not rows:
        return
    cols: Dict[str, None] = {}
    for r in rows:
        cols.update(dict.fromkeys(r))
    with path.open("w", newline="", encoding="utf-8") as f:
        w = csv.DictWriter(f, fieldnames=list(cols))
        w.writeheader()
        w.writerows(rows)


def main(argv: Optional[List[str]] = None) -> int:
    a = sweep_parser().parse_args(argv)
    if a.seeds is not None:
        seeds = a.seeds
    else:
        if a.seed_count < 1:
            raise ValueError("--seed-count must be positive")
        seeds = [a.seed + i * a.seed_stride for i in range(a.seed_count)]
    out_dir = Path(a.output_dir)
    out_dir.mkdir(parents=True, exist_ok=True)
    rows: List[Dict[str, Any]] = []
    records: List[Dict[str, Any]] = []
    pure_vt: Dict[int, float] = {}
    last_pure: Optional[float] = None
    for si, seed in enumerate(seeds):
        suffix = "" if len(seeds) == 1 else f"_seed{seed}"
        if not a.skip_pure:
            path = out_dir / f"pure_wos{suffix}.json"
            _run([a.executable, "--method", "pure_wos", "--samples", str(a.pure_samples), "--output", str(path)]
                 + solver_flags(a, seed), a.dry_run)
            if not a.dry_run:
                doc = json.loads(path.read_text(encoding="utf-8"))
                last_pure = pure_vt[seed] = vt_product(doc.get("estimator") or {})
                rows.append(summary_row("pure_wos", doc, {"json_path": str(path), "seed": seed, "seed_index": si},
                                        last_pure))
                records.append({"label": "pure_wos", "seed": seed, "json_path": str(path), "document": doc})
        ref_vt = pure_vt.get(seed, last_pure)
        for depth in a.depths:
            for ratio in a.coarse_ratios:
                label = f"oracle_2lmc_m{depth}_r{ratio:g}"
                path = out_dir / f"{label}{suffix}.json"
                coarse = max(1, int(round(a.residual_samples * ratio)))
                _run([a.executable, "--method", "oracle_2lmc", "--coarse-samples", str(coarse),
                      "--residual-samples", str(a.residual_samples), "--depth-m", str(depth), "--output", str(path)]
                     + solver_flags(a, seed), a.dry_run)
                if a.dry_run:
                    continue
                doc = json.loads(path.read_text(encoding="utf-8"))
                extra = {"json_path": str(path), "coarse_ratio_requested": ratio, "seed": seed, "seed_index": si}
                extra.update(lmc_metrics(doc, ref_vt))
                rows.append(summary_row(label, doc, extra, ref_vt))
                records.append({"label": label, "seed": seed, "json_path": str(path), "document": doc,
                                "metrics": extra})
    if a.dry_run:
        return 0
    by_label = rows_by_label(rows)
    csv_path, label_path = out_dir / f"{a.summary_name}.csv", out_dir / f"{a.summary_name}_by_label.csv"
    json_path = out_dir / f"{a.summary_name}.json"
    write_rows(csv_path, rows)
    write_rows(label_path, by_label)
    json_path.write_text(json.dumps({
        "schema": SWEEP_SCHEMA, "generated_unix_time": time.time(), "executable": a.executable,
        "output_dir": str(out_dir), "pure_variance_time_product_ms": last_pure, "seeds": seeds, "rows": rows,
        "rows_by_label": by_label, "records": records}, indent=2), encoding="utf-8")
    for p in (csv_path, label_path, json_path):
        print(f"wrote {p}")
    return 0


# ---- several seeds ---------------------------------------------------------------

def multiseed_parser() -> argparse.ArgumentParser:
    ap = argparse.ArgumentParser(description="oracle_2lmc sweeps over several RNG seeds, aggregated")
    ap.add_argument("--executable", default=str(DEFAULT_EXECUTABLE))
    ap.add_argument("--output-dir", default="results/persistent_oracle_multiseed")
    ap.add_argument("--seeds", type=_ints, default=_ints("12345,23456,34567,45678,56789"))
    _solver_flags(ap, engine="persistent", list_type=str)
    ap.add_argument("--dry-run", action="store_true")
    return ap


def _cell(text: str) -> Any:
    """A CSV cell back as a number where it is one."""
    if text == "":
        return ""
    try:
        return float(text)
    except ValueError:
        return text


def seed_aggregate(label: str, rows: List[Dict[str, Any]]) -> Dict[str, Any]:
    """Across-seed statistics of one label.  The pooled standard error of the
    seed-mean uses each run's own estimator variance: sqrt(sum var_i) / n."""
    n = len(rows)
    exact = _f(rows[0].get("exact"))
    means = [_f(r.get("mean")) for r in rows]
    errs = [m - exact for m in means if math.isfinite(m) and math.isfinite(exact)]
    var_sum = sum(_finite(r.get("estimator_variance") for r in rows))
    pooled = math.sqrt(var_sum) / n if n else NAN
    m_est = _mean(means)
    bias = m_est - exact if math.isfinite(m_est) and math.isfinite(exact) else NAN

    def col(name):
        return [r.get(name) for r in rows]

    vt, spd = _finite(col("variance_time_product_ms")), _finite(col("score_speedup_vs_pure"))
    opt = _finite(col("optimal_speedup_vs_pure_predicted"))
    el = _finite(col("elapsed_ms_total"))
    return {
        "label": label, "method": rows[0].get("method"), "engine": rows[0].get("engine"),
        "depth_m": rows[0].get("depth_m"), "coarse_ratio_requested": rows[0].get("coarse_ratio_requested"),
        "num_seeds": n, "mean_estimate_across_seeds": m_est, "exact": exact, "bias_of_seed_mean": bias,
        "abs_bias_of_seed_mean": abs(bias), "pooled_stderr_of_seed_mean": pooled,
        "bias_z_score": bias / pooled if pooled > 0 else NAN,
        "rmse_of_seed_estimates": math.sqrt(sum(e * e for e in errs) / len(errs)) if errs else NAN,
        "elapsed_ms_total_mean": _mean(el), "elapsed_ms_total_stdev": _std(el) if len(el) > 1 else NAN,
        "estimator_variance_mean": _mean(col("estimator_variance")),
        "variance_time_product_ms_mean": _mean(vt), "variance_time_product_ms_min": min(vt, default=NAN),
        "variance_time_product_ms_max": max(vt, default=NAN),
        "score_speedup_vs_pure_mean": _mean(spd), "score_speedup_vs_pure_min": min(spd, default=NAN),
        "score_speedup_vs_pure_max": max(spd, default=NAN),
        "actual_speedup_vs_pure_mean": _mean(col("actual_speedup_vs_pure")),
        "optimal_speedup_vs_pure_predicted_mean": _mean(opt),
        "optimal_speedup_vs_pure_predicted_max": max(opt, default=NAN),
        "optimal_coarse_to_residual_sample_ratio_mean": _mean(col("optimal_coarse_to_residual_sample_ratio")),
        "residual_variance_ratio_vs_coarse_mean": _mean(col("residual_variance_ratio_vs_coarse")),
        "forced_max_steps_total_sum": int(sum(_finite(col("forced_max_steps_total")))),
        "overflow_count_total_sum": int(sum(_finite(col("overflow_count_total")))),
    }


def multiseed_main(argv: Optional[List[str]] = None) -> int:
    a = multiseed_parser().parse_args(argv)
    out_dir = Path(a.output_dir)
    out_dir.mkdir(parents=True, exist_ok=True)
    manifest: Dict[str, Any] = {"schema": MULTISEED_SCHEMA, "generated_unix_time": time.time(),
                                "executable": a.executable, "engine": a.engine, "seeds": a.seeds,
                                "output_dir": str(out_dir), "seed_runs": []}
    by_seed: List[Dict[str, Any]] = []
    for seed in a.seeds:
        seed_dir = out_dir / f"seed_{seed}"
        seed_dir.mkdir(parents=True, exist_ok=True)
        argv_seed = ["--executable", a.executable, "--output-dir", str(seed_dir), "--summary-name", "summary",
                     "--pure-samples", str(a.pure_samples), "--residual-samples", str(a.residual_samples),
                     "--coarse-ratios", a.coarse_ratios, "--depths", a.depths] + solver_flags(a, seed)
        print("+ sweep " + " ".join(shlex.quote(x) for x in argv_seed), flush=True)
        if a.dry_run:
            continue
        main(argv_seed)
        csv_path = seed_dir / "summary.csv"
        with csv_path.open(newline="", encoding="utf-8") as f:
            rows = [{k: _cell(v) for k, v in r.items()} for r in csv.DictReader(f)]
        for r in rows:
            r["seed"] = seed
            r["seed_summary_path"] = str(csv_path)
        by_seed += rows
        manifest["seed_runs"].append({"seed": seed, "summary_csv": str(csv_path), "rows": len(rows)})
    if a.dry_run:
        return 0
    groups: Dict[str, List[Dict[str, Any]]] = {}
    for r in by_seed:
        groups.setdefault(str(r.get("label", "")), []).append(r)
    agg = [seed_aggregate(k, groups[k]) for k in sorted(groups)]
    by_seed_csv, agg_csv = out_dir / "summary_by_seed.csv", out_dir / "summary_aggregate.csv"
    write_rows(by_seed_csv, by_seed)
    write_rows(agg_csv, agg)
    lmc = [r for r in agg if r.get("method") == "oracle_2lmc"]

    def best(key):
        return max(lmc, key=lambda r: _f(r.get(key)) if math.isfinite(_f(r.get(key))) else -math.inf,
                   default=None)

    manifest.update({"summary_by_seed_csv": str(by_seed_csv), "summary_aggregate_csv": str(agg_csv),
                     "best_actual_oracle_2lmc": best("score_speedup_vs_pure_mean"),
                     "best_predicted_oracle_2lmc": best("optimal_speedup_vs_pure_predicted_mean"),
                     "aggregate_rows": agg})
    (out_dir / "summary_aggregate.json").write_text(json.dumps(manifest, indent=2), encoding="utf-8")
    for p in (by_seed_csv, agg_csv, out_dir / "summary_aggregate.json"):
        print(f"wrote {p}")
    return 0


if __name__ == "__main__":
    if len(sys.argv) > 1 and sys.argv[1] == "multiseed":
        sys.exit(multiseed_main(sys.argv[2:]))
    sys.exit(main(sys.argv[1:]))
