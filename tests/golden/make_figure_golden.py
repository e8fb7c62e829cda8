"""Generates tests/golden/figure_runs.json and tests/golden/figure_masks.npz
from the reference's two published evaluation runs.

The reference commits the JSON result and the slice mask of two runs of its
own n2wos_eval_tcnn_nc_wos (RTX 3070, cuBQL SAH leaf 8, tiny-cuda-nn):

* figures/zebra_k8_m2.json + figures/zebra_k8_m2_slice_mask.ppm — its bumpy
  sphere (128 x 256, amplitude 0.15), boundary harmonic_zebra_k8, z = 0 slice
  512 x 512, eps = 1e-4, 64 pure walks per pixel;
* figures/bunny_zebra_k8_m2.json + figures/bunny_zebra_k8_m2_slice_mask.ppm —
  the bundled bunny PLY, z = 0.12 slice, same settings.

Kept: each run's command line, mesh_stats, bvh_stats, slice_eval and the
runs.* statistics (pure_wos in full; nc_wos / nc_2lmc RMSE and timings), and
each mask as packed bits (1 = interior pixel, row 0 = the PPM's first row).

    python tests/golden/make_figure_golden.py    (needs the reference checkout)
"""
from __future__ import annotations

import json
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT))

from oracle import build as ob  # noqa: E402

RUNS = ("zebra_k8_m2", "bunny_zebra_k8_m2")
MASK_INSIDE, MASK_OUTSIDE = 235, 20  # grey levels of the reference's mask PPM


def read_mask(path: Path) -> np.ndarray:
    raw = path.read_bytes()
    magic, dims, maxval, body = raw.split(b"\n", 3)
    if magic != b"P6" or maxval != b"255":
        raise SystemExit(f"{path}: not an 8-bit P6 PPM")
    w, h = map(int, dims.split())
    rgb = np.frombuffer(body, np.uint8).reshape(h, w, 3)
    if not (np.all(rgb == rgb[..., :1]) and np.isin(rgb, (MASK_INSIDE, MASK_OUTSIDE)).all()):
        raise SystemExit(f"{path}: unexpected mask colours")
    return rgb[..., 0] == MASK_INSIDE


def main() -> None:
    figs = ob.reference_root() / "figures"
    if not figs.is_dir():
        raise SystemExit(f"reference figures not found under {figs}")
    out, masks = {}, {}
    for name in RUNS:
        d = json.loads((figs / f"{name}.json").read_text())
        runs = d["runs"]
        keep_runs = {"pure_wos": runs["pure_wos"]}
        for k in ("nc_wos", "nc_2lmc"):
            keep_runs[k] = {kk: runs[k][kk] for kk in ("rmse", "elapsed_ms") if kk in runs[k]}
        out[name] = {"command_line": d["command_line"], "options": d["options"], "mesh_stats": d["mesh_stats"],
                     "bvh_stats": d["bvh_stats"], "slice_eval": d["slice_eval"], "runs": keep_runs,
                     "training": d.get("training"), "device": d.get("cuda", {}).get("device")}
        m = read_mask(figs / f"{name}_slice_mask.ppm")
        if int(m.sum()) != d["slice_eval"]["inside_pixels"]:
            raise SystemExit(f"{name}: mask count {int(m.sum())} != inside_pixels")
        masks[name] = np.packbits(m.reshape(-1))
        masks[name + "_shape"] = np.array(m.shape, np.int32)
    (HERE / "figure_runs.json").write_text(json.dumps(out, indent=1, sort_keys=True) + "\n")
    np.savez_compressed(HERE / "figure_masks.npz", **masks)
    print("wrote", HERE / "figure_runs.json", HERE / "figure_masks.npz")


if __name__ == "__main__":
    main()
