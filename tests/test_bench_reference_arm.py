"""The bench's reference arm builds and walks the headline workload with the
oracle and the reference's own sources only: no module or shared object of
the product is loaded, and its workload is the product's point for point."""
import json
import subprocess
import sys

import numpy as np
import pytest

import oracle
from conftest import ROOT

pytestmark = pytest.mark.skipif(not oracle.ref_available(), reason="oracle/_ref not built (reference sources absent)")

PROBE = r"""
import sys, json
sys.path.insert(0, {root!r})
import numpy as np
import bench
scene = bench.reference_cpu_scene()
bvh, pts, problem = scene
s = bench.reference_cpu_sample((bvh, pts[:64 * bench.REF_SAMPLE_STRIDE], problem), 8, threads=2)
print(json.dumps({{"n2w_modules": sorted(m for m in sys.modules if m == "n2w" or m.startswith("n2w.")),
                   "libs": bench.loaded_libraries(), "points": len(pts), "steps_per_s": s["value"]}}))
np.save({out!r}, pts)
"""


def test_reference_arm_loads_no_product_code(tmp_path, n2w):
    out = tmp_path / "ref_pts.npy"
    r = subprocess.run([sys.executable, "-c", PROBE.format(root=str(ROOT), out=str(out))], capture_output=True,
                       text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    d = json.loads(r.stdout.strip().splitlines()[-1])
    assert d["n2w_modules"] == []
    assert all(lib.startswith("oracle/") for lib in d["libs"]), d["libs"]
    assert d["steps_per_s"] > 0
    # the same interior points as the product's headline slice
    m = n2w.Mesh.icosphere_displaced(6, 0.12, 3.0, 4, 0.5, 12345)
    m.normalize()
    lo, hi = m.bounds()
    grid, _ = n2w.slice_points(lo, hi, "xy", 0.12, 512, 512, 0.02, True)
    ref_pts = np.load(out)
    v, t = m.arrays()
    # inside test on a strided subset with the oracle's brute-force reference rule
    sub = grid[::97]
    inside = oracle.inside_bruteforce(v, t, sub).astype(bool)
    ref_sub = set(map(tuple, ref_pts.tolist()))
    assert all((tuple(p) in ref_sub) == bool(i) for p, i in zip(sub.tolist(), inside))
    assert d["points"] == 170364


def test_reference_arm_other_ranks_exit_without_work():
    """Under torchrun only rank 0 runs the reference arm; the others exit 0
    at once and print nothing."""
    import os

    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--gpus", "2"],
                       capture_output=True, text=True, timeout=120, env=env, cwd=str(ROOT))
    assert r.returncode == 0, r.stderr
    assert r.stdout.strip() == ""
