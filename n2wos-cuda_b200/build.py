"""Build recipe for libn2w.so and the CLI executables (sm_100a only).

Run ``python n2wos-cuda_b200/build.py`` (or ``__graft_entry__.build()``).
Objects go to ``n2wos-cuda_b200/_build/``; the shared library to
``n2wos-cuda_b200/lib/libn2w.so``; executables to ``n2wos-cuda_b200/bin/``.
Rebuilds are incremental on file modification times (any header change
rebuilds everything).
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
TOOLS = PKG / "tools"
BUILD = PKG / "_build"
LIB = PKG / "lib"
BIN = PKG / "bin"
INCLUDE = ROOT / "include"
CUDA_HOME = Path(os.environ.get("CUDA_HOME", "/usr/local/cuda"))
NVCC = str(CUDA_HOME / "bin" / "nvcc")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + [
    "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-O2",
    "--expt-relaxed-constexpr", f"-I{INCLUDE}", f"-I{CSRC}",
]
CXX_FLAGS = ["-O2", "-fPIC", "-std=c++17", "-ffp-contract=off", f"-I{INCLUDE}", f"-I{CSRC}",
             f"-I{CUDA_HOME / 'include'}"]

LIB_CU = ["closest_point.cu", "walker.cu", "cache.cu", "nc.cu", "util.cu", "batch.cu", "server.cu", "probe.cu", "comm.cu"]
LIB_CPP = ["mesh.cpp", "bvh_build.cpp", "capi.cpp"]
EXECUTABLES = {
    "n2wos_probe_cuda_bvh": ["probe_cuda_bvh.cpp"],
    "n2wos_probe_geometry_backends": ["probe_geometry_backends.cpp"],
    "n2wos_eval_wavefront_wos": ["eval_wavefront_wos.cpp"],
    "n2wos_eval_tcnn_nc_wos": ["eval_tcnn_nc_wos.cpp"],
    "n2wos_probe_tcnn_cache": ["probe_tcnn_cache.cpp"],
    "n2wos_render_harmonic_slice": ["render_harmonic_slice.cpp"],
}


def _headers() -> list[Path]:
    hs = list(CSRC.glob("*.h")) + list(CSRC.glob("*.hpp")) + list(CSRC.glob("*.cuh"))
    hs += list(INCLUDE.glob("*.h")) + list(INCLUDE.glob("*.hpp")) + list(TOOLS.glob("*.hpp"))
    return hs


def _stale(target: Path, sources: list[Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(s.stat().st_mtime > t for s in sources)


def _run(cmd: list[str]) -> None:
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"build step failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")


def _compile(src: Path, obj: Path, headers: list[Path]) -> Path:
    if _stale(obj, [src] + headers):
        if src.suffix == ".cu":
            _run([NVCC] + NVCC_FLAGS + ["-c", str(src), "-o", str(obj)])
        else:
            _run(["g++"] + CXX_FLAGS + ["-c", str(src), "-o", str(obj)])
    return obj


def build(verbose: bool = False, jobs: int | None = None) -> Path:
    BUILD.mkdir(exist_ok=True)
    LIB.mkdir(exist_ok=True)
    BIN.mkdir(exist_ok=True)
    headers = _headers()
    srcs = [CSRC / s for s in LIB_CU + LIB_CPP]
    tool_srcs = sorted({s for v in EXECUTABLES.values() for s in v})
    jobs = jobs or max(2, min(8, os.cpu_count() or 2))
    with cf.ThreadPoolExecutor(jobs) as ex:
        futs = [ex.submit(_compile, s, BUILD / (s.name + ".o"), headers) for s in srcs]
        tfuts = [ex.submit(_compile, TOOLS / s, BUILD / ("tool_" + s + ".o"), headers)
                 for s in tool_srcs if (TOOLS / s).exists()]
        objs = [f.result() for f in futs]
        tobjs = {Path(f.result()).name: f.result() for f in tfuts}
    so = LIB / "libn2w.so"
    if _stale(so, objs):
        _run([NVCC] + ARCH + ["-shared", "-o", str(so)] + [str(o) for o in objs] + ["-lcudart", "-lnccl"])
        if verbose:
            print(f"linked {so}")
    for exe, parts in EXECUTABLES.items():
        pobjs = [tobjs.get("tool_" + p + ".o") for p in parts]
        if any(o is None for o in pobjs):
            continue
        out = BIN / exe
        if _stale(out, pobjs + [so]):
            _run(["g++", "-o", str(out)] + [str(o) for o in pobjs] +
                 [f"-L{LIB}", "-ln2w", f"-Wl,-rpath,$ORIGIN/../lib", f"-L{CUDA_HOME / 'lib64'}",
                  "-lcudart", "-lpthread"])
    return so


if __name__ == "__main__":
    p = build(verbose=True)
    print(p)
    sys.exit(0)
