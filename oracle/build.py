"""ORACLE build recipe — test infrastructure only.

* ``oracle/liboracle.so``: the CPU restatement (oracle.cpp), g++ -O2
  -ffp-contract=off so every float operation rounds like the reference's g++
  build (no FMA contraction).
* ``oracle/_ref/libn2wos_ref.so``: the reference's own CPU sources compiled where
  they lie under the reference checkout (src/mesh/*.cpp,
  src/geometry/closest_point.cpp, src/cuda/bvh_build_host.cpp) plus
  ref_shim.cpp.  Built only when the checkout is present.
* ``oracle/_ref/libn2wos_ref_gpu.so``: the reference's in-tree GPU kernel
  (src/cuda/bvh_query.cu + bvh_build_host.cpp) compiled unmodified for sm_100a,
  plus ref_gpu_shim.cu.
* ``oracle/_ref/meshes/bunny_zipper_wataertight.ply``: a copy of the reference's
  bundled bunny mesh (data the GPU checks load where the checkout is absent).

The reference checkout is located by ``reference_root()``: the environment
variable N2W_REFERENCE_ROOT when set, else the checkout's default location.
Everything under oracle/_ref is a build output: never committed, but it travels
with the repository snapshot to GPU machines.

The reference's cuBQL / tiny-cuda-nn targets are not buildable (those
third-party sources are not vendored), so they are not attempted.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
REF_OUT = HERE / "_ref"
DEFAULT_REFERENCE_ROOT = "/root/reference"
REF_BUNNY = REF_OUT / "meshes" / "bunny_zipper_wataertight.ply"


def reference_root() -> Path:
    """The reference checkout: $N2W_REFERENCE_ROOT, else the default location."""
    return Path(os.environ.get("N2W_REFERENCE_ROOT", DEFAULT_REFERENCE_ROOT))
CUDA_HOME = Path(os.environ.get("CUDA_HOME", "/usr/local/cuda"))

REF_CPU_SOURCES = ["src/mesh/normalize.cpp", "src/mesh/ply_loader.cpp", "src/mesh/obj_loader.cpp",
                   "src/mesh/procedural_bumpy_sphere.cpp", "src/geometry/closest_point.cpp",
                   "src/cuda/bvh_build_host.cpp"]


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"oracle build failed: {' '.join(map(str, cmd))}\n{r.stdout}\n{r.stderr}")


def _stale(target: Path, sources) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(Path(s).stat().st_mtime > t for s in sources)


def build_oracle() -> Path:
    out = HERE / "liboracle.so"
    src = HERE / "oracle.cpp"
    if _stale(out, [src]):
        _run(["g++", "-O2", "-ffp-contract=off", "-fPIC", "-shared", "-std=c++17", "-pthread",
              str(src), "-o", str(out)])
    return out


def build_ref() -> list[Path]:
    """Builds oracle/_ref from the reference sources when they are present."""
    REFERENCE = reference_root()
    if not (REFERENCE / "src").is_dir():
        return []
    REF_OUT.mkdir(exist_ok=True)
    bunny = REFERENCE / "meshes" / REF_BUNNY.name
    if bunny.exists() and _stale(REF_BUNNY, [bunny]):
        REF_BUNNY.parent.mkdir(exist_ok=True)
        shutil.copyfile(bunny, REF_BUNNY)
    inc = [f"-I{REFERENCE / 'include'}", f"-I{REFERENCE / 'src' / 'cuda'}", f"-I{CUDA_HOME / 'include'}"]
    built = []
    cpu = REF_OUT / "libn2wos_ref.so"
    srcs = [REFERENCE / s for s in REF_CPU_SOURCES] + [HERE / "ref_shim.cpp"]
    if _stale(cpu, srcs):
        _run(["g++", "-O2", "-fPIC", "-shared", "-std=c++17"] + inc + [str(s) for s in srcs] + ["-o", str(cpu)])
    built.append(cpu)
    gpu = REF_OUT / "libn2wos_ref_gpu.so"
    gsrcs = [REFERENCE / "src/cuda/bvh_query.cu", REFERENCE / "src/cuda/bvh_build_host.cpp",
             HERE / "ref_gpu_shim.cu"]
    if _stale(gpu, gsrcs):
        objs = []
        for s in gsrcs:
            o = REF_OUT / (s.name + ".o")
            _run([str(CUDA_HOME / "bin" / "nvcc"), "-gencode", "arch=compute_100a,code=sm_100a", "-O3",
                  "-std=c++17", "-Xcompiler", "-fPIC", "-x", "cu" if s.suffix == ".cu" else "c++"] + inc +
                 ["-c", str(s), "-o", str(o)])
            objs.append(o)
        _run([str(CUDA_HOME / "bin" / "nvcc"), "-gencode", "arch=compute_100a,code=sm_100a", "-shared",
              "-o", str(gpu)] + [str(o) for o in objs] + ["-lcudart"])
    built.append(gpu)
    return built


def build() -> None:
    build_oracle()
    build_ref()


if __name__ == "__main__":
    build()
    print("oracle built:", HERE / "liboracle.so", [str(p) for p in REF_OUT.glob("*.so")])
    sys.exit(0)
