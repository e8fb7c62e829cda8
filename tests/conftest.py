"""Shared pytest setup: import paths, the `gpu` marker, device fixtures.

Tests marked ``gpu`` need a CUDA device and fail (they never skip) when none is
visible, so a GPU run can not pass on a silent CPU path.  Everything else runs
on the CPU and covers the oracle, the host logic and the ABI surface.
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
PKG = ROOT / "n2wos-cuda_b200"
for p in (str(ROOT), str(PKG)):
    if p not in sys.path:
        sys.path.insert(0, p)

GOLDEN = ROOT / "tests" / "golden"


def _reference_bunny() -> Path:
    """The reference's bunny PLY: the copy oracle/build.py stages in oracle/_ref
    (it travels to GPU machines), else the reference checkout's own file."""
    from oracle import build as ob

    return ob.REF_BUNNY if ob.REF_BUNNY.exists() else ob.reference_root() / "meshes" / ob.REF_BUNNY.name


REFERENCE_BUNNY = _reference_bunny()


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); run with -m gpu")


def _ensure_built():
    lib = PKG / "lib" / "libn2w.so"
    sys.path.insert(0, str(PKG))
    import build as pkg_build

    tools = [PKG / "bin" / exe for exe in pkg_build.EXECUTABLES]
    if not lib.exists() or not all(t.exists() for t in tools):
        pkg_build.build()
    orc = ROOT / "oracle" / "liboracle.so"
    if not orc.exists():
        from oracle import build as ob

        ob.build_oracle()


_ensure_built()


@pytest.fixture(scope="session")
def n2w():
    import n2w as mod

    return mod


@pytest.fixture(scope="session")
def gpu(n2w):
    if n2w.device_count() < 1:
        pytest.fail("no CUDA device visible: GPU tests must run on a GPU box")
    return n2w


@pytest.fixture(scope="session")
def bumpy_ref_mesh(n2w):
    """Reference-formula bumpy sphere 128x256, amplitude 0.15, normalised."""
    m = n2w.Mesh.bumpy_sphere_ref(128, 256, 0.15)
    m.normalize()
    return m


@pytest.fixture(scope="session")
def golden_closest():
    return dict(np.load(GOLDEN / "closest_golden.npz"))


def uniform_box(n, extent, seed):
    return np.random.default_rng(seed).uniform(-extent, extent, (n, 3)).astype(np.float32)
