"""The allocation-free walker entry point, n2w_wos_estimate_noalloc.

It serves callers that may not allocate device memory while they solve (an
application that gives the library a fixed share of HBM and forbids other
allocations, or a serving loop that must keep cudaMalloc off its request path).
Its scratch is a static device array, so its results must equal those of the
ordinary entry point, n2w_wos_estimate, which allocates its workspace: the same
Philox streams give the same walks, and the per-point FP64 sums can differ only
in the order of their atomic additions (relative tolerance 1e-9 below).  Two
calls in a row check that the shared array is re-initialised between calls.
Kept in its own file, collected last, so a failure here comes after every
other test has run.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

RTOL = 1e-9


def test_noalloc_matches_allocating_entry_point_on_two_calls(gpu):
    from n2w._lib import call, lib

    mesh = gpu.Mesh.bumpy_sphere_trig(32, 64, 0.08, 6, 8)
    mesh.normalize()
    bvh = gpu.Bvh(mesh, 4, "sah")
    rng = np.random.default_rng(11)
    pts = rng.uniform(-0.5, 0.5, (3000, 3)).astype(np.float32)
    problem = gpu.problem_charges_seeded(8, 1.6, 2.0, 12345)
    opts = gpu.walk_options(walks_per_point=256, epsilon=1e-3, seed=42)
    want, _ = gpu.wos_estimate(bvh, problem, pts, options=opts)  # allocates its workspace

    n = len(pts)
    d_pts = gpu.DeviceBuffer.from_array(pts)
    stats = gpu.PointStatsBuffers.allocate(n)
    counters = gpu.DeviceBuffer(C.sizeof(gpu._lib.WalkCounters))
    for _ in range(2):
        call("n2w_wos_estimate_noalloc", bvh.handle, C.byref(problem), d_pts.ptr, n, C.byref(opts),
             stats.struct(), counters.ptr, None)
        call("n2w_device_sync")
        got = stats.download()
        assert np.array_equal(got["count"], want["count"])
        assert np.allclose(got["sum"], want["sum"], rtol=RTOL, atol=1e-12)
        assert np.allclose(got["sum_sq"], want["sum_sq"], rtol=RTOL, atol=1e-12)
        assert np.array_equal(got["mean_steps"], want["mean_steps"])
        walks = counters.download(np.uint64, 8)[0]
        assert walks == 256 * n


def test_noalloc_rejects_sizes_beyond_its_scratch(gpu):
    from n2w._lib import lib

    mesh = gpu.Mesh.bumpy_sphere_trig(16, 32, 0.08, 6, 8)
    mesh.normalize()
    bvh = gpu.Bvh(mesh, 4, "sah")
    problem = gpu.problem_charges_seeded()
    opts = gpu.walk_options(walks_per_point=4)
    stats = gpu.PointStatsBuffers.allocate(1)
    d = gpu.DeviceBuffer(16)
    limit = (4 << 20) - 512
    too_many = limit // 24 + 1
    st = lib.n2w_wos_estimate_noalloc(bvh.handle, C.byref(problem), d.ptr, too_many, C.byref(opts),
                                      stats.struct(), None, None)
    assert st == 1
    assert b"exceed the limit" in lib.n2w_last_error()


def test_noalloc_at_its_maximum_size(gpu):
    """Exactly N2W_NOALLOC_MAX_POINTS points (the scratch's 512 + 24 n bytes
    fill the 4 MiB array) with a few walks each: the same counts and steps as
    the allocating entry point."""
    from n2w._lib import call

    limit = ((4 << 20) - 512) // 24
    mesh = gpu.Mesh.bumpy_sphere_trig(32, 64, 0.08, 6, 8)
    mesh.normalize()
    bvh = gpu.Bvh(mesh, 4, "sah")
    pts = np.random.default_rng(5).uniform(-0.4, 0.4, (limit, 3)).astype(np.float32)
    problem = gpu.problem_charges_seeded(8, 1.6, 2.0, 12345)
    opts = gpu.walk_options(walks_per_point=4, epsilon=1e-3, seed=9)
    want, _ = gpu.wos_estimate(bvh, problem, pts, options=opts)
    d_pts = gpu.DeviceBuffer.from_array(pts)
    stats = gpu.PointStatsBuffers.allocate(limit)
    call("n2w_wos_estimate_noalloc", bvh.handle, C.byref(problem), d_pts.ptr, limit, C.byref(opts),
         stats.struct(), None, None)
    call("n2w_device_sync")
    got = stats.download()
    assert np.array_equal(got["count"], want["count"]) and (got["count"] == 4).all()
    assert np.array_equal(got["mean_steps"], want["mean_steps"])
    assert np.allclose(got["sum"], want["sum"], rtol=RTOL, atol=1e-12)
