"""Per-sample, NC prefix / 2LMC continuation, combine and label-update paths
against the oracle's restatement of the reference kernels (8 seeds).

Reference kernels (src/cuda/cubql_bvh.cu) and the product entry points:
  nc_pure_wos_samples_kernel       1422-1449  n2w_wos_pure_samples
  nc_hybrid_prefix_kernel          1451-1516  n2w_wos_prefix_samples(PREFIX)
  nc_2lmc_prefix_continue_kernel   1519-1606  n2w_wos_prefix_samples(RESIDUAL)
  nc_combine_cache_and_residual    1608-1627  n2w_wos_combine
  nc_update_labels_kernel          1372-1420  n2w_nc_update_labels
Statistics pooled over 8 seeds agree within 3 sigma of the combined Monte
Carlo error (walks differ between the two only by the few-ulp distances of
the walker's contracted arithmetic, so the tests are distributional); the
combine kernel is deterministic and is compared bit for bit.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu

W = 256
SEEDS = range(1, 9)
EPS = 1e-3
IN_MIN = np.full(3, -1.1, np.float32)
IN_EXT = np.full(3, 2.2, np.float32)


def key_words(seed, tag=0):
    k0 = (seed & 0xFFFFFFFF) ^ ((tag * 0x85EBCA6B) & 0xFFFFFFFF)
    k1 = (seed >> 32) ^ ((tag * 0xC2B2AE35) & 0xFFFFFFFF)
    return k0, k1


@pytest.fixture(scope="module")
def scene(gpu):
    m = gpu.Mesh.bumpy_sphere_trig(32, 64, 0.08, 6, 8)
    m.normalize()
    bvh = gpu.Bvh(m, 4, "sah")
    nodes, tris = bvh.layout()
    pts = np.array([[0.0, 0.0, 0.0], [0.3, -0.2, 0.1], [-0.5, 0.2, -0.3], [0.1, 0.6, 0.2],
                    [0.7, 0.1, -0.1], [-0.2, -0.7, 0.05]], np.float32)
    return bvh, nodes, tris, pts


def problems(gpu):
    ball = gpu.problem_sinprod(3.0 * np.pi, gpu.N2W_SOURCE_BALL)
    center = gpu.problem_sinprod(3.0 * np.pi, gpu.N2W_SOURCE_CENTER)
    return {"sinprod_ball": ball, "sinprod_center": center, "zebra_k8": gpu.problem_from_name("harmonic_zebra_k8")}


def gpu_samples(gpu, bvh, p, pts, seed, mode, depth_m):
    """Per-sample arrays from the CUDA walker (mode 0 pure, 1 prefix, 2 residual)."""
    from n2w._lib import call
    n = len(pts)
    S = n * W
    dp = gpu.DeviceBuffer.from_array(pts)
    o = gpu.walk_options(walks_per_point=W, epsilon=EPS, seed=seed, depth_m=depth_m)
    st, fo, ov = (gpu.DeviceBuffer(4 * S) for _ in range(3))
    if mode == oracle.MODE_PURE:
        val = gpu.DeviceBuffer(4 * S)
        call("n2w_wos_pure_samples", bvh.handle, C.byref(p), dp.ptr, n, C.byref(o), val.ptr, st.ptr, fo.ptr, ov.ptr,
             None)
        call("n2w_device_sync")
        return {"value": val.download(np.float32), "steps": st.download(np.int32), "forced": fo.download(np.int32),
                "overflow": ov.download(np.int32)}
    inp, bnd, cont = gpu.DeviceBuffer(12 * S), gpu.DeviceBuffer(4 * S), gpu.DeviceBuffer(4 * S)
    needs = gpu.DeviceBuffer(S)
    call("n2w_wos_prefix_samples", bvh.handle, C.byref(p), dp.ptr, n, C.byref(o), mode,
         IN_MIN.ctypes.data_as(C.c_void_p), IN_EXT.ctypes.data_as(C.c_void_p), inp.ptr, bnd.ptr,
         cont.ptr if mode == oracle.MODE_RESIDUAL else None, needs.ptr, st.ptr, fo.ptr, ov.ptr, None)
    call("n2w_device_sync")
    out = {"value": bnd.download(np.float32), "inputs": inp.download(np.float32).reshape(S, 3),
           "needs_cache": needs.download(np.uint8), "steps": st.download(np.int32), "forced": fo.download(np.int32),
           "overflow": ov.download(np.int32)}
    if mode == oracle.MODE_RESIDUAL:
        out["continuation"] = cont.download(np.float32)
    return out


def oracle_samples(nodes, tris, p, pts, seed, mode, depth_m):
    return oracle.walk_samples(nodes, tris, bytes(p), pts, W, mode, depth_m, 256, EPS, 0.999, *key_words(seed, mode),
                               IN_MIN, IN_EXT)


def per_point(x, n):
    """Per-point mean and variance of a per-sample quantity (sample i*W + j)."""
    x = np.asarray(x, np.float64).reshape(n, W)
    return x.mean(1), x.var(1, ddof=1)


def assert_pooled_close(gm, gv, om, ov, what):
    """gm/om: [seeds, points] means; gv/ov: per-sample variances."""
    gm, gv, om, ov = map(np.asarray, (gm, gv, om, ov))
    k = len(gm)
    diff = gm.mean(0) - om.mean(0)
    sigma = np.sqrt(gv.mean(0) / (W * k) + ov.mean(0) / (W * k))
    ok = np.abs(diff) <= 3 * sigma + 1e-7
    assert ok.all(), f"{what}: diff {diff[~ok]} sigma {sigma[~ok]}"


@pytest.mark.parametrize("name", ["sinprod_ball", "zebra_k8"])
def test_pure_samples_match_oracle(gpu, scene, name):
    bvh, nodes, tris, pts = scene
    p = problems(gpu)[name]
    n = len(pts)
    acc = {k: [] for k in ("gv", "gvv", "ov", "ovv", "gs", "gsv", "os", "osv")}
    for seed in SEEDS:
        g = gpu_samples(gpu, bvh, p, pts, seed, oracle.MODE_PURE, 0)
        o = oracle_samples(nodes, tris, p, pts, seed, oracle.MODE_PURE, 0)
        assert g["overflow"].sum() == 0 and g["forced"].sum() == o["forced"].sum() == 0
        for pre, src in (("g", g), ("o", o)):
            m, v = per_point(src["value"], n)
            acc[pre + "v"].append(m)
            acc[pre + "vv"].append(v)
            m, v = per_point(src["steps"], n)
            acc[pre + "s"].append(m)
            acc[pre + "sv"].append(v)
    assert_pooled_close(acc["gv"], acc["gvv"], acc["ov"], acc["ovv"], "walk value")
    assert_pooled_close(acc["gs"], acc["gsv"], acc["os"], acc["osv"], "steps per walk")


@pytest.mark.parametrize("name", ["sinprod_center", "sinprod_ball", "zebra_k8"])
@pytest.mark.parametrize("depth_m", [1, 4])
def test_prefix_samples_match_oracle(gpu, scene, name, depth_m):
    bvh, nodes, tris, pts = scene
    p = problems(gpu)[name]
    n = len(pts)
    qs = {k: ([], [], [], []) for k in ("A", "needs", "x", "y", "z")}
    for seed in SEEDS:
        g = gpu_samples(gpu, bvh, p, pts, seed, oracle.MODE_PREFIX, depth_m)
        o = oracle_samples(nodes, tris, p, pts, seed, oracle.MODE_PREFIX, depth_m)
        for src, (im, iv) in ((g, (0, 1)), (o, (2, 3))):
            needs = src["needs_cache"].astype(bool)
            # walks that need the cache stopped exactly at depth m; the others
            # reached the epsilon shell at or before it (the shell test comes first)
            assert (src["steps"][needs] == depth_m).all() and (src["steps"][~needs] <= depth_m).all()
            assert ((src["inputs"] >= 0) & (src["inputs"] <= 1)).all()
            for key, arr in (("A", src["value"]), ("needs", needs.astype(np.float64)), ("x", src["inputs"][:, 0]),
                             ("y", src["inputs"][:, 1]), ("z", src["inputs"][:, 2])):
                m, v = per_point(arr, n)
                qs[key][im].append(m)
                qs[key][iv].append(v)
    for key, (gm, gv, om, ov) in qs.items():
        assert_pooled_close(gm, gv, om, ov, f"prefix {key}")


@pytest.mark.parametrize("name", ["sinprod_ball", "zebra_k8"])
def test_two_level_estimate_matches_oracle_with_analytic_cache(gpu, scene, name):
    """Coarse = prefix + C(X_m), residual = continuation - C(X_m) with C the exact
    solution; the combine kernel equals the restated one bit for bit, and the
    two-level estimate per point matches the oracle's and the exact value."""
    from n2w._lib import call
    bvh, nodes, tris, pts = scene
    p = problems(gpu)[name]
    n, S, m = len(pts), len(pts) * W, 2
    lo, ext = IN_MIN.astype(np.float64), IN_EXT.astype(np.float64)
    est = {"g": [], "gv": [], "o": [], "ov": []}
    for seed in SEEDS:
        parts = {}
        for who in ("g", "o"):
            coarse = (gpu_samples if who == "g" else None)
            if who == "g":
                c = gpu_samples(gpu, bvh, p, pts, seed, oracle.MODE_PREFIX, m)
                r = gpu_samples(gpu, bvh, p, pts, seed, oracle.MODE_RESIDUAL, m)
            else:
                c = oracle_samples(nodes, tris, p, pts, seed, oracle.MODE_PREFIX, m)
                r = oracle_samples(nodes, tris, p, pts, seed, oracle.MODE_RESIDUAL, m)
            del coarse
            cache_c = gpu.problem_exact(p, lo + c["inputs"].astype(np.float64) * ext).astype(np.float32)
            cache_r = gpu.problem_exact(p, lo + r["inputs"].astype(np.float64) * ext).astype(np.float32)
            if who == "g":
                # the product's combine kernel on these arrays, against the restatement
                outs = {}
                for tag, smp, cache in (("c", c, cache_c), ("r", r, cache_r)):
                    cont = smp.get("continuation", smp["value"])
                    bufs = [gpu.DeviceBuffer.from_array(np.ascontiguousarray(a)) for a in
                            (cache, smp["value"], cont, smp["needs_cache"])]
                    d_nc, d_res = gpu.DeviceBuffer(4 * S), gpu.DeviceBuffer(4 * S)
                    call("n2w_wos_combine", *[b.ptr for b in bufs], S, d_nc.ptr, d_res.ptr, 256, None)
                    call("n2w_device_sync")
                    got = (d_nc.download(np.float32), d_res.download(np.float32))
                    want = oracle.nc_combine(cache, smp["value"], cont, smp["needs_cache"])
                    assert np.array_equal(got[0].view(np.uint32), want[0].view(np.uint32))
                    assert np.array_equal(got[1].view(np.uint32), want[1].view(np.uint32))
                    outs[tag] = got
                nc_vals, res_vals = outs["c"][0], outs["r"][1]
            else:
                nc_vals, _ = oracle.nc_combine(cache_c, c["value"], c["value"], c["needs_cache"])
                _, res_vals = oracle.nc_combine(cache_r, r["value"], r["continuation"], r["needs_cache"])
            mc, vc = per_point(nc_vals, n)
            mr, vr = per_point(res_vals, n)
            parts[who] = (mc + mr, vc + vr)
        est["g"].append(parts["g"][0]); est["gv"].append(parts["g"][1])
        est["o"].append(parts["o"][0]); est["ov"].append(parts["o"][1])
    assert_pooled_close(est["g"], est["gv"], est["o"], est["ov"], "two-level estimate")
    exact = gpu.problem_exact(p, pts.astype(np.float64))
    g = np.array(est["g"]).mean(0)
    sig = np.sqrt(np.array(est["gv"]).mean(0) / (W * len(SEEDS)))
    assert np.all(np.abs(g - exact) <= 3 * sig + 5e-3), (g, exact, sig)


def test_label_update_matches_oracle(gpu, scene):
    """Two refreshes of WoS labels: counts are exact, inputs bit-equal, running
    targets agree with the oracle's within 3 sigma (8 seeds); exact labels equal
    the solution."""
    from n2w._lib import call
    bvh, nodes, tris, pts = scene
    p = gpu.problem_charges_seeded(8, 1.6, 2.0, 12345)
    n = len(pts)
    dp = gpu.DeviceBuffer.from_array(pts)
    Wl = 64
    gt, ot, gvar = [], [], []
    for seed in SEEDS:
        acc = gpu.PointStatsBuffers.allocate(n)
        acc.zero()  # the running accumulators start at zero before refresh 0
        d_in, d_tg = gpu.DeviceBuffer(12 * n), gpu.DeviceBuffer(4 * n)
        otg, ocnt = np.zeros(n, np.float32), np.zeros(n, np.int32)
        for refresh in range(2):
            lo = gpu.label_options(walks_per_point=Wl, epsilon=EPS, seed=seed, refresh_index=refresh,
                                   input_min=IN_MIN, input_extent=IN_EXT)
            call("n2w_nc_update_labels", bvh.handle, C.byref(p), dp.ptr, n, C.byref(lo), acc.struct(), d_in.ptr,
                 d_tg.ptr, None, None)
            wseed = (seed + 0x9E3779B97F4A7C15 * (refresh + 1)) & 0xFFFFFFFFFFFFFFFF
            oin = oracle.nc_update_labels(nodes, tris, bytes(p), pts, Wl, 256, EPS, 0.999, *key_words(wseed), 1,
                                          IN_MIN, IN_EXT, otg, ocnt)
        call("n2w_device_sync")
        r = acc.download()
        assert (r["count"] == 2 * Wl).all() and (ocnt == 2 * Wl).all()
        assert np.array_equal(d_in.download(np.float32).reshape(n, 3), oin)
        gt.append(d_tg.download(np.float32))
        ot.append(otg.copy())
        gvar.append(r["sample_variance"])
    gt, ot, gvar = map(np.array, (gt, ot, gvar))
    diff = gt.mean(0) - ot.mean(0)
    sigma = np.sqrt(2 * gvar.mean(0) / (2 * Wl * len(SEEDS)))
    assert np.all(np.abs(diff) <= 3 * sigma), (diff, sigma)
    # exact labels
    lo = gpu.label_options(walks_per_point=1, epsilon=EPS, seed=1, refresh_index=0, input_min=IN_MIN,
                           input_extent=IN_EXT, label_source=0)
    d_in, d_tg = gpu.DeviceBuffer(12 * n), gpu.DeviceBuffer(4 * n)
    call("n2w_nc_update_labels", bvh.handle, C.byref(p), dp.ptr, n, C.byref(lo), gpu.PointStatsBuffers.allocate(n)
         .struct(), d_in.ptr, d_tg.ptr, None, None)
    call("n2w_device_sync")
    otg, ocnt = np.zeros(n, np.float32), np.zeros(n, np.int32)
    oracle.nc_update_labels(nodes, tris, bytes(p), pts, 1, 256, EPS, 0.999, 0, 0, 0, IN_MIN, IN_EXT, otg, ocnt)
    np.testing.assert_allclose(d_tg.download(np.float32), otg, rtol=2e-6, atol=1e-6)
