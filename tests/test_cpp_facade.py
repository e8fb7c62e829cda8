"""The C++ facade (include/n2w.hpp): the reference's class shapes over the C
ABI, with failures rethrown as std::runtime_error like the reference's
N2WOS_CUDA_CHECK (src/cuda/bvh_query.cu:16-23).  A small program is compiled
against the header and libn2w.so; the CPU test covers mesh calls and the error
path, the GPU test the device-pointer query against the host brute force."""
import subprocess

import pytest

from conftest import PKG, ROOT

PROGRAM = r"""
#define N2W_PROVIDE_N2WOS_NAMESPACE
#include "n2w.hpp"
#include <cstdio>
#include <random>
#include <vector>

int main(int argc, char** argv) {
  const bool gpu = argc > 1;
  n2wos::Mesh mesh = n2wos::make_procedural_bumpy_sphere(128, 256, 0.15f);
  const n2wos::NormalizeTransform tr = n2wos::normalize_to_unit_radius(mesh);
  std::printf("triangles %zu vertices %zu scale %.9g\n", mesh.triangle_count(), mesh.vertex_count(), tr.scale);
  try {
    n2wos::make_procedural_bumpy_sphere(2, 8, 0.1f);
    std::printf("no exception\n");
    return 1;
  } catch (const std::runtime_error& e) {
    std::printf("caught: %s\n", e.what());
  }
  if (!gpu) {
    try {
      n2wos::CudaBvh bvh(mesh, 8);
      std::printf("bvh built without a device\n");
    } catch (const std::runtime_error& e) {
      std::printf("caught: %s\n", e.what());
    }
    return 0;
  }
  n2wos::CuBqlBvh bvh(mesh, 4, "sah");
  const int n = 4096;
  std::vector<float> pts(3 * n);
  std::mt19937 rng(12345);
  std::uniform_real_distribution<float> u(-1.2f, 1.2f);
  for (float& x : pts) x = u(rng);
  void *dp, *dd, *dc, *di, *dov;
  N2W_CPP_CHECK(n2w_malloc(&dp, 12 * n));
  N2W_CPP_CHECK(n2w_malloc(&dd, 4 * n));
  N2W_CPP_CHECK(n2w_malloc(&dc, 12 * n));
  N2W_CPP_CHECK(n2w_malloc(&di, 4 * n));
  N2W_CPP_CHECK(n2w_malloc(&dov, 4 * n));
  N2W_CPP_CHECK(n2w_memcpy_h2d(dp, pts.data(), 12 * n, nullptr));
  bvh.query_device(static_cast<const n2wos::DeviceVec3*>(dp), n, static_cast<float*>(dd),
                   static_cast<n2wos::DeviceVec3*>(dc), static_cast<int*>(di), static_cast<int*>(dov));
  std::vector<float> d2(n), want_d2(n);
  std::vector<int> id(n), want_id(n);
  N2W_CPP_CHECK(n2w_memcpy_d2h(d2.data(), dd, 4 * n, nullptr));
  N2W_CPP_CHECK(n2w_memcpy_d2h(id.data(), di, 4 * n, nullptr));
  N2W_CPP_CHECK(n2w_stream_sync(nullptr));
  N2W_CPP_CHECK(n2w_mesh_closest_point_host(mesh.handle(), pts.data(), n, want_d2.data(), nullptr,
                                            want_id.data(), 0));
  int bad = 0;
  for (int i = 0; i < n; ++i) bad += (d2[i] != want_d2[i] || id[i] != want_id[i]);
  std::printf("queries %d mismatches %d nodes %zu\n", n, bad, bvh.node_count());
  try {
    bvh.query_device(nullptr, n, static_cast<float*>(dd), static_cast<n2wos::DeviceVec3*>(dc),
                     static_cast<int*>(di), static_cast<int*>(dov));
  } catch (const std::runtime_error& e) {
    std::printf("caught: %s\n", e.what());
  }
  for (void* p : {dp, dd, dc, di, dov}) N2W_CPP_CHECK(n2w_free(p));
  return bad == 0 ? 0 : 2;
}
"""


@pytest.fixture(scope="module")
def facade_exe(tmp_path_factory):
    d = tmp_path_factory.mktemp("facade")
    src = d / "facade.cpp"
    src.write_text(PROGRAM)
    exe = d / "facade"
    lib = PKG / "lib"
    r = subprocess.run(["g++", "-std=c++17", "-O1", "-Wall", "-Wextra", f"-I{ROOT / 'include'}", str(src), "-o",
                        str(exe), f"-L{lib}", "-ln2w", f"-Wl,-rpath,{lib}"], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


def test_facade_mesh_calls_and_error_path(facade_exe):
    r = subprocess.run([str(facade_exe)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    lines = r.stdout.splitlines()
    assert lines[0].startswith("triangles 65024 vertices 32514")
    assert lines[1].startswith("caught: n2w error 1 in n2w_mesh_bumpy_sphere_ref") and "stacks >= 4" in lines[1]


@pytest.mark.gpu
def test_facade_query_device_matches_bruteforce(facade_exe, gpu):
    r = subprocess.run([str(facade_exe), "gpu"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "queries 4096 mismatches 0" in r.stdout
    assert "caught: n2w error 1 in n2w_bvh_query_device" in r.stdout
