/*
 * n2w.hpp — header-only C++ facade over the C ABI (n2w.h), in the shape of the
 * reference's C++ API so a caller of n2wos::CudaBvh / n2wos::CuBqlBvh
 * (include/n2wos/cuda_bvh.hpp:34-79, include/n2wos/cubql_bvh.hpp:29-70) and of
 * the mesh functions (include/n2wos/mesh.hpp:9-19) can switch by changing the
 * include and the namespace.
 *
 * Errors: every failing C call is rethrown as std::runtime_error carrying
 * "n2w error <status> in <call>: <n2w_last_error()>", the way the reference's
 * N2WOS_CUDA_CHECK turns CUDA errors into std::runtime_error
 * (src/cuda/bvh_query.cu:16-23).  Asynchronous kernel faults surface at the
 * next checked call, as in the reference.
 *
 * Ownership follows the reference: Mesh is a value-like host object, the BVH
 * classes own their device arrays (move-only), query_device takes caller-owned
 * device pointers and neither allocates nor copies to or from the host.
 *
 * To keep the reference's spelling, a translation unit may define
 * N2W_PROVIDE_N2WOS_NAMESPACE before including this header: the classes then
 * also appear as n2wos::Mesh, n2wos::CudaBvh, n2wos::CuBqlBvh, ...
 */
#ifndef N2W_HPP_
#define N2W_HPP_

#include <cstddef>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "n2w.h"

namespace n2w {

using DeviceVec3 = n2w_vec3;

struct Vec3f {
  float x = 0.0f, y = 0.0f, z = 0.0f;
};

/* Throws std::runtime_error for a non-zero status of a C ABI call. */
inline void check(int status, const char* call) {
  if (status != N2W_OK) {
    throw std::runtime_error(std::string("n2w error ") + std::to_string(status) + " in " + call + ": " +
                             n2w_last_error());
  }
}

#define N2W_CPP_CHECK(expr) ::n2w::check((expr), #expr)

/* Host triangle mesh (reference n2wos::Mesh + its free functions). */
class Mesh {
 public:
  Mesh() = default;
  explicit Mesh(n2w_mesh* handle) : m_(handle) {}
  Mesh(const std::vector<Vec3f>& vertices, const std::vector<std::uint32_t>& triangle_indices,
       const std::string& name = "mesh") {
    static_assert(sizeof(Vec3f) == 3 * sizeof(float), "Vec3f must be three packed floats");
    N2W_CPP_CHECK(n2w_mesh_create(reinterpret_cast<const float*>(vertices.data()),
                                  static_cast<int64_t>(vertices.size()), triangle_indices.data(),
                                  static_cast<int64_t>(triangle_indices.size() / 3), name.c_str(), &m_));
  }
  ~Mesh() { n2w_mesh_free(m_); }
  Mesh(const Mesh&) = delete;
  Mesh& operator=(const Mesh&) = delete;
  Mesh(Mesh&& o) noexcept : m_(std::exchange(o.m_, nullptr)) {}
  Mesh& operator=(Mesh&& o) noexcept {
    if (this != &o) {
      n2w_mesh_free(m_);
      m_ = std::exchange(o.m_, nullptr);
    }
    return *this;
  }

  const n2w_mesh* handle() const { return m_; }
  n2w_mesh* handle() { return m_; }
  std::size_t vertex_count() const { return counts().first; }
  std::size_t triangle_count() const { return counts().second; }

 private:
  std::pair<std::size_t, std::size_t> counts() const {
    int64_t nv = 0, nt = 0;
    N2W_CPP_CHECK(n2w_mesh_counts(m_, &nv, &nt));
    return {static_cast<std::size_t>(nv), static_cast<std::size_t>(nt)};
  }
  n2w_mesh* m_ = nullptr;
};

struct NormalizeTransform {
  Vec3f center;
  float scale = 1.0f;
};

inline Mesh make_procedural_bumpy_sphere(int stacks, int slices, float bump_amplitude = 0.15f) {
  n2w_mesh* m = nullptr;
  N2W_CPP_CHECK(n2w_mesh_bumpy_sphere_ref(stacks, slices, bump_amplitude, &m));
  return Mesh(m);
}

inline Mesh load_ply_mesh(const std::string& path) {
  n2w_mesh* m = nullptr;
  N2W_CPP_CHECK(n2w_mesh_load_ply(path.c_str(), &m));
  return Mesh(m);
}

inline Mesh load_obj_mesh(const std::string& path) {
  n2w_mesh* m = nullptr;
  N2W_CPP_CHECK(n2w_mesh_load_obj(path.c_str(), &m));
  return Mesh(m);
}

inline NormalizeTransform normalize_to_unit_radius(Mesh& mesh) {
  NormalizeTransform t;
  float c[3];
  N2W_CPP_CHECK(n2w_mesh_normalize(mesh.handle(), c, &t.scale));
  t.center = {c[0], c[1], c[2]};
  return t;
}

/* Device-resident BVH + triangles with the reference's query shape.
 * build_method: "sah" or "spatial_median"; leaf_size in [1, 8]. */
class CuBqlBvh {
 public:
  CuBqlBvh() = default;
  explicit CuBqlBvh(const Mesh& mesh, int leaf_size = 8, const std::string& build_method = "spatial_median") {
    N2W_CPP_CHECK(n2w_bvh_create(mesh.handle(), leaf_size, build_method.c_str(), &b_));
  }
  ~CuBqlBvh() { n2w_bvh_destroy(b_); }
  CuBqlBvh(const CuBqlBvh&) = delete;
  CuBqlBvh& operator=(const CuBqlBvh&) = delete;
  CuBqlBvh(CuBqlBvh&& o) noexcept : b_(std::exchange(o.b_, nullptr)) {}
  CuBqlBvh& operator=(CuBqlBvh&& o) noexcept {
    if (this != &o) {
      n2w_bvh_destroy(b_);
      b_ = std::exchange(o.b_, nullptr);
    }
    return *this;
  }

  /* Caller-owned device pointers; no allocation, no host transfer. */
  void query_device(const DeviceVec3* d_points, int query_count, float* d_distance2, DeviceVec3* d_closest,
                    int* d_triangle_id, int* d_overflow, int block_size = 128, n2w_stream_t stream = nullptr) const {
    N2W_CPP_CHECK(n2w_bvh_query_device(b_, d_points, query_count, d_distance2, d_closest, d_triangle_id,
                                       d_overflow, block_size, stream));
  }

  void query_device_masked(const DeviceVec3* d_points, const std::uint8_t* d_active, int query_count,
                           float* d_distance2, DeviceVec3* d_closest, int* d_triangle_id, int* d_overflow,
                           int block_size = 128, n2w_stream_t stream = nullptr) const {
    N2W_CPP_CHECK(n2w_bvh_query_device_masked(b_, d_points, d_active, query_count, d_distance2, d_closest,
                                              d_triangle_id, d_overflow, block_size, stream));
  }

  std::size_t triangle_count() const { return static_cast<std::size_t>(stats().triangles); }
  std::size_t node_count() const { return static_cast<std::size_t>(stats().nodes); }
  std::size_t prim_id_count() const { return static_cast<std::size_t>(stats().triangles); }
  int leaf_size() const { return stats().leaf_size; }
  int max_depth() const { return stats().max_depth; }
  const n2w_bvh* handle() const { return b_; }

 private:
  n2w_bvh_stats stats() const {
    n2w_bvh_stats s{};
    N2W_CPP_CHECK(n2w_bvh_stats_get(b_, &s));
    return s;
  }
  n2w_bvh* b_ = nullptr;
};

/* The reference's in-tree backend name: same object, leaf size only
 * (its builder was the median split). */
class CudaBvh : public CuBqlBvh {
 public:
  CudaBvh() = default;
  explicit CudaBvh(const Mesh& mesh, int leaf_size = 8) : CuBqlBvh(mesh, leaf_size, "spatial_median") {}
};

inline std::string cuda_runtime_version_string() {
  char buf[256];
  N2W_CPP_CHECK(n2w_cuda_runtime_version_string(buf, sizeof(buf)));
  return buf;
}

inline std::string cuda_device_summary() {
  char buf[512];
  N2W_CPP_CHECK(n2w_cuda_device_summary(buf, sizeof(buf)));
  return buf;
}

}  // namespace n2w

#ifdef N2W_PROVIDE_N2WOS_NAMESPACE
namespace n2wos {
using n2w::CuBqlBvh;
using n2w::CudaBvh;
using n2w::DeviceVec3;
using n2w::load_obj_mesh;
using n2w::load_ply_mesh;
using n2w::make_procedural_bumpy_sphere;
using n2w::Mesh;
using n2w::normalize_to_unit_radius;
using n2w::NormalizeTransform;
using n2w::Vec3f;
using n2w::cuda_device_summary;
using n2w::cuda_runtime_version_string;
}  // namespace n2wos
#endif

#endif  // N2W_HPP_
