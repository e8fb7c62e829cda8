// ORACLE — test infrastructure only.  C entry points over the reference's own
// CPU sources, compiled where they lie (src/mesh/*.cpp,
// src/geometry/closest_point.cpp, src/cuda/bvh_build_host.cpp) by
// oracle/build.py into oracle/_ref/libn2wos_ref.so.  Used to pin the oracle
// and to generate golden vectors; never part of the product.
#include <cstdint>
#include <cstring>
#include <exception>
#include <string>

#include "n2wos/closest_point.hpp"
#include "n2wos/cuda_bvh.hpp"
#include "n2wos/mesh.hpp"
#include "n2wos/nc_harmonic_mixture.hpp"
#include "n2wos/nc_poisson_manufactured.hpp"

namespace {
thread_local std::string g_err;
n2wos::Mesh* as_mesh(void* h) { return static_cast<n2wos::Mesh*>(h); }
}  // namespace

extern "C" {

const char* ref_last_error() { return g_err.c_str(); }

void* ref_bumpy_sphere(int stacks, int slices, float amplitude) {
  try {
    return new n2wos::Mesh(n2wos::make_procedural_bumpy_sphere(stacks, slices, amplitude));
  } catch (const std::exception& e) {
    g_err = e.what();
    return nullptr;
  }
}

void* ref_load_ply(const char* path) {
  try {
    return new n2wos::Mesh(n2wos::load_ply_mesh(path));
  } catch (const std::exception& e) {
    g_err = e.what();
    return nullptr;
  }
}

void* ref_load_obj(const char* path) {
  try {
    return new n2wos::Mesh(n2wos::load_obj_mesh(path));
  } catch (const std::exception& e) {
    g_err = e.what();
    return nullptr;
  }
}

void* ref_mesh_from_arrays(const float* v, int64_t nv, const uint32_t* t, int64_t nt) {
  auto* m = new n2wos::Mesh();
  m->vertices.resize(static_cast<size_t>(nv));
  m->triangles.resize(static_cast<size_t>(nt));
  for (int64_t i = 0; i < nv; ++i) m->vertices[i] = {v[3 * i], v[3 * i + 1], v[3 * i + 2]};
  for (int64_t i = 0; i < nt; ++i) m->triangles[i] = {t[3 * i], t[3 * i + 1], t[3 * i + 2]};
  return m;
}

void ref_mesh_free(void* h) { delete as_mesh(h); }

void ref_mesh_counts(void* h, int64_t* nv, int64_t* nt) {
  *nv = static_cast<int64_t>(as_mesh(h)->vertices.size());
  *nt = static_cast<int64_t>(as_mesh(h)->triangles.size());
}

void ref_mesh_copy(void* h, float* v, uint32_t* t) {
  const auto* m = as_mesh(h);
  for (size_t i = 0; i < m->vertices.size(); ++i) {
    v[3 * i] = m->vertices[i].x;
    v[3 * i + 1] = m->vertices[i].y;
    v[3 * i + 2] = m->vertices[i].z;
  }
  for (size_t i = 0; i < m->triangles.size(); ++i) {
    t[3 * i] = m->triangles[i].v0;
    t[3 * i + 1] = m->triangles[i].v1;
    t[3 * i + 2] = m->triangles[i].v2;
  }
}

int ref_normalize(void* h, float* center, float* scale) {
  try {
    const n2wos::NormalizeTransform tr = n2wos::normalize_to_unit_radius(*as_mesh(h));
    center[0] = tr.center.x;
    center[1] = tr.center.y;
    center[2] = tr.center.z;
    *scale = tr.scale;
    return 0;
  } catch (const std::exception& e) {
    g_err = e.what();
    return 1;
  }
}

void ref_bruteforce(void* h, const float* points, int64_t n, float* d2, float* cp, int32_t* id) {
  const auto& m = *as_mesh(h);
  for (int64_t i = 0; i < n; ++i) {
    const n2wos::ClosestPointResult r =
        n2wos::closest_point_bruteforce(m, {points[3 * i], points[3 * i + 1], points[3 * i + 2]});
    d2[i] = r.distance2;
    cp[3 * i] = r.closest.x;
    cp[3 * i + 1] = r.closest.y;
    cp[3 * i + 2] = r.closest.z;
    id[i] = r.triangle_id;
  }
}

int64_t ref_count_degenerate(void* h) {
  return static_cast<int64_t>(n2wos::count_degenerate_triangles(*as_mesh(h)));
}

// Reference host median-split BVH (bvh_build_host.cpp): node count and depth.
int ref_host_bvh_stats(void* h, int leaf_size, int64_t* nodes, int32_t* depth) {
  try {
    const n2wos::HostBvhData b = n2wos::build_host_bvh(*as_mesh(h), leaf_size);
    *nodes = static_cast<int64_t>(b.nodes.size());
    *depth = b.max_depth;
    return 0;
  } catch (const std::exception& e) {
    g_err = e.what();
    return 1;
  }
}

// The reference host BVH itself (bvh_build_host.cpp:129-158): triangles in
// mesh order (36 B each), nodes in DFS order (40 B each), the leaf triangle
// index list.  Walked by the oracle's restatement of closest_point_bvh_kernel.
void* ref_host_bvh_build(void* h, int leaf_size) {
  try {
    return new n2wos::HostBvhData(n2wos::build_host_bvh(*as_mesh(h), leaf_size));
  } catch (const std::exception& e) {
    g_err = e.what();
    return nullptr;
  }
}

void ref_host_bvh_counts(void* b, int64_t* tris, int64_t* nodes, int64_t* idx, int32_t* depth) {
  const auto* d = static_cast<const n2wos::HostBvhData*>(b);
  *tris = static_cast<int64_t>(d->triangles.size());
  *nodes = static_cast<int64_t>(d->nodes.size());
  *idx = static_cast<int64_t>(d->triangle_indices.size());
  *depth = d->max_depth;
}

void ref_host_bvh_copy(void* b, void* tris, void* nodes, int32_t* idx) {
  const auto* d = static_cast<const n2wos::HostBvhData*>(b);
  static_assert(sizeof(n2wos::DeviceTriangle) == 36 && sizeof(n2wos::DeviceBvhNode) == 40, "reference layout");
  std::memcpy(tris, d->triangles.data(), d->triangles.size() * sizeof(n2wos::DeviceTriangle));
  std::memcpy(nodes, d->nodes.data(), d->nodes.size() * sizeof(n2wos::DeviceBvhNode));
  for (size_t i = 0; i < d->triangle_indices.size(); ++i) idx[i] = d->triangle_indices[i];
}

void ref_host_bvh_free(void* b) { delete static_cast<n2wos::HostBvhData*>(b); }

// Boundary data u and source f of the reference's header-only analytic modes
// (harmonic mixtures 13-16, manufactured Poisson 30, 31, 32), evaluated by the
// reference's own inline functions.  Returns 0, or -1 for another mode.
struct RefP {
  float x, y, z;
};
int ref_analytic_mode(int mode, const float* xyz, int64_t n, float* u_out, float* f_out) {
  for (int64_t i = 0; i < n; ++i) {
    const RefP p{xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2]};
    float u = 0.0f, f = 0.0f;
    switch (mode) {
      case 13: u = n2wos::nc_harmonic_mixture_smooth_value(p); break;
      case 14: u = n2wos::nc_harmonic_mixture_figlike_value(p); break;
      case 15: u = n2wos::nc_harmonic_mixture_multiscale_value(p); break;
      case 16: u = n2wos::nc_harmonic_mixture_figlike_hf_value(p); break;
      case 30:
      case 31:
        u = n2wos::nc_poisson_manufactured_u(p, mode);
        f = n2wos::nc_poisson_manufactured_f(p, mode);
        break;
      case 32:
        u = ::nc_poisson_figlike_hf_x5_value(p);  // declared outside namespace n2wos
        f = ::nc_poisson_figlike_hf_x5_source(p);
        break;
      default: return -1;
    }
    u_out[i] = u;
    f_out[i] = f;
  }
  return 0;
}

}  // extern "C"
