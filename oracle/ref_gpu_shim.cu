// ORACLE — test infrastructure only.  C entry points over the reference's
// in-tree GPU closest-point kernel (src/cuda/bvh_query.cu, CudaBvh with the
// host median BVH of src/cuda/bvh_build_host.cpp), compiled unmodified for
// sm_100a by oracle/build.py into oracle/_ref/libn2wos_ref_gpu.so.  Used only by
// GPU tests that compare the product kernel with the reference kernel on the
// same device.
#include <cstdint>
#include <exception>
#include <string>

#include "n2wos/cuda_bvh.hpp"

namespace {
thread_local std::string g_err;
}

extern "C" {

const char* ref_gpu_last_error() { return g_err.c_str(); }

void* ref_gpu_bvh_create(const float* v, int64_t nv, const uint32_t* t, int64_t nt, int leaf_size) {
  try {
    n2wos::Mesh m;
    m.vertices.resize(static_cast<size_t>(nv));
    m.triangles.resize(static_cast<size_t>(nt));
    for (int64_t i = 0; i < nv; ++i) m.vertices[i] = {v[3 * i], v[3 * i + 1], v[3 * i + 2]};
    for (int64_t i = 0; i < nt; ++i) m.triangles[i] = {t[3 * i], t[3 * i + 1], t[3 * i + 2]};
    return new n2wos::CudaBvh(m, leaf_size);
  } catch (const std::exception& e) {
    g_err = e.what();
    return nullptr;
  }
}

int ref_gpu_query_device(void* h, const void* d_points, int n, float* d2, void* cp, int* id, int* ov,
                         int block_size, void* stream) {
  try {
    static_cast<n2wos::CudaBvh*>(h)->query_device(static_cast<const n2wos::DeviceVec3*>(d_points), n, d2,
                                                  static_cast<n2wos::DeviceVec3*>(cp), id, ov, block_size,
                                                  static_cast<cudaStream_t>(stream));
    return 0;
  } catch (const std::exception& e) {
    g_err = e.what();
    return 1;
  }
}

void ref_gpu_bvh_destroy(void* h) { delete static_cast<n2wos::CudaBvh*>(h); }

}  // extern "C"
