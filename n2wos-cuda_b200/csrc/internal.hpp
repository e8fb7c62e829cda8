// Host-side internals shared by the library's translation units.
#pragma once

#include <cuda_runtime.h>

#include <array>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

#include "layout.h"
#include "n2w.h"

struct n2w_mesh {
  std::vector<std::array<float, 3>> vertices;
  std::vector<std::array<uint32_t, 3>> triangles;
  std::string name;
};

struct n2w_bvh {
  n2w::Node4* d_nodes = nullptr;
  n2w::TriRec* d_tris = nullptr;
  int* d_seed = nullptr;  // seed grid: leaf slot of the nearest triangle per lattice node
  float seed_lo[3] = {0, 0, 0};
  float seed_h = 0.0f;
  int seed_n = 0;
  n2w_bvh_stats stats{};
  int device = 0;
};

namespace n2w {

class Error : public std::runtime_error {
 public:
  Error(int code, const std::string& msg) : std::runtime_error(msg), code_(code) {}
  int code() const { return code_; }

 private:
  int code_;
};

void set_last_error(const std::string& msg);

#define N2W_CUDA(expr)                                                                         \
  do {                                                                                         \
    cudaError_t err__ = (expr);                                                                \
    if (err__ != cudaSuccess) {                                                                \
      throw ::n2w::Error(N2W_ECUDA, std::string("CUDA error at ") + __FILE__ + ":" +          \
                                        std::to_string(__LINE__) + ": " +                      \
                                        cudaGetErrorString(err__));                            \
    }                                                                                          \
  } while (false)

#define N2W_REQUIRE(cond, msg)                        \
  do {                                                \
    if (!(cond)) throw ::n2w::Error(N2W_EINVAL, msg); \
  } while (false)

// Runs f, converting exceptions into status codes + last-error text.
template <typename F>
int guarded(F&& f) {
  try {
    f();
    return N2W_OK;
  } catch (const Error& e) {
    set_last_error(e.what());
    return e.code();
  } catch (const std::bad_alloc&) {
    set_last_error("host allocation failed");
    return N2W_ENOMEM;
  } catch (const std::exception& e) {
    set_last_error(e.what());
    return N2W_EINTERNAL;
  }
}

// ---- host BVH build (bvh_build.cpp) ----
struct HostBvh {
  std::vector<Node4> nodes;
  std::vector<TriRec> tris;
  int64_t binary_nodes = 0;
  int64_t leaves = 0;
  int max_depth = 0;
  double sah_cost = 0.0;
};
HostBvh build_bvh4(const n2w_mesh& mesh, int leaf_size, const std::string& method);
n2w_bvh_stats host_stats(const HostBvh& h, int leaf_size, double ms);

// ---- device query launch (closest_point.cu) ----
void launch_closest_point(const n2w_bvh& bvh, const n2w_vec3* d_points, const uint8_t* d_active,
                          int n, float* d_d2, n2w_vec3* d_cp, int* d_id, int* d_overflow,
                          int* d_nodes, int* d_tris, int block_size, cudaStream_t stream);

void build_seed_grid(n2w_bvh& b, const n2w_mesh& mesh, int n);

void launch_inside(const n2w_bvh& bvh, const n2w_vec3* d_points, int n, uint8_t* d_inside, int* d_overflow,
                   int block_size, cudaStream_t stream);

int sm_count_current();

// ---- device utilities (util.cu) ----
void launch_oracle_cache(const n2w_problem& pb, const float* d_inputs, int64_t n, const float* in_min,
                         const float* in_ext, float* d_out, cudaStream_t s);
void launch_count_samples(const uint8_t* needs, const int* forced, const int* overflow, int64_t n,
                          unsigned long long* d_counts, cudaStream_t s);
void launch_exact(const n2w_problem& pb, const n2w_vec3* d_points, int64_t n, float* d_out, cudaStream_t s);

// ---- stream-ordered scratch (util.cu) ----
// Allocations come from a memory pool the library owns on each device, which
// keeps up to kScratchRetainBytes cached across synchronisations, so repeated
// calls reuse mapped memory instead of remapping it (the device's default
// pool, left untouched, releases everything at each synchronisation).
constexpr uint64_t kScratchRetainBytes = uint64_t{2} << 30;
void* scratch_alloc(size_t bytes, cudaStream_t s);
void scratch_free(void* p, cudaStream_t s);

}  // namespace n2w
