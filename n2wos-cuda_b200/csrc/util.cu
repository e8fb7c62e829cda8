// Small device utilities that the evaluation tools and the Python layer share:
// exact solutions evaluated on the device, the analytic stand-in for the cache
// (an "oracle cache" that returns the exact solution), seeded unit-cube sample
// batches with their targets, and FP64 reductions of per-sample arrays.
//
// Reference counterparts: the wavefront engine's analytic cache
// (src/cuda/wos_wavefront.cu:140-149, harmonic_device at X_m), the cache
// probe's batch generator and downstream consumer
// (src/tools/probe_tcnn_cache.cu:217-262), and the per-sample counting of
// cache queries / forced / overflow walks in the NC evaluator's host summary
// (src/tools/eval_tcnn_nc_wos.cu:527-533), done here on the device.
#include <cuda_runtime.h>

#include <algorithm>
#include <mutex>

#include "internal.hpp"
#include "philox.cuh"
#include "problem.cuh"

namespace n2w {
namespace {

constexpr int kBlock = 256;

unsigned blocks_for(int64_t n) { return static_cast<unsigned>((n + kBlock - 1) / kBlock); }

__global__ void exact_kernel(n2w_problem pb, const n2w_vec3* __restrict__ pts, int64_t n, float* __restrict__ out) {
  const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const n2w_vec3 p = pts[i];
  out[i] = static_cast<float>(problem_u<double>(pb, p.x, p.y, p.z));
}

// Unit-cube input u -> world point in_min + u * in_ext (FP32, as the walker
// maps it forward) -> exact solution there.
__global__ void oracle_cache_kernel(n2w_problem pb, const float* __restrict__ in, int64_t n, float3 lo, float3 ext,
                                    float* __restrict__ out) {
  const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float x = lo.x + in[3 * i + 0] * ext.x;
  const float y = lo.y + in[3 * i + 1] * ext.y;
  const float z = lo.z + in[3 * i + 2] * ext.z;
  out[i] = static_cast<float>(problem_u<double>(pb, x, y, z));
}

// Sample i of batch `step`: Philox(seed; i, step) -> 3 uniforms in [0,1).
__global__ void fill_unit_kernel(n2w_problem pb, int64_t n, uint32_t k0, uint32_t k1, uint32_t step, float3 lo,
                                 float3 ext, float* __restrict__ inputs, float* __restrict__ targets) {
  const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const U4 r = philox4x32_10(U4{static_cast<uint32_t>(i), static_cast<uint32_t>(i >> 32), step, 0x7Au}, k0, k1);
  const float ux = u01(r.x), uy = u01(r.y), uz = u01(r.z);
  inputs[3 * i + 0] = ux;
  inputs[3 * i + 1] = uy;
  inputs[3 * i + 2] = uz;
  if (targets) {
    targets[i] = static_cast<float>(
        problem_u<double>(pb, lo.x + ux * ext.x, lo.y + uy * ext.y, lo.z + uz * ext.z));
  }
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

__device__ __forceinline__ unsigned long long warp_sum_u64(unsigned long long v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// acc[0..3] += sum pred, sum exact, sum (pred-exact)^2, sum |pred-exact| (FP64),
// one atomic per warp and quantity.
__global__ void compare_kernel(const float* __restrict__ pred, const float* __restrict__ exact, int64_t n,
                               double* __restrict__ acc) {
  double s0 = 0, s1 = 0, s2 = 0, s3 = 0;
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const double p = pred[i], e = exact[i], d = p - e;
    s0 += p;
    s1 += e;
    s2 += d * d;
    s3 += fabs(d);
  }
  s0 = warp_sum(s0);
  s1 = warp_sum(s1);
  s2 = warp_sum(s2);
  s3 = warp_sum(s3);
  if ((threadIdx.x & 31) == 0) {
    atomicAdd(acc + 0, s0);
    atomicAdd(acc + 1, s1);
    atomicAdd(acc + 2, s2);
    atomicAdd(acc + 3, s3);
  }
}

// counts[0..2] += nonzero entries of needs (u8), forced (i32), overflow (i32).
__global__ void count_kernel(const uint8_t* __restrict__ needs, const int* __restrict__ forced,
                             const int* __restrict__ overflow, int64_t n, unsigned long long* __restrict__ counts) {
  unsigned long long c0 = 0, c1 = 0, c2 = 0;
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    if (needs) c0 += needs[i] ? 1 : 0;
    if (forced) c1 += forced[i] ? 1 : 0;
    if (overflow) c2 += overflow[i] ? 1 : 0;
  }
  c0 = warp_sum_u64(c0);
  c1 = warp_sum_u64(c1);
  c2 = warp_sum_u64(c2);
  if ((threadIdx.x & 31) == 0) {
    if (c0) atomicAdd(counts + 0, c0);
    if (c1) atomicAdd(counts + 1, c1);
    if (c2) atomicAdd(counts + 2, c2);
  }
}

unsigned reduce_grid(int64_t n) {
  const int64_t want = (n + kBlock - 1) / kBlock;
  const int64_t cap = static_cast<int64_t>(sm_count_current()) * 8;
  return static_cast<unsigned>(want < 1 ? 1 : (want < cap ? want : cap));
}

}  // namespace

void launch_oracle_cache(const n2w_problem& pb, const float* d_inputs, int64_t n, const float* in_min,
                         const float* in_ext, float* d_out, cudaStream_t s) {
  if (n == 0) return;
  oracle_cache_kernel<<<blocks_for(n), kBlock, 0, s>>>(pb, d_inputs, n, make_float3(in_min[0], in_min[1], in_min[2]),
                                                       make_float3(in_ext[0], in_ext[1], in_ext[2]), d_out);
  N2W_CUDA(cudaGetLastError());
}

void launch_count_samples(const uint8_t* needs, const int* forced, const int* overflow, int64_t n,
                          unsigned long long* d_counts, cudaStream_t s) {
  if (n == 0) return;
  count_kernel<<<reduce_grid(n), kBlock, 0, s>>>(needs, forced, overflow, n, d_counts);
  N2W_CUDA(cudaGetLastError());
}

namespace {
constexpr int kScratchMaxDevices = 64;
std::mutex g_scratch_mutex;
cudaMemPool_t g_scratch_pool[kScratchMaxDevices] = {};

cudaMemPool_t scratch_pool_current_device() {
  int dev = 0;
  N2W_CUDA(cudaGetDevice(&dev));
  N2W_REQUIRE(dev >= 0 && dev < kScratchMaxDevices, "device index beyond the scratch pool table");
  std::lock_guard<std::mutex> lock(g_scratch_mutex);
  if (!g_scratch_pool[dev]) {
    cudaMemPoolProps props{};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = dev;
    cudaMemPool_t pool = nullptr;
    N2W_CUDA(cudaMemPoolCreate(&pool, &props));
    uint64_t retain = kScratchRetainBytes;
    N2W_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &retain));
    g_scratch_pool[dev] = pool;
  }
  return g_scratch_pool[dev];
}
}  // namespace

void* scratch_alloc(size_t bytes, cudaStream_t s) {
  void* p = nullptr;
  N2W_CUDA(cudaMallocFromPoolAsync(&p, std::max<size_t>(bytes, 1), scratch_pool_current_device(), s));
  return p;
}

void scratch_free(void* p, cudaStream_t s) {
  if (p) N2W_CUDA(cudaFreeAsync(p, s));
}

void launch_exact(const n2w_problem& pb, const n2w_vec3* d_points, int64_t n, float* d_out, cudaStream_t s) {
  if (n == 0) return;
  exact_kernel<<<blocks_for(n), kBlock, 0, s>>>(pb, d_points, n, d_out);
  N2W_CUDA(cudaGetLastError());
}

}  // namespace n2w

using namespace n2w;

extern "C" {

int n2w_problem_exact_device(const n2w_problem* problem, const n2w_vec3* d_points, int64_t n, float* d_u_out,
                             n2w_stream_t stream) {
  return guarded([&] {
    N2W_REQUIRE(problem && n >= 0, "n2w_problem_exact_device: invalid arguments");
    if (n == 0) return;
    N2W_REQUIRE(d_points && d_u_out, "n2w_problem_exact_device: null device pointer");
    launch_exact(*problem, d_points, n, d_u_out, stream);
  });
}

int n2w_oracle_cache_infer(const n2w_problem* problem, const float* d_inputs, int64_t n, const float* input_min,
                           const float* input_extent, float* d_outputs, n2w_stream_t stream) {
  return guarded([&] {
    N2W_REQUIRE(problem && input_min && input_extent && n >= 0, "n2w_oracle_cache_infer: invalid arguments");
    if (n == 0) return;
    N2W_REQUIRE(d_inputs && d_outputs, "n2w_oracle_cache_infer: null device pointer");
    launch_oracle_cache(*problem, d_inputs, n, input_min, input_extent, d_outputs, stream);
  });
}

int n2w_fill_unit_samples(const n2w_problem* problem, int64_t n, uint64_t seed, uint32_t step,
                          const float* input_min, const float* input_extent, float* d_inputs, float* d_targets,
                          n2w_stream_t stream) {
  return guarded([&] {
    N2W_REQUIRE(n >= 0, "n must be non-negative");
    if (n == 0) return;
    N2W_REQUIRE(d_inputs, "n2w_fill_unit_samples: null inputs");
    N2W_REQUIRE(!d_targets || (problem && input_min && input_extent), "targets need a problem and an input map");
    uint32_t k0, k1;
    philox_key(seed, 0x5EEDu, k0, k1);
    const n2w_problem pb = problem ? *problem : n2w_problem{};
    const float3 lo = input_min ? make_float3(input_min[0], input_min[1], input_min[2]) : make_float3(0, 0, 0);
    const float3 ext = input_extent ? make_float3(input_extent[0], input_extent[1], input_extent[2]) : make_float3(1, 1, 1);
    fill_unit_kernel<<<blocks_for(n), kBlock, 0, stream>>>(pb, n, k0, k1, step, lo, ext, d_inputs, d_targets);
    N2W_CUDA(cudaGetLastError());
  });
}

int n2w_compare_accumulate(const float* d_pred, const float* d_exact, int64_t n, double* d_acc4,
                           n2w_stream_t stream) {
  return guarded([&] {
    N2W_REQUIRE(n >= 0, "n must be non-negative");
    if (n == 0) return;
    N2W_REQUIRE(d_pred && d_exact && d_acc4, "n2w_compare_accumulate: null device pointer");
    compare_kernel<<<reduce_grid(n), kBlock, 0, stream>>>(d_pred, d_exact, n, d_acc4);
    N2W_CUDA(cudaGetLastError());
  });
}

int n2w_count_samples(const uint8_t* d_needs_cache, const int* d_forced, const int* d_overflow, int64_t n,
                      unsigned long long* d_counts3, n2w_stream_t stream) {
  return guarded([&] {
    N2W_REQUIRE(n >= 0, "n must be non-negative");
    if (n == 0) return;
    N2W_REQUIRE(d_counts3, "n2w_count_samples: null counts");
    launch_count_samples(d_needs_cache, d_forced, d_overflow, n, d_counts3, stream);
  });
}

}  // extern "C"
