// Read-bandwidth probes of the on-chip memory levels.  The closest-point
// traversal and the walkers fetch nodes and triangles that are L1 / L2 hits
// (the BVH and triangles of an 80 k-triangle mesh are ~7 MB), so their
// roofline denominator is the sustained read bandwidth of those levels, which
// the copy and GEMM peaks measured elsewhere do not give.  No counterpart in
// the reference.
//
//  level 2: every thread streams 16-byte loads that bypass L1 (ld.global.cg)
//           over a buffer that fits in L2, four loads in flight per thread;
//  level 1: every block re-reads its own 16 KiB slice with L1-caching loads.
// Both run a full grid (SMs x 8 blocks of 256 threads) and report the bytes
// loaded divided by the CUDA-event time of the timed launch.
#include <cuda_runtime.h>

#include "internal.hpp"

namespace n2w {
namespace {

constexpr int kProbeThreads = 256;
constexpr int kProbeBlocksPerSm = 8;
constexpr size_t kL1Slice4 = 1024;  // float4 per block slice: 16 KiB

// Loads the compiler may not hoist out of the repeat loop or merge across
// iterations (volatile): L1-caching (.ca) and L2-only (.cg) 16-byte reads.
__device__ __forceinline__ float4 load_ca(const float4* p) {
  float4 v;
  asm volatile("ld.global.ca.v4.f32 {%0, %1, %2, %3}, [%4];" : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w) : "l"(p));
  return v;
}
__device__ __forceinline__ float4 load_cg(const float4* p) {
  float4 v;
  asm volatile("ld.global.cg.v4.f32 {%0, %1, %2, %3}, [%4];" : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w) : "l"(p));
  return v;
}

__device__ __forceinline__ void acc4(float4& a, float4 v) {
  a.x += v.x;
  a.y += v.y;
  a.z += v.z;
  a.w += v.w;
}

// The buffer holds zeros, so the sink store never happens; the compiler cannot
// know that and keeps every load.
__global__ void __launch_bounds__(kProbeThreads) read_l2_kernel(const float4* __restrict__ buf, size_t n4, int iters,
                                                                float4* __restrict__ sink) {
  float4 a0 = make_float4(0, 0, 0, 0), a1 = a0, a2 = a0, a3 = a0;
  const size_t stride = static_cast<size_t>(gridDim.x) * blockDim.x;
  const size_t start = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  for (int it = 0; it < iters; ++it) {
    size_t i = start;
    for (; i + 3 * stride < n4; i += 4 * stride) {
      const float4 v0 = load_cg(buf + i), v1 = load_cg(buf + i + stride), v2 = load_cg(buf + i + 2 * stride),
                   v3 = load_cg(buf + i + 3 * stride);
      acc4(a0, v0);
      acc4(a1, v1);
      acc4(a2, v2);
      acc4(a3, v3);
    }
    for (; i < n4; i += stride) acc4(a0, load_cg(buf + i));
  }
  const float s = a0.x + a1.y + a2.z + a3.w + a0.w + a1.x + a2.y + a3.z;
  if (s != 0.0f) sink[start] = make_float4(s, s, s, s);
}

__global__ void __launch_bounds__(kProbeThreads) read_l1_kernel(const float4* __restrict__ buf, int iters,
                                                                float4* __restrict__ sink) {
  const float4* slice = buf + static_cast<size_t>(blockIdx.x) * kL1Slice4;
  float4 a0 = make_float4(0, 0, 0, 0), a1 = a0, a2 = a0, a3 = a0;
  constexpr unsigned kMask = static_cast<unsigned>(kL1Slice4) - 1u;
  for (int it = 0; it < iters; ++it) {
    // the lane's offsets rotate every pass (a pass still reads the whole
    // slice, a coalesced 512 B per warp load), so no load repeats the
    // previous pass's address and none can be hoisted out of the loop
    const unsigned j = (threadIdx.x + static_cast<unsigned>(it) * 32u) & kMask;
    acc4(a0, load_ca(slice + j));
    acc4(a1, load_ca(slice + ((j + kProbeThreads) & kMask)));
    acc4(a2, load_ca(slice + ((j + 2 * kProbeThreads) & kMask)));
    acc4(a3, load_ca(slice + ((j + 3 * kProbeThreads) & kMask)));
  }
  const float s = a0.x + a1.y + a2.z + a3.w + a0.w + a1.x + a2.y + a3.z;
  if (s != 0.0f) sink[static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x] = make_float4(s, s, s, s);
}

}  // namespace
}  // namespace n2w

using namespace n2w;

extern "C" int n2w_probe_read_bandwidth(int level, size_t bytes, int iterations, double* gbs_out) {
  return guarded([&] {
    N2W_REQUIRE(gbs_out, "null output");
    N2W_REQUIRE(level == 1 || level == 2, "level must be 1 (L1) or 2 (L2)");
    N2W_REQUIRE(iterations > 0, "iterations must be positive");
    int dev = 0, sms = 0;
    N2W_CUDA(cudaGetDevice(&dev));
    N2W_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    const unsigned grid = static_cast<unsigned>(sms * kProbeBlocksPerSm);
    const size_t n4 = level == 2 ? bytes / 16 : static_cast<size_t>(grid) * kL1Slice4;
    N2W_REQUIRE(level == 1 || n4 >= static_cast<size_t>(grid) * kProbeThreads, "buffer too small for one pass");
    float4* buf = nullptr;
    float4* sink = nullptr;
    N2W_CUDA(cudaMalloc(&buf, n4 * sizeof(float4)));
    cudaError_t e = cudaMalloc(&sink, static_cast<size_t>(grid) * kProbeThreads * sizeof(float4));
    cudaEvent_t t0 = nullptr, t1 = nullptr;
    float ms = 0.0f;
    if (e == cudaSuccess) e = cudaMemset(buf, 0, n4 * sizeof(float4));
    if (e == cudaSuccess) e = cudaEventCreate(&t0);
    if (e == cudaSuccess) e = cudaEventCreate(&t1);
    for (int pass = 0; pass < 2 && e == cudaSuccess; ++pass) {  // pass 0 warms the cache level
      if (pass == 1) e = cudaEventRecord(t0);
      if (level == 2) read_l2_kernel<<<grid, kProbeThreads>>>(buf, n4, iterations, sink);
      else read_l1_kernel<<<grid, kProbeThreads>>>(buf, iterations, sink);
      if (e == cudaSuccess) e = cudaGetLastError();
      if (pass == 1 && e == cudaSuccess) e = cudaEventRecord(t1);
    }
    if (e == cudaSuccess) e = cudaEventSynchronize(t1);
    if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, t0, t1);
    if (t0) cudaEventDestroy(t0);
    if (t1) cudaEventDestroy(t1);
    cudaFree(sink);
    cudaFree(buf);
    N2W_CUDA(e);
    N2W_REQUIRE(ms > 0.0f, "probe launch took no measurable time");
    *gbs_out = static_cast<double>(n4) * 16.0 * iterations / (ms * 1e-3) / 1e9;
  });
}
