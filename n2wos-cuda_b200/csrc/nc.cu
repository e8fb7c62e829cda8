// Neural-cache estimators on the device: interior sampling, online training of
// the cache from WoS labels, and the NC+2LMC estimate (coarse walks truncated
// at depth m and closed with the cache, plus an unbiased residual from fewer
// walks continued to the boundary).
//
// Reference semantics (Somatic-Cell/n2wos-cuda):
//   labels     nc_update_labels_kernel   src/cuda/cubql_bvh.cu:1372-1420 (W walks -> mean)
//   coarse     nc_hybrid_prefix_kernel   1451-1516 -> tcnn inference -> combine 1608-1627
//   residual   nc_2lmc_prefix_continue   1519-1606 -> inference -> combine
//   estimator  mean(coarse) + mean(residual), variances add
//              (src/tools/eval_wavefront_wos.cu:327-342, eval_tcnn_nc_wos.cu:562)
//   input map  (x - input_min) / input_extent clamped to [0,1] (cubql_bvh.cu:1311-1315)
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <chrono>
#include <cstring>
#include <vector>

#include "geom.cuh"
#include "internal.hpp"
#include "philox.cuh"

namespace n2w {
namespace {

// Rejection sampling of points uniform in the interior: candidate k is drawn
// from Philox(seed; k) uniformly in the box and kept when the +x ray parity
// says it is inside.  counters[0] = candidates taken, counters[1] = accepted.
__global__ void __launch_bounds__(256) sample_interior_kernel(const float4* __restrict__ nodes,
                                                              const float4* __restrict__ tris, float3 lo, float3 ext,
                                                              int64_t n, uint32_t k0, uint32_t k1,
                                                              unsigned long long* counters, int64_t max_candidates,
                                                              n2w_vec3* __restrict__ out) {
  for (;;) {
    if (*reinterpret_cast<volatile unsigned long long*>(counters + 1) >= static_cast<unsigned long long>(n)) return;
    const unsigned long long k = atomicAdd(counters, 1ull);
    if (k >= static_cast<unsigned long long>(max_candidates)) return;
    const U4 r = philox4x32_10(U4{static_cast<uint32_t>(k), static_cast<uint32_t>(k >> 32), 0x51u, 0u}, k0, k1);
    const float x = lo.x + ext.x * u01(r.x), y = lo.y + ext.y * u01(r.y), z = lo.z + ext.z * u01(r.z);
    int ov = 0;
    const int hits = dev::ray_x_crossings(nodes, tris, dev::v3(x, y + 1.928371e-6f, z + 3.141593e-6f), ov);
    if ((hits & 1) && !ov) {
      const unsigned long long s = atomicAdd(counters + 1, 1ull);
      if (s < static_cast<unsigned long long>(n)) out[s] = n2w_vec3{x, y, z};
    }
  }
}

// Adds one block's per-point statistics into running totals (fields that are
// null in either struct are skipped).
__global__ void accumulate_stats_kernel(n2w_point_stats part, n2w_point_stats total, int64_t n) {
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    total.d_sum[i] += part.d_sum[i];
    total.d_sum_sq[i] += part.d_sum_sq[i];
    total.d_count[i] += part.d_count[i];
    if (total.d_steps && part.d_steps) total.d_steps[i] += part.d_steps[i];
    if (total.d_forced && part.d_forced) total.d_forced[i] += part.d_forced[i];
  }
}

// Per-point label = mean of the walks; inputs mapped to the unit cube.
__global__ void labels_kernel(const n2w_vec3* __restrict__ pts, const double* __restrict__ sum,
                              const uint32_t* __restrict__ count, int64_t n, float3 in_min, float3 in_ext,
                              float* __restrict__ inputs, float* __restrict__ targets) {
  const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const n2w_vec3 p = pts[i];
  inputs[3 * i + 0] = fminf(1.0f, fmaxf(0.0f, (p.x - in_min.x) / fmaxf(in_ext.x, 1.0e-6f)));
  inputs[3 * i + 1] = fminf(1.0f, fmaxf(0.0f, (p.y - in_min.y) / fmaxf(in_ext.y, 1.0e-6f)));
  inputs[3 * i + 2] = fminf(1.0f, fmaxf(0.0f, (p.z - in_min.z) / fmaxf(in_ext.z, 1.0e-6f)));
  const uint32_t c = count[i];
  targets[i] = c ? static_cast<float>(sum[i] / static_cast<double>(c)) : 0.0f;
}

__global__ void map_to_unit_kernel(const n2w_vec3* __restrict__ pts, int64_t n, float3 in_min, float3 in_ext,
                                   float* __restrict__ inputs) {
  const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const n2w_vec3 p = pts[i];
  inputs[3 * i + 0] = fminf(1.0f, fmaxf(0.0f, (p.x - in_min.x) / fmaxf(in_ext.x, 1.0e-6f)));
  inputs[3 * i + 1] = fminf(1.0f, fmaxf(0.0f, (p.y - in_min.y) / fmaxf(in_ext.y, 1.0e-6f)));
  inputs[3 * i + 2] = fminf(1.0f, fmaxf(0.0f, (p.z - in_min.z) / fmaxf(in_ext.z, 1.0e-6f)));
}

template <typename T>
T* stream_alloc(size_t count, cudaStream_t s) {
  return static_cast<T*>(scratch_alloc(std::max<size_t>(count, 1) * sizeof(T), s));
}

void sample_interior(const n2w_bvh& bvh, const float* lo, const float* hi, int64_t n, uint64_t seed,
                     n2w_vec3* d_out, unsigned long long* d_counters, cudaStream_t s) {
  N2W_CUDA(cudaMemsetAsync(d_counters, 0, 2 * sizeof(unsigned long long), s));
  uint32_t k0, k1;
  philox_key(seed, 9u, k0, k1);
  const int block = 256;
  const int grid = sm_count_current() * 8;
  sample_interior_kernel<<<grid, block, 0, s>>>(
      reinterpret_cast<const float4*>(bvh.d_nodes), reinterpret_cast<const float4*>(bvh.d_tris),
      make_float3(lo[0], lo[1], lo[2]), make_float3(hi[0] - lo[0], hi[1] - lo[1], hi[2] - lo[2]), n, k0, k1,
      d_counters, 1000 * n + 1000000, d_out);
  N2W_CUDA(cudaGetLastError());
}

}  // namespace
}  // namespace n2w

using namespace n2w;

extern "C" {

int n2w_sample_interior(const n2w_bvh* bvh, const float* box_lo, const float* box_hi, int64_t n, uint64_t seed,
                        n2w_vec3* d_points_out, int64_t* h_accepted_out, n2w_stream_t stream) {
  return n2w_sample_interior_ex(bvh, box_lo, box_hi, n, seed, d_points_out, h_accepted_out, nullptr, stream);
}

int n2w_sample_interior_ex(const n2w_bvh* bvh, const float* box_lo, const float* box_hi, int64_t n, uint64_t seed,
                           n2w_vec3* d_points_out, int64_t* h_accepted_out, int64_t* h_candidates_out,
                           n2w_stream_t stream) {
  return guarded([&] {
    N2W_REQUIRE(bvh && bvh->d_nodes && box_lo && box_hi, "null argument");
    N2W_REQUIRE(n >= 0, "n must be non-negative");
    if (n == 0) return;
    N2W_REQUIRE(d_points_out, "null output");
    for (int a = 0; a < 3; ++a) N2W_REQUIRE(box_hi[a] > box_lo[a], "empty sampling box");
    unsigned long long* d_c = stream_alloc<unsigned long long>(2, stream);
    sample_interior(*bvh, box_lo, box_hi, n, seed, d_points_out, d_c, stream);
    unsigned long long c[2] = {0, 0};
    N2W_CUDA(cudaMemcpyAsync(c, d_c, sizeof(c), cudaMemcpyDeviceToHost, stream));
    scratch_free(d_c, stream);
    N2W_CUDA(cudaStreamSynchronize(stream));
    const int64_t acc = static_cast<int64_t>(std::min<unsigned long long>(c[1], static_cast<unsigned long long>(n)));
    if (h_accepted_out) *h_accepted_out = acc;
    // Threads race past the n-th acceptance, so the raw counters overshoot; their
    // ratio is still an unbiased acceptance estimate: report n / (hits / draws).
    if (h_candidates_out) {
      *h_candidates_out = c[1] ? static_cast<int64_t>(std::llround(static_cast<double>(n) * static_cast<double>(c[0]) /
                                                                   static_cast<double>(c[1])))
                               : static_cast<int64_t>(c[0]);
    }
    if (acc < n) throw Error(N2W_EINTERNAL, "interior sampling gave up: the box holds too little interior");
  });
}

int n2w_map_to_unit(const n2w_vec3* d_points, int64_t n, const float* input_min, const float* input_extent,
                    float* d_inputs, n2w_stream_t stream) {
  return guarded([&] {
    N2W_REQUIRE(n >= 0 && input_min && input_extent, "invalid arguments");
    if (n == 0) return;
    N2W_REQUIRE(d_points && d_inputs, "null device pointer");
    const int b = 256;
    map_to_unit_kernel<<<static_cast<unsigned>((n + b - 1) / b), b, 0, stream>>>(
        d_points, n, make_float3(input_min[0], input_min[1], input_min[2]),
        make_float3(input_extent[0], input_extent[1], input_extent[2]), d_inputs);
    N2W_CUDA(cudaGetLastError());
  });
}

int n2w_nc_train(n2w_cache* cache, const n2w_bvh* bvh, const n2w_problem* problem,
                 const n2w_nc_train_options* o, float* h_losses, n2w_stream_t stream) {
  return guarded([&] {
    N2W_REQUIRE(cache && bvh && problem && o, "null argument");
    N2W_REQUIRE(o->steps >= 0 && o->batch > 0 && o->walks_per_label > 0, "invalid training options");
    const int64_t B = o->batch;
    n2w_vec3* pts = stream_alloc<n2w_vec3>(B, stream);
    float* inputs = stream_alloc<float>(3 * B, stream);
    float* targets = stream_alloc<float>(B, stream);
    double* sum = stream_alloc<double>(B, stream);
    double* sum2 = stream_alloc<double>(B, stream);
    uint32_t* cnt = stream_alloc<uint32_t>(B, stream);
    uint64_t* steps = stream_alloc<uint64_t>(B, stream);
    uint32_t* forced = stream_alloc<uint32_t>(B, stream);
    unsigned long long* sc = stream_alloc<unsigned long long>(2, stream);
    void* ws = stream_alloc<char>(n2w_wos_workspace_bytes(B), stream);
    n2w_point_stats st{sum, sum2, cnt, steps, forced};
    n2w_walk_options wo{};
    wo.walks_per_point = o->walks_per_label;
    wo.max_steps = o->max_steps;
    wo.epsilon = o->epsilon;
    wo.step_scale = o->step_scale;
    int status = N2W_OK;
    std::string err;
    for (int s = 0; s < o->steps && status == N2W_OK; ++s) {
      const uint64_t seed = o->seed + 0x9E3779B97F4A7C15ull * static_cast<uint64_t>(s + 1);
      sample_interior(*bvh, o->sample_lo, o->sample_hi, B, seed, pts, sc, stream);
      wo.seed = seed ^ 0xD1B54A32D192ED03ull;
      status = n2w_wos_estimate(bvh, problem, pts, B, &wo, st, nullptr, ws, stream);
      if (status != N2W_OK) {
        err = n2w_last_error();
        break;
      }
      const int b = 256;
      labels_kernel<<<static_cast<unsigned>((B + b - 1) / b), b, 0, stream>>>(
          pts, sum, cnt, B, make_float3(o->input_min[0], o->input_min[1], o->input_min[2]),
          make_float3(o->input_extent[0], o->input_extent[1], o->input_extent[2]), inputs, targets);
      N2W_CUDA(cudaGetLastError());
      status = n2w_cache_train_step(cache, inputs, targets, B, h_losses ? h_losses + s : nullptr, stream);
      if (status != N2W_OK) err = n2w_last_error();
    }
    for (void* p : {static_cast<void*>(pts), static_cast<void*>(inputs), static_cast<void*>(targets),
                    static_cast<void*>(sum), static_cast<void*>(sum2), static_cast<void*>(cnt),
                    static_cast<void*>(steps), static_cast<void*>(forced), static_cast<void*>(sc), ws}) {
      scratch_free(p, stream);
    }
    if (status != N2W_OK) throw Error(status, err);
  });
}

int n2w_nc_train_dp(n2w_cache* cache, const n2w_bvh* bvh, const n2w_problem* problem,
                    const n2w_nc_train_options* o, n2w_comm* comm, float* h_losses, n2w_stream_t stream) {
  return guarded([&] {
    N2W_REQUIRE(cache && bvh && problem && o && comm, "null argument");
    N2W_REQUIRE(o->steps >= 0 && o->batch > 0 && o->walks_per_label > 0, "invalid training options");
    auto ok = [](int st) {
      if (st != N2W_OK) throw Error(st, n2w_last_error());
    };
    int rank = 0, world = 1;
    ok(n2w_comm_info(comm, &rank, &world));
    float* d_grad = nullptr;
    float* d_loss = nullptr;
    int64_t n_params = 0;
    ok(n2w_cache_gradient_buffer(cache, &d_grad, &n_params, &d_loss));
    const int64_t B = o->batch;
    n2w_vec3* pts = stream_alloc<n2w_vec3>(B, stream);
    float* inputs = stream_alloc<float>(3 * B, stream);
    float* targets = stream_alloc<float>(B, stream);
    double* sum = stream_alloc<double>(B, stream);
    double* sum2 = stream_alloc<double>(B, stream);
    uint32_t* cnt = stream_alloc<uint32_t>(B, stream);
    uint64_t* steps = stream_alloc<uint64_t>(B, stream);
    uint32_t* forced = stream_alloc<uint32_t>(B, stream);
    unsigned long long* sc = stream_alloc<unsigned long long>(2, stream);
    void* ws = stream_alloc<char>(n2w_wos_workspace_bytes(B), stream);
    n2w_point_stats st{sum, sum2, cnt, steps, forced};
    n2w_walk_options wo{};
    wo.walks_per_point = o->walks_per_label;
    wo.max_steps = o->max_steps;
    wo.epsilon = o->epsilon;
    wo.step_scale = o->step_scale;
    // rank r draws its own points and walks; rank 0 draws what n2w_nc_train draws
    const uint64_t rank_seed = o->seed + 0xD6E8FEB86659FD93ull * static_cast<uint64_t>(rank);
    int status = N2W_OK;
    std::string err;
    for (int s = 0; s < o->steps && status == N2W_OK; ++s) {
      const uint64_t seed = rank_seed + 0x9E3779B97F4A7C15ull * static_cast<uint64_t>(s + 1);
      sample_interior(*bvh, o->sample_lo, o->sample_hi, B, seed, pts, sc, stream);
      wo.seed = seed ^ 0xD1B54A32D192ED03ull;
      status = n2w_wos_estimate(bvh, problem, pts, B, &wo, st, nullptr, ws, stream);
      if (status != N2W_OK) {
        err = n2w_last_error();
        break;
      }
      const int b = 256;
      labels_kernel<<<static_cast<unsigned>((B + b - 1) / b), b, 0, stream>>>(
          pts, sum, cnt, B, make_float3(o->input_min[0], o->input_min[1], o->input_min[2]),
          make_float3(o->input_extent[0], o->input_extent[1], o->input_extent[2]), inputs, targets);
      N2W_CUDA(cudaGetLastError());
      // local mean gradient and loss sum -> summed over ranks -> Adam on the mean
      status = n2w_cache_gradients(cache, inputs, targets, B, nullptr, stream);
      if (status == N2W_OK && world > 1) {
        status = n2w_comm_allreduce(comm, d_grad, d_grad, n_params, N2W_DTYPE_F32, N2W_OP_SUM, stream);
        if (status == N2W_OK) status = n2w_comm_allreduce(comm, d_loss, d_loss, 1, N2W_DTYPE_F32, N2W_OP_SUM, stream);
      }
      if (status == N2W_OK) status = n2w_cache_apply_gradients(cache, 1.0f / static_cast<float>(world), stream);
      if (status != N2W_OK) {
        err = n2w_last_error();
        break;
      }
      if (h_losses) {
        float l = 0.0f;
        N2W_CUDA(cudaMemcpyAsync(&l, d_loss, sizeof(float), cudaMemcpyDeviceToHost, stream));
        N2W_CUDA(cudaStreamSynchronize(stream));
        h_losses[s] = l / static_cast<float>(B * world);
      }
    }
    for (void* p : {static_cast<void*>(pts), static_cast<void*>(inputs), static_cast<void*>(targets),
                    static_cast<void*>(sum), static_cast<void*>(sum2), static_cast<void*>(cnt),
                    static_cast<void*>(steps), static_cast<void*>(forced), static_cast<void*>(sc), ws}) {
      scratch_free(p, stream);
    }
    if (status != N2W_OK) throw Error(status, err);
  });
}

int n2w_nc_progressive(n2w_cache* theta_train, n2w_cache* theta_infer, const n2w_bvh* bvh,
                       const n2w_problem* problem, const n2w_vec3* d_points, int64_t n,
                       const n2w_nc_progressive_options* o, n2w_point_stats coarse, n2w_point_stats residual,
                       n2w_nc_progressive_block* h_blocks, n2w_stream_t eval_stream, n2w_stream_t train_stream) {
  std::vector<cudaEvent_t> ev;
  void* scratch = nullptr;
  const int st = guarded([&] {
    N2W_REQUIRE(theta_train && theta_infer && bvh && problem && o, "n2w_nc_progressive: null argument");
    N2W_REQUIRE(theta_train != theta_infer, "theta_train and theta_infer must be different caches");
    N2W_REQUIRE(o->blocks >= 1 && o->train_steps_per_block >= 0, "invalid block options");
    N2W_REQUIRE(o->overlap == 0 || o->overlap == 1, "overlap must be 0 or 1");
    N2W_REQUIRE(n >= 1 && d_points, "n2w_nc_progressive: need points");
    const n2w_nc2lmc_options& eo = o->estimate;
    N2W_REQUIRE(eo.coarse_walks >= 0 && eo.residual_walks >= 0 && (eo.coarse_walks > 0 || eo.residual_walks > 0),
                "invalid walk counts");
    N2W_REQUIRE(eo.coarse_walks == 0 || (coarse.d_sum && coarse.d_sum_sq && coarse.d_count), "null coarse outputs");
    N2W_REQUIRE(eo.residual_walks == 0 || (residual.d_sum && residual.d_sum_sq && residual.d_count),
                "null residual outputs");
    const cudaStream_t es = eval_stream;
    const cudaStream_t ts = o->overlap ? train_stream : eval_stream;
    N2W_REQUIRE(!o->overlap || ts != es, "overlap needs two distinct streams");
    auto zero = [&](const n2w_point_stats& s) {
      if (!s.d_sum) return;
      N2W_CUDA(cudaMemsetAsync(s.d_sum, 0, sizeof(double) * n, es));
      N2W_CUDA(cudaMemsetAsync(s.d_sum_sq, 0, sizeof(double) * n, es));
      N2W_CUDA(cudaMemsetAsync(s.d_count, 0, sizeof(uint32_t) * n, es));
      if (s.d_steps) N2W_CUDA(cudaMemsetAsync(s.d_steps, 0, sizeof(uint64_t) * n, es));
      if (s.d_forced) N2W_CUDA(cudaMemsetAsync(s.d_forced, 0, sizeof(uint32_t) * n, es));
    };
    zero(coarse);
    zero(residual);
    // one block's statistics: coarse sum, sum_sq, steps; residual sum, sum_sq, steps (8 B);
    // coarse count, forced; residual count, forced (4 B)
    const size_t per = static_cast<size_t>(n);
    scratch = scratch_alloc(per * (6 * 8 + 4 * 4), es);
    double* d = static_cast<double*>(scratch);
    n2w_point_stats bc{d, d + per, reinterpret_cast<uint32_t*>(d + 6 * per),
                       reinterpret_cast<uint64_t*>(d + 2 * per), reinterpret_cast<uint32_t*>(d + 6 * per) + per};
    n2w_point_stats br{d + 3 * per, d + 4 * per, reinterpret_cast<uint32_t*>(d + 6 * per) + 2 * per,
                       reinterpret_cast<uint64_t*>(d + 5 * per), reinterpret_cast<uint32_t*>(d + 6 * per) + 3 * per};
    ev.resize(6);
    for (auto& e : ev) N2W_CUDA(cudaEventCreate(&e));
    for (int k = 0; k < o->blocks; ++k) {
      // 1. freeze the snapshot (both streams are idle here)
      N2W_CUDA(cudaEventRecord(ev[0], es));
      const int rc_copy = n2w_cache_copy_params(theta_infer, theta_train, es);
      if (rc_copy != N2W_OK) throw Error(rc_copy, n2w_last_error());
      N2W_CUDA(cudaEventRecord(ev[1], es));
      // 2. estimate with theta_infer
      n2w_nc2lmc_options bo = eo;
      bo.seed = eo.seed + 0x9E3779B97F4A7C15ull * static_cast<uint64_t>(k + 1) * 0x100000001ull;
      const int rc_est = n2w_nc2lmc_estimate_ex(bvh, problem, theta_infer, d_points, n, &bo, bc, br, nullptr, es);
      if (rc_est != N2W_OK) throw Error(rc_est, n2w_last_error());
      const int g = static_cast<int>(std::min<int64_t>((n + 255) / 256, 65535));
      if (eo.coarse_walks > 0) accumulate_stats_kernel<<<g, 256, 0, es>>>(bc, coarse, n);
      if (eo.residual_walks > 0) accumulate_stats_kernel<<<g, 256, 0, es>>>(br, residual, n);
      N2W_CUDA(cudaGetLastError());
      N2W_CUDA(cudaEventRecord(ev[2], es));
      // 3. train toward the next snapshot
      const bool train = k + 1 < o->blocks && o->train_steps_per_block > 0;
      N2W_CUDA(cudaEventRecord(ev[3], ts));
      if (train) {
        n2w_nc_train_options to = o->train;
        to.steps = o->train_steps_per_block;
        to.seed = o->train.seed + 0xD1B54A32D192ED03ull * static_cast<uint64_t>(k + 1);
        const int rc_tr = n2w_nc_train(theta_train, bvh, problem, &to, nullptr, ts);
        if (rc_tr != N2W_OK) throw Error(rc_tr, n2w_last_error());
      }
      N2W_CUDA(cudaEventRecord(ev[4], ts));
      // 4. block boundary
      N2W_CUDA(cudaStreamSynchronize(es));
      if (ts != es) N2W_CUDA(cudaStreamSynchronize(ts));
      if (h_blocks) {
        float e_ms = 0.0f, t_ms = 0.0f, w0 = 0.0f, w1 = 0.0f;
        N2W_CUDA(cudaEventElapsedTime(&e_ms, ev[1], ev[2]));
        N2W_CUDA(cudaEventElapsedTime(&t_ms, ev[3], ev[4]));
        N2W_CUDA(cudaEventElapsedTime(&w0, ev[0], ev[2]));
        N2W_CUDA(cudaEventElapsedTime(&w1, ev[0], ev[4]));
        h_blocks[k] = n2w_nc_progressive_block{e_ms, train ? t_ms : 0.0f, std::max(w0, w1), 0.0f};
      }
    }
  });
  if (scratch) cudaFreeAsync(scratch, eval_stream);  // no throw on the error path
  for (auto& e : ev) {
    if (e) cudaEventDestroy(e);
  }
  return st;
}

int n2w_nc_update_labels(const n2w_bvh* bvh, const n2w_problem* problem, const n2w_vec3* d_points, int64_t n,
                         const n2w_nc_label_options* o, n2w_point_stats accum, float* d_inputs, float* d_targets,
                         void* d_workspace, n2w_stream_t stream) {
  return guarded([&] {
    N2W_REQUIRE(bvh && problem && o, "n2w_nc_update_labels: null argument");
    N2W_REQUIRE(n >= 0, "n must be non-negative");
    N2W_REQUIRE(o->label_source == N2W_LABEL_EXACT || o->label_source == N2W_LABEL_WOS, "bad label_source");
    if (n == 0) return;
    N2W_REQUIRE(d_points && d_inputs && d_targets, "n2w_nc_update_labels: null device pointer");
    const float3 in_min = make_float3(o->input_min[0], o->input_min[1], o->input_min[2]);
    const float3 in_ext = make_float3(o->input_extent[0], o->input_extent[1], o->input_extent[2]);
    const int b = 256;
    const unsigned grid = static_cast<unsigned>((n + b - 1) / b);
    if (o->label_source == N2W_LABEL_EXACT) {
      map_to_unit_kernel<<<grid, b, 0, stream>>>(d_points, n, in_min, in_ext, d_inputs);
      N2W_CUDA(cudaGetLastError());
      launch_exact(*problem, d_points, n, d_targets, stream);
      return;
    }
    N2W_REQUIRE(o->walks_per_point > 0, "walks_per_point must be positive");
    N2W_REQUIRE(accum.d_sum && accum.d_sum_sq && accum.d_count && accum.d_steps && accum.d_forced,
                "WoS labels need the running accumulators");
    n2w_walk_options wo{};
    wo.walks_per_point = o->walks_per_point;
    wo.max_steps = o->max_steps;
    wo.epsilon = o->epsilon;
    wo.step_scale = o->step_scale;
    wo.seed = o->seed + 0x9E3779B97F4A7C15ull * static_cast<uint64_t>(o->refresh_index + 1);
    wo.block_size = o->block_size;
    wo.accumulate = 1;
    const int st = n2w_wos_estimate(bvh, problem, d_points, n, &wo, accum, nullptr, d_workspace, stream);
    if (st != N2W_OK) throw Error(st, n2w_last_error());
    labels_kernel<<<grid, b, 0, stream>>>(d_points, accum.d_sum, accum.d_count, n, in_min, in_ext, d_inputs,
                                          d_targets);
    N2W_CUDA(cudaGetLastError());
  });
}

int n2w_nc2lmc_estimate(const n2w_bvh* bvh, const n2w_problem* problem, const n2w_cache* cache,
                        const n2w_vec3* d_points, int64_t n, const n2w_nc2lmc_options* o,
                        n2w_point_stats coarse, n2w_point_stats residual, n2w_stream_t stream) {
  if (!cache) {
    set_last_error("n2w_nc2lmc_estimate: null cache (n2w_nc2lmc_estimate_ex takes NULL for the analytic cache)");
    return N2W_EINVAL;
  }
  return n2w_nc2lmc_estimate_ex(bvh, problem, cache, d_points, n, o, coarse, residual, nullptr, stream);
}

int n2w_nc2lmc_estimate_ex(const n2w_bvh* bvh, const n2w_problem* problem, const n2w_cache* cache,
                           const n2w_vec3* d_points, int64_t n, const n2w_nc2lmc_options* o,
                           n2w_point_stats coarse, n2w_point_stats residual, n2w_nc2lmc_counters* d_counters,
                           n2w_stream_t stream) {
  return guarded([&] {
    N2W_REQUIRE(bvh && problem && o, "null argument");
    N2W_REQUIRE(n >= 0, "n must be non-negative");
    N2W_REQUIRE(o->coarse_walks >= 0 && o->residual_walks >= 0 && o->depth_m >= 0 &&
                    (o->coarse_walks > 0 || o->residual_walks > 0),
                "invalid walk counts");
    if (n == 0) return;
    N2W_REQUIRE(d_points, "null points");
    N2W_REQUIRE(o->coarse_walks == 0 || (coarse.d_sum && coarse.d_sum_sq && coarse.d_count), "null coarse outputs");
    N2W_REQUIRE(o->residual_walks == 0 || (residual.d_sum && residual.d_sum_sq && residual.d_count),
                "null residual outputs");
    const int64_t wmax = std::max(o->coarse_walks, o->residual_walks);
    // Auto batch: up to 2^24 samples per level launch (45 B of per-sample
    // scratch each, ~0.75 GB), so a launch holds enough walks to fill the GPU
    // (with 2^22, 1,024 coarse walks meant 4,096-point launches whose tails
    // cost ~30 % of a block of the time-to-MSE run).
    const int64_t batch = std::min<int64_t>(
        n, o->point_batch > 0 ? o->point_batch : std::max<int64_t>(1, (int64_t{1} << 24) / wmax));
    const int64_t maxS = batch * std::max(o->coarse_walks, o->residual_walks);
    float* inp = stream_alloc<float>(3 * maxS, stream);
    float* bnd = stream_alloc<float>(maxS, stream);
    float* cont = stream_alloc<float>(maxS, stream);
    uint8_t* needs = stream_alloc<uint8_t>(maxS, stream);
    int* stp = stream_alloc<int>(maxS, stream);
    int* frc = stream_alloc<int>(maxS, stream);
    int* ovf = stream_alloc<int>(maxS, stream);
    float* cval = stream_alloc<float>(maxS, stream);
    float* ncv = stream_alloc<float>(maxS, stream);
    float* res = stream_alloc<float>(maxS, stream);
    auto zero = [&](const n2w_point_stats& s) {
      N2W_CUDA(cudaMemsetAsync(s.d_sum, 0, sizeof(double) * n, stream));
      N2W_CUDA(cudaMemsetAsync(s.d_sum_sq, 0, sizeof(double) * n, stream));
      N2W_CUDA(cudaMemsetAsync(s.d_count, 0, sizeof(uint32_t) * n, stream));
      if (s.d_steps) N2W_CUDA(cudaMemsetAsync(s.d_steps, 0, sizeof(uint64_t) * n, stream));
      if (s.d_forced) N2W_CUDA(cudaMemsetAsync(s.d_forced, 0, sizeof(uint32_t) * n, stream));
    };
    if (o->coarse_walks > 0) zero(coarse);
    if (o->residual_walks > 0) zero(residual);
    int status = N2W_OK;
    std::string err;
    auto run_level = [&](int mode, int walks, n2w_point_stats& out, int64_t p0, int64_t np) {
      if (status != N2W_OK || walks == 0) return;
      n2w_walk_options wo{};
      wo.walks_per_point = walks;
      wo.max_steps = o->max_steps;
      wo.depth_m = o->depth_m;
      wo.epsilon = o->epsilon;
      wo.step_scale = o->step_scale;
      wo.seed = o->seed + static_cast<uint64_t>(p0) * 0x9E3779B97F4A7C15ull;
      const int64_t S = np * walks;
      status = n2w_wos_prefix_samples(bvh, problem, d_points + p0, np, &wo, mode, o->input_min, o->input_extent,
                                      inp, bnd, mode == N2W_WALK_RESIDUAL ? cont : nullptr, needs, stp, frc, ovf,
                                      stream);
      if (status == N2W_OK) {
        if (cache) {
          status = n2w_cache_infer(cache, inp, S, cval, stream);
        } else {
          launch_oracle_cache(*problem, inp, S, o->input_min, o->input_extent, cval, stream);
        }
      }
      if (status == N2W_OK && d_counters) {
        unsigned long long* c = reinterpret_cast<unsigned long long*>(d_counters) + (mode == N2W_WALK_PREFIX ? 0 : 3);
        launch_count_samples(needs, frc, ovf, S, c, stream);
      }
      if (status == N2W_OK && mode == N2W_WALK_PREFIX) {
        // coarse value = A + needs * C; the combine kernel needs a continuation array
        status = n2w_wos_combine(cval, bnd, bnd, needs, S, ncv, res, 256, stream);
      } else if (status == N2W_OK) {
        status = n2w_wos_combine(cval, bnd, cont, needs, S, ncv, res, 256, stream);
      }
      n2w_point_stats part = out;
      part.d_sum += p0;
      part.d_sum_sq += p0;
      part.d_count += p0;
      if (part.d_steps) part.d_steps += p0;
      if (part.d_forced) part.d_forced += p0;
      if (status == N2W_OK) {
        status = n2w_reduce_samples(mode == N2W_WALK_PREFIX ? ncv : res, part.d_steps ? stp : nullptr,
                                    part.d_forced ? frc : nullptr, np, walks, part, 1, stream);
      }
      if (status != N2W_OK) err = n2w_last_error();
    };
    for (int64_t p0 = 0; p0 < n && status == N2W_OK; p0 += batch) {
      const int64_t np = std::min(batch, n - p0);
      run_level(N2W_WALK_PREFIX, o->coarse_walks, coarse, p0, np);
      run_level(N2W_WALK_RESIDUAL, o->residual_walks, residual, p0, np);
    }
    for (void* p : {static_cast<void*>(inp), static_cast<void*>(bnd), static_cast<void*>(cont),
                    static_cast<void*>(needs), static_cast<void*>(stp), static_cast<void*>(frc),
                    static_cast<void*>(ovf), static_cast<void*>(cval), static_cast<void*>(ncv),
                    static_cast<void*>(res)}) {
      scratch_free(p, stream);
    }
    if (status != N2W_OK) throw Error(status, err);
  });
}

}  // extern "C"
