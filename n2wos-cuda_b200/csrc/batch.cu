// Batched Walk-on-Spheres: many PDE instances of uneven sizes, on several
// meshes, in ONE persistent walker launch.
//
//  * A scene merges the BVHs of several meshes into one device layout: node
//    arrays, triangle arrays and seed-grid slots are concatenated and every
//    child reference / slot is rebased, so a walker only needs its instance's
//    root node index to query its own mesh.
//  * A batch is a fixed table of instances (mesh, problem, points, walks per
//    point, seed, per-point accumulators).  Their chunks form one global queue,
//    so instances with few points or short walks never leave SMs idle while
//    others still have work.
//  * A launch is memsets + two kernels and is stream-capturable; the batch can
//    hold an instantiated CUDA graph of itself and replay it.
//  * An autotuner times candidate launch shapes (threads per block, register
//    budget, chunk size, regeneration threshold) on a subsample of the batch
//    and keeps the fastest.
//
// Each instance's walks are keyed by (instance seed; point index within the
// instance, walk index), exactly as n2w_wos_estimate keys them, so an
// instance's estimates do not depend on what else is in the batch (up to the
// order of FP64 additions).  The reference runs one problem per launch; this
// is the batched form of its persistent walker (src/cuda/cubql_bvh.cu:263-336).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "internal.hpp"
#include "philox.cuh"
#include "problem.cuh"
#include "scene.hpp"
#include "walker.cuh"

struct n2w_batch {
  const n2w_scene* scene = nullptr;
  int n_items = 0;
  int64_t total_points = 0, total_chunks = 0;
  n2w_walk_options opt{};
  int reg_variant = 0;
  std::vector<n2w_batch_item> items;
  std::vector<n2w_problem> problems;
  std::vector<n2w::BatchInst> h_insts;
  n2w::BatchInst* d_insts = nullptr;
  n2w_problem* d_problems = nullptr;
  float4* d_cpd = nullptr;
  int2* d_ids = nullptr;
  char* d_hdr = nullptr;  // [0,8) queue counter, [256,320) run counters
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
};

namespace n2w {
namespace {

__global__ void rebase_nodes_kernel(const Node4* __restrict__ src, int64_t n, Node4* __restrict__ dst,
                                    int32_t node_off, int32_t tri_off) {
  const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n) return;
  Node4 nd = src[i];
#pragma unroll
  for (int c = 0; c < 4; ++c) {
    const int32_t r = nd.child[c];
    if (r >= 0) nd.child[c] = r + node_off;
    else if (r != kEmptyChild) nd.child[c] = leaf_ref(leaf_first(r) + tri_off, leaf_count(r));
  }
  dst[i] = nd;
}

__global__ void rebase_slots_kernel(const int* __restrict__ src, int64_t n, int* __restrict__ dst, int32_t tri_off) {
  const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i < n) dst[i] = src[i] + tri_off;
}

// Zeroes the per-point accumulators of every instance (global point index i).
__global__ void zero_batch_stats_kernel(const BatchInst* __restrict__ insts, int n_insts, int64_t n) {
  const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int lo = 0, hi = n_insts - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (insts[mid].point_base <= i) lo = mid;
    else hi = mid - 1;
  }
  const BatchInst& I = insts[lo];
  const int64_t q = i - I.point_base;
  I.sum[q] = 0.0;
  I.sum_sq[q] = 0.0;
  I.count[q] = 0u;
  I.steps[q] = 0ull;
  I.forced[q] = 0u;
}

unsigned blocks_of(int64_t n, int b) { return static_cast<unsigned>((n + b - 1) / b); }

void free_graph(n2w_batch& b) {
  if (b.exec) cudaGraphExecDestroy(b.exec);
  if (b.graph) cudaGraphDestroy(b.graph);
  b.exec = nullptr;
  b.graph = nullptr;
}

// Builds the instance table (host) from the items and current options.
void build_instances(n2w_batch& b) {
  const n2w_scene& sc = *b.scene;
  const int chunk = b.opt.chunk > 0 ? b.opt.chunk : kDefaultChunk;
  b.h_insts.assign(b.n_items, BatchInst{});
  int64_t pbase = 0, cbase = 0;
  for (int k = 0; k < b.n_items; ++k) {
    const n2w_batch_item& it = b.items[k];
    BatchInst& I = b.h_insts[k];
    I.points = it.d_points;
    I.sum = it.stats.d_sum;
    I.sum_sq = it.stats.d_sum_sq;
    I.count = it.stats.d_count;
    I.steps = it.stats.d_steps;
    I.forced = it.stats.d_forced;
    I.point_base = pbase;
    I.point_count = it.point_count;
    I.chunk_base = cbase;
    I.chunks_per_point = (it.walks_per_point + chunk - 1) / chunk;
    I.walks_per_point = it.walks_per_point;
    set_instance_geometry(I, sc, it.mesh);
    set_instance_problem(I, b.problems[it.problem], b.d_problems + it.problem);
    philox_key(it.seed, 0u, I.k0, I.k1);
    I.wid_base = 0;
    pbase += it.point_count;
    cbase += it.point_count * I.chunks_per_point;
  }
  b.total_points = pbase;
  b.total_chunks = cbase;
}

void upload_instances(n2w_batch& b, cudaStream_t s) {
  N2W_CUDA(cudaMemcpyAsync(b.d_insts, b.h_insts.data(), sizeof(BatchInst) * b.h_insts.size(),
                           cudaMemcpyHostToDevice, s));
  N2W_CUDA(cudaStreamSynchronize(s));
}

WalkArgs batch_args(const n2w_batch& b, n2w_walk_counters* d_counters) {
  WalkArgs a{};
  a.nodes = reinterpret_cast<const float4*>(b.scene->d_nodes);
  a.tris = reinterpret_cast<const float4*>(b.scene->d_tris);
  a.first_cpd = b.d_cpd;
  a.first_ids = b.d_ids;
  a.total_chunks = b.total_chunks;
  a.chunk = b.opt.chunk > 0 ? b.opt.chunk : kDefaultChunk;
  a.regen = b.opt.regen_threshold > 0 ? b.opt.regen_threshold : kDefaultRegen;
  a.max_steps = b.opt.max_steps;
  a.eps = b.opt.epsilon;
  a.step_scale = b.opt.step_scale;
  a.deadline_ns = b.opt.deadline_ns;
  a.queue = reinterpret_cast<unsigned long long*>(b.d_hdr);
  a.counters = d_counters ? d_counters : reinterpret_cast<n2w_walk_counters*>(b.d_hdr + 256);
  a.insts = b.d_insts;
  a.n_insts = b.n_items;
  return a;
}

// The launch itself: stream-ordered, no allocation, no host synchronisation.
void launch_batch(const n2w_batch& b, n2w_walk_counters* d_counters, cudaStream_t s) {
  N2W_CUDA(cudaMemsetAsync(b.d_hdr, 0, 512, s));
  if (d_counters) N2W_CUDA(cudaMemsetAsync(d_counters, 0, sizeof(n2w_walk_counters), s));
  if (b.total_points == 0) return;
  if (!b.opt.accumulate) {
    zero_batch_stats_kernel<<<blocks_of(b.total_points, 256), 256, 0, s>>>(b.d_insts, b.n_items, b.total_points);
    N2W_CUDA(cudaGetLastError());
  }
  const WalkArgs a = batch_args(b, d_counters);
  launch_first_query_batch(a, b.total_points, b.d_cpd, b.d_ids, s);
  launch_walker_batch(a, b.opt.block_size > 0 ? b.opt.block_size : kDefaultWalkerThreads, b.opt.blocks_per_sm,
                      b.reg_variant, s);
}

void release_batch(n2w_batch* b) {
  if (!b) return;
  free_graph(*b);
  cudaFree(b->d_insts);
  cudaFree(b->d_problems);
  cudaFree(b->d_cpd);
  cudaFree(b->d_ids);
  cudaFree(b->d_hdr);
  delete b;
}

void check_tunables(const n2w_walk_options& o) {
  N2W_REQUIRE(o.max_steps > 0, "max_steps must be positive");
  N2W_REQUIRE(o.epsilon > 0.0f, "epsilon must be positive");
  N2W_REQUIRE(o.step_scale > 0.0f && o.step_scale <= 1.0f, "step_scale must be in (0, 1]");
  N2W_REQUIRE(o.block_size == 0 || (o.block_size >= 32 && o.block_size <= kWalkerMaxThreads && o.block_size % 32 == 0),
              "walker block_size must be 0 or a multiple of 32 in [32, 256]");
  N2W_REQUIRE(o.chunk >= 0 && o.chunk <= 1024, "chunk must be in [0, 1024]");
  N2W_REQUIRE(o.regen_threshold >= 0 && o.regen_threshold <= 32, "regen_threshold must be in [0, 32]");
  N2W_REQUIRE(o.blocks_per_sm >= 0, "blocks_per_sm must be non-negative");
}

}  // namespace
}  // namespace n2w

using namespace n2w;

extern "C" {

int n2w_scene_create(const n2w_bvh* const* bvhs, int count, n2w_scene** out) {
  n2w_scene* sc = nullptr;
  const int st = guarded([&] {
    N2W_REQUIRE(out && bvhs && count > 0, "n2w_scene_create: invalid arguments");
    sc = new n2w_scene();
    N2W_CUDA(cudaGetDevice(&sc->device));
    sc->meshes.resize(count);
    for (int k = 0; k < count; ++k) {
      const n2w_bvh* b = bvhs[k];
      N2W_REQUIRE(b && b->d_nodes && b->d_tris, "n2w_scene_create: null BVH");
      N2W_REQUIRE(b->device == sc->device, "n2w_scene_create: BVH on another device");
      auto& m = sc->meshes[k];
      m.node_off = sc->nodes;
      m.tri_off = sc->tris;
      m.root = static_cast<int32_t>(m.node_off);
      m.triangles = b->stats.triangles;
      sc->nodes += b->stats.nodes;
      sc->tris += b->stats.triangles;
      if (b->d_seed) {
        const int64_t s = static_cast<int64_t>(b->seed_n) + 1;
        m.slot_off = sc->slots;
        sc->slots += s * s * s;
        for (int a = 0; a < 3; ++a) {
          m.seed_lo[a] = b->seed_lo[a];
          m.box_lo[a] = b->seed_lo[a];
          m.box_hi[a] = b->seed_lo[a] + b->seed_h * static_cast<float>(b->seed_n);
        }
        m.seed_h = b->seed_h;
        m.seed_n = b->seed_n;
      }
    }
    N2W_REQUIRE(sc->nodes < (int64_t{1} << 31) && sc->tris < (int64_t{1} << 28),
                "n2w_scene_create: merged scene exceeds 2^31 nodes or 2^28 triangles");
    N2W_CUDA(cudaMalloc(&sc->d_nodes, sizeof(Node4) * sc->nodes));
    N2W_CUDA(cudaMalloc(&sc->d_tris, sizeof(TriRec) * sc->tris));
    if (sc->slots) N2W_CUDA(cudaMalloc(&sc->d_slots, sizeof(int) * sc->slots));
    for (int k = 0; k < count; ++k) {
      const n2w_bvh* b = bvhs[k];
      const auto& m = sc->meshes[k];
      rebase_nodes_kernel<<<blocks_of(b->stats.nodes, 256), 256>>>(b->d_nodes, b->stats.nodes,
                                                                    sc->d_nodes + m.node_off,
                                                                    static_cast<int32_t>(m.node_off),
                                                                    static_cast<int32_t>(m.tri_off));
      N2W_CUDA(cudaGetLastError());
      N2W_CUDA(cudaMemcpy(sc->d_tris + m.tri_off, b->d_tris, sizeof(TriRec) * b->stats.triangles,
                          cudaMemcpyDeviceToDevice));
      if (m.slot_off >= 0) {
        const int64_t s = static_cast<int64_t>(b->seed_n) + 1;
        rebase_slots_kernel<<<blocks_of(s * s * s, 256), 256>>>(b->d_seed, s * s * s, sc->d_slots + m.slot_off,
                                                                static_cast<int32_t>(m.tri_off));
        N2W_CUDA(cudaGetLastError());
      }
    }
    N2W_CUDA(cudaDeviceSynchronize());
    *out = sc;
  });
  if (st != N2W_OK && sc) n2w_scene_destroy(sc);
  return st;
}

int n2w_scene_info(const n2w_scene* scene, int* mesh_count, int64_t* nodes, int64_t* triangles,
                   int64_t* device_bytes) {
  return guarded([&] {
    N2W_REQUIRE(scene, "null scene");
    if (mesh_count) *mesh_count = static_cast<int>(scene->meshes.size());
    if (nodes) *nodes = scene->nodes;
    if (triangles) *triangles = scene->tris;
    if (device_bytes) {
      *device_bytes = scene->nodes * static_cast<int64_t>(sizeof(Node4)) +
                      scene->tris * static_cast<int64_t>(sizeof(TriRec)) + scene->slots * 4;
    }
  });
}

void n2w_scene_destroy(n2w_scene* scene) {
  if (!scene) return;
  cudaFree(scene->d_nodes);
  cudaFree(scene->d_tris);
  cudaFree(scene->d_slots);
  delete scene;
}

int n2w_batch_create(const n2w_scene* scene, const n2w_problem* problems, int problem_count,
                     const n2w_batch_item* items, int item_count, const n2w_walk_options* options,
                     n2w_batch** out) {
  n2w_batch* b = nullptr;
  const int st = guarded([&] {
    N2W_REQUIRE(scene && problems && items && options && out, "n2w_batch_create: null argument");
    N2W_REQUIRE(problem_count > 0 && item_count > 0, "n2w_batch_create: empty problem or item list");
    check_tunables(*options);
    for (int p = 0; p < problem_count; ++p) validate_problem(problems[p]);
    const int nm = static_cast<int>(scene->meshes.size());
    for (int k = 0; k < item_count; ++k) {
      const n2w_batch_item& it = items[k];
      const std::string where = "item " + std::to_string(k) + ": ";
      N2W_REQUIRE(it.mesh >= 0 && it.mesh < nm, where + "mesh index out of range");
      N2W_REQUIRE(it.problem >= 0 && it.problem < problem_count, where + "problem index out of range");
      N2W_REQUIRE(it.point_count >= 0, where + "negative point count");
      N2W_REQUIRE(it.walks_per_point > 0, where + "walks_per_point must be positive");
      N2W_REQUIRE(it.point_count == 0 || (it.d_points && it.stats.d_sum && it.stats.d_sum_sq && it.stats.d_count &&
                                          it.stats.d_steps && it.stats.d_forced),
                  where + "null device pointer");
    }
    b = new n2w_batch();
    b->scene = scene;
    b->n_items = item_count;
    b->opt = *options;
    b->items.assign(items, items + item_count);
    b->problems.assign(problems, problems + problem_count);
    N2W_CUDA(cudaMalloc(&b->d_problems, sizeof(n2w_problem) * problem_count));
    N2W_CUDA(cudaMemcpy(b->d_problems, problems, sizeof(n2w_problem) * problem_count, cudaMemcpyHostToDevice));
    N2W_CUDA(cudaMalloc(&b->d_insts, sizeof(BatchInst) * item_count));
    N2W_CUDA(cudaMalloc(&b->d_hdr, 512));
    build_instances(*b);
    N2W_CUDA(cudaMalloc(&b->d_cpd, sizeof(float4) * std::max<int64_t>(b->total_points, 1)));
    N2W_CUDA(cudaMalloc(&b->d_ids, sizeof(int2) * std::max<int64_t>(b->total_points, 1)));
    upload_instances(*b, nullptr);
    *out = b;
  });
  if (st != N2W_OK && b) release_batch(b);
  return st;
}

int n2w_batch_info(const n2w_batch* batch, int64_t* total_points, int64_t* total_walks,
                   n2w_walk_options* options_out, int* reg_variant_out) {
  return guarded([&] {
    N2W_REQUIRE(batch, "null batch");
    if (total_points) *total_points = batch->total_points;
    if (total_walks) {
      int64_t w = 0;
      for (const auto& it : batch->items) w += it.point_count * static_cast<int64_t>(it.walks_per_point);
      *total_walks = w;
    }
    if (options_out) *options_out = batch->opt;
    if (reg_variant_out) *reg_variant_out = batch->reg_variant;
  });
}

int n2w_batch_set_seeds(n2w_batch* batch, const uint64_t* seeds, n2w_stream_t stream) {
  return guarded([&] {
    N2W_REQUIRE(batch && seeds, "null argument");
    for (int k = 0; k < batch->n_items; ++k) {
      batch->items[k].seed = seeds[k];
      philox_key(seeds[k], 0u, batch->h_insts[k].k0, batch->h_insts[k].k1);
    }
    // The instance table lives at a fixed address, so a captured graph sees the new keys.
    upload_instances(*batch, stream);
  });
}

int n2w_batch_launch(n2w_batch* batch, n2w_walk_counters* d_counters, n2w_stream_t stream) {
  return guarded([&] {
    N2W_REQUIRE(batch, "null batch");
    launch_batch(*batch, d_counters, stream);
  });
}

int n2w_batch_capture_graph(n2w_batch* batch, n2w_walk_counters* d_counters, n2w_stream_t stream) {
  return guarded([&] {
    N2W_REQUIRE(batch, "null batch");
    N2W_REQUIRE(stream != nullptr, "graph capture needs a non-default stream");
    free_graph(*batch);
    N2W_CUDA(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
    try {
      launch_batch(*batch, d_counters, stream);
    } catch (...) {
      cudaGraph_t g = nullptr;
      cudaStreamEndCapture(stream, &g);
      if (g) cudaGraphDestroy(g);
      throw;
    }
    N2W_CUDA(cudaStreamEndCapture(stream, &batch->graph));
    N2W_CUDA(cudaGraphInstantiate(&batch->exec, batch->graph, 0));
  });
}

int n2w_batch_graph_launch(n2w_batch* batch, n2w_stream_t stream) {
  return guarded([&] {
    N2W_REQUIRE(batch && batch->exec, "no captured graph (call n2w_batch_capture_graph first)");
    N2W_CUDA(cudaGraphLaunch(batch->exec, stream));
  });
}

int n2w_batch_autotune(n2w_batch* batch, double sample_fraction, n2w_batch_tuning* best_out,
                       n2w_batch_tuning* trials_out, int trials_cap, int* trials_count, n2w_stream_t stream) {
  return guarded([&] {
    N2W_REQUIRE(batch, "null batch");
    N2W_REQUIRE(sample_fraction > 0.0 && sample_fraction <= 1.0, "sample_fraction must be in (0, 1]");
    // Probe batch: the first max(min(n, 64), ceil(f * n)) points of every item,
    // written into scratch accumulators so the caller's statistics are untouched.
    std::vector<n2w_batch_item> probe(batch->items);
    int64_t total = 0;
    for (auto& it : probe) {
      const int64_t want = static_cast<int64_t>(std::ceil(sample_fraction * static_cast<double>(it.point_count)));
      it.point_count = std::min(it.point_count, std::max<int64_t>(want, std::min<int64_t>(it.point_count, 64)));
      total += it.point_count;
    }
    void* scratch = nullptr;
    N2W_CUDA(cudaMalloc(&scratch, 32 * static_cast<size_t>(std::max<int64_t>(total, 1))));
    char* base = static_cast<char*>(scratch);
    int64_t off = 0;
    for (auto& it : probe) {
      it.stats.d_sum = reinterpret_cast<double*>(base) + off;
      it.stats.d_sum_sq = reinterpret_cast<double*>(base + 8 * total) + off;
      it.stats.d_steps = reinterpret_cast<uint64_t*>(base + 16 * total) + off;
      it.stats.d_count = reinterpret_cast<uint32_t*>(base + 24 * total) + off;
      it.stats.d_forced = reinterpret_cast<uint32_t*>(base + 28 * total) + off;
      off += it.point_count;
    }
    n2w_batch* pb = nullptr;
    n2w_walk_options o = batch->opt;
    o.accumulate = 0;
    const int st = n2w_batch_create(batch->scene, batch->problems.data(), static_cast<int>(batch->problems.size()),
                                    probe.data(), static_cast<int>(probe.size()), &o, &pb);
    if (st != N2W_OK) {
      cudaFree(scratch);
      throw Error(st, n2w_last_error());
    }
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    std::vector<n2w_batch_tuning> trials;
    auto cleanup = [&] {
      if (e0) cudaEventDestroy(e0);
      if (e1) cudaEventDestroy(e1);
      release_batch(pb);
      cudaFree(scratch);
    };
    int bb = batch->opt.block_size > 0 ? batch->opt.block_size : kDefaultWalkerThreads;
    int br = batch->reg_variant;
    int bc = batch->opt.chunk > 0 ? batch->opt.chunk : kDefaultChunk;
    int bg = batch->opt.regen_threshold > 0 ? batch->opt.regen_threshold : kDefaultRegen;
    float best = INFINITY;
    try {
      N2W_CUDA(cudaEventCreate(&e0));
      N2W_CUDA(cudaEventCreate(&e1));
      auto time_cfg = [&](int block, int regv, int chunk, int regen) -> float {
        pb->opt.block_size = block;
        pb->opt.chunk = chunk;
        pb->opt.regen_threshold = regen;
        pb->reg_variant = regv;
        build_instances(*pb);  // the chunk size changes the queue layout
        upload_instances(*pb, stream);
        float t_best = INFINITY;
        for (int r = 0; r < 3; ++r) {  // the first run warms up; keep the best of the other two
          N2W_CUDA(cudaEventRecord(e0, stream));
          launch_batch(*pb, nullptr, stream);
          N2W_CUDA(cudaEventRecord(e1, stream));
          N2W_CUDA(cudaEventSynchronize(e1));
          float ms = 0.0f;
          N2W_CUDA(cudaEventElapsedTime(&ms, e0, e1));
          if (r > 0) t_best = std::min(t_best, ms);
        }
        n2w_batch_tuning t{};
        t.block_size = block;
        t.chunk = chunk;
        t.regen_threshold = regen;
        t.reg_variant = regv;
        t.ms = t_best;
        trials.push_back(t);
        return t_best;
      };
      // Coordinate search: (threads per block x register budget), then chunk, then regeneration.
      const int c0 = bc, g0 = bg;
      for (int block : {64, 128, 256}) {
        for (int regv : {0, 1}) {
          const float t = time_cfg(block, regv, c0, g0);
          if (t < best) {
            best = t;
            bb = block;
            br = regv;
          }
        }
      }
      for (int chunk : {2, 4, 8, 16}) {
        if (chunk == c0) continue;
        const float t = time_cfg(bb, br, chunk, g0);
        if (t < best) {
          best = t;
          bc = chunk;
        }
      }
      for (int regen : {4, 8, 12, 16, 24}) {
        if (regen == g0) continue;
        const float t = time_cfg(bb, br, bc, regen);
        if (t < best) {
          best = t;
          bg = regen;
        }
      }
    } catch (...) {
      cleanup();
      throw;
    }
    cleanup();
    // Apply the winner (the queue layout depends on the chunk size).
    batch->opt.block_size = bb;
    batch->opt.chunk = bc;
    batch->opt.regen_threshold = bg;
    batch->reg_variant = br;
    free_graph(*batch);
    build_instances(*batch);
    upload_instances(*batch, stream);
    if (best_out) {
      *best_out = n2w_batch_tuning{};
      best_out->block_size = bb;
      best_out->chunk = bc;
      best_out->regen_threshold = bg;
      best_out->reg_variant = br;
      best_out->ms = best;
    }
    if (trials_count) *trials_count = static_cast<int>(trials.size());
    if (trials_out) {
      for (int i = 0; i < std::min<int>(trials_cap, static_cast<int>(trials.size())); ++i) trials_out[i] = trials[i];
    }
  });
}

int n2w_batch_set_tuning(n2w_batch* batch, const n2w_batch_tuning* t, n2w_stream_t stream) {
  return guarded([&] {
    N2W_REQUIRE(batch && t, "null argument");
    n2w_walk_options o = batch->opt;
    o.block_size = t->block_size;
    o.blocks_per_sm = t->blocks_per_sm;
    o.chunk = t->chunk;
    o.regen_threshold = t->regen_threshold;
    check_tunables(o);
    N2W_REQUIRE(t->reg_variant == 0 || t->reg_variant == 1, "reg_variant must be 0 or 1");
    batch->opt = o;
    batch->reg_variant = t->reg_variant;
    free_graph(*batch);
    build_instances(*batch);
    upload_instances(*batch, stream);
  });
}

void n2w_batch_destroy(n2w_batch* batch) { release_batch(batch); }

}  // extern "C"
