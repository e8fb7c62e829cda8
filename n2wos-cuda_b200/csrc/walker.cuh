// Kernel argument block of the persistent walker (walker.cu).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "geom.cuh"
#include "n2w.h"

namespace n2w {

constexpr int kOutStats = 0;    // per-point FP64 accumulators
constexpr int kOutSamples = 1;  // per-sample value / steps / flags (reference layout)
constexpr int kOutPrefix = 2;   // per-sample prefix records for the cache levels

constexpr int kWalkerMaxThreads = 256;
// Resident 256-thread blocks the register budget must allow (64 registers per
// thread): the traversal hides L1/L2 latency with warps, so occupancy matters.
constexpr int kWalkerMinBlocks = 4;
constexpr int kDefaultWalkerThreads = 128;
constexpr int kDefaultChunk = 8;
constexpr int kDefaultRegen = 12;

// One instance of a batched launch: its geometry inside the merged scene, its
// problem, its points and accumulators, and its slice of the global chunk queue.
struct alignas(16) BatchInst {
  const n2w_vec3* points;       // this instance's points
  const n2w_problem* problem;   // device copy of its problem
  double* sum;                  // per-point accumulators (local point index)
  double* sum_sq;
  uint32_t* count;
  uint64_t* steps;
  uint32_t* forced;
  int64_t point_base;           // first global point index (first-query cache)
  int64_t point_count;
  int64_t chunk_base;           // first global chunk of this instance
  int64_t chunks_per_point;
  dev::SeedGrid grid;           // slots already rebased into the merged scene
  float box_lo[3], box_hi[3];   // domain box (walks never leave it)
  int32_t walks_per_point;
  int32_t root;                 // root node of this instance's mesh in the scene
  uint32_t k0, k1;              // Philox key of the instance
  int32_t has_source, source_center, source_samples, pad;
  int64_t wid_base;             // added to every walk id (a point range of a larger request)
};

struct WalkArgs {
  const float4* nodes;
  const float4* tris;
  dev::SeedGrid grid;
  float box_lo[3], box_hi[3];  // domain box: the mesh box grown by 20 % (walks never leave it)
  const n2w_vec3* points;
  // Per-point first query (closest point + d2, id + slot): every walk of a
  // point starts with the same query, computed once by a pre-pass.
  const float4* first_cpd;
  const int2* first_ids;
  int64_t total_chunks;
  int64_t chunks_per_point;
  int walks_per_point;
  int chunk;
  int regen;  // waiting lanes that trigger the walk-update phase
  int max_steps;
  int depth_m;
  float eps;
  float step_scale;
  uint32_t k0, k1;
  int has_source;
  int source_center;
  int source_samples;  // points averaged per ball (>= 1)
  int64_t deadline_ns;
  n2w_problem problem;
  // kOutStats
  double* sum;
  double* sum_sq;
  uint32_t* count;
  uint64_t* steps;
  uint32_t* forced;
  // kOutSamples / kOutPrefix
  float* s_value;
  int* s_steps;
  int* s_forced;
  int* s_overflow;
  float* p_inputs;
  float* p_boundary;
  float* p_cont;
  uint8_t* p_needs;
  float in_min[3];
  float in_ext[3];
  // scratch
  unsigned long long* queue;
  n2w_walk_counters* counters;
  // batched launches: instance table sorted by chunk_base / point_base
  const BatchInst* insts;
  int n_insts;
};

dev::SeedGrid seed_grid_of(const n2w_bvh& b);
void validate_problem(const n2w_problem& p);
void validate_walk_options(const n2w_walk_options& o);

// Batched launches (walker.cu): per-point first queries of every instance, and
// the persistent walker over the concatenated chunk queue of all instances.
// reg_variant 0: 64 registers / 4 blocks per SM; 1: 80 registers / 3 blocks.
void launch_first_query_batch(const WalkArgs& a, int64_t total_points, float4* cpd, int2* ids, cudaStream_t s);
void launch_walker_batch(const WalkArgs& a, int block, int blocks_per_sm, int reg_variant, cudaStream_t s);
int walker_batch_occupancy(int block, int reg_variant);

}  // namespace n2w
