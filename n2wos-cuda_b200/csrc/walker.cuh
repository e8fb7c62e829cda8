// Kernel argument block of the persistent walker (walker.cu).
#pragma once

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
};

dev::SeedGrid seed_grid_of(const n2w_bvh& b);

}  // namespace n2w
