// Merged multi-mesh device layout shared by batched launches and the serving
// loop: concatenated 4-wide nodes, leaf-ordered triangles and seed-grid slots
// of several BVHs, with every index rebased, plus per-mesh metadata.
#pragma once

#include <cuda_runtime.h>

#include <vector>

#include "internal.hpp"
#include "problem.cuh"
#include "walker.cuh"

struct n2w_scene {
  n2w::Node4* d_nodes = nullptr;
  n2w::TriRec* d_tris = nullptr;
  int* d_slots = nullptr;
  int64_t nodes = 0, tris = 0, slots = 0;
  struct MeshEntry {
    int32_t root = 0;
    int64_t node_off = 0, tri_off = 0, slot_off = -1;
    float seed_lo[3] = {0, 0, 0};
    float seed_h = 0.0f;
    int seed_n = 0;
    float box_lo[3] = {-1.0e30f, -1.0e30f, -1.0e30f};
    float box_hi[3] = {1.0e30f, 1.0e30f, 1.0e30f};
    int64_t triangles = 0;
  };
  std::vector<MeshEntry> meshes;
  int device = 0;
};

namespace n2w {

// Geometry fields of a batch instance on scene mesh `mesh`.
inline void set_instance_geometry(BatchInst& I, const n2w_scene& sc, int mesh) {
  const auto& m = sc.meshes[mesh];
  I.root = m.root;
  I.grid.slots = m.slot_off >= 0 ? sc.d_slots + m.slot_off : nullptr;
  I.grid.lo_x = m.seed_lo[0];
  I.grid.lo_y = m.seed_lo[1];
  I.grid.lo_z = m.seed_lo[2];
  I.grid.inv_h = m.seed_h > 0.0f ? 1.0f / m.seed_h : 0.0f;
  I.grid.n = m.seed_n;
  for (int a = 0; a < 3; ++a) {
    I.box_lo[a] = m.box_lo[a];
    I.box_hi[a] = m.box_hi[a];
  }
}

// Problem fields of a batch instance (host copy for the flags, device copy for the kernel).
inline void set_instance_problem(BatchInst& I, const n2w_problem& pb, const n2w_problem* d_pb) {
  I.problem = d_pb;
  I.has_source = problem_has_source(pb) ? 1 : 0;
  I.source_center = pb.source_sampling == N2W_SOURCE_CENTER ? 1 : 0;
  I.source_samples = pb.source_samples > 1 ? pb.source_samples : 1;
}

}  // namespace n2w
