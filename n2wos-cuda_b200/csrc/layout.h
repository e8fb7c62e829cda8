// Device layout of the 4-wide BVH and the leaf-ordered triangle array.
//
// Node (128 B, one L2 line): six float4 rows hold the four child boxes in
// structure-of-arrays form (lo.x, hi.x, lo.y, hi.y, lo.z, hi.z), one int4 row
// holds the child references, the last 16 B are padding.  A thread fetches the
// 112 used bytes with seven 16-byte vector loads.
//
// Child reference r:  r >= 0      inner node index
//                     r == kEmpty  unused slot (its box is +inf/-inf)
//                     otherwise    leaf: ~r = (first_triangle << 3) | (count - 1)
//
// Triangle (48 B): three float4 rows (v0.xyz, original id as int bits),
// (v1.xyz, 0), (v2.xyz, 0).  Triangles are permuted into leaf order, so a leaf
// is a contiguous run; the original id is kept for results and tie-breaking.
#pragma once

#include <stdint.h>

#ifdef __CUDACC__
#define N2W_HD __host__ __device__ __forceinline__
#else
#define N2W_HD inline
#endif

namespace n2w {

constexpr int32_t kEmptyChild = INT32_MIN;
constexpr int kMaxLeafSize = 8;
constexpr int kTraversalStack = 64;
constexpr int kSeedGridCells = 128;  // seed-grid cells per axis

struct alignas(128) Node4 {
  float lo_x[4];
  float hi_x[4];
  float lo_y[4];
  float hi_y[4];
  float lo_z[4];
  float hi_z[4];
  int32_t child[4];
  int32_t pad[4];
};
static_assert(sizeof(Node4) == 128, "Node4 must be one 128-byte line");

struct alignas(16) TriRec {
  float v0[3];
  int32_t id;
  float v1[3];
  int32_t pad1;
  float v2[3];
  int32_t pad2;
};
static_assert(sizeof(TriRec) == 48, "TriRec must be 48 bytes");

N2W_HD int32_t leaf_ref(int32_t first, int32_t count) { return ~((first << 3) | (count - 1)); }
N2W_HD bool ref_is_leaf(int32_t r) { return r < 0 && r != kEmptyChild; }
N2W_HD int32_t leaf_first(int32_t r) { return (~r) >> 3; }
N2W_HD int32_t leaf_count(int32_t r) { return ((~r) & 7) + 1; }

}  // namespace n2w
