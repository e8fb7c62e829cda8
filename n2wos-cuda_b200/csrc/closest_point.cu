// Device-pointer closest-point queries over the 4-wide BVH (reference
// CudaBvh::query_device, src/cuda/bvh_query.cu:228-261, and the masked cuBQL
// variant, src/cuda/cubql_bvh.cu:187-214).  Each query is seeded with the
// triangle stored at the nearest seed-grid node (a real candidate, so the
// exact answer is unchanged), then finished by the ordered traversal of
// geom.cuh, advanced one node or one triangle per loop iteration.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstring>

#include "geom.cuh"
#include "internal.hpp"

namespace n2w {

dev::SeedGrid seed_grid_of(const n2w_bvh& b) {
  dev::SeedGrid g;
  g.slots = b.d_seed;
  g.lo_x = b.seed_lo[0];
  g.lo_y = b.seed_lo[1];
  g.lo_z = b.seed_lo[2];
  g.inv_h = b.seed_h > 0.0f ? 1.0f / b.seed_h : 0.0f;
  g.n = b.seed_n;
  return g;
}

namespace {

// Persistent state machine, one lane per query.  Every iteration each busy
// lane advances its query by ONE unit of traversal work (one 4-wide node
// expansion or one triangle test, dev::trav_step), and a lane whose query is
// complete writes it and takes the next query in the same iteration.  Each
// block owns the contiguous range [b n / B, (b + 1) n / B) of the queries and
// its lanes take them from a shared-memory counter as they finish, so a lane
// that drew slow queries does not hold up queries that idle lanes of its
// block could run (with a fixed grid-stride sequence, launches of ~1-2
// queries per lane last as long as their unluckiest lane's pair).  Lanes therefore never wait for another lane's whole
// traversal (one-query-per-thread loops leave ~3.6 of 32 lanes active on
// incoherent queries); short work units keep the warp's two code paths
// (node / triangle) busy.  The visit order, pruning and pushes are those of
// dev::traverse, so results and node-visit / triangle-test counts are
// identical to the one-query-per-thread traversal.
constexpr int kQueryBlock = 256;
// Traversal units (node expansions + triangle tests) a lane spends on one
// query before handing it to the warp-cooperative finisher, when the launch
// holds about one query per resident lane; the few queries far from the
// surface in every direction (near the centre of a closed mesh) need
// thousands, and one of them per lane would set the launch's length.  With
// more queries per lane the lanes' totals even out and the budget grows in
// proportion, so a full GPU hands off only the extreme queries (measured on
// 262,144 / 4,194,304 uniform queries: budget 384 -> 1.4x / 1.0x the
// single-phase rate; a fixed 192 -> 1.35x / 0.67x).
constexpr uint32_t kQueryBudget = 384;
constexpr int kHandOff = 2;         // overflow-slot mark of a handed-off query
constexpr int kFinishWarps = 4;     // warps per finisher block
constexpr int kFinishStack = 2048;  // work-list entries per finisher warp (16 KiB)
// Resident blocks per SM the traversal is compiled for (kMinBlocks).  Launches
// of up to a few queries per lane run faster with 4 (up to 64 registers, no
// spills) and larger ones with 5 (more warps to hide load latency): measured
// 152.5 / 224.2 / 285.1 against 149.5 / 213.0 / 276.0 M queries/s at 131,072 /
// 262,144 / 524,288 queries, equal at 1 M and 2 M, 391 against 405 at 4 M.
constexpr int64_t kSmallLaunch = int64_t{1} << 21;

template <bool kMasked, bool kCount, int kMinBlocks>
__global__ void __launch_bounds__(kQueryBlock, kMinBlocks) closest_point_kernel(
    const float4* __restrict__ nodes, const float4* __restrict__ tris, const dev::SeedGrid grid,
    const n2w_vec3* __restrict__ points, const uint8_t* __restrict__ active, int n,
    float* __restrict__ out_d2, n2w_vec3* __restrict__ out_cp, int* __restrict__ out_id,
    int* __restrict__ out_overflow, int* __restrict__ out_nodes, int* __restrict__ out_tris, uint32_t budget) {
  // next unclaimed query of this block's range (unsigned: after the range
  // runs out each lane claims once more, up to b_end + blockDim.x <= 2^31 + 1023)
  __shared__ unsigned s_next;
  const unsigned b_end = static_cast<unsigned>((static_cast<int64_t>(blockIdx.x) + 1) * n / gridDim.x);
  if (threadIdx.x == 0) s_next = static_cast<unsigned>(static_cast<int64_t>(blockIdx.x) * n / gridDim.x);
  __syncthreads();
  int q = 0;
  bool busy = false, drained = false;
  dev::V3 p = dev::v3(0.0f, 0.0f, 0.0f);
  dev::ClosestHit hit;
  hit.d2 = FLT_MAX;
  hit.id = INT32_MAX;
  hit.slot = -1;
  hit.cp = p;
  dev::TravState tv{0, kEmptyChild, 0, 0};
  int2 stack_mem[kTraversalStack];
  dev::LocalStack stack{stack_mem};
  uint32_t c_nodes = 0, c_tris = 0;
  bool overflow = false;
  for (;;) {
    while (!busy && !drained) {
      const unsigned claim = atomicAdd(&s_next, 1u);
      if (claim >= b_end) {
        drained = true;  // stop claiming
        break;
      }
      q = static_cast<int>(claim);
      const n2w_vec3 pt = points[q];
      if (kMasked && active[q] == 0) {
        out_d2[q] = 0.0f;
        out_cp[q] = pt;
        out_id[q] = -1;
        out_overflow[q] = 0;
        if (kCount) {
          out_nodes[q] = 0;
          out_tris[q] = 0;
        }
        continue;
      }
      p = dev::v3(pt.x, pt.y, pt.z);
      hit.d2 = FLT_MAX;
      hit.id = INT32_MAX;
      hit.slot = -1;
      hit.cp = dev::v3(0.0f, 0.0f, 0.0f);
      c_nodes = c_tris = 0;
      overflow = false;
      if (grid.slots) {
        dev::test_slot(tris, dev::seed_slot(grid, p), p, hit);
        ++c_tris;
      }
      tv.sp = 0;
      tv.ref = 0;
      tv.leaf_cur = tv.leaf_end = 0;
      busy = true;
    }
    if (!__any_sync(0xffffffffu, busy)) break;
    // Two units per iteration, written out twice: the claim loop and the vote
    // cost about as much as a unit (262,144 / 1,048,576 / 4,194,304 queries:
    // 229.8 / 347.1 / 412.4 against 225.9 / 338.2 / 404.1 M queries/s with one;
    // 229.8 / 345.8 / 410.9 as an unrolled loop).
    if (busy) {
      bool ov = false;
      if (!kCount && budget && c_nodes + c_tris > budget) {
        // Over budget: hand the query to the warp-cooperative finisher with its
        // best so far (a bound on the answer) in its own output slots.
        out_d2[q] = hit.d2;
        out_cp[q] = n2w_vec3{hit.cp.x, hit.cp.y, hit.cp.z};
        out_id[q] = hit.id == INT32_MAX ? -1 : hit.id;
        out_overflow[q] = kHandOff;
        busy = false;
      } else if (!dev::trav_step(nodes, tris, p, hit, tv, stack, c_nodes, c_tris, ov)) {
        out_d2[q] = hit.d2;
        out_cp[q] = n2w_vec3{hit.cp.x, hit.cp.y, hit.cp.z};
        out_id[q] = hit.id == INT32_MAX ? -1 : hit.id;
        out_overflow[q] = overflow ? 1 : 0;
        if (kCount) {
          out_nodes[q] = static_cast<int>(c_nodes);
          out_tris[q] = static_cast<int>(c_tris);
        }
        busy = false;
      }
      if (ov) overflow = true;
    }
    if (busy) {
      bool ov = false;
      if (!kCount && budget && c_nodes + c_tris > budget) {
        // Over budget: hand the query to the warp-cooperative finisher with its
        // best so far (a bound on the answer) in its own output slots.
        out_d2[q] = hit.d2;
        out_cp[q] = n2w_vec3{hit.cp.x, hit.cp.y, hit.cp.z};
        out_id[q] = hit.id == INT32_MAX ? -1 : hit.id;
        out_overflow[q] = kHandOff;
        busy = false;
      } else if (!dev::trav_step(nodes, tris, p, hit, tv, stack, c_nodes, c_tris, ov)) {
        out_d2[q] = hit.d2;
        out_cp[q] = n2w_vec3{hit.cp.x, hit.cp.y, hit.cp.z};
        out_id[q] = hit.id == INT32_MAX ? -1 : hit.id;
        out_overflow[q] = overflow ? 1 : 0;
        if (kCount) {
          out_nodes[q] = static_cast<int>(c_nodes);
          out_tris[q] = static_cast<int>(c_tris);
        }
        busy = false;
      }
      if (ov) overflow = true;
    }
  }
}

// Warp-cooperative finisher for the queries that ran over the per-lane
// budget (marked kHandOff in their overflow slot): one warp per group of 32
// consecutive queries takes its marked queries one at a time and traverses
// the BVH from the root with the lane's best so far as the bound.  A
// shared-memory work list of (node or leaf, box distance) entries feeds the 32
// lanes: each iteration every lane takes one entry, expands a node (children
// whose box is within the warp's best are pushed) or tests a leaf's
// triangles, and the warp's best (d2, id) -- a 64-bit key, lowest d2 then
// lowest id -- is the minimum over lanes.  Pruning is conservative, so the
// answer is the exact one a single-lane traversal gives.  Blocks whose groups
// hold no marked query exit at once, so the block scheduler balances the work.
__device__ __forceinline__ unsigned long long hit_key(float d2, int id) {
  return (static_cast<unsigned long long>(__float_as_uint(d2)) << 32) | static_cast<unsigned>(id);
}

__global__ void __launch_bounds__(32 * kFinishWarps) closest_point_finish_kernel(
    const float4* __restrict__ nodes, const float4* __restrict__ tris, const n2w_vec3* __restrict__ points, int n,
    float* __restrict__ out_d2, n2w_vec3* __restrict__ out_cp, int* __restrict__ out_id,
    int* __restrict__ out_overflow) {
  extern __shared__ int2 s_work[];
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  int2* work = s_work + warp * kFinishStack;
  const int64_t q0 = (static_cast<int64_t>(blockIdx.x) * kFinishWarps + warp) * 32;
  if (q0 >= n) return;
  const int64_t mine = q0 + lane;
  unsigned pending = __ballot_sync(0xffffffffu, mine < n && out_overflow[mine] == kHandOff);
  while (pending) {
    const int q = static_cast<int>(q0) + __ffs(pending) - 1;
    pending &= pending - 1;
    const n2w_vec3 pt = points[q];
    const dev::V3 p = dev::v3(pt.x, pt.y, pt.z);
    const int id0 = out_id[q];
    const unsigned long long start_key = hit_key(out_d2[q], id0 < 0 ? INT32_MAX : id0);
    unsigned long long best_key = start_key;  // warp-uniform
    unsigned long long my_key = start_key;
    dev::V3 my_cp = p;
    bool dropped = false;  // warp-uniform: the work list was full
    if (lane == 0) work[0] = make_int2(0, __float_as_int(0.0f));
    int sp = 1;  // warp-uniform
    __syncwarp();
    while (sp > 0) {
      const int take = min(sp, 32);
      int2 e = make_int2(kEmptyChild, 0);
      if (lane < take) e = work[sp - take + lane];
      __syncwarp();
      sp -= take;
      const float bound = __uint_as_float(static_cast<unsigned>(best_key >> 32));
      int2 c0 = make_int2(kEmptyChild, 0), c1 = c0, c2 = c0, c3 = c0;
      int nc = 0;
      if (e.x != kEmptyChild && __int_as_float(e.y) <= bound) {
        if (e.x >= 0) {
          float4 lox, hix, loy, hiy, loz, hiz;
          int4 ch;
          dev::load_node(nodes, e.x, lox, hix, loy, hiy, loz, hiz, ch);
          float d[4] = {dev::box_d2(p, lox.x, hix.x, loy.x, hiy.x, loz.x, hiz.x),
                        dev::box_d2(p, lox.y, hix.y, loy.y, hiy.y, loz.y, hiz.y),
                        dev::box_d2(p, lox.z, hix.z, loy.z, hiy.z, loz.z, hiz.z),
                        dev::box_d2(p, lox.w, hix.w, loy.w, hiy.w, loz.w, hiz.w)};
          const int r[4] = {ch.x, ch.y, ch.z, ch.w};
#pragma unroll
          for (int k = 0; k < 4; ++k) {
            if (r[k] != kEmptyChild && d[k] <= bound) {
              const int2 ce = make_int2(r[k], __float_as_int(d[k]));
              if (nc == 0) c0 = ce;
              else if (nc == 1) c1 = ce;
              else if (nc == 2) c2 = ce;
              else c3 = ce;
              ++nc;
            }
          }
        } else {
          const int first = leaf_first(e.x), count = leaf_count(e.x);
          for (int i = 0; i < count; ++i) {
            dev::ClosestHit h;
            h.d2 = FLT_MAX;
            h.id = INT32_MAX;
            h.slot = 0;
            h.cp = p;
            dev::test_slot(tris, first + i, p, h);
            const unsigned long long k = hit_key(h.d2, h.id);
            if (k < my_key) {
              my_key = k;
              my_cp = h.cp;
            }
          }
        }
      }
      unsigned long long wk = my_key;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) wk = min(wk, __shfl_xor_sync(0xffffffffu, wk, o));
      best_key = min(best_key, wk);
      // append this iteration's children (lane order, each lane's nearest last)
      int incl = nc;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int v = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += v;
      }
      const int total = __shfl_sync(0xffffffffu, incl, 31);
      int at = sp + incl - nc;
      const int2 cs[4] = {c0, c1, c2, c3};
      for (int j = nc - 1; j >= 0; --j, ++at) {
        if (at < kFinishStack) work[at] = cs[j];
      }
      if (sp + total > kFinishStack) dropped = true;
      sp = min(sp + total, kFinishStack);
      __syncwarp();
    }
    // the lane holding the winning key writes it (a triangle is tested by one
    // lane only); if nothing beat the hand-off bound, the written hit stands
    if (best_key != start_key && my_key == best_key) {
      out_d2[q] = __uint_as_float(static_cast<unsigned>(best_key >> 32));
      out_id[q] = static_cast<int>(best_key & 0xffffffffu);
      out_cp[q] = n2w_vec3{my_cp.x, my_cp.y, my_cp.z};
    }
    if (lane == 0) out_overflow[q] = dropped ? 1 : 0;
    __syncwarp();
  }
}

// Builds the seed grid: a cold exact query at every lattice node.
__global__ void __launch_bounds__(256) seed_grid_kernel(const float4* __restrict__ nodes,
                                                        const float4* __restrict__ tris, float lox, float loy,
                                                        float loz, float h, int n, int* __restrict__ slots,
                                                        int* __restrict__ overflow) {
  const int s = n + 1;
  const int64_t total = static_cast<int64_t>(s) * s * s;
  const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= total) return;
  const int ix = static_cast<int>(i % s), iy = static_cast<int>((i / s) % s), iz = static_cast<int>(i / (static_cast<int64_t>(s) * s));
  // Lattice position lo + h * i, rounded per operation (no FMA) so a host
  // float32 evaluation of the same expression gives the same point.
  const dev::V3 p = dev::v3(__fadd_rn(lox, __fmul_rn(h, static_cast<float>(ix))),
                            __fadd_rn(loy, __fmul_rn(h, static_cast<float>(iy))),
                            __fadd_rn(loz, __fmul_rn(h, static_cast<float>(iz))));
  dev::ClosestHit hit;
  hit.d2 = FLT_MAX;
  hit.id = INT32_MAX;
  hit.slot = 0;
  hit.cp = p;
  dev::TraversalStats st{0, 0, 0};
  dev::traverse<false>(nodes, tris, p, hit, st);
  slots[i] = hit.slot;
  if (st.overflow) atomicOr(overflow, 1);
}

// Inside/outside by ray parity along +x with the reference's deterministic
// offset (src/cuda/cubql_bvh.cu:446-455).
__global__ void __launch_bounds__(1024) inside_kernel(const float4* __restrict__ nodes,
                                                      const float4* __restrict__ tris,
                                                      const n2w_vec3* __restrict__ points, int n,
                                                      uint8_t* __restrict__ inside, int* __restrict__ overflow) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= n) return;
  const n2w_vec3 p = points[q];
  int ov = 0;
  const int hits = dev::ray_x_crossings(nodes, tris, dev::v3(p.x, p.y + 1.928371e-6f, p.z + 3.141593e-6f), ov);
  inside[q] = (hits & 1) ? 1 : 0;
  if (ov) atomicOr(overflow, 1);
}

}  // namespace

void launch_inside(const n2w_bvh& bvh, const n2w_vec3* d_points, int n, uint8_t* d_inside, int* d_overflow,
                   int block_size, cudaStream_t stream) {
  const int grid = (n + block_size - 1) / block_size;
  inside_kernel<<<grid, block_size, 0, stream>>>(reinterpret_cast<const float4*>(bvh.d_nodes),
                                                 reinterpret_cast<const float4*>(bvh.d_tris), d_points, n,
                                                 d_inside, d_overflow);
  N2W_CUDA(cudaGetLastError());
}

void launch_closest_point(const n2w_bvh& bvh, const n2w_vec3* d_points, const uint8_t* d_active,
                          int n, float* d_d2, n2w_vec3* d_cp, int* d_id, int* d_overflow,
                          int* d_nodes, int* d_tris, int block_size, cudaStream_t stream) {
  // block_size (the reference's launch knob, validated to [1, 1024]) is a hint:
  // the kernel runs 256-thread blocks, each over its own range of the queries,
  // with the grid sized to the resident capacity of the GPU.
  (void)block_size;
  const float4* nodes = reinterpret_cast<const float4*>(bvh.d_nodes);
  const float4* tris = reinterpret_cast<const float4*>(bvh.d_tris);
  const dev::SeedGrid sg = seed_grid_of(bvh);
  auto launch = [&](auto kern, const uint8_t* act, int* dn, int* dt) {
    int occ = 0;
    N2W_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, kQueryBlock, 0));
    const int64_t blocks_needed = (static_cast<int64_t>(n) + kQueryBlock - 1) / kQueryBlock;
    const int64_t resident = static_cast<int64_t>(sm_count_current()) * std::max(occ, 1);
    const int grid = static_cast<int>(std::max<int64_t>(1, std::min(blocks_needed, resident)));
    const int64_t lanes = resident * kQueryBlock;
    const int64_t per_lane = (static_cast<int64_t>(n) + 2 * lanes - 1) / (2 * lanes);  // ceil(n / (2 lanes))
    const uint32_t budget = static_cast<uint32_t>(std::min<int64_t>(kQueryBudget * std::max<int64_t>(per_lane, 1),
                                                                    1 << 30));
    kern<<<grid, kQueryBlock, 0, stream>>>(nodes, tris, sg, d_points, act, n, d_d2, d_cp, d_id, d_overflow, dn, dt,
                                           dn ? 0u : budget);
  };
  if (d_nodes) {
    // the counting variant runs every query to completion in one lane, so its
    // counts are the single-lane traversal's (the algorithmic work)
    launch(closest_point_kernel<false, true, 5>, d_active, d_nodes, d_tris);
    N2W_CUDA(cudaGetLastError());
    return;
  }
  const bool small = n < kSmallLaunch;
  if (d_active) {
    if (small) launch(closest_point_kernel<true, false, 4>, d_active, nullptr, nullptr);
    else launch(closest_point_kernel<true, false, 5>, d_active, nullptr, nullptr);
  } else {
    if (small) launch(closest_point_kernel<false, false, 4>, nullptr, nullptr, nullptr);
    else launch(closest_point_kernel<false, false, 5>, nullptr, nullptr, nullptr);
  }
  N2W_CUDA(cudaGetLastError());
  const size_t smem = sizeof(int2) * kFinishWarps * kFinishStack;
  static thread_local int configured_device = -1;
  int dev = 0;
  N2W_CUDA(cudaGetDevice(&dev));
  if (configured_device != dev) {
    N2W_CUDA(cudaFuncSetAttribute(closest_point_finish_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  static_cast<int>(smem)));
    configured_device = dev;
  }
  const int64_t groups = (static_cast<int64_t>(n) + 31) / 32;
  const unsigned blocks = static_cast<unsigned>((groups + kFinishWarps - 1) / kFinishWarps);
  closest_point_finish_kernel<<<blocks, 32 * kFinishWarps, smem, stream>>>(nodes, tris, d_points, n, d_d2, d_cp,
                                                                          d_id, d_overflow);
  N2W_CUDA(cudaGetLastError());
}

int sm_count_current() {
  int dev = 0, sms = 0;
  N2W_CUDA(cudaGetDevice(&dev));
  N2W_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  return sms;
}

// Seed grid over the mesh box grown by 20 % of its largest extent on every side.
void build_seed_grid(n2w_bvh& b, const n2w_mesh& mesh, int n) {
  float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
  for (const auto& v : mesh.vertices) {
    for (int a = 0; a < 3; ++a) {
      lo[a] = std::min(lo[a], v[a]);
      hi[a] = std::max(hi[a], v[a]);
    }
  }
  const float ext = std::max(std::max(hi[0] - lo[0], hi[1] - lo[1]), hi[2] - lo[2]);
  const float pad = 0.2f * ext + 1e-6f;
  const float h = (ext + 2.0f * pad) / static_cast<float>(n);
  for (int a = 0; a < 3; ++a) b.seed_lo[a] = 0.5f * (lo[a] + hi[a]) - 0.5f * (ext + 2.0f * pad);
  b.seed_h = h;
  b.seed_n = n;
  const int64_t total = static_cast<int64_t>(n + 1) * (n + 1) * (n + 1);
  N2W_CUDA(cudaMalloc(&b.d_seed, total * sizeof(int)));
  int* d_ov = nullptr;
  N2W_CUDA(cudaMalloc(&d_ov, sizeof(int)));
  N2W_CUDA(cudaMemset(d_ov, 0, sizeof(int)));
  const int block = 256;
  seed_grid_kernel<<<static_cast<unsigned>((total + block - 1) / block), block>>>(
      reinterpret_cast<const float4*>(b.d_nodes), reinterpret_cast<const float4*>(b.d_tris), b.seed_lo[0],
      b.seed_lo[1], b.seed_lo[2], h, n, b.d_seed, d_ov);
  N2W_CUDA(cudaGetLastError());
  int ov = 0;
  N2W_CUDA(cudaMemcpy(&ov, d_ov, sizeof(int), cudaMemcpyDeviceToHost));
  cudaFree(d_ov);
  if (ov) throw Error(N2W_EINTERNAL, "traversal stack overflow while building the seed grid");
}

}  // namespace n2w

using namespace n2w;

namespace {

void check_query_args(const n2w_bvh* bvh, const void* pts, int n, const void* d2, const void* cp,
                      const void* id, const void* ov, int block_size) {
  N2W_REQUIRE(bvh && bvh->d_nodes && bvh->d_tris, "query_device called on empty BVH");
  N2W_REQUIRE(n >= 0, "query_device query_count must be non-negative");
  if (n == 0) return;
  N2W_REQUIRE(pts && d2 && cp && id && ov, "query_device received a null device pointer");
  N2W_REQUIRE(block_size >= 1 && block_size <= 1024, "CUDA block size must be in [1, 1024]");
}

void release(n2w_bvh* b) {
  if (b->d_nodes) cudaFree(b->d_nodes);
  if (b->d_tris) cudaFree(b->d_tris);
  if (b->d_seed) cudaFree(b->d_seed);
  delete b;
}

}  // namespace

extern "C" {

int n2w_bvh_create(const n2w_mesh* mesh, int leaf_size, const char* build_method, n2w_bvh** out) {
  return guarded([&] {
    N2W_REQUIRE(mesh && out, "n2w_bvh_create: null argument");
    const auto t0 = std::chrono::steady_clock::now();
    HostBvh h = build_bvh4(*mesh, leaf_size, build_method ? build_method : "sah");
    auto* b = new n2w_bvh();
    try {
      N2W_CUDA(cudaGetDevice(&b->device));
      N2W_CUDA(cudaMalloc(&b->d_nodes, h.nodes.size() * sizeof(Node4)));
      N2W_CUDA(cudaMalloc(&b->d_tris, h.tris.size() * sizeof(TriRec)));
      N2W_CUDA(cudaMemcpy(b->d_nodes, h.nodes.data(), h.nodes.size() * sizeof(Node4), cudaMemcpyHostToDevice));
      N2W_CUDA(cudaMemcpy(b->d_tris, h.tris.data(), h.tris.size() * sizeof(TriRec), cudaMemcpyHostToDevice));
      build_seed_grid(*b, *mesh, kSeedGridCells);
      N2W_CUDA(cudaDeviceSynchronize());
    } catch (...) {
      release(b);
      throw;
    }
    const auto t1 = std::chrono::steady_clock::now();
    b->stats = host_stats(h, leaf_size, std::chrono::duration<double, std::milli>(t1 - t0).count());
    b->stats.device_bytes += static_cast<int64_t>(kSeedGridCells + 1) * (kSeedGridCells + 1) * (kSeedGridCells + 1) * 4;
    *out = b;
  });
}

int n2w_bvh_stats_get(const n2w_bvh* bvh, n2w_bvh_stats* out) {
  return guarded([&] {
    N2W_REQUIRE(bvh && out, "null argument");
    *out = bvh->stats;
  });
}

void n2w_bvh_destroy(n2w_bvh* bvh) {
  if (bvh) release(bvh);
}

int n2w_bvh_query_device(const n2w_bvh* bvh, const n2w_vec3* d_points, int query_count,
                         float* d_distance2, n2w_vec3* d_closest, int* d_triangle_id,
                         int* d_overflow, int block_size, n2w_stream_t stream) {
  return guarded([&] {
    check_query_args(bvh, d_points, query_count, d_distance2, d_closest, d_triangle_id, d_overflow, block_size);
    if (query_count == 0) return;
    launch_closest_point(*bvh, d_points, nullptr, query_count, d_distance2, d_closest, d_triangle_id,
                         d_overflow, nullptr, nullptr, block_size, stream);
  });
}

int n2w_bvh_query_device_masked(const n2w_bvh* bvh, const n2w_vec3* d_points,
                                const uint8_t* d_active, int query_count, float* d_distance2,
                                n2w_vec3* d_closest, int* d_triangle_id, int* d_overflow,
                                int block_size, n2w_stream_t stream) {
  return guarded([&] {
    check_query_args(bvh, d_points, query_count, d_distance2, d_closest, d_triangle_id, d_overflow, block_size);
    if (query_count == 0) return;
    N2W_REQUIRE(d_active, "query_device_masked received a null mask");
    launch_closest_point(*bvh, d_points, d_active, query_count, d_distance2, d_closest, d_triangle_id,
                         d_overflow, nullptr, nullptr, block_size, stream);
  });
}

int n2w_bvh_query_device_counted(const n2w_bvh* bvh, const n2w_vec3* d_points, int query_count,
                                 float* d_distance2, n2w_vec3* d_closest, int* d_triangle_id,
                                 int* d_overflow, int* d_node_visits, int* d_tri_tests,
                                 int block_size, n2w_stream_t stream) {
  return guarded([&] {
    check_query_args(bvh, d_points, query_count, d_distance2, d_closest, d_triangle_id, d_overflow, block_size);
    if (query_count == 0) return;
    N2W_REQUIRE(d_node_visits && d_tri_tests, "counted query needs counter outputs");
    launch_closest_point(*bvh, d_points, nullptr, query_count, d_distance2, d_closest, d_triangle_id,
                         d_overflow, d_node_visits, d_tri_tests, block_size, stream);
  });
}

int n2w_bvh_inside_device(const n2w_bvh* bvh, const n2w_vec3* d_points, int query_count, uint8_t* d_inside,
                          int* d_overflow, int block_size, n2w_stream_t stream) {
  return guarded([&] {
    N2W_REQUIRE(bvh && bvh->d_nodes && bvh->d_tris, "inside_device called on empty BVH");
    N2W_REQUIRE(query_count >= 0, "query_count must be non-negative");
    if (query_count == 0) return;
    N2W_REQUIRE(d_points && d_inside && d_overflow, "inside_device received a null device pointer");
    N2W_REQUIRE(block_size >= 1 && block_size <= 1024, "CUDA block size must be in [1, 1024]");
    launch_inside(*bvh, d_points, query_count, d_inside, d_overflow, block_size, stream);
  });
}

int n2w_bvh_copy_layout(const n2w_bvh* bvh, void* nodes_out, void* tris_out) {
  return guarded([&] {
    N2W_REQUIRE(bvh, "null bvh");
    if (nodes_out) {
      N2W_CUDA(cudaMemcpy(nodes_out, bvh->d_nodes, static_cast<size_t>(bvh->stats.nodes) * sizeof(Node4),
                          cudaMemcpyDeviceToHost));
    }
    if (tris_out) {
      N2W_CUDA(cudaMemcpy(tris_out, bvh->d_tris, static_cast<size_t>(bvh->stats.triangles) * sizeof(TriRec),
                          cudaMemcpyDeviceToHost));
    }
  });
}

int n2w_bvh_seed_grid(const n2w_bvh* bvh, float* lo_out, float* h_out, int* n_out, int* slots_out) {
  return guarded([&] {
    N2W_REQUIRE(bvh && bvh->d_seed, "BVH has no seed grid");
    if (lo_out) std::memcpy(lo_out, bvh->seed_lo, sizeof(bvh->seed_lo));
    if (h_out) *h_out = bvh->seed_h;
    if (n_out) *n_out = bvh->seed_n;
    if (slots_out) {
      const size_t s = static_cast<size_t>(bvh->seed_n) + 1;
      N2W_CUDA(cudaMemcpy(slots_out, bvh->d_seed, s * s * s * sizeof(int), cudaMemcpyDeviceToHost));
    }
  });
}

}  // extern "C"
