// Persistent Walk-on-Spheres walkers with on-device estimator reductions.
//
// Semantics follow the reference walk (src/cuda/cubql_bvh.cu:1323-1357,
// 263-336): for step = 0..max_steps query the closest point P at x, d = |x-P|;
// stop if d <= epsilon, step >= max_steps or d is not finite and score g(P);
// otherwise add the ball's source contribution, move x += step_scale*d*dir with
// dir uniform on the unit sphere (z = 1-2u, phi = 2 pi v, reference 254-261).
//
// B200 design:
//  * a grid of SMs x resident blocks that lives until the work runs out; each
//    lane owns one walker and pops `chunk` consecutive walks of one point from
//    a global queue with one warp-aggregated atomic, so uneven walk lengths
//    never idle a lane while work remains;
//  * counter-based Philox keyed by (seed; walk id, step, stream), so a walk's
//    path is independent of scheduling (serving "alone == in the mix");
//  * the first query of every walk of a point is computed once per point
//    (exact arithmetic); every later query is seeded with two real candidate
//    triangles (the previous closest one and the seed-grid one at x), which
//    bounds the traversal to the walker's neighbourhood, and runs the
//    contracted-FP32 box and triangle routines of geom.cuh (FMA, fast
//    division; within a few ulps of the exact query, as the reference's own
//    nvcc-compiled walker is);
//  * per-point FP64 sum / sum of squares accumulated per lane over its chunk,
//    merged across lanes with warp shuffles and flushed with FP64 atomics.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <mutex>

#include "geom.cuh"
#include "internal.hpp"
#include "philox.cuh"
#include "problem.cuh"
#include "walker.cuh"

namespace n2w {

__device__ __forceinline__ uint64_t global_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ dev::V3 unit_sphere(uint32_t a, uint32_t b) {
  const float z = 1.0f - 2.0f * u01(a);
  float s, c;
  sincospif(2.0f * u01(b), &s, &c);
  const float r = sqrtf(fmaxf(0.0f, 1.0f - z * z));
  return dev::v3(r * c, r * s, z);
}

// Beta(2,2) inverse CDF: the radius fraction t of a point drawn from the ball's
// Green's function density G(x,y) ∝ 1/|y-x| - 1/R (radial density ∝ t(1-t)).
// Solves 3t^2 - 2t^3 = u with the trigonometric root of the depressed cubic.
// The cosine's argument lies in [-2 pi / 3, -pi / 3], where the SFU cosine
// __cosf has an absolute error of at most 2^-21.19 (CUDA programming guide).
__device__ __forceinline__ float green_radius_fraction(float u) {
  const float a = acosf(fminf(1.0f, fmaxf(-1.0f, 1.0f - 2.0f * u)));
  return 0.5f + __cosf((a - 6.283185307179586f) * (1.0f / 3.0f));
}

// sin x with x first reduced to about [-pi, pi] (Cody-Waite: 2 pi split as
// 6.28125, exact in a few bits, plus 1.9353071795864769e-3), so the SFU sine
// __sinf keeps its documented absolute error of at most 2^-21.41.
__device__ __forceinline__ float sin_sfu(float x) {
  const float k = rintf(x * 0.15915494309189535f);
  return __sinf(fmaf(-k, 1.9353071795864769e-3f, fmaf(-k, 6.28125f, x)));
}

// Source f at an in-ball sample.  The manufactured sin-product source uses the
// SFU sines: an absolute error below 3 x 2^-21.4 on the product of sines, i.e.
// ~1e-6 relative to f's scale 3 omega^2, far below the Monte Carlo error of
// any estimate (16 samples per ball: 29.6 -> 25.7 ns per walk).  Other
// sources use the accurate routines of problem_f.
__device__ __forceinline__ float source_f_sample(const n2w_problem& pb, float x, float y, float z) {
  if (pb.mode == N2W_BC_POISSON_SINPROD) {
    const float w = pb.omega;
    return 3.0f * w * w * sin_sfu(w * x) * sin_sfu(w * y) * sin_sfu(w * z);
  }
  return problem_f<float>(pb, x, y, z);
}

__device__ __forceinline__ double shfl_xor_d(double v, int o) { return __shfl_xor_sync(0xffffffffu, v, o); }


// Source contribution of the ball B(x, R): (R^2/6) * f at the ball centre
// (reference rule) or averaged over `source_samples` points drawn from the
// ball's Green's function.  Sample 0 takes its radius fraction from word u2 of
// the step's stream-0 draw and its direction from stream 1; samples k >= 1 use
// stream 1 + k.
__device__ __forceinline__ float ball_source(const n2w_problem& pb, uint32_t k0, uint32_t k1, int source_center,
                                             int source_samples, dev::V3 x, float R, uint64_t wid, int step,
                                             uint32_t u2) {
  float f;
  if (source_center) {
    f = problem_f<float>(pb, x.x, x.y, x.z);
  } else {
    const float tfrac = green_radius_fraction(u01(u2));
    const U4 r2 = philox4x32_10(U4{static_cast<uint32_t>(wid), static_cast<uint32_t>(wid >> 32),
                                   static_cast<uint32_t>(step), 1u},
                                k0, k1);
    const dev::V3 w = unit_sphere(r2.x, r2.y);
    const float rho = R * tfrac;
    f = source_f_sample(pb, x.x + rho * w.x, x.y + rho * w.y, x.z + rho * w.z);
    for (int k = 1; k < source_samples; ++k) {
      const U4 rk = philox4x32_10(U4{static_cast<uint32_t>(wid), static_cast<uint32_t>(wid >> 32),
                                     static_cast<uint32_t>(step), 1u + static_cast<uint32_t>(k)},
                                  k0, k1);
      const float rk_rho = R * green_radius_fraction(u01(rk.x));
      const dev::V3 wk = unit_sphere(rk.y, rk.z);
      f += source_f_sample(pb, x.x + rk_rho * wk.x, x.y + rk_rho * wk.y, x.z + rk_rho * wk.z);
    }
    if (source_samples > 1) f *= 1.0f / static_cast<float>(source_samples);
  }
  return (R * R) * (1.0f / 6.0f) * f;
}

// Warp-collective flush of per-lane chunk accumulators into per-point FP64
// totals: lanes are grouped by point id, each group is reduced by a shuffle
// butterfly (non-members contribute zero) and its lowest lane issues the atomics.
template <bool kBatch>
__device__ __forceinline__ void warp_flush(bool want, int64_t pid, int inst, double s, double s2, uint32_t n,
                                           uint64_t steps, uint32_t forced, const WalkArgs& a) {
  unsigned pending = __ballot_sync(0xffffffffu, want);
  const int lane = threadIdx.x & 31;
  while (pending) {
    const int leader = __ffs(pending) - 1;
    const long long lp = __shfl_sync(0xffffffffu, static_cast<long long>(pid), leader);
    const bool in = want && pid == lp;
    const unsigned grp = __ballot_sync(0xffffffffu, in);
    double vs = in ? s : 0.0, vs2 = in ? s2 : 0.0;
    unsigned long long vst = in ? steps : 0ull;
    unsigned vn = in ? n : 0u, vf = in ? forced : 0u;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      vs += shfl_xor_d(vs, o);
      vs2 += shfl_xor_d(vs2, o);
      vst += __shfl_xor_sync(0xffffffffu, vst, o);
      vn += __shfl_xor_sync(0xffffffffu, vn, o);
      vf += __shfl_xor_sync(0xffffffffu, vf, o);
    }
    if (kBatch) {
      // pid is the global point index; the leader's instance owns the accumulators.
      const int li = __shfl_sync(0xffffffffu, inst, leader);
      if (lane == leader) {
        const BatchInst& I = a.insts[li];
        const int64_t q = lp - I.point_base;
        atomicAdd(I.sum + q, vs);
        atomicAdd(I.sum_sq + q, vs2);
        atomicAdd(I.count + q, vn);
        atomicAdd(reinterpret_cast<unsigned long long*>(I.steps) + q, vst);
        atomicAdd(I.forced + q, vf);
      }
    } else if (lane == leader) {
      atomicAdd(a.sum + lp, vs);
      atomicAdd(a.sum_sq + lp, vs2);
      atomicAdd(a.count + lp, vn);
      atomicAdd(reinterpret_cast<unsigned long long*>(a.steps) + lp, vst);
      atomicAdd(a.forced + lp, vf);
    }
    pending &= ~grp;
  }
}

__device__ __forceinline__ unsigned long long warp_sum_u64(unsigned long long v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Persistent walker: a two-phase loop per warp.
//  Phase A (warp-uniform): finished queries are consumed — the walk stops and
//    is scored, or moves to its next ball and seeds its next query; finished
//    chunks are flushed into the per-point FP64 totals; idle lanes pop new
//    chunks from the global queue.
//  Phase B: every lane with a query in flight performs traversal steps; the
//    warp returns to Phase A once `regen` lanes are waiting (or none is busy),
//    so the walk updates run for many lanes at once and no lane waits for
//    another lane's whole traversal.
template <int kOut, int kWalk, bool kBatch = false, int kMinBlocks = kWalkerMinBlocks, int kUnits = 1>
__global__ void __launch_bounds__(kWalkerMaxThreads, kMinBlocks) walker_kernel(const __grid_constant__ WalkArgs a) {
  static_assert(!kBatch || (kOut == kOutStats && kWalk == N2W_WALK_PURE),
                "batched launches run plain walks into per-point statistics");
  const int lane = threadIdx.x & 31;
  const uint64_t t_start = (a.deadline_ns > 0) ? global_ns() : 0;

  bool alive = false;     // a walk is in progress on this lane
  bool querying = false;  // its closest-point query is in flight
  bool exhausted = false; // the global queue has no chunk left for this lane
  int64_t pid = -1;  // global point index
  int inst = 0;      // batched launches: instance of the current chunk
  int walk = 0, walk_end = 0;
  dev::V3 x = dev::v3(0, 0, 0), xm = dev::v3(0, 0, 0);
  float src = 0.0f, am = 0.0f;
  int step = 0, cont0 = 0;
  bool has_xm = false, w_overflow = false;
  uint64_t wid = 0;

  dev::ClosestHit hit;
  hit.d2 = FLT_MAX;
  hit.id = INT32_MAX;
  hit.slot = 0;
  hit.cp = x;
  dev::TravState tv{0, kEmptyChild, 0, 0};
  int2 stack_mem[kTraversalStack];
  dev::LocalStack stack{stack_mem};

  double acc_s = 0.0, acc_s2 = 0.0;
  uint32_t acc_n = 0, acc_forced = 0, acc_steps = 0;

  // Per-thread run counters (32-bit; spilled to the 64-bit totals when large).
  uint32_t c_walks = 0, c_steps = 0, c_queries = 0, c_nodes = 0, c_tris = 0, c_overflow = 0, c_forced = 0,
           c_timeout = 0;

  // Per-instance parameters: kernel arguments for a single problem, the
  // instance table (L1-resident) for batched launches.
  auto problem_of = [&]() -> const n2w_problem& {
    if constexpr (kBatch) return *a.insts[inst].problem;
    else return a.problem;
  };
  auto start_point = [&]() -> n2w_vec3 {
    if constexpr (kBatch) return a.insts[inst].points[pid - a.insts[inst].point_base];
    else return a.points[pid];
  };

  for (;;) {
    // ================= Phase A =================
    // (1) deadline: abandon the current walk and stop taking work.
    if (a.deadline_ns > 0 && !exhausted && (global_ns() - t_start) > static_cast<uint64_t>(a.deadline_ns)) {
      if (alive) ++c_timeout;
      alive = false;
      querying = false;
      exhausted = true;
      walk = walk_end;
    }
    // (2) consume finished queries: score and finish, or move and seed the next
    //     query.  A finished walk with more walks left in its chunk starts the
    //     next one at once from the point's cached first query.
    while (alive && !querying) {
      ++c_queries;
      const float d = sqrtf(fmaxf(hit.d2, 0.0f));
      const int rel = step - cont0;  // steps since the walk (or its continuation) began
      const bool forced = rel >= a.max_steps;
      const bool stop = d <= a.eps || forced || !isfinite(d) || hit.id == INT32_MAX;
      if (stop || (kWalk == N2W_WALK_PREFIX && step >= a.depth_m)) {
        const float value = stop ? src + problem_u<float>(problem_of(), hit.cp.x, hit.cp.y, hit.cp.z) : src;
        ++c_walks;
        c_steps += static_cast<uint32_t>(step);
        c_forced += forced ? 1u : 0u;
        if (kOut == kOutStats) {
          acc_s += static_cast<double>(value);
          acc_s2 += static_cast<double>(value) * static_cast<double>(value);
          ++acc_n;
          acc_steps += static_cast<uint32_t>(step);
          acc_forced += forced ? 1u : 0u;
        } else {
          const uint64_t s = wid;
          if (kOut == kOutSamples) {
            a.s_value[s] = value;
          } else {
            // Prefix outputs (reference cubql_bvh.cu:1451-1606): X is X_m when the
            // cache is needed, else the position where the walk stopped.
            const bool needs = (kWalk == N2W_WALK_PREFIX) ? !stop : has_xm;
            const dev::V3 xo = (kWalk == N2W_WALK_RESIDUAL && has_xm) ? xm : x;
            a.p_inputs[3 * s + 0] = fminf(1.0f, fmaxf(0.0f, (xo.x - a.in_min[0]) / fmaxf(a.in_ext[0], 1.0e-6f)));
            a.p_inputs[3 * s + 1] = fminf(1.0f, fmaxf(0.0f, (xo.y - a.in_min[1]) / fmaxf(a.in_ext[1], 1.0e-6f)));
            a.p_inputs[3 * s + 2] = fminf(1.0f, fmaxf(0.0f, (xo.z - a.in_min[2]) / fmaxf(a.in_ext[2], 1.0e-6f)));
            a.p_needs[s] = needs ? 1 : 0;
            if (kWalk == N2W_WALK_PREFIX) {
              a.p_boundary[s] = value;
            } else {
              a.p_boundary[s] = needs ? am : value;
              a.p_cont[s] = needs ? (value - am) : value;
            }
          }
          a.s_steps[s] = step;
          a.s_forced[s] = forced ? 1 : 0;
          a.s_overflow[s] = w_overflow ? 1 : 0;
        }
        ++walk;
        if (walk < walk_end) {
          // next walk of the same chunk: same point, cached first query
          const n2w_vec3 p0 = start_point();
          x = dev::v3(p0.x, p0.y, p0.z);
          src = 0.0f;
          step = 0;
          cont0 = 0;
          has_xm = false;
          w_overflow = false;
          ++wid;
          const float4 c = __ldg(a.first_cpd + pid);
          const int2 ii = __ldg(a.first_ids + pid);
          hit.cp = dev::v3(c.x, c.y, c.z);
          hit.d2 = c.w;
          hit.id = ii.x;
          hit.slot = ii.y;
        } else {
          alive = false;
        }
        continue;
      }
      if (kWalk == N2W_WALK_RESIDUAL && step == a.depth_m && !has_xm) {
        // X_m reached: remember it and the prefix source; the continuation gets a
        // fresh max_steps budget like the reference's nc_wos_from_point(X_m).
        xm = x;
        am = src;
        has_xm = true;
        cont0 = step;
      }
      const float R = a.step_scale * d;
      uint32_t k0 = a.k0, k1 = a.k1;
      if constexpr (kBatch) {
        k0 = a.insts[inst].k0;
        k1 = a.insts[inst].k1;
      }
      const U4 r = philox4x32_10(U4{static_cast<uint32_t>(wid), static_cast<uint32_t>(wid >> 32),
                                    static_cast<uint32_t>(step), 0u},
                                 k0, k1);
      const dev::V3 dir = unit_sphere(r.x, r.y);
      if constexpr (kBatch) {
        const BatchInst& I = a.insts[inst];
        if (I.has_source) src += ball_source(*I.problem, k0, k1, I.source_center, I.source_samples, x, R, wid, step, r.z);
      } else {
        if (a.has_source) src += ball_source(a.problem, k0, k1, a.source_center, a.source_samples, x, R, wid, step, r.z);
      }
      const int prev_slot = hit.slot;
      const dev::V3 xn = dev::v3(x.x + R * dir.x, x.y + R * dir.y, x.z + R * dir.z);
      const float* blo = a.box_lo;
      const float* bhi = a.box_hi;
      if constexpr (kBatch) {
        blo = a.insts[inst].box_lo;
        bhi = a.insts[inst].box_hi;
      }
      if (!(xn.x >= blo[0] && xn.x <= bhi[0] && xn.y >= blo[1] && xn.y <= bhi[1] && xn.z >= blo[2] &&
            xn.z <= bhi[2])) {
        // A walk from an interior point stays inside the mesh; leaving the
        // domain box means the start point was outside (a misclassified sample).
        // Stop it as forced, scored at the current closest point, instead of
        // letting it wander the unbounded exterior.
        step = cont0 + a.max_steps;
        continue;
      }
      x = xn;
      ++step;
      // Seed the next query with two real candidates (previous closest
      // triangle, seed-grid triangle at x); the exact answer is unchanged.
      hit.d2 = FLT_MAX;
      hit.id = INT32_MAX;
      hit.cp = x;
      dev::test_slot_fast(a.tris, prev_slot, x, hit);
      ++c_tris;
      const dev::SeedGrid& grid = [&]() -> const dev::SeedGrid& {
        if constexpr (kBatch) return a.insts[inst].grid;
        else return a.grid;
      }();
      if (grid.slots) {
        const int sg = dev::seed_slot(grid, x);
        if (sg != prev_slot) {
          dev::test_slot_fast(a.tris, sg, x, hit);
          ++c_tris;
        }
      }
      tv.sp = 0;
      if constexpr (kBatch) tv.ref = a.insts[inst].root;
      else tv.ref = 0;
      tv.leaf_cur = tv.leaf_end = 0;
      querying = true;
    }
    // (3) flush finished (or abandoned) chunks' accumulators; always before the
    //     exit test below, so nothing accumulated is ever dropped.
    if (kOut == kOutStats) {
      const bool want = !alive && walk >= walk_end && acc_n > 0;
      warp_flush<kBatch>(want, pid, inst, acc_s, acc_s2, acc_n, acc_steps, acc_forced, a);
      if (want) {
        acc_s = acc_s2 = 0.0;
        acc_n = acc_forced = acc_steps = 0;
      }
    }
    // (4) pop new chunks for idle lanes (one warp-aggregated atomic).
    const bool need = !alive && !exhausted;
    const unsigned need_mask = __ballot_sync(0xffffffffu, need);
    if (need_mask) {
      const int leader = __ffs(need_mask) - 1;
      unsigned long long base = 0;
      if (lane == leader) base = atomicAdd(a.queue, static_cast<unsigned long long>(__popc(need_mask)));
      base = __shfl_sync(0xffffffffu, base, leader);
      if (need) {
        const unsigned long long c = base + __popc(need_mask & ((1u << lane) - 1u));
        if (c < static_cast<unsigned long long>(a.total_chunks)) {
          int64_t lpid;  // point index within the instance (keys its walks' random streams)
          int wpp;
          if constexpr (kBatch) {
            // Instance of chunk c: the last one whose chunk_base <= c.
            int lo = 0, hi = a.n_insts - 1;
            while (lo < hi) {
              const int mid = (lo + hi + 1) >> 1;
              if (static_cast<unsigned long long>(a.insts[mid].chunk_base) <= c) lo = mid;
              else hi = mid - 1;
            }
            inst = lo;
            const BatchInst& I = a.insts[inst];
            const unsigned long long lc = c - static_cast<unsigned long long>(I.chunk_base);
            const unsigned long long cpp = static_cast<unsigned long long>(I.chunks_per_point);
            lpid = static_cast<int64_t>(lc / cpp);
            wpp = I.walks_per_point;
            walk = static_cast<int>((lc % cpp) * a.chunk);
            pid = I.point_base + lpid;
            wid = static_cast<uint64_t>(I.wid_base);
          } else {
            lpid = static_cast<int64_t>(c / static_cast<unsigned long long>(a.chunks_per_point));
            wpp = a.walks_per_point;
            walk = static_cast<int>((c % static_cast<unsigned long long>(a.chunks_per_point)) * a.chunk);
            pid = lpid;
            wid = 0;
          }
          walk_end = min(walk + a.chunk, wpp);
          const n2w_vec3 p0 = start_point();
          x = dev::v3(p0.x, p0.y, p0.z);
          src = 0.0f;
          step = 0;
          cont0 = 0;
          has_xm = false;
          w_overflow = false;
          wid += static_cast<uint64_t>(lpid) * static_cast<uint64_t>(wpp) + static_cast<uint64_t>(walk);
          const float4 cc = __ldg(a.first_cpd + pid);
          const int2 ii = __ldg(a.first_ids + pid);
          hit.cp = dev::v3(cc.x, cc.y, cc.z);
          hit.d2 = cc.w;
          hit.id = ii.x;
          hit.slot = ii.y;
          alive = true;  // its (cached) first query is consumed in the next Phase A
        } else {
          exhausted = true;
        }
      }
    }
    if (!__any_sync(0xffffffffu, alive)) break;

    // ================= Phase B =================
    for (;;) {
      const unsigned busy = __ballot_sync(0xffffffffu, querying);
      const unsigned waiting = __ballot_sync(0xffffffffu, !querying && alive);
      if (busy == 0 || __popc(waiting) >= a.regen) break;
      // kUnits = 2 runs two units of traversal per vote, written out twice: the
      // votes and the exit test cost about as much as a unit, and a lane that
      // finishes on the first unit waits at most one unit longer (headline
      // slice, same box: one unit 1,031, two 1,070, three 1,040 M
      // walk-steps/s; the two units as an unrolled loop 1,054).  Compiled in,
      // the second unit slows walks whose steps carry several source samples
      // (16 per ball: 29.4 ns per walk with one unit, 31.4 with the second
      // unit present even when it is skipped), so they run the kUnits = 1
      // kernel.
      if (querying) {
        bool ov = false;
        if (!dev::trav_step_fast(a.nodes, a.tris, x, hit, tv, stack, c_nodes, c_tris, ov)) querying = false;
        if (ov) {
          w_overflow = true;
          ++c_overflow;
        }
      }
      if constexpr (kUnits == 2) {
        if (querying) {
          bool ov = false;
          if (!dev::trav_step_fast(a.nodes, a.tris, x, hit, tv, stack, c_nodes, c_tris, ov)) querying = false;
          if (ov) {
            w_overflow = true;
            ++c_overflow;
          }
        }
      }
    }
    if (a.counters && (c_nodes >= 0x40000000u || c_tris >= 0x40000000u)) {
      atomicAdd(&a.counters->node_visits, static_cast<unsigned long long>(c_nodes));
      atomicAdd(&a.counters->tri_tests, static_cast<unsigned long long>(c_tris));
      c_nodes = c_tris = 0;
    }
  }

  if (a.counters) {
    const unsigned long long s_walks = warp_sum_u64(c_walks), s_steps = warp_sum_u64(c_steps),
                             s_queries = warp_sum_u64(c_queries), s_nodes = warp_sum_u64(c_nodes),
                             s_tris = warp_sum_u64(c_tris), s_over = warp_sum_u64(c_overflow),
                             s_forced = warp_sum_u64(c_forced), s_timeout = warp_sum_u64(c_timeout);
    if (lane == 0) {
      atomicAdd(&a.counters->walks, s_walks);
      atomicAdd(&a.counters->steps, s_steps);
      atomicAdd(&a.counters->queries, s_queries);
      atomicAdd(&a.counters->node_visits, s_nodes);
      atomicAdd(&a.counters->tri_tests, s_tris);
      atomicAdd(&a.counters->overflow, s_over);
      atomicAdd(&a.counters->forced, s_forced);
      atomicAdd(&a.counters->timed_out, s_timeout);
    }
  }
}

// ---- per-point first query ----------------------------------------------------
__global__ void __launch_bounds__(256) first_query_kernel(const float4* __restrict__ nodes,
                                                          const float4* __restrict__ tris, const dev::SeedGrid grid,
                                                          const n2w_vec3* __restrict__ points, int64_t n,
                                                          float4* __restrict__ cpd, int2* __restrict__ ids,
                                                          n2w_walk_counters* counters) {
  const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const n2w_vec3 pt = points[i];
  const dev::V3 p = dev::v3(pt.x, pt.y, pt.z);
  dev::ClosestHit hit;
  hit.d2 = FLT_MAX;
  hit.id = INT32_MAX;
  hit.slot = -1;
  hit.cp = p;
  dev::TraversalStats st{0, 0, 0};
  if (grid.slots) {
    dev::test_slot(tris, dev::seed_slot(grid, p), p, hit);
    ++st.tri_tests;
  }
  dev::traverse<true>(nodes, tris, p, hit, st);
  cpd[i] = make_float4(hit.cp.x, hit.cp.y, hit.cp.z, hit.d2);
  ids[i] = make_int2(hit.id, hit.slot);
  if (counters) {
    atomicAdd(&counters->node_visits, static_cast<unsigned long long>(st.node_visits));
    atomicAdd(&counters->tri_tests, static_cast<unsigned long long>(st.tri_tests));
    if (st.overflow) atomicAdd(&counters->overflow, 1ull);
  }
}

// First queries of a batched launch: point i belongs to the last instance whose
// point_base <= i; its query starts at that instance's root in the merged scene.
__global__ void __launch_bounds__(256) first_query_batch_kernel(const __grid_constant__ WalkArgs a, int64_t n,
                                                                float4* __restrict__ cpd, int2* __restrict__ ids) {
  const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int lo = 0, hi = a.n_insts - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (a.insts[mid].point_base <= i) lo = mid;
    else hi = mid - 1;
  }
  const BatchInst& I = a.insts[lo];
  const n2w_vec3 pt = I.points[i - I.point_base];
  const dev::V3 p = dev::v3(pt.x, pt.y, pt.z);
  dev::ClosestHit hit;
  hit.d2 = FLT_MAX;
  hit.id = INT32_MAX;
  hit.slot = -1;
  hit.cp = p;
  dev::TraversalStats st{0, 0, 0};
  if (I.grid.slots) {
    dev::test_slot(a.tris, dev::seed_slot(I.grid, p), p, hit);
    ++st.tri_tests;
  }
  dev::traverse<true>(a.nodes, a.tris, p, hit, st, I.root);
  cpd[i] = make_float4(hit.cp.x, hit.cp.y, hit.cp.z, hit.d2);
  ids[i] = make_int2(hit.id, hit.slot);
  if (a.counters) {
    atomicAdd(&a.counters->node_visits, static_cast<unsigned long long>(st.node_visits));
    atomicAdd(&a.counters->tri_tests, static_cast<unsigned long long>(st.tri_tests));
    if (st.overflow) atomicAdd(&a.counters->overflow, 1ull);
  }
}

// ---- per-sample reduction and 2LMC combination ------------------------------
__global__ void reduce_samples_kernel(const float* __restrict__ values, const int* __restrict__ steps,
                                      const int* __restrict__ forced, int64_t points, int W,
                                      double* sum, double* sum_sq, uint32_t* count, uint64_t* st,
                                      uint32_t* fc) {
  // One warp per (point, 32*k slice): lanes stride the point's samples, then a
  // shuffle butterfly and one FP64 atomic per warp.
  const int64_t warp = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  const int64_t warps_per_point = (W + 1023) / 1024;
  const int64_t pid = warp / warps_per_point;
  if (pid >= points) return;
  const int64_t part = warp % warps_per_point;
  const int j0 = static_cast<int>(part * 1024);
  const int j1 = min(W, j0 + 1024);
  double s = 0.0, s2 = 0.0;
  unsigned long long ns = 0;
  unsigned n = 0, f = 0;
  for (int j = j0 + lane; j < j1; j += 32) {
    const int64_t k = pid * W + j;
    const double v = values[k];
    s += v;
    s2 += v * v;
    ++n;
    if (steps) ns += static_cast<unsigned long long>(steps[k]);
    if (forced) f += forced[k] ? 1u : 0u;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    s += shfl_xor_d(s, o);
    s2 += shfl_xor_d(s2, o);
    ns += __shfl_xor_sync(0xffffffffu, ns, o);
    n += __shfl_xor_sync(0xffffffffu, n, o);
    f += __shfl_xor_sync(0xffffffffu, f, o);
  }
  if (lane == 0) {
    atomicAdd(sum + pid, s);
    atomicAdd(sum_sq + pid, s2);
    atomicAdd(count + pid, n);
    if (st) atomicAdd(reinterpret_cast<unsigned long long*>(st) + pid, ns);
    if (fc) atomicAdd(fc + pid, f);
  }
}

__global__ void combine_kernel(const float* __restrict__ cache, const float* __restrict__ boundary,
                               const float* __restrict__ cont, const uint8_t* __restrict__ needs,
                               int64_t n, float* __restrict__ nc, float* __restrict__ residual) {
  const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n) return;
  if (needs[i]) {
    const float c = cache[i];
    nc[i] = boundary[i] + c;
    residual[i] = cont[i] - c;
  } else {
    nc[i] = boundary[i];
    residual[i] = 0.0f;
  }
}

// ---- host side -----------------------------------------------------------
namespace {

template <int kOut, int kWalk, bool kBatch = false, int kMinBlocks = kWalkerMinBlocks, int kUnits = 1>
void launch_walker(const WalkArgs& a, int block, int blocks_per_sm, cudaStream_t stream) {
  auto kern = walker_kernel<kOut, kWalk, kBatch, kMinBlocks, kUnits>;
  int occ = 0;
  N2W_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, block, 0));
  if (occ < 1) occ = 1;
  const int per_sm = blocks_per_sm > 0 ? std::min(blocks_per_sm, occ) : occ;
  const int64_t lanes_needed = a.total_chunks;
  int64_t grid = static_cast<int64_t>(sm_count_current()) * per_sm;
  grid = std::min<int64_t>(grid, (lanes_needed + block - 1) / block);
  grid = std::max<int64_t>(grid, 1);
  kern<<<static_cast<unsigned>(grid), block, 0, stream>>>(a);
  N2W_CUDA(cudaGetLastError());
}

}  // namespace

void launch_first_query_batch(const WalkArgs& a, int64_t total_points, float4* cpd, int2* ids, cudaStream_t s) {
  if (total_points == 0) return;
  const int block = 256;
  first_query_batch_kernel<<<static_cast<unsigned>((total_points + block - 1) / block), block, 0, s>>>(
      a, total_points, cpd, ids);
  N2W_CUDA(cudaGetLastError());
}

// Two register budgets for the batched walker: 64 registers (4 resident
// 256-thread blocks per SM, some spills of the per-instance state) or 80
// registers (3 blocks, fewer spills); the autotuner picks one per workload.
void launch_walker_batch(const WalkArgs& a, int block, int blocks_per_sm, int reg_variant, cudaStream_t s) {
  if (a.total_chunks == 0) return;
  if (reg_variant == 1) launch_walker<kOutStats, N2W_WALK_PURE, true, 3>(a, block, blocks_per_sm, s);
  else launch_walker<kOutStats, N2W_WALK_PURE, true, 4>(a, block, blocks_per_sm, s);
}

int walker_batch_occupancy(int block, int reg_variant) {
  int occ = 0;
  if (reg_variant == 1) {
    N2W_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, walker_kernel<kOutStats, N2W_WALK_PURE, true, 3>,
                                                            block, 0));
  } else {
    N2W_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, walker_kernel<kOutStats, N2W_WALK_PURE, true, 4>,
                                                            block, 0));
  }
  return occ;
}

void validate_walk_options(const n2w_walk_options& o) {
  N2W_REQUIRE(o.walks_per_point > 0, "walks_per_point must be positive");
  N2W_REQUIRE(o.max_steps > 0, "max_steps must be positive");
  N2W_REQUIRE(o.depth_m >= 0, "depth_m must be non-negative");
  N2W_REQUIRE(o.epsilon > 0.0f, "epsilon must be positive");
  N2W_REQUIRE(o.step_scale > 0.0f && o.step_scale <= 1.0f, "step_scale must be in (0, 1]");
  N2W_REQUIRE(o.block_size == 0 || (o.block_size >= 32 && o.block_size <= kWalkerMaxThreads && o.block_size % 32 == 0),
              "walker block_size must be 0 or a multiple of 32 in [32, 256]");
  N2W_REQUIRE(o.chunk >= 0, "chunk must be non-negative");
  N2W_REQUIRE(o.regen_threshold >= 0 && o.regen_threshold <= 32, "regen_threshold must be in [0, 32]");
  N2W_REQUIRE(o.blocks_per_sm >= 0, "blocks_per_sm must be non-negative");
}

void validate_problem(const n2w_problem& p) {
  const int m = p.mode;
  const bool ok = (m >= 0 && m <= 16) || m == N2W_BC_POISSON_MULTISCALE || m == N2W_BC_POISSON_FIGLIKE_HF ||
                  m == N2W_BC_POISSON_FIGLIKE_HF_X5 || m == N2W_BC_CHARGES_SEEDED || m == N2W_BC_POISSON_SINPROD;
  N2W_REQUIRE(ok, "unsupported boundary mode " + std::to_string(m));
  N2W_REQUIRE(p.source_sampling == N2W_SOURCE_BALL || p.source_sampling == N2W_SOURCE_CENTER,
              "source_sampling must be N2W_SOURCE_BALL or N2W_SOURCE_CENTER");
  N2W_REQUIRE(p.source_samples >= 0 && p.source_samples <= 64, "source_samples must be in [0, 64]");
  if (m == N2W_BC_CHARGES_SEEDED) {
    N2W_REQUIRE(p.charge_count >= 1 && p.charge_count <= N2W_MAX_CHARGES, "charge_count must be in [1, 16]");
  }
}

WalkArgs make_walk_args(const n2w_bvh& bvh, const n2w_problem& problem, const n2w_vec3* d_points,
                        int64_t point_count, const n2w_walk_options& o, uint32_t stream_tag) {
  WalkArgs a{};
  a.nodes = reinterpret_cast<const float4*>(bvh.d_nodes);
  a.tris = reinterpret_cast<const float4*>(bvh.d_tris);
  a.grid = seed_grid_of(bvh);
  for (int k = 0; k < 3; ++k) {
    a.box_lo[k] = bvh.d_seed ? bvh.seed_lo[k] : -1.0e30f;
    a.box_hi[k] = bvh.d_seed ? bvh.seed_lo[k] + bvh.seed_h * static_cast<float>(bvh.seed_n) : 1.0e30f;
  }
  a.points = d_points;
  a.walks_per_point = o.walks_per_point;
  a.chunk = o.chunk > 0 ? std::min(o.chunk, o.walks_per_point) : std::min(kDefaultChunk, o.walks_per_point);
  a.chunks_per_point = (o.walks_per_point + a.chunk - 1) / a.chunk;
  a.regen = o.regen_threshold > 0 ? o.regen_threshold : kDefaultRegen;
  a.total_chunks = point_count * a.chunks_per_point;
  a.max_steps = o.max_steps;
  a.depth_m = o.depth_m;
  a.eps = o.epsilon;
  a.step_scale = o.step_scale;
  philox_key(o.seed, stream_tag, a.k0, a.k1);
  a.problem = problem;
  a.has_source = problem_has_source(problem) ? 1 : 0;
  a.source_center = problem.source_sampling == N2W_SOURCE_CENTER ? 1 : 0;
  a.source_samples = problem.source_samples > 1 ? problem.source_samples : 1;
  a.deadline_ns = o.deadline_ns;
  return a;
}

// Workspace layout: [0, 8) queue counter, [256, 320) run counters when the
// caller passes none, [512, 512 + 16 n) first-query points+d2 (float4),
// then 8 n bytes of first-query (id, slot) pairs.
constexpr size_t kWsHeader = 512;

void run_walker(WalkArgs& a, int64_t point_count, int out_kind, int walk_mode, const n2w_walk_options& o,
                n2w_walk_counters* d_counters, void* d_workspace, cudaStream_t stream) {
  if (a.total_chunks == 0) return;
  const size_t ws_bytes = n2w_wos_workspace_bytes(point_count);
  void* ws = d_workspace;
  bool own = false;
  if (!ws) {
    ws = scratch_alloc(ws_bytes, stream);
    own = true;
  }
  char* base = reinterpret_cast<char*>(ws);
  N2W_CUDA(cudaMemsetAsync(ws, 0, kWsHeader, stream));
  a.queue = reinterpret_cast<unsigned long long*>(base);
  a.counters = d_counters ? d_counters : reinterpret_cast<n2w_walk_counters*>(base + 256);
  if (d_counters) N2W_CUDA(cudaMemsetAsync(d_counters, 0, sizeof(n2w_walk_counters), stream));
  float4* cpd = reinterpret_cast<float4*>(base + kWsHeader);
  int2* ids = reinterpret_cast<int2*>(base + kWsHeader + 16 * static_cast<size_t>(point_count));
  a.first_cpd = cpd;
  a.first_ids = ids;
  {
    const int block = 256;
    const int64_t grid = (point_count + block - 1) / block;
    first_query_kernel<<<static_cast<unsigned>(grid), block, 0, stream>>>(a.nodes, a.tris, a.grid, a.points,
                                                                          point_count, cpd, ids, a.counters);
    N2W_CUDA(cudaGetLastError());
  }
  const int block = o.block_size > 0 ? o.block_size : kDefaultWalkerThreads;
  if (out_kind == kOutStats) {
    // two traversal units per vote unless the steps carry several source samples
    if (a.has_source && a.source_samples > 1) launch_walker<kOutStats, N2W_WALK_PURE>(a, block, o.blocks_per_sm, stream);
    else launch_walker<kOutStats, N2W_WALK_PURE, false, kWalkerMinBlocks, 2>(a, block, o.blocks_per_sm, stream);
  }
  else if (out_kind == kOutSamples) launch_walker<kOutSamples, N2W_WALK_PURE>(a, block, o.blocks_per_sm, stream);
  else if (walk_mode == N2W_WALK_PREFIX) launch_walker<kOutPrefix, N2W_WALK_PREFIX>(a, block, o.blocks_per_sm, stream);
  else launch_walker<kOutPrefix, N2W_WALK_RESIDUAL>(a, block, o.blocks_per_sm, stream);
  if (own) scratch_free(ws, stream);
}

void zero_stats(const n2w_point_stats& s, int64_t n, cudaStream_t stream) {
  N2W_CUDA(cudaMemsetAsync(s.d_sum, 0, sizeof(double) * n, stream));
  N2W_CUDA(cudaMemsetAsync(s.d_sum_sq, 0, sizeof(double) * n, stream));
  N2W_CUDA(cudaMemsetAsync(s.d_count, 0, sizeof(uint32_t) * n, stream));
  N2W_CUDA(cudaMemsetAsync(s.d_steps, 0, sizeof(uint64_t) * n, stream));
  N2W_CUDA(cudaMemsetAsync(s.d_forced, 0, sizeof(uint32_t) * n, stream));
}

}  // namespace n2w

using namespace n2w;

extern "C" {

size_t n2w_wos_workspace_bytes(int64_t point_count) {
  return kWsHeader + 24 * static_cast<size_t>(point_count < 0 ? 0 : point_count);
}

int n2w_wos_estimate(const n2w_bvh* bvh, const n2w_problem* problem, const n2w_vec3* d_points,
                     int64_t point_count, const n2w_walk_options* options, n2w_point_stats stats,
                     n2w_walk_counters* d_counters, void* d_workspace, n2w_stream_t stream) {
  return guarded([&] {
    N2W_REQUIRE(bvh && bvh->d_nodes && problem && options, "n2w_wos_estimate: null argument");
    N2W_REQUIRE(point_count >= 0, "point_count must be non-negative");
    validate_walk_options(*options);
    validate_problem(*problem);
    if (point_count == 0) return;
    N2W_REQUIRE(d_points && stats.d_sum && stats.d_sum_sq && stats.d_count && stats.d_steps && stats.d_forced,
                "n2w_wos_estimate: null device pointer");
    if (!options->accumulate) zero_stats(stats, point_count, stream);
    WalkArgs a = make_walk_args(*bvh, *problem, d_points, point_count, *options, 0);
    a.sum = stats.d_sum;
    a.sum_sq = stats.d_sum_sq;
    a.count = stats.d_count;
    a.steps = stats.d_steps;
    a.forced = stats.d_forced;
    run_walker(a, point_count, kOutStats, N2W_WALK_PURE, *options, d_counters, d_workspace, stream);
  });
}

}  // extern "C"

// ---- allocation-free variant of n2w_wos_estimate ----------------------------
// Some callers cannot allocate device memory while they solve: applications
// that give the library a fixed share of HBM up front and forbid it any other
// allocation, and serving loops that must never call cudaMalloc or
// cudaMallocAsync on the request path (cudaMalloc can synchronise the device
// and stall every stream).  For them, the walker's scratch (queue counter, run
// counters, each point's cached first query) lives in this static device
// array.  Every GPU that loads the library holds it until the process exits.
static __device__ __align__(256) unsigned char g_noalloc_scratch[N2W_NOALLOC_SCRATCH_BYTES];

namespace {

// In host code the array's name is only a host-side stand-in; its device
// address is looked up with the current device on every call
// (cudaGetSymbolAddress allocates nothing), so the address stays right after a
// cudaDeviceReset has reloaded the module.  The first lookup on a device loads
// the module, which is why the first call must come before any stream capture.
void* noalloc_scratch_current_device() {
  void* p = nullptr;
  const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
  if (e != cudaSuccess || !p) {
    throw Error(N2W_ECUDA, std::string("cudaGetSymbolAddress for the allocation-free scratch failed: ") +
                               cudaGetErrorString(e));
  }
  return p;
}

}  // namespace

extern "C" {

int n2w_wos_estimate_noalloc(const n2w_bvh* bvh, const n2w_problem* problem, const n2w_vec3* d_points,
                             int64_t point_count, const n2w_walk_options* options, n2w_point_stats stats,
                             n2w_walk_counters* d_counters, n2w_stream_t stream) {
  void* scratch = nullptr;
  const int st = guarded([&] {
    N2W_REQUIRE(point_count <= static_cast<int64_t>(N2W_NOALLOC_MAX_POINTS),
                "n2w_wos_estimate_noalloc: " + std::to_string(point_count) + " points exceed the limit of " +
                    std::to_string(N2W_NOALLOC_MAX_POINTS) + " points of the static " +
                    std::to_string(N2W_NOALLOC_SCRATCH_BYTES) +
                    "-byte scratch; split the points or call n2w_wos_estimate with a workspace");
    scratch = noalloc_scratch_current_device();
  });
  if (st != N2W_OK) return st;
  // The scratch is passed as the caller workspace, so nothing is allocated.
  return n2w_wos_estimate(bvh, problem, d_points, point_count, options, stats, d_counters, scratch, stream);
}

int n2w_wos_pure_samples(const n2w_bvh* bvh, const n2w_problem* problem, const n2w_vec3* d_points,
                         int64_t point_count, const n2w_walk_options* options,
                         float* d_sample_values, int* d_step_count, int* d_forced_max_steps,
                         int* d_query_overflow, n2w_stream_t stream) {
  return guarded([&] {
    N2W_REQUIRE(bvh && bvh->d_nodes && problem && options, "n2w_wos_pure_samples: null argument");
    N2W_REQUIRE(point_count >= 0, "point_count must be non-negative");
    validate_walk_options(*options);
    validate_problem(*problem);
    if (point_count == 0) return;
    N2W_REQUIRE(d_points && d_sample_values && d_step_count && d_forced_max_steps && d_query_overflow,
                "n2w_wos_pure_samples: null device pointer");
    WalkArgs a = make_walk_args(*bvh, *problem, d_points, point_count, *options, 0);
    a.s_value = d_sample_values;
    a.s_steps = d_step_count;
    a.s_forced = d_forced_max_steps;
    a.s_overflow = d_query_overflow;
    run_walker(a, point_count, kOutSamples, N2W_WALK_PURE, *options, nullptr, nullptr, stream);
  });
}

int n2w_wos_prefix_samples(const n2w_bvh* bvh, const n2w_problem* problem,
                           const n2w_vec3* d_points, int64_t point_count,
                           const n2w_walk_options* options, int mode, const float* input_min,
                           const float* input_extent, float* d_prefix_inputs,
                           float* d_boundary_values, float* d_continuation_values,
                           uint8_t* d_needs_cache, int* d_step_count, int* d_forced_max_steps,
                           int* d_query_overflow, n2w_stream_t stream) {
  return guarded([&] {
    N2W_REQUIRE(bvh && bvh->d_nodes && problem && options && input_min && input_extent,
                "n2w_wos_prefix_samples: null argument");
    N2W_REQUIRE(mode == N2W_WALK_PREFIX || mode == N2W_WALK_RESIDUAL, "mode must be PREFIX or RESIDUAL");
    N2W_REQUIRE(point_count >= 0, "point_count must be non-negative");
    validate_walk_options(*options);
    validate_problem(*problem);
    if (point_count == 0) return;
    N2W_REQUIRE(d_points && d_prefix_inputs && d_boundary_values && d_needs_cache && d_step_count &&
                    d_forced_max_steps && d_query_overflow,
                "n2w_wos_prefix_samples: null device pointer");
    N2W_REQUIRE(mode == N2W_WALK_PREFIX || d_continuation_values, "RESIDUAL needs continuation values");
    WalkArgs a = make_walk_args(*bvh, *problem, d_points, point_count, *options, mode == N2W_WALK_PREFIX ? 1 : 2);
    for (int k = 0; k < 3; ++k) {
      a.in_min[k] = input_min[k];
      a.in_ext[k] = input_extent[k];
    }
    a.p_inputs = d_prefix_inputs;
    a.p_boundary = d_boundary_values;
    a.p_cont = d_continuation_values;
    a.p_needs = d_needs_cache;
    a.s_steps = d_step_count;
    a.s_forced = d_forced_max_steps;
    a.s_overflow = d_query_overflow;
    run_walker(a, point_count, kOutPrefix, mode, *options, nullptr, nullptr, stream);
  });
}

int n2w_wos_combine(const float* d_cache_outputs, const float* d_boundary_values,
                    const float* d_continuation_values, const uint8_t* d_needs_cache,
                    int64_t sample_count, float* d_nc_values, float* d_residual_values,
                    int block_size, n2w_stream_t stream) {
  return guarded([&] {
    N2W_REQUIRE(sample_count >= 0, "sample_count must be non-negative");
    if (sample_count == 0) return;
    N2W_REQUIRE(d_cache_outputs && d_boundary_values && d_continuation_values && d_needs_cache && d_nc_values &&
                    d_residual_values,
                "n2w_wos_combine: null pointer");
    N2W_REQUIRE(block_size >= 1 && block_size <= 1024, "block_size must be in [1,1024]");
    const int64_t grid = (sample_count + block_size - 1) / block_size;
    combine_kernel<<<static_cast<unsigned>(grid), block_size, 0, stream>>>(
        d_cache_outputs, d_boundary_values, d_continuation_values, d_needs_cache, sample_count, d_nc_values,
        d_residual_values);
    N2W_CUDA(cudaGetLastError());
  });
}

int n2w_reduce_samples(const float* d_values, const int* d_step_count, const int* d_forced,
                       int64_t point_count, int walks_per_point, n2w_point_stats stats, int accumulate,
                       n2w_stream_t stream) {
  return guarded([&] {
    N2W_REQUIRE(point_count >= 0 && walks_per_point > 0, "invalid sizes");
    if (point_count == 0) return;
    N2W_REQUIRE(d_values && stats.d_sum && stats.d_sum_sq && stats.d_count, "n2w_reduce_samples: null pointer");
    if (!accumulate) {
      N2W_CUDA(cudaMemsetAsync(stats.d_sum, 0, sizeof(double) * point_count, stream));
      N2W_CUDA(cudaMemsetAsync(stats.d_sum_sq, 0, sizeof(double) * point_count, stream));
      N2W_CUDA(cudaMemsetAsync(stats.d_count, 0, sizeof(uint32_t) * point_count, stream));
      if (stats.d_steps) N2W_CUDA(cudaMemsetAsync(stats.d_steps, 0, sizeof(uint64_t) * point_count, stream));
      if (stats.d_forced) N2W_CUDA(cudaMemsetAsync(stats.d_forced, 0, sizeof(uint32_t) * point_count, stream));
    }
    const int64_t warps = point_count * ((walks_per_point + 1023) / 1024);
    const int block = 256;
    const int64_t grid = (warps * 32 + block - 1) / block;
    reduce_samples_kernel<<<static_cast<unsigned>(grid), block, 0, stream>>>(
        d_values, d_step_count, d_forced, point_count, walks_per_point, stats.d_sum, stats.d_sum_sq, stats.d_count,
        d_step_count ? stats.d_steps : nullptr, d_forced ? stats.d_forced : nullptr);
    N2W_CUDA(cudaGetLastError());
  });
}

}  // extern "C"
