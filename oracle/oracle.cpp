// ORACLE — test infrastructure only.  CPU restatement of the reference's hot
// path, used by tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg
// as the checker.  Never linked into or called by the product library.
//
// Parity pinning: the closest-point functions are checked bit-for-bit against
// the reference's own CPU code compiled from its sources (oracle/_ref) and
// against committed golden vectors generated from it (tests/golden/).
//
// Contents (reference paths inside Somatic-Cell/n2wos-cuda):
//   oracle_closest_point_on_triangle  src/geometry/closest_point.cpp:7-48
//   oracle_bruteforce                 src/geometry/closest_point.cpp:50-68 (+ tie counts)
//   oracle_traverse4                  the product's 4-wide traversal restated over
//                                     its copied layout, to count node visits and
//                                     triangle tests (algorithmic bytes)
//   oracle_wos                        one-walk-per-sample WoS restating
//                                     nc_wos_from_point, src/cuda/cubql_bvh.cu:1323-1357,
//                                     with the unit-sphere sampler of 254-261 and the
//                                     Poisson centre rule of
//                                     include/n2wos/nc_poisson_manufactured.hpp:151-157
//                                     or the in-ball Green's-function sample.
//   oracle_philox4x32_10              Philox4x32-10, Salmon et al. SC'11
// Build: g++ -O2 -ffp-contract=off (no FMA contraction: IEEE float per operation,
// the same arithmetic as the reference's g++ build).
#include <algorithm>
#include <array>
#include <atomic>
#include <cfloat>
#include <climits>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <map>
#include <thread>
#include <utility>
#include <vector>

namespace {

struct V {
  float x, y, z;
};
inline V sub(V a, V b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline V add(V a, V b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline V mul(V a, float s) { return {a.x * s, a.y * s, a.z * s}; }
inline float dot(V a, V b) { return a.x * b.x + a.y * b.y + a.z * b.z; }

V closest_on_triangle(V p, V a, V b, V c) {
  const V ab = sub(b, a);
  const V ac = sub(c, a);
  const V ap = sub(p, a);
  const float d1 = dot(ab, ap);
  const float d2 = dot(ac, ap);
  if (d1 <= 0.0f && d2 <= 0.0f) return a;
  const V bp = sub(p, b);
  const float d3 = dot(ab, bp);
  const float d4 = dot(ac, bp);
  if (d3 >= 0.0f && d4 <= d3) return b;
  const float vc = d1 * d4 - d3 * d2;
  if (vc <= 0.0f && d1 >= 0.0f && d3 <= 0.0f) {
    const float v = d1 / (d1 - d3);
    return add(a, mul(ab, v));
  }
  const V cp = sub(p, c);
  const float d5 = dot(ab, cp);
  const float d6 = dot(ac, cp);
  if (d6 >= 0.0f && d5 <= d6) return c;
  const float vb = d5 * d2 - d1 * d6;
  if (vb <= 0.0f && d2 >= 0.0f && d6 <= 0.0f) {
    const float w = d2 / (d2 - d6);
    return add(a, mul(ac, w));
  }
  const float va = d3 * d6 - d5 * d4;
  if (va <= 0.0f && (d4 - d3) >= 0.0f && (d5 - d6) >= 0.0f) {
    const float w = (d4 - d3) / ((d4 - d3) + (d5 - d6));
    return add(b, mul(sub(c, b), w));
  }
  const float denom = 1.0f / (va + vb + vc);
  const float v = vb * denom;
  const float w = vc * denom;
  return add(add(a, mul(ab, v)), mul(ac, w));
}

template <typename F>
void parallel_for(int64_t n, int threads, F&& f) {
  if (threads <= 1 || n < 64) {
    for (int64_t i = 0; i < n; ++i) f(i);
    return;
  }
  std::atomic<int64_t> next{0};
  std::vector<std::thread> pool;
  for (int t = 0; t < threads; ++t) {
    pool.emplace_back([&] {
      for (;;) {
        const int64_t i0 = next.fetch_add(16);
        if (i0 >= n) break;
        for (int64_t i = i0; i < std::min<int64_t>(n, i0 + 16); ++i) f(i);
      }
    });
  }
  for (auto& th : pool) th.join();
}

// ---- the product's 4-wide layout, restated ----
struct Node4 {
  float lo_x[4], hi_x[4], lo_y[4], hi_y[4], lo_z[4], hi_z[4];
  int32_t child[4];
  int32_t pad[4];
};
struct TriRec {
  float v0[3];
  int32_t id;
  float v1[3];
  int32_t p1;
  float v2[3];
  int32_t p2;
};
constexpr int32_t kEmpty = INT32_MIN;

inline float gap(float p, float lo, float hi) { return std::fmax(std::fmax(lo - p, p - hi), 0.0f); }

struct Hit {
  float d2;
  int32_t id;
  V cp;
  int nodes, tris, overflow;
};

void traverse4(const Node4* nodes, const TriRec* tris, V p, Hit& h) {
  struct E {
    int32_t ref;
    float d;
  };
  E stack[64];
  int sp = 0;
  int32_t ref = 0;
  for (;;) {
    if (ref >= 0) {
      const Node4& n = nodes[ref];
      ++h.nodes;
      float d[4];
      int32_t r[4];
      for (int k = 0; k < 4; ++k) {
        const float dx = gap(p.x, n.lo_x[k], n.hi_x[k]);
        const float dy = gap(p.y, n.lo_y[k], n.hi_y[k]);
        const float dz = gap(p.z, n.lo_z[k], n.hi_z[k]);
        d[k] = dx * dx + dy * dy + dz * dz;
        r[k] = n.child[k];
      }
      auto cs = [&](int i, int j) {
        if (d[j] < d[i]) {
          std::swap(d[i], d[j]);
          std::swap(r[i], r[j]);
        }
      };
      cs(0, 1);
      cs(2, 3);
      cs(0, 2);
      cs(1, 3);
      cs(1, 2);
      const float best = h.d2;
      for (int k = 3; k >= 1; --k) {
        if (d[k] <= best) {
          if (sp < 64) stack[sp++] = {r[k], d[k]};
          else h.overflow = 1;
        }
      }
      ref = d[0] <= best ? r[0] : kEmpty;
    } else if (ref != kEmpty) {
      const int32_t first = (~ref) >> 3, count = ((~ref) & 7) + 1;
      for (int i = 0; i < count; ++i) {
        const TriRec& t = tris[first + i];
        ++h.tris;
        const V cp = closest_on_triangle(p, {t.v0[0], t.v0[1], t.v0[2]}, {t.v1[0], t.v1[1], t.v1[2]},
                                         {t.v2[0], t.v2[1], t.v2[2]});
        const V dv = sub(cp, p);
        const float dd = dot(dv, dv);
        if (dd < h.d2 || (dd == h.d2 && t.id < h.id)) {
          h.d2 = dd;
          h.id = t.id;
          h.cp = cp;
        }
      }
      ref = kEmpty;
    }
    if (ref == kEmpty) {
      bool found = false;
      while (sp > 0) {
        const E e = stack[--sp];
        if (e.d <= h.d2) {
          ref = e.ref;
          found = true;
          break;
        }
      }
      if (!found) break;
    }
  }
}

// ---- Philox4x32-10 ----
struct U4 {
  uint32_t x, y, z, w;
};
U4 philox(U4 c, uint32_t k0, uint32_t k1) {
  for (int r = 0; r < 10; ++r) {
    const uint64_t p0 = static_cast<uint64_t>(0xD2511F53u) * c.x;
    const uint64_t p1 = static_cast<uint64_t>(0xCD9E8D57u) * c.z;
    c = U4{static_cast<uint32_t>(p1 >> 32) ^ c.y ^ k0, static_cast<uint32_t>(p1),
           static_cast<uint32_t>(p0 >> 32) ^ c.w ^ k1, static_cast<uint32_t>(p0)};
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
  return c;
}
inline float u01(uint32_t v) { return static_cast<float>(v >> 8) * (1.0f / 16777216.0f); }

// ---- boundary problems used by the parity tests ----
struct Problem {
  int32_t mode;
  int32_t source_sampling;
  int32_t charge_count;
  float omega;
  float charges[16][4];
  int32_t source_samples;
  int32_t reserved;
};

float safe_sqrt(float r2) { return std::sqrt(std::fmax(r2, 1.0e-12f)); }

float g_value(const Problem& pb, V p) {
  switch (pb.mode) {
    case 0: return p.x * p.x - p.y * p.y;
    case 4: {  // Re((x + i y)^8)
      float ar = 1.0f, ai = 0.0f;
      for (int i = 0; i < 8; ++i) {
        const float nr = ar * p.x - ai * p.y;
        const float ni = ar * p.y + ai * p.x;
        ar = nr;
        ai = ni;
      }
      return ar;
    }
    case 12: return 1.0f;
    case 100: {
      float v = 0.0f;
      for (int k = 0; k < pb.charge_count; ++k) {
        const float dx = p.x - pb.charges[k][0], dy = p.y - pb.charges[k][1], dz = p.z - pb.charges[k][2];
        v += pb.charges[k][3] / safe_sqrt(dx * dx + dy * dy + dz * dz);
      }
      return v;
    }
    case 101: return std::sin(pb.omega * p.x) * std::sin(pb.omega * p.y) * std::sin(pb.omega * p.z);
    default: return NAN;
  }
}

float f_value(const Problem& pb, V p) {
  if (pb.mode == 101) return 3.0f * pb.omega * pb.omega * g_value(pb, p);
  return 0.0f;
}

}  // namespace

extern "C" {

int oracle_abi_version() { return 1; }

void oracle_closest_point_on_triangle(const float* p, const float* a, const float* b, const float* c, float* out) {
  const V r = closest_on_triangle({p[0], p[1], p[2]}, {a[0], a[1], a[2]}, {b[0], b[1], b[2]}, {c[0], c[1], c[2]});
  out[0] = r.x;
  out[1] = r.y;
  out[2] = r.z;
}

// Brute force over all triangles in index order; strict '<' keeps the lowest
// index among exact ties; tie_count = number of triangles at the minimum.
void oracle_bruteforce(const float* verts, const uint32_t* tris, int64_t nt, const float* points, int64_t n,
                       float* out_d2, float* out_cp, int32_t* out_id, int32_t* out_ties, int threads) {
  parallel_for(n, threads, [&](int64_t q) {
    const V p{points[3 * q], points[3 * q + 1], points[3 * q + 2]};
    float best = INFINITY;
    V bcp{0, 0, 0};
    int32_t bid = -1, ties = 0;
    for (int64_t i = 0; i < nt; ++i) {
      const uint32_t* t = tris + 3 * i;
      const V a{verts[3 * t[0]], verts[3 * t[0] + 1], verts[3 * t[0] + 2]};
      const V b{verts[3 * t[1]], verts[3 * t[1] + 1], verts[3 * t[1] + 2]};
      const V c{verts[3 * t[2]], verts[3 * t[2] + 1], verts[3 * t[2] + 2]};
      const V cp = closest_on_triangle(p, a, b, c);
      const V dv = sub(cp, p);
      const float d2 = dot(dv, dv);
      if (d2 < best) {
        best = d2;
        bcp = cp;
        bid = static_cast<int32_t>(i);
        ties = 1;
      } else if (d2 == best) {
        ++ties;
      }
    }
    out_d2[q] = best;
    out_cp[3 * q] = bcp.x;
    out_cp[3 * q + 1] = bcp.y;
    out_cp[3 * q + 2] = bcp.z;
    out_id[q] = bid;
    if (out_ties) out_ties[q] = ties;
  });
}

// Restated 4-wide traversal over the product layout (nodes 128 B, tris 48 B).
// When seed_slots is given, the triangle stored at the nearest seed-grid node
// (lattice lo + i/inv_h, n cells per axis) is tested first, as the kernel does.
void oracle_traverse4(const void* nodes, const void* tris, const float* points, int64_t n, float* out_d2,
                      float* out_cp, int32_t* out_id, int32_t* out_nodes, int32_t* out_tris, int threads,
                      const int32_t* seed_slots, const float* seed_lo, float seed_inv_h, int seed_n) {
  const Node4* nd = static_cast<const Node4*>(nodes);
  const TriRec* tr = static_cast<const TriRec*>(tris);
  parallel_for(n, threads, [&](int64_t q) {
    Hit h{FLT_MAX, INT32_MAX, {0, 0, 0}, 0, 0, 0};
    const V p{points[3 * q], points[3 * q + 1], points[3 * q + 2]};
    if (seed_slots) {
      auto idx = [&](float c, float lo) {
        const float f = (c - lo) * seed_inv_h;
        return static_cast<int64_t>(std::nearbyint(std::fmin(std::fmax(f, 0.0f), static_cast<float>(seed_n))));
      };
      const int64_t s = seed_n + 1;
      const int32_t slot = seed_slots[(idx(p.z, seed_lo[2]) * s + idx(p.y, seed_lo[1])) * s + idx(p.x, seed_lo[0])];
      const TriRec& t = tr[slot];
      ++h.tris;
      const V cp = closest_on_triangle(p, {t.v0[0], t.v0[1], t.v0[2]}, {t.v1[0], t.v1[1], t.v1[2]},
                                       {t.v2[0], t.v2[1], t.v2[2]});
      const V dv = sub(cp, p);
      const float dd = dot(dv, dv);
      if (dd < h.d2 || (dd == h.d2 && t.id < h.id)) {
        h.d2 = dd;
        h.id = t.id;
        h.cp = cp;
      }
    }
    traverse4(nd, tr, p, h);
    out_d2[q] = h.d2;
    out_cp[3 * q] = h.cp.x;
    out_cp[3 * q + 1] = h.cp.y;
    out_cp[3 * q + 2] = h.cp.z;
    out_id[q] = h.id == INT32_MAX ? -1 : h.id;
    if (out_nodes) out_nodes[q] = h.nodes;
    if (out_tris) out_tris[q] = h.tris;
  });
}

// Reference slice mask (src/cuda/cubql_bvh.cu:407-455): +x ray from
// p + (0, 1.928371e-6, 3.141593e-6), Möller–Trumbore with the reference's
// tolerances, against every triangle; inside iff the hit count is odd.
void oracle_inside_bruteforce(const float* verts, const uint32_t* tris, int64_t nt, const float* points, int64_t n,
                              uint8_t* out_inside, int threads) {
  parallel_for(n, threads, [&](int64_t q) {
    const V p{points[3 * q], points[3 * q + 1] + 1.928371e-6f, points[3 * q + 2] + 3.141593e-6f};
    int hits = 0;
    for (int64_t i = 0; i < nt; ++i) {
      const uint32_t* t = tris + 3 * i;
      const V a{verts[3 * t[0]], verts[3 * t[0] + 1], verts[3 * t[0] + 2]};
      const V b{verts[3 * t[1]], verts[3 * t[1] + 1], verts[3 * t[1] + 2]};
      const V c{verts[3 * t[2]], verts[3 * t[2] + 1], verts[3 * t[2] + 2]};
      const float y_min = std::min({a.y, b.y, c.y}), y_max = std::max({a.y, b.y, c.y});
      const float z_min = std::min({a.z, b.z, c.z}), z_max = std::max({a.z, b.z, c.z});
      const float x_max = std::max({a.x, b.x, c.x});
      if (p.y < y_min || p.y > y_max || p.z < z_min || p.z > z_max || p.x > x_max) continue;
      const V e1 = sub(b, a), e2 = sub(c, a);
      const V h{0.0f * e2.z - 0.0f * e2.y, 0.0f * e2.x - 1.0f * e2.z, 1.0f * e2.y - 0.0f * e2.x};
      const float det = dot(e1, h);
      if (std::fabs(det) < 1.0e-12f) continue;
      const float inv_det = 1.0f / det;
      const V s = sub(p, a);
      const float u = inv_det * dot(s, h);
      if (u < -1.0e-7f || u > 1.0f + 1.0e-7f) continue;
      const V qv{s.y * e1.z - s.z * e1.y, s.z * e1.x - s.x * e1.z, s.x * e1.y - s.y * e1.x};
      const float v = inv_det * dot(V{1.0f, 0.0f, 0.0f}, qv);
      if (v < -1.0e-7f || u + v > 1.0f + 1.0e-7f) continue;
      const float tt = inv_det * dot(e2, qv);
      if (tt > 1.0e-7f) ++hits;
    }
    out_inside[q] = (hits & 1) ? 1 : 0;
  });
}

void oracle_philox4x32_10(const uint32_t* ctr, uint32_t k0, uint32_t k1, uint32_t* out) {
  const U4 r = philox(U4{ctr[0], ctr[1], ctr[2], ctr[3]}, k0, k1);
  out[0] = r.x;
  out[1] = r.y;
  out[2] = r.z;
  out[3] = r.w;
}

}  // extern "C"

namespace {

// ---- the reference's host BVH layout (src/cuda/bvh_types.cuh:17-36) ----
struct RefVec {
  float x, y, z;
};
struct RefTri {
  RefVec v0, v1, v2;
};
struct RefNode {
  RefVec lo, hi;
  int32_t left, right, first, count;
};
static_assert(sizeof(RefTri) == 36 && sizeof(RefNode) == 40, "reference layout");

inline V rv(RefVec a) { return {a.x, a.y, a.z}; }

// d_aabb_distance2 (src/cuda/bvh_types.cuh:79-90), same operation order.
inline float ref_aabb_d2(V p, RefVec lo, RefVec hi) {
  float dx = 0.0f;
  if (p.x < lo.x) dx = lo.x - p.x;
  if (p.x > hi.x) dx = p.x - hi.x;
  float dy = 0.0f;
  if (p.y < lo.y) dy = lo.y - p.y;
  if (p.y > hi.y) dy = p.y - hi.y;
  float dz = 0.0f;
  if (p.z < lo.z) dz = lo.z - p.z;
  if (p.z > hi.z) dz = p.z - hi.z;
  return dx * dx + dy * dy + dz * dz;
}

// Closest point over the reference's binary BVH, restating
// closest_point_bvh_kernel (src/cuda/bvh_query.cu:75-160): a 128-entry stack,
// cull when the node's box is farther than the best so far, the far child
// pushed before the near one, strict '<' on triangle distances (the first
// visited triangle wins a tie), triangles through triangle_indices.
struct RefBvh {
  const RefNode* nodes;
  const RefTri* tris;
  const int32_t* idx;

  void query(V p, Hit& h) const {
    constexpr int kStack = 128;
    int stack[kStack];
    int sp = 0;
    stack[sp++] = 0;
    while (sp > 0) {
      const RefNode& node = nodes[stack[--sp]];
      ++h.nodes;
      if (ref_aabb_d2(p, node.lo, node.hi) > h.d2) continue;
      if (node.count > 0) {
        for (int i = 0; i < node.count; ++i) {
          const int32_t t = idx[node.first + i];
          const RefTri& tr = tris[t];
          ++h.tris;
          const V cp = closest_on_triangle(p, rv(tr.v0), rv(tr.v1), rv(tr.v2));
          const V dv = sub(cp, p);
          const float d2 = dot(dv, dv);
          if (d2 < h.d2) {
            h.d2 = d2;
            h.cp = cp;
            h.id = t;
          }
        }
      } else if (node.left >= 0 && node.right >= 0) {
        const float dl = ref_aabb_d2(p, nodes[node.left].lo, nodes[node.left].hi);
        const float dr = ref_aabb_d2(p, nodes[node.right].lo, nodes[node.right].hi);
        int near_id = node.left, far_id = node.right;
        float near_d2 = dl, far_d2 = dr;
        if (dr < dl) {
          near_id = node.right;
          far_id = node.left;
          near_d2 = dr;
          far_d2 = dl;
        }
        if (far_d2 <= h.d2) {
          if (sp < kStack) stack[sp++] = far_id;
          else h.overflow = 1;
        }
        if (near_d2 <= h.d2) {
          if (sp < kStack) stack[sp++] = near_id;
          else h.overflow = 1;
        }
      }
    }
  }
};

// The product's 4-wide layout as a query.
struct Bvh4 {
  const Node4* nodes;
  const TriRec* tris;
  void query(V p, Hit& h) const { traverse4(nodes, tris, p, h); }
};

// +x ray test of one triangle, ray_x_intersects_triangle
// (src/cuda/cubql_bvh.cu:407-426) with its tolerances.
bool ray_x_hits(V p, V a, V b, V c) {
  const float y_min = std::min({a.y, b.y, c.y}), y_max = std::max({a.y, b.y, c.y});
  const float z_min = std::min({a.z, b.z, c.z}), z_max = std::max({a.z, b.z, c.z});
  const float x_max = std::max({a.x, b.x, c.x});
  if (p.y < y_min || p.y > y_max || p.z < z_min || p.z > z_max || p.x > x_max) return false;
  const V e1 = sub(b, a), e2 = sub(c, a);
  const V h{0.0f * e2.z - 0.0f * e2.y, 0.0f * e2.x - 1.0f * e2.z, 1.0f * e2.y - 0.0f * e2.x};
  const float det = dot(e1, h);
  if (std::fabs(det) < 1.0e-12f) return false;
  const float inv_det = 1.0f / det;
  const V s = sub(p, a);
  const float u = inv_det * dot(s, h);
  if (u < -1.0e-7f || u > 1.0f + 1.0e-7f) return false;
  const V qv{s.y * e1.z - s.z * e1.y, s.z * e1.x - s.x * e1.z, s.x * e1.y - s.y * e1.x};
  const float v = inv_det * dot(V{1.0f, 0.0f, 0.0f}, qv);
  if (v < -1.0e-7f || u + v > 1.0f + 1.0e-7f) return false;
  const float tt = inv_det * dot(e2, qv);
  return tt > 1.0e-7f;
}

// ---- one walk (reference nc_wos_from_point, src/cuda/cubql_bvh.cu:1323-1357,
//      and the prefix / 2LMC walks of 1451-1606) ----
constexpr int kModePure = 0;      // walk to the boundary
constexpr int kModePrefix = 1;    // nc_hybrid_prefix_kernel: stop at depth m (needs the cache)
constexpr int kModeResidual = 2;  // nc_2lmc_prefix_continue_kernel: prefix to m, then continue

struct WalkRec {
  float value;     // pure: the walk's value; prefix / residual: boundary_values[]
  float cont;      // residual: continuation_values[] (prefix source excluded)
  V xo;            // position mapped to prefix_inputs[] (X_m, or where the walk stopped)
  int needs;       // needs_cache[]
  int steps;       // step_count[] (prefix + continuation steps)
  int forced;      // forced_max_steps[]
};

// Directions and source samples use the product's Philox streams, so a walk
// (w, key) is reproducible: stream 0 gives (z, phi, source radius word), stream
// 1 + k the k-th in-ball source sample.  Parity with the product is statistical.
inline V sphere_dir(uint32_t a, uint32_t b) {
  const float z = 1.0f - 2.0f * u01(a);
  const float phi = 2.0f * 3.14159265358979323846f * u01(b);
  const float rr = std::sqrt(std::fmax(0.0f, 1.0f - z * z));
  return {rr * std::cos(phi), rr * std::sin(phi), z};
}

inline float green_fraction(uint32_t u) {
  const float a = std::acos(std::fmin(1.0f, std::fmax(-1.0f, 1.0f - 2.0f * u01(u))));
  return 0.5f + std::cos((a - 6.283185307179586f) / 3.0f);
}

float ball_source(const Problem& pb, V x, float R, uint64_t w, int step, uint32_t u2, uint32_t k0, uint32_t k1) {
  float f;
  if (pb.source_sampling == 1) {
    // centre rule (include/n2wos/nc_poisson_manufactured.hpp:151-157)
    f = f_value(pb, x);
  } else {
    const U4 r2 = philox(U4{static_cast<uint32_t>(w), static_cast<uint32_t>(w >> 32), static_cast<uint32_t>(step), 1u},
                         k0, k1);
    const float rho = R * green_fraction(u2);
    const V d = sphere_dir(r2.x, r2.y);
    f = f_value(pb, {x.x + rho * d.x, x.y + rho * d.y, x.z + rho * d.z});
    const int K = pb.source_samples > 1 ? pb.source_samples : 1;
    for (int k = 1; k < K; ++k) {
      const U4 rk = philox(U4{static_cast<uint32_t>(w), static_cast<uint32_t>(w >> 32), static_cast<uint32_t>(step),
                              1u + static_cast<uint32_t>(k)},
                           k0, k1);
      const float rk_rho = R * green_fraction(rk.x);
      const V dk = sphere_dir(rk.y, rk.z);
      f += f_value(pb, {x.x + rk_rho * dk.x, x.y + rk_rho * dk.y, x.z + rk_rho * dk.z});
    }
    if (K > 1) f *= 1.0f / static_cast<float>(K);
  }
  return R * R * (1.0f / 6.0f) * f;
}

template <class G>
WalkRec walk(const G& geo, const Problem& pb, V x, uint64_t w, uint32_t k0, uint32_t k1, int max_steps, float eps,
             float step_scale, int mode, int depth_m) {
  const bool has_source = pb.mode == 101;
  WalkRec rec{0.0f, 0.0f, x, 0, 0, 0};
  float src = 0.0f;     // source accumulated by the current walk segment
  float prefix = 0.0f;  // residual mode: the prefix source A_m
  int seg_step = 0;     // steps of the current segment (the continuation restarts at 0)
  bool continuing = false;
  V xm = x;
  for (int step = 0;; ++step, ++seg_step) {
    Hit h{FLT_MAX, INT32_MAX, x, 0, 0, 0};
    geo.query(x, h);
    const float d = std::sqrt(std::fmax(h.d2, 0.0f));
    bool forced = seg_step >= max_steps;
    bool stop = d <= eps || forced || !std::isfinite(d);
    if (!stop && mode == kModeResidual && !continuing && step >= depth_m) {
      // X_m reached: the continuation is nc_wos_from_point(X_m) with its own
      // source sum and step budget; its first query is this one.
      continuing = true;
      prefix = src;
      src = 0.0f;
      xm = x;
      seg_step = 0;
      forced = seg_step >= max_steps;
      stop = forced;
    }
    if (stop) {
      const float gb = g_value(pb, h.cp);
      rec.steps = step;
      rec.forced = forced ? 1 : 0;
      if (continuing) {
        rec.value = prefix;   // boundary_values = A_m
        rec.cont = src + gb;  // continuation_values
        rec.xo = xm;
        rec.needs = 1;
      } else {
        rec.value = src + gb;
        rec.cont = src + gb;
        rec.xo = x;
        rec.needs = 0;
      }
      return rec;
    }
    if (mode == kModePrefix && step >= depth_m) {
      rec.value = src;
      rec.xo = x;
      rec.needs = 1;
      rec.steps = step;
      return rec;
    }
    const float R = step_scale * d;
    const U4 r = philox(U4{static_cast<uint32_t>(w), static_cast<uint32_t>(w >> 32), static_cast<uint32_t>(step), 0u},
                        k0, k1);
    const V dir = sphere_dir(r.x, r.y);
    if (has_source) src += ball_source(pb, x, R, w, step, r.z, k0, k1);
    x = {x.x + R * dir.x, x.y + R * dir.y, x.z + R * dir.z};
  }
}

// nc_map_to_unit (src/cuda/cubql_bvh.cu:1311-1315).
inline float clamp01(float v) { return std::fmin(1.0f, std::fmax(0.0f, v)); }
inline void map_to_unit(V p, const float* in_min, const float* in_ext, float* out) {
  out[0] = clamp01((p.x - in_min[0]) / std::fmax(in_ext[0], 1.0e-6f));
  out[1] = clamp01((p.y - in_min[1]) / std::fmax(in_ext[1], 1.0e-6f));
  out[2] = clamp01((p.z - in_min[2]) / std::fmax(in_ext[2], 1.0e-6f));
}

template <class G>
void wos_points(const G& geo, const Problem& pb, const float* points, int64_t n, int W, int max_steps, float eps,
                float step_scale, uint32_t k0, uint32_t k1, double* out_sum, double* out_sum_sq, double* out_steps,
                int threads) {
  parallel_for(n, threads, [&](int64_t i) {
    double s = 0.0, s2 = 0.0, st = 0.0;
    for (int j = 0; j < W; ++j) {
      const uint64_t w = static_cast<uint64_t>(i) * static_cast<uint64_t>(W) + static_cast<uint64_t>(j);
      const WalkRec r = walk(geo, pb, {points[3 * i], points[3 * i + 1], points[3 * i + 2]}, w, k0, k1, max_steps,
                             eps, step_scale, kModePure, 0);
      s += r.value;
      s2 += static_cast<double>(r.value) * r.value;
      st += r.steps;
    }
    out_sum[i] = s;
    out_sum_sq[i] = s2;
    out_steps[i] = st;
  });
}

// ---- procedural meshes ----
uint64_t splitmix_next(uint64_t& state) {
  uint64_t z = (state += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
double splitmix_unit(uint64_t& state) { return static_cast<double>(splitmix_next(state) >> 11) * (1.0 / 9007199254740992.0); }

// Seeded value noise: lattice values in [-1, 1] hashed from the integer
// coordinates, trilinear with the quintic fade, octaves normalised by the total
// amplitude (the displaced-icosphere surface of the Poisson slice workload).
double lattice(int64_t ix, int64_t iy, int64_t iz, uint64_t seed) {
  uint64_t s = seed ^ (static_cast<uint64_t>(ix) * 0x9E3779B97F4A7C15ull) ^
               (static_cast<uint64_t>(iy) * 0xC2B2AE3D27D4EB4Full) ^ (static_cast<uint64_t>(iz) * 0x165667B19E3779F9ull);
  return 2.0 * splitmix_unit(s) - 1.0;
}
double quintic(double t) { return t * t * t * (t * (t * 6.0 - 15.0) + 10.0); }
double noise3(double x, double y, double z, uint64_t seed) {
  const double fx = std::floor(x), fy = std::floor(y), fz = std::floor(z);
  const int64_t ix = static_cast<int64_t>(fx), iy = static_cast<int64_t>(fy), iz = static_cast<int64_t>(fz);
  const double tx = quintic(x - fx), ty = quintic(y - fy), tz = quintic(z - fz);
  double c[2][2][2];
  for (int a = 0; a < 2; ++a)
    for (int b = 0; b < 2; ++b)
      for (int d = 0; d < 2; ++d) c[a][b][d] = lattice(ix + a, iy + b, iz + d, seed);
  const double x00 = c[0][0][0] + tx * (c[1][0][0] - c[0][0][0]);
  const double x10 = c[0][1][0] + tx * (c[1][1][0] - c[0][1][0]);
  const double x01 = c[0][0][1] + tx * (c[1][0][1] - c[0][0][1]);
  const double x11 = c[0][1][1] + tx * (c[1][1][1] - c[0][1][1]);
  const double y0 = x00 + ty * (x10 - x00);
  const double y1 = x01 + ty * (x11 - x01);
  return y0 + tz * (y1 - y0);
}
double fractal(double x, double y, double z, double freq, int octaves, double persistence, uint64_t seed) {
  double sum = 0.0, norm = 0.0, amp = 1.0;
  for (int o = 0; o < octaves; ++o) {
    uint64_t os = seed + 0x632BE59BD9B4E019ull * static_cast<uint64_t>(o + 1);
    sum += amp * noise3(x * freq, y * freq, z * freq, splitmix_next(os));
    norm += amp;
    amp *= persistence;
    freq *= 2.0;
  }
  return norm > 0.0 ? sum / norm : 0.0;
}

struct IcoMesh {
  std::vector<std::array<double, 3>> v;
  std::vector<std::array<uint32_t, 3>> f;
};

// Icosahedron subdivided `level` times, midpoints pushed to the unit sphere
// (shared edges keyed by their sorted vertex pair), children (a, ab, ca),
// (b, bc, ab), (c, ca, bc), (ab, bc, ca).
IcoMesh icosphere(int level) {
  const double t = (1.0 + std::sqrt(5.0)) / 2.0;
  IcoMesh m;
  m.v = {{-1, t, 0}, {1, t, 0}, {-1, -t, 0}, {1, -t, 0}, {0, -1, t}, {0, 1, t},
         {0, -1, -t}, {0, 1, -t}, {t, 0, -1}, {t, 0, 1}, {-t, 0, -1}, {-t, 0, 1}};
  for (auto& p : m.v) {
    const double n = std::sqrt(p[0] * p[0] + p[1] * p[1] + p[2] * p[2]);
    for (double& c : p) c /= n;
  }
  m.f = {{0, 11, 5}, {0, 5, 1},  {0, 1, 7},   {0, 7, 10}, {0, 10, 11}, {1, 5, 9},  {5, 11, 4},
         {11, 10, 2}, {10, 7, 6}, {7, 1, 8},  {3, 9, 4},  {3, 4, 2},   {3, 2, 6},  {3, 6, 8},
         {3, 8, 9},  {4, 9, 5},  {2, 4, 11}, {6, 2, 10}, {8, 6, 7},   {9, 8, 1}};
  for (int l = 0; l < level; ++l) {
    std::map<std::pair<uint32_t, uint32_t>, uint32_t> mid;
    auto midpoint = [&](uint32_t a, uint32_t b) {
      const auto key = std::make_pair(std::min(a, b), std::max(a, b));
      const auto it = mid.find(key);
      if (it != mid.end()) return it->second;
      std::array<double, 3> p{(m.v[a][0] + m.v[b][0]) * 0.5, (m.v[a][1] + m.v[b][1]) * 0.5,
                              (m.v[a][2] + m.v[b][2]) * 0.5};
      const double n = std::sqrt(p[0] * p[0] + p[1] * p[1] + p[2] * p[2]);
      for (double& c : p) c /= n;
      m.v.push_back(p);
      const uint32_t id = static_cast<uint32_t>(m.v.size() - 1);
      mid.emplace(key, id);
      return id;
    };
    std::vector<std::array<uint32_t, 3>> nf;
    nf.reserve(m.f.size() * 4);
    for (const auto& tri : m.f) {
      const uint32_t ab = midpoint(tri[0], tri[1]), bc = midpoint(tri[1], tri[2]), ca = midpoint(tri[2], tri[0]);
      nf.push_back({tri[0], ab, ca});
      nf.push_back({tri[1], bc, ab});
      nf.push_back({tri[2], ca, bc});
      nf.push_back({ab, bc, ca});
    }
    m.f.swap(nf);
  }
  return m;
}

}  // namespace

extern "C" {

// Scalar WoS: W walks from each of n points over the product's 4-wide layout
// (restated traversal, identical to brute force).  Per-point FP64 sums and
// total steps.  Walk (point i, walk j) uses Philox key (k0, k1) and walk id
// w = i*W + j.
void oracle_wos(const void* nodes, const void* tris, const void* problem, const float* points, int64_t n, int W,
                int max_steps, float eps, float step_scale, uint32_t k0, uint32_t k1, double* out_sum,
                double* out_sum_sq, double* out_steps, int threads) {
  const Bvh4 geo{static_cast<const Node4*>(nodes), static_cast<const TriRec*>(tris)};
  wos_points(geo, *static_cast<const Problem*>(problem), points, n, W, max_steps, eps, step_scale, k0, k1, out_sum,
             out_sum_sq, out_steps, threads);
}

// The same walk over the reference's own host BVH (bvh_build_host.cpp output:
// 40-byte nodes, 36-byte triangles, triangle index list), traversed as
// closest_point_bvh_kernel does: the reference path's CPU form.
void oracle_wos_ref_bvh(const void* ref_nodes, const void* ref_tris, const int32_t* ref_idx, const void* problem,
                        const float* points, int64_t n, int W, int max_steps, float eps, float step_scale, uint32_t k0,
                        uint32_t k1, double* out_sum, double* out_sum_sq, double* out_steps, int threads) {
  const RefBvh geo{static_cast<const RefNode*>(ref_nodes), static_cast<const RefTri*>(ref_tris), ref_idx};
  wos_points(geo, *static_cast<const Problem*>(problem), points, n, W, max_steps, eps, step_scale, k0, k1, out_sum,
             out_sum_sq, out_steps, threads);
}

// Closest point over the reference's host BVH (restated bvh_query.cu:75-160);
// node visits and triangle tests per query.
void oracle_ref_bvh_query(const void* ref_nodes, const void* ref_tris, const int32_t* ref_idx, const float* points,
                          int64_t n, float* out_d2, float* out_cp, int32_t* out_id, int32_t* out_nodes,
                          int32_t* out_tris, int threads) {
  const RefBvh geo{static_cast<const RefNode*>(ref_nodes), static_cast<const RefTri*>(ref_tris), ref_idx};
  parallel_for(n, threads, [&](int64_t q) {
    Hit h{FLT_MAX, -1, {0.0f, 0.0f, 0.0f}, 0, 0, 0};
    geo.query({points[3 * q], points[3 * q + 1], points[3 * q + 2]}, h);
    out_d2[q] = h.d2;
    out_cp[3 * q] = h.cp.x;
    out_cp[3 * q + 1] = h.cp.y;
    out_cp[3 * q + 2] = h.cp.z;
    out_id[q] = h.id;
    if (out_nodes) out_nodes[q] = h.nodes;
    if (out_tris) out_tris[q] = h.tris;
  });
}

// Reference slice mask (point_inside_closed_mesh_ray_x, cubql_bvh.cu:446-455)
// with the reference BVH's boxes as a cull: a node whose box the +x ray from p
// misses (p.y or p.z outside it, or p.x beyond its max x) holds no triangle the
// per-triangle test could count, so the hit count equals the brute force one.
void oracle_inside_ref_bvh(const void* ref_nodes, const void* ref_tris, const int32_t* ref_idx, const float* points,
                           int64_t n, uint8_t* out_inside, int threads) {
  const RefNode* nodes = static_cast<const RefNode*>(ref_nodes);
  const RefTri* tris = static_cast<const RefTri*>(ref_tris);
  parallel_for(n, threads, [&](int64_t q) {
    const V p{points[3 * q], points[3 * q + 1] + 1.928371e-6f, points[3 * q + 2] + 3.141593e-6f};
    std::vector<int> stack{0};
    int hits = 0;
    while (!stack.empty()) {
      const RefNode& nd = nodes[stack.back()];
      stack.pop_back();
      if (p.y < nd.lo.y || p.y > nd.hi.y || p.z < nd.lo.z || p.z > nd.hi.z || p.x > nd.hi.x) continue;
      if (nd.count > 0) {
        for (int i = 0; i < nd.count; ++i) {
          const RefTri& t = tris[ref_idx[nd.first + i]];
          if (ray_x_hits(p, rv(t.v0), rv(t.v1), rv(t.v2))) ++hits;
        }
      } else {
        if (nd.left >= 0) stack.push_back(nd.left);
        if (nd.right >= 0) stack.push_back(nd.right);
      }
    }
    out_inside[q] = (hits & 1) ? 1 : 0;
  });
}

// Per-sample walks over the product's 4-wide layout, restating
//   mode 0: nc_pure_wos_samples_kernel      (cubql_bvh.cu:1422-1449)
//   mode 1: nc_hybrid_prefix_kernel         (cubql_bvh.cu:1451-1516)
//   mode 2: nc_2lmc_prefix_continue_kernel  (cubql_bvh.cu:1519-1606)
// Sample s = i*W + j.  Outputs (any may be NULL): value (pure value, or
// boundary_values), continuation values (mode 2), prefix inputs (3 per sample,
// unit cube), needs_cache, step_count, forced_max_steps.
void oracle_walk_samples(const void* nodes, const void* tris, const void* problem, const float* points, int64_t n,
                         int W, int mode, int depth_m, int max_steps, float eps, float step_scale, uint32_t k0,
                         uint32_t k1, const float* in_min, const float* in_ext, float* out_value, float* out_cont,
                         float* out_inputs, uint8_t* out_needs, int32_t* out_steps, int32_t* out_forced,
                         int threads) {
  const Bvh4 geo{static_cast<const Node4*>(nodes), static_cast<const TriRec*>(tris)};
  const Problem& pb = *static_cast<const Problem*>(problem);
  parallel_for(n, threads, [&](int64_t i) {
    for (int j = 0; j < W; ++j) {
      const uint64_t s = static_cast<uint64_t>(i) * static_cast<uint64_t>(W) + static_cast<uint64_t>(j);
      const WalkRec r = walk(geo, pb, {points[3 * i], points[3 * i + 1], points[3 * i + 2]}, s, k0, k1, max_steps, eps,
                             step_scale, mode, depth_m);
      if (out_value) out_value[s] = r.value;
      if (out_cont) out_cont[s] = r.cont;
      if (out_inputs && in_min && in_ext) map_to_unit(r.xo, in_min, in_ext, out_inputs + 3 * s);
      if (out_needs) out_needs[s] = static_cast<uint8_t>(r.needs);
      if (out_steps) out_steps[s] = r.steps;
      if (out_forced) out_forced[s] = r.forced;
    }
  });
}

// nc_combine_cache_and_residual_kernel (cubql_bvh.cu:1608-1627).
void oracle_nc_combine(const float* cache_out, const float* boundary, const float* cont, const uint8_t* needs,
                       int64_t n, float* nc_out, float* residual_out) {
  for (int64_t s = 0; s < n; ++s) {
    if (needs[s]) {
      nc_out[s] = boundary[s] + cache_out[s];
      residual_out[s] = cont[s] - cache_out[s];
    } else {
      nc_out[s] = boundary[s];
      residual_out[s] = 0.0f;
    }
  }
}

// nc_update_labels_kernel (cubql_bvh.cu:1372-1420): inputs = the point mapped
// to the unit cube; label y = g(p) (label_source 0, exact) or the mean of W
// walks (label_source 1); running float average
// targets = (targets*count + y*add) / (count + add), count += add.
// Walk j of point i uses walk id i*W + j under key (k0, k1).
void oracle_nc_update_labels(const void* nodes, const void* tris, const void* problem, const float* points, int64_t n,
                             int W, int max_steps, float eps, float step_scale, uint32_t k0, uint32_t k1,
                             int label_source, const float* in_min, const float* in_ext, float* inputs,
                             float* targets, int32_t* counts, int threads) {
  const Bvh4 geo{static_cast<const Node4*>(nodes), static_cast<const TriRec*>(tris)};
  const Problem& pb = *static_cast<const Problem*>(problem);
  parallel_for(n, threads, [&](int64_t i) {
    const V p0{points[3 * i], points[3 * i + 1], points[3 * i + 2]};
    map_to_unit(p0, in_min, in_ext, inputs + 3 * i);
    float y = 0.0f;
    int add = 1;
    if (label_source == 0) {
      y = g_value(pb, p0);
    } else {
      const int walks = W > 1 ? W : 1;
      add = walks;
      float sum = 0.0f;
      for (int j = 0; j < walks; ++j) {
        const uint64_t w = static_cast<uint64_t>(i) * static_cast<uint64_t>(walks) + static_cast<uint64_t>(j);
        sum += walk(geo, pb, p0, w, k0, k1, max_steps, eps, step_scale, kModePure, 0).value;
      }
      y = sum / static_cast<float>(walks);
    }
    const int old_count = std::max(0, counts[i]);
    const int new_count = old_count + add;
    const float old_total = targets[i] * static_cast<float>(old_count);
    targets[i] = (old_total + y * static_cast<float>(add)) / static_cast<float>(new_count);
    counts[i] = new_count;
  });
}

// Displaced icosphere: subdivision `level`, each unit-sphere vertex moved to
// radius 1 + amplitude * fractal value noise (base frequency, octaves,
// persistence, seed).  Call with null outputs for the counts.
void oracle_icosphere_displaced(int level, float amplitude, float base_frequency, int octaves, float persistence,
                                uint64_t seed, int64_t* nv, int64_t* nt, float* out_v, uint32_t* out_t) {
  const IcoMesh m = icosphere(level);
  *nv = static_cast<int64_t>(m.v.size());
  *nt = static_cast<int64_t>(m.f.size());
  if (!out_v || !out_t) return;
  for (size_t i = 0; i < m.v.size(); ++i) {
    // the unit-sphere vertex is stored as float first, then displaced
    const double x = static_cast<float>(m.v[i][0]), y = static_cast<float>(m.v[i][1]),
                 z = static_cast<float>(m.v[i][2]);
    const double r = 1.0 + static_cast<double>(amplitude) *
                               fractal(x, y, z, base_frequency, octaves, persistence, seed);
    out_v[3 * i] = static_cast<float>(x * r);
    out_v[3 * i + 1] = static_cast<float>(y * r);
    out_v[3 * i + 2] = static_cast<float>(z * r);
  }
  for (size_t i = 0; i < m.f.size(); ++i) {
    for (int k = 0; k < 3; ++k) out_t[3 * i + k] = m.f[i][k];
  }
}

// Slice grid of the evaluation / render tools: frame = bounds of the view's
// axes padded by `padding` of their extent, widened to the image aspect when
// preserve_aspect (reference cubql_bvh.cu:90-112, 974-995); pixel (ix, iy) at
// u_min + du * (ix / (W-1)) (render rule 0) or u_min + du * ix / (W-1)
// (evaluation rule 1).  points_out: W*H*3 floats, row-major from v_min.
int oracle_slice_points(const float* b, int view, float plane, int width, int height, float padding,
                        int preserve_aspect, int rule, float* points_out, float* frame_out) {
  int ua, va, fa;
  if (view == 0) { ua = 0; va = 1; fa = 2; }
  else if (view == 1) { ua = 0; va = 2; fa = 1; }
  else if (view == 2) { ua = 1; va = 2; fa = 0; }
  else return 1;
  const float du0 = b[3 + ua] - b[ua], dv0 = b[3 + va] - b[va];
  float u_min = b[ua] - padding * du0, u_max = b[3 + ua] + padding * du0;
  float v_min = b[va] - padding * dv0, v_max = b[3 + va] + padding * dv0;
  if (preserve_aspect) {
    const float du = u_max - u_min, dv = v_max - v_min;
    if (du > 0.0f && dv > 0.0f) {
      const float image_aspect = static_cast<float>(width) / static_cast<float>(height);
      const float frame_aspect = du / dv;
      if (frame_aspect < image_aspect) {
        const float nd = image_aspect * dv, c = 0.5f * (u_min + u_max);
        u_min = c - 0.5f * nd;
        u_max = c + 0.5f * nd;
      } else if (frame_aspect > image_aspect) {
        const float nd = du / image_aspect, c = 0.5f * (v_min + v_max);
        v_min = c - 0.5f * nd;
        v_max = c + 0.5f * nd;
      }
    }
  }
  if (frame_out) {
    frame_out[0] = u_min;
    frame_out[1] = u_max;
    frame_out[2] = v_min;
    frame_out[3] = v_max;
  }
  for (int iy = 0; iy < height; ++iy) {
    const float fy = static_cast<float>(iy), ny = static_cast<float>(height - 1);
    const float pv = height == 1 ? 0.5f * (v_min + v_max)
                     : rule == 0 ? v_min + (v_max - v_min) * (fy / ny)
                                 : v_min + (v_max - v_min) * fy / ny;
    for (int ix = 0; ix < width; ++ix) {
      const float fx = static_cast<float>(ix), nx = static_cast<float>(width - 1);
      const float pu = width == 1 ? 0.5f * (u_min + u_max)
                       : rule == 0 ? u_min + (u_max - u_min) * (fx / nx)
                                   : u_min + (u_max - u_min) * fx / nx;
      float* o = points_out + 3 * (static_cast<size_t>(iy) * width + ix);
      o[ua] = pu;
      o[va] = pv;
      o[fa] = plane;
    }
  }
  return 0;
}

}  // extern "C"
