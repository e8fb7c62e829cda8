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
#include <atomic>
#include <cfloat>
#include <climits>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <thread>
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

// Scalar WoS: W walks from each of n points; closest points by the restated
// traversal (identical to brute force).  Per-point FP64 sums and total steps.
// source_center: 1 = r^2/6 f(centre) (reference rule), 0 = in-ball Green sample.
// Walk (point i, walk j) uses Philox key (k0, k1) and counter (w, w>>32, step, 0|1)
// with w = i*W + j.
void oracle_wos(const void* nodes, const void* tris, const void* problem, const float* points, int64_t n, int W,
                int max_steps, float eps, float step_scale, uint32_t k0, uint32_t k1, double* out_sum,
                double* out_sum_sq, double* out_steps, int threads) {
  const Node4* nd = static_cast<const Node4*>(nodes);
  const TriRec* tr = static_cast<const TriRec*>(tris);
  const Problem& pb = *static_cast<const Problem*>(problem);
  const bool has_source = pb.mode == 101;
  parallel_for(n, threads, [&](int64_t i) {
    double s = 0.0, s2 = 0.0, st = 0.0;
    for (int j = 0; j < W; ++j) {
      const uint64_t w = static_cast<uint64_t>(i) * static_cast<uint64_t>(W) + static_cast<uint64_t>(j);
      V x{points[3 * i], points[3 * i + 1], points[3 * i + 2]};
      float src = 0.0f;
      float value = 0.0f;
      int steps = 0;
      for (int step = 0; step <= max_steps; ++step) {
        Hit h{FLT_MAX, INT32_MAX, x, 0, 0, 0};
        traverse4(nd, tr, x, h);
        const float d = std::sqrt(std::fmax(h.d2, 0.0f));
        if (d <= eps || step >= max_steps || !std::isfinite(d)) {
          value = src + g_value(pb, h.cp);
          steps = step;
          break;
        }
        const float R = step_scale * d;
        const U4 r = philox(U4{static_cast<uint32_t>(w), static_cast<uint32_t>(w >> 32), static_cast<uint32_t>(step), 0u},
                            k0, k1);
        const float z = 1.0f - 2.0f * u01(r.x);
        const float phi = 2.0f * 3.14159265358979323846f * u01(r.y);
        const float rr = std::sqrt(std::fmax(0.0f, 1.0f - z * z));
        const V dir{rr * std::cos(phi), rr * std::sin(phi), z};
        if (has_source) {
          float f;
          if (pb.source_sampling == 1) {
            f = f_value(pb, x);
          } else {
            const float a = std::acos(std::fmin(1.0f, std::fmax(-1.0f, 1.0f - 2.0f * u01(r.z))));
            const float t = 0.5f + std::cos((a - 6.283185307179586f) / 3.0f);
            const U4 r2 = philox(
                U4{static_cast<uint32_t>(w), static_cast<uint32_t>(w >> 32), static_cast<uint32_t>(step), 1u}, k0, k1);
            const float z2 = 1.0f - 2.0f * u01(r2.x);
            const float phi2 = 2.0f * 3.14159265358979323846f * u01(r2.y);
            const float rr2 = std::sqrt(std::fmax(0.0f, 1.0f - z2 * z2));
            const float rho = R * t;
            f = f_value(pb, {x.x + rho * rr2 * std::cos(phi2), x.y + rho * rr2 * std::sin(phi2), x.z + rho * z2});
            const int K = pb.source_samples > 1 ? pb.source_samples : 1;
            for (int k = 1; k < K; ++k) {
              // extra in-ball samples: Philox stream 1 + k (radius, direction)
              const U4 rk = philox(U4{static_cast<uint32_t>(w), static_cast<uint32_t>(w >> 32),
                                      static_cast<uint32_t>(step), 1u + static_cast<uint32_t>(k)},
                                   k0, k1);
              const float ak = std::acos(std::fmin(1.0f, std::fmax(-1.0f, 1.0f - 2.0f * u01(rk.x))));
              const float rhok = R * (0.5f + std::cos((ak - 6.283185307179586f) / 3.0f));
              const float zk = 1.0f - 2.0f * u01(rk.y);
              const float phk = 2.0f * 3.14159265358979323846f * u01(rk.z);
              const float rrk = std::sqrt(std::fmax(0.0f, 1.0f - zk * zk));
              f += f_value(pb, {x.x + rhok * rrk * std::cos(phk), x.y + rhok * rrk * std::sin(phk), x.z + rhok * zk});
            }
            if (K > 1) f *= 1.0f / static_cast<float>(K);
          }
          src += R * R * (1.0f / 6.0f) * f;
        }
        x = {x.x + R * dir.x, x.y + R * dir.y, x.z + R * dir.z};
      }
      s += value;
      s2 += static_cast<double>(value) * value;
      st += steps;
    }
    out_sum[i] = s;
    out_sum_sq[i] = s2;
    out_steps[i] = st;
  });
}

}  // extern "C"
