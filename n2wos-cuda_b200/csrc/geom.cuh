// Exact point-triangle closest point and the 4-wide BVH traversal (device).
//
// The triangle routine restates Ericson, Real-Time Collision Detection §5.1.5,
// in the operation order of the reference CPU oracle
// (src/geometry/closest_point.cpp:7-48, device twin src/cuda/bvh_query.cu:33-73).
// Every arithmetic step uses a round-to-nearest intrinsic (__fadd_rn etc.), which
// the compiler never fuses into an FMA, so results are bit-identical to the
// reference's g++ build of the same expressions.  The box distance uses the
// same non-fused operations, which keeps it a rounding-monotone lower bound of
// every contained triangle's computed distance: pruning with `box_d2 > best_d2`
// therefore never drops a triangle whose distance ties the current best, and the
// (d2, id) tie-break returns the lowest triangle id among exact ties — the
// answer of the reference brute force, which keeps the first minimum in index
// order (closest_point.cpp:57-65).
#pragma once

#include <float.h>
#include <stdint.h>

#include "layout.h"

namespace n2w {
namespace dev {

struct V3 {
  float x, y, z;
};

__device__ __forceinline__ float fa(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float fs(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float fm(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float fd(float a, float b) { return __fdiv_rn(a, b); }

__device__ __forceinline__ V3 v3(float x, float y, float z) { return V3{x, y, z}; }
__device__ __forceinline__ V3 vsub(V3 a, V3 b) { return V3{fs(a.x, b.x), fs(a.y, b.y), fs(a.z, b.z)}; }
__device__ __forceinline__ V3 vadd(V3 a, V3 b) { return V3{fa(a.x, b.x), fa(a.y, b.y), fa(a.z, b.z)}; }
__device__ __forceinline__ V3 vscale(V3 a, float s) { return V3{fm(a.x, s), fm(a.y, s), fm(a.z, s)}; }
__device__ __forceinline__ float vdot(V3 a, V3 b) { return fa(fa(fm(a.x, b.x), fm(a.y, b.y)), fm(a.z, b.z)); }

// Ericson closest point on triangle abc to p, reference operation order.
// Branch-free form for SIMT: all six dot products and the three barycentric
// numerators are computed, the Voronoi region is chosen with Ericson's tests in
// his order, and only the chosen region's expression is evaluated (one IEEE
// division); each region's result uses exactly the reference's operations:
//   edge ab: a + ab*(d1/(d1-d3))           edge ac: a + ac*(d2/(d2-d6))
//   edge bc: b + (c-b)*((d4-d3)/((d4-d3)+(d5-d6)))
//   face:    (a + ab*(vb*r)) + ac*(vc*r),  r = 1/((va+vb)+vc)
//   vertex regions return the vertex itself.
__device__ __forceinline__ V3 closest_point_triangle(V3 p, V3 a, V3 b, V3 c) {
  const V3 ab = vsub(b, a);
  const V3 ac = vsub(c, a);
  const V3 ap = vsub(p, a);
  const float d1 = vdot(ab, ap);
  const float d2 = vdot(ac, ap);
  const V3 bp = vsub(p, b);
  const float d3 = vdot(ab, bp);
  const float d4 = vdot(ac, bp);
  const V3 cq = vsub(p, c);
  const float d5 = vdot(ab, cq);
  const float d6 = vdot(ac, cq);
  const float vc = fs(fm(d1, d4), fm(d3, d2));
  const float vb = fs(fm(d5, d2), fm(d1, d6));
  const float va = fs(fm(d3, d6), fm(d5, d4));
  const float d43 = fs(d4, d3);
  const float d56 = fs(d5, d6);

  const bool rA = d1 <= 0.0f && d2 <= 0.0f;
  const bool rB = !rA && d3 >= 0.0f && d4 <= d3;
  const bool rAB = !rA && !rB && vc <= 0.0f && d1 >= 0.0f && d3 <= 0.0f;
  const bool r3 = rA || rB || rAB;
  const bool rC = !r3 && d6 >= 0.0f && d5 <= d6;
  const bool rAC = !r3 && !rC && vb <= 0.0f && d2 >= 0.0f && d6 <= 0.0f;
  const bool rBC = !r3 && !rC && !rAC && va <= 0.0f && d43 >= 0.0f && d56 >= 0.0f;
  const bool rF = !r3 && !rC && !rAC && !rBC;

  float num = 0.0f, den = 1.0f;
  if (rAB) { num = d1; den = fs(d1, d3); }
  if (rAC) { num = d2; den = fs(d2, d6); }
  if (rBC) { num = d43; den = fa(d43, d56); }
  if (rF) { num = 1.0f; den = fa(fa(va, vb), vc); }
  const float q = fd(num, den);
  const float s = rF ? fm(vb, q) : q;
  const V3 base = rBC ? b : a;
  const V3 e1 = rBC ? vsub(c, b) : (rAC ? ac : ab);
  V3 r = vadd(base, vscale(e1, s));
  if (rF) r = vadd(r, vscale(ac, fm(vc, q)));
  if (rA) r = a;
  if (rB) r = b;
  if (rC) r = c;
  return r;
}

// Signed gap from p to [lo, hi] along one axis: p - clamp(p, lo, hi).  Its
// square equals that of max(lo - p, p - hi, 0) bit for bit (IEEE subtraction
// is sign-symmetric), with one subtraction instead of two; empty slots
// (lo = +inf, hi = -inf) give an infinite gap.
__device__ __forceinline__ float axis_gap(float p, float lo, float hi) {
  return fs(p, fminf(fmaxf(p, lo), hi));
}

__device__ __forceinline__ float box_d2(V3 p, float lox, float hix, float loy, float hiy, float loz,
                                        float hiz) {
  const float dx = axis_gap(p.x, lox, hix);
  const float dy = axis_gap(p.y, loy, hiy);
  const float dz = axis_gap(p.z, loz, hiz);
  return fa(fa(fm(dx, dx), fm(dy, dy)), fm(dz, dz));
}

// ---- contracted-FP32 variants for the walker -------------------------------
// A walk only needs each step's distance (and the closest point at the
// terminal step) to FP32 accuracy: the reference's GPU walker is compiled
// with FMA contraction and IEEE division, and its parity with any CPU
// evaluation is statistical.  These variants evaluate the same Ericson region
// tests with fused multiply-adds and the fast division intrinsic, cutting the
// instruction count of a triangle test by about a quarter.  Results differ
// from the exact routine above by a few ulps, so the walker's queries are not
// bit-identical to n2w_bvh_query_device's; the query API keeps the exact path.
__device__ __forceinline__ float vdot_fast(V3 a, V3 b) { return fmaf(a.z, b.z, fmaf(a.y, b.y, a.x * b.x)); }
__device__ __forceinline__ V3 vsub_fast(V3 a, V3 b) { return V3{a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ V3 vmad_fast(V3 e, float s, V3 base) {
  return V3{fmaf(e.x, s, base.x), fmaf(e.y, s, base.y), fmaf(e.z, s, base.z)};
}

__device__ __forceinline__ V3 closest_point_triangle_fast(V3 p, V3 a, V3 b, V3 c) {
  const V3 ab = vsub_fast(b, a);
  const V3 ac = vsub_fast(c, a);
  const V3 ap = vsub_fast(p, a);
  const float d1 = vdot_fast(ab, ap);
  const float d2 = vdot_fast(ac, ap);
  const V3 bp = vsub_fast(p, b);
  const float d3 = vdot_fast(ab, bp);
  const float d4 = vdot_fast(ac, bp);
  const V3 cq = vsub_fast(p, c);
  const float d5 = vdot_fast(ab, cq);
  const float d6 = vdot_fast(ac, cq);
  const float vc = fmaf(d1, d4, -(d3 * d2));
  const float vb = fmaf(d5, d2, -(d1 * d6));
  const float va = fmaf(d3, d6, -(d5 * d4));
  const float d43 = d4 - d3;
  const float d56 = d5 - d6;

  const bool rA = d1 <= 0.0f && d2 <= 0.0f;
  const bool rB = !rA && d3 >= 0.0f && d4 <= d3;
  const bool rAB = !rA && !rB && vc <= 0.0f && d1 >= 0.0f && d3 <= 0.0f;
  const bool r3 = rA || rB || rAB;
  const bool rC = !r3 && d6 >= 0.0f && d5 <= d6;
  const bool rAC = !r3 && !rC && vb <= 0.0f && d2 >= 0.0f && d6 <= 0.0f;
  const bool rBC = !r3 && !rC && !rAC && va <= 0.0f && d43 >= 0.0f && d56 >= 0.0f;
  const bool rF = !r3 && !rC && !rAC && !rBC;

  float num = 0.0f, den = 1.0f;
  if (rAB) { num = d1; den = d1 - d3; }
  if (rAC) { num = d2; den = d2 - d6; }
  if (rBC) { num = d43; den = d43 + d56; }
  if (rF) { num = 1.0f; den = (va + vb) + vc; }
  const float q = __fdividef(num, den);
  const float s = rF ? vb * q : q;
  const V3 base = rBC ? b : a;
  const V3 e1 = rBC ? vsub_fast(c, b) : (rAC ? ac : ab);
  V3 r = vmad_fast(e1, s, base);
  if (rF) r = vmad_fast(ac, vc * q, r);
  if (rA) r = a;
  if (rB) r = b;
  if (rC) r = c;
  return r;
}

__device__ __forceinline__ float box_d2_fast(V3 p, float lox, float hix, float loy, float hiy, float loz,
                                             float hiz) {
  const float dx = p.x - fminf(fmaxf(p.x, lox), hix);
  const float dy = p.y - fminf(fmaxf(p.y, loy), hiy);
  const float dz = p.z - fminf(fmaxf(p.z, loz), hiz);
  return fmaf(dz, dz, fmaf(dy, dy, dx * dx));
}

__device__ __forceinline__ void cswap(float& da, int& ra, float& db, int& rb) {
  if (db < da) {
    const float td = da;
    da = db;
    db = td;
    const int tr = ra;
    ra = rb;
    rb = tr;
  }
}

// One 4-wide node (layout.h Node4: lo_x, hi_x, lo_y, hi_y, lo_z, hi_z float4,
// then the child refs) in four 256-bit read-only loads (ld.global.nc.v8,
// sm_100) instead of seven 128-bit ones: a warp's divergent gathers touch
// the same sectors with fewer L1 wavefronts.  Node arrays are cudaMalloc'd
// (256-byte aligned) and nodes are 128 bytes, so every load is 32-byte
// aligned.  The last load also brings the node's 16 pad bytes (same sector).
__device__ __forceinline__ void ldg_v8f(const float4* p, float4& a, float4& b) {
  asm("ld.global.nc.v8.f32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
      : "=f"(a.x), "=f"(a.y), "=f"(a.z), "=f"(a.w), "=f"(b.x), "=f"(b.y), "=f"(b.z), "=f"(b.w)
      : "l"(p));
}
__device__ __forceinline__ int4 ldg_v8_first_int4(const float4* p) {
  int4 a;
  int d0, d1, d2, d3;
  asm("ld.global.nc.v8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
      : "=r"(a.x), "=r"(a.y), "=r"(a.z), "=r"(a.w), "=r"(d0), "=r"(d1), "=r"(d2), "=r"(d3)
      : "l"(p));
  return a;
}
__device__ __forceinline__ void load_node(const float4* __restrict__ nodes, int32_t ref, float4& lox, float4& hix,
                                          float4& loy, float4& hiy, float4& loz, float4& hiz, int4& ch) {
  static_assert(sizeof(Node4) == 128, "node loads assume 128-byte nodes");
  const float4* n = nodes + static_cast<size_t>(ref) * 8;
  ldg_v8f(n + 0, lox, hix);
  ldg_v8f(n + 2, loy, hiy);
  ldg_v8f(n + 4, loz, hiz);
  ch = ldg_v8_first_int4(n + 6);
}

struct ClosestHit {
  float d2;
  int id;    // original triangle id; INT32_MAX when nothing was found below the bound
  int slot;  // leaf-order index of that triangle (used to re-seed the next query)
  V3 cp;
};

// Tests one triangle (by leaf-order slot) and keeps it if it beats the hit in
// (d2, id) order.  Seeding a query with real candidates gives the traversal a
// tight bound without changing its answer.  kFast selects the contracted-FP32
// triangle routine (walker); callers use the test_slot / test_slot_fast wrappers.
template <bool kFast>
__device__ __forceinline__ void test_slot_impl(const float4* __restrict__ tris, int slot, V3 p, ClosestHit& hit) {
  // three 128-bit loads: a 256-bit + 128-bit split by record parity measured
  // slower (the selects cost more than the saved load)
  const float4* t = tris + static_cast<size_t>(slot) * 3;
  const float4 a = __ldg(t + 0);
  const float4 b = __ldg(t + 1);
  const float4 c = __ldg(t + 2);
  V3 cp;
  float dd;
  if (kFast) {
    cp = closest_point_triangle_fast(p, v3(a.x, a.y, a.z), v3(b.x, b.y, b.z), v3(c.x, c.y, c.z));
    const V3 dv = vsub_fast(cp, p);
    dd = vdot_fast(dv, dv);
  } else {
    cp = closest_point_triangle(p, v3(a.x, a.y, a.z), v3(b.x, b.y, b.z), v3(c.x, c.y, c.z));
    const V3 dv = vsub(cp, p);
    dd = vdot(dv, dv);
  }
  const int id = __float_as_int(a.w);
  if (dd < hit.d2 || (dd == hit.d2 && id < hit.id)) {
    hit.d2 = dd;
    hit.id = id;
    hit.slot = slot;
    hit.cp = cp;
  }
}

__device__ __forceinline__ void test_slot(const float4* __restrict__ tris, int slot, V3 p, ClosestHit& hit) {
  test_slot_impl<false>(tris, slot, p, hit);
}
__device__ __forceinline__ void test_slot_fast(const float4* __restrict__ tris, int slot, V3 p, ClosestHit& hit) {
  test_slot_impl<true>(tris, slot, p, hit);
}

// Seed grid: (n+1)^3 lattice nodes over a padded mesh box; node value = leaf
// slot of the triangle closest to the node.  The nearest node's triangle is a
// candidate within (node distance + |x - node|) of x.
struct SeedGrid {
  const int* slots;  // nullptr when absent
  float lo_x, lo_y, lo_z;
  float inv_h;
  int n;  // cells per axis
};

__device__ __forceinline__ int seed_slot(const SeedGrid& g, V3 p) {
  const float fx = (p.x - g.lo_x) * g.inv_h, fy = (p.y - g.lo_y) * g.inv_h, fz = (p.z - g.lo_z) * g.inv_h;
  const int ix = __float2int_rn(fminf(fmaxf(fx, 0.0f), static_cast<float>(g.n)));
  const int iy = __float2int_rn(fminf(fmaxf(fy, 0.0f), static_cast<float>(g.n)));
  const int iz = __float2int_rn(fminf(fmaxf(fz, 0.0f), static_cast<float>(g.n)));
  const int s = g.n + 1;
  return __ldg(g.slots + (static_cast<size_t>(iz) * s + iy) * s + ix);
}

struct TraversalStats {
  int node_visits;
  int tri_tests;
  int overflow;
};

// Ordered depth-first traversal: at each inner node the four child boxes are
// measured, sorted ascending (fixed 5-comparator network), the nearest child
// is entered and the others are pushed far-to-near.  Popped entries are
// re-checked against the current best.  Candidates are any triangles whose box
// distance is <= best_d2; `hit` must be initialised by the caller (cold query:
// d2 = FLT_MAX, id = INT32_MAX; warm start: d2 = an upper bound).
template <bool kCount>
__device__ __forceinline__ void traverse(const float4* __restrict__ nodes,
                                         const float4* __restrict__ tris, V3 p, ClosestHit& hit,
                                         TraversalStats& st, int32_t root = 0) {
  int2 stack[kTraversalStack];
  int sp = 0;
  int32_t ref = root;
  for (;;) {
    if (ref >= 0) {
      const float4* n = nodes + static_cast<size_t>(ref) * 8;
      const float4 lox = __ldg(n + 0);
      const float4 hix = __ldg(n + 1);
      const float4 loy = __ldg(n + 2);
      const float4 hiy = __ldg(n + 3);
      const float4 loz = __ldg(n + 4);
      const float4 hiz = __ldg(n + 5);
      const int4 ch = __ldg(reinterpret_cast<const int4*>(n + 6));
      if (kCount) ++st.node_visits;
      float d0 = box_d2(p, lox.x, hix.x, loy.x, hiy.x, loz.x, hiz.x);
      float d1 = box_d2(p, lox.y, hix.y, loy.y, hiy.y, loz.y, hiz.y);
      float d2 = box_d2(p, lox.z, hix.z, loy.z, hiy.z, loz.z, hiz.z);
      float d3 = box_d2(p, lox.w, hix.w, loy.w, hiy.w, loz.w, hiz.w);
      int r0 = ch.x, r1 = ch.y, r2 = ch.z, r3 = ch.w;
      cswap(d0, r0, d1, r1);
      cswap(d2, r2, d3, r3);
      cswap(d0, r0, d2, r2);
      cswap(d1, r1, d3, r3);
      cswap(d1, r1, d2, r2);
      const float best = hit.d2;
      if (d3 <= best) {
        if (sp < kTraversalStack) stack[sp++] = make_int2(r3, __float_as_int(d3));
        else st.overflow = 1;
      }
      if (d2 <= best) {
        if (sp < kTraversalStack) stack[sp++] = make_int2(r2, __float_as_int(d2));
        else st.overflow = 1;
      }
      if (d1 <= best) {
        if (sp < kTraversalStack) stack[sp++] = make_int2(r1, __float_as_int(d1));
        else st.overflow = 1;
      }
      ref = (d0 <= best) ? r0 : kEmptyChild;
    } else if (ref != kEmptyChild) {
      const int first = leaf_first(ref);
      const int count = leaf_count(ref);
      const float4* t = tris + static_cast<size_t>(first) * 3;
      for (int i = 0; i < count; ++i) {
        const float4 a = __ldg(t + 3 * i + 0);
        const float4 b = __ldg(t + 3 * i + 1);
        const float4 c = __ldg(t + 3 * i + 2);
        if (kCount) ++st.tri_tests;
        const V3 cp = closest_point_triangle(p, v3(a.x, a.y, a.z), v3(b.x, b.y, b.z), v3(c.x, c.y, c.z));
        const V3 dv = vsub(cp, p);
        const float dd = vdot(dv, dv);
        const int id = __float_as_int(a.w);
        if (dd < hit.d2 || (dd == hit.d2 && id < hit.id)) {
          hit.d2 = dd;
          hit.id = id;
          hit.slot = first + i;
          hit.cp = cp;
        }
      }
      ref = kEmptyChild;
    }
    if (ref == kEmptyChild) {
      bool found = false;
      while (sp > 0) {
        const int2 e = stack[--sp];
        if (__int_as_float(e.y) <= hit.d2) {
          ref = e.x;
          found = true;
          break;
        }
      }
      if (!found) break;
    }
  }
}

// Traversal stack in the lane's local array (kTraversalStack entries):
// push(sp, e) stores entry sp; pop(sp) returns entry sp (the caller has
// already decremented sp).  (A shared-memory ring holding the top 8 entries
// measured slower: its shared-memory carve-out costs more L1 hits on node
// fetches than it saves on pops.)
struct LocalStack {
  int2* a;
  __device__ __forceinline__ void push(int sp, int2 e) { a[sp] = e; }
  __device__ __forceinline__ int2 pop(int sp) { return a[sp]; }
};

// Per-lane state of one closest-point query in flight.
struct TravState {
  int sp;
  int ref;       // inner node to expand next, or kEmptyChild
  int leaf_cur;  // next triangle slot of the leaf being tested
  int leaf_end;
};

// One unit of traversal work for one lane: test ONE triangle of the current
// leaf, or expand ONE 4-wide node (same ordering and pruning as
// dev::traverse: children sorted by box distance, nearest entered, others
// pushed far-to-near, popped entries re-checked).  Returns false once the
// query is complete.  Splitting the traversal into equal-sized steps is what
// lets lanes with short queries move on while others are still searching.
// kFast selects the contracted-FP32 box and triangle routines (walker);
// callers use the trav_step / trav_step_fast wrappers.
template <bool kFast, class Stack>
__device__ __forceinline__ bool trav_step_impl(const float4* __restrict__ nodes, const float4* __restrict__ tris,
                                          V3 p, ClosestHit& hit, TravState& t, Stack& stack,
                                          uint32_t& c_nodes, uint32_t& c_tris, bool& overflow) {
  if (t.leaf_cur >= t.leaf_end && t.ref == kEmptyChild) {
    bool found = false;
    while (t.sp > 0) {
      const int2 e = stack.pop(--t.sp);
      if (__int_as_float(e.y) <= hit.d2) {
        if (e.x >= 0) {
          t.ref = e.x;
        } else {
          t.leaf_cur = leaf_first(e.x);
          t.leaf_end = t.leaf_cur + leaf_count(e.x);
        }
        found = true;
        break;
      }
    }
    if (!found) return false;
  }
  if (t.leaf_cur < t.leaf_end) {
    test_slot_impl<kFast>(tris, t.leaf_cur, p, hit);
    ++t.leaf_cur;
    ++c_tris;
    return true;
  }
  float4 lox, hix, loy, hiy, loz, hiz;
  int4 ch;
  load_node(nodes, t.ref, lox, hix, loy, hiy, loz, hiz, ch);
  ++c_nodes;
  float d0, d1, d2, d3;
  if (kFast) {
    d0 = box_d2_fast(p, lox.x, hix.x, loy.x, hiy.x, loz.x, hiz.x);
    d1 = box_d2_fast(p, lox.y, hix.y, loy.y, hiy.y, loz.y, hiz.y);
    d2 = box_d2_fast(p, lox.z, hix.z, loy.z, hiy.z, loz.z, hiz.z);
    d3 = box_d2_fast(p, lox.w, hix.w, loy.w, hiy.w, loz.w, hiz.w);
  } else {
    d0 = box_d2(p, lox.x, hix.x, loy.x, hiy.x, loz.x, hiz.x);
    d1 = box_d2(p, lox.y, hix.y, loy.y, hiy.y, loz.y, hiz.y);
    d2 = box_d2(p, lox.z, hix.z, loy.z, hiy.z, loz.z, hiz.z);
    d3 = box_d2(p, lox.w, hix.w, loy.w, hiy.w, loz.w, hiz.w);
  }
  int r0 = ch.x, r1 = ch.y, r2 = ch.z, r3 = ch.w;
  cswap(d0, r0, d1, r1);
  cswap(d2, r2, d3, r3);
  cswap(d0, r0, d2, r2);
  cswap(d1, r1, d3, r3);
  cswap(d1, r1, d2, r2);
  const float best = hit.d2;
  if (d3 <= best) {
    if (t.sp < kTraversalStack) stack.push(t.sp++, make_int2(r3, __float_as_int(d3)));
    else overflow = true;
  }
  if (d2 <= best) {
    if (t.sp < kTraversalStack) stack.push(t.sp++, make_int2(r2, __float_as_int(d2)));
    else overflow = true;
  }
  if (d1 <= best) {
    if (t.sp < kTraversalStack) stack.push(t.sp++, make_int2(r1, __float_as_int(d1)));
    else overflow = true;
  }
  t.ref = kEmptyChild;
  if (d0 <= best) {
    if (r0 >= 0) {
      t.ref = r0;
    } else {
      t.leaf_cur = leaf_first(r0);
      t.leaf_end = t.leaf_cur + leaf_count(r0);
    }
  }
  return true;
}

__device__ __forceinline__ bool trav_step(const float4* __restrict__ nodes, const float4* __restrict__ tris, V3 p,
                                          ClosestHit& hit, TravState& t, LocalStack& stack, uint32_t& c_nodes,
                                          uint32_t& c_tris, bool& overflow) {
  return trav_step_impl<false>(nodes, tris, p, hit, t, stack, c_nodes, c_tris, overflow);
}
__device__ __forceinline__ bool trav_step_fast(const float4* __restrict__ nodes, const float4* __restrict__ tris,
                                               V3 p, ClosestHit& hit, TravState& t, LocalStack& stack,
                                               uint32_t& c_nodes, uint32_t& c_tris, bool& overflow) {
  return trav_step_impl<true>(nodes, tris, p, hit, t, stack, c_nodes, c_tris, overflow);
}

// +x ray / triangle test of the reference's slice mask
// (src/cuda/cubql_bvh.cu:407-428, Möller–Trumbore with its tolerances), in the
// same non-fused float operations, so the parity count matches the CPU test.
__device__ __forceinline__ bool ray_x_hits(V3 p, V3 a, V3 b, V3 c) {
  const float y_min = fminf(fminf(a.y, b.y), c.y), y_max = fmaxf(fmaxf(a.y, b.y), c.y);
  const float z_min = fminf(fminf(a.z, b.z), c.z), z_max = fmaxf(fmaxf(a.z, b.z), c.z);
  const float x_max = fmaxf(fmaxf(a.x, b.x), c.x);
  if (p.y < y_min || p.y > y_max || p.z < z_min || p.z > z_max || p.x > x_max) return false;
  const V3 e1 = vsub(b, a);
  const V3 e2 = vsub(c, a);
  // h = cross((1,0,0), e2)
  const V3 h = v3(fs(fm(0.0f, e2.z), fm(0.0f, e2.y)), fs(fm(0.0f, e2.x), fm(1.0f, e2.z)),
                  fs(fm(1.0f, e2.y), fm(0.0f, e2.x)));
  const float det = vdot(e1, h);
  if (fabsf(det) < 1.0e-12f) return false;
  const float inv_det = fd(1.0f, det);
  const V3 s = vsub(p, a);
  const float u = fm(inv_det, vdot(s, h));
  if (u < -1.0e-7f || u > 1.0f + 1.0e-7f) return false;
  const V3 q = v3(fs(fm(s.y, e1.z), fm(s.z, e1.y)), fs(fm(s.z, e1.x), fm(s.x, e1.z)),
                  fs(fm(s.x, e1.y), fm(s.y, e1.x)));
  const float v = fm(inv_det, vdot(v3(1.0f, 0.0f, 0.0f), q));
  if (v < -1.0e-7f || fa(u, v) > 1.0f + 1.0e-7f) return false;
  const float t = fm(inv_det, vdot(e2, q));
  return t > 1.0e-7f;
}

// Number of mesh triangles crossed by the +x ray from p (every node whose
// child box meets the ray {x >= p.x, y = p.y, z = p.z} is visited).
__device__ __forceinline__ int ray_x_crossings(const float4* __restrict__ nodes, const float4* __restrict__ tris,
                                               V3 p, int& overflow) {
  int stack[kTraversalStack];
  int sp = 0;
  int hits = 0;
  stack[sp++] = 0;
  while (sp > 0) {
    const int ref = stack[--sp];
    if (ref >= 0) {
      const float4* n = nodes + static_cast<size_t>(ref) * 8;
      const float4 hix = __ldg(n + 1), loy = __ldg(n + 2), hiy = __ldg(n + 3), loz = __ldg(n + 4),
                   hiz = __ldg(n + 5);
      const int4 ch = __ldg(reinterpret_cast<const int4*>(n + 6));
      const float hx[4] = {hix.x, hix.y, hix.z, hix.w}, ly[4] = {loy.x, loy.y, loy.z, loy.w},
                  hy[4] = {hiy.x, hiy.y, hiy.z, hiy.w}, lz[4] = {loz.x, loz.y, loz.z, loz.w},
                  hz[4] = {hiz.x, hiz.y, hiz.z, hiz.w};
      const int cr[4] = {ch.x, ch.y, ch.z, ch.w};
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        if (cr[k] == kEmptyChild) continue;
        if (p.y < ly[k] || p.y > hy[k] || p.z < lz[k] || p.z > hz[k] || p.x > hx[k]) continue;
        if (sp < kTraversalStack) stack[sp++] = cr[k];
        else overflow = 1;
      }
    } else {
      const int first = leaf_first(ref), count = leaf_count(ref);
      const float4* t = tris + static_cast<size_t>(first) * 3;
      for (int i = 0; i < count; ++i) {
        const float4 a = __ldg(t + 3 * i), b = __ldg(t + 3 * i + 1), c = __ldg(t + 3 * i + 2);
        if (ray_x_hits(p, v3(a.x, a.y, a.z), v3(b.x, b.y, b.z), v3(c.x, c.y, c.z))) ++hits;
      }
    }
  }
  return hits;
}

}  // namespace dev
}  // namespace n2w
