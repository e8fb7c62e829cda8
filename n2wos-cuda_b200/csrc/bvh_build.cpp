// Host BVH construction: a binary tree built top-down (binned SAH, or the
// reference's largest-centroid-axis median split, src/cuda/bvh_build_host.cpp:74-120),
// collapsed into a 4-wide tree whose nodes are one 128-byte line each, with
// triangles permuted into leaf order (see layout.h).
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <limits>
#include <numeric>

#include "internal.hpp"

namespace n2w {
namespace {

struct Box {
  float lo[3] = {INFINITY, INFINITY, INFINITY};
  float hi[3] = {-INFINITY, -INFINITY, -INFINITY};
  void grow(const float* p) {
    for (int a = 0; a < 3; ++a) {
      lo[a] = std::min(lo[a], p[a]);
      hi[a] = std::max(hi[a], p[a]);
    }
  }
  void grow(const Box& b) {
    for (int a = 0; a < 3; ++a) {
      lo[a] = std::min(lo[a], b.lo[a]);
      hi[a] = std::max(hi[a], b.hi[a]);
    }
  }
  double area() const {
    const double ex = std::max(0.0f, hi[0] - lo[0]), ey = std::max(0.0f, hi[1] - lo[1]),
                 ez = std::max(0.0f, hi[2] - lo[2]);
    return 2.0 * (ex * ey + ey * ez + ez * ex);
  }
};

struct BNode {
  Box box;
  int left = -1, right = -1;  // left < 0 -> leaf
  int first = 0, count = 0;   // leaf range in the primitive order
};

struct Builder {
  const n2w_mesh& mesh;
  int leaf_size;
  bool sah;
  std::vector<Box> prim_box;
  std::vector<std::array<float, 3>> centroid;
  std::vector<int> order;
  std::vector<BNode> nodes;

  Builder(const n2w_mesh& m, int ls, bool use_sah) : mesh(m), leaf_size(ls), sah(use_sah) {
    const size_t n = m.triangles.size();
    prim_box.resize(n);
    centroid.resize(n);
    for (size_t i = 0; i < n; ++i) {
      const auto& t = m.triangles[i];
      const auto& a = m.vertices[t[0]];
      const auto& b = m.vertices[t[1]];
      const auto& c = m.vertices[t[2]];
      prim_box[i].grow(a.data());
      prim_box[i].grow(b.data());
      prim_box[i].grow(c.data());
      for (int k = 0; k < 3; ++k) centroid[i][k] = (a[k] + b[k] + c[k]) / 3.0f;
    }
    order.resize(n);
    std::iota(order.begin(), order.end(), 0);
  }

  int make_leaf(int begin, int end, const Box& box) {
    BNode nd;
    nd.box = box;
    nd.first = begin;
    nd.count = end - begin;
    nodes.push_back(nd);
    return static_cast<int>(nodes.size() - 1);
  }

  // Median split on the largest centroid axis (ties: x, then y, then z).
  int median_split(int begin, int end, const Box& cbox) {
    const float ex = cbox.hi[0] - cbox.lo[0], ey = cbox.hi[1] - cbox.lo[1], ez = cbox.hi[2] - cbox.lo[2];
    const int axis = (ex >= ey && ex >= ez) ? 0 : ((ey >= ex && ey >= ez) ? 1 : 2);
    const int mid = begin + (end - begin) / 2;
    std::nth_element(order.begin() + begin, order.begin() + mid, order.begin() + end,
                     [&](int a, int b) { return centroid[a][axis] < centroid[b][axis]; });
    return mid;
  }

  // Binned SAH (32 bins per axis); returns the split position or -1 when no
  // split beats a leaf and the range already fits in one.
  int sah_split(int begin, int end, const Box& box, const Box& cbox) {
    constexpr int kBins = 32;
    const int n = end - begin;
    double best_cost = std::numeric_limits<double>::infinity();
    int best_axis = -1, best_bin = -1;
    for (int axis = 0; axis < 3; ++axis) {
      const float ext = cbox.hi[axis] - cbox.lo[axis];
      if (!(ext > 0.0f)) continue;
      Box bb[kBins];
      int bc[kBins] = {0};
      const float scale = static_cast<float>(kBins) / ext;
      for (int i = begin; i < end; ++i) {
        const int p = order[i];
        int b = static_cast<int>((centroid[p][axis] - cbox.lo[axis]) * scale);
        b = std::min(kBins - 1, std::max(0, b));
        bb[b].grow(prim_box[p]);
        ++bc[b];
      }
      double right_area[kBins];
      int right_count[kBins];
      Box acc;
      int cnt = 0;
      for (int b = kBins - 1; b > 0; --b) {
        acc.grow(bb[b]);
        cnt += bc[b];
        right_area[b] = acc.area();
        right_count[b] = cnt;
      }
      Box lacc;
      int lcnt = 0;
      for (int b = 1; b < kBins; ++b) {
        lacc.grow(bb[b - 1]);
        lcnt += bc[b - 1];
        if (lcnt == 0 || right_count[b] == 0) continue;
        const double cost = lacc.area() * lcnt + right_area[b] * right_count[b];
        if (cost < best_cost) {
          best_cost = cost;
          best_axis = axis;
          best_bin = b;
        }
      }
    }
    const double parent_area = std::max(box.area(), 1e-30);
    if (best_axis < 0) return median_split(begin, end, cbox);
    const double split_cost = 1.0 + best_cost / parent_area;
    if (n <= leaf_size && split_cost >= static_cast<double>(n)) return -1;
    const float ext = cbox.hi[best_axis] - cbox.lo[best_axis];
    const float scale = static_cast<float>(kBins) / ext;
    auto it = std::partition(order.begin() + begin, order.begin() + end, [&](int p) {
      int b = static_cast<int>((centroid[p][best_axis] - cbox.lo[best_axis]) * scale);
      b = std::min(kBins - 1, std::max(0, b));
      return b < best_bin;
    });
    int mid = static_cast<int>(it - order.begin());
    if (mid == begin || mid == end) mid = median_split(begin, end, cbox);
    return mid;
  }

  int build(int begin, int end) {
    Box box, cbox;
    for (int i = begin; i < end; ++i) {
      box.grow(prim_box[order[i]]);
      cbox.grow(centroid[order[i]].data());
    }
    const int n = end - begin;
    if (n == 1) return make_leaf(begin, end, box);
    int mid;
    if (sah) {
      mid = sah_split(begin, end, box, cbox);
      if (mid < 0) return make_leaf(begin, end, box);
    } else {
      if (n <= leaf_size) return make_leaf(begin, end, box);
      mid = median_split(begin, end, cbox);
    }
    const int self = static_cast<int>(nodes.size());
    nodes.emplace_back();
    nodes[self].box = box;
    const int l = build(begin, mid);
    const int r = build(mid, end);
    nodes[self].left = l;
    nodes[self].right = r;
    return self;
  }

  double sah_cost(int id) const {
    const BNode& nd = nodes[id];
    if (nd.left < 0) return nd.count * nd.box.area();
    return nd.box.area() + sah_cost(nd.left) + sah_cost(nd.right);
  }
};

// Outward pad so that rounding in the closest-point arithmetic can never place
// a computed closest point outside its leaf box (relative 2^-20 >> a few ulps).
void pad_box(const Box& in, float lo[3], float hi[3]) {
  for (int a = 0; a < 3; ++a) {
    const float m = std::max(std::fabs(in.lo[a]), std::fabs(in.hi[a]));
    const float pad = m * 9.5367431640625e-07f + 1e-30f;
    lo[a] = in.lo[a] - pad;
    hi[a] = in.hi[a] + pad;
  }
}

struct Collapser {
  const Builder& b;
  HostBvh& out;

  int emit_leaf(const BNode& leaf) {
    const int first = static_cast<int>(out.tris.size());
    for (int i = 0; i < leaf.count; ++i) {
      const int p = b.order[leaf.first + i];
      const auto& t = b.mesh.triangles[p];
      TriRec r{};
      std::memcpy(r.v0, b.mesh.vertices[t[0]].data(), 12);
      std::memcpy(r.v1, b.mesh.vertices[t[1]].data(), 12);
      std::memcpy(r.v2, b.mesh.vertices[t[2]].data(), 12);
      r.id = p;
      out.tris.push_back(r);
    }
    ++out.leaves;
    return leaf_ref(first, leaf.count);
  }

  // Emits the 4-wide node covering binary node `id` (pre-order); returns its index.
  int emit(int id, int depth) {
    out.max_depth = std::max(out.max_depth, depth);
    int kids[4];
    int nk = 0;
    const BNode& root = b.nodes[id];
    if (root.left < 0) {
      kids[nk++] = id;  // the whole tree is a single leaf
    } else {
      kids[nk++] = root.left;
      kids[nk++] = root.right;
      while (nk < 4) {
        int pick = -1;
        double best = -1.0;
        for (int k = 0; k < nk; ++k) {
          const BNode& c = b.nodes[kids[k]];
          if (c.left >= 0 && c.box.area() > best) {
            best = c.box.area();
            pick = k;
          }
        }
        if (pick < 0) break;
        const BNode& c = b.nodes[kids[pick]];
        kids[pick] = c.left;
        kids[nk++] = c.right;
      }
    }
    const int self = static_cast<int>(out.nodes.size());
    out.nodes.emplace_back();
    Node4 nd{};
    for (int k = 0; k < 4; ++k) {
      if (k < nk) {
        float lo[3], hi[3];
        pad_box(b.nodes[kids[k]].box, lo, hi);
        nd.lo_x[k] = lo[0];
        nd.hi_x[k] = hi[0];
        nd.lo_y[k] = lo[1];
        nd.hi_y[k] = hi[1];
        nd.lo_z[k] = lo[2];
        nd.hi_z[k] = hi[2];
      } else {
        nd.lo_x[k] = nd.lo_y[k] = nd.lo_z[k] = INFINITY;
        nd.hi_x[k] = nd.hi_y[k] = nd.hi_z[k] = -INFINITY;
        nd.child[k] = kEmptyChild;
      }
      nd.pad[k] = 0;
    }
    for (int k = 0; k < nk; ++k) {
      const BNode& c = b.nodes[kids[k]];
      nd.child[k] = (c.left < 0) ? emit_leaf(c) : emit(kids[k], depth + 1);
    }
    out.nodes[self] = nd;
    return self;
  }
};

}  // namespace

HostBvh build_bvh4(const n2w_mesh& mesh, int leaf_size, const std::string& method) {
  N2W_REQUIRE(leaf_size >= 1 && leaf_size <= kMaxLeafSize, "leaf size must be in [1, 8]");
  N2W_REQUIRE(!mesh.triangles.empty(), "cannot build BVH with no triangles");
  N2W_REQUIRE(mesh.triangles.size() < (1u << 27), "mesh too large for the 27-bit leaf encoding");
  bool sah = true;
  if (method == "sah" || method == "binned_sah" || method.empty()) sah = true;
  else if (method == "spatial_median" || method == "median") sah = false;
  else throw Error(N2W_EINVAL, "unknown build method '" + method + "' (expected sah or spatial_median)");
  Builder b(mesh, leaf_size, sah);
  b.nodes.reserve(2 * mesh.triangles.size());
  const int root = b.build(0, static_cast<int>(mesh.triangles.size()));
  HostBvh out;
  out.binary_nodes = static_cast<int64_t>(b.nodes.size());
  out.sah_cost = b.sah_cost(root) / std::max(b.nodes[root].box.area(), 1e-30);
  out.tris.reserve(mesh.triangles.size());
  Collapser c{b, out};
  c.emit(root, 0);
  if (out.tris.size() != mesh.triangles.size()) throw Error(N2W_EINTERNAL, "internal BVH build error");
  return out;
}

n2w_bvh_stats host_stats(const HostBvh& h, int leaf_size, double ms) {
  n2w_bvh_stats s{};
  s.triangles = static_cast<int64_t>(h.tris.size());
  s.nodes = static_cast<int64_t>(h.nodes.size());
  s.binary_nodes = h.binary_nodes;
  s.leaves = h.leaves;
  s.leaf_size = leaf_size;
  s.max_depth = h.max_depth;
  s.sah_cost = h.sah_cost;
  s.build_milliseconds = ms;
  s.device_bytes = static_cast<int64_t>(h.nodes.size() * sizeof(Node4) + h.tris.size() * sizeof(TriRec));
  return s;
}

}  // namespace n2w

struct n2w_bvh_host {
  n2w::HostBvh h;
  n2w_bvh_stats stats;
};

extern "C" {

int n2w_bvh_host_build(const n2w_mesh* mesh, int leaf_size, const char* build_method,
                       n2w_bvh_host** out) {
  return n2w::guarded([&] {
    N2W_REQUIRE(mesh && out, "null argument");
    const auto t0 = std::chrono::steady_clock::now();
    auto* hb = new n2w_bvh_host();
    try {
      hb->h = n2w::build_bvh4(*mesh, leaf_size, build_method ? build_method : "sah");
    } catch (...) {
      delete hb;
      throw;
    }
    const auto t1 = std::chrono::steady_clock::now();
    hb->stats = n2w::host_stats(hb->h, leaf_size, std::chrono::duration<double, std::milli>(t1 - t0).count());
    *out = hb;
  });
}

int n2w_bvh_host_stats(const n2w_bvh_host* h, n2w_bvh_stats* out) {
  return n2w::guarded([&] {
    N2W_REQUIRE(h && out, "null argument");
    *out = h->stats;
  });
}

int n2w_bvh_host_copy(const n2w_bvh_host* h, void* nodes_out, void* tris_out) {
  return n2w::guarded([&] {
    N2W_REQUIRE(h, "null argument");
    if (nodes_out) std::memcpy(nodes_out, h->h.nodes.data(), h->h.nodes.size() * sizeof(n2w::Node4));
    if (tris_out) std::memcpy(tris_out, h->h.tris.data(), h->h.tris.size() * sizeof(n2w::TriRec));
  });
}

void n2w_bvh_host_free(n2w_bvh_host* h) { delete h; }

}  // extern "C"
