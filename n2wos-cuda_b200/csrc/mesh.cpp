// Host triangle meshes: procedural generators, PLY/OBJ loaders, normalisation.
//
// The bumpy UV sphere keeps the reference topology (poles + (stacks-1) rings
// of `slices` vertices, 2*slices*(stacks-1) triangles, cap/band/cap emission
// order; src/mesh/procedural_bumpy_sphere.cpp:32-90) so triangle ids agree with
// the reference for the reference radius function.  Loaders follow the
// reference's accepted inputs (ASCII + binary little-endian PLY with fan
// triangulation, OBJ v/f with negative indices; src/mesh/ply_loader.cpp,
// src/mesh/obj_loader.cpp:63-109).
#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstring>
#include <fstream>
#include <map>
#include <sstream>
#include <thread>
#include <utility>

#include "internal.hpp"
#include "philox.cuh"

namespace n2w {
namespace {

constexpr float kPiF = 3.14159265358979323846f;

void require_valid(const n2w_mesh& m) {
  if (m.vertices.empty()) throw Error(N2W_EINVAL, "mesh has no vertices");
  if (m.triangles.empty()) throw Error(N2W_EINVAL, "mesh has no triangles");
  const size_t nv = m.vertices.size();
  for (const auto& t : m.triangles) {
    if (t[0] >= nv || t[1] >= nv || t[2] >= nv) {
      throw Error(N2W_EINVAL, "mesh triangle contains out-of-range vertex index");
    }
  }
}

// Closest point on triangle abc to p (Ericson, Real-Time Collision Detection
// 5.1.5) with the device kernel's operation order, one IEEE operation per
// step (this file is compiled without FP contraction), so host and device
// agree bit for bit.
struct HostHit {
  float d2;
  int id;
  float cp[3];
};

inline float hdot(const float* a, const float* b) { return (a[0] * b[0] + a[1] * b[1]) + a[2] * b[2]; }

void closest_on_triangle(const float* p, const float* a, const float* b, const float* c, float* r) {
  const float ab[3] = {b[0] - a[0], b[1] - a[1], b[2] - a[2]};
  const float ac[3] = {c[0] - a[0], c[1] - a[1], c[2] - a[2]};
  const float ap[3] = {p[0] - a[0], p[1] - a[1], p[2] - a[2]};
  const float d1 = hdot(ab, ap), d2 = hdot(ac, ap);
  if (d1 <= 0.0f && d2 <= 0.0f) { std::memcpy(r, a, 12); return; }
  const float bp[3] = {p[0] - b[0], p[1] - b[1], p[2] - b[2]};
  const float d3 = hdot(ab, bp), d4 = hdot(ac, bp);
  if (d3 >= 0.0f && d4 <= d3) { std::memcpy(r, b, 12); return; }
  const float vc = d1 * d4 - d3 * d2;
  if (vc <= 0.0f && d1 >= 0.0f && d3 <= 0.0f) {
    const float v = d1 / (d1 - d3);
    for (int k = 0; k < 3; ++k) r[k] = a[k] + ab[k] * v;
    return;
  }
  const float cq[3] = {p[0] - c[0], p[1] - c[1], p[2] - c[2]};
  const float d5 = hdot(ab, cq), d6 = hdot(ac, cq);
  if (d6 >= 0.0f && d5 <= d6) { std::memcpy(r, c, 12); return; }
  const float vb = d5 * d2 - d1 * d6;
  if (vb <= 0.0f && d2 >= 0.0f && d6 <= 0.0f) {
    const float w = d2 / (d2 - d6);
    for (int k = 0; k < 3; ++k) r[k] = a[k] + ac[k] * w;
    return;
  }
  const float va = d3 * d6 - d5 * d4;
  const float d43 = d4 - d3, d56 = d5 - d6;
  if (va <= 0.0f && d43 >= 0.0f && d56 >= 0.0f) {
    const float w = d43 / (d43 + d56);
    for (int k = 0; k < 3; ++k) r[k] = b[k] + (c[k] - b[k]) * w;
    return;
  }
  const float q = 1.0f / ((va + vb) + vc);
  const float v = vb * q, w = vc * q;
  for (int k = 0; k < 3; ++k) r[k] = (a[k] + ab[k] * v) + ac[k] * w;
}

// Every triangle in id order; strict '<' keeps the lowest id on exact ties.
HostHit closest_bruteforce(const n2w_mesh& m, float x, float y, float z) {
  const float p[3] = {x, y, z};
  HostHit best{INFINITY, -1, {x, y, z}};
  for (size_t t = 0; t < m.triangles.size(); ++t) {
    const auto& tri = m.triangles[t];
    float r[3];
    closest_on_triangle(p, m.vertices[tri[0]].data(), m.vertices[tri[1]].data(), m.vertices[tri[2]].data(), r);
    const float dv[3] = {r[0] - p[0], r[1] - p[1], r[2] - p[2]};
    const float dd = hdot(dv, dv);
    if (dd < best.d2) {
      best.d2 = dd;
      best.id = static_cast<int>(t);
      std::memcpy(best.cp, r, 12);
    }
  }
  return best;
}

// Radius function of the reference generator (procedural_bumpy_sphere.cpp:12-17),
// evaluated with the same float expressions.
float ref_bump_radius(float theta, float phi, float amplitude) {
  const float low = std::sin(3.0f * theta + 0.35f * std::cos(5.0f * phi));
  const float high = std::sin(7.0f * phi + 0.5f * std::cos(2.0f * theta));
  const float mid = std::cos(5.0f * theta - 2.0f * phi);
  return 1.0f + amplitude * (0.45f * low * high + 0.35f * mid * std::sin(theta) + 0.20f * std::sin(4.0f * theta));
}

template <typename RadiusFn>
n2w_mesh* uv_sphere(int stacks, int slices, const char* name, RadiusFn radius) {
  auto* m = new n2w_mesh();
  m->name = name;
  auto point = [&](float theta, float phi) {
    const float r = radius(theta, phi);
    const float st = std::sin(theta);
    return std::array<float, 3>{r * st * std::cos(phi), r * st * std::sin(phi), r * std::cos(theta)};
  };
  auto ring = [&](int i, int j) { return static_cast<uint32_t>(1 + (i - 1) * slices + (j % slices)); };
  m->vertices.reserve(2 + static_cast<size_t>(stacks - 1) * slices);
  m->vertices.push_back(point(0.0f, 0.0f));
  for (int i = 1; i <= stacks - 1; ++i) {
    const float theta = kPiF * static_cast<float>(i) / static_cast<float>(stacks);
    for (int j = 0; j < slices; ++j) {
      const float phi = 2.0f * kPiF * static_cast<float>(j) / static_cast<float>(slices);
      m->vertices.push_back(point(theta, phi));
    }
  }
  const uint32_t south = static_cast<uint32_t>(m->vertices.size());
  m->vertices.push_back(point(kPiF, 0.0f));
  m->triangles.reserve(static_cast<size_t>(2) * slices * (stacks - 1));
  for (int j = 0; j < slices; ++j) m->triangles.push_back({0u, ring(1, j), ring(1, j + 1)});
  for (int i = 1; i < stacks - 1; ++i) {
    for (int j = 0; j < slices; ++j) {
      const uint32_t a = ring(i, j), b = ring(i, j + 1), c = ring(i + 1, j), d = ring(i + 1, j + 1);
      m->triangles.push_back({a, c, b});
      m->triangles.push_back({b, c, d});
    }
  }
  for (int j = 0; j < slices; ++j) m->triangles.push_back({ring(stacks - 1, j), south, ring(stacks - 1, j + 1)});
  return m;
}

// ---- seeded value noise ------------------------------------------------
// Lattice values in [-1, 1] hashed from integer coordinates and the seed,
// trilinearly interpolated with the quintic fade 6t^5 - 15t^4 + 10t^3.
double lattice_value(int64_t ix, int64_t iy, int64_t iz, uint64_t seed) {
  uint64_t s = seed ^ (static_cast<uint64_t>(ix) * 0x9E3779B97F4A7C15ull) ^
               (static_cast<uint64_t>(iy) * 0xC2B2AE3D27D4EB4Full) ^
               (static_cast<uint64_t>(iz) * 0x165667B19E3779F9ull);
  return 2.0 * splitmix64_unit(s) - 1.0;
}

double fade(double t) { return t * t * t * (t * (t * 6.0 - 15.0) + 10.0); }

double value_noise(double x, double y, double z, uint64_t seed) {
  const double fx = std::floor(x), fy = std::floor(y), fz = std::floor(z);
  const int64_t ix = static_cast<int64_t>(fx), iy = static_cast<int64_t>(fy), iz = static_cast<int64_t>(fz);
  const double tx = fade(x - fx), ty = fade(y - fy), tz = fade(z - fz);
  double c[2][2][2];
  for (int a = 0; a < 2; ++a)
    for (int b = 0; b < 2; ++b)
      for (int d = 0; d < 2; ++d) c[a][b][d] = lattice_value(ix + a, iy + b, iz + d, seed);
  const double x00 = c[0][0][0] + tx * (c[1][0][0] - c[0][0][0]);
  const double x10 = c[0][1][0] + tx * (c[1][1][0] - c[0][1][0]);
  const double x01 = c[0][0][1] + tx * (c[1][0][1] - c[0][0][1]);
  const double x11 = c[0][1][1] + tx * (c[1][1][1] - c[0][1][1]);
  const double y0 = x00 + ty * (x10 - x00);
  const double y1 = x01 + ty * (x11 - x01);
  return y0 + tz * (y1 - y0);
}

// Octave sum normalised by the total amplitude, so the result stays in [-1, 1].
double fractal_noise(double x, double y, double z, double base_freq, int octaves, double persistence,
                     uint64_t seed) {
  double sum = 0.0, norm = 0.0, amp = 1.0, freq = base_freq;
  for (int o = 0; o < octaves; ++o) {
    uint64_t os = seed + 0x632BE59BD9B4E019ull * static_cast<uint64_t>(o + 1);
    sum += amp * value_noise(x * freq, y * freq, z * freq, splitmix64_next(os));
    norm += amp;
    amp *= persistence;
    freq *= 2.0;
  }
  return norm > 0.0 ? sum / norm : 0.0;
}

n2w_mesh* icosphere(int level) {
  const double t = (1.0 + std::sqrt(5.0)) / 2.0;
  std::vector<std::array<double, 3>> v = {{-1, t, 0}, {1, t, 0}, {-1, -t, 0}, {1, -t, 0},
                                          {0, -1, t}, {0, 1, t}, {0, -1, -t}, {0, 1, -t},
                                          {t, 0, -1}, {t, 0, 1}, {-t, 0, -1}, {-t, 0, 1}};
  for (auto& p : v) {
    const double n = std::sqrt(p[0] * p[0] + p[1] * p[1] + p[2] * p[2]);
    for (double& c : p) c /= n;
  }
  std::vector<std::array<uint32_t, 3>> f = {{0, 11, 5}, {0, 5, 1},  {0, 1, 7},   {0, 7, 10}, {0, 10, 11},
                                            {1, 5, 9},  {5, 11, 4}, {11, 10, 2}, {10, 7, 6}, {7, 1, 8},
                                            {3, 9, 4},  {3, 4, 2},  {3, 2, 6},   {3, 6, 8},  {3, 8, 9},
                                            {4, 9, 5},  {2, 4, 11}, {6, 2, 10},  {8, 6, 7},  {9, 8, 1}};
  for (int l = 0; l < level; ++l) {
    std::map<std::pair<uint32_t, uint32_t>, uint32_t> mid;
    auto midpoint = [&](uint32_t a, uint32_t b) {
      const auto key = std::make_pair(std::min(a, b), std::max(a, b));
      auto it = mid.find(key);
      if (it != mid.end()) return it->second;
      std::array<double, 3> p{(v[a][0] + v[b][0]) * 0.5, (v[a][1] + v[b][1]) * 0.5, (v[a][2] + v[b][2]) * 0.5};
      const double n = std::sqrt(p[0] * p[0] + p[1] * p[1] + p[2] * p[2]);
      for (double& c : p) c /= n;
      v.push_back(p);
      const uint32_t id = static_cast<uint32_t>(v.size() - 1);
      mid.emplace(key, id);
      return id;
    };
    std::vector<std::array<uint32_t, 3>> nf;
    nf.reserve(f.size() * 4);
    for (const auto& tri : f) {
      const uint32_t a = midpoint(tri[0], tri[1]);
      const uint32_t b = midpoint(tri[1], tri[2]);
      const uint32_t c = midpoint(tri[2], tri[0]);
      nf.push_back({tri[0], a, c});
      nf.push_back({tri[1], b, a});
      nf.push_back({tri[2], c, b});
      nf.push_back({a, b, c});
    }
    f.swap(nf);
  }
  auto* m = new n2w_mesh();
  m->vertices.reserve(v.size());
  for (const auto& p : v) {
    m->vertices.push_back({static_cast<float>(p[0]), static_cast<float>(p[1]), static_cast<float>(p[2])});
  }
  m->triangles = std::move(f);
  return m;
}

// ---- loaders ------------------------------------------------------------
std::string base_name(const std::string& path) {
  const size_t s = path.find_last_of("/\\");
  return s == std::string::npos ? path : path.substr(s + 1);
}

void fan(n2w_mesh& m, const std::vector<int64_t>& face, size_t nv, const char* what) {
  if (face.size() < 3) throw Error(N2W_EIO, std::string(what) + " face has fewer than 3 vertices");
  for (int64_t idx : face) {
    if (idx < 0 || idx >= static_cast<int64_t>(nv)) throw Error(N2W_EIO, std::string(what) + " face vertex index out of range");
  }
  for (size_t i = 1; i + 1 < face.size(); ++i) {
    m.triangles.push_back({static_cast<uint32_t>(face[0]), static_cast<uint32_t>(face[i]),
                           static_cast<uint32_t>(face[i + 1])});
  }
}

struct PlyProp {
  std::string name;
  std::string type;       // scalar type, or item type for lists
  std::string count_type; // non-empty for lists
};
struct PlyElem {
  std::string name;
  size_t count = 0;
  std::vector<PlyProp> props;
};

size_t ply_type_size(const std::string& t) {
  if (t == "char" || t == "int8" || t == "uchar" || t == "uint8") return 1;
  if (t == "short" || t == "int16" || t == "ushort" || t == "uint16") return 2;
  if (t == "int" || t == "int32" || t == "uint" || t == "uint32" || t == "float" || t == "float32") return 4;
  if (t == "double" || t == "float64") return 8;
  throw Error(N2W_EIO, "unsupported PLY scalar type: " + t);
}

double ply_read(const unsigned char*& p, const unsigned char* end, const std::string& t) {
  const size_t n = ply_type_size(t);
  if (static_cast<size_t>(end - p) < n) throw Error(N2W_EIO, "truncated binary PLY data");
  double v = 0.0;
  if (t == "char" || t == "int8") { int8_t x; std::memcpy(&x, p, 1); v = x; }
  else if (t == "uchar" || t == "uint8") { uint8_t x; std::memcpy(&x, p, 1); v = x; }
  else if (t == "short" || t == "int16") { int16_t x; std::memcpy(&x, p, 2); v = x; }
  else if (t == "ushort" || t == "uint16") { uint16_t x; std::memcpy(&x, p, 2); v = x; }
  else if (t == "int" || t == "int32") { int32_t x; std::memcpy(&x, p, 4); v = x; }
  else if (t == "uint" || t == "uint32") { uint32_t x; std::memcpy(&x, p, 4); v = x; }
  else if (t == "float" || t == "float32") { float x; std::memcpy(&x, p, 4); v = x; }
  else { double x; std::memcpy(&x, p, 8); v = x; }
  p += n;
  return v;
}

n2w_mesh* load_ply(const std::string& path) {
  std::ifstream in(path, std::ios::binary);
  if (!in) throw Error(N2W_EIO, "failed to open PLY file: " + path);
  std::string line;
  if (!std::getline(in, line) || line.substr(0, 3) != "ply") throw Error(N2W_EIO, "not a PLY file: " + path);
  bool binary = false, have_format = false;
  std::vector<PlyElem> elems;
  for (;;) {
    if (!std::getline(in, line)) throw Error(N2W_EIO, "PLY header ended before end_header");
    if (!line.empty() && line.back() == '\r') line.pop_back();
    std::istringstream ss(line);
    std::string kw;
    ss >> kw;
    if (kw == "format") {
      std::string fmt;
      ss >> fmt;
      if (fmt == "ascii") binary = false;
      else if (fmt == "binary_little_endian") binary = true;
      else throw Error(N2W_EIO, "unsupported PLY format: " + fmt);
      have_format = true;
    } else if (kw == "element") {
      PlyElem e;
      ss >> e.name >> e.count;
      elems.push_back(e);
    } else if (kw == "property") {
      if (elems.empty()) throw Error(N2W_EIO, "PLY property before element");
      PlyProp p;
      std::string t;
      ss >> t;
      if (t == "list") ss >> p.count_type >> p.type >> p.name;
      else { p.type = t; ss >> p.name; }
      elems.back().props.push_back(p);
    } else if (kw == "end_header") {
      break;
    }
  }
  if (!have_format) throw Error(N2W_EIO, "PLY header has no format line");
  auto* m = new n2w_mesh();
  m->name = base_name(path);
  try {
    auto face_list_index = [](const PlyElem& e) {
      for (size_t i = 0; i < e.props.size(); ++i) {
        const auto& p = e.props[i];
        if (!p.count_type.empty() && (p.name == "vertex_indices" || p.name == "vertex_index" || p.name == "vertices")) return static_cast<int>(i);
      }
      for (size_t i = 0; i < e.props.size(); ++i) if (!e.props[i].count_type.empty()) return static_cast<int>(i);
      return -1;
    };
    if (binary) {
      std::vector<unsigned char> buf((std::istreambuf_iterator<char>(in)), std::istreambuf_iterator<char>());
      const unsigned char* p = buf.data();
      const unsigned char* end = buf.data() + buf.size();
      for (const auto& e : elems) {
        const int fi = face_list_index(e);
        for (size_t r = 0; r < e.count; ++r) {
          std::array<float, 3> xyz{0, 0, 0};
          std::vector<int64_t> face;
          for (size_t k = 0; k < e.props.size(); ++k) {
            const auto& pr = e.props[k];
            if (!pr.count_type.empty()) {
              const int64_t cnt = static_cast<int64_t>(ply_read(p, end, pr.count_type));
              if (cnt < 0) throw Error(N2W_EIO, "negative PLY list count");
              for (int64_t c = 0; c < cnt; ++c) {
                const double v = ply_read(p, end, pr.type);
                if (e.name == "face" && static_cast<int>(k) == fi) face.push_back(static_cast<int64_t>(v));
              }
            } else {
              const double v = ply_read(p, end, pr.type);
              if (e.name == "vertex") {
                if (pr.name == "x") xyz[0] = static_cast<float>(v);
                if (pr.name == "y") xyz[1] = static_cast<float>(v);
                if (pr.name == "z") xyz[2] = static_cast<float>(v);
              }
            }
          }
          if (e.name == "vertex") m->vertices.push_back(xyz);
          if (e.name == "face") fan(*m, face, m->vertices.size(), "PLY");
        }
      }
    } else {
      for (const auto& e : elems) {
        const int fi = face_list_index(e);
        for (size_t r = 0; r < e.count; ++r) {
          if (!std::getline(in, line)) throw Error(N2W_EIO, "unexpected end of ASCII PLY data");
          std::istringstream ss(line);
          std::array<float, 3> xyz{0, 0, 0};
          std::vector<int64_t> face;
          for (size_t k = 0; k < e.props.size(); ++k) {
            const auto& pr = e.props[k];
            if (!pr.count_type.empty()) {
              int64_t cnt = 0;
              if (!(ss >> cnt) || cnt < 0) throw Error(N2W_EIO, "invalid ASCII PLY list count");
              for (int64_t c = 0; c < cnt; ++c) {
                double v;
                if (!(ss >> v)) throw Error(N2W_EIO, "truncated ASCII PLY list");
                if (e.name == "face" && static_cast<int>(k) == fi) face.push_back(static_cast<int64_t>(v));
              }
            } else {
              std::string tok;
              if (!(ss >> tok)) throw Error(N2W_EIO, "truncated ASCII PLY line");
              if (e.name == "vertex") {
                const float v = static_cast<float>(std::stod(tok));
                if (pr.name == "x") xyz[0] = v;
                if (pr.name == "y") xyz[1] = v;
                if (pr.name == "z") xyz[2] = v;
              }
            }
          }
          if (e.name == "vertex") m->vertices.push_back(xyz);
          if (e.name == "face") fan(*m, face, m->vertices.size(), "PLY");
        }
      }
    }
    require_valid(*m);
  } catch (...) {
    delete m;
    throw;
  }
  return m;
}

n2w_mesh* load_obj(const std::string& path) {
  std::ifstream in(path);
  if (!in) throw Error(N2W_EIO, "failed to open OBJ file: " + path);
  auto* m = new n2w_mesh();
  m->name = base_name(path);
  try {
    std::string line;
    size_t lineno = 0;
    while (std::getline(in, line)) {
      ++lineno;
      std::istringstream ss(line);
      std::string tag;
      if (!(ss >> tag) || tag[0] == '#') continue;
      if (tag == "v") {
        std::array<float, 3> p;
        if (!(ss >> p[0] >> p[1] >> p[2])) throw Error(N2W_EIO, "invalid OBJ vertex at line " + std::to_string(lineno));
        m->vertices.push_back(p);
      } else if (tag == "f") {
        std::vector<int64_t> face;
        std::string tok;
        while (ss >> tok) {
          const std::string head = tok.substr(0, tok.find('/'));
          size_t used = 0;
          const long long raw = std::stoll(head, &used);
          if (used != head.size() || raw == 0) throw Error(N2W_EIO, "invalid OBJ face index at line " + std::to_string(lineno));
          face.push_back(raw > 0 ? raw - 1 : static_cast<int64_t>(m->vertices.size()) + raw);
        }
        fan(*m, face, m->vertices.size(), "OBJ");
      }
    }
    require_valid(*m);
  } catch (...) {
    delete m;
    throw;
  }
  return m;
}

void normalize(n2w_mesh& m, float* center_out, float* scale_out) {
  require_valid(m);
  float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
  for (const auto& p : m.vertices) {
    for (int a = 0; a < 3; ++a) {
      lo[a] = std::min(lo[a], p[a]);
      hi[a] = std::max(hi[a], p[a]);
    }
  }
  // Same float sequence as the reference (normalize.cpp:21-36): centre of the
  // AABB, radius = max |p - centre|, p <- (p - centre) / radius.
  const float c[3] = {(lo[0] + hi[0]) * 0.5f, (lo[1] + hi[1]) * 0.5f, (lo[2] + hi[2]) * 0.5f};
  float radius = 0.0f;
  for (const auto& p : m.vertices) {
    const float dx = p[0] - c[0], dy = p[1] - c[1], dz = p[2] - c[2];
    radius = std::max(radius, std::sqrt(dx * dx + dy * dy + dz * dz));
  }
  if (!(radius > 0.0f)) throw Error(N2W_EINVAL, "cannot normalize mesh with zero radius");
  for (auto& p : m.vertices) {
    p = {(p[0] - c[0]) / radius, (p[1] - c[1]) / radius, (p[2] - c[2]) / radius};
  }
  if (center_out) std::memcpy(center_out, c, sizeof(c));
  if (scale_out) *scale_out = 1.0f / radius;
}

}  // namespace
}  // namespace n2w

using namespace n2w;

extern "C" {

int n2w_mesh_create(const float* vertices, int64_t nv, const uint32_t* triangles, int64_t nt,
                    const char* name, n2w_mesh** out) {
  return guarded([&] {
    N2W_REQUIRE(out && vertices && triangles && nv > 0 && nt > 0, "n2w_mesh_create: invalid arguments");
    auto* m = new n2w_mesh();
    m->name = name ? name : "mesh";
    m->vertices.resize(static_cast<size_t>(nv));
    m->triangles.resize(static_cast<size_t>(nt));
    std::memcpy(m->vertices.data(), vertices, sizeof(float) * 3 * static_cast<size_t>(nv));
    std::memcpy(m->triangles.data(), triangles, sizeof(uint32_t) * 3 * static_cast<size_t>(nt));
    try {
      require_valid(*m);
    } catch (...) {
      delete m;
      throw;
    }
    *out = m;
  });
}

int n2w_mesh_bumpy_sphere_ref(int stacks, int slices, float amplitude, n2w_mesh** out) {
  return guarded([&] {
    N2W_REQUIRE(out, "null output");
    N2W_REQUIRE(stacks >= 4, "bumpy sphere requires stacks >= 4");
    N2W_REQUIRE(slices >= 8, "bumpy sphere requires slices >= 8");
    N2W_REQUIRE(amplitude >= 0.0f && amplitude <= 0.5f, "bumpy sphere bump amplitude must be in [0, 0.5]");
    *out = uv_sphere(stacks, slices, "procedural_bumpy_sphere",
                     [&](float th, float ph) { return ref_bump_radius(th, ph, amplitude); });
  });
}

int n2w_mesh_bumpy_sphere_trig(int stacks, int slices, float amplitude, int k_theta, int k_phi,
                               n2w_mesh** out) {
  return guarded([&] {
    N2W_REQUIRE(out, "null output");
    N2W_REQUIRE(stacks >= 4 && slices >= 8, "bumpy sphere requires stacks >= 4 and slices >= 8");
    N2W_REQUIRE(amplitude >= 0.0f && amplitude < 1.0f, "amplitude must be in [0, 1)");
    *out = uv_sphere(stacks, slices, "bumpy_sphere_trig", [&](float th, float ph) {
      return 1.0f + amplitude * std::sin(static_cast<float>(k_theta) * th) * std::cos(static_cast<float>(k_phi) * ph);
    });
  });
}

int n2w_mesh_icosphere_displaced(int level, float amplitude, float base_frequency, int octaves,
                                 float persistence, uint64_t seed, n2w_mesh** out) {
  return guarded([&] {
    N2W_REQUIRE(out, "null output");
    N2W_REQUIRE(level >= 0 && level <= 9, "icosphere level must be in [0, 9]");
    N2W_REQUIRE(amplitude >= 0.0f && amplitude < 1.0f, "amplitude must be in [0, 1)");
    N2W_REQUIRE(octaves >= 1 && octaves <= 16, "octaves must be in [1, 16]");
    n2w_mesh* m = icosphere(level);
    m->name = "icosphere_displaced";
    for (auto& p : m->vertices) {
      const double x = p[0], y = p[1], z = p[2];
      const double n = fractal_noise(x, y, z, base_frequency, octaves, persistence, seed);
      const double r = 1.0 + static_cast<double>(amplitude) * n;
      p = {static_cast<float>(x * r), static_cast<float>(y * r), static_cast<float>(z * r)};
    }
    *out = m;
  });
}

int n2w_mesh_load_ply(const char* path, n2w_mesh** out) {
  return guarded([&] {
    N2W_REQUIRE(path && out, "null argument");
    *out = load_ply(path);
  });
}

int n2w_mesh_load_obj(const char* path, n2w_mesh** out) {
  return guarded([&] {
    N2W_REQUIRE(path && out, "null argument");
    *out = load_obj(path);
  });
}

int n2w_mesh_normalize(n2w_mesh* mesh, float* center_out, float* scale_out) {
  return guarded([&] {
    N2W_REQUIRE(mesh, "null mesh");
    normalize(*mesh, center_out, scale_out);
  });
}

int n2w_mesh_counts(const n2w_mesh* mesh, int64_t* nv, int64_t* nt) {
  return guarded([&] {
    N2W_REQUIRE(mesh, "null mesh");
    if (nv) *nv = static_cast<int64_t>(mesh->vertices.size());
    if (nt) *nt = static_cast<int64_t>(mesh->triangles.size());
  });
}

int n2w_mesh_copy_out(const n2w_mesh* mesh, float* vertices, uint32_t* triangles) {
  return guarded([&] {
    N2W_REQUIRE(mesh, "null mesh");
    if (vertices) std::memcpy(vertices, mesh->vertices.data(), mesh->vertices.size() * 3 * sizeof(float));
    if (triangles) std::memcpy(triangles, mesh->triangles.data(), mesh->triangles.size() * 3 * sizeof(uint32_t));
  });
}

int n2w_mesh_bounds(const n2w_mesh* mesh, float* b) {
  return guarded([&] {
    N2W_REQUIRE(mesh && b, "null argument");
    require_valid(*mesh);
    for (int a = 0; a < 3; ++a) {
      b[a] = INFINITY;
      b[3 + a] = -INFINITY;
    }
    for (const auto& p : mesh->vertices) {
      for (int a = 0; a < 3; ++a) {
        b[a] = std::min(b[a], p[a]);
        b[3 + a] = std::max(b[3 + a], p[a]);
      }
    }
  });
}

int n2w_mesh_count_degenerate(const n2w_mesh* mesh, float eps, int64_t* out) {
  return guarded([&] {
    N2W_REQUIRE(mesh && out, "null argument");
    int64_t count = 0;
    for (const auto& t : mesh->triangles) {
      const auto& a = mesh->vertices[t[0]];
      const auto& b = mesh->vertices[t[1]];
      const auto& c = mesh->vertices[t[2]];
      const float ux = b[0] - a[0], uy = b[1] - a[1], uz = b[2] - a[2];
      const float vx = c[0] - a[0], vy = c[1] - a[1], vz = c[2] - a[2];
      const float cx = uy * vz - uz * vy, cy = uz * vx - ux * vz, cz = ux * vy - uy * vx;
      if (cx * cx + cy * cy + cz * cz <= eps) ++count;
    }
    *out = count;
  });
}

int n2w_mesh_closest_point_host(const n2w_mesh* mesh, const float* xyz, int64_t n, float* d2_out,
                                float* closest_out, int* tri_out, int threads) {
  return guarded([&] {
    N2W_REQUIRE(mesh && (n == 0 || xyz), "null argument");
    N2W_REQUIRE(n >= 0, "n must be non-negative");
    require_valid(*mesh);
    if (n == 0) return;
    int nt = threads > 0 ? threads : static_cast<int>(std::max(1u, std::thread::hardware_concurrency()));
    nt = static_cast<int>(std::min<int64_t>(nt, std::max<int64_t>(1, n / 16)));
    auto work = [&](int64_t lo, int64_t hi) {
      for (int64_t i = lo; i < hi; ++i) {
        const HostHit h = closest_bruteforce(*mesh, xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2]);
        if (d2_out) d2_out[i] = h.d2;
        if (closest_out) {
          closest_out[3 * i + 0] = h.cp[0];
          closest_out[3 * i + 1] = h.cp[1];
          closest_out[3 * i + 2] = h.cp[2];
        }
        if (tri_out) tri_out[i] = h.id;
      }
    };
    if (nt == 1) {
      work(0, n);
      return;
    }
    std::vector<std::thread> pool;
    const int64_t per = (n + nt - 1) / nt;
    for (int t = 0; t < nt; ++t) {
      const int64_t lo = t * per, hi = std::min<int64_t>(n, lo + per);
      if (lo < hi) pool.emplace_back(work, lo, hi);
    }
    for (auto& th : pool) th.join();
  });
}

const char* n2w_mesh_name(const n2w_mesh* mesh) { return mesh ? mesh->name.c_str() : ""; }

void n2w_mesh_free(n2w_mesh* mesh) { delete mesh; }

}  // extern "C"
