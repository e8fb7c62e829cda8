// Shared plumbing of the command-line tools: strict option parsing, JSON
// helpers, the CUDA description block, mesh selection and RAII wrappers over
// the C ABI (include/n2w.h).  The tools keep the reference tools' flags, JSON
// schemas and exit codes (src/tools/*.cpp|cu); everything they compute goes
// through libn2w.
#pragma once

#include <algorithm>
#include <array>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <ctime>
#include <filesystem>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <numeric>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "n2w.h"

namespace tool {

// Throws with the library's message when a C-ABI call fails.
inline void check(int status, const char* what) {
  if (status != N2W_OK) {
    throw std::runtime_error(std::string(what) + " failed (status " + std::to_string(status) +
                             "): " + n2w_last_error());
  }
}
#define N2W_CHECK(expr) ::tool::check((expr), #expr)

inline std::string require_value(int& i, int argc, char** argv) {
  if (i + 1 >= argc) throw std::runtime_error(std::string("missing value for ") + argv[i]);
  return argv[++i];
}

inline int parse_int(const std::string& s, const std::string& name) {
  try {
    size_t pos = 0;
    const int v = std::stoi(s, &pos);
    if (pos != s.size()) throw std::runtime_error("trailing characters");
    return v;
  } catch (const std::exception&) {
    throw std::runtime_error("failed to parse integer for " + name + ": " + s);
  }
}

inline float parse_float(const std::string& s, const std::string& name) {
  try {
    size_t pos = 0;
    const float v = std::stof(s, &pos);
    if (pos != s.size()) throw std::runtime_error("trailing characters");
    return v;
  } catch (const std::exception&) {
    throw std::runtime_error("failed to parse float for " + name + ": " + s);
  }
}

inline uint64_t parse_u64(const std::string& s, const std::string& name) {
  try {
    size_t pos = 0;
    const unsigned long long v = std::stoull(s, &pos);
    if (pos != s.size()) throw std::runtime_error("trailing characters");
    return static_cast<uint64_t>(v);
  } catch (const std::exception&) {
    throw std::runtime_error("failed to parse unsigned integer for " + name + ": " + s);
  }
}

inline std::vector<float> parse_float_list(const std::string& s, size_t count, const std::string& name) {
  std::stringstream ss(s);
  std::string tok;
  std::vector<float> v;
  while (std::getline(ss, tok, ',')) {
    if (!tok.empty()) v.push_back(parse_float(tok, name));
  }
  if (v.size() != count) {
    throw std::runtime_error(name + " expects " + std::to_string(count) + " comma-separated values");
  }
  return v;
}

inline std::vector<int> parse_int_list(const std::string& s, const std::string& name) {
  std::stringstream ss(s);
  std::string tok;
  std::vector<int> v;
  while (std::getline(ss, tok, ',')) {
    if (!tok.empty()) v.push_back(parse_int(tok, name));
  }
  if (v.empty()) throw std::runtime_error(name + " expects a comma-separated list");
  return v;
}

inline std::vector<std::string> parse_str_list(const std::string& s) {
  std::stringstream ss(s);
  std::string tok;
  std::vector<std::string> v;
  while (std::getline(ss, tok, ',')) {
    if (!tok.empty()) v.push_back(tok);
  }
  return v;
}

inline std::string json_quote(const std::string& s) {
  std::string o = "\"";
  for (const char ch : s) {
    switch (ch) {
      case '"': o += "\\\""; break;
      case '\\': o += "\\\\"; break;
      case '\n': o += "\\n"; break;
      case '\r': o += "\\r"; break;
      case '\t': o += "\\t"; break;
      default:
        if (static_cast<unsigned char>(ch) < 0x20) {
          char buf[8];
          std::snprintf(buf, sizeof(buf), "\\u%04x", ch);
          o += buf;
        } else {
          o += ch;
        }
    }
  }
  return o + "\"";
}

// Finite doubles print as numbers; NaN / inf as null so the file stays JSON.
inline std::string num(double v) {
  if (!std::isfinite(v)) return "null";
  std::ostringstream o;
  o << std::setprecision(9) << v;
  return o.str();
}

inline std::string vec3_json(const float* p) { return "[" + num(p[0]) + ", " + num(p[1]) + ", " + num(p[2]) + "]"; }

inline std::string floats_json(const std::vector<float>& v) {
  std::string o = "[";
  for (size_t i = 0; i < v.size(); ++i) o += (i ? ", " : "") + num(v[i]);
  return o + "]";
}

inline std::string utc_now() {
  const std::time_t t = std::time(nullptr);
  std::tm tm{};
  gmtime_r(&t, &tm);
  char buf[64];
  std::strftime(buf, sizeof(buf), "%Y-%m-%dT%H:%M:%SZ", &tm);
  return buf;
}

inline std::string join_argv(int argc, char** argv) {
  std::string o;
  for (int i = 0; i < argc; ++i) o += (i ? " " : "") + std::string(argv[i]);
  return o;
}

// {"runtime": "runtime=..,driver=..", "device": "<name> sm_XY global_mem=.."}
inline std::string cuda_json(const std::string& indent = "  ") {
  char rt[128] = {0}, dev[256] = {0};
  N2W_CHECK(n2w_cuda_runtime_version_string(rt, sizeof(rt)));
  N2W_CHECK(n2w_cuda_device_summary(dev, sizeof(dev)));
  return "{\n" + indent + "  \"runtime\": " + json_quote(rt) + ",\n" + indent + "  \"device\": " + json_quote(dev) +
         "\n" + indent + "}";
}

inline float median(std::vector<float> v) {
  if (v.empty()) return 0.0f;
  std::sort(v.begin(), v.end());
  const size_t m = v.size() / 2;
  return v.size() % 2 ? v[m] : 0.5f * (v[m - 1] + v[m]);
}

inline float mean(const std::vector<float>& v) {
  if (v.empty()) return 0.0f;
  return std::accumulate(v.begin(), v.end(), 0.0f) / static_cast<float>(v.size());
}

inline void ensure_parent_dir(const std::string& path) {
  const std::filesystem::path p(path);
  if (p.has_parent_path()) std::filesystem::create_directories(p.parent_path());
}

inline void write_text(const std::string& path, const std::string& text) {
  ensure_parent_dir(path);
  std::ofstream f(path);
  if (!f) throw std::runtime_error("failed to open output: " + path);
  f << text;
}

// ---- mesh selection (reference tools' --mesh/--mesh-path/--normalize/--bumpy-*) ----

struct MeshOptions {
  std::string mesh = "procedural_bumpy_sphere";
  std::string mesh_path;
  int normalize = 1;
  int bumpy_stacks = 128;
  int bumpy_slices = 256;
  float bumpy_amplitude = 0.15f;

  // Consumes a mesh flag; returns false when `arg` is not one.
  bool parse(const std::string& arg, int& i, int argc, char** argv) {
    if (arg == "--mesh") mesh = require_value(i, argc, argv);
    else if (arg == "--mesh-path") mesh_path = require_value(i, argc, argv);
    else if (arg == "--normalize") normalize = parse_int(require_value(i, argc, argv), arg);
    else if (arg == "--bumpy-stacks") bumpy_stacks = parse_int(require_value(i, argc, argv), arg);
    else if (arg == "--bumpy-slices") bumpy_slices = parse_int(require_value(i, argc, argv), arg);
    else if (arg == "--bumpy-amplitude") bumpy_amplitude = parse_float(require_value(i, argc, argv), arg);
    else return false;
    return true;
  }

  void validate() const {
    if (mesh != "procedural_bumpy_sphere" && mesh != "obj" && mesh != "ply") {
      throw std::runtime_error("--mesh must be procedural_bumpy_sphere, obj, or ply");
    }
    if ((mesh == "obj" || mesh == "ply") && mesh_path.empty()) {
      throw std::runtime_error("--mesh-path is required when --mesh obj or ply");
    }
  }
};

class Mesh {
 public:
  n2w_mesh* m = nullptr;
  bool normalized = false;
  float center[3] = {0, 0, 0};
  float scale = 1.0f;

  explicit Mesh(const MeshOptions& o) {
    if (o.mesh == "procedural_bumpy_sphere") {
      N2W_CHECK(n2w_mesh_bumpy_sphere_ref(o.bumpy_stacks, o.bumpy_slices, o.bumpy_amplitude, &m));
    } else if (o.mesh == "obj") {
      N2W_CHECK(n2w_mesh_load_obj(o.mesh_path.c_str(), &m));
    } else {
      N2W_CHECK(n2w_mesh_load_ply(o.mesh_path.c_str(), &m));
    }
    // The procedural sphere is always normalised (reference probe_cuda_bvh.cpp:349-352).
    if (o.mesh == "procedural_bumpy_sphere" || o.normalize != 0) {
      N2W_CHECK(n2w_mesh_normalize(m, center, &scale));
      normalized = true;
    }
  }
  ~Mesh() { n2w_mesh_free(m); }
  Mesh(const Mesh&) = delete;
  Mesh& operator=(const Mesh&) = delete;

  int64_t vertices() const {
    int64_t nv = 0, nt = 0;
    N2W_CHECK(n2w_mesh_counts(m, &nv, &nt));
    return nv;
  }
  int64_t triangles() const {
    int64_t nv = 0, nt = 0;
    N2W_CHECK(n2w_mesh_counts(m, &nv, &nt));
    return nt;
  }
  void bounds(float* b6) const { N2W_CHECK(n2w_mesh_bounds(m, b6)); }
  int64_t degenerate() const {
    int64_t d = 0;
    N2W_CHECK(n2w_mesh_count_degenerate(m, 1.0e-24f, &d));
    return d;
  }
};

// mesh_stats block: name, vertices, triangles, degenerate count, bounds, normalisation.
inline std::string mesh_stats_json(const Mesh& mesh, const std::string& name, bool always_normalization) {
  float b[6];
  mesh.bounds(b);
  std::ostringstream o;
  o << "{\n"
    << "    \"name\": " << json_quote(name) << ",\n"
    << "    \"vertices\": " << mesh.vertices() << ",\n"
    << "    \"triangles\": " << mesh.triangles() << ",\n"
    << "    \"degenerate_triangles\": " << mesh.degenerate() << ",\n"
    << "    \"bounds_min\": " << vec3_json(b) << ",\n"
    << "    \"bounds_max\": " << vec3_json(b + 3);
  if (mesh.normalized || always_normalization) {
    o << ",\n    \"normalization\": {\"center\": " << vec3_json(mesh.center) << ", \"scale\": " << num(mesh.scale)
      << "}\n";
  } else {
    o << "\n";
  }
  o << "  }";
  return o.str();
}

class Bvh {
 public:
  n2w_bvh* b = nullptr;
  n2w_bvh_stats stats{};
  std::string method;
  Bvh(const Mesh& mesh, int leaf_size, const std::string& build_method) : method(build_method) {
    N2W_CHECK(n2w_bvh_create(mesh.m, leaf_size, build_method.c_str(), &b));
    N2W_CHECK(n2w_bvh_stats_get(b, &stats));
  }
  ~Bvh() { n2w_bvh_destroy(b); }
  Bvh(const Bvh&) = delete;
  Bvh& operator=(const Bvh&) = delete;
};

// Device buffer of T (n2w_malloc / n2w_free).
template <typename T>
class DeviceArray {
 public:
  T* p = nullptr;
  size_t n = 0;
  DeviceArray() = default;
  explicit DeviceArray(size_t count) { reset(count); }
  ~DeviceArray() { release(); }
  DeviceArray(const DeviceArray&) = delete;
  DeviceArray& operator=(const DeviceArray&) = delete;
  void reset(size_t count) {
    release();
    n = count;
    void* q = nullptr;
    N2W_CHECK(n2w_malloc(&q, std::max<size_t>(count, 1) * sizeof(T)));
    p = static_cast<T*>(q);
  }
  void release() {
    if (p) n2w_free(p);
    p = nullptr;
    n = 0;
  }
  void upload(const T* h, size_t count, n2w_stream_t s = nullptr) {
    N2W_CHECK(n2w_memcpy_h2d(p, h, count * sizeof(T), s));
  }
  void download(T* h, size_t count, n2w_stream_t s = nullptr) const {
    N2W_CHECK(n2w_memcpy_d2h(h, p, count * sizeof(T), s));
  }
  std::vector<T> to_host(size_t count, n2w_stream_t s = nullptr) const {
    std::vector<T> v(count);
    if (count) download(v.data(), count, s);
    N2W_CHECK(n2w_stream_sync(s));
    return v;
  }
  void zero(n2w_stream_t s = nullptr) { N2W_CHECK(n2w_memset(p, 0, std::max<size_t>(n, 1) * sizeof(T), s)); }
};

class Stream {
 public:
  n2w_stream_t s = nullptr;
  Stream() { N2W_CHECK(n2w_stream_create(&s)); }
  ~Stream() {
    if (s) n2w_stream_destroy(s);
  }
  void sync() { N2W_CHECK(n2w_stream_sync(s)); }
};

class Timer {
 public:
  n2w_timer* t = nullptr;
  Timer() { N2W_CHECK(n2w_timer_create(&t)); }
  ~Timer() { n2w_timer_destroy(t); }
  void start(n2w_stream_t s) { N2W_CHECK(n2w_timer_start(t, s)); }
  float stop_ms(n2w_stream_t s) {
    N2W_CHECK(n2w_timer_stop(t, s));
    float ms = 0;
    N2W_CHECK(n2w_timer_elapsed_ms(t, &ms));
    return ms;
  }
};

// Per-point FP64 accumulators on the device plus their host copies.
struct PointStats {
  DeviceArray<double> sum, sum_sq;
  DeviceArray<uint32_t> count;
  DeviceArray<uint64_t> steps;
  DeviceArray<uint32_t> forced;
  size_t n = 0;
  explicit PointStats(size_t points) : sum(points), sum_sq(points), count(points), steps(points), forced(points), n(points) {
    zero();
  }
  void zero(n2w_stream_t s = nullptr) {
    sum.zero(s);
    sum_sq.zero(s);
    count.zero(s);
    steps.zero(s);
    forced.zero(s);
  }
  n2w_point_stats view() { return n2w_point_stats{sum.p, sum_sq.p, count.p, steps.p, forced.p}; }

  struct Host {
    std::vector<double> sum, sum_sq;
    std::vector<uint32_t> count;
    std::vector<uint64_t> steps;
    std::vector<uint32_t> forced;
    double mean(size_t i) const { return count[i] ? sum[i] / count[i] : 0.0; }
    // Unbiased sample variance from (sum, sum of squares, n).
    double variance(size_t i) const {
      const double c = count[i];
      if (c < 2) return 0.0;
      const double m = sum[i] / c;
      return std::max(0.0, sum_sq[i] - c * m * m) / (c - 1.0);
    }
    double mean_steps(size_t i) const { return count[i] ? static_cast<double>(steps[i]) / count[i] : 0.0; }
  };
  Host to_host(n2w_stream_t s = nullptr) const {
    Host h;
    h.sum = sum.to_host(n, s);
    h.sum_sq = sum_sq.to_host(n, s);
    h.count = count.to_host(n, s);
    h.steps = steps.to_host(n, s);
    h.forced = forced.to_host(n, s);
    return h;
  }
};

// The reference tools' --block-size is a plain CUDA block size; the persistent
// walker takes a multiple of 32 in [32, 256].  Other values select its default.
inline int walker_block(int block_size) {
  return (block_size >= 32 && block_size <= 256 && block_size % 32 == 0) ? block_size : 0;
}

// Reference boundary-name normalisation (eval_tcnn_nc_wos.cu:147-162):
// lower case, '-', ' ', '.' -> '_', outer underscores trimmed.
inline std::string normalize_mode_text(const std::string& s) {
  std::string o;
  for (const char ch : s) {
    if (ch == '-' || ch == ' ' || ch == '.') o.push_back('_');
    else if (ch >= 'A' && ch <= 'Z') o.push_back(static_cast<char>(ch - 'A' + 'a'));
    else o.push_back(ch);
  }
  while (!o.empty() && o.front() == '_') o.erase(o.begin());
  while (!o.empty() && o.back() == '_') o.pop_back();
  return o;
}

// Runs a tool body; validation and runtime failures print "error: ..." and
// return 1, as the reference tools do.
template <typename F>
int run_main(F&& body) {
  try {
    return body();
  } catch (const std::exception& e) {
    std::cerr << "error: " << e.what() << "\n";
    return 1;
  }
}

}  // namespace tool
