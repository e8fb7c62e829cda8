// n2wos_probe_geometry_backends: closest-point stress probe over query
// distributions (uniform box, interior slice, exact surface, near-boundary
// shell, WoS-like mix) and a sweep of BVH builders and leaf sizes.
//
// Flags, query generators, JSON schema (n2wos_geometry_backend_probe_v2) and
// exit codes follow src/tools/probe_geometry_backends.cu: options 155-183,
// generators 295-395 (std::mt19937 streams consumed in the same order, so the
// same seed gives the same points), JSON 760-847, exit 1 when no backend
// built and 2 when validation or overflow failed (996-997).
//
// Backends here are this library's 4-wide BVH.  Builders it provides: "sah"
// (binned SAH) and "spatial_median" (the reference's in-tree median split).
// The reference's cuBQL-only builders ("radix", "elh") and leaf sizes above 8
// are reported as backends that did not build, with the reason.
#include <limits>
#include <random>

#include "common.hpp"

namespace {

struct Options {
  tool::MeshOptions mesh;
  int leaf_size = 8;
  std::vector<int> leaf_sizes = {8};
  std::vector<std::string> build_methods = {"spatial_median", "radix", "sah", "elh"};
  int queries = 262144;
  int validate = 2048;
  int repeat = 10;
  int block_size = 128;
  unsigned int seed = 12345;
  float query_extent = 1.35f;
  std::string query_mode = "uniform_box";
  float shell_min = 1.0e-4f;
  float shell_max = 2.5e-1f;
  float plane_z = 0.0f;
  int run_custom = 1;
  int run_cubql = 1;
  std::string output = "results/probe_geometry_backends.json";
};

std::string trim(const std::string& s) {
  const size_t a = s.find_first_not_of(" \t\n\r");
  if (a == std::string::npos) return "";
  return s.substr(a, s.find_last_not_of(" \t\n\r") - a + 1);
}

// Builder aliases of the reference (probe_geometry_backends.cu:84-95).
std::string canonical_method(std::string m) {
  m = trim(m);
  if (m == "sm" || m == "spatial-median") return "spatial_median";
  if (m == "surface_area_heuristic") return "sah";
  if (m == "morton" || m == "radix_morton") return "radix";
  if (m == "rebin" || m == "robust_radix" || m == "modified_radix" || m == "rebin_radix" || m == "rebin-radix") {
    throw std::runtime_error("build method rebin_radix is disabled");
  }
  return m;
}

std::vector<std::string> parse_methods(const std::string& text) {
  std::vector<std::string> out;
  for (const std::string& item : tool::parse_str_list(text)) {
    const std::string t = trim(item);
    if (t == "sweep" || t == "all") {
      out.insert(out.end(), {"spatial_median", "radix", "sah", "elh"});
    } else if (!t.empty()) {
      out.push_back(canonical_method(t));
    }
  }
  return out;
}

std::string canonical_query_mode(std::string m) {
  m = trim(m);
  if (m == "plane_slice") return "interior_slice";
  if (m == "near_surface_shell") return "near_boundary_shell";
  if (m == "mixed_wos_like") return "wos_like_prefix";
  return m;
}

void usage(std::ostream& out, const char* argv0) {
  out << "Usage: " << argv0 << " [options]\n\n"
      << "Options:\n"
      << "  --mesh procedural_bumpy_sphere|obj|ply\n"
      << "  --mesh-path <path>                 Required when --mesh obj or ply\n"
      << "  --normalize 0|1                    Normalize a loaded mesh to centered unit radius [1]\n"
      << "  --bumpy-stacks <int>               Procedural sphere stacks [128]\n"
      << "  --bumpy-slices <int>               Procedural sphere slices [256]\n"
      << "  --bumpy-amplitude <float>          Procedural bump amplitude [0.15]\n"
      << "  --leaf-size <int>                  Leaf size of the median-split comparison BVH [8]\n"
      << "  --cubql-leaf-sizes <csv>           Leaf sizes of the builder sweep, e.g. 1,4,8 [8]\n"
      << "  --queries <int>                    Number of device-resident query points [262144]\n"
      << "  --validate <int>                   Number of points checked by CPU brute force [2048]\n"
      << "  --repeat <int>                     Repeated timed device-query launches [10]\n"
      << "  --block-size <int>                 CUDA block size [128]\n"
      << "  --seed <int>                       Host query generation seed [12345]\n"
      << "  --query-extent <float>             Uniform cube/slice half-width [1.35]\n"
      << "  --query-mode <mode>                uniform_box|interior_slice|surface_exact|near_boundary_shell|wos_like_prefix [uniform_box]\n"
      << "  --shell-min <float>                near_boundary_shell minimum offset [1e-4]\n"
      << "  --shell-max <float>                near_boundary_shell maximum offset [0.25]\n"
      << "  --plane-z <float>                  z coordinate for interior_slice [0]\n"
      << "  --cubql-build-method <name>        Single builder of the sweep\n"
      << "  --cubql-build-methods <csv>        spatial_median,radix,sah,elh or sweep/all [spatial_median,radix,sah,elh]\n"
      << "  --run-custom 0|1                   Run the median-split comparison backend [1]\n"
      << "  --run-cubql 0|1                    Run the builder sweep [1]\n"
      << "  --output <path>                    JSON output [results/probe_geometry_backends.json]\n"
      << "  --help\n";
}

Options parse(int argc, char** argv) {
  Options o;
  for (int i = 1; i < argc; ++i) {
    const std::string a = argv[i];
    auto val = [&] { return tool::require_value(i, argc, argv); };
    if (a == "--help" || a == "-h") {
      usage(std::cout, argv[0]);
      std::exit(0);
    } else if (o.mesh.parse(a, i, argc, argv)) {
    } else if (a == "--leaf-size") o.leaf_size = tool::parse_int(val(), a);
    else if (a == "--cubql-leaf-sizes") o.leaf_sizes = tool::parse_int_list(val(), a);
    else if (a == "--queries") o.queries = tool::parse_int(val(), a);
    else if (a == "--validate") o.validate = tool::parse_int(val(), a);
    else if (a == "--repeat") o.repeat = tool::parse_int(val(), a);
    else if (a == "--block-size") o.block_size = tool::parse_int(val(), a);
    else if (a == "--seed") o.seed = static_cast<unsigned>(tool::parse_u64(val(), a));
    else if (a == "--query-extent") o.query_extent = tool::parse_float(val(), a);
    else if (a == "--query-mode") o.query_mode = canonical_query_mode(val());
    else if (a == "--shell-min") o.shell_min = tool::parse_float(val(), a);
    else if (a == "--shell-max") o.shell_max = tool::parse_float(val(), a);
    else if (a == "--plane-z") o.plane_z = tool::parse_float(val(), a);
    else if (a == "--cubql-build-method") o.build_methods = {canonical_method(val())};
    else if (a == "--cubql-build-methods") o.build_methods = parse_methods(val());
    else if (a == "--run-custom") o.run_custom = tool::parse_int(val(), a);
    else if (a == "--run-cubql") o.run_cubql = tool::parse_int(val(), a);
    else if (a == "--output") o.output = val();
    else throw std::runtime_error("unknown option: " + a);
  }
  o.mesh.validate();
  if (o.build_methods.empty()) throw std::runtime_error("--cubql-build-methods cannot be empty");
  for (const auto& m : o.build_methods) {
    if (m != "spatial_median" && m != "sah" && m != "elh" && m != "radix") {
      throw std::runtime_error("build method must be one of: spatial_median, sah, elh, radix");
    }
  }
  for (const int l : o.leaf_sizes) {
    if (l <= 0) throw std::runtime_error("--cubql-leaf-sizes entries must be positive");
  }
  const std::string& q = o.query_mode;
  if (q != "uniform_box" && q != "interior_slice" && q != "surface_exact" && q != "near_boundary_shell" &&
      q != "wos_like_prefix") {
    throw std::runtime_error(
        "--query-mode must be uniform_box, interior_slice, surface_exact, near_boundary_shell, or wos_like_prefix");
  }
  if (o.queries <= 0) throw std::runtime_error("--queries must be positive");
  if (o.validate < 0) throw std::runtime_error("--validate must be non-negative");
  if (o.repeat <= 0) throw std::runtime_error("--repeat must be positive");
  if (o.leaf_size <= 0) throw std::runtime_error("--leaf-size must be positive");
  if (!(o.query_extent > 0.0f)) throw std::runtime_error("--query-extent must be positive");
  if (!(o.shell_min >= 0.0f) || !(o.shell_max >= o.shell_min)) {
    throw std::runtime_error("require 0 <= --shell-min <= --shell-max");
  }
  return o;
}

// ---- query point generators --------------------------------------------------

using P3 = std::array<float, 3>;

std::vector<P3> uniform_box(int n, unsigned seed, float extent) {
  std::mt19937 rng(seed);
  std::uniform_real_distribution<float> u(-extent, extent);
  std::vector<P3> pts(n);
  for (auto& p : pts) {
    const float x = u(rng), y = u(rng), z = u(rng);
    p = {x, y, z};
  }
  return pts;
}

std::vector<P3> plane_slice(int n, unsigned seed, float extent, float z) {
  std::mt19937 rng(seed);
  std::uniform_real_distribution<float> u(-extent, extent);
  std::vector<P3> pts(n);
  for (auto& p : pts) {
    const float x = u(rng), y = u(rng);
    p = {x, y, z};
  }
  return pts;
}

// Area-weighted surface points pushed along the face normal by a log-uniform
// offset in [shell_min, shell_max] with a random sign (zero_offset: on the surface).
std::vector<P3> surface_shell(const std::vector<float>& V, const std::vector<uint32_t>& T, int n, unsigned seed,
                              float shell_min, float shell_max, bool zero_offset) {
  const size_t nt = T.size() / 3;
  auto vert = [&](uint32_t k) { return P3{V[3 * k], V[3 * k + 1], V[3 * k + 2]}; };
  auto sub = [](const P3& a, const P3& b) { return P3{a[0] - b[0], a[1] - b[1], a[2] - b[2]}; };
  auto cross = [](const P3& a, const P3& b) {
    return P3{a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]};
  };
  auto len = [](const P3& a) { return std::sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]); };
  std::mt19937 rng(seed);
  std::vector<double> w(nt);
  for (size_t t = 0; t < nt; ++t) {
    const P3 a = vert(T[3 * t]), b = vert(T[3 * t + 1]), c = vert(T[3 * t + 2]);
    w[t] = std::max<double>(0.5f * len(cross(sub(b, a), sub(c, a))), 1.0e-30);
  }
  std::discrete_distribution<size_t> pick(w.begin(), w.end());
  std::uniform_real_distribution<float> unit(0.0f, 1.0f);
  const float min_pos = std::max(shell_min, 1.0e-8f);
  const bool log_sample = shell_max > min_pos;
  std::vector<P3> pts(n);
  for (auto& p : pts) {
    const size_t t = pick(rng);
    const P3 a = vert(T[3 * t]), b = vert(T[3 * t + 1]), c = vert(T[3 * t + 2]);
    const float su = std::sqrt(unit(rng));
    const float v = unit(rng);
    const float wa = 1.0f - su, wb = su * (1.0f - v), wc = su * v;
    P3 q;
    for (int k = 0; k < 3; ++k) q[k] = (a[k] * wa + b[k] * wb) + c[k] * wc;
    P3 nrm = cross(sub(b, a), sub(c, a));
    const float l = len(nrm);
    if (l > 0.0f) {
      for (float& x : nrm) x = x / l;
    } else {
      nrm = {1.0f, 0.0f, 0.0f};
    }
    float off = 0.0f;
    if (!zero_offset) {
      if (log_sample) {
        const float s = unit(rng);
        off = min_pos * std::exp(std::log(shell_max / min_pos) * s);
      } else {
        off = shell_max;
      }
      if (unit(rng) < 0.5f) off = -off;
    }
    for (int k = 0; k < 3; ++k) p[k] = q[k] + nrm[k] * off;
  }
  return pts;
}

std::vector<P3> make_points(const Options& o, const tool::Mesh& mesh) {
  if (o.query_mode == "uniform_box") return uniform_box(o.queries, o.seed, o.query_extent);
  if (o.query_mode == "interior_slice") return plane_slice(o.queries, o.seed, o.query_extent, o.plane_z);
  std::vector<float> V(3 * mesh.vertices());
  std::vector<uint32_t> T(3 * mesh.triangles());
  N2W_CHECK(n2w_mesh_copy_out(mesh.m, V.data(), T.data()));
  if (o.query_mode == "surface_exact") return surface_shell(V, T, o.queries, o.seed, 0.0f, 0.0f, true);
  std::vector<P3> shell = surface_shell(V, T, o.queries, o.seed, o.shell_min, o.shell_max, false);
  if (o.query_mode == "near_boundary_shell") return shell;
  // wos_like_prefix: every fourth point from the plane slice, the rest from the shell.
  const std::vector<P3> slice = plane_slice(o.queries, o.seed ^ 0x9e3779b9u, o.query_extent, o.plane_z);
  for (int i = 0; i < o.queries; i += 4) shell[i] = slice[i];
  return shell;
}

// ---- backends -------------------------------------------------------------------

struct Run {
  std::string name, builder, error;
  bool enabled = true, built = false, production_candidate = false;
  n2w_bvh_stats stats{};
  int leaf_size = 0;
  std::vector<float> ms;
  std::vector<float> d2, cp;
  std::vector<int> ids;
  long long overflow = 0;
  int checked = 0, bad = 0, id_disagree = 0;
  float max_err = 0, rms_err = 0, max_cp_err = 0, rms_cp_err = 0, max_backend_delta = 0;
  bool passed() const { return enabled && built && bad == 0 && overflow == 0 && !ms.empty(); }
  double median_us(int queries) const {
    return ms.empty() ? std::numeric_limits<double>::infinity() : tool::median(ms) * 1000.0 / queries;
  }
};

struct Reference {
  std::vector<float> d2, cp;
  std::vector<int> ids;
};

void run_backend(Run& r, const tool::Mesh& mesh, const Options& o, const std::string& method, int leaf,
                 tool::DeviceArray<n2w_vec3>& d_pts, tool::Stream& stream, const Reference& cpu,
                 const Run* comparison) {
  r.leaf_size = leaf;
  try {
    if (method != "sah" && method != "spatial_median") {
      throw std::runtime_error("build method '" + method + "' is a cuBQL builder that this library does not provide");
    }
    tool::Bvh bvh(mesh, leaf, method);
    r.stats = bvh.stats;
    r.built = true;
    const size_t n = o.queries;
    tool::DeviceArray<n2w_vec3> d_cp(n);
    tool::DeviceArray<float> d_d2(n);
    tool::DeviceArray<int> d_id(n), d_ov(n);
    auto launch = [&] {
      N2W_CHECK(n2w_bvh_query_device(bvh.b, d_pts.p, o.queries, d_d2.p, d_cp.p, d_id.p, d_ov.p, o.block_size,
                                     stream.s));
    };
    launch();
    stream.sync();
    tool::Timer timer;
    for (int k = 0; k < o.repeat; ++k) {
      timer.start(stream.s);
      launch();
      r.ms.push_back(timer.stop_ms(stream.s));
      std::cerr << r.name << " repeat " << (k + 1) << "/" << o.repeat << ": kernel_ms=" << r.ms.back() << "\n";
    }
    r.d2 = d_d2.to_host(n, stream.s);
    const std::vector<n2w_vec3> cpv = d_cp.to_host(n, stream.s);
    r.cp.resize(3 * n);
    std::memcpy(r.cp.data(), cpv.data(), 12 * n);
    r.ids = d_id.to_host(n, stream.s);
    for (const int v : d_ov.to_host(n, stream.s)) r.overflow += v ? 1 : 0;
  } catch (const std::exception& e) {
    r.error = e.what();
    std::cerr << "backend failed: " << r.name << ": " << e.what() << "\n";
    return;
  }
  r.checked = static_cast<int>(cpu.d2.size());
  double sd = 0, sc = 0;
  for (int i = 0; i < r.checked; ++i) {
    const float dc = std::sqrt(std::max(cpu.d2[i], 0.0f)), dg = std::sqrt(std::max(r.d2[i], 0.0f));
    const float e = std::fabs(dc - dg);
    const float ex = cpu.cp[3 * i] - r.cp[3 * i], ey = cpu.cp[3 * i + 1] - r.cp[3 * i + 1],
                ez = cpu.cp[3 * i + 2] - r.cp[3 * i + 2];
    const float ce = std::sqrt(ex * ex + ey * ey + ez * ez);
    r.max_err = std::max(r.max_err, e);
    r.max_cp_err = std::max(r.max_cp_err, ce);
    sd += static_cast<double>(e) * e;
    sc += static_cast<double>(ce) * ce;
    if (e > 2.0e-4f) ++r.bad;
    if (cpu.ids[i] != r.ids[i]) ++r.id_disagree;
    if (comparison && comparison->built) {
      const float od = std::sqrt(std::max(comparison->d2[i], 0.0f));
      r.max_backend_delta = std::max(r.max_backend_delta, std::fabs(od - dg));
    }
  }
  if (r.checked) {
    r.rms_err = static_cast<float>(std::sqrt(sd / r.checked));
    r.rms_cp_err = static_cast<float>(std::sqrt(sc / r.checked));
  }
}

std::string backend_json(const Run& r, int queries) {
  std::ostringstream o;
  o << "    " << tool::json_quote(r.name) << ": {\n"
    << "      \"enabled\": " << (r.enabled ? "true" : "false") << ",\n"
    << "      \"built\": " << (r.built ? "true" : "false") << ",\n"
    << "      \"builder\": " << tool::json_quote(r.builder) << ",\n";
  if (!r.error.empty()) o << "      \"error\": " << tool::json_quote(r.error) << ",\n";
  o << "      \"production_candidate\": " << (r.production_candidate ? "true" : "false") << ",\n"
    << "      \"device_resident_query_api\": true,\n"
    << "      \"host_transfer_in_timing\": false,\n"
    << "      \"bvh_stats\": {\n"
    << "        \"triangles\": " << r.stats.triangles << ",\n"
    << "        \"nodes\": " << r.stats.nodes << ",\n"
    << "        \"prim_ids\": " << r.stats.triangles << ",\n"
    << "        \"leaf_size\": " << r.leaf_size << ",\n"
    << "        \"max_depth\": " << r.stats.max_depth << ",\n"
    << "        \"sah_cost\": " << tool::num(r.stats.sah_cost) << ",\n"
    << "        \"build_milliseconds\": " << tool::num(r.stats.build_milliseconds) << "\n"
    << "      },\n";
  const float med = tool::median(r.ms), avg = tool::mean(r.ms);
  o << "      \"timing\": {\n"
    << "        \"kernel_ms\": " << tool::floats_json(r.ms) << ",\n"
    << "        \"kernel_ms_median\": " << tool::num(med) << ",\n"
    << "        \"kernel_ms_mean\": " << tool::num(avg) << ",\n"
    << "        \"median_us_per_query\": " << tool::num(r.ms.empty() ? 0.0 : med * 1000.0 / queries) << ",\n"
    << "        \"mean_us_per_query\": " << tool::num(r.ms.empty() ? 0.0 : avg * 1000.0 / queries) << ",\n"
    << "        \"median_mqueries_per_second\": " << tool::num(r.ms.empty() ? 0.0 : queries / (med * 1000.0)) << "\n"
    << "      },\n"
    << "      \"validation\": {\n"
    << "        \"checked\": " << r.checked << ",\n"
    << "        \"bad_distance_count_threshold_2e_4\": " << r.bad << ",\n"
    << "        \"max_abs_distance_error\": " << tool::num(r.max_err) << ",\n"
    << "        \"rms_distance_error\": " << tool::num(r.rms_err) << ",\n"
    << "        \"max_closest_point_error\": " << tool::num(r.max_cp_err) << ",\n"
    << "        \"rms_closest_point_error\": " << tool::num(r.rms_cp_err) << ",\n"
    << "        \"max_backend_distance_delta\": " << tool::num(r.max_backend_delta) << ",\n"
    << "        \"triangle_id_disagreement_count\": " << r.id_disagree << "\n"
    << "      },\n"
    << "      \"validation_passed\": " << (r.passed() ? "true" : "false") << ",\n"
    << "      \"overflow_count\": " << r.overflow << "\n"
    << "    }";
  return o.str();
}

const Run* fastest(const std::vector<Run>& runs, int queries, bool production_only) {
  const Run* best = nullptr;
  double best_us = std::numeric_limits<double>::infinity();
  for (const Run& r : runs) {
    if (!r.passed() || (production_only && !r.production_candidate)) continue;
    if (r.median_us(queries) < best_us) {
      best_us = r.median_us(queries);
      best = &r;
    }
  }
  return best;
}

std::string str_array(const std::vector<std::string>& v) {
  std::string o = "[";
  for (size_t i = 0; i < v.size(); ++i) o += (i ? ", " : "") + tool::json_quote(v[i]);
  return o + "]";
}

std::string int_array(const std::vector<int>& v) {
  std::string o = "[";
  for (size_t i = 0; i < v.size(); ++i) o += (i ? ", " : "") + std::to_string(v[i]);
  return o + "]";
}

}  // namespace

int main(int argc, char** argv) {
  return tool::run_main([&]() -> int {
    const Options o = parse(argc, argv);
    tool::Mesh mesh(o.mesh);
    const std::vector<P3> pts = make_points(o, mesh);
    std::cerr << "mesh: " << n2w_mesh_name(mesh.m) << " vertices=" << mesh.vertices()
              << " triangles=" << mesh.triangles() << "\n"
              << "query_mode=" << o.query_mode
              << " query points uploaded once; timed queries do not include H2D/D2H transfers\n";
    tool::Stream stream;
    tool::DeviceArray<n2w_vec3> d_pts(pts.size());
    d_pts.upload(reinterpret_cast<const n2w_vec3*>(pts.data()), pts.size(), stream.s);

    Reference cpu;
    const int nval = std::min(o.validate, o.queries);
    cpu.d2.resize(nval);
    cpu.cp.resize(3 * static_cast<size_t>(nval));
    cpu.ids.resize(nval);
    if (nval > 0) {
      N2W_CHECK(n2w_mesh_closest_point_host(mesh.m, reinterpret_cast<const float*>(pts.data()), nval, cpu.d2.data(),
                                            cpu.cp.data(), cpu.ids.data(), 0));
    }

    std::vector<Run> runs;
    runs.reserve(1 + o.leaf_sizes.size() * o.build_methods.size());
    if (o.run_custom) {
      Run r;
      r.name = "n2w_median_bvh_leaf" + std::to_string(o.leaf_size);
      r.builder = "in_tree_cpu_largest_axis_centroid_median_split";
      r.production_candidate = false;
      run_backend(r, mesh, o, "spatial_median", o.leaf_size, d_pts, stream, cpu, nullptr);
      runs.push_back(std::move(r));
    }
    const Run* comparison = o.run_custom && !runs.empty() ? &runs.front() : nullptr;
    if (o.run_cubql) {
      for (const int leaf : o.leaf_sizes) {
        for (const std::string& m : o.build_methods) {
          Run r;
          r.name = "n2w_sm100a_bvh_" + m + "_leaf" + std::to_string(leaf);
          r.builder = m == "sah" ? "n2w_binned_sah_4wide" : (m == "spatial_median" ? "n2w_median_split_4wide" : m);
          r.production_candidate = true;
          run_backend(r, mesh, o, m, leaf, d_pts, stream, cpu, comparison);
          if (!r.built) r.production_candidate = false;
          runs.push_back(std::move(r));
          comparison = o.run_custom ? &runs.front() : nullptr;
        }
      }
    }

    const Run* best_prod = fastest(runs, o.queries, true);
    const Run* best_all = fastest(runs, o.queries, false);
    std::ostringstream j;
    j << "{\n"
      << "  \"schema\": \"n2wos_geometry_backend_probe_v2\",\n"
      << "  \"patch\": \"n2w-sm100a-geometry-backend-probe\",\n"
      << "  \"generated_at_utc\": " << tool::json_quote(tool::utc_now()) << ",\n"
      << "  \"command_line\": " << tool::json_quote(tool::join_argv(argc, argv)) << ",\n"
      << "  \"cuda\": " << tool::cuda_json() << ",\n"
      << "  \"backend_policy\": {\n"
      << "    \"production_requires_gpu_resident_geometry_query\": true,\n"
      << "    \"production_forbids_per_step_host_transfer\": true,\n"
      << "    \"production_forbids_fcpw_public_host_vector_loop\": true,\n"
      << "    \"probe_timing_scope\": \"device_query_kernel_only_excludes_query_upload_result_readback; build time is separately reported\",\n"
      << "    \"median_split_bvh_role\": \"comparison_only\",\n"
      << "    \"n2w_sm100a_bvh_role\": \"production_candidate_when_it_builds_and_validates\"\n"
      << "  },\n"
      << "  \"options\": {\n"
      << "    \"mesh\": " << tool::json_quote(o.mesh.mesh) << ",\n"
      << "    \"mesh_path\": " << tool::json_quote(o.mesh.mesh_path) << ",\n"
      << "    \"normalize\": " << o.mesh.normalize << ",\n"
      << "    \"bumpy_stacks\": " << o.mesh.bumpy_stacks << ",\n"
      << "    \"bumpy_slices\": " << o.mesh.bumpy_slices << ",\n"
      << "    \"bumpy_amplitude\": " << tool::num(o.mesh.bumpy_amplitude) << ",\n"
      << "    \"leaf_size\": " << o.leaf_size << ",\n"
      << "    \"cubql_leaf_sizes\": " << int_array(o.leaf_sizes) << ",\n"
      << "    \"queries\": " << o.queries << ",\n"
      << "    \"validate\": " << o.validate << ",\n"
      << "    \"repeat\": " << o.repeat << ",\n"
      << "    \"block_size\": " << o.block_size << ",\n"
      << "    \"seed\": " << o.seed << ",\n"
      << "    \"query_extent\": " << tool::num(o.query_extent) << ",\n"
      << "    \"query_mode\": " << tool::json_quote(o.query_mode) << ",\n"
      << "    \"shell_min\": " << tool::num(o.shell_min) << ",\n"
      << "    \"shell_max\": " << tool::num(o.shell_max) << ",\n"
      << "    \"plane_z\": " << tool::num(o.plane_z) << ",\n"
      << "    \"cubql_build_methods\": " << str_array(o.build_methods) << "\n"
      << "  },\n"
      << "  \"mesh_stats\": " << tool::mesh_stats_json(mesh, n2w_mesh_name(mesh.m), false) << ",\n"
      << "  \"build_features\": {\n"
      << "    \"N2WOS_HAS_CUBQL\": false,\n"
      << "    \"n2w_sm100a_bvh\": true\n"
      << "  },\n"
      << "  \"recommendation\": {\n"
      << "    \"selection_policy\": \"fastest validated device-resident production candidate for the tested mesh/query mode\",\n"
      << "    \"selected_production_candidate\": " << (best_prod ? tool::json_quote(best_prod->name) : "null") << ",\n"
      << "    \"selected_median_us_per_query\": " << (best_prod ? tool::num(best_prod->median_us(o.queries)) : "null")
      << ",\n"
      << "    \"fastest_validated_overall\": " << (best_all ? tool::json_quote(best_all->name) : "null") << ",\n"
      << "    \"fastest_validated_overall_median_us_per_query\": "
      << (best_all ? tool::num(best_all->median_us(o.queries)) : "null") << ",\n"
      << "    \"median_split_bvh_excluded_from_production_selection\": true\n"
      << "  },\n"
      << "  \"backends\": {\n";
    bool first = true;
    for (const Run& r : runs) {
      j << (first ? "" : ",\n") << backend_json(r, o.queries);
      first = false;
    }
    if (!o.run_cubql) {
      j << (first ? "" : ",\n") << "    \"n2w_sm100a_bvh\": {\n      \"enabled\": false,\n      \"built\": false,\n"
        << "      \"reason\": \"disabled by --run-cubql 0\",\n      \"production_candidate\": false,\n"
        << "      \"device_resident_query_api\": true,\n      \"host_transfer_in_timing\": false\n    }";
    }
    j << "\n  }\n}\n";
    tool::write_text(o.output, j.str());

    int built = 0;
    long long bad = 0, overflow = 0;
    for (const Run& r : runs) {
      if (!r.built) continue;
      ++built;
      bad += r.bad;
      overflow += r.overflow;
      std::cout << r.name << " median_us_per_query=" << r.median_us(o.queries)
                << " build_ms=" << r.stats.build_milliseconds << " validation_max_abs_distance_error=" << r.max_err
                << " overflow=" << r.overflow << "\n";
    }
    if (best_prod) {
      std::cout << "selected_production_candidate=" << best_prod->name
                << " median_us_per_query=" << best_prod->median_us(o.queries) << "\n";
    }
    std::cout << "wrote " << o.output << "\n";
    if (built == 0) return 1;
    return bad == 0 && overflow == 0 ? 0 : 2;
  });
}
