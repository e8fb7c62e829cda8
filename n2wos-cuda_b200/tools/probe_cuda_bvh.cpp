// n2wos_probe_cuda_bvh: closest-point throughput of the device BVH on uniform
// query points, validated against the CPU brute force.
//
// Flags, JSON schema (n2wos_cuda_probe_bvh_v1) and exit codes follow the
// reference tool src/tools/probe_cuda_bvh.cpp:42-61 (flags), 239-316 (JSON),
// 386 (exit 2 when validation or overflow fails).  Query points come from
// std::mt19937 with uniform_real_distribution<float> in [-extent, extent]^3, as
// the reference generates them (124-132), so the same seed gives the same points.
#include <random>

#include "common.hpp"

namespace {

struct Options {
  tool::MeshOptions mesh;
  int leaf_size = 8;
  std::string build_method = "sah";
  int queries = 262144;
  int validate = 512;
  int repeat = 10;
  int block_size = 128;
  unsigned int seed = 12345;
  float query_extent = 1.35f;
  std::string output = "results/probe_cuda_bvh.json";
};

void usage(std::ostream& out, const char* argv0) {
  out << "Usage: " << argv0 << " [options]\n\n"
      << "Options:\n"
      << "  --mesh procedural_bumpy_sphere|obj|ply\n"
      << "  --mesh-path <path>                 Required when --mesh obj or ply\n"
      << "  --normalize 0|1                    Normalize a loaded mesh to centered unit radius [1]\n"
      << "  --bumpy-stacks <int>               Procedural sphere stacks [128]\n"
      << "  --bumpy-slices <int>               Procedural sphere slices [256]\n"
      << "  --bumpy-amplitude <float>          Procedural bump amplitude [0.15]\n"
      << "  --leaf-size <int>                  BVH leaf triangle count, 1..8 [8]\n"
      << "  --build-method sah|spatial_median  BVH builder [sah]\n"
      << "  --queries <int>                    Number of device query points [262144]\n"
      << "  --validate <int>                   Number of points checked by CPU brute force [512]\n"
      << "  --repeat <int>                     Repeated timed kernel launches [10]\n"
      << "  --block-size <int>                 CUDA block size [128]\n"
      << "  --seed <int>                       Host query generation seed [12345]\n"
      << "  --query-extent <float>             Uniform query cube half-width [1.35]\n"
      << "  --output <path>                    JSON output [results/probe_cuda_bvh.json]\n"
      << "  --help\n";
}

Options parse(int argc, char** argv) {
  Options o;
  for (int i = 1; i < argc; ++i) {
    const std::string a = argv[i];
    if (a == "--help" || a == "-h") {
      usage(std::cout, argv[0]);
      std::exit(0);
    } else if (o.mesh.parse(a, i, argc, argv)) {
    } else if (a == "--leaf-size") o.leaf_size = tool::parse_int(tool::require_value(i, argc, argv), a);
    else if (a == "--build-method") o.build_method = tool::require_value(i, argc, argv);
    else if (a == "--queries") o.queries = tool::parse_int(tool::require_value(i, argc, argv), a);
    else if (a == "--validate") o.validate = tool::parse_int(tool::require_value(i, argc, argv), a);
    else if (a == "--repeat") o.repeat = tool::parse_int(tool::require_value(i, argc, argv), a);
    else if (a == "--block-size") o.block_size = tool::parse_int(tool::require_value(i, argc, argv), a);
    else if (a == "--seed") o.seed = static_cast<unsigned>(tool::parse_u64(tool::require_value(i, argc, argv), a));
    else if (a == "--query-extent") o.query_extent = tool::parse_float(tool::require_value(i, argc, argv), a);
    else if (a == "--output") o.output = tool::require_value(i, argc, argv);
    else throw std::runtime_error("unknown option: " + a);
  }
  o.mesh.validate();
  if (o.queries <= 0) throw std::runtime_error("--queries must be positive");
  if (o.validate < 0) throw std::runtime_error("--validate must be non-negative");
  if (o.repeat <= 0) throw std::runtime_error("--repeat must be positive");
  if (o.leaf_size <= 0) throw std::runtime_error("--leaf-size must be positive");
  if (!(o.query_extent > 0.0f)) throw std::runtime_error("--query-extent must be positive");
  return o;
}

struct Validation {
  int checked = 0;
  int bad = 0;
  int id_mismatch = 0;
  float max_abs_distance_error = 0, rms_distance_error = 0;
  float max_closest_point_error = 0, rms_closest_point_error = 0;
};

Validation validate(const tool::Mesh& mesh, const std::vector<float>& pts, const std::vector<float>& d2,
                    const std::vector<float>& cp, const std::vector<int>& ids, int requested) {
  Validation v;
  v.checked = std::min<int>(requested, static_cast<int>(d2.size()));
  if (v.checked == 0) return v;
  std::vector<float> cd2(v.checked), ccp(3 * v.checked);
  std::vector<int> cid(v.checked);
  N2W_CHECK(n2w_mesh_closest_point_host(mesh.m, pts.data(), v.checked, cd2.data(), ccp.data(), cid.data(), 0));
  double sd = 0, sc = 0;
  for (int i = 0; i < v.checked; ++i) {
    const float dc = std::sqrt(std::max(cd2[i], 0.0f)), dg = std::sqrt(std::max(d2[i], 0.0f));
    const float e = std::fabs(dc - dg);
    const float ex = ccp[3 * i] - cp[3 * i], ey = ccp[3 * i + 1] - cp[3 * i + 1], ez = ccp[3 * i + 2] - cp[3 * i + 2];
    const float ce = std::sqrt(ex * ex + ey * ey + ez * ez);
    v.max_abs_distance_error = std::max(v.max_abs_distance_error, e);
    v.max_closest_point_error = std::max(v.max_closest_point_error, ce);
    sd += static_cast<double>(e) * e;
    sc += static_cast<double>(ce) * ce;
    if (e > 2.0e-4f) ++v.bad;
    if (cid[i] != ids[i]) ++v.id_mismatch;
  }
  v.rms_distance_error = static_cast<float>(std::sqrt(sd / v.checked));
  v.rms_closest_point_error = static_cast<float>(std::sqrt(sc / v.checked));
  return v;
}

}  // namespace

int main(int argc, char** argv) {
  return tool::run_main([&]() -> int {
    const Options o = parse(argc, argv);
    tool::Mesh mesh(o.mesh);
    std::cerr << "mesh: " << n2w_mesh_name(mesh.m) << " vertices=" << mesh.vertices()
              << " triangles=" << mesh.triangles() << "\n";
    tool::Bvh bvh(mesh, o.leaf_size, o.build_method);
    std::cerr << "BVH: nodes=" << bvh.stats.nodes << " max_depth=" << bvh.stats.max_depth << "\n";

    std::mt19937 rng(o.seed);
    std::uniform_real_distribution<float> uni(-o.query_extent, o.query_extent);
    std::vector<float> pts(3 * static_cast<size_t>(o.queries));
    for (int i = 0; i < o.queries; ++i) {
      pts[3 * i] = uni(rng);
      pts[3 * i + 1] = uni(rng);
      pts[3 * i + 2] = uni(rng);
    }
    const size_t n = o.queries;
    tool::Stream stream;
    tool::DeviceArray<n2w_vec3> d_pts(n), d_cp(n);
    tool::DeviceArray<float> d_d2(n);
    tool::DeviceArray<int> d_id(n), d_ov(n);
    d_pts.upload(reinterpret_cast<const n2w_vec3*>(pts.data()), n, stream.s);
    auto launch = [&] {
      N2W_CHECK(n2w_bvh_query_device(bvh.b, d_pts.p, o.queries, d_d2.p, d_cp.p, d_id.p, d_ov.p, o.block_size,
                                     stream.s));
    };
    launch();  // warm-up
    stream.sync();
    tool::Timer timer;
    std::vector<float> ms;
    for (int r = 0; r < o.repeat; ++r) {
      timer.start(stream.s);
      launch();
      ms.push_back(timer.stop_ms(stream.s));
      std::cerr << "repeat " << (r + 1) << "/" << o.repeat << ": kernel_ms=" << ms.back() << "\n";
    }
    const std::vector<float> d2 = d_d2.to_host(n, stream.s);
    std::vector<n2w_vec3> cpv = d_cp.to_host(n, stream.s);
    const std::vector<int> ids = d_id.to_host(n, stream.s), ov = d_ov.to_host(n, stream.s);
    std::vector<float> cp(3 * n);
    std::memcpy(cp.data(), cpv.data(), 12 * n);
    long long overflow = 0;
    for (const int v : ov) overflow += v ? 1 : 0;

    std::cerr << "validating " << std::min(o.validate, o.queries) << " points by CPU brute force...\n";
    const Validation v = validate(mesh, pts, d2, cp, ids, o.validate);

    const float med = tool::median(ms), avg = tool::mean(ms);
    const double med_us = static_cast<double>(med) * 1000.0 / o.queries;
    std::ostringstream j;
    j << "{\n"
      << "  \"schema\": \"n2wos_cuda_probe_bvh_v1\",\n"
      << "  \"patch\": \"n2w-sm100a-bvh-probe\",\n"
      << "  \"generated_at_utc\": " << tool::json_quote(tool::utc_now()) << ",\n"
      << "  \"command_line\": " << tool::json_quote(tool::join_argv(argc, argv)) << ",\n"
      << "  \"cuda\": " << tool::cuda_json() << ",\n"
      << "  \"implementation_mode\": {\n"
      << "    \"gpu_resident_geometry_query\": true,\n"
      << "    \"geometry_query\": \"n2w_sm100a_bvh\",\n"
      << "    \"bvh_layout\": \"4-wide SoA nodes (128 B), leaf-ordered float4 triangles (48 B)\",\n"
      << "    \"fcpw_gpu_public_api\": false,\n"
      << "    \"host_driven_walker_loop\": false,\n"
      << "    \"cache_inference\": \"none\",\n"
      << "    \"rng\": \"host_query_generation_only\",\n"
      << "    \"accumulation\": \"not_applicable\",\n"
      << "    \"timing_scope\": \"cuda_kernel_only_excludes_h2d_d2h_and_allocation\"\n"
      << "  },\n"
      << "  \"options\": {\n"
      << "    \"mesh\": " << tool::json_quote(o.mesh.mesh) << ",\n"
      << "    \"mesh_path\": " << tool::json_quote(o.mesh.mesh_path) << ",\n"
      << "    \"normalize\": " << o.mesh.normalize << ",\n"
      << "    \"bumpy_stacks\": " << o.mesh.bumpy_stacks << ",\n"
      << "    \"bumpy_slices\": " << o.mesh.bumpy_slices << ",\n"
      << "    \"bumpy_amplitude\": " << tool::num(o.mesh.bumpy_amplitude) << ",\n"
      << "    \"leaf_size\": " << o.leaf_size << ",\n"
      << "    \"build_method\": " << tool::json_quote(o.build_method) << ",\n"
      << "    \"queries\": " << o.queries << ",\n"
      << "    \"validate\": " << o.validate << ",\n"
      << "    \"repeat\": " << o.repeat << ",\n"
      << "    \"block_size\": " << o.block_size << ",\n"
      << "    \"seed\": " << o.seed << ",\n"
      << "    \"query_extent\": " << tool::num(o.query_extent) << "\n"
      << "  },\n"
      << "  \"mesh_stats\": " << tool::mesh_stats_json(mesh, n2w_mesh_name(mesh.m), false) << ",\n"
      << "  \"bvh_stats\": {\n"
      << "    \"nodes\": " << bvh.stats.nodes << ",\n"
      << "    \"triangle_indices\": " << bvh.stats.triangles << ",\n"
      << "    \"leaf_size\": " << bvh.stats.leaf_size << ",\n"
      << "    \"max_depth\": " << bvh.stats.max_depth << ",\n"
      << "    \"binary_nodes\": " << bvh.stats.binary_nodes << ",\n"
      << "    \"sah_cost\": " << tool::num(bvh.stats.sah_cost) << ",\n"
      << "    \"build_milliseconds\": " << tool::num(bvh.stats.build_milliseconds) << ",\n"
      << "    \"device_bytes\": " << bvh.stats.device_bytes << "\n"
      << "  },\n"
      << "  \"timing\": {\n"
      << "    \"kernel_ms\": " << tool::floats_json(ms) << ",\n"
      << "    \"kernel_ms_median\": " << tool::num(med) << ",\n"
      << "    \"kernel_ms_mean\": " << tool::num(avg) << ",\n"
      << "    \"median_us_per_query\": " << tool::num(med_us) << ",\n"
      << "    \"mean_us_per_query\": " << tool::num(static_cast<double>(avg) * 1000.0 / o.queries) << ",\n"
      << "    \"median_mqueries_per_second\": " << tool::num(o.queries / (static_cast<double>(med) * 1000.0)) << "\n"
      << "  },\n"
      << "  \"validation\": {\n"
      << "    \"checked\": " << v.checked << ",\n"
      << "    \"bad_distance_count_threshold_2e_4\": " << v.bad << ",\n"
      << "    \"triangle_id_mismatch_count\": " << v.id_mismatch << ",\n"
      << "    \"max_abs_distance_error\": " << tool::num(v.max_abs_distance_error) << ",\n"
      << "    \"rms_distance_error\": " << tool::num(v.rms_distance_error) << ",\n"
      << "    \"max_closest_point_error\": " << tool::num(v.max_closest_point_error) << ",\n"
      << "    \"rms_closest_point_error\": " << tool::num(v.rms_closest_point_error) << ",\n"
      << "    \"cuda_stack_overflow_count\": " << overflow << "\n"
      << "  }\n"
      << "}\n";
    tool::write_text(o.output, j.str());
    std::cout << "wrote " << o.output << "\n";
    std::cout << "median_us_per_query=" << med_us << " validation_max_abs_distance_error=" << v.max_abs_distance_error
              << " overflow=" << overflow << "\n";
    return v.bad == 0 && overflow == 0 ? 0 : 2;
  });
}
