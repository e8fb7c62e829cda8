// n2wos_eval_wavefront_wos: single-point harmonic estimator check for
// u = x^2 - y^2 at x0 with plain WoS and the analytic-cache two-level levels.
//
// Flags, methods, JSON schema (n2wos_wavefront_wos_eval_v1) and the estimator
// algebra follow src/tools/eval_wavefront_wos.cu: options 96-114, methods
// 268-302 (oracle_2lmc = coarse with `samples` walks + residual with
// max(1, samples/8) walks and seed ^ 0x517cc1b727220a95), per-run fields
// 206-226, JSON 320-395.  The "analytic oracle" cache is the exact solution
// C(x) = u(x) (src/cuda/wos_wavefront.cu:140-149).
//
// Both --engine values run this library's persistent walker (one launch per
// level; lanes take new walks from a queue as theirs finish); the flag is
// recorded but does not switch implementations.
#include "common.hpp"

namespace {

struct Options {
  tool::MeshOptions mesh;
  std::string method = "pure_wos";
  std::string engine = "wavefront";
  int samples = 65536;
  int coarse_samples = 0;
  int residual_samples = 0;
  int depth_m = 8;
  int max_steps = 256;
  float epsilon = 1.0e-4f;
  float step_scale = 0.999f;
  float x0[3] = {0.1f, 0.05f, 0.0f};
  uint64_t seed = 12345;
  int block_size = 128;
  int leaf_size = 8;
  std::string build_method = "sah";
  std::string output = "results/eval_wavefront_wos.json";
};

void usage(const char* argv0) {
  std::cerr << "usage: " << argv0 << " [options]\n"
            << "  --mesh procedural_bumpy_sphere|obj|ply\n"
            << "  --mesh-path PATH\n"
            << "  --normalize 0|1 --bumpy-stacks N --bumpy-slices N --bumpy-amplitude A\n"
            << "  --method pure_wos|oracle_coarse|oracle_residual|oracle_2lmc\n"
            << "  --engine wavefront|persistent   both run the persistent queue walker\n"
            << "  --samples N\n"
            << "  --coarse-samples N       for oracle_2lmc; default samples\n"
            << "  --residual-samples N     for oracle_2lmc; default max(1, samples/8)\n"
            << "  --depth-m M\n"
            << "  --max-steps N\n"
            << "  --epsilon EPS\n"
            << "  --step-scale S\n"
            << "  --x0 x,y,z\n"
            << "  --seed N\n"
            << "  --block-size N           walker threads per block\n"
            << "  --cubql-build-method sah|spatial_median\n"
            << "  --cubql-leaf-size N      1..8\n"
            << "  --output PATH\n";
}

Options parse(int argc, char** argv) {
  Options o;
  for (int i = 1; i < argc; ++i) {
    const std::string a = argv[i];
    auto val = [&] { return tool::require_value(i, argc, argv); };
    if (a == "--help" || a == "-h") {
      usage(argv[0]);
      std::exit(0);
    } else if (o.mesh.parse(a, i, argc, argv)) {
    } else if (a == "--method") o.method = val();
    else if (a == "--engine") o.engine = val();
    else if (a == "--samples") o.samples = tool::parse_int(val(), a);
    else if (a == "--coarse-samples") o.coarse_samples = tool::parse_int(val(), a);
    else if (a == "--residual-samples") o.residual_samples = tool::parse_int(val(), a);
    else if (a == "--depth-m") o.depth_m = tool::parse_int(val(), a);
    else if (a == "--max-steps") o.max_steps = tool::parse_int(val(), a);
    else if (a == "--epsilon") o.epsilon = tool::parse_float(val(), a);
    else if (a == "--step-scale") o.step_scale = tool::parse_float(val(), a);
    else if (a == "--x0") {
      const auto v = tool::parse_float_list(val(), 3, "--x0");
      o.x0[0] = v[0];
      o.x0[1] = v[1];
      o.x0[2] = v[2];
    } else if (a == "--seed") o.seed = tool::parse_u64(val(), a);
    else if (a == "--block-size") o.block_size = tool::parse_int(val(), a);
    else if (a == "--cubql-leaf-size") o.leaf_size = tool::parse_int(val(), a);
    else if (a == "--cubql-build-method") o.build_method = val();
    else if (a == "--output") o.output = val();
    else throw std::runtime_error("unknown argument: " + a);
  }
  o.mesh.validate();
  if (o.method != "pure_wos" && o.method != "oracle_coarse" && o.method != "oracle_residual" &&
      o.method != "oracle_2lmc") {
    throw std::runtime_error("--method must be pure_wos, oracle_coarse, oracle_residual, or oracle_2lmc");
  }
  if (o.engine != "wavefront" && o.engine != "persistent") {
    throw std::runtime_error("--engine must be wavefront or persistent");
  }
  if (o.samples <= 0 || o.max_steps <= 0 || o.block_size <= 0) {
    throw std::runtime_error("samples, max-steps, and block-size must be positive");
  }
  if (o.depth_m < 0) throw std::runtime_error("depth_m must be non-negative");
  return o;
}

struct RunStats {
  int samples = 0;
  double mean = 0, sample_variance = 0, estimator_variance = 0, stderr_ = 0, mean_steps = 0;
  float elapsed_ms = 0;
  unsigned long long queries = 0, forced = 0, overflow = 0;
};

RunStats finish(const tool::PointStats& st, int samples, float ms, unsigned long long queries,
                unsigned long long forced, unsigned long long overflow) {
  const auto h = st.to_host();
  RunStats s;
  s.samples = samples;
  s.mean = h.mean(0);
  s.sample_variance = h.variance(0);
  s.estimator_variance = s.sample_variance / samples;
  s.stderr_ = std::sqrt(s.estimator_variance);
  s.mean_steps = h.mean_steps(0);
  s.elapsed_ms = ms;
  s.queries = queries;
  s.forced = forced;
  s.overflow = overflow;
  return s;
}

std::string run_json(const std::string& name, const RunStats& s, double exact) {
  const double err = s.mean - exact;
  std::ostringstream o;
  o << "    " << tool::json_quote(name) << ": {\n"
    << "      \"samples\": " << s.samples << ",\n"
    << "      \"mean\": " << tool::num(s.mean) << ",\n"
    << "      \"exact_target\": " << tool::num(exact) << ",\n"
    << "      \"error\": " << tool::num(err) << ",\n"
    << "      \"abs_error\": " << tool::num(std::fabs(err)) << ",\n"
    << "      \"sample_variance\": " << tool::num(s.sample_variance) << ",\n"
    << "      \"estimator_variance\": " << tool::num(s.estimator_variance) << ",\n"
    << "      \"stderr\": " << tool::num(s.stderr_) << ",\n"
    << "      \"mean_steps\": " << tool::num(s.mean_steps) << ",\n"
    << "      \"elapsed_ms\": " << tool::num(s.elapsed_ms) << ",\n"
    << "      \"us_per_sample\": " << tool::num(1000.0 * s.elapsed_ms / s.samples) << ",\n"
    << "      \"launched_query_slots\": " << s.queries << ",\n"
    << "      \"mean_launched_query_slots_per_sample\": " << tool::num(static_cast<double>(s.queries) / s.samples)
    << ",\n"
    << "      \"scheduled_query_rounds\": 1,\n"
    << "      \"forced_max_steps\": " << s.forced << ",\n"
    << "      \"overflow_count\": " << s.overflow << "\n"
    << "    }";
  return o.str();
}

}  // namespace

int main(int argc, char** argv) {
  return tool::run_main([&]() -> int {
    const Options o = parse(argc, argv);
    tool::Mesh mesh(o.mesh);
    std::cerr << "building BVH method=" << o.build_method << " leaf=" << o.leaf_size << "...\n";
    tool::Bvh bvh(mesh, o.leaf_size, o.build_method);
    n2w_problem pb{};
    N2W_CHECK(n2w_problem_reference_mode(N2W_BC_HARMONIC_X2_MINUS_Y2, N2W_SOURCE_CENTER, &pb));
    const double exact = static_cast<double>(o.x0[0]) * o.x0[0] - static_cast<double>(o.x0[1]) * o.x0[1];

    float b6[6];
    mesh.bounds(b6);
    // Unit-cube map of the cache inputs: mesh bounds padded by 5 % per side.
    float in_min[3], in_ext[3];
    for (int k = 0; k < 3; ++k) {
      const float e = b6[3 + k] - b6[k];
      in_min[k] = b6[k] - 0.05f * e;
      in_ext[k] = e * 1.1f;
    }
    tool::Stream stream;
    tool::DeviceArray<n2w_vec3> d_x0(1);
    d_x0.upload(reinterpret_cast<const n2w_vec3*>(o.x0), 1, stream.s);
    tool::Timer timer;

    // Plain WoS: one point, `samples` walks, FP64 per-point reduction.
    auto run_pure = [&](int samples, uint64_t seed) {
      tool::PointStats st(1);
      tool::DeviceArray<n2w_walk_counters> d_c(1);
      n2w_walk_options wo{};
      wo.walks_per_point = samples;
      wo.max_steps = o.max_steps;
      wo.epsilon = o.epsilon;
      wo.step_scale = o.step_scale;
      wo.seed = seed;
      wo.block_size = tool::walker_block(o.block_size);
      timer.start(stream.s);
      N2W_CHECK(n2w_wos_estimate(bvh.b, &pb, d_x0.p, 1, &wo, st.view(), d_c.p, nullptr, stream.s));
      const float ms = timer.stop_ms(stream.s);
      const n2w_walk_counters c = d_c.to_host(1, stream.s)[0];
      return finish(st, samples, ms, c.queries, c.forced, c.overflow);
    };
    // Oracle levels: coarse (PREFIX closed by the exact u) or residual.
    auto run_level = [&](bool coarse, int samples, uint64_t seed) {
      tool::PointStats st(1);
      tool::DeviceArray<n2w_nc2lmc_counters> d_c(1);
      d_c.zero(stream.s);
      n2w_nc2lmc_options no{};
      no.coarse_walks = coarse ? samples : 0;
      no.residual_walks = coarse ? 0 : samples;
      no.depth_m = o.depth_m;
      no.max_steps = o.max_steps;
      no.epsilon = o.epsilon;
      no.step_scale = o.step_scale;
      no.seed = seed;
      for (int k = 0; k < 3; ++k) {
        no.input_min[k] = in_min[k];
        no.input_extent[k] = in_ext[k];
      }
      timer.start(stream.s);
      N2W_CHECK(n2w_nc2lmc_estimate_ex(bvh.b, &pb, nullptr, d_x0.p, 1, &no, coarse ? st.view() : n2w_point_stats{},
                                       coarse ? n2w_point_stats{} : st.view(), d_c.p, stream.s));
      const float ms = timer.stop_ms(stream.s);
      const n2w_nc2lmc_counters c = d_c.to_host(1, stream.s)[0];
      const auto h = st.to_host();
      // Each walk queries once per position: steps + 1 per walk.
      const unsigned long long q = h.steps[0] + static_cast<unsigned long long>(samples);
      return finish(st, samples, ms, q, coarse ? c.coarse_forced : c.residual_forced,
                    coarse ? c.coarse_overflow : c.residual_overflow);
    };

    std::ostringstream runs;
    double est_mean = 0, est_var = 0, est_stderr = 0, elapsed = 0;
    if (o.method == "pure_wos") {
      const RunStats s = run_pure(o.samples, o.seed);
      est_mean = s.mean;
      est_var = s.estimator_variance;
      est_stderr = s.stderr_;
      elapsed = s.elapsed_ms;
      runs << run_json("pure_wos", s, exact);
    } else if (o.method == "oracle_coarse") {
      const RunStats s = run_level(true, o.samples, o.seed);
      est_mean = s.mean;
      est_var = s.estimator_variance;
      est_stderr = s.stderr_;
      elapsed = s.elapsed_ms;
      runs << run_json("oracle_coarse", s, exact);
    } else if (o.method == "oracle_residual") {
      const RunStats s = run_level(false, o.samples, o.seed);
      est_mean = s.mean;
      est_var = s.estimator_variance;
      est_stderr = s.stderr_;
      elapsed = s.elapsed_ms;
      runs << run_json("oracle_residual", s, 0.0);
    } else {
      const int nc = o.coarse_samples > 0 ? o.coarse_samples : o.samples;
      const int nr = o.residual_samples > 0 ? o.residual_samples : std::max(1, o.samples / 8);
      const RunStats c = run_level(true, nc, o.seed);
      const RunStats r = run_level(false, nr, o.seed ^ 0x517cc1b727220a95ull);
      est_mean = c.mean + r.mean;
      est_var = c.estimator_variance + r.estimator_variance;
      est_stderr = std::sqrt(est_var);
      elapsed = static_cast<double>(c.elapsed_ms) + r.elapsed_ms;
      runs << run_json("coarse", c, exact) << ",\n" << run_json("residual", r, 0.0);
    }
    const double est_err = est_mean - exact;
    const auto& st = bvh.stats;
    std::ostringstream j;
    j << "{\n"
      << "  \"schema\": \"n2wos_wavefront_wos_eval_v1\",\n"
      << "  \"patch\": \"n2w-sm100a-persistent-walker\",\n"
      << "  \"generated_at_utc\": " << tool::json_quote(tool::utc_now()) << ",\n"
      << "  \"command_line\": " << tool::json_quote(tool::join_argv(argc, argv)) << ",\n"
      << "  \"cuda\": " << tool::cuda_json() << ",\n"
      << "  \"implementation_mode\": {\n"
      << "    \"engine\": \"n2w_persistent_walker_queue_regeneration\",\n"
      << "    \"geometry_backend\": \"n2w_sm100a_bvh\",\n"
      << "    \"geometry_build_method\": " << tool::json_quote(o.build_method) << ",\n"
      << "    \"gpu_resident_walker_state\": true,\n"
      << "    \"gpu_rng\": \"philox4x32_10_counter_based\",\n"
      << "    \"cpu_gpu_transfer_inside_sampling_loop\": false,\n"
      << "    \"host_controls_global_step_loop\": false,\n"
      << "    \"per_walk_kernel_launch\": false,\n"
      << "    \"active_compaction\": true,\n"
      << "    \"inactive_slots_skip_bvh_traversal\": true,\n"
      << "    \"coarse_query_rounds_capped_at_depth_m\": true,\n"
      << "    \"cache_backend\": \"analytic_oracle_debug_only\",\n"
      << "    \"tcnn_in_solver\": false,\n"
      << "    \"reduction\": \"per_point_fp64_warp_shuffle_atomics\",\n"
      << "    \"timing_scope\": \"cuda_events_include_walks_cache_and_reduction_exclude_bvh_build_allocation_final_readback\",\n"
      << "    \"launched_query_slots_meaning\": \"closest-point queries actually issued (steps + 1 per walk)\"\n"
      << "  },\n"
      << "  \"options\": {\n"
      << "    \"mesh\": " << tool::json_quote(o.mesh.mesh) << ",\n"
      << "    \"mesh_path\": " << tool::json_quote(o.mesh.mesh_path) << ",\n"
      << "    \"normalize\": " << (o.mesh.normalize ? "true" : "false") << ",\n"
      << "    \"method\": " << tool::json_quote(o.method) << ",\n"
      << "    \"engine\": " << tool::json_quote(o.engine) << ",\n"
      << "    \"samples\": " << o.samples << ",\n"
      << "    \"coarse_samples\": " << o.coarse_samples << ",\n"
      << "    \"residual_samples\": " << o.residual_samples << ",\n"
      << "    \"depth_m\": " << o.depth_m << ",\n"
      << "    \"max_steps\": " << o.max_steps << ",\n"
      << "    \"epsilon\": " << tool::num(o.epsilon) << ",\n"
      << "    \"step_scale\": " << tool::num(o.step_scale) << ",\n"
      << "    \"x0\": " << tool::vec3_json(o.x0) << ",\n"
      << "    \"seed\": " << o.seed << ",\n"
      << "    \"block_size\": " << o.block_size << ",\n"
      << "    \"cubql_leaf_size\": " << o.leaf_size << ",\n"
      << "    \"cubql_build_method\": " << tool::json_quote(o.build_method) << "\n"
      << "  },\n"
      << "  \"mesh_stats\": " << tool::mesh_stats_json(mesh, n2w_mesh_name(mesh.m), true) << ",\n"
      << "  \"bvh_stats\": {\n"
      << "    \"triangles\": " << st.triangles << ",\n"
      << "    \"nodes\": " << st.nodes << ",\n"
      << "    \"prim_ids\": " << st.triangles << ",\n"
      << "    \"leaf_size\": " << st.leaf_size << ",\n"
      << "    \"build_method\": " << tool::json_quote(o.build_method) << ",\n"
      << "    \"build_milliseconds\": " << tool::num(st.build_milliseconds) << "\n"
      << "  },\n"
      << "  \"target\": {\"boundary_condition\": \"harmonic_x2_minus_y2\", \"exact_u_x0\": " << tool::num(exact)
      << "},\n"
      << "  \"runs\": {\n"
      << runs.str() << "\n  },\n"
      << "  \"estimator\": {\n"
      << "    \"method\": " << tool::json_quote(o.method) << ",\n"
      << "    \"engine\": " << tool::json_quote(o.engine) << ",\n"
      << "    \"mean\": " << tool::num(est_mean) << ",\n"
      << "    \"exact\": " << tool::num(exact) << ",\n"
      << "    \"error\": " << tool::num(est_err) << ",\n"
      << "    \"abs_error\": " << tool::num(std::fabs(est_err)) << ",\n"
      << "    \"estimator_variance\": " << tool::num(est_var) << ",\n"
      << "    \"stderr\": " << tool::num(est_stderr) << ",\n"
      << "    \"elapsed_ms_total\": " << tool::num(elapsed) << "\n"
      << "  }\n"
      << "}\n";
    tool::write_text(o.output, j.str());
    std::cout << j.str();
    return 0;
  });
}
