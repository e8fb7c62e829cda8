// n2wos_eval_tcnn_nc_wos: neural-cache WoS evaluator.  Trains the hash-grid +
// MLP cache on a fixed training set with refreshed WoS (or exact) labels, then
// compares plain WoS, NC-WoS (walks truncated at depth m, closed by the cache)
// and NC+2LMC (NC-WoS plus a residual level) on ball, slice or training points.
//
// Flags, presets, samplers, seeds and the JSON schema (n2wos_tcnn_nc_wos_eval_v4)
// follow src/tools/eval_tcnn_nc_wos.cu: options 268-347, presets 240-257,
// ball points 385-391, slice grid 392-395, training set 437-491 (padded to a
// multiple of 256 by reusing accepted points), input map 522-523, level seeds
// 735-770, summaries 525-569, estimates CSV 605-646, JSON 782-849.
//
// Everything runs through libn2w: the training set is drawn on the device by
// rejection with +x ray parity over the BVH (the reference does the same test
// on the host), labels are refreshed with n2w_nc_update_labels, each training
// step is one full-batch Adam step of the n2w cache, and per-point statistics
// are FP64 reductions on the device.
#include <random>

#include "common.hpp"

namespace {

struct Options {
  tool::MeshOptions mesh;
  std::string build_method = "sah";
  int leaf_size = 8;
  std::string bc = "external_charges_high";
  int mode = N2W_BC_EXTERNAL_CHARGES_HIGH;
  std::string label_source = "wos_supervision";
  std::string source_sampling = "center";
  int train_points = 20000;
  int eval_points = 8192;
  std::string eval_mode = "ball";
  int slice_width = 512, slice_height = 512;
  std::string slice_view = "xy";
  float slice_plane = 0.0f;
  bool slice_use_mesh_bounds = true;
  bool slice_preserve_world_aspect = true;
  float slice_frame[4] = {-1.0f, 1.0f, -1.0f, 1.0f};
  float slice_padding_fraction = 0.02f;
  std::string slice_output_prefix;
  std::string train_sampler = "rejection";
  std::string save_train_points_prefix;
  int label_refreshes = 4;
  int walks_per_label_refresh = 50;
  int train_steps_per_refresh = 5000;
  int pure_wpp = 64, hybrid_wpp = 4, coarse_wpp = 64, residual_wpp = 4;
  int enable_2lmc = 1;
  int depth_m = 1;
  int max_steps = 256;
  float epsilon = 1.0e-4f;
  float step_scale = 0.999f;
  int seed = 12345;
  int block_size = 128;
  std::string cache_preset = "baseline";
  int n_levels = 12, n_features_per_level = 2, log2_hashmap_size = 18, base_resolution = 8;
  float per_level_scale = 1.5f;
  int n_neurons = 32, n_hidden_layers = 2;
  float learning_rate = 1.0e-2f;
  std::string network = "FullyFusedMLP";
  int jit = 0;
  std::string output = "results/eval_tcnn_nc_wos.json";
  std::string save_estimates_prefix;
  int skip_training = 0;
  int eval_use_train_points = 0;
};

void apply_preset(Options& o, const std::string& p) {
  o.cache_preset = p;
  auto set = [&](int L, int F, int T, int N0, float b, int H, int D) {
    o.n_levels = L;
    o.n_features_per_level = F;
    o.log2_hashmap_size = T;
    o.base_resolution = N0;
    o.per_level_scale = b;
    o.n_neurons = H;
    o.n_hidden_layers = D;
  };
  if (p == "baseline" || p == "paper_like") set(12, 2, 18, 8, 1.5f, 32, 2);
  else if (p == "light") set(8, 2, 15, 8, 1.5f, 16, 1);
  else if (p == "nano") set(6, 2, 13, 8, 1.5f, 16, 1);
  else if (p == "heavy") set(16, 2, 19, 8, 1.4f, 64, 3);
  else if (p == "xlarge") set(16, 4, 20, 8, 1.35f, 64, 4);
  else if (p != "custom") {
    throw std::runtime_error("unknown cache preset: " + p + " (expected baseline, light, nano, heavy, xlarge, custom)");
  }
}

void usage(const char* argv0) {
  std::cout << "Usage: " << argv0 << " [options]\n"
            << "  --mesh procedural_bumpy_sphere|obj|ply\n"
            << "  --mesh-path <path>\n"
            << "  --bc constant_one|harmonic_x2_minus_y2|external_charges_medium|external_charges_high|"
               "harmonic_zebra_k8|external_charges_shell_k16|boundary_texture_stripes_k16|"
               "boundary_texture_checker_k16|poisson_multiscale|poisson_figlike_hf|...\n"
            << "  --label-source wos_supervision|exact_analytic\n"
            << "  --source-sampling center|ball   (Poisson source rule; center = reference) [center]\n"
            << "  --cache-preset baseline|light|nano|heavy|xlarge|custom\n"
            << "  --train-points <int> --eval-points <int>\n"
            << "  --train-sampler rejection|ball\n"
            << "  --save-train-points-prefix <prefix>\n"
            << "  --eval-mode ball|slice|train_points\n"
            << "  --slice-width <int> --slice-height <int> --slice-view xy|xz|yz --slice-plane <float>\n"
            << "  --slice-frame u_min,u_max,v_min,v_max --slice-padding-fraction <f>\n"
            << "  --slice-preserve-world-aspect 0|1 --slice-output-prefix <prefix>\n"
            << "  --label-refreshes <int> --walks-per-label-refresh <int>\n"
            << "  --train-steps-per-refresh <int>\n"
            << "  --pure-walks-per-point <int> --hybrid-walks-per-point <int>\n"
            << "  --coarse-walks-per-point <int> --residual-walks-per-point <int>\n"
            << "  --depth-m <int> --enable-2lmc 0|1 --max-steps <int> --epsilon <f> --step-scale <f>\n"
            << "  --seed <int> --block-size <int> --cubql-build-method sah|spatial_median --cubql-leaf-size <int>\n"
            << "  --network FullyFusedMLP|CutlassMLP --n-levels --n-features-per-level --log2-hashmap-size\n"
            << "  --base-resolution --per-level-scale --n-neurons --n-hidden-layers --learning-rate --jit 0|1\n"
            << "  --output <path> --save-estimates-prefix <prefix>\n"
            << "  --skip-training 0|1 --eval-use-train-points 0|1\n";
}

Options parse(int argc, char** argv) {
  Options o;
  for (int i = 1; i < argc; ++i) {
    const std::string a = argv[i];
    auto val = [&] { return tool::require_value(i, argc, argv); };
    auto ival = [&] { return tool::parse_int(val(), a); };
    auto fval = [&] { return tool::parse_float(val(), a); };
    if (a == "--help" || a == "-h") {
      usage(argv[0]);
      std::exit(0);
    } else if (o.mesh.parse(a, i, argc, argv)) {
    } else if (a == "--cubql-build-method") o.build_method = val();
    else if (a == "--cubql-leaf-size") o.leaf_size = ival();
    else if (a == "--bc" || a == "--boundary") {
      o.bc = tool::normalize_mode_text(val());
      N2W_CHECK(n2w_problem_mode_from_name(o.bc.c_str(), &o.mode));
    } else if (a == "--label-source") {
      const std::string s = val();
      if (s == "exact" || s == "exact_analytic") o.label_source = "exact_analytic";
      else if (s == "wos" || s == "wos_supervision") o.label_source = "wos_supervision";
      else throw std::runtime_error("unknown NC label source: " + s);
    } else if (a == "--source-sampling") {
      o.source_sampling = val();
      if (o.source_sampling != "center" && o.source_sampling != "ball") {
        throw std::runtime_error("--source-sampling must be center or ball");
      }
    } else if (a == "--cache-preset") apply_preset(o, val());
    else if (a == "--train-points") o.train_points = ival();
    else if (a == "--train-sampler") {
      o.train_sampler = tool::normalize_mode_text(val());
      if (o.train_sampler == "bbox_rejection") o.train_sampler = "rejection";
      if (o.train_sampler != "rejection" && o.train_sampler != "ball") {
        throw std::runtime_error("--train-sampler must be rejection or ball");
      }
    } else if (a == "--save-train-points-prefix") o.save_train_points_prefix = val();
    else if (a == "--eval-points") o.eval_points = ival();
    else if (a == "--eval-mode" || a == "--eval-sampler") {
      o.eval_mode = val();
      if (o.eval_mode != "ball" && o.eval_mode != "slice" && o.eval_mode != "train_points") {
        throw std::runtime_error("--eval-mode must be ball, slice, or train_points");
      }
    } else if (a == "--slice-width") o.slice_width = ival();
    else if (a == "--slice-height") o.slice_height = ival();
    else if (a == "--slice-view") {
      o.slice_view = val();
      if (o.slice_view != "xy" && o.slice_view != "xz" && o.slice_view != "yz") {
        throw std::runtime_error("--slice-view must be xy, xz, or yz");
      }
    } else if (a == "--slice-plane") o.slice_plane = fval();
    else if (a == "--slice-frame") {
      const auto f = tool::parse_float_list(val(), 4, "--slice-frame");
      for (int k = 0; k < 4; ++k) o.slice_frame[k] = f[k];
      o.slice_use_mesh_bounds = false;
    } else if (a == "--slice-padding-fraction") o.slice_padding_fraction = fval();
    else if (a == "--slice-preserve-world-aspect") o.slice_preserve_world_aspect = ival() != 0;
    else if (a == "--slice-output-prefix") o.slice_output_prefix = val();
    else if (a == "--label-refreshes") o.label_refreshes = ival();
    else if (a == "--walks-per-label-refresh") o.walks_per_label_refresh = ival();
    else if (a == "--train-steps-per-refresh") o.train_steps_per_refresh = ival();
    else if (a == "--pure-walks-per-point") o.pure_wpp = ival();
    else if (a == "--hybrid-walks-per-point") o.hybrid_wpp = ival();
    else if (a == "--coarse-walks-per-point") o.coarse_wpp = ival();
    else if (a == "--residual-walks-per-point") o.residual_wpp = ival();
    else if (a == "--enable-2lmc") o.enable_2lmc = ival();
    else if (a == "--depth-m") o.depth_m = ival();
    else if (a == "--max-steps") o.max_steps = ival();
    else if (a == "--epsilon") o.epsilon = fval();
    else if (a == "--step-scale") o.step_scale = fval();
    else if (a == "--seed") o.seed = ival();
    else if (a == "--block-size") o.block_size = ival();
    else if (a == "--network") o.network = val();
    else if (a == "--n-levels") { o.n_levels = ival(); o.cache_preset = "custom"; }
    else if (a == "--n-features-per-level") { o.n_features_per_level = ival(); o.cache_preset = "custom"; }
    else if (a == "--log2-hashmap-size") { o.log2_hashmap_size = ival(); o.cache_preset = "custom"; }
    else if (a == "--base-resolution") { o.base_resolution = ival(); o.cache_preset = "custom"; }
    else if (a == "--per-level-scale") { o.per_level_scale = fval(); o.cache_preset = "custom"; }
    else if (a == "--n-neurons") { o.n_neurons = ival(); o.cache_preset = "custom"; }
    else if (a == "--n-hidden-layers") { o.n_hidden_layers = ival(); o.cache_preset = "custom"; }
    else if (a == "--learning-rate") o.learning_rate = fval();
    else if (a == "--jit") o.jit = ival();
    else if (a == "--output") o.output = val();
    else if (a == "--save-estimates-prefix") o.save_estimates_prefix = val();
    else if (a == "--skip-training") o.skip_training = ival();
    else if (a == "--eval-use-train-points") {
      o.eval_use_train_points = ival();
      if (o.eval_use_train_points) o.eval_mode = "train_points";
    } else throw std::runtime_error("unknown argument: " + a);
  }
  o.mesh.validate();
  if (o.train_points <= 0 || o.eval_points <= 0 || o.pure_wpp <= 0 || o.hybrid_wpp <= 0) {
    throw std::runtime_error("invalid sample counts");
  }
  if (o.eval_mode == "slice" && (o.slice_width <= 0 || o.slice_height <= 0)) {
    throw std::runtime_error("invalid slice dimensions");
  }
  if (o.coarse_wpp <= 0 || o.residual_wpp <= 0) throw std::runtime_error("invalid 2LMC sample counts");
  if (o.label_refreshes <= 0 || o.walks_per_label_refresh <= 0 || o.train_steps_per_refresh < 0) {
    throw std::runtime_error("invalid training schedule");
  }
  if (o.depth_m < 0 || o.max_steps <= 0 || !(o.epsilon > 0.0f)) throw std::runtime_error("invalid WoS options");
  if (o.network != "FullyFusedMLP" && o.network != "CutlassMLP") {
    throw std::runtime_error("--network must be FullyFusedMLP or CutlassMLP");
  }
  return o;
}

using P3 = std::array<float, 3>;

// Uniform points in the ball of radius 0.42 * (smallest box extent) about the
// box centre (mt19937_64; z, phi, cube-root radius per point).
std::vector<P3> ball_points(int n, const float* b6, uint64_t seed) {
  const float cx = 0.5f * (b6[0] + b6[3]), cy = 0.5f * (b6[1] + b6[4]), cz = 0.5f * (b6[2] + b6[5]);
  const float radius = 0.42f * std::min({b6[3] - b6[0], b6[4] - b6[1], b6[5] - b6[2]});
  std::mt19937_64 rng(seed);
  std::uniform_real_distribution<float> u(0.0f, 1.0f);
  std::vector<P3> pts;
  pts.reserve(n);
  for (int i = 0; i < n; ++i) {
    const float z = 1.0f - 2.0f * u(rng);
    const float phi = 6.283185307179586f * u(rng);
    const float rr = radius * std::cbrt(std::max(0.0f, u(rng)));
    const float s = std::sqrt(std::max(0.0f, 1.0f - z * z));
    pts.push_back({cx + rr * s * std::cos(phi), cy + rr * s * std::sin(phi), cz + rr * z});
  }
  return pts;
}

struct TrainSet {
  std::vector<P3> points;
  std::vector<int> source;
  std::string sampler;
  int requested = 0, padded = 0, unique = 0;
  long long candidates = 0, accepted = 0;
  double acceptance = 0.0;
  bool padding_reuses = false;
  std::string inside_test;
};

TrainSet make_train_set(const Options& o, const tool::Bvh& bvh, const float* b6, tool::Stream& stream) {
  TrainSet t;
  t.requested = o.train_points;
  t.padded = (o.train_points + 255) / 256 * 256;
  if (o.train_sampler == "ball") {
    t.sampler = "ball";
    t.unique = t.padded;
    t.candidates = t.accepted = t.padded;
    t.acceptance = 1.0;
    t.inside_test = "not_applied_debug_ball_sampler";
    t.points = ball_points(t.padded, b6, static_cast<uint64_t>(o.seed));
    t.source.resize(t.padded);
    for (int i = 0; i < t.padded; ++i) t.source[i] = i;
    return t;
  }
  t.sampler = "bbox_rejection";
  t.unique = t.requested;
  t.padding_reuses = t.padded > t.requested;
  t.inside_test = "device_ray_parity_x_over_bvh";
  tool::DeviceArray<n2w_vec3> d(t.requested);
  int64_t acc = 0, cand = 0;
  N2W_CHECK(n2w_sample_interior_ex(bvh.b, b6, b6 + 3, t.requested, static_cast<uint64_t>(o.seed), d.p, &acc, &cand,
                                   stream.s));
  const std::vector<n2w_vec3> h = d.to_host(t.requested, stream.s);
  t.accepted = acc;
  t.candidates = cand;
  t.acceptance = cand > 0 ? static_cast<double>(acc) / cand : 0.0;
  for (int i = 0; i < t.requested; ++i) {
    t.points.push_back({h[i].x, h[i].y, h[i].z});
    t.source.push_back(i);
  }
  std::mt19937_64 rng(static_cast<uint64_t>(o.seed));
  std::uniform_int_distribution<int> pick(0, t.requested - 1);
  while (static_cast<int>(t.points.size()) < t.padded) {
    const int s = pick(rng);
    t.points.push_back(t.points[s]);
    t.source.push_back(s);
  }
  return t;
}

struct Slice {
  int width = 0, height = 0, candidates = 0, inside = 0;
  float frame[4] = {0, 0, 0, 0};
  std::vector<uint8_t> mask;
  std::string prefix;
};

// Per-point statistics of one level (or of plain WoS) against the exact solution.
struct Summary {
  double rmse = 0, mae = 0, max_abs = 0, mean_est = 0, mean_exact = 0, mean_var = 0, mean_steps = 0;
  unsigned long long cache_queries = 0, forced = 0, overflow = 0;
};

Summary summarize(const tool::PointStats::Host& h, const std::vector<double>& exact) {
  Summary s;
  const size_t n = exact.size();
  double se = 0;
  for (size_t i = 0; i < n; ++i) {
    const double m = h.mean(i), e = m - exact[i];
    se += e * e;
    s.mae += std::fabs(e);
    s.max_abs = std::max(s.max_abs, std::fabs(e));
    s.mean_est += m;
    s.mean_exact += exact[i];
    s.mean_var += h.variance(i);
    s.mean_steps += h.mean_steps(i);
    s.forced += h.forced[i];
  }
  s.rmse = std::sqrt(se / n);
  s.mae /= n;
  s.mean_est /= n;
  s.mean_exact /= n;
  s.mean_var /= n;
  s.mean_steps /= n;
  return s;
}

struct TwoLevel {
  double rmse = 0, mae = 0, max_abs = 0, mean_est = 0, mean_exact = 0, mean_c = 0, mean_r = 0, var_c = 0, var_r = 0,
         steps_c = 0, steps_r = 0;
};

TwoLevel summarize2(const tool::PointStats::Host& c, const tool::PointStats::Host& r, const std::vector<double>& exact) {
  TwoLevel t;
  const size_t n = exact.size();
  double se = 0;
  for (size_t i = 0; i < n; ++i) {
    const double cm = c.mean(i), rm = r.mean(i), est = cm + rm, e = est - exact[i];
    se += e * e;
    t.mae += std::fabs(e);
    t.max_abs = std::max(t.max_abs, std::fabs(e));
    t.mean_est += est;
    t.mean_exact += exact[i];
    t.mean_c += cm;
    t.mean_r += rm;
    t.var_c += c.variance(i);
    t.var_r += r.variance(i);
    t.steps_c += c.mean_steps(i);
    t.steps_r += r.mean_steps(i);
  }
  t.rmse = std::sqrt(se / n);
  for (double* v : {&t.mae, &t.mean_est, &t.mean_exact, &t.mean_c, &t.mean_r, &t.var_c, &t.var_r, &t.steps_c,
                    &t.steps_r}) {
    *v /= n;
  }
  return t;
}

std::string stats_json(const Summary& s, int points, int wpp, float ms, float training_ms) {
  const double samples = static_cast<double>(points) * wpp;
  std::ostringstream o;
  o << "{\n"
    << "      \"eval_points\": " << points << ",\n"
    << "      \"walks_per_point\": " << wpp << ",\n"
    << "      \"samples\": " << static_cast<long long>(samples) << ",\n"
    << "      \"rmse\": " << tool::num(s.rmse) << ",\n"
    << "      \"mae\": " << tool::num(s.mae) << ",\n"
    << "      \"max_abs_error\": " << tool::num(s.max_abs) << ",\n"
    << "      \"mean_estimate\": " << tool::num(s.mean_est) << ",\n"
    << "      \"mean_exact\": " << tool::num(s.mean_exact) << ",\n"
    << "      \"mean_bias\": " << tool::num(s.mean_est - s.mean_exact) << ",\n"
    << "      \"mean_sample_variance\": " << tool::num(s.mean_var) << ",\n"
    << "      \"mean_steps\": " << tool::num(s.mean_steps) << ",\n"
    << "      \"cache_queries\": " << s.cache_queries << ",\n"
    << "      \"cache_query_fraction\": " << tool::num(samples > 0 ? s.cache_queries / samples : 0.0) << ",\n"
    << "      \"forced_max_steps\": " << s.forced << ",\n"
    << "      \"overflow_count\": " << s.overflow << ",\n"
    << "      \"elapsed_ms\": " << tool::num(ms) << ",\n"
    << "      \"training_plus_elapsed_ms\": " << tool::num(training_ms + ms) << ",\n"
    << "      \"us_per_point\": " << tool::num(1000.0 * ms / points) << ",\n"
    << "      \"us_per_sample\": " << tool::num(1000.0 * ms / samples) << "\n"
    << "    }";
  return o.str();
}

std::string two_level_json(const TwoLevel& t, const n2w_nc2lmc_counters& c, int points, int cw, int rw, float cms,
                           float rms, float training_ms) {
  const double cs = static_cast<double>(points) * cw, rs = static_cast<double>(points) * rw;
  const float el = cms + rms;
  std::ostringstream o;
  o << "{\n"
    << "      \"eval_points\": " << points << ",\n"
    << "      \"coarse_walks_per_point\": " << cw << ",\n"
    << "      \"residual_walks_per_point\": " << rw << ",\n"
    << "      \"coarse_samples\": " << static_cast<long long>(cs) << ",\n"
    << "      \"residual_samples\": " << static_cast<long long>(rs) << ",\n"
    << "      \"rmse\": " << tool::num(t.rmse) << ",\n"
    << "      \"mae\": " << tool::num(t.mae) << ",\n"
    << "      \"max_abs_error\": " << tool::num(t.max_abs) << ",\n"
    << "      \"mean_estimate\": " << tool::num(t.mean_est) << ",\n"
    << "      \"mean_exact\": " << tool::num(t.mean_exact) << ",\n"
    << "      \"mean_bias\": " << tool::num(t.mean_est - t.mean_exact) << ",\n"
    << "      \"mean_coarse\": " << tool::num(t.mean_c) << ",\n"
    << "      \"mean_residual\": " << tool::num(t.mean_r) << ",\n"
    << "      \"mean_coarse_sample_variance\": " << tool::num(t.var_c) << ",\n"
    << "      \"mean_residual_sample_variance\": " << tool::num(t.var_r) << ",\n"
    << "      \"mean_coarse_steps\": " << tool::num(t.steps_c) << ",\n"
    << "      \"mean_residual_steps\": " << tool::num(t.steps_r) << ",\n"
    << "      \"coarse_cache_queries\": " << c.coarse_cache_queries << ",\n"
    << "      \"residual_cache_queries\": " << c.residual_cache_queries << ",\n"
    << "      \"coarse_cache_query_fraction\": " << tool::num(cs > 0 ? c.coarse_cache_queries / cs : 0.0) << ",\n"
    << "      \"residual_cache_query_fraction\": " << tool::num(rs > 0 ? c.residual_cache_queries / rs : 0.0) << ",\n"
    << "      \"coarse_forced_max_steps\": " << c.coarse_forced << ",\n"
    << "      \"residual_forced_max_steps\": " << c.residual_forced << ",\n"
    << "      \"coarse_overflow_count\": " << c.coarse_overflow << ",\n"
    << "      \"residual_overflow_count\": " << c.residual_overflow << ",\n"
    << "      \"coarse_elapsed_ms\": " << tool::num(cms) << ",\n"
    << "      \"residual_elapsed_ms\": " << tool::num(rms) << ",\n"
    << "      \"elapsed_ms\": " << tool::num(el) << ",\n"
    << "      \"training_plus_elapsed_ms\": " << tool::num(training_ms + el) << ",\n"
    << "      \"us_per_point\": " << tool::num(1000.0 * el / points) << ",\n"
    << "      \"us_per_effective_sample\": " << tool::num(1000.0 * el / (cs + rs)) << "\n"
    << "    }";
  return o.str();
}

void write_ppm_mask(const std::string& path, const Slice& s) {
  tool::ensure_parent_dir(path);
  std::ofstream f(path, std::ios::binary);
  if (!f) throw std::runtime_error("failed to open slice mask for writing: " + path);
  f << "P6\n" << s.width << " " << s.height << "\n255\n";
  for (int iy = 0; iy < s.height; ++iy) {
    const int sy = s.height - 1 - iy;
    for (int ix = 0; ix < s.width; ++ix) {
      const char c = static_cast<char>(s.mask[static_cast<size_t>(sy) * s.width + ix] ? 235 : 20);
      f.put(c);
      f.put(c);
      f.put(c);
    }
  }
}

void write_points_csv(const std::string& path, const std::vector<P3>& pts) {
  tool::ensure_parent_dir(path);
  std::ofstream f(path);
  if (!f) throw std::runtime_error("failed to open points CSV for writing: " + path);
  f << "point_id,x,y,z\n" << std::setprecision(10);
  for (size_t i = 0; i < pts.size(); ++i) f << i << ',' << pts[i][0] << ',' << pts[i][1] << ',' << pts[i][2] << '\n';
}

}  // namespace

int main(int argc, char** argv) {
  return tool::run_main([&]() -> int {
    const Options o = parse(argc, argv);
    const std::string cmd = tool::join_argv(argc, argv);
    tool::Mesh mesh(o.mesh);
    tool::Bvh bvh(mesh, o.leaf_size, o.build_method);
    float b6[6];
    mesh.bounds(b6);
    n2w_problem pb{};
    const int sampling = o.source_sampling == "ball" ? N2W_SOURCE_BALL : N2W_SOURCE_CENTER;
    if (o.mode == N2W_BC_POISSON_SINPROD) {
      N2W_CHECK(n2w_problem_sinprod(3.0f * 3.14159265358979f, sampling, &pb));
    } else if (o.mode == N2W_BC_CHARGES_SEEDED) {
      N2W_CHECK(n2w_problem_charges_seeded(8, 1.6f, 2.0f, static_cast<uint64_t>(o.seed), &pb));
    } else {
      N2W_CHECK(n2w_problem_reference_mode(o.mode, sampling, &pb));
    }
    tool::Stream stream;

    const TrainSet train = make_train_set(o, bvh, b6, stream);
    if (!o.save_train_points_prefix.empty()) {
      const std::string path = o.save_train_points_prefix + "_train_points.csv";
      tool::ensure_parent_dir(path);
      std::ofstream f(path);
      if (!f) throw std::runtime_error("failed to open training points CSV for writing: " + path);
      f << "point_id,x,y,z,is_padding,padding_source\n" << std::setprecision(10);
      for (size_t i = 0; i < train.points.size(); ++i) {
        f << i << ',' << train.points[i][0] << ',' << train.points[i][1] << ',' << train.points[i][2] << ','
          << (static_cast<int>(i) >= train.requested ? 1 : 0) << ',' << train.source[i] << '\n';
      }
    }

    std::vector<P3> eval;
    Slice slice;
    if (o.eval_mode == "train_points") {
      eval = train.points;
    } else if (o.eval_mode == "slice") {
      slice.width = o.slice_width;
      slice.height = o.slice_height;
      slice.candidates = o.slice_width * o.slice_height;
      std::vector<float> grid(3 * static_cast<size_t>(slice.candidates));
      N2W_CHECK(n2w_slice_points_ex(b6, o.slice_use_mesh_bounds ? nullptr : o.slice_frame, o.slice_view.c_str(),
                                    o.slice_plane, o.slice_width, o.slice_height, o.slice_padding_fraction,
                                    o.slice_preserve_world_aspect ? 1 : 0, N2W_SLICE_RULE_EVAL, grid.data(),
                                    slice.frame));
      tool::DeviceArray<n2w_vec3> d_grid(slice.candidates);
      tool::DeviceArray<uint8_t> d_in(slice.candidates);
      tool::DeviceArray<int> d_ov(1);
      d_ov.zero(stream.s);
      d_grid.upload(reinterpret_cast<const n2w_vec3*>(grid.data()), slice.candidates, stream.s);
      N2W_CHECK(n2w_bvh_inside_device(bvh.b, d_grid.p, slice.candidates, d_in.p, d_ov.p, 256, stream.s));
      slice.mask = d_in.to_host(slice.candidates, stream.s);
      for (int i = 0; i < slice.candidates; ++i) {
        if (slice.mask[i]) eval.push_back({grid[3 * i], grid[3 * i + 1], grid[3 * i + 2]});
      }
      slice.inside = static_cast<int>(eval.size());
      if (slice.inside == 0) {
        throw std::runtime_error("slice contains no interior pixels; adjust --slice-view, --slice-plane, or --slice-frame");
      }
      if (!o.slice_output_prefix.empty()) {
        slice.prefix = o.slice_output_prefix;
      } else {
        std::filesystem::path p(o.output);
        if (p.extension() == ".json") p.replace_extension("");
        slice.prefix = p.string() + "_slice";
      }
      write_ppm_mask(slice.prefix + "_mask.ppm", slice);
      write_points_csv(slice.prefix + "_points.csv", eval);
    } else {
      eval = ball_points(o.eval_points, b6, static_cast<uint64_t>(o.seed) ^ 0x8da6b343ull);
    }
    const int ne = static_cast<int>(eval.size());
    const int nt = static_cast<int>(train.points.size());
    std::vector<double> exact(ne);
    {
      std::vector<double> xyz(3 * static_cast<size_t>(ne));
      for (int i = 0; i < ne; ++i) {
        for (int k = 0; k < 3; ++k) xyz[3 * i + k] = eval[i][k];
      }
      N2W_CHECK(n2w_problem_exact(&pb, xyz.data(), ne, exact.data()));
    }

    // Cache inputs: mesh bounds padded by 5 % of the extent per side, mapped to [0,1]^3.
    float in_min[3], in_ext[3];
    for (int k = 0; k < 3; ++k) {
      const float e = b6[3 + k] - b6[k];
      in_min[k] = b6[k] - 0.05f * e;
      in_ext[k] = e * (1.0f + 2.0f * 0.05f);
    }

    n2w_cache_config cfg{};
    N2W_CHECK(n2w_cache_config_default(&cfg));
    cfg.n_levels = o.n_levels;
    cfg.n_features_per_level = o.n_features_per_level;
    cfg.log2_hashmap_size = o.log2_hashmap_size;
    cfg.base_resolution = static_cast<float>(o.base_resolution);
    cfg.per_level_scale = o.per_level_scale;
    cfg.n_neurons = o.n_neurons;
    cfg.n_hidden_layers = o.n_hidden_layers;
    cfg.learning_rate = o.learning_rate;
    cfg.beta1 = 0.9f;
    cfg.beta2 = 0.99f;
    cfg.seed = static_cast<uint64_t>(o.seed);
    n2w_cache* cache = nullptr;
    N2W_CHECK(n2w_cache_create(&cfg, &cache));
    struct Guard {
      n2w_cache* c;
      ~Guard() { n2w_cache_destroy(c); }
    } guard{cache};

    tool::DeviceArray<n2w_vec3> d_train(nt), d_eval(ne);
    d_train.upload(reinterpret_cast<const n2w_vec3*>(train.points.data()), nt, stream.s);
    d_eval.upload(reinterpret_cast<const n2w_vec3*>(eval.data()), ne, stream.s);
    tool::Timer timer;

    float label_ms = 0.0f, train_ms = 0.0f;
    if (!o.skip_training) {
      tool::PointStats labels_acc(nt);
      tool::DeviceArray<float> tin(3 * static_cast<size_t>(nt)), ttg(nt);
      n2w_nc_label_options lo{};
      lo.walks_per_point = o.walks_per_label_refresh;
      lo.max_steps = o.max_steps;
      lo.epsilon = o.epsilon;
      lo.step_scale = o.step_scale;
      lo.seed = static_cast<uint64_t>(o.seed);
      lo.label_source = o.label_source == "exact_analytic" ? N2W_LABEL_EXACT : N2W_LABEL_WOS;
      lo.block_size = tool::walker_block(o.block_size);
      for (int k = 0; k < 3; ++k) {
        lo.input_min[k] = in_min[k];
        lo.input_extent[k] = in_ext[k];
      }
      for (int r = 0; r < o.label_refreshes; ++r) {
        lo.refresh_index = r;
        timer.start(stream.s);
        N2W_CHECK(n2w_nc_update_labels(bvh.b, &pb, d_train.p, nt, &lo, labels_acc.view(), tin.p, ttg.p, nullptr,
                                       stream.s));
        label_ms += timer.stop_ms(stream.s);
        timer.start(stream.s);
        for (int s = 0; s < o.train_steps_per_refresh; ++s) {
          N2W_CHECK(n2w_cache_train_step(cache, tin.p, ttg.p, nt, nullptr, stream.s));
        }
        train_ms += timer.stop_ms(stream.s);
      }
    }
    const float training_ms = label_ms + train_ms;

    // Plain WoS.
    tool::PointStats pure(ne);
    tool::DeviceArray<n2w_walk_counters> d_wc(1);
    n2w_walk_options wo{};
    wo.walks_per_point = o.pure_wpp;
    wo.max_steps = o.max_steps;
    wo.epsilon = o.epsilon;
    wo.step_scale = o.step_scale;
    wo.seed = static_cast<uint64_t>(o.seed) ^ 0x44d2a123ull;
    wo.block_size = tool::walker_block(o.block_size);
    timer.start(stream.s);
    N2W_CHECK(n2w_wos_estimate(bvh.b, &pb, d_eval.p, ne, &wo, pure.view(), d_wc.p, nullptr, stream.s));
    const float pure_ms = timer.stop_ms(stream.s);
    const n2w_walk_counters wc = d_wc.to_host(1, stream.s)[0];

    auto level_options = [&](int coarse, int residual, uint64_t seed) {
      n2w_nc2lmc_options no{};
      no.coarse_walks = coarse;
      no.residual_walks = residual;
      no.depth_m = o.depth_m;
      no.max_steps = o.max_steps;
      no.epsilon = o.epsilon;
      no.step_scale = o.step_scale;
      no.seed = seed;
      for (int k = 0; k < 3; ++k) {
        no.input_min[k] = in_min[k];
        no.input_extent[k] = in_ext[k];
      }
      return no;
    };
    // NC-WoS: walks truncated at depth m and closed by the cache.
    tool::PointStats hyb(ne);
    tool::DeviceArray<n2w_nc2lmc_counters> d_hc(1);
    d_hc.zero(stream.s);
    const n2w_nc2lmc_options ho = level_options(o.hybrid_wpp, 0, static_cast<uint64_t>(o.seed) ^ 0x89abcdefull);
    timer.start(stream.s);
    N2W_CHECK(n2w_nc2lmc_estimate_ex(bvh.b, &pb, cache, d_eval.p, ne, &ho, hyb.view(), n2w_point_stats{}, d_hc.p,
                                     stream.s));
    const float hybrid_ms = timer.stop_ms(stream.s);
    const n2w_nc2lmc_counters hc = d_hc.to_host(1, stream.s)[0];

    // NC+2LMC: coarse level + residual level, timed separately.
    tool::PointStats c2(o.enable_2lmc ? ne : 1), r2(o.enable_2lmc ? ne : 1);
    n2w_nc2lmc_counters tc{};
    float coarse_ms = 0.0f, residual_ms = 0.0f;
    if (o.enable_2lmc) {
      tool::DeviceArray<n2w_nc2lmc_counters> d_tc(1);
      d_tc.zero(stream.s);
      const n2w_nc2lmc_options co =
          level_options(o.coarse_wpp, 0, static_cast<uint64_t>(o.seed) ^ 0xf1357aea2e62a9c5ull);
      const n2w_nc2lmc_options ro =
          level_options(0, o.residual_wpp, static_cast<uint64_t>(o.seed) ^ 0x5f4dca4f0a2bbf27ull);
      timer.start(stream.s);
      N2W_CHECK(n2w_nc2lmc_estimate_ex(bvh.b, &pb, cache, d_eval.p, ne, &co, c2.view(), n2w_point_stats{}, d_tc.p,
                                       stream.s));
      coarse_ms = timer.stop_ms(stream.s);
      timer.start(stream.s);
      N2W_CHECK(n2w_nc2lmc_estimate_ex(bvh.b, &pb, cache, d_eval.p, ne, &ro, n2w_point_stats{}, r2.view(), d_tc.p,
                                       stream.s));
      residual_ms = timer.stop_ms(stream.s);
      tc = d_tc.to_host(1, stream.s)[0];
    }

    const auto hp = pure.to_host(stream.s), hh = hyb.to_host(stream.s);
    Summary sp = summarize(hp, exact);
    sp.overflow = wc.overflow;
    Summary sh = summarize(hh, exact);
    sh.cache_queries = hc.coarse_cache_queries;
    sh.overflow = hc.coarse_overflow;
    TwoLevel tl;
    tool::PointStats::Host hc2, hr2;
    if (o.enable_2lmc) {
      hc2 = c2.to_host(stream.s);
      hr2 = r2.to_host(stream.s);
      tl = summarize2(hc2, hr2, exact);
    }

    if (!o.save_estimates_prefix.empty()) {
      const std::string path = o.save_estimates_prefix + "_estimates.csv";
      tool::ensure_parent_dir(path);
      std::ofstream f(path);
      if (!f) throw std::runtime_error("failed to open estimates CSV for writing: " + path);
      f << "point_id,x,y,z,analytic_value,pure_mean,pure_sample_variance,nc_wos_mean,nc_wos_sample_variance";
      if (o.enable_2lmc) {
        f << ",nc_2lmc_mean,nc_2lmc_coarse_mean,nc_2lmc_residual_mean,nc_2lmc_coarse_sample_variance,"
             "nc_2lmc_residual_sample_variance";
      }
      f << "\n" << std::setprecision(10);
      for (int i = 0; i < ne; ++i) {
        f << i << ',' << eval[i][0] << ',' << eval[i][1] << ',' << eval[i][2] << ',' << exact[i] << ','
          << hp.mean(i) << ',' << hp.variance(i) << ',' << hh.mean(i) << ',' << hh.variance(i);
        if (o.enable_2lmc) {
          f << ',' << (hc2.mean(i) + hr2.mean(i)) << ',' << hc2.mean(i) << ',' << hr2.mean(i) << ','
            << hc2.variance(i) << ',' << hr2.variance(i);
        }
        f << '\n';
      }
    }

    const char* point_sampler = o.eval_mode == "slice" ? "fixed_slice_interior_pixels"
                                : o.eval_mode == "train_points" ? "training_points_reused_for_eval_sanity"
                                                                : "inscribed_ball_screening_sampler";
    const auto& bs = bvh.stats;
    std::ostringstream j;
    j << "{\n"
      << "  \"schema\": \"n2wos_tcnn_nc_wos_eval_v4\",\n"
      << "  \"patch\": \"n2w-sm100a-nc-2lmc\",\n"
      << "  \"generated_at_utc\": " << tool::json_quote(tool::utc_now()) << ",\n"
      << "  \"command_line\": " << tool::json_quote(cmd) << ",\n"
      << "  \"cuda\": " << tool::cuda_json() << ",\n"
      << "  \"implementation_mode\": {\n"
      << "    \"solver\": \"neural_cache_wos_and_nc_2lmc_depth_sweep_screening\",\n"
      << "    \"geometry_backend\": \"n2w_sm100a_bvh\",\n"
      << "    \"cache_backend\": \"n2w_hashgrid_mlp_native\",\n"
      << "    \"walker\": \"n2w_persistent_walker_queue_regeneration\",\n"
      << "    \"training_schedule\": \"fixed_refresh_count_and_fixed_train_steps\",\n"
      << "    \"training_labels\": " << tool::json_quote(o.label_source) << ",\n"
      << "    \"poisson_source_rule\": " << tool::json_quote(o.source_sampling) << ",\n"
      << "    \"host_transfer_between_prefix_and_tcnn\": false,\n"
      << "    \"host_transfer_between_tcnn_and_residual_consumer\": false,\n"
      << "    \"csv_postprocess\": false,\n"
      << "    \"python_bindings\": false,\n"
      << "    \"nc_wos_biased\": true,\n"
      << "    \"nc_2lmc_correction_enabled\": " << (o.enable_2lmc ? "true" : "false") << ",\n"
      << "    \"nc_and_2lmc_share_depth_m\": true,\n"
      << "    \"point_sampler\": " << tool::json_quote(point_sampler) << ",\n"
      << "    \"per_point_statistics\": \"device_fp64_reductions\",\n"
      << "    \"production_status\": \"screening_diagnostic_not_final_wall_clock\"\n"
      << "  },\n"
      << "  \"options\": {\n"
      << "    \"mesh\": " << tool::json_quote(o.mesh.mesh) << ",\n"
      << "    \"mesh_path\": " << tool::json_quote(o.mesh.mesh_path) << ",\n"
      << "    \"boundary_condition\": " << tool::json_quote(n2w_problem_mode_name(o.mode)) << ",\n"
      << "    \"label_source\": " << tool::json_quote(o.label_source) << ",\n"
      << "    \"train_points_requested\": " << o.train_points << ",\n"
      << "    \"train_points_padded\": " << nt << ",\n"
      << "    \"train_sampler\": " << tool::json_quote(o.train_sampler) << ",\n"
      << "    \"eval_points_requested\": " << o.eval_points << ",\n"
      << "    \"eval_points\": " << ne << ",\n"
      << "    \"eval_mode\": " << tool::json_quote(o.eval_mode) << ",\n"
      << "    \"eval_use_train_points\": " << (o.eval_mode == "train_points" ? "true" : "false") << ",\n"
      << "    \"label_refreshes\": " << o.label_refreshes << ",\n"
      << "    \"walks_per_label_refresh\": " << o.walks_per_label_refresh << ",\n"
      << "    \"train_steps_per_refresh\": " << o.train_steps_per_refresh << ",\n"
      << "    \"pure_walks_per_point\": " << o.pure_wpp << ",\n"
      << "    \"hybrid_walks_per_point\": " << o.hybrid_wpp << ",\n"
      << "    \"coarse_walks_per_point\": " << o.coarse_wpp << ",\n"
      << "    \"residual_walks_per_point\": " << o.residual_wpp << ",\n"
      << "    \"depth_m\": " << o.depth_m << ",\n"
      << "    \"max_steps\": " << o.max_steps << ",\n"
      << "    \"epsilon\": " << tool::num(o.epsilon) << ",\n"
      << "    \"cache_preset\": " << tool::json_quote(o.cache_preset) << ",\n"
      << "    \"network\": " << tool::json_quote(o.network) << ",\n"
      << "    \"n_levels\": " << o.n_levels << ",\n"
      << "    \"n_features_per_level\": " << o.n_features_per_level << ",\n"
      << "    \"log2_hashmap_size\": " << o.log2_hashmap_size << ",\n"
      << "    \"base_resolution\": " << o.base_resolution << ",\n"
      << "    \"per_level_scale\": " << tool::num(o.per_level_scale) << ",\n"
      << "    \"n_neurons\": " << o.n_neurons << ",\n"
      << "    \"n_hidden_layers\": " << o.n_hidden_layers << ",\n"
      << "    \"jit_requested\": " << (o.jit ? "true" : "false") << ",\n"
      << "    \"jit_supported\": false,\n"
      << "    \"jit_enabled\": false\n"
      << "  },\n";
    if (o.eval_mode == "slice") {
      j << "  \"slice_eval\": {\n"
        << "    \"width\": " << slice.width << ",\n"
        << "    \"height\": " << slice.height << ",\n"
        << "    \"candidate_pixels\": " << slice.candidates << ",\n"
        << "    \"inside_pixels\": " << slice.inside << ",\n"
        << "    \"view\": " << tool::json_quote(o.slice_view) << ",\n"
        << "    \"plane\": " << tool::num(o.slice_plane) << ",\n"
        << "    \"frame_u_min\": " << tool::num(slice.frame[0]) << ",\n"
        << "    \"frame_u_max\": " << tool::num(slice.frame[1]) << ",\n"
        << "    \"frame_v_min\": " << tool::num(slice.frame[2]) << ",\n"
        << "    \"frame_v_max\": " << tool::num(slice.frame[3]) << ",\n"
        << "    \"mask_ppm\": " << tool::json_quote(slice.prefix + "_mask.ppm") << ",\n"
        << "    \"points_csv\": " << tool::json_quote(slice.prefix + "_points.csv") << "\n"
        << "  },\n";
    }
    if (!o.save_estimates_prefix.empty()) {
      j << "  \"estimate_outputs\": {\n"
        << "    \"estimates_csv\": " << tool::json_quote(o.save_estimates_prefix + "_estimates.csv") << "\n"
        << "  },\n";
    }
    j << "  \"training_point_sampler\": {\n"
      << "    \"mode\": " << tool::json_quote(train.sampler) << ",\n"
      << "    \"requested_points\": " << train.requested << ",\n"
      << "    \"padded_points\": " << train.padded << ",\n"
      << "    \"unique_points\": " << train.unique << ",\n"
      << "    \"candidate_points\": " << train.candidates << ",\n"
      << "    \"accepted_points\": " << train.accepted << ",\n"
      << "    \"acceptance_rate\": " << tool::num(train.acceptance) << ",\n"
      << "    \"inside_test\": " << tool::json_quote(train.inside_test) << ",\n"
      << "    \"padding_reuses_accepted_points\": " << (train.padding_reuses ? "true" : "false") << ",\n"
      << "    \"train_points_csv\": "
      << tool::json_quote(o.save_train_points_prefix.empty() ? "" : o.save_train_points_prefix + "_train_points.csv")
      << "\n"
      << "  },\n"
      << "  \"mesh_stats\": " << tool::mesh_stats_json(mesh, n2w_mesh_name(mesh.m), true) << ",\n"
      << "  \"bvh_stats\": {\n"
      << "    \"triangles\": " << bs.triangles << ",\n"
      << "    \"nodes\": " << bs.nodes << ",\n"
      << "    \"prim_ids\": " << bs.triangles << ",\n"
      << "    \"leaf_size\": " << bs.leaf_size << ",\n"
      << "    \"build_method\": " << tool::json_quote(o.build_method) << ",\n"
      << "    \"build_milliseconds\": " << tool::num(bs.build_milliseconds) << "\n"
      << "  },\n"
      << "  \"training\": {\n"
      << "    \"label_update_ms\": " << tool::num(label_ms) << ",\n"
      << "    \"tcnn_training_ms\": " << tool::num(train_ms) << ",\n"
      << "    \"total_training_ms\": " << tool::num(training_ms) << ",\n"
      << "    \"host_readback_in_training_loop\": false\n"
      << "  },\n"
      << "  \"runs\": {\n"
      << "    \"pure_wos\": " << stats_json(sp, ne, o.pure_wpp, pure_ms, 0.0f) << ",\n"
      << "    \"nc_wos\": " << stats_json(sh, ne, o.hybrid_wpp, hybrid_ms, training_ms);
    if (o.enable_2lmc) {
      const std::string two = two_level_json(tl, tc, ne, o.coarse_wpp, o.residual_wpp, coarse_ms, residual_ms,
                                             training_ms);
      j << ",\n    \"nc_2lmc\": " << two << ",\n    \"nc_2lmc_m" << o.depth_m << "\": " << two;
    }
    j << "\n  },\n"
      << "  \"comparison\": {\n"
      << "    \"nc_wos_rmse_div_pure_wos_rmse\": " << tool::num(sp.rmse > 0 ? sh.rmse / sp.rmse : 0.0) << ",\n";
    if (o.enable_2lmc) {
      const double lv = coarse_ms + residual_ms;
      j << "    \"nc_2lmc_rmse_div_pure_wos_rmse\": " << tool::num(sp.rmse > 0 ? tl.rmse / sp.rmse : 0.0) << ",\n"
        << "    \"nc_2lmc_rmse_div_nc_wos_rmse\": " << tool::num(sh.rmse > 0 ? tl.rmse / sh.rmse : 0.0) << ",\n"
        << "    \"nc_wos_mean_bias\": " << tool::num(sh.mean_est - sh.mean_exact) << ",\n"
        << "    \"nc_2lmc_mean_bias\": " << tool::num(tl.mean_est - tl.mean_exact) << ",\n"
        << "    \"pure_elapsed_div_nc_2lmc_inference_elapsed\": " << tool::num(lv > 0 ? pure_ms / lv : 0.0) << ",\n"
        << "    \"pure_elapsed_div_nc_2lmc_total_with_training\": "
        << tool::num(lv + training_ms > 0 ? pure_ms / (lv + training_ms) : 0.0) << ",\n";
    }
    j << "    \"pure_elapsed_div_nc_inference_elapsed\": " << tool::num(hybrid_ms > 0 ? pure_ms / hybrid_ms : 0.0)
      << ",\n"
      << "    \"pure_elapsed_div_nc_total_with_training\": "
      << tool::num(hybrid_ms + training_ms > 0 ? pure_ms / (hybrid_ms + training_ms) : 0.0) << ",\n"
      << "    \"training_cost_counted_in_total_speedup\": true\n"
      << "  }\n"
      << "}\n";
    tool::write_text(o.output, j.str());
    std::cout << "wrote " << o.output << "\n"
              << "pure RMSE " << sp.rmse << " in " << pure_ms << " ms\n"
              << "NC+WoS RMSE " << sh.rmse << " in " << hybrid_ms << " ms\n";
    if (o.enable_2lmc) std::cout << "NC+2LMC RMSE " << tl.rmse << " in " << (coarse_ms + residual_ms) << " ms\n";
    return 0;
  });
}
