// n2wos_probe_tcnn_cache: trains the hash-grid + MLP cache on the harmonic
// target x^2 - y^2 over [-1,1]^3 (fed as unit-cube coordinates) and times
// device-resident inference with and without a downstream consumer.
//
// Flags, JSON schema (n2wos_tcnn_cache_probe_v1) and the protocol (fresh
// device-generated batch per training step, warm-ups, repeated timed
// inference, validation of every repeat by the consumer) follow
// src/tools/probe_tcnn_cache.cu: options 73-93, protocol 311-433, JSON 435-507.
// The cache is this library's (n2w_cache_*); there is no tiny-cuda-nn.  The
// consumer is two device kernels (analytic target, FP64 error sums) where the
// reference fuses one.
#include "common.hpp"

namespace {

struct Options {
  int samples = 262144;
  int batch_size = 262144;
  int train_steps = 200;
  int repeat = 20;
  int warmup = 3;
  int seed = 12345;
  std::string network = "FullyFusedMLP";
  int n_levels = 12;
  int n_features_per_level = 2;
  int log2_hashmap_size = 18;
  int base_resolution = 8;
  float per_level_scale = 1.5f;
  int n_neurons = 32;
  int n_hidden_layers = 2;
  float learning_rate = 1.0e-2f;
  int jit = 0;
  std::string output = "results/probe_tcnn_cache.json";
};

void usage(std::ostream& out, const char* argv0) {
  out << "Usage: " << argv0 << " [options]\n\n"
      << "Options:\n"
      << "  --samples <int>                Inference sample count [262144]\n"
      << "  --batch-size <int>             Training batch size [262144]\n"
      << "  --train-steps <int>            Training steps [200]\n"
      << "  --repeat <int>                 Repeated inference timings [20]\n"
      << "  --warmup <int>                 Untimed inference warmups [3]\n"
      << "  --seed <int>                   GPU sample-generation seed [12345]\n"
      << "  --network FullyFusedMLP|CutlassMLP [FullyFusedMLP] (both select the n2w MLP)\n"
      << "  --n-levels <int>               HashGrid levels [12]\n"
      << "  --n-features-per-level <int>   HashGrid features per level [2]\n"
      << "  --log2-hashmap-size <int>      HashGrid log2 hashmap size [18]\n"
      << "  --base-resolution <int>        HashGrid base resolution [8]\n"
      << "  --per-level-scale <float>      HashGrid scale per level [1.5]\n"
      << "  --n-neurons <int>              MLP neurons per hidden layer [32]\n"
      << "  --n-hidden-layers <int>        MLP hidden layers [2]\n"
      << "  --learning-rate <float>        Adam learning rate [1e-2]\n"
      << "  --jit 0|1                      Accepted for compatibility; no JIT fusion here [0]\n"
      << "  --output <path>                JSON output [results/probe_tcnn_cache.json]\n"
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
    } else if (a == "--samples") o.samples = tool::parse_int(val(), a);
    else if (a == "--batch-size") o.batch_size = tool::parse_int(val(), a);
    else if (a == "--train-steps") o.train_steps = tool::parse_int(val(), a);
    else if (a == "--repeat") o.repeat = tool::parse_int(val(), a);
    else if (a == "--warmup") o.warmup = tool::parse_int(val(), a);
    else if (a == "--seed") o.seed = tool::parse_int(val(), a);
    else if (a == "--network") o.network = val();
    else if (a == "--n-levels") o.n_levels = tool::parse_int(val(), a);
    else if (a == "--n-features-per-level") o.n_features_per_level = tool::parse_int(val(), a);
    else if (a == "--log2-hashmap-size") o.log2_hashmap_size = tool::parse_int(val(), a);
    else if (a == "--base-resolution") o.base_resolution = tool::parse_int(val(), a);
    else if (a == "--per-level-scale") o.per_level_scale = tool::parse_float(val(), a);
    else if (a == "--n-neurons") o.n_neurons = tool::parse_int(val(), a);
    else if (a == "--n-hidden-layers") o.n_hidden_layers = tool::parse_int(val(), a);
    else if (a == "--learning-rate") o.learning_rate = tool::parse_float(val(), a);
    else if (a == "--jit") o.jit = tool::parse_int(val(), a);
    else if (a == "--output") o.output = val();
    else throw std::runtime_error("unknown argument: " + a);
  }
  if (o.samples <= 0 || o.batch_size <= 0 || o.train_steps < 0 || o.repeat <= 0 || o.warmup < 0) {
    throw std::runtime_error(
        "samples, batch-size, repeat must be positive; train-steps and warmup must be nonnegative");
  }
  if (o.network != "FullyFusedMLP" && o.network != "CutlassMLP") {
    throw std::runtime_error("--network must be FullyFusedMLP or CutlassMLP");
  }
  return o;
}

}  // namespace

int main(int argc, char** argv) {
  return tool::run_main([&]() -> int {
    const Options o = parse(argc, argv);
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

    // Target u = x^2 - y^2 at x = -1 + 2 * input (the reference's unit-cube harmonic target).
    n2w_problem pb{};
    N2W_CHECK(n2w_problem_reference_mode(N2W_BC_HARMONIC_X2_MINUS_Y2, N2W_SOURCE_CENTER, &pb));
    const float in_min[3] = {-1.0f, -1.0f, -1.0f}, in_ext[3] = {2.0f, 2.0f, 2.0f};
    const size_t nb = o.batch_size, ns = o.samples;
    tool::Stream stream;
    tool::DeviceArray<float> tr_in(3 * nb), tr_t(nb), inf_in(3 * ns), inf_out(ns), exact(ns);
    tool::DeviceArray<double> acc(4 * static_cast<size_t>(o.repeat));
    acc.zero(stream.s);
    const uint64_t seed = static_cast<uint64_t>(static_cast<uint32_t>(o.seed));
    N2W_CHECK(n2w_fill_unit_samples(&pb, static_cast<int64_t>(ns), seed ^ 0xa341316cull, 0, in_min, in_ext, inf_in.p,
                                    nullptr, stream.s));

    tool::Timer timer;
    float train_ms = 0.0f;
    if (o.train_steps > 0) {
      timer.start(stream.s);
      for (int s = 0; s < o.train_steps; ++s) {
        N2W_CHECK(n2w_fill_unit_samples(&pb, static_cast<int64_t>(nb), seed, static_cast<uint32_t>(s), in_min, in_ext,
                                        tr_in.p, tr_t.p, stream.s));
        N2W_CHECK(n2w_cache_train_step(cache, tr_in.p, tr_t.p, static_cast<int64_t>(nb), nullptr, stream.s));
      }
      train_ms = timer.stop_ms(stream.s);
    }
    for (int i = 0; i < o.warmup; ++i) {
      N2W_CHECK(n2w_cache_infer(cache, inf_in.p, static_cast<int64_t>(ns), inf_out.p, stream.s));
    }
    stream.sync();
    std::vector<float> inf_ms, cons_ms;
    for (int r = 0; r < o.repeat; ++r) {
      timer.start(stream.s);
      N2W_CHECK(n2w_cache_infer(cache, inf_in.p, static_cast<int64_t>(ns), inf_out.p, stream.s));
      inf_ms.push_back(timer.stop_ms(stream.s));
    }
    for (int r = 0; r < o.repeat; ++r) {
      timer.start(stream.s);
      N2W_CHECK(n2w_cache_infer(cache, inf_in.p, static_cast<int64_t>(ns), inf_out.p, stream.s));
      N2W_CHECK(n2w_oracle_cache_infer(&pb, inf_in.p, static_cast<int64_t>(ns), in_min, in_ext, exact.p, stream.s));
      N2W_CHECK(n2w_compare_accumulate(inf_out.p, exact.p, static_cast<int64_t>(ns), acc.p + 4 * r, stream.s));
      cons_ms.push_back(timer.stop_ms(stream.s));
    }
    const std::vector<double> h = acc.to_host(4 * static_cast<size_t>(o.repeat), stream.s);
    double sp = 0, se = 0, ssq = 0, sab = 0;
    for (int r = 0; r < o.repeat; ++r) {
      sp += h[4 * r];
      se += h[4 * r + 1];
      ssq += h[4 * r + 2];
      sab += h[4 * r + 3];
    }
    const double denom = static_cast<double>(ns) * o.repeat;
    const double mse = ssq / denom;
    const float inf_med = tool::median(inf_ms), cons_med = tool::median(cons_ms);
    const double us_per_sample = 1000.0 * inf_med / ns;
    int64_t grid_params = 0, mlp_params = 0;
    n2w_cache_config got{};
    N2W_CHECK(n2w_cache_info(cache, &got, &grid_params, &mlp_params, nullptr, nullptr));

    std::ostringstream j;
    j << "{\n"
      << "  \"schema\": \"n2wos_tcnn_cache_probe_v1\",\n"
      << "  \"patch\": \"n2w-sm100a-hashgrid-mlp-cache-probe\",\n"
      << "  \"generated_at_utc\": " << tool::json_quote(tool::utc_now()) << ",\n"
      << "  \"command_line\": " << tool::json_quote(tool::join_argv(argc, argv)) << ",\n"
      << "  \"cuda\": " << tool::cuda_json() << ",\n"
      << "  \"implementation_mode\": {\n"
      << "    \"cache_backend\": \"n2w_hashgrid_mlp_native\",\n"
      << "    \"mlp_arithmetic\": \"fp16 mma.sync m16n8k16, fp32 accumulate, fp32 Adam master weights\",\n"
      << "    \"python_bindings\": false,\n"
      << "    \"csv_postprocess\": false,\n"
      << "    \"training_batch_generation\": \"cuda_kernel\",\n"
      << "    \"training_inputs_location\": \"cuda_device_memory\",\n"
      << "    \"training_targets_location\": \"cuda_device_memory\",\n"
      << "    \"inference_inputs_location\": \"cuda_device_memory\",\n"
      << "    \"inference_outputs_location\": \"cuda_device_memory\",\n"
      << "    \"downstream_consumer\": \"cuda_kernels\",\n"
      << "    \"host_transfer_between_tcnn_and_consumer\": false,\n"
      << "    \"timing_scope\": \"cuda_events; inference timing excludes final validation readback\"\n"
      << "  },\n"
      << "  \"options\": {\n"
      << "    \"samples\": " << o.samples << ",\n"
      << "    \"samples_padded_to_tcnn_granularity\": " << o.samples << ",\n"
      << "    \"batch_size\": " << o.batch_size << ",\n"
      << "    \"batch_size_padded_to_tcnn_granularity\": " << o.batch_size << ",\n"
      << "    \"train_steps\": " << o.train_steps << ",\n"
      << "    \"repeat\": " << o.repeat << ",\n"
      << "    \"warmup\": " << o.warmup << ",\n"
      << "    \"seed\": " << o.seed << ",\n"
      << "    \"target_function\": \"harmonic_x2_minus_y2_on_unit_cube_coordinates\",\n"
      << "    \"network\": " << tool::json_quote(o.network) << ",\n"
      << "    \"jit_requested\": " << (o.jit ? "true" : "false") << ",\n"
      << "    \"jit_supported\": false,\n"
      << "    \"jit_enabled\": false,\n"
      << "    \"n_levels\": " << o.n_levels << ",\n"
      << "    \"n_features_per_level\": " << o.n_features_per_level << ",\n"
      << "    \"log2_hashmap_size\": " << o.log2_hashmap_size << ",\n"
      << "    \"base_resolution\": " << o.base_resolution << ",\n"
      << "    \"per_level_scale\": " << tool::num(o.per_level_scale) << ",\n"
      << "    \"n_neurons\": " << o.n_neurons << ",\n"
      << "    \"n_hidden_layers\": " << o.n_hidden_layers << ",\n"
      << "    \"learning_rate\": " << tool::num(o.learning_rate) << ",\n"
      << "    \"grid_params\": " << grid_params << ",\n"
      << "    \"mlp_params\": " << mlp_params << "\n"
      << "  },\n"
      << "  \"training\": {\n"
      << "    \"total_ms\": " << tool::num(train_ms) << ",\n"
      << "    \"ms_per_step\": " << tool::num(o.train_steps > 0 ? train_ms / o.train_steps : 0.0f) << ",\n"
      << "    \"includes_gpu_batch_generation\": true,\n"
      << "    \"host_readback_in_training_loop\": false\n"
      << "  },\n"
      << "  \"inference\": {\n"
      << "    \"kernel_ms\": " << tool::floats_json(inf_ms) << ",\n"
      << "    \"kernel_ms_median\": " << tool::num(inf_med) << ",\n"
      << "    \"kernel_ms_mean\": " << tool::num(tool::mean(inf_ms)) << ",\n"
      << "    \"median_us_per_sample\": " << tool::num(us_per_sample) << ",\n"
      << "    \"median_msamples_per_second\": " << tool::num(ns / (1000.0 * inf_med)) << "\n"
      << "  },\n"
      << "  \"inference_plus_downstream_consumer\": {\n"
      << "    \"kernel_ms\": " << tool::floats_json(cons_ms) << ",\n"
      << "    \"kernel_ms_median\": " << tool::num(cons_med) << ",\n"
      << "    \"kernel_ms_mean\": " << tool::num(tool::mean(cons_ms)) << ",\n"
      << "    \"median_us_per_sample\": " << tool::num(1000.0 * cons_med / ns) << ",\n"
      << "    \"host_transfer_between_stages\": false\n"
      << "  },\n"
      << "  \"validation\": {\n"
      << "    \"checked_repeated_samples\": " << static_cast<unsigned long long>(ns) * o.repeat << ",\n"
      << "    \"mean_prediction\": " << tool::num(sp / denom) << ",\n"
      << "    \"mean_exact\": " << tool::num(se / denom) << ",\n"
      << "    \"mse\": " << tool::num(mse) << ",\n"
      << "    \"rmse\": " << tool::num(std::sqrt(mse)) << ",\n"
      << "    \"mae\": " << tool::num(sab / denom) << "\n"
      << "  }\n"
      << "}\n";
    tool::write_text(o.output, j.str());
    std::cout << "wrote " << o.output << "\n"
              << "median inference: " << us_per_sample << " us/sample\n"
              << "RMSE after training: " << std::sqrt(mse) << "\n";
    return 0;
  });
}
