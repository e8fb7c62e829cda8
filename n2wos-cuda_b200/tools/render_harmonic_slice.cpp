// n2wos_render_harmonic_slice: WoS estimate of u = x^2 - y^2 on a planar slice
// through the mesh, written as CSV, five PPM heat maps and a JSON summary.
//
// Flags, file formats and the JSON schema (n2wos_harmonic_slice_render_v2)
// follow src/tools/render_harmonic_slice.cu: options 126-180, CSV columns
// 242-258, heat-map colour rules 260-340, JSON 365-450; the slice frame, pixel
// grid and per-pixel statistics follow src/cuda/cubql_bvh.cu:963-1152.
//
// Differences, by design: the inside mask is computed on the device by +x ray
// parity over the BVH (the reference tests every triangle on the host), only
// inside pixels launch walks, and per-pixel statistics are FP64 reductions on
// the device instead of per-sample arrays reduced on the host.
#include <limits>

#include "common.hpp"

namespace {

struct Options {
  tool::MeshOptions mesh;
  int width = 128;
  int height = 128;
  int samples_per_pixel = 256;
  std::string view = "xy";
  float plane_z = 0.0f;
  bool use_mesh_bounds = true;
  bool preserve_world_aspect = true;
  float frame[4] = {-1.0f, 1.0f, -1.0f, 1.0f};
  float padding_fraction = 0.02f;
  bool mask_outside_mesh = true;
  int max_steps = 256;
  float epsilon = 1.0e-4f;
  float step_scale = 0.999f;
  uint64_t seed = 12345;
  int block_size = 128;
  int leaf_size = 8;
  std::string build_method = "sah";
  std::string output_prefix = "results/harmonic_slice";
};

void usage(const char* argv0) {
  std::cerr << "usage: " << argv0 << " [options]\n"
            << "  --mesh procedural_bumpy_sphere|obj|ply\n"
            << "  --mesh-path PATH\n"
            << "  --normalize 0|1 --bumpy-stacks N --bumpy-slices N --bumpy-amplitude A\n"
            << "  --width N --height N\n"
            << "  --samples-per-pixel N\n"
            << "  --view xy|xz|yz\n"
            << "  --plane-z Z      fixed coordinate: z for xy, y for xz, x for yz\n"
            << "  --frame u_min,u_max,v_min,v_max   overrides mesh bounds for selected view\n"
            << "  --padding-fraction F\n"
            << "  --preserve-world-aspect 0|1\n"
            << "  --mask-outside-mesh 0|1\n"
            << "  --max-steps N --epsilon EPS --step-scale S --seed N --block-size N\n"
            << "  --cubql-build-method sah|spatial_median --cubql-leaf-size N\n"
            << "  --output-prefix PATH_PREFIX\n";
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
    } else if (a == "--width") o.width = tool::parse_int(val(), a);
    else if (a == "--height") o.height = tool::parse_int(val(), a);
    else if (a == "--samples-per-pixel" || a == "--spp") o.samples_per_pixel = tool::parse_int(val(), a);
    else if (a == "--view") {
      o.view = val();
      if (o.view != "xy" && o.view != "xz" && o.view != "yz") throw std::runtime_error("--view must be one of: xy, xz, yz");
    } else if (a == "--plane-z" || a == "--plane") o.plane_z = tool::parse_float(val(), a);
    else if (a == "--frame") {
      const auto f = tool::parse_float_list(val(), 4, "--frame");
      for (int k = 0; k < 4; ++k) o.frame[k] = f[k];
      o.use_mesh_bounds = false;
    } else if (a == "--padding-fraction") o.padding_fraction = tool::parse_float(val(), a);
    else if (a == "--preserve-world-aspect") o.preserve_world_aspect = tool::parse_int(val(), a) != 0;
    else if (a == "--mask-outside-mesh") o.mask_outside_mesh = tool::parse_int(val(), a) != 0;
    else if (a == "--max-steps") o.max_steps = tool::parse_int(val(), a);
    else if (a == "--epsilon") o.epsilon = tool::parse_float(val(), a);
    else if (a == "--step-scale") o.step_scale = tool::parse_float(val(), a);
    else if (a == "--seed") o.seed = tool::parse_u64(val(), a);
    else if (a == "--block-size") o.block_size = tool::parse_int(val(), a);
    else if (a == "--cubql-leaf-size") o.leaf_size = tool::parse_int(val(), a);
    else if (a == "--cubql-build-method") o.build_method = val();
    else if (a == "--output-prefix") o.output_prefix = val();
    else throw std::runtime_error("unknown argument: " + a);
  }
  o.mesh.validate();
  if (o.width <= 0 || o.height <= 0 || o.samples_per_pixel <= 0) {
    throw std::runtime_error("width, height and samples-per-pixel must be positive");
  }
  if (o.max_steps <= 0 || !(o.epsilon > 0.0f)) throw std::runtime_error("invalid WoS options");
  return o;
}

struct Pixel {
  float x = 0, y = 0, z = 0;
  bool inside = false;
  int samples = 0;
  double mean = 0, exact = 0, error = 0, stderr_ = 0, variance = 0, mean_steps = 0;
  long long forced = 0, overflow = 0;
};

struct Rgb {
  unsigned char r, g, b;
};

unsigned char to_byte(double x) { return static_cast<unsigned char>(std::lround(255.0 * std::clamp(x, 0.0, 1.0))); }

// Grey ramp over [vmin, vmax]; dark grey for non-finite, mid grey for an empty range.
Rgb grey(double v, double vmin, double vmax) {
  if (!std::isfinite(v)) return {30, 30, 30};
  if (!(vmax > vmin)) return {128, 128, 128};
  const unsigned char c = to_byte((v - vmin) / (vmax - vmin));
  return {c, c, c};
}

// Blue (negative) - white - red (positive), saturating at |v| = max_abs.
Rgb diverging(double v, double max_abs) {
  if (!std::isfinite(v)) return {30, 30, 30};
  if (!(max_abs > 0.0)) return {255, 255, 255};
  const double t = std::clamp(v / max_abs, -1.0, 1.0);
  if (t < 0.0) return {to_byte(1.0 + t), to_byte(1.0 + t), 255};
  return {255, to_byte(1.0 - t), to_byte(1.0 - t)};
}

void write_ppm(const std::string& path, int w, int h, const std::vector<Rgb>& px) {
  tool::ensure_parent_dir(path);
  std::ofstream f(path, std::ios::binary);
  if (!f) throw std::runtime_error("failed to open PPM for writing: " + path);
  f << "P6\n" << w << " " << h << "\n255\n";
  f.write(reinterpret_cast<const char*>(px.data()), static_cast<std::streamsize>(px.size() * 3));
}

// Row 0 of the slice (v_min) is the bottom row of the image.
void write_heatmaps(const std::string& prefix, int w, int h, const std::vector<Pixel>& px) {
  double emin = INFINITY, emax = -INFINITY, smin = INFINITY, smax = -INFINITY, sd_max = 0, err_max = 0;
  for (const Pixel& p : px) {
    if (!p.inside) continue;
    emin = std::min(emin, p.exact);
    emax = std::max(emax, p.exact);
    smin = std::min(smin, p.mean);
    smax = std::max(smax, p.mean);
    sd_max = std::max(sd_max, p.stderr_);
    err_max = std::max(err_max, std::fabs(p.error));
  }
  const double vmin = std::min(emin, smin), vmax = std::max(emax, smax);
  const size_t n = static_cast<size_t>(w) * h;
  std::vector<Rgb> mask(n), exact(n), est(n), err(n), sd(n);
  for (int iy = 0; iy < h; ++iy) {
    for (int ix = 0; ix < w; ++ix) {
      const Pixel& p = px[static_cast<size_t>(iy) * w + ix];
      const size_t d = static_cast<size_t>(h - 1 - iy) * w + ix;
      if (!p.inside) {
        mask[d] = exact[d] = est[d] = err[d] = sd[d] = Rgb{20, 20, 20};
        continue;
      }
      mask[d] = {235, 235, 235};
      exact[d] = grey(p.exact, vmin, vmax);
      est[d] = grey(p.mean, vmin, vmax);
      err[d] = diverging(p.error, err_max);
      sd[d] = grey(p.stderr_, 0.0, sd_max);
    }
  }
  write_ppm(prefix + "_mask.ppm", w, h, mask);
  write_ppm(prefix + "_exact.ppm", w, h, exact);
  write_ppm(prefix + "_estimate.ppm", w, h, est);
  write_ppm(prefix + "_error.ppm", w, h, err);
  write_ppm(prefix + "_stderr.ppm", w, h, sd);
}

std::string csv_num(double v) {
  if (std::isnan(v)) return "nan";
  std::ostringstream o;
  o << std::setprecision(10) << v;
  return o.str();
}

}  // namespace

int main(int argc, char** argv) {
  return tool::run_main([&]() -> int {
    const Options o = parse(argc, argv);
    tool::Mesh mesh(o.mesh);
    tool::Bvh bvh(mesh, o.leaf_size, o.build_method);
    float b6[6];
    mesh.bounds(b6);
    const int W = o.width, H = o.height;
    const size_t npx = static_cast<size_t>(W) * H;
    std::vector<float> pts(3 * npx);
    float frame[4];
    N2W_CHECK(n2w_slice_points_ex(b6, o.use_mesh_bounds ? nullptr : o.frame, o.view.c_str(), o.plane_z, W, H,
                                  o.padding_fraction, o.preserve_world_aspect ? 1 : 0, N2W_SLICE_RULE_RENDER,
                                  pts.data(), frame));
    tool::Stream stream;
    tool::DeviceArray<n2w_vec3> d_px(npx);
    d_px.upload(reinterpret_cast<const n2w_vec3*>(pts.data()), npx, stream.s);
    std::vector<uint8_t> inside(npx, 1);
    if (o.mask_outside_mesh) {
      tool::DeviceArray<uint8_t> d_in(npx);
      tool::DeviceArray<int> d_ov(1);
      d_ov.zero(stream.s);
      N2W_CHECK(n2w_bvh_inside_device(bvh.b, d_px.p, static_cast<int>(npx), d_in.p, d_ov.p, 256, stream.s));
      inside = d_in.to_host(npx, stream.s);
      if (d_ov.to_host(1, stream.s)[0]) throw std::runtime_error("inside test: traversal stack overflow");
    }
    std::vector<float> ipts;
    std::vector<size_t> ids;
    for (size_t i = 0; i < npx; ++i) {
      if (!inside[i]) continue;
      ids.push_back(i);
      ipts.insert(ipts.end(), {pts[3 * i], pts[3 * i + 1], pts[3 * i + 2]});
    }
    const size_t nin = ids.size();

    n2w_problem pb{};
    N2W_CHECK(n2w_problem_reference_mode(N2W_BC_HARMONIC_X2_MINUS_Y2, N2W_SOURCE_CENTER, &pb));
    tool::PointStats st(std::max<size_t>(nin, 1));
    tool::DeviceArray<n2w_vec3> d_in_pts(std::max<size_t>(nin, 1));
    tool::DeviceArray<n2w_walk_counters> d_c(1);
    d_c.zero(stream.s);
    float ms = 0.0f;
    if (nin) {
      d_in_pts.upload(reinterpret_cast<const n2w_vec3*>(ipts.data()), nin, stream.s);
      n2w_walk_options wo{};
      wo.walks_per_point = o.samples_per_pixel;
      wo.max_steps = o.max_steps;
      wo.epsilon = o.epsilon;
      wo.step_scale = o.step_scale;
      wo.seed = o.seed;
      wo.block_size = tool::walker_block(o.block_size);
      tool::Timer timer;
      timer.start(stream.s);
      N2W_CHECK(n2w_wos_estimate(bvh.b, &pb, d_in_pts.p, static_cast<int64_t>(nin), &wo, st.view(), d_c.p, nullptr,
                                 stream.s));
      ms = timer.stop_ms(stream.s);
    }
    const n2w_walk_counters c = d_c.to_host(1, stream.s)[0];
    const auto h = st.to_host(stream.s);

    std::vector<Pixel> px(npx);
    const double qnan = std::numeric_limits<double>::quiet_NaN();
    for (size_t i = 0; i < npx; ++i) {
      Pixel& p = px[i];
      p.x = pts[3 * i];
      p.y = pts[3 * i + 1];
      p.z = pts[3 * i + 2];
      p.exact = static_cast<double>(p.x) * p.x - static_cast<double>(p.y) * p.y;
      p.mean = p.error = p.variance = p.stderr_ = p.mean_steps = qnan;
    }
    double sum_abs = 0, sum_sq = 0, max_abs = 0;
    long long forced_total = 0;
    for (size_t k = 0; k < nin; ++k) {
      Pixel& p = px[ids[k]];
      p.inside = true;
      p.samples = static_cast<int>(h.count[k]);
      p.mean = h.mean(k);
      p.variance = h.variance(k);
      p.stderr_ = std::sqrt(p.variance / std::max<uint32_t>(h.count[k], 1));
      p.mean_steps = h.mean_steps(k);
      p.forced = h.forced[k];
      // Traversal overflows are counted per run, not per pixel: -1 marks "unknown" when any occurred.
      p.overflow = c.overflow ? -1 : 0;
      p.error = p.mean - p.exact;
      sum_abs += std::fabs(p.error);
      sum_sq += p.error * p.error;
      max_abs = std::max(max_abs, std::fabs(p.error));
      forced_total += p.forced;
    }

    {
      const std::string path = o.output_prefix + ".csv";
      tool::ensure_parent_dir(path);
      std::ofstream f(path);
      if (!f) throw std::runtime_error("failed to open CSV for writing: " + path);
      f << "ix,iy,x,y,z,inside,samples,mean,exact,error,stderr,sample_variance,mean_steps,forced_max_steps,"
           "overflow_count\n";
      for (int iy = 0; iy < H; ++iy) {
        for (int ix = 0; ix < W; ++ix) {
          const Pixel& p = px[static_cast<size_t>(iy) * W + ix];
          f << ix << ',' << iy << ',' << csv_num(p.x) << ',' << csv_num(p.y) << ',' << csv_num(p.z) << ','
            << (p.inside ? 1 : 0) << ',' << p.samples << ',' << csv_num(p.mean) << ',' << csv_num(p.exact) << ','
            << csv_num(p.error) << ',' << csv_num(p.stderr_) << ',' << csv_num(p.variance) << ','
            << csv_num(p.mean_steps) << ',' << p.forced << ',' << p.overflow << '\n';
        }
      }
    }
    write_heatmaps(o.output_prefix, W, H, px);

    const double total_samples = static_cast<double>(npx) * o.samples_per_pixel;
    const auto& bs = bvh.stats;
    const std::string P = o.output_prefix;
    std::ostringstream j;
    j << "{\n"
      << "  \"schema\": \"n2wos_harmonic_slice_render_v2\",\n"
      << "  \"patch\": \"n2w-sm100a-slice-render\",\n"
      << "  \"generated_at_utc\": " << tool::json_quote(tool::utc_now()) << ",\n"
      << "  \"command_line\": " << tool::json_quote(tool::join_argv(argc, argv)) << ",\n"
      << "  \"cuda\": " << tool::cuda_json() << ",\n"
      << "  \"implementation_mode\": {\n"
      << "    \"engine\": \"n2w_persistent_walker_inside_pixels_only\",\n"
      << "    \"geometry_backend\": \"n2w_sm100a_bvh\",\n"
      << "    \"geometry_build_method\": " << tool::json_quote(o.build_method) << ",\n"
      << "    \"inside_mask\": \"device_ray_parity_x_over_bvh\",\n"
      << "    \"pixel_reduction\": \"device_fp64_per_pixel\",\n"
      << "    \"cpu_gpu_transfer_inside_sampling_loop\": false,\n"
      << "    \"host_controls_global_step_loop\": false,\n"
      << "    \"field_rendering_role\": \"visual_diagnostic_not_final_time_to_mse_benchmark\"\n"
      << "  },\n"
      << "  \"options\": {\n"
      << "    \"mesh\": " << tool::json_quote(o.mesh.mesh) << ",\n"
      << "    \"mesh_path\": " << tool::json_quote(o.mesh.mesh_path) << ",\n"
      << "    \"normalize\": " << (o.mesh.normalize ? "true" : "false") << ",\n"
      << "    \"width\": " << W << ",\n"
      << "    \"height\": " << H << ",\n"
      << "    \"samples_per_pixel\": " << o.samples_per_pixel << ",\n"
      << "    \"slice_view\": " << tool::json_quote(o.view) << ",\n"
      << "    \"plane_z\": " << tool::num(o.plane_z) << ",\n"
      << "    \"plane_z_note\": \"fixed coordinate: z for xy, y for xz, x for yz\",\n"
      << "    \"preserve_world_aspect\": " << (o.preserve_world_aspect ? "true" : "false") << ",\n"
      << "    \"mask_outside_mesh\": " << (o.mask_outside_mesh ? "true" : "false") << ",\n"
      << "    \"max_steps\": " << o.max_steps << ",\n"
      << "    \"epsilon\": " << tool::num(o.epsilon) << ",\n"
      << "    \"step_scale\": " << tool::num(o.step_scale) << ",\n"
      << "    \"seed\": " << o.seed << "\n"
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
      << "  \"outputs\": {\n"
      << "    \"csv\": " << tool::json_quote(P + ".csv") << ",\n"
      << "    \"mask_ppm\": " << tool::json_quote(P + "_mask.ppm") << ",\n"
      << "    \"exact_ppm\": " << tool::json_quote(P + "_exact.ppm") << ",\n"
      << "    \"estimate_ppm\": " << tool::json_quote(P + "_estimate.ppm") << ",\n"
      << "    \"error_ppm\": " << tool::json_quote(P + "_error.ppm") << ",\n"
      << "    \"stderr_ppm\": " << tool::json_quote(P + "_stderr.ppm") << "\n"
      << "  },\n"
      << "  \"slice_frame\": {\n"
      << "    \"view\": " << tool::json_quote(o.view) << ",\n"
      << "    \"u_min\": " << tool::num(frame[0]) << ",\n"
      << "    \"u_max\": " << tool::num(frame[1]) << ",\n"
      << "    \"v_min\": " << tool::num(frame[2]) << ",\n"
      << "    \"v_max\": " << tool::num(frame[3]) << ",\n"
      << "    \"world_units_per_pixel_u\": "
      << tool::num(W > 1 ? static_cast<double>(frame[1] - frame[0]) / (W - 1) : 0.0) << ",\n"
      << "    \"world_units_per_pixel_v\": "
      << tool::num(H > 1 ? static_cast<double>(frame[3] - frame[2]) / (H - 1) : 0.0) << "\n"
      << "  },\n"
      << "  \"summary\": {\n"
      << "    \"inside_pixels\": " << nin << ",\n"
      << "    \"elapsed_ms\": " << tool::num(ms) << ",\n"
      << "    \"us_per_active_pixel\": " << tool::num(nin ? 1000.0 * ms / nin : 0.0) << ",\n"
      << "    \"us_per_launched_sample\": " << tool::num(1000.0 * ms / total_samples) << ",\n"
      << "    \"us_per_walked_sample\": "
      << tool::num(nin ? 1000.0 * ms / (static_cast<double>(nin) * o.samples_per_pixel) : 0.0) << ",\n"
      << "    \"rmse_inside\": " << tool::num(nin ? std::sqrt(sum_sq / nin) : 0.0) << ",\n"
      << "    \"mae_inside\": " << tool::num(nin ? sum_abs / nin : 0.0) << ",\n"
      << "    \"max_abs_error_inside\": " << tool::num(max_abs) << ",\n"
      << "    \"forced_max_steps\": " << forced_total << ",\n"
      << "    \"overflow_count\": " << c.overflow << "\n"
      << "  }\n"
      << "}\n";
    tool::write_text(P + ".json", j.str());
    std::cout << "wrote " << P << ".json/.csv and PPM heatmaps\n";
    return 0;
  });
}
