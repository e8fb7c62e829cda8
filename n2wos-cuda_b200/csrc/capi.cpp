// Error reporting, boundary-value problem helpers and thin CUDA runtime
// helpers of the C ABI.
#include <cuda_runtime.h>

#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>

#include "internal.hpp"
#include "philox.cuh"
#include "problem.cuh"

namespace n2w {
namespace {
thread_local std::string g_last_error;

struct ModeName {
  int mode;
  const char* canonical;
  const char* aliases[6];
};

// Canonical names and CLI aliases (reference src/cuda/cubql_bvh.cu:1704-1800).
const ModeName kModes[] = {
    {N2W_BC_HARMONIC_X2_MINUS_Y2, "harmonic_x2_minus_y2", {"harmonic", nullptr}},
    {N2W_BC_EXTERNAL_CHARGES_MEDIUM, "external_charges_medium", {"medium", "charges_medium", nullptr}},
    {N2W_BC_EXTERNAL_CHARGES_HIGH, "external_charges_high", {"high", "charges_high", nullptr}},
    {N2W_BC_HARMONIC_ZEBRA_K4, "harmonic_zebra_k4", {"zebra4", nullptr}},
    {N2W_BC_HARMONIC_ZEBRA_K8, "harmonic_zebra_k8", {"zebra8", nullptr}},
    {N2W_BC_HARMONIC_ZEBRA_K12, "harmonic_zebra_k12", {"zebra12", nullptr}},
    {N2W_BC_EXTERNAL_CHARGES_SHELL_K8, "external_charges_shell_k8", {"shell8", "charges_shell_k8", nullptr}},
    {N2W_BC_EXTERNAL_CHARGES_SHELL_K16, "external_charges_shell_k16", {"shell16", "charges_shell_k16", nullptr}},
    {N2W_BC_TEXTURE_STRIPES_K8, "boundary_texture_stripes_k8", {"texture_stripes_k8", "stripes8", "stripes_k8", nullptr}},
    {N2W_BC_TEXTURE_STRIPES_K16, "boundary_texture_stripes_k16", {"texture_stripes_k16", "stripes16", "stripes_k16", nullptr}},
    {N2W_BC_TEXTURE_CHECKER_K8, "boundary_texture_checker_k8", {"texture_checker_k8", "checker8", "checker_k8", nullptr}},
    {N2W_BC_TEXTURE_CHECKER_K16, "boundary_texture_checker_k16", {"texture_checker_k16", "checker16", "checker_k16", nullptr}},
    {N2W_BC_CONSTANT_ONE, "constant_one", {"constant", "one", "const1", nullptr}},
    {N2W_BC_HARMONIC_MIXTURE_SMOOTH, "harmonic_mixture_smooth", {"mixture_smooth", "hm_smooth", "fig_smooth", nullptr}},
    {N2W_BC_HARMONIC_MIXTURE_FIGLIKE, "harmonic_mixture_figlike",
     {"mixture_figlike", "hm_figlike", "figlike", "fig1", "fig4", nullptr}},
    {N2W_BC_HARMONIC_MIXTURE_MULTISCALE, "harmonic_mixture_multiscale",
     {"mixture_multiscale", "hmix_multiscale", "multiscale", nullptr}},
    {N2W_BC_HARMONIC_MIXTURE_FIGLIKE_HF, "harmonic_mixture_figlike_hf",
     {"mixture_figlike_hf", "hmix_figlike_hf", "figlike_hf", "fig_hf", nullptr}},
    {N2W_BC_POISSON_MULTISCALE, "poisson_multiscale",
     {"manufactured_poisson_multiscale", "poisson_mscale", "poisson", nullptr}},
    {N2W_BC_POISSON_FIGLIKE_HF, "poisson_figlike_hf", {"manufactured_poisson_figlike_hf", "poisson_hf", nullptr}},
    {N2W_BC_POISSON_FIGLIKE_HF_X5, "poisson_figlike_hf_x5", {"poisson_hf_x5", "poisson_figlike_x5", nullptr}},
    {N2W_BC_CHARGES_SEEDED, "charges_seeded", {"charges8_seeded", "seeded_charges", nullptr}},
    {N2W_BC_POISSON_SINPROD, "poisson_sinprod", {"sinprod", "manufactured_poisson_sinprod", nullptr}},
};

}  // namespace

void set_last_error(const std::string& msg) { g_last_error = msg; }

}  // namespace n2w

using namespace n2w;

namespace {
void copy_string(const std::string& s, char* buf, size_t cap) {
  N2W_REQUIRE(buf && cap > 0, "null buffer");
  std::snprintf(buf, cap, "%s", s.c_str());
}
}  // namespace

extern "C" {

const char* n2w_last_error(void) { return g_last_error.c_str(); }
int n2w_abi_version(void) { return N2W_ABI_VERSION; }

int n2w_cuda_runtime_version_string(char* buf, size_t cap) {
  return guarded([&] {
    int rt = 0, drv = 0;
    N2W_CUDA(cudaRuntimeGetVersion(&rt));
    N2W_CUDA(cudaDriverGetVersion(&drv));
    copy_string("runtime=" + std::to_string(rt) + ",driver=" + std::to_string(drv), buf, cap);
  });
}

int n2w_cuda_device_summary(char* buf, size_t cap) {
  return guarded([&] {
    int dev = 0;
    N2W_CUDA(cudaGetDevice(&dev));
    cudaDeviceProp prop{};
    N2W_CUDA(cudaGetDeviceProperties(&prop, dev));
    copy_string(std::string(prop.name) + " sm_" + std::to_string(prop.major) + std::to_string(prop.minor) +
                    " global_mem=" + std::to_string(static_cast<unsigned long long>(prop.totalGlobalMem)),
                buf, cap);
  });
}

// ---- problems ---------------------------------------------------------------
int n2w_problem_charges_seeded(int count, float r_min, float r_max, uint64_t seed, n2w_problem* out) {
  return guarded([&] {
    N2W_REQUIRE(out, "null output");
    N2W_REQUIRE(count >= 1 && count <= N2W_MAX_CHARGES, "count must be in [1, 16]");
    N2W_REQUIRE(r_min > 0.0f && r_max >= r_min, "require 0 < r_min <= r_max");
    std::memset(out, 0, sizeof(*out));
    out->mode = N2W_BC_CHARGES_SEEDED;
    out->source_sampling = N2W_SOURCE_BALL;
    out->charge_count = count;
    uint64_t s = seed;
    const double lo3 = static_cast<double>(r_min) * r_min * r_min;
    const double hi3 = static_cast<double>(r_max) * r_max * r_max;
    for (int k = 0; k < count; ++k) {
      // Direction: z uniform in [-1,1], azimuth uniform; radius uniform in volume.
      const double z = 2.0 * splitmix64_unit(s) - 1.0;
      const double phi = 2.0 * M_PI * splitmix64_unit(s);
      const double r = std::cbrt(lo3 + (hi3 - lo3) * splitmix64_unit(s));
      const double q = 2.0 * splitmix64_unit(s) - 1.0;
      const double rxy = std::sqrt(std::max(0.0, 1.0 - z * z));
      out->charges[k][0] = static_cast<float>(r * rxy * std::cos(phi));
      out->charges[k][1] = static_cast<float>(r * rxy * std::sin(phi));
      out->charges[k][2] = static_cast<float>(r * z);
      out->charges[k][3] = static_cast<float>(q);
    }
  });
}

int n2w_problem_sinprod(float omega, int source_sampling, n2w_problem* out) {
  return guarded([&] {
    N2W_REQUIRE(out, "null output");
    N2W_REQUIRE(source_sampling == N2W_SOURCE_BALL || source_sampling == N2W_SOURCE_CENTER, "bad source_sampling");
    std::memset(out, 0, sizeof(*out));
    out->mode = N2W_BC_POISSON_SINPROD;
    out->source_sampling = source_sampling;
    out->omega = omega;
  });
}

int n2w_problem_reference_mode(int mode, int source_sampling, n2w_problem* out) {
  return guarded([&] {
    N2W_REQUIRE(out, "null output");
    const bool ok = (mode >= 0 && mode <= 16) || mode == N2W_BC_POISSON_MULTISCALE || mode == N2W_BC_POISSON_FIGLIKE_HF ||
                    mode == N2W_BC_POISSON_FIGLIKE_HF_X5;
    N2W_REQUIRE(ok, "mode " + std::to_string(mode) + " is not a supported reference mode");
    N2W_REQUIRE(source_sampling == N2W_SOURCE_BALL || source_sampling == N2W_SOURCE_CENTER, "bad source_sampling");
    std::memset(out, 0, sizeof(*out));
    out->mode = mode;
    out->source_sampling = source_sampling;
  });
}

int n2w_problem_exact(const n2w_problem* problem, const double* xyz, int64_t n, double* u_out) {
  return guarded([&] {
    N2W_REQUIRE(problem && (n == 0 || (xyz && u_out)), "null argument");
    for (int64_t i = 0; i < n; ++i) u_out[i] = problem_u<double>(*problem, xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2]);
  });
}

int n2w_problem_eval_f32(const n2w_problem* problem, const float* xyz, int64_t n, float* g_out, float* f_out) {
  return guarded([&] {
    N2W_REQUIRE(problem && (n == 0 || xyz), "null argument");
    for (int64_t i = 0; i < n; ++i) {
      if (g_out) g_out[i] = problem_u<float>(*problem, xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2]);
      if (f_out) f_out[i] = problem_f<float>(*problem, xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2]);
    }
  });
}

int n2w_problem_mode_from_name(const char* name, int* mode_out) {
  return guarded([&] {
    N2W_REQUIRE(name && mode_out, "null argument");
    std::string s(name);
    for (char& c : s) c = static_cast<char>(std::tolower(static_cast<unsigned char>(c)));
    for (const auto& m : kModes) {
      if (s == m.canonical) {
        *mode_out = m.mode;
        return;
      }
      for (int k = 0; k < 6 && m.aliases[k]; ++k) {
        if (s == m.aliases[k]) {
          *mode_out = m.mode;
          return;
        }
      }
    }
    throw Error(N2W_EINVAL, "unknown boundary mode: " + s);
  });
}

const char* n2w_problem_mode_name(int mode) {
  for (const auto& m : kModes) {
    if (m.mode == mode) return m.canonical;
  }
  return "unknown";
}

int n2w_slice_points(const float* b, const char* view, float plane, int width, int height, float padding,
                     int preserve_aspect, float* points_out, float* frame_out) {
  return n2w_slice_points_ex(b, nullptr, view, plane, width, height, padding, preserve_aspect, N2W_SLICE_RULE_RENDER,
                             points_out, frame_out);
}

int n2w_slice_points_ex(const float* b, const float* frame_in, const char* view, float plane, int width, int height,
                        float padding, int preserve_aspect, int rule, float* points_out, float* frame_out) {
  return guarded([&] {
    N2W_REQUIRE(view && (b || frame_in), "null argument");
    N2W_REQUIRE(rule == N2W_SLICE_RULE_RENDER || rule == N2W_SLICE_RULE_EVAL, "bad pixel coordinate rule");
    N2W_REQUIRE(width > 0 && height > 0, "slice width/height must be positive");
    const std::string v(view);
    int ua, va, fa;
    if (v == "xy") { ua = 0; va = 1; fa = 2; }
    else if (v == "xz") { ua = 0; va = 2; fa = 1; }
    else if (v == "yz") { ua = 1; va = 2; fa = 0; }
    else throw Error(N2W_EINVAL, "slice view must be one of: xy, xz, yz");
    // Frame from the bounds, padded, then widened to the image aspect
    // (reference cubql_bvh.cu:90-112, 974-995), in the same float operations.
    float u_min, u_max, v_min, v_max;
    if (frame_in) {
      u_min = frame_in[0];
      u_max = frame_in[1];
      v_min = frame_in[2];
      v_max = frame_in[3];
    } else {
      const float du0 = b[3 + ua] - b[ua], dv0 = b[3 + va] - b[va];
      u_min = b[ua] - padding * du0;
      u_max = b[3 + ua] + padding * du0;
      v_min = b[va] - padding * dv0;
      v_max = b[3 + va] + padding * dv0;
    }
    if (preserve_aspect) {
      const float du = u_max - u_min, dv = v_max - v_min;
      if (du > 0.0f && dv > 0.0f) {
        const float image_aspect = static_cast<float>(width) / static_cast<float>(height);
        const float frame_aspect = du / dv;
        if (frame_aspect < image_aspect) {
          const float nd = image_aspect * dv, c = 0.5f * (u_min + u_max);
          u_min = c - 0.5f * nd;
          u_max = c + 0.5f * nd;
        } else if (frame_aspect > image_aspect) {
          const float nd = du / image_aspect, c = 0.5f * (v_min + v_max);
          v_min = c - 0.5f * nd;
          v_max = c + 0.5f * nd;
        }
      }
    }
    N2W_REQUIRE(u_max > u_min && v_max > v_min, "invalid slice frame");
    if (frame_out) {
      frame_out[0] = u_min;
      frame_out[1] = u_max;
      frame_out[2] = v_min;
      frame_out[3] = v_max;
    }
    if (!points_out) return;
    for (int iy = 0; iy < height; ++iy) {
      // The reference renderer scales by (i / (n-1)); its NC evaluator by (d * i) / (n-1).
      const float fy = static_cast<float>(iy), ny = static_cast<float>(height - 1);
      const float pv = height == 1 ? 0.5f * (v_min + v_max)
                       : rule == N2W_SLICE_RULE_RENDER ? v_min + (v_max - v_min) * (fy / ny)
                                                       : v_min + (v_max - v_min) * fy / ny;
      for (int ix = 0; ix < width; ++ix) {
        const float fx = static_cast<float>(ix), nx = static_cast<float>(width - 1);
        const float pu = width == 1 ? 0.5f * (u_min + u_max)
                         : rule == N2W_SLICE_RULE_RENDER ? u_min + (u_max - u_min) * (fx / nx)
                                                         : u_min + (u_max - u_min) * fx / nx;
        float* p = points_out + 3 * (static_cast<int64_t>(iy) * width + ix);
        p[ua] = pu;
        p[va] = pv;
        p[fa] = plane;
      }
    }
  });
}

int n2w_rng_philox4x32_10(const uint32_t* ctr, uint64_t seed, uint32_t tag, uint32_t* out) {
  return guarded([&] {
    N2W_REQUIRE(ctr && out, "null argument");
    uint32_t k0, k1;
    philox_key(seed, tag, k0, k1);
    const U4 r = philox4x32_10(U4{ctr[0], ctr[1], ctr[2], ctr[3]}, k0, k1);
    out[0] = r.x;
    out[1] = r.y;
    out[2] = r.z;
    out[3] = r.w;
  });
}

// ---- device helpers -----------------------------------------------------------
int n2w_device_count(int* out) {
  return guarded([&] {
    N2W_REQUIRE(out, "null output");
    N2W_CUDA(cudaGetDeviceCount(out));
  });
}
int n2w_set_device(int device) { return guarded([&] { N2W_CUDA(cudaSetDevice(device)); }); }
int n2w_malloc(void** p, size_t bytes) {
  return guarded([&] {
    N2W_REQUIRE(p, "null output");
    *p = nullptr;
    if (bytes == 0) return;
    const cudaError_t e = cudaMalloc(p, bytes);
    if (e == cudaErrorMemoryAllocation) {
      cudaGetLastError();
      throw Error(N2W_ENOMEM, "device allocation of " + std::to_string(bytes) + " bytes failed");
    }
    N2W_CUDA(e);
  });
}
int n2w_free(void* p) { return guarded([&] { N2W_CUDA(cudaFree(p)); }); }
int n2w_malloc_host(void** p, size_t bytes) {
  return guarded([&] {
    N2W_REQUIRE(p, "null output");
    N2W_CUDA(cudaMallocHost(p, bytes));
  });
}
int n2w_free_host(void* p) { return guarded([&] { N2W_CUDA(cudaFreeHost(p)); }); }
int n2w_memcpy_h2d(void* d, const void* h, size_t bytes, n2w_stream_t s) {
  return guarded([&] { N2W_CUDA(cudaMemcpyAsync(d, h, bytes, cudaMemcpyHostToDevice, s)); });
}
int n2w_memcpy_d2h(void* h, const void* d, size_t bytes, n2w_stream_t s) {
  return guarded([&] { N2W_CUDA(cudaMemcpyAsync(h, d, bytes, cudaMemcpyDeviceToHost, s)); });
}
int n2w_memset(void* d, int v, size_t bytes, n2w_stream_t s) {
  return guarded([&] { N2W_CUDA(cudaMemsetAsync(d, v, bytes, s)); });
}
int n2w_stream_create(n2w_stream_t* out) {
  return guarded([&] {
    N2W_REQUIRE(out, "null output");
    N2W_CUDA(cudaStreamCreateWithFlags(out, cudaStreamNonBlocking));
  });
}
int n2w_stream_destroy(n2w_stream_t s) { return guarded([&] { N2W_CUDA(cudaStreamDestroy(s)); }); }
int n2w_stream_sync(n2w_stream_t s) { return guarded([&] { N2W_CUDA(cudaStreamSynchronize(s)); }); }
int n2w_device_sync(void) { return guarded([&] { N2W_CUDA(cudaDeviceSynchronize()); }); }

}  // extern "C"

struct n2w_timer {
  cudaEvent_t start = nullptr;
  cudaEvent_t stop = nullptr;
};

extern "C" {

int n2w_timer_create(n2w_timer** out) {
  return guarded([&] {
    N2W_REQUIRE(out, "null output");
    auto* t = new n2w_timer();
    if (cudaEventCreate(&t->start) != cudaSuccess || cudaEventCreate(&t->stop) != cudaSuccess) {
      delete t;
      throw Error(N2W_ECUDA, "cudaEventCreate failed");
    }
    *out = t;
  });
}
int n2w_timer_start(n2w_timer* t, n2w_stream_t s) {
  return guarded([&] { N2W_CUDA(cudaEventRecord(t->start, s)); });
}
int n2w_timer_stop(n2w_timer* t, n2w_stream_t s) {
  return guarded([&] { N2W_CUDA(cudaEventRecord(t->stop, s)); });
}
int n2w_timer_elapsed_ms(n2w_timer* t, float* ms) {
  return guarded([&] {
    N2W_CUDA(cudaEventSynchronize(t->stop));
    N2W_CUDA(cudaEventElapsedTime(ms, t->start, t->stop));
  });
}
void n2w_timer_destroy(n2w_timer* t) {
  if (!t) return;
  cudaEventDestroy(t->start);
  cudaEventDestroy(t->stop);
  delete t;
}
int n2w_sm_count(int* out) {
  return guarded([&] {
    N2W_REQUIRE(out, "null output");
    *out = sm_count_current();
  });
}
int n2w_mem_info(size_t* f, size_t* t) {
  return guarded([&] {
    N2W_REQUIRE(f && t, "null output");
    N2W_CUDA(cudaMemGetInfo(f, t));
  });
}

}  // extern "C"
