// Dirichlet data g, source f (for -Lap u = f) and exact solutions, evaluated
// identically on host and device.  Template parameter T is float for the
// walkers and double for the FP64 analytic solution used to score estimates.
//
// Reference modes keep the reference's formulas (src/cuda/cubql_bvh.cu:1180-1300,
// include/n2wos/nc_poisson_manufactured.hpp:41-160): the boundary data must be
// the same function for the estimates to be comparable.  Modes 100/101 are the
// seeded charge shell and the sin-product manufactured Poisson problem.
#pragma once

#include <math.h>
#include <stdint.h>

#include "n2w.h"

#ifdef __CUDACC__
#define N2W_PHD __host__ __device__ __forceinline__
#else
#define N2W_PHD inline
#endif

namespace n2w {

template <typename T>
struct Math;
template <>
struct Math<float> {
  static N2W_PHD float s(float x) { return sinf(x); }
  static N2W_PHD float c(float x) { return cosf(x); }
  static N2W_PHD float e(float x) { return expf(x); }
  static N2W_PHD float sq(float x) { return sqrtf(x); }
  static N2W_PHD float th(float x) { return tanhf(x); }
  static N2W_PHD float mx(float a, float b) { return fmaxf(a, b); }
};
template <>
struct Math<double> {
  static N2W_PHD double s(double x) { return sin(x); }
  static N2W_PHD double c(double x) { return cos(x); }
  static N2W_PHD double e(double x) { return exp(x); }
  static N2W_PHD double sq(double x) { return sqrt(x); }
  static N2W_PHD double th(double x) { return tanh(x); }
  static N2W_PHD double mx(double a, double b) { return fmax(a, b); }
};

template <typename T>
N2W_PHD T charge_term(T x, T y, T z, T q, T ax, T ay, T az) {
  const T dx = x - ax, dy = y - ay, dz = z - az;
  // sqrt(max(r^2, 1e-12)) keeps the reference's guard (cubql_bvh.cu:1197-1199).
  return q / Math<T>::sq(Math<T>::mx(dx * dx + dy * dy + dz * dz, T(1.0e-12)));
}

template <typename T>
N2W_PHD T complex_power_real(T x, T y, int k) {
  T ar = T(1), ai = T(0);
  for (int i = 0; i < k; ++i) {
    const T nr = ar * x - ai * y;
    const T ni = ar * y + ai * x;
    ar = nr;
    ai = ni;
  }
  return ar;
}

template <typename T>
N2W_PHD T texture_stripes(T x, T y, T z, int k) {
  const T pi = T(3.14159265358979323846);
  const T u = T(0.83) * x + T(0.41) * y + T(0.29) * z;
  const T v = T(-0.21) * x + T(0.77) * y - T(0.43) * z;
  const T a = Math<T>::s(T(k) * pi * u);
  const T b = T(0.45) * Math<T>::s(T(k / 2 + 1) * pi * v + T(0.7));
  const T c = T(0.25) * Math<T>::c(T(k + 3) * pi * (T(0.35) * x - T(0.62) * z));
  return a + b + c;
}

template <typename T>
N2W_PHD T texture_checker(T x, T y, T z, int k) {
  const T pi = T(3.14159265358979323846);
  const T sx = Math<T>::s(T(k) * pi * x);
  const T sy = Math<T>::s(T(k) * pi * y + T(0.31));
  const T sz = Math<T>::s(T(k / 2 + 1) * pi * z - T(0.17));
  return Math<T>::th(T(2.25) * sx * sy) + T(0.25) * sz;
}

// One manufactured Poisson term A exp(k a.x) {cos|sin}(k b.x + phi) with a.b = 0:
// harmonic source f, particular solution u = -(a.x)/(2k) f
// (include/n2wos/nc_poisson_manufactured.hpp:41-73).
template <typename T>
N2W_PHD void poisson_term(T x, T y, T z, T amp, T k, T ax, T ay, T az, T bx, T by, T bz, T phi,
                          bool use_sin, T& u, T& f) {
  const T adot = ax * x + ay * y + az * z;
  const T bdot = bx * x + by * y + bz * z;
  const T arg = k * bdot + phi;
  const T ff = amp * Math<T>::e(k * adot) * (use_sin ? Math<T>::s(arg) : Math<T>::c(arg));
  u += -(adot / (T(2) * k)) * ff;
  f += ff;
}

template <typename T>
N2W_PHD void poisson_multiscale(T x, T y, T z, T& u, T& f) {
  const T r = T(0.70710678118);
  poisson_term<T>(x, y, z, T(0.32), T(1.8), T(1), T(0), T(0), T(0), T(1), T(0), T(0.15), false, u, f);
  poisson_term<T>(x, y, z, T(-0.26), T(2.1), T(0), T(1), T(0), T(0), T(0), T(1), T(-0.40), true, u, f);
  poisson_term<T>(x, y, z, T(0.22), T(2.7), r, r, T(0), -r, r, T(0), T(0.50), false, u, f);
  poisson_term<T>(x, y, z, T(0.18), T(3.0), r, T(0), r, -r, T(0), r, T(-0.10), true, u, f);
  u += T(0.10) * x - T(0.07) * y + T(0.04) * z;
}

template <typename T>
N2W_PHD void poisson_figlike_hf(T x, T y, T z, T& u, T& f) {
  const T r = T(0.70710678118);
  poisson_term<T>(x, y, z, T(0.28), T(2.4), T(1), T(0), T(0), T(0), T(1), T(0), T(0.25), false, u, f);
  poisson_term<T>(x, y, z, T(-0.22), T(2.7), T(0), T(1), T(0), T(0), T(0), T(1), T(-0.30), true, u, f);
  poisson_term<T>(x, y, z, T(0.18), T(3.4), r, r, T(0), -r, r, T(0), T(0.85), false, u, f);
  poisson_term<T>(x, y, z, T(0.14), T(3.8), r, T(0), r, -r, T(0), r, T(0.10), true, u, f);
  poisson_term<T>(x, y, z, T(-0.12), T(4.2), T(0), T(0.8), T(0.6), T(0), T(-0.6), T(0.8), T(-0.20), false, u, f);
  u += T(0.08) * x + T(0.05) * y - T(0.03) * z;
}

// Fixed charge sets of the reference (cubql_bvh.cu:1266-1296).
template <typename T>
N2W_PHD T fixed_charges(T x, T y, T z, int mode) {
  T v = T(0);
  if (mode == N2W_BC_EXTERNAL_CHARGES_SHELL_K8 || mode == N2W_BC_EXTERNAL_CHARGES_SHELL_K16) {
    const bool k16 = mode == N2W_BC_EXTERNAL_CHARGES_SHELL_K16;
    const float rs = k16 ? 1.08f : 1.14f;
    const int n = k16 ? 16 : 8;
    for (int i = 0; i < n; ++i) {
      // Charge positions are computed in FP32 as the reference does.
      const float a = 6.283185307179586f * static_cast<float>(i) / static_cast<float>(n);
      const float q = (i & 1) ? -0.45f : 0.45f;
      const float cz = (i & 2) ? 0.18f : -0.18f;
      const float rr = sqrtf(fmaxf(rs * rs - cz * cz, 0.0f));
      v += charge_term<T>(x, y, z, T(q), T(rr * cosf(a)), T(rr * sinf(a)), T(cz));
    }
  } else if (mode == N2W_BC_EXTERNAL_CHARGES_HIGH) {
    v += charge_term<T>(x, y, z, T(1.20f), T(1.18f), T(0.16f), T(0.10f));
    v += charge_term<T>(x, y, z, T(-1.00f), T(-1.16f), T(-0.20f), T(0.22f));
    v += charge_term<T>(x, y, z, T(0.85f), T(0.08f), T(1.17f), T(-0.30f));
    v += charge_term<T>(x, y, z, T(-0.70f), T(-0.18f), T(-1.18f), T(0.36f));
    v += charge_term<T>(x, y, z, T(0.58f), T(0.35f), T(-0.20f), T(1.19f));
    v += charge_term<T>(x, y, z, T(-0.53f), T(-0.38f), T(0.24f), T(-1.19f));
    v += charge_term<T>(x, y, z, T(0.32f), T(0.90f), T(-0.82f), T(0.70f));
    v += charge_term<T>(x, y, z, T(-0.30f), T(-0.86f), T(0.78f), T(-0.66f));
  } else {
    v += charge_term<T>(x, y, z, T(1.00f), T(1.55f), T(0.30f), T(0.18f));
    v += charge_term<T>(x, y, z, T(-0.85f), T(-1.45f), T(-0.28f), T(0.36f));
    v += charge_term<T>(x, y, z, T(0.55f), T(0.20f), T(1.48f), T(-0.42f));
    v += charge_term<T>(x, y, z, T(-0.45f), T(-0.34f), T(-1.52f), T(0.24f));
  }
  return v;
}

// Solution u (which equals the Dirichlet data g on the boundary) at x.
template <typename T>
N2W_PHD T problem_u(const n2w_problem& pb, T x, T y, T z) {
  switch (pb.mode) {
    case N2W_BC_HARMONIC_X2_MINUS_Y2: return x * x - y * y;
    case N2W_BC_HARMONIC_ZEBRA_K4: return complex_power_real<T>(x, y, 4);
    case N2W_BC_HARMONIC_ZEBRA_K8: return complex_power_real<T>(x, y, 8);
    case N2W_BC_HARMONIC_ZEBRA_K12: return complex_power_real<T>(x, y, 12);
    case N2W_BC_TEXTURE_STRIPES_K8: return texture_stripes<T>(x, y, z, 8);
    case N2W_BC_TEXTURE_STRIPES_K16: return texture_stripes<T>(x, y, z, 16);
    case N2W_BC_TEXTURE_CHECKER_K8: return texture_checker<T>(x, y, z, 8);
    case N2W_BC_TEXTURE_CHECKER_K16: return texture_checker<T>(x, y, z, 16);
    case N2W_BC_CONSTANT_ONE: return T(1);
    case N2W_BC_POISSON_MULTISCALE: {
      T u = T(0), f = T(0);
      poisson_multiscale<T>(x, y, z, u, f);
      return u;
    }
    case N2W_BC_POISSON_FIGLIKE_HF: {
      T u = T(0), f = T(0);
      poisson_figlike_hf<T>(x, y, z, u, f);
      return u;
    }
    case N2W_BC_CHARGES_SEEDED: {
      T v = T(0);
      for (int k = 0; k < pb.charge_count; ++k) {
        v += charge_term<T>(x, y, z, T(pb.charges[k][3]), T(pb.charges[k][0]), T(pb.charges[k][1]),
                            T(pb.charges[k][2]));
      }
      return v;
    }
    case N2W_BC_POISSON_SINPROD: {
      const T w = T(pb.omega);
      return Math<T>::s(w * x) * Math<T>::s(w * y) * Math<T>::s(w * z);
    }
    default: return fixed_charges<T>(x, y, z, pb.mode);
  }
}

// Source f of -Lap u = f (zero for harmonic problems).
template <typename T>
N2W_PHD T problem_f(const n2w_problem& pb, T x, T y, T z) {
  switch (pb.mode) {
    case N2W_BC_POISSON_MULTISCALE: {
      T u = T(0), f = T(0);
      poisson_multiscale<T>(x, y, z, u, f);
      return f;
    }
    case N2W_BC_POISSON_FIGLIKE_HF: {
      T u = T(0), f = T(0);
      poisson_figlike_hf<T>(x, y, z, u, f);
      return f;
    }
    case N2W_BC_POISSON_SINPROD: {
      const T w = T(pb.omega);
      return T(3) * w * w * Math<T>::s(w * x) * Math<T>::s(w * y) * Math<T>::s(w * z);
    }
    default: return T(0);
  }
}

N2W_PHD bool problem_has_source(const n2w_problem& pb) {
  return pb.mode == N2W_BC_POISSON_MULTISCALE || pb.mode == N2W_BC_POISSON_FIGLIKE_HF ||
         pb.mode == N2W_BC_POISSON_SINPROD;
}

// Whether u is a known solution in the interior (false for the texture modes,
// whose boundary data has no closed-form harmonic extension).
N2W_PHD bool problem_exact_known(const n2w_problem& pb) {
  return !(pb.mode >= N2W_BC_TEXTURE_STRIPES_K8 && pb.mode <= N2W_BC_TEXTURE_CHECKER_K16);
}

}  // namespace n2w
