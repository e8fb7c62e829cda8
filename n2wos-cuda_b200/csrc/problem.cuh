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

// One harmonic term A exp(k a.x) {cos|sin}(k b.x + phi) with a, b orthonormal:
// the exponential's second derivative along a cancels the oscillation's along
// b.  The reference's analytic mixtures (include/n2wos/nc_harmonic_mixture.hpp)
// are scaled sums of such terms plus a linear part; their coefficient tables
// are kept as given there so the boundary data are the same functions.
template <typename T>
N2W_PHD T harmonic_term(T x, T y, T z, T amp, T k, T ax, T ay, T az, T bx, T by, T bz, T phi, bool use_sin) {
  const T adot = ax * x + ay * y + az * z;
  const T arg = k * (bx * x + by * y + bz * z) + phi;
  return amp * Math<T>::e(k * adot) * (use_sin ? Math<T>::s(arg) : Math<T>::c(arg));
}

template <typename T>
N2W_PHD T harmonic_mixture(T x, T y, T z, int mode) {
  const T r = T(0.70710678118), s3 = T(0.57735026919);
  T t = T(0), lin = T(0), scale = T(1);
  switch (mode) {
    case N2W_BC_HARMONIC_MIXTURE_SMOOTH:
      t += harmonic_term<T>(x, y, z, T(0.42), T(1.15), T(1), T(0), T(0), T(0), T(1), T(0), T(0.15), false);
      t += harmonic_term<T>(x, y, z, T(-0.30), T(1.05), T(0), T(-1), T(0), T(0), T(0), T(1), T(-0.25), true);
      t += harmonic_term<T>(x, y, z, T(0.24), T(1.25), T(0.6), T(0), T(0.8), T(-0.8), T(0), T(0.6), T(0.70), false);
      t += harmonic_term<T>(x, y, z, T(0.18), T(1.10), -s3, -s3, -s3, r, -r, T(0), T(1.10), true);
      lin = T(0.12) * x - T(0.08) * y + T(0.06) * z;
      scale = T(0.72);
      break;
    case N2W_BC_HARMONIC_MIXTURE_FIGLIKE:
      t += harmonic_term<T>(x, y, z, T(0.36), T(1.65), T(1), T(0), T(0), T(0), T(1), T(0), T(0.35), false);
      t += harmonic_term<T>(x, y, z, T(-0.30), T(1.45), T(0), T(-1), T(0), T(0), T(0), T(1), T(-0.20), false);
      t += harmonic_term<T>(x, y, z, T(0.27), T(1.85), r, T(0), r, -r, T(0), r, T(0.55), true);
      t += harmonic_term<T>(x, y, z, T(0.18), T(1.30), T(0), T(-0.8), T(-0.6), T(0), T(-0.6), T(0.8), T(-0.90),
                            false);
      lin = T(0.10) * x + T(0.14) * y - T(0.05) * z;
      scale = T(0.58);
      break;
    case N2W_BC_HARMONIC_MIXTURE_MULTISCALE:
      t += harmonic_term<T>(x, y, z, T(0.20), T(1.35), T(1), T(0), T(0), T(0), T(1), T(0), T(0.20), false);
      t += harmonic_term<T>(x, y, z, T(-0.17), T(1.55), T(0), T(-1), T(0), T(0), T(0), T(1), T(-0.45), true);
      t += harmonic_term<T>(x, y, z, T(0.15), T(1.70), T(0), T(0), T(1), T(1), T(0), T(0), T(0.80), false);
      t += harmonic_term<T>(x, y, z, T(0.095), T(2.55), r, r, T(0), -r, r, T(0), T(0.15), false);
      t += harmonic_term<T>(x, y, z, T(-0.080), T(2.85), T(0), -r, -r, T(0), -r, r, T(-0.65), true);
      t += harmonic_term<T>(x, y, z, T(0.070), T(3.15), r, T(0), r, -r, T(0), r, T(1.10), false);
      t += harmonic_term<T>(x, y, z, T(0.060), T(3.35), -s3, -s3, -s3, r, -r, T(0), T(0.40), true);
      t += harmonic_term<T>(x, y, z, T(0.035), T(4.00), T(0.81649658093), T(-0.40824829046), T(-0.40824829046),
                            T(0), r, -r, T(-0.35), false);
      lin = T(0.035) * x - T(0.025) * y + T(0.020) * z;
      scale = T(0.62);
      break;
    default:  // N2W_BC_HARMONIC_MIXTURE_FIGLIKE_HF
      t += harmonic_term<T>(x, y, z, T(0.18), T(1.65), T(1), T(0), T(0), T(0), T(1), T(0), T(0.35), false);
      t += harmonic_term<T>(x, y, z, T(-0.15), T(1.75), T(0), T(-1), T(0), T(0), T(0), T(1), T(-0.20), false);
      t += harmonic_term<T>(x, y, z, T(0.13), T(1.85), T(0), T(0), T(1), T(1), T(0), T(0), T(0.70), true);
      t += harmonic_term<T>(x, y, z, T(0.095), T(2.90), r, T(0), r, -r, T(0), r, T(0.55), true);
      t += harmonic_term<T>(x, y, z, T(-0.085), T(3.25), -r, -r, T(0), -r, r, T(0), T(-0.75), false);
      t += harmonic_term<T>(x, y, z, T(0.070), T(3.55), T(0), r, r, T(0), -r, r, T(1.20), true);
      t += harmonic_term<T>(x, y, z, T(0.040), T(4.20), T(0.86602540378), T(0), T(0.5), T(-0.5), T(0),
                            T(0.86602540378), T(0.25), false);
      t += harmonic_term<T>(x, y, z, T(-0.032), T(4.50), T(0), T(-0.8), T(-0.6), T(0), T(-0.6), T(0.8), T(-0.30), true);
      lin = T(0.025) * x + T(0.020) * y - T(0.015) * z;
      scale = T(0.55);
      break;
  }
  return scale * (t + lin);
}

// Higher-frequency manufactured Poisson field of the reference
// (include/n2wos/nc_poisson_manufactured.hpp:160-209): a Fourier mixture
// u = sum A trig(k.x + phi) + a weak linear part, f = -Lap u = sum A |k|^2 trig(...).
template <typename T>
N2W_PHD void fourier_term(T x, T y, T z, T amp, T kx, T ky, T kz, T phi, bool use_sin, T& u, T& f) {
  const T arg = kx * x + ky * y + kz * z + phi;
  const T v = amp * (use_sin ? Math<T>::s(arg) : Math<T>::c(arg));
  u += v;
  f += (kx * kx + ky * ky + kz * kz) * v;
}

template <typename T>
N2W_PHD void poisson_figlike_hf_x5(T x, T y, T z, T& u, T& f) {
  fourier_term<T>(x, y, z, T(0.090), T(12.0), T(4.0), T(1.5), T(0.30), true, u, f);
  fourier_term<T>(x, y, z, T(0.075), T(-5.0), T(13.5), T(2.0), T(-0.70), false, u, f);
  fourier_term<T>(x, y, z, T(0.060), T(7.5), T(-3.5), T(15.0), T(1.10), true, u, f);
  fourier_term<T>(x, y, z, T(0.050), T(14.0), T(-10.0), T(4.0), T(2.20), false, u, f);
  fourier_term<T>(x, y, z, T(0.045), T(-9.0), T(6.5), T(12.0), T(-1.30), true, u, f);
  fourier_term<T>(x, y, z, T(0.035), T(18.0), T(2.5), T(-7.0), T(0.80), false, u, f);
  u += T(0.030) * (T(0.60) * x - T(0.35) * y + T(0.20) * z);
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
    case N2W_BC_HARMONIC_MIXTURE_SMOOTH:
    case N2W_BC_HARMONIC_MIXTURE_FIGLIKE:
    case N2W_BC_HARMONIC_MIXTURE_MULTISCALE:
    case N2W_BC_HARMONIC_MIXTURE_FIGLIKE_HF: return harmonic_mixture<T>(x, y, z, pb.mode);
    case N2W_BC_POISSON_FIGLIKE_HF_X5: {
      T u = T(0), f = T(0);
      poisson_figlike_hf_x5<T>(x, y, z, u, f);
      return u;
    }
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
    case N2W_BC_POISSON_FIGLIKE_HF_X5: {
      T u = T(0), f = T(0);
      poisson_figlike_hf_x5<T>(x, y, z, u, f);
      return f;
    }
    default: return T(0);
  }
}

N2W_PHD bool problem_has_source(const n2w_problem& pb) {
  return pb.mode == N2W_BC_POISSON_MULTISCALE || pb.mode == N2W_BC_POISSON_FIGLIKE_HF ||
         pb.mode == N2W_BC_POISSON_FIGLIKE_HF_X5 || pb.mode == N2W_BC_POISSON_SINPROD;
}

// Whether u is a known solution in the interior (false for the texture modes,
// whose boundary data has no closed-form harmonic extension).
N2W_PHD bool problem_exact_known(const n2w_problem& pb) {
  return !(pb.mode >= N2W_BC_TEXTURE_STRIPES_K8 && pb.mode <= N2W_BC_TEXTURE_CHECKER_K16);
}

}  // namespace n2w
