// Counter-based Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel Random
// Numbers: As Easy as 1, 2, 3", SC 2011): four 32-bit words per call from a
// 128-bit counter and a 64-bit key.  Walk w of a run draws step s from counter
// (w.lo, w.hi, s, stream), so a walk's random numbers depend only on
// (seed, walk id, step) and never on which thread or launch runs it.
#pragma once

#include <stdint.h>

#ifdef __CUDACC__
#define N2W_RNG_HD __host__ __device__ __forceinline__
#else
#define N2W_RNG_HD inline
#endif

namespace n2w {

struct U4 {
  uint32_t x, y, z, w;
};

N2W_RNG_HD void mulhilo32(uint32_t a, uint32_t b, uint32_t& hi, uint32_t& lo) {
#if defined(__CUDA_ARCH__)
  lo = a * b;
  hi = __umulhi(a, b);
#else
  const uint64_t p = static_cast<uint64_t>(a) * static_cast<uint64_t>(b);
  lo = static_cast<uint32_t>(p);
  hi = static_cast<uint32_t>(p >> 32);
#endif
}

N2W_RNG_HD U4 philox4x32_10(U4 c, uint32_t k0, uint32_t k1) {
  // Round multipliers and Weyl key increments from the SC'11 paper.
  const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;
  const uint32_t W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    uint32_t hi0, lo0, hi1, lo1;
    mulhilo32(M0, c.x, hi0, lo0);
    mulhilo32(M1, c.z, hi1, lo1);
    c = U4{hi1 ^ c.y ^ k0, lo1, hi0 ^ c.w ^ k1, lo0};
    k0 += W0;
    k1 += W1;
  }
  return c;
}

// Uniform in [0, 1) with 24 random bits.
N2W_RNG_HD float u01(uint32_t v) { return static_cast<float>(v >> 8) * (1.0f / 16777216.0f); }

// Key words from a 64-bit seed and a small stream tag (coarse / residual / training).
N2W_RNG_HD void philox_key(uint64_t seed, uint32_t tag, uint32_t& k0, uint32_t& k1) {
  k0 = static_cast<uint32_t>(seed) ^ (tag * 0x85EBCA6Bu);
  k1 = static_cast<uint32_t>(seed >> 32) ^ (tag * 0xC2B2AE35u);
}

// splitmix64 (Steele, Lea, Flood, OOPSLA 2014) for host-side seeded generators.
inline uint64_t splitmix64_next(uint64_t& state) {
  uint64_t z = (state += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
inline double splitmix64_unit(uint64_t& state) {
  return static_cast<double>(splitmix64_next(state) >> 11) * (1.0 / 9007199254740992.0);
}

}  // namespace n2w
