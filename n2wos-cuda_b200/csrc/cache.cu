// Neural cache: multiresolution hash-grid encoding + small ReLU MLP, trained
// online with Adam.  Replaces tiny-cuda-nn's HashGrid + FullyFusedMLP + Adam
// as used by the reference (src/tools/eval_tcnn_nc_wos.cu:747-750,759).
//
// Encoding (Mueller, Evans, Schied, Keller, "Instant Neural Graphics
// Primitives with a Multiresolution Hash Encoding", SIGGRAPH 2022): level l has
// resolution N_l = floor(N_min * b^l); a point x in [0,1]^3 is scaled by N_l,
// its 8 lattice corners are looked up densely while (N_l+1)^3 fits the level's
// table and through the spatial hash (x*1 ^ y*2654435761 ^ z*805459861) mod T
// otherwise, and the F features are trilinearly interpolated.
//
// MLP: inputs L*F (= 32 for 16 levels x 2), hidden width W in {16, 32, 64},
// H hidden layers, scalar output, ReLU, no output activation.  FP16 weights
// and activations on mma.sync.m16n8k16 with FP32 accumulation; FP32 master
// parameters and Adam moments.
//
// Warp tiling: a warp owns 16 samples.  Lane (g = lane/4, c = lane%4) holds
// rows g and g+8 of every fragment.  It computes the encoding of exactly the
// (sample, level) pairs its layer-1 A fragment needs — levels c, c+4, c+8,
// c+12 of samples g and g+8 — so features go straight into registers; each
// layer's FP32 C fragments become the next layer's FP16 A fragments in place;
// in the backward pass dX arrives in the same (sample, level) ownership, so the
// grid-gradient scatter needs no reshuffle.
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <string>
#include <vector>

#include "internal.hpp"
#include "philox.cuh"

namespace n2w {
namespace {

constexpr int kMaxLevels = 16;
constexpr int kMaxHidden = 4;
constexpr int kTrainBlock = 128;  // 4 warps
constexpr int kTrainRound = 64;   // samples staged per block round

struct GridMeta {
  int levels;
  int features;  // fixed to 2
  uint32_t table_size[kMaxLevels];
  uint32_t offset[kMaxLevels];  // entry offset of each level
  float scale[kMaxLevels];      // N_l
  uint32_t res[kMaxLevels];     // N_l
  uint32_t dense[kMaxLevels];   // 1 = dense indexing
};

struct MlpMeta {
  int width;   // 16 / 32 / 64
  int hidden;  // hidden layers
  int in_dim;  // 16 or 32 (levels*2 padded to 16)
  // parameter offsets (elements) inside the MLP block
  int w_in;                // [width x in_dim]
  int w_hid[kMaxHidden];   // [width x width], hidden-1 of them used
  int w_out;               // [width] (output row)
  int total;
};

__host__ __device__ __forceinline__ uint32_t hash3(uint32_t x, uint32_t y, uint32_t z) {
  return x * 1u ^ y * 2654435761u ^ z * 805459861u;
}

__device__ __forceinline__ uint32_t corner_index(const GridMeta& g, int l, uint32_t x, uint32_t y, uint32_t z) {
  if (g.dense[l]) {
    const uint32_t s = g.res[l] + 1;
    return x + s * (y + s * z);
  }
  return hash3(x, y, z) % g.table_size[l];
}

// Trilinear corner setup of level l for input u in [0,1]^3.
struct Corners {
  uint32_t base[3];
  float w[3];  // fractional parts
};

__device__ __forceinline__ Corners level_corners(const GridMeta& g, int l, float ux, float uy, float uz) {
  Corners c;
  const float s = g.scale[l];
  const float px = ux * s, py = uy * s, pz = uz * s;
  const float fx = floorf(px), fy = floorf(py), fz = floorf(pz);
  const float lim = s - 1.0f;
  const float cx = fminf(fmaxf(fx, 0.0f), lim), cy = fminf(fmaxf(fy, 0.0f), lim), cz = fminf(fmaxf(fz, 0.0f), lim);
  c.base[0] = static_cast<uint32_t>(cx);
  c.base[1] = static_cast<uint32_t>(cy);
  c.base[2] = static_cast<uint32_t>(cz);
  c.w[0] = px - cx;
  c.w[1] = py - cy;
  c.w[2] = pz - cz;
  return c;
}

// Encoded feature pair (F = 2) of one (sample, level).
__device__ __forceinline__ float2 encode_level(const GridMeta& g, const __half2* __restrict__ table, int l,
                                               float ux, float uy, float uz) {
  const Corners c = level_corners(g, l, ux, uy, uz);
  float2 acc = make_float2(0.0f, 0.0f);
  const __half2* t = table + g.offset[l];
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    const uint32_t dx = k & 1, dy = (k >> 1) & 1, dz = (k >> 2) & 1;
    const float w = (dx ? c.w[0] : 1.0f - c.w[0]) * (dy ? c.w[1] : 1.0f - c.w[1]) * (dz ? c.w[2] : 1.0f - c.w[2]);
    const float2 v = __half22float2(__ldg(t + corner_index(g, l, c.base[0] + dx, c.base[1] + dy, c.base[2] + dz)));
    acc.x += w * v.x;
    acc.y += w * v.y;
  }
  return acc;
}

__device__ __forceinline__ void scatter_level(const GridMeta& g, float2* __restrict__ grad, int l, float ux, float uy,
                                              float uz, float2 d) {
  const Corners c = level_corners(g, l, ux, uy, uz);
  float2* t = grad + g.offset[l];
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    const uint32_t dx = k & 1, dy = (k >> 1) & 1, dz = (k >> 2) & 1;
    const float w = (dx ? c.w[0] : 1.0f - c.w[0]) * (dy ? c.w[1] : 1.0f - c.w[1]) * (dz ? c.w[2] : 1.0f - c.w[2]);
    atomicAdd(t + corner_index(g, l, c.base[0] + dx, c.base[1] + dy, c.base[2] + dz), make_float2(w * d.x, w * d.y));
  }
}

__device__ __forceinline__ uint32_t pack_h2(float a, float b) {
  const __half2 h = __floats2half2_rn(a, b);
  return *reinterpret_cast<const uint32_t*>(&h);
}

__device__ __forceinline__ float2 unpack_h2(uint32_t u) {
  return __half22float2(*reinterpret_cast<const __half2*>(&u));
}

// D = A(16x16 f16, row) * B(16x8 f16, col) + C (f32).
__device__ __forceinline__ void mma16816(float* d, const uint32_t* a, const uint32_t* b) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.f16.f16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// B fragment of W^T (B[k][n] = W[n][k], W row-major [out x in], leading dim ld):
// lane (g,c) needs W[n0+g][k0+2c..2c+1] and W[n0+g][k0+2c+8..2c+9].
__device__ __forceinline__ void load_b_wt(uint32_t* b, const __half* W, int ld, int n0, int k0, int g, int c) {
  const __half* r = W + (n0 + g) * ld + k0 + 2 * c;
  b[0] = *reinterpret_cast<const uint32_t*>(r);
  b[1] = *reinterpret_cast<const uint32_t*>(r + 8);
}

// C fragments of n-tiles (2t, 2t+1) -> A fragment of k-step t, with ReLU.
__device__ __forceinline__ void c_to_a_relu(uint32_t* a, const float* c0, const float* c1) {
  a[0] = pack_h2(fmaxf(c0[0], 0.0f), fmaxf(c0[1], 0.0f));
  a[1] = pack_h2(fmaxf(c0[2], 0.0f), fmaxf(c0[3], 0.0f));
  a[2] = pack_h2(fmaxf(c1[0], 0.0f), fmaxf(c1[1], 0.0f));
  a[3] = pack_h2(fmaxf(c1[2], 0.0f), fmaxf(c1[3], 0.0f));
}

__device__ __forceinline__ void c_to_a(uint32_t* a, const float* c0, const float* c1) {
  a[0] = pack_h2(c0[0], c0[1]);
  a[1] = pack_h2(c0[2], c0[3]);
  a[2] = pack_h2(c1[0], c1[1]);
  a[3] = pack_h2(c1[2], c1[3]);
}

struct NetArgs {
  GridMeta grid;
  MlpMeta mlp;
  const __half2* table;   // fp16 grid features
  const __half* mlp_h;    // fp16 MLP weights
  float2* grid_grad;      // fp32 grid gradient accumulators
  float* mlp_grad;        // fp32 MLP gradient accumulators
  const float* inputs;    // [n x 3], unit cube
  const float* targets;   // [n]
  float* outputs;         // [n]
  int64_t n;
  float loss_scale;       // dL/dy = loss_scale * (y - t)
  float* loss_sum;        // optional: sum of (y - t)^2
};

// Loads every MLP weight matrix into shared memory (fp16), plus transposed
// copies for the backward products.
template <int W>
__device__ void stage_weights(const NetArgs& a, __half* sm, __half* smT) {
  const int n = a.mlp.total;
  for (int i = threadIdx.x; i < n; i += blockDim.x) sm[i] = a.mlp_h[i];
  if (smT) {
    // transposes: w_in [W x in] -> [in x W]; hidden [W x W] -> [W x W]^T
    const int in = a.mlp.in_dim;
    for (int i = threadIdx.x; i < W * in; i += blockDim.x) {
      const int o = i / in, k = i % in;
      smT[a.mlp.w_in + k * W + o] = a.mlp_h[a.mlp.w_in + i];
    }
    for (int h = 0; h < a.mlp.hidden - 1; ++h) {
      const int off = a.mlp.w_hid[h];
      for (int i = threadIdx.x; i < W * W; i += blockDim.x) {
        const int o = i / W, k = i % W;
        smT[off + k * W + o] = a.mlp_h[off + i];
      }
    }
  }
  __syncthreads();
}

// Encodes the 16-sample tile into layer-1 A fragments (KS k-steps of 16 inputs).
template <int KS>
__device__ __forceinline__ void encode_tile(const NetArgs& a, int64_t s0, int64_t s1, int g, int c,
                                            uint32_t (&x)[KS][4], float (&u)[2][3]) {
  const bool v0 = s0 < a.n, v1 = s1 < a.n;
  for (int k = 0; k < 3; ++k) {
    u[0][k] = v0 ? a.inputs[3 * s0 + k] : 0.0f;
    u[1][k] = v1 ? a.inputs[3 * s1 + k] : 0.0f;
  }
#pragma unroll
  for (int kk = 0; kk < KS; ++kk) {
#pragma unroll
    for (int half = 0; half < 2; ++half) {
      const int l = 8 * kk + c + 4 * half;
      float2 e0 = make_float2(0.0f, 0.0f), e1 = make_float2(0.0f, 0.0f);
      if (l < a.grid.levels) {
        e0 = encode_level(a.grid, a.table, l, u[0][0], u[0][1], u[0][2]);
        e1 = encode_level(a.grid, a.table, l, u[1][0], u[1][1], u[1][2]);
      }
      x[kk][2 * half + 0] = pack_h2(e0.x, e0.y);
      x[kk][2 * half + 1] = pack_h2(e1.x, e1.y);
    }
  }
}

// Forward pass of one tile; returns activations' fragments for the backward.
template <int W, int KS, int H>
__device__ __forceinline__ void forward_tile(const NetArgs& a, const __half* sm, const uint32_t (&x)[KS][4], int g,
                                             int c, uint32_t (&act)[H][W / 16][4], float& y0, float& y1) {
  constexpr int NT = W / 8;
  float acc[NT][4];
#pragma unroll
  for (int j = 0; j < NT; ++j) acc[j][0] = acc[j][1] = acc[j][2] = acc[j][3] = 0.0f;
#pragma unroll
  for (int kk = 0; kk < KS; ++kk) {
#pragma unroll
    for (int j = 0; j < NT; ++j) {
      uint32_t b[2];
      load_b_wt(b, sm + a.mlp.w_in, a.mlp.in_dim, 8 * j, 16 * kk, g, c);
      mma16816(acc[j], x[kk], b);
    }
  }
#pragma unroll
  for (int t = 0; t < W / 16; ++t) c_to_a_relu(act[0][t], acc[2 * t], acc[2 * t + 1]);
#pragma unroll
  for (int h = 1; h < H; ++h) {
#pragma unroll
    for (int j = 0; j < NT; ++j) acc[j][0] = acc[j][1] = acc[j][2] = acc[j][3] = 0.0f;
#pragma unroll
    for (int kk = 0; kk < W / 16; ++kk) {
#pragma unroll
      for (int j = 0; j < NT; ++j) {
        uint32_t b[2];
        load_b_wt(b, sm + a.mlp.w_hid[h - 1], W, 8 * j, 16 * kk, g, c);
        mma16816(acc[j], act[h - 1][kk], b);
      }
    }
#pragma unroll
    for (int t = 0; t < W / 16; ++t) c_to_a_relu(act[h][t], acc[2 * t], acc[2 * t + 1]);
  }
  // output row: n-tile of 8 where only column 0 is the output neuron
  float o[4] = {0.0f, 0.0f, 0.0f, 0.0f};
  const __half* wo = sm + a.mlp.w_out;
#pragma unroll
  for (int kk = 0; kk < W / 16; ++kk) {
    uint32_t b[2] = {0u, 0u};
    if (g == 0) {
      b[0] = *reinterpret_cast<const uint32_t*>(wo + 16 * kk + 2 * c);
      b[1] = *reinterpret_cast<const uint32_t*>(wo + 16 * kk + 2 * c + 8);
    }
    mma16816(o, act[H - 1][kk], b);
  }
  y0 = o[0];  // valid in lanes with c == 0: row g, column 0
  y1 = o[2];  // row g + 8
}

template <int W, int KS, int H>
__global__ void __launch_bounds__(kTrainBlock) infer_kernel(const NetArgs a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __half* sm = reinterpret_cast<__half*>(smem_raw);
  stage_weights<W>(a, sm, nullptr);
  const int lane = threadIdx.x & 31, g = lane >> 2, c = lane & 3;
  const int64_t warps = static_cast<int64_t>(gridDim.x) * (blockDim.x >> 5);
  const int64_t tiles = (a.n + 15) / 16;
  for (int64_t tile = static_cast<int64_t>(blockIdx.x) * (blockDim.x >> 5) + (threadIdx.x >> 5); tile < tiles;
       tile += warps) {
    const int64_t s0 = tile * 16 + g, s1 = s0 + 8;
    uint32_t x[KS][4];
    float u[2][3];
    encode_tile<KS>(a, s0, s1, g, c, x, u);
    uint32_t act[H][W / 16][4];
    float y0, y1;
    forward_tile<W, KS, H>(a, sm, x, g, c, act, y0, y1);
    if (c == 0) {
      if (s0 < a.n) a.outputs[s0] = y0;
      if (s1 < a.n) a.outputs[s1] = y1;
    }
  }
}

// Forward + backward over rounds of 64 samples per block (16 per warp).
// Gradients: grid features by vector FP32 atomics; MLP weights accumulated per
// warp in registers (warp w owns output rows [16w, 16w+16) of each matrix)
// from the round's activations staged in shared memory, flushed at the end.
template <int W, int KS, int H>
__global__ void __launch_bounds__(kTrainBlock) train_kernel(const NetArgs a) {
  static_assert(W == 64 || W == 32 || W == 16, "width");
  constexpr int NT = W / 8;
  constexpr int IN = 16 * KS;
  constexpr int MT = W / 16;  // m-tiles of a weight matrix (rows)
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __half* sm = reinterpret_cast<__half*>(smem_raw);
  __half* smT = sm + a.mlp.total;
  // staged per round: X [64 x IN], act[h] [64 x W], dpre[h] [64 x W], dy [64] (fp32)
  __half* sX = smT + a.mlp.total;
  __half* sAct = sX + kTrainRound * IN;
  __half* sD = sAct + kMaxHidden * kTrainRound * W;
  float* sDy = reinterpret_cast<float*>(sD + kMaxHidden * kTrainRound * W);
  stage_weights<W>(a, sm, smT);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, c = lane & 3;
  constexpr int HG = H > 1 ? H - 1 : 1;
  // weight-gradient accumulators: this warp's m-tile (rows 16*warp..) of each matrix
  float gin[IN / 8][4];
  float ghid[HG][NT][4];
#pragma unroll
  for (int j = 0; j < IN / 8; ++j) gin[j][0] = gin[j][1] = gin[j][2] = gin[j][3] = 0.0f;
#pragma unroll
  for (int h = 0; h < HG; ++h)
#pragma unroll
    for (int j = 0; j < NT; ++j) ghid[h][j][0] = ghid[h][j][1] = ghid[h][j][2] = ghid[h][j][3] = 0.0f;
  float loss = 0.0f;

  const int64_t rounds = (a.n + kTrainRound - 1) / kTrainRound;
  for (int64_t r = blockIdx.x; r < rounds; r += gridDim.x) {
    const int64_t s0 = r * kTrainRound + warp * 16 + g, s1 = s0 + 8;
    const int row0 = warp * 16 + g, row1 = row0 + 8;  // rows within the staged round
    uint32_t x[KS][4];
    float u[2][3];
    encode_tile<KS>(a, s0, s1, g, c, x, u);
    uint32_t act[H][W / 16][4];
    float y0, y1;
    forward_tile<W, KS, H>(a, sm, x, g, c, act, y0, y1);
    // dL/dy (lanes c==0 hold the outputs); broadcast to the quad
    float dy0 = 0.0f, dy1 = 0.0f;
    if (c == 0) {
      if (s0 < a.n) {
        const float e = y0 - a.targets[s0];
        dy0 = a.loss_scale * e;
        loss += e * e;
      }
      if (s1 < a.n) {
        const float e = y1 - a.targets[s1];
        dy1 = a.loss_scale * e;
        loss += e * e;
      }
      if (a.outputs) {
        if (s0 < a.n) a.outputs[s0] = y0;
        if (s1 < a.n) a.outputs[s1] = y1;
      }
    }
    dy0 = __shfl_sync(0xffffffffu, dy0, lane & ~3);
    dy1 = __shfl_sync(0xffffffffu, dy1, lane & ~3);
    // stage X, activations, dy
#pragma unroll
    for (int kk = 0; kk < KS; ++kk) {
      *reinterpret_cast<uint32_t*>(sX + row0 * IN + 16 * kk + 2 * c) = x[kk][0];
      *reinterpret_cast<uint32_t*>(sX + row1 * IN + 16 * kk + 2 * c) = x[kk][1];
      *reinterpret_cast<uint32_t*>(sX + row0 * IN + 16 * kk + 2 * c + 8) = x[kk][2];
      *reinterpret_cast<uint32_t*>(sX + row1 * IN + 16 * kk + 2 * c + 8) = x[kk][3];
    }
#pragma unroll
    for (int h = 0; h < H; ++h) {
      __half* base = sAct + h * kTrainRound * W;
#pragma unroll
      for (int t = 0; t < W / 16; ++t) {
        *reinterpret_cast<uint32_t*>(base + row0 * W + 16 * t + 2 * c) = act[h][t][0];
        *reinterpret_cast<uint32_t*>(base + row1 * W + 16 * t + 2 * c) = act[h][t][1];
        *reinterpret_cast<uint32_t*>(base + row0 * W + 16 * t + 2 * c + 8) = act[h][t][2];
        *reinterpret_cast<uint32_t*>(base + row1 * W + 16 * t + 2 * c + 8) = act[h][t][3];
      }
    }
    if (c == 0) {
      sDy[row0] = dy0;
      sDy[row1] = dy1;
    }
    // backward: dpre of the last hidden layer = dy * w_out, masked by ReLU'
    float dpre[NT][4];
    {
      const __half* wo = sm + a.mlp.w_out;
      const int H1 = H - 1;
#pragma unroll
      for (int j = 0; j < NT; ++j) {
        const float w0 = __half2float(wo[8 * j + 2 * c]), w1 = __half2float(wo[8 * j + 2 * c + 1]);
        const float2 h0 = unpack_h2(act[H1][j / 2][(j & 1) ? 2 : 0]);
        const float2 h1 = unpack_h2(act[H1][j / 2][(j & 1) ? 3 : 1]);
        dpre[j][0] = h0.x > 0.0f ? dy0 * w0 : 0.0f;
        dpre[j][1] = h0.y > 0.0f ? dy0 * w1 : 0.0f;
        dpre[j][2] = h1.x > 0.0f ? dy1 * w0 : 0.0f;
        dpre[j][3] = h1.y > 0.0f ? dy1 * w1 : 0.0f;
      }
    }
#pragma unroll
    for (int h = H - 1; h >= 0; --h) {
      uint32_t da[W / 16][4];
#pragma unroll
      for (int t = 0; t < W / 16; ++t) c_to_a(da[t], dpre[2 * t], dpre[2 * t + 1]);
      __half* dbase = sD + h * kTrainRound * W;
#pragma unroll
      for (int t = 0; t < W / 16; ++t) {
        *reinterpret_cast<uint32_t*>(dbase + row0 * W + 16 * t + 2 * c) = da[t][0];
        *reinterpret_cast<uint32_t*>(dbase + row1 * W + 16 * t + 2 * c) = da[t][1];
        *reinterpret_cast<uint32_t*>(dbase + row0 * W + 16 * t + 2 * c + 8) = da[t][2];
        *reinterpret_cast<uint32_t*>(dbase + row1 * W + 16 * t + 2 * c + 8) = da[t][3];
      }
      if (h > 0) {
        // d act[h-1] = dpre[h] * W_hid[h-1]  (B[k][n] = W[k][n] = W^T[n][k])
        float nd[NT][4];
#pragma unroll
        for (int j = 0; j < NT; ++j) nd[j][0] = nd[j][1] = nd[j][2] = nd[j][3] = 0.0f;
#pragma unroll
        for (int kk = 0; kk < W / 16; ++kk) {
#pragma unroll
          for (int j = 0; j < NT; ++j) {
            uint32_t b[2];
            load_b_wt(b, smT + a.mlp.w_hid[h - 1], W, 8 * j, 16 * kk, g, c);
            mma16816(nd[j], da[kk], b);
          }
        }
#pragma unroll
        for (int j = 0; j < NT; ++j) {
          const float2 h0 = unpack_h2(act[h - 1][j / 2][(j & 1) ? 2 : 0]);
          const float2 h1 = unpack_h2(act[h - 1][j / 2][(j & 1) ? 3 : 1]);
          dpre[j][0] = h0.x > 0.0f ? nd[j][0] : 0.0f;
          dpre[j][1] = h0.y > 0.0f ? nd[j][1] : 0.0f;
          dpre[j][2] = h1.x > 0.0f ? nd[j][2] : 0.0f;
          dpre[j][3] = h1.y > 0.0f ? nd[j][3] : 0.0f;
        }
      } else {
        // dX = dpre[0] * W_in  -> grid gradient scatter (same (sample, level) pairs as the encode)
        float dx[IN / 8][4];
#pragma unroll
        for (int j = 0; j < IN / 8; ++j) dx[j][0] = dx[j][1] = dx[j][2] = dx[j][3] = 0.0f;
#pragma unroll
        for (int kk = 0; kk < W / 16; ++kk) {
#pragma unroll
          for (int j = 0; j < IN / 8; ++j) {
            uint32_t b[2];
            load_b_wt(b, smT + a.mlp.w_in, W, 8 * j, 16 * kk, g, c);
            mma16816(dx[j], da[kk], b);
          }
        }
        // n-tile j covers inputs 8j..8j+7; lane holds inputs 8j+2c, +1 = level 4j + c
#pragma unroll
        for (int j = 0; j < IN / 8; ++j) {
          const int l = 4 * j + c;
          if (l < a.grid.levels) {
            if (s0 < a.n) scatter_level(a.grid, a.grid_grad, l, u[0][0], u[0][1], u[0][2], make_float2(dx[j][0], dx[j][1]));
            if (s1 < a.n) scatter_level(a.grid, a.grid_grad, l, u[1][0], u[1][1], u[1][2], make_float2(dx[j][2], dx[j][3]));
          }
        }
      }
    }
    __syncthreads();
    // weight gradients over the staged 64 samples: G = dpre^T (W x 64) * input (64 x in)
    // this warp: rows [16*warp, 16*warp+16) of each matrix (only if warp < MT)
    if (warp < MT) {
      const int m0 = 16 * warp;
#pragma unroll
      for (int h = 0; h < H; ++h) {
        const __half* D = sD + h * kTrainRound * W;                  // [64 x W] dpre of layer h
        const __half* X = (h == 0) ? sX : sAct + (h - 1) * kTrainRound * W;  // layer input
        const int ld = (h == 0) ? IN : W;
        const int ntiles = (h == 0) ? IN / 8 : NT;
#pragma unroll
        for (int ks = 0; ks < kTrainRound / 16; ++ks) {
          // A[m][k] = D[k][m0+m]: lane needs A[g][2c..2c+1], A[g+8][..], A[g][2c+8..], A[g+8][2c+8..]
          const int k0 = 16 * ks;
          uint32_t af[4];
          {
            const __half* p = D + (k0 + 2 * c) * W + m0 + g;
            __half2 v;
            v = __halves2half2(p[0], p[W]);
            af[0] = *reinterpret_cast<uint32_t*>(&v);
            v = __halves2half2(p[8], p[W + 8]);
            af[1] = *reinterpret_cast<uint32_t*>(&v);
            v = __halves2half2(p[8 * W], p[9 * W]);
            af[2] = *reinterpret_cast<uint32_t*>(&v);
            v = __halves2half2(p[8 * W + 8], p[9 * W + 8]);
            af[3] = *reinterpret_cast<uint32_t*>(&v);
          }
          for (int j = 0; j < ntiles; ++j) {
            // B[k][n] = X[k0+k][8j+n]: lane needs B[2c..2c+1][g], B[2c+8..2c+9][g]
            const __half* q = X + (k0 + 2 * c) * ld + 8 * j + g;
            uint32_t bf[2];
            __half2 v = __halves2half2(q[0], q[ld]);
            bf[0] = *reinterpret_cast<uint32_t*>(&v);
            v = __halves2half2(q[8 * ld], q[9 * ld]);
            bf[1] = *reinterpret_cast<uint32_t*>(&v);
            if (h == 0) mma16816(gin[j], af, bf);
            else mma16816(ghid[h - 1][j], af, bf);
          }
        }
      }
    }
    // output-row gradient: sum_s dy[s] * act[H-1][s][n] (CUDA cores)
    {
      const __half* Xl = sAct + (H - 1) * kTrainRound * W;
      for (int n = threadIdx.x; n < W; n += blockDim.x) {
        float s = 0.0f;
        for (int k = 0; k < kTrainRound; ++k) s += sDy[k] * __half2float(Xl[k * W + n]);
        atomicAdd(a.mlp_grad + a.mlp.w_out + n, s);
      }
    }
    __syncthreads();
  }
  // flush this warp's weight-gradient tiles: C fragment rows m0+g, m0+g+8, cols 8j+2c..
  if (warp < MT) {
    const int m0 = 16 * warp;
    for (int j = 0; j < IN / 8; ++j) {
      float* G = a.mlp_grad + a.mlp.w_in;
      atomicAdd(G + (m0 + g) * IN + 8 * j + 2 * c, gin[j][0]);
      atomicAdd(G + (m0 + g) * IN + 8 * j + 2 * c + 1, gin[j][1]);
      atomicAdd(G + (m0 + g + 8) * IN + 8 * j + 2 * c, gin[j][2]);
      atomicAdd(G + (m0 + g + 8) * IN + 8 * j + 2 * c + 1, gin[j][3]);
    }
#pragma unroll
    for (int h = 1; h < H; ++h) {
      float* G = a.mlp_grad + a.mlp.w_hid[h - 1];
      for (int j = 0; j < NT; ++j) {
        atomicAdd(G + (m0 + g) * W + 8 * j + 2 * c, ghid[h - 1][j][0]);
        atomicAdd(G + (m0 + g) * W + 8 * j + 2 * c + 1, ghid[h - 1][j][1]);
        atomicAdd(G + (m0 + g + 8) * W + 8 * j + 2 * c, ghid[h - 1][j][2]);
        atomicAdd(G + (m0 + g + 8) * W + 8 * j + 2 * c + 1, ghid[h - 1][j][3]);
      }
    }
  }
  if (a.loss_sum) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) loss += __shfl_xor_sync(0xffffffffu, loss, o);
    if (lane == 0) atomicAdd(a.loss_sum, loss);
  }
}

// Adam (Kingma & Ba) on FP32 master parameters; refreshes the FP16 copy and
// clears the gradient.
__global__ void adam_kernel(float* __restrict__ p, __half* __restrict__ ph, float* __restrict__ g,
                            float* __restrict__ m, float* __restrict__ v, int64_t n, float lr, float b1, float b2,
                            float eps, float bc1, float bc2, float gscale) {
  const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float gi = g[i] * gscale;
  const float mi = b1 * m[i] + (1.0f - b1) * gi;
  const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  const float upd = lr * (mi / bc1) / (sqrtf(vi / bc2) + eps);
  const float pn = p[i] - upd;
  p[i] = pn;
  ph[i] = __float2half_rn(pn);
  g[i] = 0.0f;
}

__global__ void scale_kernel(float* __restrict__ g, int64_t n, float s) {
  const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i < n) g[i] *= s;
}

__global__ void to_half_kernel(const float* __restrict__ p, __half* __restrict__ ph, int64_t n) {
  const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i < n) ph[i] = __float2half_rn(p[i]);
}

__global__ void init_params_kernel(float* __restrict__ p, int64_t n_grid, const int* __restrict__ mlp_fan,
                                   int64_t n_total, uint64_t seed) {
  const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n_total) return;
  uint32_t k0, k1;
  philox_key(seed, 7u, k0, k1);
  const U4 r = philox4x32_10(U4{static_cast<uint32_t>(i), static_cast<uint32_t>(i >> 32), 0u, 0u}, k0, k1);
  const float u = 2.0f * u01(r.x) - 1.0f;
  if (i < n_grid) {
    p[i] = 1.0e-4f * u;  // hash-grid features: U(-1e-4, 1e-4)
  } else {
    // MLP weights: U(-s, s), s = sqrt(6 / (fan_in + fan_out))
    const int j = static_cast<int>(i - n_grid);
    p[i] = u * sqrtf(6.0f / static_cast<float>(mlp_fan[j]));
  }
}

}  // namespace
}  // namespace n2w

struct n2w_cache {
  n2w_cache_config cfg;
  n2w::GridMeta grid;
  n2w::MlpMeta mlp;
  int64_t n_grid = 0;  // floats of grid parameters (entries * F)
  int64_t n_total = 0;
  float* d_p = nullptr;     // fp32 master [grid | mlp]
  __half* d_ph = nullptr;   // fp16 working copy
  float* d_g = nullptr;     // fp32 gradient
  float* d_m = nullptr;
  float* d_v = nullptr;
  float* d_loss = nullptr;  // device scalar
  int64_t step = 0;
  int device = 0;
};

namespace n2w {
namespace {

void build_meta(n2w_cache& c) {
  const n2w_cache_config& k = c.cfg;
  N2W_REQUIRE(k.n_levels >= 1 && k.n_levels <= kMaxLevels, "n_levels must be in [1, 16]");
  N2W_REQUIRE(k.n_features_per_level == 2, "n_features_per_level must be 2");
  N2W_REQUIRE(k.log2_hashmap_size >= 10 && k.log2_hashmap_size <= 24, "log2_hashmap_size must be in [10, 24]");
  N2W_REQUIRE(k.base_resolution >= 2.0f, "base_resolution must be >= 2");
  N2W_REQUIRE(k.n_neurons == 16 || k.n_neurons == 32 || k.n_neurons == 64, "n_neurons must be 16, 32 or 64");
  N2W_REQUIRE(k.n_hidden_layers >= 1 && k.n_hidden_layers <= kMaxHidden, "n_hidden_layers must be in [1, 4]");
  float b = k.per_level_scale;
  if (!(b > 0.0f)) {
    N2W_REQUIRE(k.max_resolution >= k.base_resolution, "max_resolution must be >= base_resolution");
    b = k.n_levels > 1 ? std::exp((std::log(k.max_resolution) - std::log(k.base_resolution)) / (k.n_levels - 1)) : 1.0f;
  }
  c.cfg.per_level_scale = b;
  GridMeta& g = c.grid;
  std::memset(&g, 0, sizeof(g));
  g.levels = k.n_levels;
  g.features = 2;
  const uint64_t T = 1ull << k.log2_hashmap_size;
  uint64_t off = 0;
  for (int l = 0; l < k.n_levels; ++l) {
    // N_l = floor(N_min * b^l), evaluated in FP64 with a 1e-6 relative guard so
    // a level that is an exact power (e.g. 2048 = 16 * 128) is not rounded down.
    const double x = static_cast<double>(k.base_resolution) * std::pow(static_cast<double>(b), static_cast<double>(l));
    const uint32_t res = static_cast<uint32_t>(std::floor(x * (1.0 + 1e-6)));
    const uint64_t dense = static_cast<uint64_t>(res + 1) * (res + 1) * (res + 1);
    const uint64_t size = dense <= T ? ((dense + 7) / 8) * 8 : T;
    g.res[l] = res;
    g.scale[l] = static_cast<float>(res);
    g.dense[l] = dense <= T ? 1u : 0u;
    g.table_size[l] = static_cast<uint32_t>(size);
    g.offset[l] = static_cast<uint32_t>(off);
    off += size;
  }
  c.n_grid = static_cast<int64_t>(off) * 2;
  MlpMeta& m = c.mlp;
  m.width = k.n_neurons;
  m.hidden = k.n_hidden_layers;
  m.in_dim = k.n_levels * 2 <= 16 ? 16 : 32;
  int o = 0;
  m.w_in = o;
  o += m.width * m.in_dim;
  for (int h = 0; h < kMaxHidden; ++h) m.w_hid[h] = 0;
  for (int h = 0; h < m.hidden - 1; ++h) {
    m.w_hid[h] = o;
    o += m.width * m.width;
  }
  m.w_out = o;
  o += m.width;
  m.total = (o + 7) / 8 * 8;
  c.n_total = c.n_grid + m.total;
}

template <int W>
size_t train_smem_bytes(const MlpMeta& m, int in_dim) {
  return sizeof(__half) * (2 * static_cast<size_t>(m.total) + kTrainRound * in_dim +
                           2 * kMaxHidden * kTrainRound * static_cast<size_t>(W)) +
         sizeof(float) * kTrainRound;
}

NetArgs net_args(const n2w_cache& c) {
  NetArgs a{};
  a.grid = c.grid;
  a.mlp = c.mlp;
  a.table = reinterpret_cast<const __half2*>(c.d_ph);
  a.mlp_h = c.d_ph + c.n_grid;
  a.grid_grad = reinterpret_cast<float2*>(c.d_g);
  a.mlp_grad = c.d_g + c.n_grid;
  return a;
}

template <int W, int KS, int H>
void launch_infer_t(const NetArgs& a, cudaStream_t s) {
  const size_t smem = sizeof(__half) * a.mlp.total;
  const int64_t tiles = (a.n + 15) / 16;
  int64_t grid = std::min<int64_t>((tiles + 3) / 4, static_cast<int64_t>(sm_count_current()) * 8);
  grid = std::max<int64_t>(grid, 1);
  infer_kernel<W, KS, H><<<static_cast<unsigned>(grid), kTrainBlock, smem, s>>>(a);
  N2W_CUDA(cudaGetLastError());
}

template <int W, int KS, int H>
void launch_train_t(const NetArgs& a, cudaStream_t s) {
  const size_t smem = train_smem_bytes<W>(a.mlp, 16 * KS);
  auto k = train_kernel<W, KS, H>;
  N2W_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)));
  const int64_t rounds = (a.n + kTrainRound - 1) / kTrainRound;
  int64_t grid = std::min<int64_t>(rounds, static_cast<int64_t>(sm_count_current()) * 2);
  grid = std::max<int64_t>(grid, 1);
  k<<<static_cast<unsigned>(grid), kTrainBlock, smem, s>>>(a);
  N2W_CUDA(cudaGetLastError());
}

// Runtime (width, input k-steps, hidden layers) -> template instance.
template <template <int, int, int> class F>
void dispatch(const NetArgs& a, cudaStream_t s) {
  const int W = a.mlp.width, KS = a.mlp.in_dim / 16, H = a.mlp.hidden;
#define N2W_CACHE_CASE(w, k, h) \
  if (W == w && KS == k && H == h) return F<w, k, h>::run(a, s);
#define N2W_CACHE_H(w, k) N2W_CACHE_CASE(w, k, 1) N2W_CACHE_CASE(w, k, 2) N2W_CACHE_CASE(w, k, 3) N2W_CACHE_CASE(w, k, 4)
  N2W_CACHE_H(64, 2) N2W_CACHE_H(64, 1) N2W_CACHE_H(32, 2) N2W_CACHE_H(32, 1) N2W_CACHE_H(16, 2) N2W_CACHE_H(16, 1)
#undef N2W_CACHE_H
#undef N2W_CACHE_CASE
  throw Error(N2W_EINTERNAL, "unsupported cache network shape");
}

template <int W, int KS, int H>
struct InferL {
  static void run(const NetArgs& a, cudaStream_t s) { launch_infer_t<W, KS, H>(a, s); }
};
template <int W, int KS, int H>
struct TrainL {
  static void run(const NetArgs& a, cudaStream_t s) { launch_train_t<W, KS, H>(a, s); }
};

void launch_infer(const NetArgs& a, cudaStream_t s) { dispatch<InferL>(a, s); }
void launch_train(const NetArgs& a, cudaStream_t s) { dispatch<TrainL>(a, s); }

// fan_in + fan_out of each MLP parameter (for the uniform init bound).
std::vector<int> mlp_fans(const MlpMeta& m) {
  std::vector<int> f(static_cast<size_t>(m.total), 1);
  for (int i = 0; i < m.width * m.in_dim; ++i) f[m.w_in + i] = m.in_dim + m.width;
  for (int h = 0; h < m.hidden - 1; ++h)
    for (int i = 0; i < m.width * m.width; ++i) f[m.w_hid[h] + i] = 2 * m.width;
  for (int i = 0; i < m.width; ++i) f[m.w_out + i] = m.width + 1;
  return f;
}

void release_cache(n2w_cache* c) {
  if (!c) return;
  cudaFree(c->d_p);
  cudaFree(c->d_ph);
  cudaFree(c->d_g);
  cudaFree(c->d_m);
  cudaFree(c->d_v);
  cudaFree(c->d_loss);
  delete c;
}

constexpr uint64_t kCacheMagic = 0x31454843574E324Eull;  // "N2WCHE1"

}  // namespace
}  // namespace n2w

using namespace n2w;

extern "C" {

int n2w_cache_config_default(n2w_cache_config* out) {
  return guarded([&] {
    N2W_REQUIRE(out, "null output");
    std::memset(out, 0, sizeof(*out));
    out->n_levels = 16;
    out->n_features_per_level = 2;
    out->log2_hashmap_size = 19;
    out->base_resolution = 16.0f;
    out->max_resolution = 2048.0f;
    out->per_level_scale = 0.0f;
    out->n_neurons = 64;
    out->n_hidden_layers = 2;
    out->learning_rate = 1.0e-2f;
    out->beta1 = 0.9f;
    out->beta2 = 0.99f;
    out->epsilon = 1.0e-15f;
    out->seed = 1337;
  });
}

int n2w_cache_describe(const n2w_cache_config* cfg, int64_t* grid_params, int64_t* mlp_params,
                       int32_t* level_resolution, int32_t* level_table_size) {
  return guarded([&] {
    N2W_REQUIRE(cfg, "null config");
    n2w_cache c;
    c.cfg = *cfg;
    build_meta(c);
    if (grid_params) *grid_params = c.n_grid;
    if (mlp_params) *mlp_params = c.mlp.total;
    for (int l = 0; l < c.grid.levels; ++l) {
      if (level_resolution) level_resolution[l] = static_cast<int32_t>(c.grid.res[l]);
      if (level_table_size) level_table_size[l] = static_cast<int32_t>(c.grid.table_size[l]);
    }
  });
}

int n2w_cache_create(const n2w_cache_config* cfg, n2w_cache** out) {
  return guarded([&] {
    N2W_REQUIRE(cfg && out, "null argument");
    auto* c = new n2w_cache();
    try {
      c->cfg = *cfg;
      build_meta(*c);
      N2W_CUDA(cudaGetDevice(&c->device));
      const size_t n = static_cast<size_t>(c->n_total);
      N2W_CUDA(cudaMalloc(&c->d_p, n * sizeof(float)));
      N2W_CUDA(cudaMalloc(&c->d_ph, n * sizeof(__half)));
      N2W_CUDA(cudaMalloc(&c->d_g, n * sizeof(float)));
      N2W_CUDA(cudaMalloc(&c->d_m, n * sizeof(float)));
      N2W_CUDA(cudaMalloc(&c->d_v, n * sizeof(float)));
      N2W_CUDA(cudaMalloc(&c->d_loss, sizeof(float)));
      N2W_CUDA(cudaMemset(c->d_g, 0, n * sizeof(float)));
      N2W_CUDA(cudaMemset(c->d_m, 0, n * sizeof(float)));
      N2W_CUDA(cudaMemset(c->d_v, 0, n * sizeof(float)));
      std::vector<int> fans = mlp_fans(c->mlp);
      int* d_fans = nullptr;
      N2W_CUDA(cudaMalloc(&d_fans, fans.size() * sizeof(int)));
      N2W_CUDA(cudaMemcpy(d_fans, fans.data(), fans.size() * sizeof(int), cudaMemcpyHostToDevice));
      const int b = 256;
      init_params_kernel<<<static_cast<unsigned>((n + b - 1) / b), b>>>(c->d_p, c->n_grid, d_fans,
                                                                          c->n_total, c->cfg.seed);
      N2W_CUDA(cudaGetLastError());
      to_half_kernel<<<static_cast<unsigned>((n + b - 1) / b), b>>>(c->d_p, c->d_ph, c->n_total);
      N2W_CUDA(cudaGetLastError());
      N2W_CUDA(cudaDeviceSynchronize());
      cudaFree(d_fans);
    } catch (...) {
      release_cache(c);
      throw;
    }
    *out = c;
  });
}

void n2w_cache_destroy(n2w_cache* c) { release_cache(c); }

int n2w_cache_info(const n2w_cache* c, n2w_cache_config* cfg_out, int64_t* grid_params, int64_t* mlp_params,
                   int32_t* level_resolution, int32_t* level_table_size) {
  return guarded([&] {
    N2W_REQUIRE(c, "null cache");
    if (cfg_out) *cfg_out = c->cfg;
    if (grid_params) *grid_params = c->n_grid;
    if (mlp_params) *mlp_params = c->mlp.total;
    for (int l = 0; l < c->grid.levels; ++l) {
      if (level_resolution) level_resolution[l] = static_cast<int32_t>(c->grid.res[l]);
      if (level_table_size) level_table_size[l] = static_cast<int32_t>(c->grid.table_size[l]);
    }
  });
}

int n2w_cache_infer(const n2w_cache* c, const float* d_inputs, int64_t n, float* d_outputs, n2w_stream_t stream) {
  return guarded([&] {
    N2W_REQUIRE(c, "null cache");
    N2W_REQUIRE(n >= 0, "n must be non-negative");
    if (n == 0) return;
    N2W_REQUIRE(d_inputs && d_outputs, "null device pointer");
    NetArgs a = net_args(*c);
    a.inputs = d_inputs;
    a.outputs = d_outputs;
    a.n = n;
    launch_infer(a, stream);
  });
}

int n2w_cache_gradients(n2w_cache* c, const float* d_inputs, const float* d_targets, int64_t n, float* d_outputs,
                        n2w_stream_t stream) {
  return guarded([&] {
    N2W_REQUIRE(c, "null cache");
    N2W_REQUIRE(n > 0 && d_inputs && d_targets, "invalid arguments");
    NetArgs a = net_args(*c);
    a.inputs = d_inputs;
    a.targets = d_targets;
    a.outputs = d_outputs;
    a.n = n;
    // The backward runs on n * dL/dy = 2 (y - t): O(1) values keep FP16
    // activations' gradients out of the subnormal range; the 1/n is applied to
    // the FP32 gradient afterwards.
    a.loss_scale = 2.0f;
    a.loss_sum = c->d_loss;
    N2W_CUDA(cudaMemsetAsync(c->d_loss, 0, sizeof(float), stream));
    launch_train(a, stream);
    const int b = 256;
    scale_kernel<<<static_cast<unsigned>((c->n_total + b - 1) / b), b, 0, stream>>>(c->d_g, c->n_total,
                                                                                     1.0f / static_cast<float>(n));
    N2W_CUDA(cudaGetLastError());
  });
}

int n2w_cache_train_step(n2w_cache* c, const float* d_inputs, const float* d_targets, int64_t n, float* h_loss_out,
                         n2w_stream_t stream) {
  return guarded([&] {
    N2W_REQUIRE(c, "null cache");
    N2W_REQUIRE(n > 0 && d_inputs && d_targets, "invalid arguments");
    NetArgs a = net_args(*c);
    a.inputs = d_inputs;
    a.targets = d_targets;
    a.n = n;
    a.loss_scale = 2.0f;  // n * dL/dy; the 1/n is applied inside the Adam update
    a.loss_sum = c->d_loss;
    N2W_CUDA(cudaMemsetAsync(c->d_loss, 0, sizeof(float), stream));
    launch_train(a, stream);
    ++c->step;
    const float b1 = c->cfg.beta1, b2 = c->cfg.beta2;
    const float bc1 = 1.0f - std::pow(b1, static_cast<float>(c->step));
    const float bc2 = 1.0f - std::pow(b2, static_cast<float>(c->step));
    const int b = 256;
    adam_kernel<<<static_cast<unsigned>((c->n_total + b - 1) / b), b, 0, stream>>>(
        c->d_p, c->d_ph, c->d_g, c->d_m, c->d_v, c->n_total, c->cfg.learning_rate, b1, b2, c->cfg.epsilon, bc1, bc2,
        1.0f / static_cast<float>(n));
    N2W_CUDA(cudaGetLastError());
    if (h_loss_out) {
      float l = 0.0f;
      N2W_CUDA(cudaMemcpyAsync(&l, c->d_loss, sizeof(float), cudaMemcpyDeviceToHost, stream));
      N2W_CUDA(cudaStreamSynchronize(stream));
      *h_loss_out = l / static_cast<float>(n);
    }
  });
}

int n2w_cache_gradient_buffer(n2w_cache* c, float** d_grad, int64_t* count, float** d_loss_sum) {
  return guarded([&] {
    N2W_REQUIRE(c, "null cache");
    if (d_grad) *d_grad = c->d_g;
    if (count) *count = c->n_total;
    if (d_loss_sum) *d_loss_sum = c->d_loss;
  });
}

int n2w_cache_apply_gradients(n2w_cache* c, float grad_scale, n2w_stream_t stream) {
  return guarded([&] {
    N2W_REQUIRE(c, "null cache");
    N2W_REQUIRE(std::isfinite(grad_scale) && grad_scale > 0.0f, "grad_scale must be positive");
    ++c->step;
    const float b1 = c->cfg.beta1, b2 = c->cfg.beta2;
    const float bc1 = 1.0f - std::pow(b1, static_cast<float>(c->step));
    const float bc2 = 1.0f - std::pow(b2, static_cast<float>(c->step));
    const int b = 256;
    adam_kernel<<<static_cast<unsigned>((c->n_total + b - 1) / b), b, 0, stream>>>(
        c->d_p, c->d_ph, c->d_g, c->d_m, c->d_v, c->n_total, c->cfg.learning_rate, b1, b2, c->cfg.epsilon, bc1, bc2,
        grad_scale);
    N2W_CUDA(cudaGetLastError());
  });
}

int n2w_cache_get_params(const n2w_cache* c, float* h_fp32, uint16_t* h_fp16, float* h_grad) {
  return guarded([&] {
    N2W_REQUIRE(c, "null cache");
    const size_t n = static_cast<size_t>(c->n_total);
    if (h_fp32) N2W_CUDA(cudaMemcpy(h_fp32, c->d_p, n * sizeof(float), cudaMemcpyDeviceToHost));
    if (h_fp16) N2W_CUDA(cudaMemcpy(h_fp16, c->d_ph, n * sizeof(__half), cudaMemcpyDeviceToHost));
    if (h_grad) N2W_CUDA(cudaMemcpy(h_grad, c->d_g, n * sizeof(float), cudaMemcpyDeviceToHost));
  });
}

int n2w_cache_set_params(n2w_cache* c, const float* h_fp32) {
  return guarded([&] {
    N2W_REQUIRE(c && h_fp32, "null argument");
    const size_t n = static_cast<size_t>(c->n_total);
    N2W_CUDA(cudaMemcpy(c->d_p, h_fp32, n * sizeof(float), cudaMemcpyHostToDevice));
    const int b = 256;
    to_half_kernel<<<static_cast<unsigned>((n + b - 1) / b), b>>>(c->d_p, c->d_ph, c->n_total);
    N2W_CUDA(cudaGetLastError());
    N2W_CUDA(cudaMemset(c->d_g, 0, n * sizeof(float)));
    N2W_CUDA(cudaDeviceSynchronize());
  });
}

int n2w_cache_copy_params(n2w_cache* dst, const n2w_cache* src, n2w_stream_t stream) {
  return guarded([&] {
    N2W_REQUIRE(dst && src, "null argument");
    const n2w_cache_config& a = dst->cfg;
    const n2w_cache_config& b = src->cfg;
    N2W_REQUIRE(dst->n_total == src->n_total && a.n_levels == b.n_levels &&
                    a.n_features_per_level == b.n_features_per_level && a.log2_hashmap_size == b.log2_hashmap_size &&
                    a.base_resolution == b.base_resolution && a.per_level_scale == b.per_level_scale &&
                    a.max_resolution == b.max_resolution && a.n_neurons == b.n_neurons &&
                    a.n_hidden_layers == b.n_hidden_layers,
                "n2w_cache_copy_params: caches of different configurations");
    if (dst == src) return;
    const size_t n = static_cast<size_t>(src->n_total);
    N2W_CUDA(cudaMemcpyAsync(dst->d_p, src->d_p, n * sizeof(float), cudaMemcpyDeviceToDevice, stream));
    N2W_CUDA(cudaMemcpyAsync(dst->d_ph, src->d_ph, n * sizeof(__half), cudaMemcpyDeviceToDevice, stream));
  });
}

int n2w_cache_zero_grad(n2w_cache* c, n2w_stream_t stream) {
  return guarded([&] {
    N2W_REQUIRE(c, "null cache");
    N2W_CUDA(cudaMemsetAsync(c->d_g, 0, static_cast<size_t>(c->n_total) * sizeof(float), stream));
  });
}

// Binary checkpoint: magic, config, step, then fp32 params, Adam m, Adam v.
int n2w_cache_save(const n2w_cache* c, const char* path) {
  return guarded([&] {
    N2W_REQUIRE(c && path, "null argument");
    const size_t n = static_cast<size_t>(c->n_total);
    std::vector<float> buf(3 * n);
    N2W_CUDA(cudaMemcpy(buf.data(), c->d_p, n * sizeof(float), cudaMemcpyDeviceToHost));
    N2W_CUDA(cudaMemcpy(buf.data() + n, c->d_m, n * sizeof(float), cudaMemcpyDeviceToHost));
    N2W_CUDA(cudaMemcpy(buf.data() + 2 * n, c->d_v, n * sizeof(float), cudaMemcpyDeviceToHost));
    std::ofstream f(path, std::ios::binary);
    if (!f) throw Error(N2W_EIO, std::string("cannot write ") + path);
    const uint64_t magic = kCacheMagic, count = n;
    const int64_t step = c->step;
    f.write(reinterpret_cast<const char*>(&magic), 8);
    f.write(reinterpret_cast<const char*>(&c->cfg), sizeof(c->cfg));
    f.write(reinterpret_cast<const char*>(&step), 8);
    f.write(reinterpret_cast<const char*>(&count), 8);
    f.write(reinterpret_cast<const char*>(buf.data()), static_cast<std::streamsize>(buf.size() * sizeof(float)));
    if (!f) throw Error(N2W_EIO, std::string("write failed: ") + path);
  });
}

int n2w_cache_load(const char* path, n2w_cache** out) {
  return guarded([&] {
    N2W_REQUIRE(path && out, "null argument");
    std::ifstream f(path, std::ios::binary);
    if (!f) throw Error(N2W_EIO, std::string("cannot read ") + path);
    uint64_t magic = 0, count = 0;
    int64_t step = 0;
    n2w_cache_config cfg{};
    f.read(reinterpret_cast<char*>(&magic), 8);
    if (magic != kCacheMagic) throw Error(N2W_EIO, "not an n2w cache checkpoint");
    f.read(reinterpret_cast<char*>(&cfg), sizeof(cfg));
    f.read(reinterpret_cast<char*>(&step), 8);
    f.read(reinterpret_cast<char*>(&count), 8);
    n2w_cache* c = nullptr;
    const int st = n2w_cache_create(&cfg, &c);
    if (st != N2W_OK) throw Error(st, n2w_last_error());
    try {
      if (count != static_cast<uint64_t>(c->n_total)) throw Error(N2W_EIO, "checkpoint size mismatch");
      std::vector<float> buf(3 * count);
      f.read(reinterpret_cast<char*>(buf.data()), static_cast<std::streamsize>(buf.size() * sizeof(float)));
      if (!f) throw Error(N2W_EIO, "truncated checkpoint");
      const size_t n = count;
      N2W_CUDA(cudaMemcpy(c->d_p, buf.data(), n * sizeof(float), cudaMemcpyHostToDevice));
      N2W_CUDA(cudaMemcpy(c->d_m, buf.data() + n, n * sizeof(float), cudaMemcpyHostToDevice));
      N2W_CUDA(cudaMemcpy(c->d_v, buf.data() + 2 * n, n * sizeof(float), cudaMemcpyHostToDevice));
      const int b = 256;
      to_half_kernel<<<static_cast<unsigned>((n + b - 1) / b), b>>>(c->d_p, c->d_ph, c->n_total);
      N2W_CUDA(cudaGetLastError());
      N2W_CUDA(cudaDeviceSynchronize());
      c->step = step;
    } catch (...) {
      release_cache(c);
      throw;
    }
    *out = c;
  });
}

}  // extern "C"
