// Learned initial guess for cons2prim: a 3 -> 64 -> 64 -> 2 MLP with SiLU.
//
// Inputs from the conserved state, with s = |S|/D and t = tau/D:
//   f0 = log1p(s) / 8                     (bulk motion)
//   f1 = log10(max(t - (sqrt(1+s^2) - 1), 1e-30)) / 10
//                                         (thermal part of tau/D: what is left
//                                          of tau/D once the cold-flow kinetic
//                                          part is removed, computed in FP64)
//   f2 = log10(D) / 6
// Outputs: y0 = (ln(p/D) + 14) / 10, y1 = ln(lfac) / 3.
// The thermal input replaces tau/D itself: for cold flow p/D sits 7-10 decades
// below tau/D, which no 8-bit-mantissa (BF16) input can resolve, while the
// difference taken in FP64 keeps it.
//
// The Newton iteration of cons2prim starts from p = D exp(10 y0 - 14) and
// still iterates to the reference tolerance: the network moves only the
// iteration count, never the converged root.
//
// Parameters are one FP32 array (layout below).  Training (mlp_train.cuh) uses
// hand-written FP32 kernels (forward, backward with block-staged weight
// gradients, Adam); inference inside cons2prim runs the three layers as BF16
// mma.sync (m16n8k16, FP32 accumulation) on a warp's 32 cells at a time.
#pragma once

#include <cuda_bf16.h>

#include "physics.cuh"

namespace gb {
namespace mlp {

constexpr int H = 64;
constexpr int OFF_W1 = 0;                // [H][3]
constexpr int OFF_B1 = OFF_W1 + H * 3;   // [H]
constexpr int OFF_W2 = OFF_B1 + H;       // [H][H]
constexpr int OFF_B2 = OFF_W2 + H * H;   // [H]
constexpr int OFF_W3 = OFF_B2 + H;       // [2][H]
constexpr int OFF_B3 = OFF_W3 + 2 * H;   // [2]
constexpr int NPARAM = OFF_B3 + 2;       // 4546

__device__ __forceinline__ float silu(float z) { return z / (1.f + __expf(-z)); }
__device__ __forceinline__ float dsilu(float z) {
  const float s = 1.f / (1.f + __expf(-z));
  return s + z * s * (1.f - s);
}

// network inputs of a conserved state (D, tau, S_r): the ratios and the
// thermal part in FP64 (the thermal part cancels), the logarithms in FP32
__device__ __forceinline__ void features(double D, double tau, double S, float f[3]) {
  const double s = fabs(S) / D, t = tau / D;
  const double th = t - (sqrt(1. + s * s) - 1.);
  f[0] = log1pf((float)s) * 0.125f;
  f[1] = __log10f(fmaxf((float)th, 1e-30f)) * 0.1f;
  f[2] = __log10f((float)D) * (1.f / 6.f);
}

__device__ __forceinline__ void targets(double D, double p, double lfac, float y[2]) {
  y[0] = (float)((log(p / D) + 14.) * 0.1);
  y[1] = (float)(log(lfac) * (1. / 3.));
}

__device__ __forceinline__ double guess_pressure(double D, float y0) {
  return D * (double)__expf(10.f * y0 - 14.f);
}

// Inside a time step the previous pressure is the better start almost
// everywhere (Newton stops after one or two iterations from it), so the steps
// start cons2prim from the network only where that warm start is poor
// (c2p_warm_start_poor in physics.cuh), and only in steps whose previous step
// found more than this fraction of its searches with a poor warm start (or
// that follow no step): the step with the guess carries the network's weights,
// its call sites and the waits of a warp's neighbours for it, which cost more
// than it saves where poor warm starts are rare.
constexpr double kGuessPolicy = 0.25;

// FP32 forward of one sample; optional pre-activations and activations for
// the backward pass (h1, h2 may be strided rows of shared memory)
__device__ __forceinline__ void forward(const float *P, const float x[3], float out[2], float *z1 = nullptr,
                                        float *h1 = nullptr, float *z2 = nullptr, float *h2 = nullptr) {
  float a1[H];
#pragma unroll 4
  for (int o = 0; o < H; ++o) {
    const float z = P[OFF_B1 + o] + P[OFF_W1 + 3 * o] * x[0] + P[OFF_W1 + 3 * o + 1] * x[1] +
                    P[OFF_W1 + 3 * o + 2] * x[2];
    if (z1) z1[o] = z;
    a1[o] = silu(z);
    if (h1) h1[o] = a1[o];
  }
  float o0 = P[OFF_B3], o1 = P[OFF_B3 + 1];
#pragma unroll 2
  for (int o = 0; o < H; ++o) {
    float z = P[OFF_B2 + o];
#pragma unroll 16
    for (int i = 0; i < H; ++i) z += P[OFF_W2 + H * o + i] * a1[i];
    if (z2) z2[o] = z;
    const float a = silu(z);
    if (h2) h2[o] = a;
    o0 += P[OFF_W3 + o] * a;
    o1 += P[OFF_W3 + H + o] * a;
  }
  out[0] = o0;
  out[1] = o1;
}

// ---------------------------------------------------------------------------
// BF16 tensor-core inference for a warp's 32 cells (two m16 tiles).
//
// B operands are stored in the m16n8k16 ".col" fragment order: for k-tile kt
// and n-tile nt, lane l holds {W[n][k0], W[n][k0+1]} and {W[n][k0+8], W[n][k0+9]}
// with n = 8 nt + l/4 and k0 = 16 kt + 2 (l%4); a warp reads one 256-byte row.
struct __align__(16) InferSmem {
  uint32_t w1[8][32][2];     // layer 1: K = 16 (3 used), N = 64
  uint32_t w2[4][8][32][2];  // layer 2: K = 64, N = 64
  uint32_t w3[4][32][2];     // layer 3: K = 64, N = 8 (2 used)
  float b1[H], b2[H], b3[2];
};

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
  __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<uint32_t *>(&v);
}

// build the fragment-ordered BF16 weights from the FP32 parameters (whole block)
__device__ inline void load_infer_weights(const float *P, InferSmem &s) {
  for (int idx = threadIdx.x; idx < 8 * 32; idx += blockDim.x) {
    const int nt = idx / 32, l = idx % 32, nn = nt * 8 + l / 4, k0 = 2 * (l % 4);
    auto w1 = [&](int k) { return k < 3 ? P[OFF_W1 + 3 * nn + k] : 0.f; };
    s.w1[nt][l][0] = pack_bf16(w1(k0), w1(k0 + 1));
    s.w1[nt][l][1] = pack_bf16(w1(k0 + 8), w1(k0 + 9));
  }
  for (int idx = threadIdx.x; idx < 4 * 8 * 32; idx += blockDim.x) {
    const int kt = idx / 256, nt = (idx / 32) % 8, l = idx % 32, nn = nt * 8 + l / 4, k0 = kt * 16 + 2 * (l % 4);
    const float *row = P + OFF_W2 + H * nn;
    s.w2[kt][nt][l][0] = pack_bf16(row[k0], row[k0 + 1]);
    s.w2[kt][nt][l][1] = pack_bf16(row[k0 + 8], row[k0 + 9]);
  }
  for (int idx = threadIdx.x; idx < 4 * 32; idx += blockDim.x) {
    const int kt = idx / 32, l = idx % 32, nn = l / 4, k0 = kt * 16 + 2 * (l % 4);
    auto w3 = [&](int k) { return nn < 2 ? P[OFF_W3 + H * nn + k] : 0.f; };
    s.w3[kt][l][0] = pack_bf16(w3(k0), w3(k0 + 1));
    s.w3[kt][l][1] = pack_bf16(w3(k0 + 8), w3(k0 + 9));
  }
  for (int i = threadIdx.x; i < H; i += blockDim.x) {
    s.b1[i] = P[OFF_B1 + i];
    s.b2[i] = P[OFF_B2 + i];
  }
  if (threadIdx.x < 2) s.b3[threadIdx.x] = P[OFF_B3 + threadIdx.x];
}

__device__ __forceinline__ void mma_bf16(float c[4], const uint32_t a[4], const uint32_t b[2]) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// bias + SiLU of one m16n8 accumulator tile and its repacking as half of an
// m16k16 A fragment of the next layer (n-tile nt -> k-tile nt/2)
__device__ __forceinline__ void act_to_a(const float c[4], const float *bias, int nt, int t, uint32_t a[4][4]) {
  const int col = nt * 8 + 2 * t;
  const float h0 = silu(c[0] + bias[col]), h1 = silu(c[1] + bias[col + 1]);
  const float h2 = silu(c[2] + bias[col]), h3 = silu(c[3] + bias[col + 1]);
  const int kt = nt >> 1, half = nt & 1;
  a[kt][half ? 2 : 0] = pack_bf16(h0, h1);  // row g
  a[kt][half ? 3 : 1] = pack_bf16(h2, h3);  // row g + 8
}

// The 32 lanes of a warp each bring one cell's inputs; each lane gets its
// cell's two network outputs.  All 32 lanes must call it together.
__device__ __forceinline__ void infer_warp(const InferSmem &s, const float f[3], float out[2]) {
  const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
#pragma unroll
  for (int mt = 0; mt < 2; ++mt) {
    // rows g and g+8 of m-tile mt are the cells of lanes 16 mt + g and 16 mt + g + 8
    const int r0 = mt * 16 + g, r1 = r0 + 8;
    float fa[3], fb[3];
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      fa[j] = __shfl_sync(0xffffffffu, f[j], r0);
      fb[j] = __shfl_sync(0xffffffffu, f[j], r1);
    }
    // layer-1 A: columns 2t, 2t+1 (inputs 0..2, zero padding up to 16)
    uint32_t a[4];
    a[0] = t == 0 ? pack_bf16(fa[0], fa[1]) : (t == 1 ? pack_bf16(fa[2], 0.f) : 0u);
    a[1] = t == 0 ? pack_bf16(fb[0], fb[1]) : (t == 1 ? pack_bf16(fb[2], 0.f) : 0u);
    a[2] = 0u;
    a[3] = 0u;
    uint32_t a2[4][4];
#pragma unroll
    for (int nt = 0; nt < 8; ++nt) {
      float c[4] = {0.f, 0.f, 0.f, 0.f};
      mma_bf16(c, a, s.w1[nt][lane]);
      act_to_a(c, s.b1, nt, t, a2);
    }
    uint32_t a3[4][4];
#pragma unroll
    for (int nt = 0; nt < 8; ++nt) {
      float c[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
      for (int kt = 0; kt < 4; ++kt) mma_bf16(c, a2[kt], s.w2[kt][nt][lane]);
      act_to_a(c, s.b2, nt, t, a3);
    }
    float c[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
    for (int kt = 0; kt < 4; ++kt) mma_bf16(c, a3[kt], s.w3[kt][lane]);
    // outputs of row r (columns 0, 1) sit in lane 4 (r & 7): c[0], c[1] for r < 8, c[2], c[3] above
    const int r = lane - mt * 16;
    const int src = 4 * (r & 7);
    const float lo0 = __shfl_sync(0xffffffffu, c[0], src);
    const float lo1 = __shfl_sync(0xffffffffu, c[1], src);
    const float hi0 = __shfl_sync(0xffffffffu, c[2], src);
    const float hi1 = __shfl_sync(0xffffffffu, c[3], src);
    if (r >= 0 && r < 16) {
      out[0] = ((r & 8) ? hi0 : lo0) + s.b3[0];
      out[1] = ((r & 8) ? hi1 : lo1) + s.b3[1];
    }
  }
}

// The network's starting pressure for the cells of a warp from their
// conserved D, tau and momentum magnitude S: every lane calls, lanes with
// on = false only take part in the tensor-core tiles (their result is 0).
// Out of line, with scalar arguments: inlined into a step's loop, the
// fragments took registers from it, which then spilled on every cell, guessed
// or not.
static __device__ __noinline__ double warp_guess_pressure(const InferSmem &s, double D, double tau, double S,
                                                          bool on) {
  float f[3] = {0.f, 0.f, 0.f}, o[2] = {0.f, 0.f};
  if (on) features(D, tau, S, f);
  __syncwarp();
  infer_warp(s, f, o);
  return on ? guess_pressure(D, o[0]) : 0.;
}

}  // namespace mlp
}  // namespace gb
