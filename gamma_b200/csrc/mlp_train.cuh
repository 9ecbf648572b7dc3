// Training side of the learned cons2prim guess: parameter initialisation,
// training pairs, FP32 forward/backward and Adam.  Included by one translation
// unit only (its kernels are not templates).
#pragma once

#include "mlp.cuh"

namespace gb {
namespace mlp {

// ---------------------------------------------------------------------------
// Parameter initialisation: uniform(-sqrt(6/(fan_in+fan_out)), +...) weights
// (Glorot), zero biases, from a counter-based hash of (seed, index).

__device__ __forceinline__ unsigned long long mix64(unsigned long long z) {
  // splitmix64 finaliser (Steele, Lea, Flood 2014)
  z += 0x9e3779b97f4a7c15ull;
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
  return z ^ (z >> 31);
}
__device__ __forceinline__ double uniform01(unsigned long long seed, unsigned long long k, int j) {
  return (double)(mix64(seed ^ mix64(8 * k + j)) >> 11) * (1.0 / 9007199254740992.0);
}

__global__ void init_kernel(float *P, unsigned long long seed) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < NPARAM; i += gridDim.x * blockDim.x) {
    float lim = 0.f;
    if (i < OFF_B1) lim = sqrtf(6.f / (3 + H));
    else if (i >= OFF_W2 && i < OFF_B2) lim = sqrtf(6.f / (H + H));
    else if (i >= OFF_W3 && i < OFF_B3) lim = sqrtf(6.f / (H + 2));
    P[i] = lim * (float)(2. * uniform01(seed, i, 0) - 1.);
  }
}

// ---------------------------------------------------------------------------
// Training pairs from primitive states [NQ rows][n] (the first n pairs) and
// uniform draws (the next nu): ln lfac ~ U(0, ln 1e3), log10 p/rho ~ U(-10, 3),
// log10 rho ~ U(-6, 6), direction of motion +-1 with equal probability.
template <class Cfg>
__global__ void pairs_kernel(Phys ph, const double *prim, long long n, long long nu, unsigned long long seed,
                             float *x, float *y) {
  constexpr int NQ = Cfg::NQ;
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n + nu;
       k += (long long)gridDim.x * blockDim.x) {
    double pr[NQ], cs[NQ];
#pragma unroll
    for (int q = 0; q < NQ; ++q) pr[q] = 0.;
    if (k < n) {
#pragma unroll
      for (int q = 0; q < NQ; ++q) pr[q] = prim[q * n + k];
      pr[UU2] = 0.;
    } else {
      const unsigned long long kk = k - n;
      const double lg = exp(uniform01(seed, kk, 0) * log(1e3));
      const double pr_rho = pow(10., -10. + 13. * uniform01(seed, kk, 1));
      const double rho = pow(10., -6. + 12. * uniform01(seed, kk, 2));
      const double sgn = uniform01(seed, kk, 3) < 0.5 ? -1. : 1.;
      pr[RHO] = rho;
      pr[PPP] = rho * pr_rho;
      pr[UU1] = sgn * sqrt(fmax(lg * lg - 1., 0.));
      pr[TR1] = 1.;
    }
    prim2cons<Cfg>(ph, pr, cs);
    float f[3], t[2];
    features(cs[DEN], cs[TAU], cs[SS1], f);
    targets(cs[DEN], pr[PPP], lfac_of(pr[UU1]), t);
    x[3 * k + 0] = f[0];
    x[3 * k + 1] = f[1];
    x[3 * k + 2] = f[2];
    y[2 * k + 0] = t[0];
    y[2 * k + 1] = t[1];
  }
}

// ---------------------------------------------------------------------------
// Training: loss = sum over a mini-batch and both outputs of (out - y)^2 / (2 m).
// One thread per sample does the forward and backward pass; per-sample deltas
// and activations are staged in shared memory (rows padded to H+1 floats), and
// every thread then owns a fixed set of parameter gradients, which it sums over
// the block's samples and adds to the global gradient once.  Sample j of the
// mini-batch is pair (perm_mul * (start + j) + perm_add) mod n_total, a
// bijection when gcd(perm_mul, n_total) = 1 (the host checks).

constexpr int TB = 128;  // samples per chunk = threads per block
constexpr int HP = H + 1;

struct TrainSmem {
  float P[NPARAM];
  float x[TB][3];
  float d1[TB][HP];  // dL/dz1
  float h1[TB][HP];
  float d2[TB][HP];  // dL/dz2
  float h2[TB][HP];
  float d3[TB][2];   // dL/dout
};

__global__ void __launch_bounds__(TB) grad_kernel(const float *Pg, const float *x, const float *y, long long n_total,
                                                  long long perm_mul, long long perm_add, long long start, int m,
                                                  float *grad, float *loss) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  TrainSmem &sm = *reinterpret_cast<TrainSmem *>(smem_raw);
  const int tid = threadIdx.x;
  for (int i = tid; i < NPARAM; i += TB) sm.P[i] = Pg[i];
  __syncthreads();
  constexpr int PER = (NPARAM + TB - 1) / TB;
  float acc[PER];
#pragma unroll
  for (int j = 0; j < PER; ++j) acc[j] = 0.f;
  const float inv_m = 1.f / (float)m;
  float lsum = 0.f;

  for (int base = blockIdx.x * TB; base < m; base += gridDim.x * TB) {
    const int j = base + tid;
    const bool valid = j < m;
    float xi[3] = {0.f, 0.f, 0.f}, yi[2] = {0.f, 0.f};
    if (valid) {
      const long long k = (long long)(((unsigned long long)perm_mul * (unsigned long long)(start + j) +
                                       (unsigned long long)perm_add) % (unsigned long long)n_total);
      xi[0] = x[3 * k];
      xi[1] = x[3 * k + 1];
      xi[2] = x[3 * k + 2];
      yi[0] = y[2 * k];
      yi[1] = y[2 * k + 1];
    }
    float z1[H], z2[H], out[2];
    forward(sm.P, xi, out, z1, sm.h1[tid], z2, sm.h2[tid]);
    float dout[2] = {0.f, 0.f};
    if (valid) {
#pragma unroll
      for (int q = 0; q < 2; ++q) {
        const float e = out[q] - yi[q];
        lsum += e * e;
        dout[q] = e * inv_m;
      }
    }
    sm.d3[tid][0] = dout[0];
    sm.d3[tid][1] = dout[1];
    sm.x[tid][0] = xi[0];
    sm.x[tid][1] = xi[1];
    sm.x[tid][2] = xi[2];
    // dL/dz2 = (W3^T dout) * silu'(z2)
#pragma unroll 8
    for (int i = 0; i < H; ++i) {
      z2[i] = (sm.P[OFF_W3 + i] * dout[0] + sm.P[OFF_W3 + H + i] * dout[1]) * dsilu(z2[i]);
      sm.d2[tid][i] = z2[i];
    }
    // dL/dz1 = (W2^T dL/dz2) * silu'(z1)
#pragma unroll 2
    for (int i = 0; i < H; ++i) {
      float s = 0.f;
#pragma unroll 16
      for (int o = 0; o < H; ++o) s += sm.P[OFF_W2 + H * o + i] * z2[o];
      sm.d1[tid][i] = s * dsilu(z1[i]);
    }
    __syncthreads();
    // parameter gradients owned by this thread
#pragma unroll
    for (int q = 0; q < PER; ++q) {
      const int g = tid + q * TB;
      if (g >= NPARAM) break;
      float s = 0.f;
      if (g < OFF_B1) {  // W1[o][i]
        const int o = g / 3, i = g % 3;
        for (int t = 0; t < TB; ++t) s += sm.d1[t][o] * sm.x[t][i];
      } else if (g < OFF_W2) {
        const int o = g - OFF_B1;
        for (int t = 0; t < TB; ++t) s += sm.d1[t][o];
      } else if (g < OFF_B2) {  // W2[o][i]
        const int o = (g - OFF_W2) / H, i = (g - OFF_W2) % H;
        for (int t = 0; t < TB; ++t) s += sm.d2[t][o] * sm.h1[t][i];
      } else if (g < OFF_W3) {
        const int o = g - OFF_B2;
        for (int t = 0; t < TB; ++t) s += sm.d2[t][o];
      } else if (g < OFF_B3) {  // W3[r][i]
        const int r = (g - OFF_W3) / H, i = (g - OFF_W3) % H;
        for (int t = 0; t < TB; ++t) s += sm.d3[t][r] * sm.h2[t][i];
      } else {
        const int r = g - OFF_B3;
        for (int t = 0; t < TB; ++t) s += sm.d3[t][r];
      }
      acc[q] += s;
    }
    __syncthreads();
  }
#pragma unroll
  for (int q = 0; q < PER; ++q) {
    const int g = tid + q * TB;
    if (g < NPARAM) atomicAdd(&grad[g], acc[q]);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) lsum += __shfl_xor_sync(0xffffffffu, lsum, o);
  if (loss && (tid & 31) == 0) atomicAdd(loss, 0.5f * lsum * inv_m);
}

// Adam (Kingma & Ba 2015) with bias corrections bc1 = 1 - b1^t, bc2 = 1 - b2^t
__global__ void adam_kernel(float *P, const float *grad, float *m, float *v, float lr, float b1, float b2, float eps,
                            float bc1, float bc2) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < NPARAM; i += gridDim.x * blockDim.x) {
    const float g = grad[i];
    const float mi = b1 * m[i] + (1.f - b1) * g;
    const float vi = b2 * v[i] + (1.f - b2) * g * g;
    m[i] = mi;
    v[i] = vi;
    P[i] -= lr * (mi / bc1) / (sqrtf(vi / bc2) + eps);
  }
}

// FP32 forward of n samples (x [n][3] -> out [n][2])
__global__ void forward_kernel(const float *P, const float *x, long long n, float *out) {
  __shared__ float sP[NPARAM];
  for (int i = threadIdx.x; i < NPARAM; i += blockDim.x) sP[i] = P[i];
  __syncthreads();
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
    const float xi[3] = {x[3 * k], x[3 * k + 1], x[3 * k + 2]};
    float o[2];
    forward(sP, xi, o);
    out[2 * k] = o[0];
    out[2 * k + 1] = o[1];
  }
}

}  // namespace mlp
}  // namespace gb
