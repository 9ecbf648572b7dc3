// C-ABI of the learned cons2prim guess (include/gamma_gpu.h): training-pair
// generation, initialisation, training (FP32 forward/backward + Adam), batched
// inference (FP32 or BF16 tensor cores) and cons2prim started from the network.
#include "gamma_gpu.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <numeric>
#include <vector>

#include "mlp_train.cuh"

namespace {

using gb::mlp::NPARAM;

int sm_count() {
  int dev = 0, nsm = 148;
  if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  return nsm;
}

int kind_of(const gamma_config_t *cfg) {
  if (!cfg || cfg->ngst != 2 || !(cfg->gamma_ad > 1.)) return -1;
  if (cfg->geometry == GAMMA_GEOM_SPHERICAL1D && cfg->hydro == GAMMA_HYDRO_REL_SPH && cfg->nq == 10) return 1;
  if (cfg->geometry == GAMMA_GEOM_CARTESIAN && cfg->hydro == GAMMA_HYDRO_REL_CART && cfg->nq == 6 &&
      cfg->eos == GAMMA_EOS_IDEAL)
    return 0;
  return -1;
}

gb::Phys phys_of(const gamma_config_t &c) {
  gb::Phys p;
  p.gamma_ad = c.gamma_ad;
  p.kgam = c.gamma_ad / (c.gamma_ad - 1.);
  p.cfl = c.cfl;
  p.vi = c.vi;
  p.eos = c.eos;
  p.ngst = c.ngst;
  p.eos_ws = c.eos_wavespeeds;
  p.euler = c.timestep == GAMMA_TS_EULER;
  return p;
}

// BF16 tensor-core inference of n samples (one warp per 32 samples)
__global__ void infer_kernel(const float *P, const float *x, long long n, float *out) {
  __shared__ gb::mlp::InferSmem s;
  gb::mlp::load_infer_weights(P, s);
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const long long warps = (long long)gridDim.x * (blockDim.x >> 5);
  for (long long base = (blockIdx.x * (long long)(blockDim.x >> 5) + (threadIdx.x >> 5)) * 32; base < n;
       base += warps * 32) {
    const long long k = base + lane;
    float f[3] = {0.f, 0.f, 0.f}, o[2] = {0.f, 0.f};
    if (k < n) {
      f[0] = x[3 * k];
      f[1] = x[3 * k + 1];
      f[2] = x[3 * k + 2];
    }
    __syncwarp();
    gb::mlp::infer_warp(s, f, o);
    if (k < n) {
      out[2 * k] = o[0];
      out[2 * k + 1] = o[1];
    }
  }
}

// cons2prim started from the network's pressure (one warp per 32 cells).
// cons/prim: [NQ rows][n] in the reference's slot order.
template <class Cfg>
__global__ void cons2prim_guess_kernel(gb::Phys ph, const float *P, double *cons, double *prim, int n, int *iters) {
  constexpr int NQ = Cfg::NQ;
  __shared__ gb::mlp::InferSmem s;
  gb::mlp::load_infer_weights(P, s);
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const int warps = gridDim.x * (blockDim.x >> 5);
  for (int base = (blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5)) * 32; base < n; base += warps * 32) {
    const int k = base + lane;
    const bool on = k < n;
    double c[NQ], p[NQ];
    float f[3] = {0.f, 0.f, 0.f}, o[2] = {0.f, 0.f};
    if (on) {
#pragma unroll
      for (int q = 0; q < NQ; ++q) {
        c[q] = cons[(long long)q * n + k];
        p[q] = prim[(long long)q * n + k];
      }
      gb::mlp::features(c[gb::DEN], c[gb::TAU], c[gb::SS1], f);
    }
    __syncwarp();
    gb::mlp::infer_warp(s, f, o);
    if (on) {
      const double pg = gb::mlp::guess_pressure(c[gb::DEN], o[0]);
      if (isfinite(pg) && pg > 0.) p[gb::PPP] = pg;
      gb::C2PStats st;
      gb::cons2prim<Cfg>(ph, c, p, &st);
#pragma unroll
      for (int q = 0; q < NQ; ++q) {
        cons[(long long)q * n + k] = c[q];
        prim[(long long)q * n + k] = p[q];
      }
      if (iters) iters[k] = st.iters;
    }
  }
}

long long gcd64(long long a, long long b) {
  while (b) {
    const long long t = a % b;
    a = b;
    b = t;
  }
  return a;
}

unsigned long long host_mix(unsigned long long z) {
  z += 0x9e3779b97f4a7c15ull;
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
  return z ^ (z >> 31);
}

}  // namespace

#define GAMMA_API __attribute__((visibility("default")))

extern "C" {

GAMMA_API int gamma_mlp_param_count(void) { return NPARAM; }

GAMMA_API int gamma_mlp_init(float *params, unsigned long long seed, void *stream) {
  if (!params) return GAMMA_ERR_INVALID;
  gb::mlp::init_kernel<<<(NPARAM + 255) / 256, 256, 0, (cudaStream_t)stream>>>(params, seed);
  return cudaGetLastError() == cudaSuccess ? GAMMA_OK : GAMMA_ERR_CUDA;
}

GAMMA_API int gamma_mlp_pairs(const gamma_config_t *cfg, const double *prim, long long n_states,
                              long long n_uniform, unsigned long long seed, float *x, float *y, void *stream) {
  const int kind = kind_of(cfg);
  if (kind < 0 || n_states < 0 || n_uniform < 0 || !x || !y || (n_states > 0 && !prim)) return GAMMA_ERR_INVALID;
  const long long n = n_states + n_uniform;
  if (n == 0) return GAMMA_OK;
  const int bs = 256;
  const int grid = (int)std::min<long long>((n + bs - 1) / bs, (long long)sm_count() * 8);
  cudaStream_t s = (cudaStream_t)stream;
  if (kind == 1)
    gb::mlp::pairs_kernel<gb::CfgSph><<<grid, bs, 0, s>>>(phys_of(*cfg), prim, n_states, n_uniform, seed, x, y);
  else
    gb::mlp::pairs_kernel<gb::CfgCart><<<grid, bs, 0, s>>>(phys_of(*cfg), prim, n_states, n_uniform, seed, x, y);
  return cudaGetLastError() == cudaSuccess ? GAMMA_OK : GAMMA_ERR_CUDA;
}

GAMMA_API int gamma_mlp_train(float *params, const float *x, const float *y, long long n,
                              const gamma_mlp_train_t *tc, float *loss_per_epoch, void *stream) {
  if (!params || !x || !y || !tc || n <= 0 || tc->epochs < 0 || tc->batch <= 0 || !(tc->lr > 0.f))
    return GAMMA_ERR_INVALID;
  cudaStream_t s = (cudaStream_t)stream;
  float *ws = nullptr;  // grad, m, v, per-epoch loss
  const size_t words = 3 * (size_t)NPARAM + (size_t)std::max(tc->epochs, 1);
  if (cudaMalloc(&ws, words * sizeof(float)) != cudaSuccess) return GAMMA_ERR_CUDA;
  float *grad = ws, *m = ws + NPARAM, *v = ws + 2 * NPARAM, *loss = ws + 3 * NPARAM;
  int rc = GAMMA_OK;
  auto check = [&](cudaError_t e) {
    if (e != cudaSuccess && rc == GAMMA_OK) rc = GAMMA_ERR_CUDA;
  };
  check(cudaMemsetAsync(ws, 0, words * sizeof(float), s));
  const size_t smem = sizeof(gb::mlp::TrainSmem);
  check(cudaFuncSetAttribute(gb::mlp::grad_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const int nsm = sm_count();
  const long long steps_per_epoch = (n + tc->batch - 1) / tc->batch;
  const long long total_steps = steps_per_epoch * tc->epochs;
  const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  float pb1 = 1.f, pb2 = 1.f;
  long long step = 0;
  // multipliers coprime with n (sample order of each epoch)
  static const long long kMul[] = {1000003, 999983, 999979, 999961, 999959, 999953, 999931, 999917};
  for (int e = 0; e < tc->epochs && rc == GAMMA_OK; ++e) {
    const unsigned long long h = host_mix(tc->seed ^ (0x1234567ull + (unsigned long long)e));
    long long mul = 1;
    for (int j = 0; j < 8; ++j) {
      const long long cand = kMul[(h + j) % 8] % n;
      if (cand > 0 && gcd64(cand, n) == 1) {
        mul = cand;
        break;
      }
    }
    const long long add = (long long)(h % (unsigned long long)n);
    for (long long b = 0; b < steps_per_epoch && rc == GAMMA_OK; ++b, ++step) {
      const long long start = b * tc->batch;
      const int cnt = (int)std::min<long long>(tc->batch, n - start);
      check(cudaMemsetAsync(grad, 0, NPARAM * sizeof(float), s));
      const int grid = std::max(1, std::min((cnt + gb::mlp::TB - 1) / gb::mlp::TB, nsm));
      gb::mlp::grad_kernel<<<grid, gb::mlp::TB, smem, s>>>(params, x, y, n, mul, add, start, cnt, grad, loss + e);
      check(cudaGetLastError());
      // cosine decay from lr to lr_final over all steps
      const double frac = total_steps > 1 ? (double)step / (double)(total_steps - 1) : 0.;
      const float lr = (float)(tc->lr_final + 0.5 * (tc->lr - tc->lr_final) * (1. + std::cos(M_PI * frac)));
      pb1 *= b1;
      pb2 *= b2;
      gb::mlp::adam_kernel<<<(NPARAM + 255) / 256, 256, 0, s>>>(params, grad, m, v, lr, b1, b2, eps, 1.f - pb1,
                                                                 1.f - pb2);
      check(cudaGetLastError());
    }
  }
  if (rc == GAMMA_OK && loss_per_epoch && tc->epochs > 0) {
    std::vector<float> h(tc->epochs);
    check(cudaMemcpyAsync(h.data(), loss, tc->epochs * sizeof(float), cudaMemcpyDeviceToHost, s));
    check(cudaStreamSynchronize(s));
    // each step added its mini-batch mean loss: the epoch value is their mean
    for (int e = 0; e < tc->epochs; ++e) loss_per_epoch[e] = h[e] / (float)steps_per_epoch;
  }
  check(cudaStreamSynchronize(s));
  cudaFree(ws);
  return rc;
}

GAMMA_API int gamma_mlp_loss_grad(const float *params, const float *x, const float *y, int n, float *grad,
                                  float *loss, void *stream) {
  if (!params || !x || !y || !grad || n <= 0) return GAMMA_ERR_INVALID;
  cudaStream_t s = (cudaStream_t)stream;
  const size_t smem = sizeof(gb::mlp::TrainSmem);
  if (cudaFuncSetAttribute(gb::mlp::grad_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
      cudaSuccess)
    return GAMMA_ERR_CUDA;
  if (cudaMemsetAsync(grad, 0, NPARAM * sizeof(float), s) != cudaSuccess) return GAMMA_ERR_CUDA;
  if (loss && cudaMemsetAsync(loss, 0, sizeof(float), s) != cudaSuccess) return GAMMA_ERR_CUDA;
  const int grid = std::max(1, std::min((n + gb::mlp::TB - 1) / gb::mlp::TB, sm_count()));
  // the samples in order (multiplier 1, offset 0), one mini-batch of n
  gb::mlp::grad_kernel<<<grid, gb::mlp::TB, smem, s>>>(params, x, y, n, 1, 0, 0, n, grad, loss);
  return cudaGetLastError() == cudaSuccess ? GAMMA_OK : GAMMA_ERR_CUDA;
}

GAMMA_API int gamma_mlp_forward(const float *params, const float *x, long long n, float *out, int tensor_cores,
                                void *stream) {
  if (!params || !x || !out || n < 0) return GAMMA_ERR_INVALID;
  if (n == 0) return GAMMA_OK;
  cudaStream_t s = (cudaStream_t)stream;
  const int nsm = sm_count();
  if (tensor_cores) {
    const long long warps = (n + 31) / 32;
    const int grid = (int)std::min<long long>((warps + 3) / 4, (long long)nsm * 8);
    infer_kernel<<<grid, 128, 0, s>>>(params, x, n, out);
  } else {
    const int grid = (int)std::min<long long>((n + 127) / 128, (long long)nsm * 8);
    gb::mlp::forward_kernel<<<grid, 128, 0, s>>>(params, x, n, out);
  }
  return cudaGetLastError() == cudaSuccess ? GAMMA_OK : GAMMA_ERR_CUDA;
}

GAMMA_API int gamma_gpu_cons2prim_guess(const gamma_config_t *cfg, double *cons, double *prim, int n, int *iters,
                                        const float *params, void *stream) {
  const int kind = kind_of(cfg);
  if (kind < 0 || !cons || !prim || !params || n < 0) return GAMMA_ERR_INVALID;
  if (n == 0) return GAMMA_OK;
  cudaStream_t s = (cudaStream_t)stream;
  const int warps = (n + 31) / 32;
  const int grid = std::min((warps + 3) / 4, sm_count() * 8);
  if (kind == 1)
    cons2prim_guess_kernel<gb::CfgSph><<<grid, 128, 0, s>>>(phys_of(*cfg), params, cons, prim, n, iters);
  else
    cons2prim_guess_kernel<gb::CfgCart><<<grid, 128, 0, s>>>(phys_of(*cfg), params, cons, prim, n, iters);
  return cudaGetLastError() == cudaSuccess ? GAMMA_OK : GAMMA_ERR_CUDA;
}

}  // extern "C"
