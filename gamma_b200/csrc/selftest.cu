// Device-side checks of numerical helpers for the test suite
// (gamma_b200/lib/libgamma_selftest.so; nothing on the product path loads it).
#include <cuda_runtime.h>

#include "physics.cuh"
#include "search.cuh"

namespace {

__global__ void pow_3_4_kernel(const double *x, double *mine, double *libm, int n) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    mine[i] = gb::pow_3_4(x[i]);
    libm[i] = pow(x[i], 0.75);
  }
}

__global__ void qdiv_kernel(const double *a, const double *b, double *mine, double *ieee, int n) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    mine[i] = gb::qdiv(a[i], b[i]);
    ieee[i] = a[i] / b[i];
  }
}

}  // namespace

extern "C" {

// gb::qdiv(a, b) and the plain IEEE quotient a / b of n host pairs, on the
// current device.  Returns 0 or the CUDA error code.
__attribute__((visibility("default"))) int gb_selftest_qdiv(const double *a, const double *b, double *mine,
                                                            double *ieee, int n) {
  if (n <= 0) return 0;
  double *d = nullptr;
  const size_t s = (size_t)n * sizeof(double);
  cudaError_t e = cudaMalloc(&d, 4 * s);
  if (e != cudaSuccess) return (int)e;
  e = cudaMemcpy(d, a, s, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(d + n, b, s, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) {
    qdiv_kernel<<<(n + 255) / 256, 256>>>(d, d + n, d + 2 * (size_t)n, d + 3 * (size_t)n, n);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpy(mine, d + 2 * (size_t)n, s, cudaMemcpyDeviceToHost);
  if (e == cudaSuccess) e = cudaMemcpy(ieee, d + 3 * (size_t)n, s, cudaMemcpyDeviceToHost);
  cudaFree(d);
  return (int)e;
}

// x^(3/4) of n host values by gb::pow_3_4 (mine) and by CUDA's pow (libm),
// both evaluated on the current device.  Returns 0 or the CUDA error code.
__attribute__((visibility("default"))) int gb_selftest_pow_3_4(const double *x, double *mine, double *libm, int n) {
  if (n <= 0) return 0;
  double *d = nullptr;
  const size_t b = (size_t)n * sizeof(double);
  cudaError_t e = cudaMalloc(&d, 3 * b);
  if (e != cudaSuccess) return (int)e;
  e = cudaMemcpy(d, x, b, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) {
    pow_3_4_kernel<<<(n + 255) / 256, 256>>>(d, d + n, d + 2 * (size_t)n, n);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpy(mine, d + n, b, cudaMemcpyDeviceToHost);
  if (e == cudaSuccess) e = cudaMemcpy(libm, d + 2 * (size_t)n, b, cudaMemcpyDeviceToHost);
  cudaFree(d);
  return (int)e;
}

// gb::d2::partition_from (the 2D passes' searches from a hint) against a
// linear scan, on the host: `cases` random sorted arrays with ties, keys in
// and around their range, hints in range and far outside it.  Returns the
// number of wrong results, or -1 if a probe left [lo0, hi0).
__attribute__((visibility("default"))) int gb_selftest_partition_from(unsigned seed, int cases) {
  unsigned long long r = seed * 6364136223846793005ULL + 1442695040888963407ULL;
  auto next = [&r](unsigned m) {  // LCG, high bits
    r = r * 6364136223846793005ULL + 1442695040888963407ULL;
    return (unsigned)((r >> 33) % m);
  };
  double X[64];
  int bad = 0;
  for (int t = 0; t < cases; ++t) {
    const int n = (int)next(41), lo0 = (int)next(3), hi0 = lo0 + n;
    double v = 0.;
    for (int k = 0; k < hi0 + 2; ++k) X[k] = (v += next(3));
    const double key = next((unsigned)v + 3);
    const long long h = next(5) == 0 ? (long long)next(2000001) - 1000000 : lo0 + (long long)next(n + 3) - 1;
    bool out = false;
    auto pred = [&](int k) {
      if (k < lo0 || k >= hi0) out = true;
      return k >= lo0 && k < hi0 && X[k] < key;
    };
    int ref = lo0;
    while (ref < hi0 && X[ref] < key) ++ref;
    const int got = gb::d2::partition_from(lo0, hi0, h, pred);
    if (out) return -1;
    if (got != ref) ++bad;
  }
  return bad;
}

}  // extern "C"
