// Launch-shape variants of the 1D step kernel for the autotuner
// (gamma_gpu_autotune).  Variant 0 is the default kernel of gamma_api.cu
// (128 threads per run, one cell per thread per sweep chunk); variants 1..
// change the threads per run (the CTA size) and the cells each thread takes
// per chunk.  The arithmetic of every cell is the same in all of them, so
// they give identical results; only the speed differs.
#pragma once

#include <cuda_runtime.h>

#include "track_step.cuh"

namespace gb {
namespace tune {

constexpr int kVariants = 8;  // variant 0 included

struct Shape {
  int threads, cells_per_thread;
};

// threads per run and cells per thread of each variant
constexpr Shape kShapes[kVariants] = {{128, 1}, {64, 1}, {256, 1}, {128, 2}, {64, 2}, {128, 4}, {512, 1}, {256, 2}};

// the register cap of each variant keeps the default's resident warps per SM
constexpr int min_blocks(int default_blocks, int threads) {
  return default_blocks * 128 / threads > 0 ? default_blocks * 128 / threads : 1;
}

// Launch shape and launch of variant v >= 1: the cartesian tubes (CfgCart)
// and the spherical BM1D runs (CfgSph).
#define GB_TUNE_DECL(cfg)                                                                                      \
  cudaError_t configure_##cfg(int v, int nruns, int max_cap, int *grid, size_t *smem);                        \
  cudaError_t launch_##cfg(int v, int grid, size_t smem, cudaStream_t s, const Tracks &T, const Phys &ph,     \
                           int nsteps, const int *order, int nruns, int *queue, StepStats *stats,             \
                           int regrid_only, unsigned words_bytes);
GB_TUNE_DECL(cart)
GB_TUNE_DECL(sph)
#undef GB_TUNE_DECL

}  // namespace tune
}  // namespace gb
