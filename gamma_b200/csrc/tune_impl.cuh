// The step-kernel variants of one configuration (Cfg = GB_TUNE_CFG, entry
// points GB_TUNE_CONFIGURE / GB_TUNE_LAUNCH); included by gamma_tune_cart.cu
// and gamma_tune_sph.cu so that the two compile apart.
#pragma once

#include <algorithm>

#include "smem_limit.h"
#include "tune.h"

namespace gb {
namespace tune {
namespace {

using C = GB_TUNE_CFG;

template <int V>
struct Kern {
  static constexpr int BS = kShapes[V].threads, CPT = kShapes[V].cells_per_thread;
  static constexpr int MINB = min_blocks(C::MIN_BLOCKS, BS);
  static constexpr auto fn = track_step_kernel<C, BS, false, CPT, MINB>;
  static size_t smem(int max_cap) {
    return sizeof(typename TrackStep<C, BS, false, CPT>::Smem) + 4u * 4u * (size_t)regrid_words(max_cap);
  }
};

template <int V>
cudaError_t configure_v(int nruns, int max_cap, int *grid, size_t *smem) {
  using K = Kern<V>;
  *smem = K::smem(max_cap);
  cudaError_t e = raise_smem_limit((const void *)K::fn, *smem);
  if (e != cudaSuccess) return e;
  int dev = 0, nsm = 0, occ = 0;
  if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
  if ((e = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
  if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, K::fn, K::BS, *smem)) != cudaSuccess) return e;
  *grid = std::min(nruns, nsm * std::max(occ, 1));
  return cudaSuccess;
}

template <int V>
cudaError_t launch_v(int grid, size_t smem, cudaStream_t s, const Tracks &T, const Phys &ph, int nsteps,
                     const int *order, int nruns, int *queue, StepStats *stats, int regrid_only, unsigned wb) {
  using K = Kern<V>;
  K::fn<<<grid, K::BS, smem, s>>>(T, ph, nsteps, order, nruns, queue, stats, regrid_only, wb);
  return cudaGetLastError();
}

}  // namespace

cudaError_t GB_TUNE_CONFIGURE(int v, int nruns, int max_cap, int *grid, size_t *smem) {
  switch (v) {
    case 1: return configure_v<1>(nruns, max_cap, grid, smem);
    case 2: return configure_v<2>(nruns, max_cap, grid, smem);
    case 3: return configure_v<3>(nruns, max_cap, grid, smem);
    case 4: return configure_v<4>(nruns, max_cap, grid, smem);
    case 5: return configure_v<5>(nruns, max_cap, grid, smem);
    case 6: return configure_v<6>(nruns, max_cap, grid, smem);
    case 7: return configure_v<7>(nruns, max_cap, grid, smem);
  }
  return cudaErrorInvalidValue;
}

cudaError_t GB_TUNE_LAUNCH(int v, int grid, size_t smem, cudaStream_t s, const Tracks &T, const Phys &ph, int nsteps,
                        const int *order, int nruns, int *queue, StepStats *stats, int regrid_only, unsigned wb) {
  switch (v) {
    case 1: return launch_v<1>(grid, smem, s, T, ph, nsteps, order, nruns, queue, stats, regrid_only, wb);
    case 2: return launch_v<2>(grid, smem, s, T, ph, nsteps, order, nruns, queue, stats, regrid_only, wb);
    case 3: return launch_v<3>(grid, smem, s, T, ph, nsteps, order, nruns, queue, stats, regrid_only, wb);
    case 4: return launch_v<4>(grid, smem, s, T, ph, nsteps, order, nruns, queue, stats, regrid_only, wb);
    case 5: return launch_v<5>(grid, smem, s, T, ph, nsteps, order, nruns, queue, stats, regrid_only, wb);
    case 6: return launch_v<6>(grid, smem, s, T, ph, nsteps, order, nruns, queue, stats, regrid_only, wb);
    case 7: return launch_v<7>(grid, smem, s, T, ph, nsteps, order, nruns, queue, stats, regrid_only, wb);
  }
  return cudaErrorInvalidValue;
}

}  // namespace tune
}  // namespace gb
