// Problem modules: what one module .cu file instantiates and registers.
//
// A module (include/gamma_problem.h) is a struct of hooks plus the module set
// it runs with.  GAMMA_PROBLEM_MODULE(name, Hooks, modules, id) at the end of
// its file instantiates the 1D step kernel for it in every launch shape of the
// autotuner (tune.h), without and with the learned cons2prim guess, and adds an entry
// to the library's registry (gamma_api.cu), through which the C ABI configures
// and launches it.  The set-up hooks run on the host (initial_state below).
#pragma once

#include <cuda_runtime.h>

#include "gamma_gpu.h"
#include "gamma_problem.h"
#include "smem_limit.h"
#include "track_step.cuh"
#include "tune.h"

namespace gb {

struct ProblemEntry {
  const char *name;
  int id;       // a fixed id (the built-in GAMMA_PROBLEM_* values), or -1
  int modules;  // gamma_problem::MODULES_*
  bool regrid;  // Hooks::REGRID
  // launch shape v of the step kernel, without or with the learned guess
  cudaError_t (*configure)(int v, bool guess, int nruns, int max_cap, int *grid, size_t *smem);
  // gate: nullptr, or the step kernels' choice (track_step_kernel)
  cudaError_t (*launch)(int v, bool guess, int grid, size_t smem, cudaStream_t s, const Tracks &T, const Phys &ph,
                        int nsteps, const int *order, int nruns, int *queue, StepStats *stats, int regrid_only,
                        int max_cap, const int *gate);
  // Simu::initialise of one run on the host (prim [NQ][cap])
  int (*initial_state)(const Phys &ph, const double *par, int cap, int *ntrack, double *t, double *prim, double *x,
                       double *dx, double *xI, double *dt_loc);
};

// The registry (gamma_api.cu).  Entries register from static initialisers.
int register_problem(ProblemEntry *e);
const ProblemEntry *find_problem(int id);
int problem_id(const char *name);

template <int M>
struct ModuleCfg;
template <>
struct ModuleCfg<gamma_problem::MODULES_CARTESIAN> {
  using type = CfgCart;
};
template <>
struct ModuleCfg<gamma_problem::MODULES_SPHERICAL1D> {
  using type = CfgSph;
};
template <>
struct ModuleCfg<gamma_problem::MODULES_CARTESIAN_REL_CYL> {
  using type = CfgCyl;
};

// Shared memory of one launch: TrackStep::Smem, the regrid bit words (modules
// with a refinement criterion only), then the learned guess's weights.
template <class Hooks>
__host__ __device__ constexpr unsigned module_words_bytes(int max_cap) {
  return Hooks::REGRID ? 4u * 4u * (unsigned)regrid_words(max_cap) : 0u;
}

template <class C, class Hooks, int V, bool GUESS>
struct ModuleKernel {
  static constexpr int BS = tune::kShapes[V].threads;
  static constexpr int CPT = tune::kShapes[V].cells_per_thread;
  static constexpr int MINB = tune::min_blocks(C::MIN_BLOCKS, BS);
  static constexpr auto fn = track_step_kernel<C, Hooks, BS, GUESS, CPT, MINB>;
  static size_t smem(int max_cap) {
    size_t b = sizeof(typename TrackStep<C, Hooks, BS, GUESS, CPT>::Smem) + module_words_bytes<Hooks>(max_cap);
    if (GUESS) b = ((b + 15u) & ~size_t(15)) + sizeof(mlp::InferSmem);
    return b;
  }
  static cudaError_t configure(int nruns, int max_cap, int *grid, size_t *sm) {
    *sm = smem(max_cap);
    cudaError_t e = raise_smem_limit((const void *)fn, *sm);
    if (e != cudaSuccess) return e;
    int dev = 0, nsm = 0, occ = 0;
    if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
    if ((e = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
    if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fn, BS, *sm)) != cudaSuccess) return e;
    if (occ < 1) occ = 1;
    *grid = nruns < nsm * occ ? nruns : nsm * occ;
    return cudaSuccess;
  }
  static cudaError_t launch(int grid, size_t sm, cudaStream_t s, const Tracks &T, const Phys &ph, int nsteps,
                            const int *order, int nruns, int *queue, StepStats *stats, int regrid_only, int max_cap,
                            const int *gate) {
    fn<<<grid, BS, sm, s>>>(T, ph, nsteps, order, nruns, queue, stats, regrid_only,
                            module_words_bytes<Hooks>(max_cap), gate);
    return cudaGetLastError();
  }
};

#define GB_MODULE_SHAPES(X) X(0) X(1) X(2) X(3) X(4) X(5) X(6) X(7)
static_assert(tune::kVariants == 8, "GB_MODULE_SHAPES lists every launch shape");

template <class C, class Hooks>
cudaError_t module_configure(int v, bool guess, int nruns, int max_cap, int *grid, size_t *smem) {
  switch (v) {
#define GB_CASE(k)                                                                       \
  case k:                                                                                \
    return guess ? ModuleKernel<C, Hooks, k, true>::configure(nruns, max_cap, grid, smem) \
                 : ModuleKernel<C, Hooks, k, false>::configure(nruns, max_cap, grid, smem);
    GB_MODULE_SHAPES(GB_CASE)
#undef GB_CASE
  }
  return cudaErrorInvalidValue;
}

template <class C, class Hooks>
cudaError_t module_launch(int v, bool guess, int grid, size_t smem, cudaStream_t s, const Tracks &T, const Phys &ph,
                          int nsteps, const int *order, int nruns, int *queue, StepStats *stats, int regrid_only,
                          int max_cap, const int *gate) {
  switch (v) {
#define GB_CASE(k)                                                                                             \
  case k:                                                                                                      \
    return guess ? ModuleKernel<C, Hooks, k, true>::launch(grid, smem, s, T, ph, nsteps, order, nruns, queue,  \
                                                           stats, regrid_only, max_cap, gate)                  \
                 : ModuleKernel<C, Hooks, k, false>::launch(grid, smem, s, T, ph, nsteps, order, nruns, queue, \
                                                            stats, regrid_only, max_cap, gate);
    GB_MODULE_SHAPES(GB_CASE)
#undef GB_CASE
  }
  return cudaErrorInvalidValue;
}

// Simu::initialise for one run, on the host (src/simu.cpp:24-38 with
// src/Dimensions/1d.cpp:53-81, 217-246, 844-856, 931-951 and
// radiation_sph.cpp:246-260): loadParams, initialGeometry and initialValues of
// the module on the active cells, FluidState's default state (rho = p = 1)
// elsewhere, prepForRun's v2u and interface positions, radiation_initGammas,
// then the first updateGhosts with the module's userBoundaries.
template <class C, class Hooks>
int module_initial_state(const Phys &ph, const double *par, int cap, int *ntrack, double *t, double *prim, double *x,
                         double *dx, double *xI, double *dt_loc) {
  constexpr int NQ = C::NQ;
  const gamma_problem::Setup s = Hooks::load_params(par);
  const int ng = ph.ngst;
  const int n = s.ncell + 2 * ng;
  if (s.ncell < 3 || s.nmax < s.ncell) return GAMMA_ERR_INVALID;
  if (s.nmax + 2 * ng > cap) return GAMMA_ERR_CAPACITY;
  for (int i = 0; i < cap; ++i) {
    for (int q = 0; q < NQ; ++q) prim[(size_t)q * cap + i] = (q == RHO || q == PPP) ? 1. : 0.;
    x[i] = dx[i] = xI[i] = 0.;
    dt_loc[i] = DT_INF;
  }
  const int iL = ng - 1, iR = n - ng;
  const gamma_problem::HookArgs a{par, ph.gamma_ad, s.tini, 0, n, iL, iR};
  for (int i = 0; i < s.ncell; ++i) Hooks::initial_geometry(a, i, s.ncell, &x[ng + i], &dx[ng + i]);
  for (int i = 0; i < s.ncell; ++i) {
    double c[NQ];
    for (int q = 0; q < NQ; ++q) c[q] = (q == RHO || q == PPP) ? 1. : 0.;
    Hooks::initial_values(a, x[ng + i], dx[ng + i], c);
    for (int q = 0; q < NQ; ++q) prim[(size_t)q * cap + ng + i] = c[q];
  }
  // v2u (1d.cpp:931-951)
  for (int i = 0; i < n; ++i) {
    double v = 0.;
    const double vv = prim[(size_t)UU1 * cap + i];
    v += vv * vv;
    v = sqrt(v);
    const double lfac = 1. / sqrt(1. - v * v);
    prim[(size_t)UU1 * cap + i] *= lfac;
  }
  // interfaceGeomFromCellPos (1d.cpp:844-856)
  for (int i = 0; i < n - 1; ++i) xI[i] = i != iL ? x[i] + dx[i] / 2. : x[i + 1] - dx[i + 1] / 2.;
  if (C::SYNCH) {  // radiation_initGammas on every cell
    for (int i = 0; i < n; ++i) {
      const double lfac = gamma_problem::lorentz_factor(prim[(size_t)UU1 * cap + i]);
      const double rho = prim[(size_t)RHO * cap + i];
      const double lim = lfac * pow(rho, 4. / 3.);
      for (int q : {GMX, GMN}) {
        double &g = prim[(size_t)q * cap + i];
        if (g > lim / (lfac * rho) || g <= 0.) g = lim / (lfac * rho);
      }
    }
  }
  // updateGhosts (1d.cpp:217-246), then userBoundaries
  for (int i = 0; i <= iL; ++i) {
    for (int q = 0; q < NQ; ++q) prim[(size_t)q * cap + i] = prim[(size_t)q * cap + iL + 1];
    x[i] = x[iL + 1] - (iL - i + 1) * dx[iL + 1];
    dx[i] = dx[iL + 1];
  }
  for (int i = 0; i <= iL - 1; ++i) xI[i] = xI[iL + 1] - (iL - i + 1) * dx[iL + 1];
  for (int i = iR; i < n; ++i) {
    for (int q = 0; q < NQ; ++q) prim[(size_t)q * cap + i] = prim[(size_t)q * cap + iR - 1];
    x[i] = x[iR - 1] + (i - iR + 1) * dx[iR - 1];
    dx[i] = dx[iR - 1];
  }
  for (int i = iR; i < n - 1; ++i) xI[i] = xI[iR - 1] + (i - iR) * dx[iR - 1];
  for (int i = 0; i < n; ++i) {
    if (i > iL && i < iR) continue;
    double c[NQ];
    for (int q = 0; q < NQ; ++q) c[q] = prim[(size_t)q * cap + i];
    Hooks::user_boundaries(a, i, x[i], c);
    for (int q = 0; q < NQ; ++q) prim[(size_t)q * cap + i] = c[q];
  }
  *ntrack = n;
  *t = s.tini;
  return GAMMA_OK;
}

template <class Hooks, int MODULES>
ProblemEntry make_problem_entry(const char *name, int id) {
  using C = typename ModuleCfg<MODULES>::type;
  return ProblemEntry{name, id, MODULES, Hooks::REGRID, &module_configure<C, Hooks>, &module_launch<C, Hooks>,
                      &module_initial_state<C, Hooks>};
}

}  // namespace gb

// Registers module Hooks (module set MODULES) under NAME.  ID: a fixed id, or -1
// for the next free one (gamma_gpu_problem_id looks modules up by name).
#define GAMMA_PROBLEM_MODULE(NAME, HOOKS, MODULES, ID)                                               \
  namespace {                                                                                        \
  gb::ProblemEntry gb_problem_entry_ = gb::make_problem_entry<HOOKS, MODULES>(NAME, ID);            \
  const int gb_problem_registered_ = gb::register_problem(&gb_problem_entry_);                       \
  }
