// gamma_gpu_step_tubes_noalloc: the batched shock-tube step for callers that
// cannot allocate device memory.
//
// Some host programs are not allowed to call cudaMalloc during a run: a solver
// embedded in a framework that owns every device allocation through its own
// pool, code running inside a memory-budgeted service, or a caller that must
// not synchronise the device (cudaMalloc/cudaFree can).  Such a caller still
// owns the state arrays and the run tables; what it cannot provide is the
// step's private workspace (step-start conserved variables, stage-1 fluxes and
// interface velocities, the work-queue counter and the statistics).  This file
// keeps that workspace in one file-scope device array of fixed size, so the
// entry point itself allocates nothing.
//
// Limits and sharing:
//   * the workspace is kNoAllocBytes (64 MiB) per device, held by every GPU that
//     loads the library until the process exits; a call needing more is
//     rejected with GAMMA_ERR_CAPACITY before anything runs;
//   * every call on a device uses the same workspace and it keeps the last
//     call's contents; the queue counter, the statistics and the per-run
//     parameter records are cleared at the start of each call, the rest is
//     written before it is read;
//   * calls that overlap on the GPU (other streams, other host threads) race on
//     the workspace: issue them one after another.
#include "gamma_gpu.h"

#include <cuda_runtime.h>

#include <mutex>

#include "problem_module.cuh"

namespace {

constexpr size_t kNoAllocBytes = size_t(64) << 20;
constexpr int kMaxDevices = 64;
constexpr size_t kParBytes = gamma_problem::PARAM_WORDS * sizeof(double);  // one run's parameter words

// The workspace.  In host code this name is only a stand-in for the device
// symbol: its device address comes from cudaGetSymbolAddress below.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

unsigned char *g_scratch_ptr[kMaxDevices];
std::mutex g_setup_mutex;

// Device address of the workspace on the current device, looked up once per
// device with that device current.
int scratch_address(unsigned char **out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return GAMMA_ERR_NO_DEVICE;
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  if (!g_scratch_ptr[dev]) {
    void *p = nullptr;
    if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) return GAMMA_ERR_CUDA;
    g_scratch_ptr[dev] = static_cast<unsigned char *>(p);
  }
  *out = g_scratch_ptr[dev];
  return GAMMA_OK;
}

size_t align256(size_t b) { return (b + 255) & ~size_t(255); }

__global__ void identity_order(int *order, int n) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) order[i] = i;
}

}  // namespace

#define GAMMA_API __attribute__((visibility("default")))

extern "C" GAMMA_API int gamma_gpu_step_tubes_noalloc(const gamma_config_t *cfg, int nruns, long long total,
                                                      const long long *offsets, const int *capacity,
                                                      gamma_run_state_t *runs, double *prim, double *x,
                                                      double *dx, double *dt_loc, double *xI, int nsteps,
                                                      void *stream, gamma_step_stats_t *stats) {
  static_assert(sizeof(gamma_run_state_t) == sizeof(gb::RunState), "run state record layout");
  if (!cfg || nruns <= 0 || total <= 0 || nsteps < 0) return GAMMA_ERR_INVALID;
  if (!(cfg->geometry == GAMMA_GEOM_CARTESIAN && cfg->hydro == GAMMA_HYDRO_REL_CART && cfg->nq == 6 &&
        !cfg->shock_detection && !cfg->local_synchrotron && cfg->problem == GAMMA_PROBLEM_TUBE &&
        cfg->eos == GAMMA_EOS_IDEAL && cfg->ngst == 2 && cfg->gamma_ad > 1. && cfg->cfl > 0. &&
        (cfg->timestep == GAMMA_TS_RK3 || cfg->timestep == GAMMA_TS_EULER)))
    return GAMMA_ERR_INVALID;
  if (!offsets || !capacity || !runs || !prim || !x || !dx || !dt_loc || !xI) return GAMMA_ERR_INVALID;

  // workspace layout; reject before touching anything if it does not fit.
  // The per-item bounds come first so that no size product below can wrap.
  constexpr int NQS = gb::CfgCart::NQ - 1;
  if ((unsigned long long)total > kNoAllocBytes / sizeof(double) || (size_t)nruns > kNoAllocBytes / kParBytes)
    return GAMMA_ERR_CAPACITY;
  const size_t n = (size_t)total;
  const size_t off_queue = 0;
  const size_t off_stats = align256(off_queue + sizeof(int));
  const size_t off_order = align256(off_stats + sizeof(gb::StepStats));
  const size_t off_par = align256(off_order + (size_t)nruns * sizeof(int));
  const size_t off_u0 = align256(off_par + (size_t)nruns * kParBytes);
  const size_t off_xI0 = align256(off_u0 + NQS * n * sizeof(double));
  const size_t off_fl1 = align256(off_xI0 + n * sizeof(double));
  const size_t off_v1 = align256(off_fl1 + NQS * n * sizeof(double));
  const size_t need = off_v1 + n * sizeof(double);
  if (need > kNoAllocBytes) return GAMMA_ERR_CAPACITY;

  unsigned char *ws = nullptr;
  int rc = scratch_address(&ws);
  if (rc != GAMMA_OK) return rc;
  cudaStream_t s = (cudaStream_t)stream;

  if (cudaMemsetAsync(ws + off_queue, 0, sizeof(int), s) != cudaSuccess) return GAMMA_ERR_CUDA;
  if (cudaMemsetAsync(ws + off_stats, 0, sizeof(gb::StepStats), s) != cudaSuccess) return GAMMA_ERR_CUDA;
  if (cudaMemsetAsync(ws + off_par, 0, (size_t)nruns * kParBytes, s) != cudaSuccess)
    return GAMMA_ERR_CUDA;
  identity_order<<<(nruns + 255) / 256, 256, 0, s>>>(reinterpret_cast<int *>(ws + off_order), nruns);

  gb::Tracks T{};
  T.prim = prim;
  T.x = x;
  T.dx = dx;
  T.dtl = dt_loc;
  T.xI = xI;
  T.u0 = reinterpret_cast<double *>(ws + off_u0);
  T.xI0 = reinterpret_cast<double *>(ws + off_xI0);
  T.fl1 = reinterpret_cast<double *>(ws + off_fl1);
  T.v1 = reinterpret_cast<double *>(ws + off_v1);
  T.N = total;
  T.off = offsets;
  T.cap = capacity;
  T.run = reinterpret_cast<gb::RunState *>(runs);
  T.par = reinterpret_cast<const double *>(ws + off_par);

  gb::Phys ph{};
  ph.gamma_ad = cfg->gamma_ad;
  ph.kgam = cfg->gamma_ad / (cfg->gamma_ad - 1.);
  ph.cfl = cfg->cfl;
  ph.vi = cfg->vi;
  ph.eos = cfg->eos;
  ph.ngst = cfg->ngst;
  ph.eos_ws = cfg->eos_wavespeeds;
  ph.euler = cfg->timestep == GAMMA_TS_EULER;

  // the tube module's step kernel in its default launch shape (the module has
  // no refinement criterion, so the capacity does not size any shared memory)
  const gb::ProblemEntry *tube = gb::find_problem(GAMMA_PROBLEM_TUBE);
  if (!tube) return GAMMA_ERR_INVALID;
  int grid = 0;
  size_t smem = 0;
  if (tube->configure(0, false, nruns, 0, &grid, &smem) != cudaSuccess) return GAMMA_ERR_CUDA;
  auto *qs = reinterpret_cast<int *>(ws + off_queue);
  auto *st = reinterpret_cast<gb::StepStats *>(ws + off_stats);
  if (tube->launch(0, false, grid, smem, s, T, ph, nsteps, reinterpret_cast<const int *>(ws + off_order), nruns, qs,
                   st, 0, 0, nullptr) != cudaSuccess)
    return GAMMA_ERR_CUDA;

  if (stats) {
    gb::StepStats h;
    if (cudaMemcpyAsync(&h, st, sizeof(h), cudaMemcpyDeviceToHost, s) != cudaSuccess) return GAMMA_ERR_CUDA;
    if (cudaStreamSynchronize(s) != cudaSuccess) return GAMMA_ERR_CUDA;
    stats->c2p_calls = h.c2p_calls;
    stats->c2p_iters = h.c2p_iters;
    stats->c2p_fallbacks = h.c2p_fallbacks;
    stats->zone_updates = h.zone_updates;
    stats->splits = h.splits;
    stats->merges = h.merges;
    stats->c2p_max_iters = h.c2p_max_iters;
    stats->c2p_guesses = h.c2p_guesses;
    stats->c2p_poor = h.c2p_poor;
    stats->learned_steps = 0;
    stats->status = h.status == 30 ? GAMMA_ERR_NEG_DT : (h.status ? GAMMA_ERR_INVALID : GAMMA_OK);
    stats->device_ms = 0.f;
  }
  return GAMMA_OK;
}
