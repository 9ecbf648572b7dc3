// C-ABI of the 2D (r, theta) moving-mesh step (include/gamma_gpu.h, gamma_2d_*).
//
// One context holds one run: NJ = ntheta + 2 ngst theta tracks of `cap` cells.
// A step is a fixed sequence of kernels over all tracks (regrid, then per RK3
// stage: ghosts, moving-direction interfaces, per-cell dt and neighbour lists,
// transverse gradients, theta fluxes, dt reduction, interface move, cell
// update), captured once into a CUDA graph and replayed.  The time step lives
// in device memory, so nothing returns to the host between steps.
#include "gamma_gpu.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <string>
#include <vector>

#include <cstring>

#include "io.h"
#include "mlp.cuh"
#include "step2d.cuh"

using namespace gb;
using namespace gb::d2;

namespace {

constexpr int kThreads = 256;
// resident blocks per SM asked of the heavy per-cell passes: their FP64 and
// load latency needs warps more than registers (measured per pass at 512
// tracks with grids of whole waves: 3 for the theta interfaces and the
// transverse gradients, 4 for the r interfaces, the theta gather and the cell
// update)
#ifndef GB2_MINB_MV
#define GB2_MINB_MV 4
#endif
#ifndef GB2_MINB_TG
#define GB2_MINB_TG 3
#endif
#ifndef GB2_MINB_F1
#define GB2_MINB_F1 3
#endif
#ifndef GB2_MINB_GA
#define GB2_MINB_GA 4
#endif
#ifndef GB2_MINB_UP
#define GB2_MINB_UP 4
#endif
// waves of resident blocks in the grid of a per-cell pass
#ifndef GB2_PASS_WAVES
#define GB2_PASS_WAVES 8
#endif
constexpr int kPassWaves = GB2_PASS_WAVES;

struct Stats2 {
  unsigned long long c2p_calls, c2p_iters, c2p_fallbacks, c2p_max_iters, splits, merges, zone_updates;
  unsigned long long c2p_guesses, c2p_poor, learned_steps;
};

// The choice between the cell update and the cell update with the learned
// guess (use_guess, nonzero: the guess), made at the start of every step from
// the previous step's cell updates: their cons2prim calls and those whose
// warm start was poor (mlp::kGuessPolicy).  With no previous step (after
// gamma_2d_set_guess or an upload) the choice stays.
struct Policy2 {
  int use_guess;
  unsigned long long calls, poor;
};

__global__ void k_guess_policy2(Policy2 *pol, Stats2 *S) {
  if (pol->calls) pol->use_guess = (double)pol->poor > mlp::kGuessPolicy * (double)pol->calls ? 1 : 0;
  pol->calls = 0;
  pol->poor = 0;
  if (pol->use_guess) S->learned_steps += 1;
}

// A warp's cons2prim statistics into the launch totals (and, with pol, into
// the learned-guess choice's counts).
__device__ void add_stats(Stats2 *S, unsigned long long calls, unsigned long long iters, unsigned long long fb,
                          unsigned long long mx, unsigned long long guesses, unsigned long long poor,
                          Policy2 *pol) {
  for (int o = 16; o > 0; o >>= 1) {
    calls += __shfl_xor_sync(0xffffffffu, calls, o);
    iters += __shfl_xor_sync(0xffffffffu, iters, o);
    fb += __shfl_xor_sync(0xffffffffu, fb, o);
    guesses += __shfl_xor_sync(0xffffffffu, guesses, o);
    poor += __shfl_xor_sync(0xffffffffu, poor, o);
    const unsigned long long m2 = __shfl_xor_sync(0xffffffffu, mx, o);
    mx = m2 > mx ? m2 : mx;
  }
  if ((threadIdx.x & 31) == 0 && calls) {
    atomicAdd(&S->c2p_calls, calls);
    atomicAdd(&S->c2p_iters, iters);
    if (fb) atomicAdd(&S->c2p_fallbacks, fb);
    if (guesses) atomicAdd(&S->c2p_guesses, guesses);
    if (poor) atomicAdd(&S->c2p_poor, poor);
    atomicMax(&S->c2p_max_iters, mx);
    if (pol) {
      atomicAdd(&pol->calls, calls);
      if (poor) atomicAdd(&pol->poor, poor);
    }
  }
}

// Per active track (one block each, from track j0 on): does any cell act
// against the first active track's current target?  flags[j] = 1 if so.  Run
// once before the first active track is regridded (for that track) and once
// after it (for the others, against its final target).
__global__ void k_regrid_check(Params2 P, Grid2 G, int *flags, int j0) {
  __shared__ int s_any;
  const int j = j0 + blockIdx.x;
  if (threadIdx.x == 0) s_any = 0;
  __syncthreads();
  const Target T = track_target(G, jL_of(G) + 1);
  if (regrid_needed(P, G, j, T, threadIdx.x, blockDim.x)) s_any = 1;
  __syncthreads();
  if (threadIdx.x == 0) flags[j] = s_any;
}

// Regrid of active tracks j0, j0+1, ... (one block each) that have an action:
// warp 0 plans the walk, the block moves the records.  live: the block's track
// is the one the criterion measures (run alone, first).
__global__ void k_regrid(Phys ph, Params2 P, Grid2 G, Stats2 *S, const int *flags, int j0, int live) {
  const int j = j0 + blockIdx.x;
  if (!flags[j]) return;
  __shared__ int s_plan[3];
  const int n0 = G.ntrack[j];
  if (threadIdx.x < 32) {
    const Target T = live ? Target{0., 0., 1} : track_target(G, jL_of(G) + 1);
    const PlanOut R = regrid_plan(ph, P, G, j, live != 0, T);
    if (threadIdx.x == 0) {
      s_plan[0] = R.nnew;
      s_plan[1] = R.nseg;
      s_plan[2] = R.first;
      if (R.splits) atomicAdd(&S->splits, R.splits);
      if (R.merges) atomicAdd(&S->merges, R.merges);
      if (R.c2p[0]) {
        atomicAdd(&S->c2p_calls, R.c2p[0]);
        atomicAdd(&S->c2p_iters, R.c2p[1]);
        if (R.c2p[2]) atomicAdd(&S->c2p_fallbacks, R.c2p[2]);
        atomicMax(&S->c2p_max_iters, R.c2p[3]);
      }
    }
  }
  __syncthreads();
  regrid_execute(G, j, n0, s_plan[0], s_plan[1], s_plan[2]);
}

// updateGhosts in two launches: (1) with `reset`, Cell::resetShock on every
// slot, and the ghost tracks' copies of the edge tracks, flat over the slots;
// (2) the ghost cells of every track (after the ghost tracks are complete).
__global__ void k_ghosts_copy(Grid2 G, int reset) {
  const long long nreset = reset ? G.NC : 0, ncopy = 2LL * G.ngst * G.cap;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < nreset + ncopy;
       t += (long long)gridDim.x * blockDim.x) {
    if (t < nreset) {
      G.sd[t] = -1.;
      G.pspec[t] = 0.;
      G.shocked[t] = 0;
    } else {
      const long long u = t - nreset;
      ghosts_track_slot(G, (int)(u / G.cap), (int)(u % G.cap), reset != 0);
    }
  }
}

__global__ void k_ghost_cells(Grid2 G) { ghosts_cells(G, blockIdx.x, threadIdx.x, blockDim.x); }

// Per-cell passes run over the live cells only: pref[j] = cells of tracks < j
// (rebuilt after every ghost pass, when the track lengths are final for the
// stage), and a fixed grid strides over [0, pref[NJ]).
__global__ void k_prefix(Grid2 G) {
  __shared__ int part[1024];
  const int t = threadIdx.x, nt = blockDim.x;
  const int chunk = (G.NJ + nt - 1) / nt;
  const int j0 = t * chunk, j1 = min(G.NJ, j0 + chunk);
  int sum = 0;
  for (int j = j0; j < j1; ++j) sum += G.ntrack[j];
  part[t] = sum;
  __syncthreads();
  for (int off = 1; off < nt; off <<= 1) {  // inclusive scan
    const int v = t >= off ? part[t - off] : 0;
    __syncthreads();
    part[t] += v;
    __syncthreads();
  }
  int run = part[t] - sum;
  for (int j = j0; j < j1; ++j) {
    G.pref[j] = run;
    run += G.ntrack[j];
  }
  if (t == nt - 1) G.pref[G.NJ] = part[t];
}

// the last track j in [0, NJ-1] with pref[j] <= g (pref: a prefix over tracks)
__device__ __forceinline__ int track_at(const int *pref, int NJ, long long g) {
  int lo = 0, hi = NJ - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (pref[mid] <= g) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// track_at of every 32nd element (live cell, theta interface), after the
// prefix is formed: an element's track is then at most a few steps past its
// group's (one step per track that starts inside the group)
__global__ void k_group_tracks(const int *pref, int NJ, int *grp) {
  const long long n = pref[NJ];
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; 32 * k < n; k += (long long)gridDim.x * blockDim.x)
    grp[k] = track_at(pref, NJ, 32 * k);
}

// track_at(pref, NJ, g) from the group table
__device__ __forceinline__ int track_from(const int *pref, const int *grp, int NJ, long long g) {
  int t = grp[g >> 5];
  while (t < NJ - 1 && pref[t + 1] <= g) ++t;
  return t;
}

// (track, index) of live cell g
__device__ __forceinline__ void cell_at(const Grid2 &G, long long g, int *j, int *i) {
  const int t = track_from(G.pref, G.gtrk, G.NJ, g);
  *j = t;
  *i = (int)(g - G.pref[t]);
}

#define FOR_LIVE_CELLS(G, j, i)                                                                     \
  for (long long g_ = blockIdx.x * (long long)blockDim.x + threadIdx.x, n_ = (G).pref[(G).NJ]; g_ < n_; \
       g_ += (long long)gridDim.x * blockDim.x)                                                     \
    if (int j = 0, i = 0; cell_at((G), g_, &j, &i), true)

__global__ void __launch_bounds__(kThreads, GB2_MINB_MV) k_mv(Phys ph, Params2 P, Grid2 G) {
  const long long it = *G.it;
  FOR_LIVE_CELLS(G, j, i) mv_interface(ph, P, G, j, i, it);
}

__global__ void k_cellmv(Grid2 G) {
  FOR_LIVE_CELLS(G, j, i) cell_mv(G, j, i);
}

// foreign stale contributors: clear, then one thread per track appends
__global__ void k_stale_clear(Grid2 G) {
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < G.NJ; t += gridDim.x * blockDim.x) G.stale_n[t] = 0;
}
__global__ void k_stale(Grid2 G) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j <= G.NJ - 2) stale_append(G, j);
}

__global__ void __launch_bounds__(kThreads, GB2_MINB_TG) k_tgrad(Grid2 G) {
  FOR_LIVE_CELLS(G, j, i) trans_grad(G, j, i);
}

// The theta interfaces of track j (one block per track, j <= NJ-2), numbered
// in cell order: a cell's first interface (if_off) is the upper-list length
// of the cells before it; if_own names the owner of each; if_tot counts them.
__global__ void k_if_scan(Grid2 G) {
  __shared__ int part[kThreads];
  const int j = blockIdx.x, n = G.ntrack[j];
  const int t = threadIdx.x, nt = blockDim.x;
  const int chunk = (n + nt - 1) / nt;
  const int i0 = min(n, t * chunk), i1 = min(n, i0 + chunk);
  const long long o = (long long)j * G.cap;
  int sum = 0;
  for (int i = i0; i < i1; ++i) sum += max(G.nbr[3 * G.NC + o + i], 0);
  part[t] = sum;
  __syncthreads();
  for (int off = 1; off < nt; off <<= 1) {  // inclusive scan
    const int v = t >= off ? part[t - off] : 0;
    __syncthreads();
    part[t] += v;
    __syncthreads();
  }
  const long long IC = if_cap(G), base = (long long)j * IC;
  int run = part[t] - sum;
  for (int i = i0; i < i1; ++i) {
    const int cnt = max(G.nbr[3 * G.NC + o + i], 0);
    G.if_off[o + i] = run;
    for (int k = 0; k < cnt; ++k)
      if (run + k < IC) G.if_own[base + run + k] = i;
    run += cnt;
  }
  if (t == nt - 1) {
    const int tot = part[t];
    if (tot > IC) *G.status = 41;
    G.if_tot[j] = tot > IC ? (int)IC : tot;
  }
}

// if_pref: the interfaces of the tracks before j (track NJ-1 owns none)
__global__ void k_if_pref(Grid2 G) {
  __shared__ int part[1024];
  const int t = threadIdx.x, nt = blockDim.x;
  const int chunk = (G.NJ + nt - 1) / nt;
  const int j0 = t * chunk, j1 = min(G.NJ, j0 + chunk);
  auto tot = [&](int j) { return j <= G.NJ - 2 ? G.if_tot[j] : 0; };
  int sum = 0;
  for (int j = j0; j < j1; ++j) sum += tot(j);
  part[t] = sum;
  __syncthreads();
  for (int off = 1; off < nt; off <<= 1) {
    const int v = t >= off ? part[t - off] : 0;
    __syncthreads();
    part[t] += v;
    __syncthreads();
  }
  int run = part[t] - sum;
  for (int j = j0; j < j1; ++j) {
    G.if_pref[j] = run;
    run += tot(j);
  }
  if (t == nt - 1) G.if_pref[G.NJ] = part[t];
}

// every theta interface, one per thread (f1_if)
__global__ void __launch_bounds__(kThreads, GB2_MINB_F1) k_f1if(Phys ph, Grid2 G) {
  const long long n = G.if_pref[G.NJ];
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n;
       t += (long long)gridDim.x * blockDim.x) {
    const int j = track_from(G.if_pref, G.iftrk, G.NJ, t);
    f1_if(ph, G, j, (int)(t - G.if_pref[j]));
  }
}

__global__ void __launch_bounds__(kThreads, GB2_MINB_GA) k_f1gather(Phys ph, Grid2 G) {
  FOR_LIVE_CELLS(G, j, i) f1_gather(ph, G, j, i);
}

// detectShock and collect_dt: per-block minima, then one block
__global__ void k_dtpart(Grid2 G) {
  __shared__ double red[kThreads / 32];
  double m = DT_INF;
  FOR_LIVE_CELLS(G, j, i) m = fmin(m, collect_cell(G, j, i));
  for (int o = 16; o > 0; o >>= 1) m = fmin(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int k = 1; k < kThreads / 32; ++k) m = fmin(m, red[k]);
    G.red[blockIdx.x] = fmin(red[0], m);
  }
}

__global__ void k_dtfinal(Grid2 G, int nblocks, double cfl) {
  __shared__ double red[kThreads / 32];
  double m = DT_INF;
  for (int k = threadIdx.x; k < nblocks; k += blockDim.x) m = fmin(m, G.red[k]);
  for (int o = 16; o > 0; o >>= 1) m = fmin(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int k = 0; k < kThreads / 32; ++k) m = fmin(m, red[k]);
    *G.dt = cfl * m;
  }
}

__global__ void k_iface(Grid2 G, int stage) {
  FOR_LIVE_CELLS(G, j, i) iface_move(G, j, i, stage);
}

// The learned start of the 2D cell update (BF16 tensor cores, mlp.cuh): the
// network's pressure for the warp's cells whose warm start was poor.  It sees
// |S| = sqrt(S_r^2 + (S_theta / r)^2), the momentum magnitude cons2prim solves
// with.
struct LearnedStart {
  static constexpr bool ON = true;
  const mlp::InferSmem *inf;
  __device__ bool any(bool need) const { return __any_sync(0xffffffffu, need); }
  __device__ double operator()(const double *cons, double r, bool need) const {
    const double s1 = cons[SS1], s2 = cons[SS2] / r;
    return mlp::warp_guess_pressure(*inf, cons[DEN], cons[TAU], sqrt(s1 * s1 + s2 * s2), need);
  }
};

// Grid::update + RK3 combines over the live cells.  With `guess` (device
// parameters of the network), the loop runs warp-uniform so that every lane
// takes part in the tensor-core inference; the weights are staged in shared
// memory once per block.
// With pol (a learned guess set), both variants are launched and the one
// k_guess_policy2 did not choose returns at once.
template <bool GUESS>
__global__ void __launch_bounds__(kThreads, GB2_MINB_UP)
    k_update(Phys ph, Params2 P, Grid2 G, int stage, Stats2 *S, const float *guess, Policy2 *pol) {
  if (pol && ((pol->use_guess != 0) != GUESS)) return;
  // calls, iterations, fallbacks, max, learned starts, poor warm starts
  unsigned long long c2p[6] = {0, 0, 0, 0, 0, 0};
  if (!GUESS) {
    FOR_LIVE_CELLS(G, j, i) update_cell(ph, P, G, j, i, stage, c2p, true, WarmStart{});
  } else {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    mlp::InferSmem &inf = *reinterpret_cast<mlp::InferSmem *>(smem_raw);
    mlp::load_infer_weights(guess, inf);
    __syncthreads();
    const LearnedStart ls{&inf};
    const long long n = G.pref[G.NJ], stride = (long long)gridDim.x * blockDim.x;
    for (long long base = blockIdx.x * (long long)blockDim.x + (threadIdx.x & ~31); base < n; base += stride) {
      const long long g = base + (threadIdx.x & 31);
      int j = 0, i = 0;
      const bool live = g < n;
      if (live) cell_at(G, g, &j, &i);
      update_cell(ph, P, G, j, i, stage, c2p, live, ls);
    }
  }
  add_stats(S, c2p[0], c2p[1], c2p[2], c2p[3], c2p[4], c2p[5], pol);
}

// Grid::printCols' side effect with shock detection (text2d.cpp:147-153):
// slot TR1+1 of every cell of every track takes Sd.
__global__ void k_mark_sd(Grid2 G) {
  for (long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x; g < G.NC; g += (long long)gridDim.x * blockDim.x)
    if ((int)(g % G.cap) < G.ntrack[g / G.cap]) G.prim[(TR1 + 1) * G.NC + g] = G.sd[g];
}

__global__ void k_advance(Grid2 G, Stats2 *S) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  *G.t += *G.dt;
  *G.it += 1;
  unsigned long long z = 0;
  for (int j = jL_of(G) + 1; j <= jR_of(G) - 1; ++j) z += (unsigned long long)(G.ntrack[j] - 2 * G.ngst);
  S->zone_updates += z;
}

}  // namespace

struct gamma_2d {
  gamma_2d_config_t cfg{};
  gamma_2d_params_t par{};
  int NJ = 0, cap = 0;
  long long NC = 0;
  cudaStream_t stream = nullptr;
  cudaGraph_t graph = nullptr;
  bool no_graphs = false;  // gamma_2d_use_graphs(ctx, 0): launch each step's kernels directly
  cudaGraphExec_t exec = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  std::vector<void *> allocs;
  Grid2 G{};
  Stats2 *d_stats = nullptr;
  const float *guess = nullptr;  // learned cons2prim start (device parameters), or none
  int *d_flags = nullptr;  // [NJ] regrid flags
  Policy2 *d_policy = nullptr;  // the learned guess's choice (k_guess_policy2)
  int nsm = 148;
  // grid of each per-cell pass (set_pass_grids)
  struct {
    int mv, cellmv, tgrad, f1if, f1gather, dtpart, iface, update, update_guess, groups, if_groups;
  } grid{};
  std::vector<double> tg;  // host copy of the per-track factors
  std::vector<double> theta, dtheta;  // of the active tracks, as given at creation
  std::string err;
};

namespace {

int fail(gamma_2d *c, cudaError_t e, const char *what) {
  if (c) c->err = std::string(what) + ": " + cudaGetErrorString(e);
  return GAMMA_ERR_CUDA;
}
#define G2_CUDA(ctx, call)                              \
  do {                                                  \
    cudaError_t e_ = (call);                            \
    if (e_ != cudaSuccess) return fail(ctx, e_, #call); \
  } while (0)

Phys phys_of(const gamma_2d_config_t &c) {
  Phys p;
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

Params2 params_of(const gamma_2d_params_t &q) {
  Params2 P;
  P.split_DR = q.split_DR;
  P.merge_DR = q.merge_DR;
  P.split_DR_slow = q.split_DR_slow;
  P.merge_DR_slow = q.merge_DR_slow;
  P.v_out = q.v_out;
  P.it_hold = q.it_hold;
  P.Nalpha = q.Nalpha;
  P.Nmp = q.Nmp;
  P.Nme = q.Nme;
  return P;
}

int blocks_of(long long n) { return (int)((n + kThreads - 1) / kThreads); }

// Grid of a per-cell pass (they stride over the live cells): whole waves of
// the kernel's resident blocks on every SM, so that no pass ends on a part
// wave, and no more blocks than the cell capacity needs.  The cells a thread
// takes change with the grid, the arithmetic of each cell does not.
template <class K>
int pass_blocks(const gamma_2d *c, K kernel, size_t smem, int waves = kPassWaves) {
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kThreads, smem) != cudaSuccess || per_sm < 1)
    per_sm = 1;
  return (int)std::max(1LL, std::min<long long>(blocks_of(c->NC), (long long)c->nsm * per_sm * waves));
}

// entries of the theta interfaces' group table: the interfaces are at most
// if_cap per owning track (status 41 past that)
long long if_groups(const gamma_2d *c) { return ((long long)(c->NJ - 1) * (2LL * c->cap + 64)) / 32 + 2; }

void set_pass_grids(gamma_2d *c) {
  c->grid.mv = pass_blocks(c, k_mv, 0);
  c->grid.cellmv = pass_blocks(c, k_cellmv, 0);
  c->grid.tgrad = pass_blocks(c, k_tgrad, 0);
  c->grid.f1if = pass_blocks(c, k_f1if, 0);
  c->grid.f1gather = pass_blocks(c, k_f1gather, 0);
  // one wave: every block ends in a block reduction, and k_dtfinal reads
  // one partial per block
  c->grid.dtpart = pass_blocks(c, k_dtpart, 0, 1);
  c->grid.iface = pass_blocks(c, k_iface, 0);
  c->grid.update = pass_blocks(c, k_update<false>, 0);
  c->grid.update_guess = pass_blocks(c, k_update<true>, sizeof(mlp::InferSmem));
  c->grid.groups = std::max(1, std::min(blocks_of(c->NC / 32 + 1), c->nsm * 8));
  c->grid.if_groups = std::max(1, std::min(blocks_of(if_groups(c)), c->nsm * 8));
}

int ghost_blocks(const gamma_2d *c, bool reset) {
  const long long n = (reset ? c->NC : 0) + 2LL * c->cfg.ngst * c->cap;
  return (int)std::max(1LL, std::min((n + kThreads - 1) / kThreads, 148LL * 8));
}

// One step's launches on the context's stream.  upto > 0 stops after the
// flux passes of stage `upto` (everything before that stage's collect_dt or
// update): the diagnostics of gamma_2d_prepare_stage.
int enqueue_step_until(gamma_2d *c, int upto) {
  const Phys ph = phys_of(c->cfg);
  const Params2 P = params_of(c->par);
  const Grid2 &G = c->G;
  cudaStream_t s = c->stream;
  if (c->guess) k_guess_policy2<<<1, 1, 0, s>>>(c->d_policy, c->d_stats);
  k_regrid_check<<<1, kThreads, 0, s>>>(P, G, c->d_flags, c->cfg.ngst);
  k_regrid<<<1, kThreads, 0, s>>>(ph, P, G, c->d_stats, c->d_flags, c->cfg.ngst, 1);
  if (c->cfg.ntheta > 1) {
    k_regrid_check<<<c->cfg.ntheta - 1, kThreads, 0, s>>>(P, G, c->d_flags, c->cfg.ngst + 1);
    k_regrid<<<c->cfg.ntheta - 1, kThreads, 0, s>>>(ph, P, G, c->d_stats, c->d_flags, c->cfg.ngst + 1, 0);
  }
  const int nstage = c->cfg.timestep == GAMMA_TS_EULER ? 1 : 3;  // Timestep/euler.cpp or rk3.cpp
  for (int stage = 1; stage <= nstage; ++stage) {
    k_ghosts_copy<<<ghost_blocks(c, stage == 1), kThreads, 0, s>>>(G, stage == 1);
    k_ghost_cells<<<c->NJ, 32, 0, s>>>(G);
    k_prefix<<<1, 1024, 0, s>>>(G);
    k_group_tracks<<<c->grid.groups, kThreads, 0, s>>>(G.pref, G.NJ, G.gtrk);
    k_mv<<<c->grid.mv, kThreads, 0, s>>>(ph, P, G);
    k_cellmv<<<c->grid.cellmv, kThreads, 0, s>>>(G);
    k_stale_clear<<<(c->NJ + 255) / 256, 256, 0, s>>>(G);
    k_stale<<<(c->NJ + 127) / 128, 128, 0, s>>>(G);
    k_tgrad<<<c->grid.tgrad, kThreads, 0, s>>>(G);
    k_if_scan<<<c->NJ - 1, kThreads, 0, s>>>(G);
    k_if_pref<<<1, 1024, 0, s>>>(G);
    k_group_tracks<<<c->grid.if_groups, kThreads, 0, s>>>(G.if_pref, G.NJ, G.iftrk);
    k_f1if<<<c->grid.f1if, kThreads, 0, s>>>(ph, G);
    k_f1gather<<<c->grid.f1gather, kThreads, 0, s>>>(ph, G);
    if (stage == upto) {
      G2_CUDA(c, cudaGetLastError());
      return GAMMA_OK;
    }
    if (stage == 1) {
      k_dtpart<<<c->grid.dtpart, kThreads, 0, s>>>(G);
      k_dtfinal<<<1, kThreads, 0, s>>>(G, c->grid.dtpart, c->cfg.cfl);
    }
    k_iface<<<c->grid.iface, kThreads, 0, s>>>(G, stage);
    Policy2 *pol = c->guess ? c->d_policy : nullptr;
    k_update<false><<<c->grid.update, kThreads, 0, s>>>(ph, P, G, stage, c->d_stats, nullptr, pol);
    if (c->guess)
      k_update<true><<<c->grid.update_guess, kThreads, sizeof(mlp::InferSmem), s>>>(ph, P, G, stage, c->d_stats, c->guess, pol);
  }
  k_advance<<<1, 32, 0, s>>>(G, c->d_stats);
  G2_CUDA(c, cudaGetLastError());
  return GAMMA_OK;
}

int enqueue_step(gamma_2d *c) { return enqueue_step_until(c, 0); }

}  // namespace

#define GAMMA_API __attribute__((visibility("default")))

extern "C" {

GAMMA_API int gamma_2d_create(const gamma_2d_config_t *cfg, const double *theta, const double *dtheta,
                              gamma_2d_t **out) {
  if (!cfg || !out || !theta || !dtheta) return GAMMA_ERR_INVALID;
  *out = nullptr;
  if (cfg->ngst != 2 || cfg->ntheta < 1 || cfg->nmax < 8 || !(cfg->gamma_ad > 1.) || !(cfg->cfl > 0.) ||
      cfg->nq != 10 || (cfg->timestep != GAMMA_TS_RK3 && cfg->timestep != GAMMA_TS_EULER))
    return GAMMA_ERR_INVALID;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return GAMMA_ERR_NO_DEVICE;
  int dev = 0;
  cudaGetDevice(&dev);
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, dev) != cudaSuccess || prop.major != 10) return GAMMA_ERR_NO_DEVICE;

  // neighbour lists hold pooled cell ids as int
  if ((long long)(cfg->ntheta + 2 * cfg->ngst) * (cfg->nmax + 2 * cfg->ngst) >= (1LL << 31)) return GAMMA_ERR_INVALID;
  gamma_2d *c = new gamma_2d();
  c->cfg = *cfg;
  c->theta.assign(theta, theta + cfg->ntheta);
  c->dtheta.assign(dtheta, dtheta + cfg->ntheta);
  const int ng = cfg->ngst;
  c->NJ = cfg->ntheta + 2 * ng;
  c->cap = cfg->nmax + 2 * ng;
  c->NC = (long long)c->NJ * c->cap;
  c->nsm = prop.multiProcessorCount;
  set_pass_grids(c);
  const long long NC = c->NC;
  // per-track angular factors; ghost tracks as updateGhosts shifts them
  // (2d.cpp:259-287: by the first active track's dtheta below, the last's above)
  const int jL = ng - 1, jR = c->NJ - ng;
  c->tg.assign((size_t)c->NJ * TG_WORDS, 0.);
  for (int j = 0; j < c->NJ; ++j) {
    double th, dth;
    if (j <= jL) {
      th = theta[0];
      dth = dtheta[0];
      th -= (jL - j + 1) * dtheta[0];
    } else if (j >= jR) {
      th = theta[cfg->ntheta - 1];
      dth = dtheta[cfg->ntheta - 1];
      th += (j - jR + 1) * dtheta[cfg->ntheta - 1];
    } else {
      th = theta[j - ng];
      dth = dtheta[j - ng];
    }
    fill_track_geo(th, dth, &c->tg[(size_t)j * TG_WORDS]);
  }

  auto bail = [&](cudaError_t e, const char *what) {
    fail(c, e, what);
    gamma_2d_destroy(c);
    return GAMMA_ERR_CUDA;
  };
  cudaError_t e;
  if ((e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking)) != cudaSuccess) return bail(e, "stream");
  if ((e = cudaEventCreate(&c->ev0)) != cudaSuccess) return bail(e, "event");
  if ((e = cudaEventCreate(&c->ev1)) != cudaSuccess) return bail(e, "event");
  auto alloc = [&](size_t bytes, void **p) -> cudaError_t {
    cudaError_t ee = cudaMalloc(p, std::max<size_t>(bytes, 16));
    if (ee == cudaSuccess) {
      c->allocs.push_back(*p);
      ee = cudaMemsetAsync(*p, 0, std::max<size_t>(bytes, 16), c->stream);
    }
    return ee;
  };
  Grid2 &G = c->G;
  G.NJ = c->NJ;
  G.cap = c->cap;
  G.ngst = ng;
  G.NC = NC;
  const size_t d = sizeof(double), q = NQ;
#define G2_ALLOC(ptr, bytes) \
  if ((e = alloc((bytes), (void **)&(ptr))) != cudaSuccess) return bail(e, "cudaMalloc " #ptr)
  double *tg_d;
  G2_ALLOC(G.ntrack, c->NJ * sizeof(int));
  G2_ALLOC(tg_d, c->tg.size() * d);
  G.tg = tg_d;
  G2_ALLOC(G.prim, q * NC * d);
  G2_ALLOC(G.x, NC * d);
  G2_ALLOC(G.dx, NC * d);
  G2_ALLOC(G.dtl, NC * d);
  G2_ALLOC(G.sd, NC * d);
  G2_ALLOC(G.pspec, NC * d);
  G2_ALLOC(G.shocked, NC);
  G2_ALLOC(G.gmv, q * NC * d);
  G2_ALLOC(G.gf1, q * NC * d);
  G2_ALLOC(G.gf1n, q * NC * d);
  G2_ALLOC(G.nbr, 4 * NC * sizeof(int));
  G2_ALLOC(G.cons0, q * NC * d);
  G2_ALLOC(G.dV0, NC * d);
  G2_ALLOC(G.f1lo, q * NC * d);
  G2_ALLOC(G.f1hi, q * NC * d);
  G2_ALLOC(G.xI, NC * d);
  G2_ALLOC(G.xI0, NC * d);
  G2_ALLOC(G.xIm, NC * d);
  G2_ALLOC(G.v, NC * d);
  G2_ALLOC(G.lL, NC * d);
  G2_ALLOC(G.lR, NC * d);
  G2_ALLOC(G.flx, q * NC * d);
  G2_ALLOC(G.stale_n, c->NJ * sizeof(int));
  G2_ALLOC(G.stale_id, (size_t)c->NJ * KMAX_STALE * sizeof(int));
  G2_ALLOC(G.t, d);
  G2_ALLOC(G.dt, d);
  G2_ALLOC(G.it, sizeof(long long));
  G2_ALLOC(G.status, sizeof(int));
  G2_ALLOC(G.red, (size_t)blocks_of(NC) * d);
  G2_ALLOC(G.pref, ((size_t)c->NJ + 1) * sizeof(int));
  G2_ALLOC(G.gtrk, ((size_t)NC / 32 + 2) * sizeof(int));
  const size_t IS = (size_t)c->NJ * (size_t)if_cap(G);
  G2_ALLOC(G.ifs, (size_t)IF_WORDS * IS * d);
  G2_ALLOC(G.if_off, NC * sizeof(int));
  G2_ALLOC(G.if_own, IS * sizeof(int));
  G2_ALLOC(G.if_tot, c->NJ * sizeof(int));
  G2_ALLOC(G.if_pref, ((size_t)c->NJ + 1) * sizeof(int));
  G2_ALLOC(G.iftrk, (size_t)if_groups(c) * sizeof(int));
  G2_ALLOC(G.rprim, q * NC * d);
  G2_ALLOC(G.rgmv, q * NC * d);
  G2_ALLOC(G.rgf1, q * NC * d);
  G2_ALLOC(G.rx, NC * d);
  G2_ALLOC(G.rdx, NC * d);
  G2_ALLOC(G.rdtl, NC * d);
  G2_ALLOC(G.rxI, NC * d);
  G2_ALLOC(G.rnbr, 4 * NC * sizeof(int));
  G2_ALLOC(G.rdV, NC * d);
  G2_ALLOC(G.rseg, 2 * NC * sizeof(int));
  G2_ALLOC(G.rnbr2, 4 * NC * sizeof(int));
  G2_ALLOC(c->d_stats, sizeof(Stats2));
  G2_ALLOC(c->d_flags, (size_t)c->NJ * sizeof(int) + 4 * d + 8);
  G2_ALLOC(c->d_policy, sizeof(Policy2));
#undef G2_ALLOC
  if ((e = cudaMemcpyAsync(tg_d, c->tg.data(), c->tg.size() * d, cudaMemcpyHostToDevice, c->stream)) != cudaSuccess)
    return bail(e, "copy track factors");
  if ((e = cudaStreamSynchronize(c->stream)) != cudaSuccess) return bail(e, "sync");
  *out = c;
  return GAMMA_OK;
}

GAMMA_API int gamma_2d_layout(const gamma_2d_t *ctx, int *ntracks, int *cap) {
  if (!ctx) return GAMMA_ERR_INVALID;
  if (ntracks) *ntracks = ctx->NJ;
  if (cap) *cap = ctx->cap;
  return GAMMA_OK;
}

// the graph holds the launch arguments: capture again on the next step
static void drop_graph(gamma_2d *ctx) {
  if (ctx->exec) {
    cudaGraphExecDestroy(ctx->exec);
    cudaGraphDestroy(ctx->graph);
    ctx->exec = nullptr;
    ctx->graph = nullptr;
  }
}

GAMMA_API int gamma_2d_set_params(gamma_2d_t *ctx, const gamma_2d_params_t *params) {
  if (!ctx || !params) return GAMMA_ERR_INVALID;
  ctx->par = *params;
  drop_graph(ctx);
  return GAMMA_OK;
}

namespace {
// the next step with a learned guess set starts with it (k_guess_policy2)
int reset_policy(gamma_2d *c) {
  const Policy2 p{1, 0ull, 0ull};
  G2_CUDA(c, cudaMemcpyAsync(c->d_policy, &p, sizeof(p), cudaMemcpyHostToDevice, c->stream));
  G2_CUDA(c, cudaStreamSynchronize(c->stream));  // p is a stack buffer
  return GAMMA_OK;
}
}  // namespace

GAMMA_API int gamma_2d_set_guess(gamma_2d_t *ctx, const float *params) {
  if (!ctx) return GAMMA_ERR_INVALID;
  if (params && !ctx->guess) {
    const int rc = reset_policy(ctx);
    if (rc != GAMMA_OK) return rc;
  }
  ctx->guess = params;
  drop_graph(ctx);
  return GAMMA_OK;
}

GAMMA_API int gamma_2d_upload(gamma_2d_t *ctx, const int *ntrack, const double *prim, const double *x,
                              const double *dx, const double *dt_loc, const double *xI, const double *grad_mv,
                              const double *grad_f1, const int *nbr, double t, long long it, int run_ghosts) {
  if (!ctx || !ntrack || !prim || !x || !dx || !xI) return GAMMA_ERR_INVALID;
  gamma_2d *c = ctx;
  for (int j = 0; j < c->NJ; ++j)
    if (ntrack[j] > c->cap || ntrack[j] < 2 * c->cfg.ngst + 3) return GAMMA_ERR_CAPACITY;
  const Grid2 &G = c->G;
  const size_t NC = (size_t)c->NC, d = sizeof(double);
  cudaStream_t s = c->stream;
  G2_CUDA(c, cudaMemcpyAsync(G.ntrack, ntrack, c->NJ * sizeof(int), cudaMemcpyHostToDevice, s));
  G2_CUDA(c, cudaMemcpyAsync(G.prim, prim, NQ * NC * d, cudaMemcpyHostToDevice, s));
  G2_CUDA(c, cudaMemcpyAsync(G.x, x, NC * d, cudaMemcpyHostToDevice, s));
  G2_CUDA(c, cudaMemcpyAsync(G.dx, dx, NC * d, cudaMemcpyHostToDevice, s));
  G2_CUDA(c, cudaMemcpyAsync(G.xI, xI, NC * d, cudaMemcpyHostToDevice, s));
  std::vector<double> inf, neg, zero;
  std::vector<int> nb0;
  if (dt_loc) {
    G2_CUDA(c, cudaMemcpyAsync(G.dtl, dt_loc, NC * d, cudaMemcpyHostToDevice, s));
  } else {
    inf.assign(NC, DT_INF);
    G2_CUDA(c, cudaMemcpyAsync(G.dtl, inf.data(), NC * d, cudaMemcpyHostToDevice, s));
  }
  if (grad_mv) G2_CUDA(c, cudaMemcpyAsync(G.gmv, grad_mv, NQ * NC * d, cudaMemcpyHostToDevice, s));
  else G2_CUDA(c, cudaMemsetAsync(G.gmv, 0, NQ * NC * d, s));
  if (grad_f1) G2_CUDA(c, cudaMemcpyAsync(G.gf1, grad_f1, NQ * NC * d, cudaMemcpyHostToDevice, s));
  else G2_CUDA(c, cudaMemsetAsync(G.gf1, 0, NQ * NC * d, s));
  if (nbr) {
    G2_CUDA(c, cudaMemcpyAsync(G.nbr, nbr, 4 * NC * sizeof(int), cudaMemcpyHostToDevice, s));
  } else {  // no neighbours yet (a Cell's lists start empty)
    nb0.assign(4 * NC, 0);
    for (size_t k = 0; k < NC; ++k) nb0[k] = nb0[2 * NC + k] = -1;
    G2_CUDA(c, cudaMemcpyAsync(G.nbr, nb0.data(), 4 * NC * sizeof(int), cudaMemcpyHostToDevice, s));
  }
  neg.assign(NC, -1.);  // Cell::Cell: Sd = -1, pspec = 0, isShocked = false
  G2_CUDA(c, cudaMemcpyAsync(G.sd, neg.data(), NC * d, cudaMemcpyHostToDevice, s));
  G2_CUDA(c, cudaMemsetAsync(G.pspec, 0, NC * d, s));
  G2_CUDA(c, cudaMemsetAsync(G.shocked, 0, NC, s));
  G2_CUDA(c, cudaMemcpyAsync(G.t, &t, d, cudaMemcpyHostToDevice, s));
  G2_CUDA(c, cudaMemcpyAsync(G.it, &it, sizeof(long long), cudaMemcpyHostToDevice, s));
  G2_CUDA(c, cudaMemsetAsync(G.dt, 0, d, s));
  G2_CUDA(c, cudaMemsetAsync(G.status, 0, sizeof(int), s));
  if (run_ghosts) {  // the updateGhosts before Simu::run's loop (simu.cpp:74)
    k_ghosts_copy<<<ghost_blocks(c, false), kThreads, 0, s>>>(G, 0);
    k_ghost_cells<<<c->NJ, 32, 0, s>>>(G);
    G2_CUDA(c, cudaGetLastError());
  }
  G2_CUDA(c, cudaStreamSynchronize(s));  // host staging vectors go out of scope
  return reset_policy(c);  // a new state: no step has measured its warm starts
}

GAMMA_API int gamma_2d_use_graphs(gamma_2d_t *ctx, int on) {
  if (!ctx) return GAMMA_ERR_INVALID;
  ctx->no_graphs = on == 0;
  return GAMMA_OK;
}

GAMMA_API int gamma_2d_step(gamma_2d_t *ctx, int nsteps, gamma_step_stats_t *stats) {
  if (!ctx || nsteps < 0) return GAMMA_ERR_INVALID;
  gamma_2d *c = ctx;
  G2_CUDA(c, cudaMemsetAsync(c->d_stats, 0, sizeof(Stats2), c->stream));
  if (c->no_graphs) {  // every launch of every step from the host
    G2_CUDA(c, cudaEventRecord(c->ev0, c->stream));
    for (int k = 0; k < nsteps; ++k) {
      const int rc = enqueue_step(c);
      if (rc != GAMMA_OK) return rc;
    }
  } else if (!c->exec && nsteps > 0) {
    G2_CUDA(c, cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
    const int rc = enqueue_step(c);
    cudaGraph_t g = nullptr;
    const cudaError_t e = cudaStreamEndCapture(c->stream, &g);
    if (rc != GAMMA_OK) return rc;
    if (e != cudaSuccess) return fail(c, e, "cudaStreamEndCapture");
    c->graph = g;
    G2_CUDA(c, cudaGraphInstantiate(&c->exec, c->graph, 0));
  }
  if (!c->no_graphs) {
    G2_CUDA(c, cudaEventRecord(c->ev0, c->stream));
    for (int k = 0; k < nsteps; ++k) G2_CUDA(c, cudaGraphLaunch(c->exec, c->stream));
  }
  G2_CUDA(c, cudaEventRecord(c->ev1, c->stream));
  if (stats) {
    Stats2 h;
    int status = 0;
    G2_CUDA(c, cudaMemcpyAsync(&h, c->d_stats, sizeof(h), cudaMemcpyDeviceToHost, c->stream));
    G2_CUDA(c, cudaMemcpyAsync(&status, c->G.status, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    G2_CUDA(c, cudaStreamSynchronize(c->stream));
    float ms = 0.f;
    G2_CUDA(c, cudaEventElapsedTime(&ms, c->ev0, c->ev1));
    stats->c2p_calls = h.c2p_calls;
    stats->c2p_iters = h.c2p_iters;
    stats->c2p_fallbacks = h.c2p_fallbacks;
    stats->zone_updates = h.zone_updates;
    stats->splits = h.splits;
    stats->merges = h.merges;
    stats->c2p_max_iters = (int)h.c2p_max_iters;
    stats->status = status == 30 ? GAMMA_ERR_NEG_DT : (status ? GAMMA_ERR_INVALID : GAMMA_OK);
    stats->device_ms = ms;
    stats->c2p_guesses = h.c2p_guesses;
    stats->c2p_poor = h.c2p_poor;
    stats->learned_steps = h.learned_steps;
  }
  return GAMMA_OK;
}

GAMMA_API int gamma_2d_download(gamma_2d_t *ctx, int *ntrack, double *t, double *dt, long long *it, int *status,
                                double *prim, double *x, double *dx, double *dt_loc, double *xI, double *grad_mv,
                                double *grad_f1, int *nbr, double *sd, double *pspec, unsigned char *shocked) {
  if (!ctx) return GAMMA_ERR_INVALID;
  gamma_2d *c = ctx;
  const Grid2 &G = c->G;
  const size_t NC = (size_t)c->NC, d = sizeof(double);
  cudaStream_t s = c->stream;
  int st = 0;
  if (ntrack) G2_CUDA(c, cudaMemcpyAsync(ntrack, G.ntrack, c->NJ * sizeof(int), cudaMemcpyDeviceToHost, s));
  if (t) G2_CUDA(c, cudaMemcpyAsync(t, G.t, d, cudaMemcpyDeviceToHost, s));
  if (dt) G2_CUDA(c, cudaMemcpyAsync(dt, G.dt, d, cudaMemcpyDeviceToHost, s));
  if (it) G2_CUDA(c, cudaMemcpyAsync(it, G.it, sizeof(long long), cudaMemcpyDeviceToHost, s));
  G2_CUDA(c, cudaMemcpyAsync(&st, G.status, sizeof(int), cudaMemcpyDeviceToHost, s));
  if (prim) G2_CUDA(c, cudaMemcpyAsync(prim, G.prim, NQ * NC * d, cudaMemcpyDeviceToHost, s));
  if (x) G2_CUDA(c, cudaMemcpyAsync(x, G.x, NC * d, cudaMemcpyDeviceToHost, s));
  if (dx) G2_CUDA(c, cudaMemcpyAsync(dx, G.dx, NC * d, cudaMemcpyDeviceToHost, s));
  if (dt_loc) G2_CUDA(c, cudaMemcpyAsync(dt_loc, G.dtl, NC * d, cudaMemcpyDeviceToHost, s));
  if (xI) G2_CUDA(c, cudaMemcpyAsync(xI, G.xI, NC * d, cudaMemcpyDeviceToHost, s));
  if (grad_mv) G2_CUDA(c, cudaMemcpyAsync(grad_mv, G.gmv, NQ * NC * d, cudaMemcpyDeviceToHost, s));
  if (grad_f1) G2_CUDA(c, cudaMemcpyAsync(grad_f1, G.gf1, NQ * NC * d, cudaMemcpyDeviceToHost, s));
  if (nbr) G2_CUDA(c, cudaMemcpyAsync(nbr, G.nbr, 4 * NC * sizeof(int), cudaMemcpyDeviceToHost, s));
  if (sd) G2_CUDA(c, cudaMemcpyAsync(sd, G.sd, NC * d, cudaMemcpyDeviceToHost, s));
  if (pspec) G2_CUDA(c, cudaMemcpyAsync(pspec, G.pspec, NC * d, cudaMemcpyDeviceToHost, s));
  if (shocked) G2_CUDA(c, cudaMemcpyAsync(shocked, G.shocked, NC, cudaMemcpyDeviceToHost, s));
  G2_CUDA(c, cudaStreamSynchronize(s));
  if (status) *status = st == 30 ? GAMMA_ERR_NEG_DT : (st ? GAMMA_ERR_INVALID : GAMMA_OK);
  return GAMMA_OK;
}

GAMMA_API int gamma_2d_prepare(gamma_2d_t *ctx) { return gamma_2d_prepare_stage(ctx, 1); }

GAMMA_API int gamma_2d_prepare_stage(gamma_2d_t *ctx, int stage) {
  if (!ctx || stage < 1 || stage > (ctx->cfg.timestep == GAMMA_TS_EULER ? 1 : 3)) return GAMMA_ERR_INVALID;
  const int rc = enqueue_step_until(ctx, stage);
  if (rc != GAMMA_OK) return rc;
  G2_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return GAMMA_OK;
}

GAMMA_API int gamma_2d_download_fluxes(gamma_2d_t *ctx, double *v, double *lL, double *lR, double *flux,
                                       double *f1lo, double *f1hi, double *grad_f1_stage) {
  if (!ctx) return GAMMA_ERR_INVALID;
  gamma_2d *c = ctx;
  const Grid2 &G = c->G;
  const size_t NC = (size_t)c->NC, d = sizeof(double);
  cudaStream_t s = c->stream;
  if (v) G2_CUDA(c, cudaMemcpyAsync(v, G.v, NC * d, cudaMemcpyDeviceToHost, s));
  if (lL) G2_CUDA(c, cudaMemcpyAsync(lL, G.lL, NC * d, cudaMemcpyDeviceToHost, s));
  if (lR) G2_CUDA(c, cudaMemcpyAsync(lR, G.lR, NC * d, cudaMemcpyDeviceToHost, s));
  if (flux) G2_CUDA(c, cudaMemcpyAsync(flux, G.flx, NQ * NC * d, cudaMemcpyDeviceToHost, s));
  if (f1lo) G2_CUDA(c, cudaMemcpyAsync(f1lo, G.f1lo, NQ * NC * d, cudaMemcpyDeviceToHost, s));
  if (f1hi) G2_CUDA(c, cudaMemcpyAsync(f1hi, G.f1hi, NQ * NC * d, cudaMemcpyDeviceToHost, s));
  if (grad_f1_stage) G2_CUDA(c, cudaMemcpyAsync(grad_f1_stage, G.gf1n, NQ * NC * d, cudaMemcpyDeviceToHost, s));
  G2_CUDA(c, cudaStreamSynchronize(s));
  return GAMMA_OK;
}

GAMMA_API void *gamma_2d_stream(gamma_2d_t *ctx) { return ctx ? (void *)ctx->stream : nullptr; }

GAMMA_API const char *gamma_2d_last_error(const gamma_2d_t *ctx) { return ctx ? ctx->err.c_str() : ""; }

GAMMA_API int gamma_2d_print_cols(gamma_2d_t *ctx, const char *dir) {
  if (!ctx) return GAMMA_ERR_INVALID;
  gamma_2d *c = ctx;
  k_mark_sd<<<ghost_blocks(c, true), kThreads, 0, c->stream>>>(c->G);
  G2_CUDA(c, cudaGetLastError());
  const size_t NC = (size_t)c->NC;
  std::vector<int> nt(c->NJ);
  std::vector<double> prim(NQ * NC), x(NC), dx(NC);
  double t = 0.;
  long long it = 0;
  int rc = gamma_2d_download(c, nt.data(), &t, nullptr, &it, nullptr, prim.data(), x.data(), dx.data(), nullptr,
                             nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr);
  if (rc != GAMMA_OK) return rc;
  const std::string path = gb::io::phys_name(dir, it);
  return gb::io::write_text2d(path.c_str(), c->cfg, c->NJ, c->cap, nt.data(), c->theta.data(), c->dtheta.data(), it,
                              t, prim.data(), x.data(), dx.data());
}

// Checkpoint: configuration, tracks, parameters, then every array that carries
// state from one step to the next -- including the gradients and the
// neighbour lists that the ghost cells keep from earlier stages.
GAMMA_API int gamma_2d_save(gamma_2d_t *ctx, const char *path) {
  if (!ctx || !path) return GAMMA_ERR_INVALID;
  gamma_2d *c = ctx;
  const size_t NC = (size_t)c->NC, d = sizeof(double);
  std::vector<int> nt(c->NJ), nbr(4 * NC);
  std::vector<double> prim(NQ * NC), x(NC), dx(NC), dtl(NC), xI(NC), gmv(NQ * NC), gf1(NQ * NC), sd(NC), ps(NC);
  std::vector<unsigned char> sh(NC);
  double sc[2] = {0., 0.};  // t, dt
  long long it = 0;
  int rc = gamma_2d_download(c, nt.data(), &sc[0], &sc[1], &it, nullptr, prim.data(), x.data(), dx.data(),
                             dtl.data(), xI.data(), gmv.data(), gf1.data(), nbr.data(), sd.data(), ps.data(),
                             sh.data());
  if (rc != GAMMA_OK) return rc;
  gb::io::CkptOut out(path);
  if (!out.ok()) return GAMMA_ERR_IO;
  const uint32_t kind = gb::io::kCkpt2D;
  out.block("kind", &kind, sizeof(kind));
  out.block("config", &c->cfg, sizeof(c->cfg));
  out.block("theta", c->theta.data(), c->theta.size() * d);
  out.block("dtheta", c->dtheta.data(), c->dtheta.size() * d);
  out.block("params", &c->par, sizeof(c->par));
  out.block("t_dt", sc, sizeof(sc));
  out.block("it", &it, sizeof(it));
  out.block("ntrack", nt.data(), nt.size() * sizeof(int));
  out.block("prim", prim.data(), prim.size() * d);
  out.block("x", x.data(), NC * d);
  out.block("dx", dx.data(), NC * d);
  out.block("dt_loc", dtl.data(), NC * d);
  out.block("xI", xI.data(), NC * d);
  out.block("grad_mv", gmv.data(), gmv.size() * d);
  out.block("grad_f1", gf1.data(), gf1.size() * d);
  out.block("nbr", nbr.data(), nbr.size() * sizeof(int));
  out.block("sd", sd.data(), NC * d);
  out.block("pspec", ps.data(), NC * d);
  out.block("shocked", sh.data(), NC);
  return out.close();
}

GAMMA_API int gamma_2d_load(gamma_2d_t *ctx, const char *path) {
  if (!ctx || !path) return GAMMA_ERR_INVALID;
  gamma_2d *c = ctx;
  const size_t NC = (size_t)c->NC, d = sizeof(double);
  gb::io::CkptIn in(path);
  if (!in.ok()) return GAMMA_ERR_IO;
  uint32_t kind = 0;
  gamma_2d_config_t cfg;
  if (!in.block("kind", &kind, sizeof(kind)) || kind != gb::io::kCkpt2D) return GAMMA_ERR_IO;
  if (!in.block("config", &cfg, sizeof(cfg)) || !gb::io::same_config(cfg, c->cfg))
    return GAMMA_ERR_INVALID;
  std::vector<double> th(c->theta.size()), dth(c->dtheta.size());
  if (!in.block("theta", th.data(), th.size() * d) || !in.block("dtheta", dth.data(), dth.size() * d) ||
      th != c->theta || dth != c->dtheta)
    return GAMMA_ERR_INVALID;
  gamma_2d_params_t par;
  double sc[2];
  long long it = 0;
  std::vector<int> nt(c->NJ), nbr(4 * NC);
  std::vector<double> prim(NQ * NC), x(NC), dx(NC), dtl(NC), xI(NC), gmv(NQ * NC), gf1(NQ * NC), sd(NC), ps(NC);
  std::vector<unsigned char> sh(NC);
  const bool ok = in.block("params", &par, sizeof(par)) && in.block("t_dt", sc, sizeof(sc)) &&
                  in.block("it", &it, sizeof(it)) && in.block("ntrack", nt.data(), nt.size() * sizeof(int)) &&
                  in.block("prim", prim.data(), prim.size() * d) && in.block("x", x.data(), NC * d) &&
                  in.block("dx", dx.data(), NC * d) && in.block("dt_loc", dtl.data(), NC * d) &&
                  in.block("xI", xI.data(), NC * d) && in.block("grad_mv", gmv.data(), gmv.size() * d) &&
                  in.block("grad_f1", gf1.data(), gf1.size() * d) &&
                  in.block("nbr", nbr.data(), nbr.size() * sizeof(int)) && in.block("sd", sd.data(), NC * d) &&
                  in.block("pspec", ps.data(), NC * d) && in.block("shocked", sh.data(), NC);
  if (!ok) return GAMMA_ERR_IO;
  int rc = gamma_2d_set_params(c, &par);
  if (rc == GAMMA_OK)
    rc = gamma_2d_upload(c, nt.data(), prim.data(), x.data(), dx.data(), dtl.data(), xI.data(), gmv.data(),
                         gf1.data(), nbr.data(), sc[0], it, 0);
  if (rc != GAMMA_OK) return rc;
  const Grid2 &G = c->G;
  G2_CUDA(c, cudaMemcpyAsync(G.sd, sd.data(), NC * d, cudaMemcpyHostToDevice, c->stream));
  G2_CUDA(c, cudaMemcpyAsync(G.pspec, ps.data(), NC * d, cudaMemcpyHostToDevice, c->stream));
  G2_CUDA(c, cudaMemcpyAsync(G.shocked, sh.data(), NC, cudaMemcpyHostToDevice, c->stream));
  G2_CUDA(c, cudaMemcpyAsync(G.dt, &sc[1], d, cudaMemcpyHostToDevice, c->stream));
  G2_CUDA(c, cudaStreamSynchronize(c->stream));
  return GAMMA_OK;
}

GAMMA_API void gamma_2d_destroy(gamma_2d_t *ctx) {
  if (!ctx) return;
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  if (ctx->exec) cudaGraphExecDestroy(ctx->exec);
  if (ctx->graph) cudaGraphDestroy(ctx->graph);
  for (void *p : ctx->allocs) cudaFree(p);
  if (ctx->ev0) cudaEventDestroy(ctx->ev0);
  if (ctx->ev1) cudaEventDestroy(ctx->ev1);
  if (ctx->stream) cudaStreamDestroy(ctx->stream);
  delete ctx;
}

}  // extern "C"
