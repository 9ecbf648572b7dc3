/*
 * gamma_gpu.h -- C ABI of the B200 moving-mesh relativistic hydro step.
 *
 * The GAMMA reference has no FFI: its "operator API" is the C++ class surface
 * (Grid / Cell / FluidState / Interface) with module bodies picked at link
 * time (Makefile:1-8, 82-92).  This header is the boundary a replacement of that
 * path binds: plain pointers and sizes, status codes, no C++ or torch types.
 * Each entry point names the reference member(s) it stands in for.
 *
 * Data model.  A context holds the physics configuration (the reference's
 * compile-time switches, src/environment.h:46-66) and nruns independent runs.
 * Each run is one 1D track of cells (Grid::Ctot / Grid::Itot of
 * src/Dimensions/1d.cpp) with its own time, time step and cell count.  Run r
 * owns cells [offset[r], offset[r] + capacity[r]) of every per-cell array;
 * the host arrays passed to upload/download use exactly that layout, so each
 * field moves in one copy:
 *   prim    [nq][total]   primitive variables (FluidState::prim slots,
 *                         src/environment.h:33-82; slot 3 is zero in 1D)
 *   x, dx   [total]       cell centre and width (s_cell_geometry x, dx)
 *   dt_loc  [total]       Cell::dt_loc (carried between steps, cell.cpp:97)
 *   xI      [total]       interface i between cells i and i+1 (Interface::x)
 * Cells [0, ngst) and [ntrack-ngst, ntrack) of a run are its ghost cells.
 *
 * Errors: every call returns GAMMA_OK (0) or a negative code;
 * gamma_gpu_strerror gives its text and gamma_gpu_last_error the detail of the
 * last failure on a context.  A context is used by one host thread at a time
 * and runs its work on its own CUDA stream.
 */
#ifndef GAMMA_GPU_H
#define GAMMA_GPU_H

#ifdef __cplusplus
extern "C" {
#endif

#define GAMMA_OK 0
#define GAMMA_ERR_INVALID (-1)     /* bad argument or unsupported module combination */
#define GAMMA_ERR_CUDA (-2)        /* a CUDA call failed; see gamma_gpu_last_error */
#define GAMMA_ERR_CAPACITY (-3)    /* a track does not fit its capacity */
#define GAMMA_ERR_NO_DEVICE (-4)   /* no usable sm_100 device */
#define GAMMA_ERR_IO (-5)          /* a snapshot file could not be opened, written or parsed */
#define GAMMA_ERR_NEG_DT (-30)     /* a CFL candidate was negative: the reference exit(30)s (cell.cpp:70-73) */

enum { GAMMA_GEOM_SPHERICAL1D = 0, GAMMA_GEOM_CARTESIAN = 1 };
enum { GAMMA_HYDRO_REL_SPH = 0, GAMMA_HYDRO_REL_CART = 1, GAMMA_HYDRO_REL_CYL = 2 };
enum { GAMMA_EOS_IDEAL = 0, GAMMA_EOS_SYNGE = 1 };
/* built-in problem modules; others by name through gamma_gpu_problem_id */
enum { GAMMA_PROBLEM_BM1D = 0, GAMMA_PROBLEM_TUBE = 1 };
/* the Timestep module: Grid::evolve of src/Timestep/rk3.cpp (SSP-RK3, three
 * stages) or of src/Timestep/euler.cpp (one forward-Euler Grid::update) */
enum { GAMMA_TS_RK3 = 0, GAMMA_TS_EULER = 1 };

/* Module selection and switches (Makefile GEOMETRY/HYDRO/RADIATION/INITIAL,
 * environment.h GAMMA_, EOS_, CFL_, VI, SHOCK_DETECTION_, LOCAL_SYNCHROTRON_).
 * Supported combinations, each with any problem module built for it:
 *   spherical1D + rel_sph + shock detection + local synchrotron (nq = 10)
 *   cartesian   + rel_cart, no shock detection, no synchrotron   (nq = 6)
 *   cartesian   + rel_cyl (Hydro/rel_cyl.cpp), the same switches  (nq = 6) */
typedef struct {
  int geometry;
  int hydro;
  int eos;
  int nq;
  int shock_detection;
  int local_synchrotron;
  int problem;
  int ngst;
  double gamma_ad;
  double cfl;
  double vi;
  /* 0: GAMMA_ in the wave speeds and the shock detector whatever the EOS, as
   * the reference does (src/Hydro/rel_sph.cpp:331-334, radiation_sph.cpp:37-39);
   * 1: each state's Gamma_eff there too (rel_sph.cpp:37-52), the Synge EOS end
   * to end -- no counterpart in the reference.  No effect with the ideal EOS. */
  int eos_wavespeeds;
  int timestep;  /* GAMMA_TS_*: the Makefile's TIMESTEP module */
} gamma_config_t;

/* Per-run parameters of the Blandford-McKee problem hooks
 * (src/Initial/Tests/BM1D.cpp: calcBM 62-86, userKinematics 188-246,
 * userBoundaries 254-274, checkCellForRegrid 277-319) and the normalised
 * synchrotron constants (src/constants.cpp:12-20).  Ignored by tubes. */
typedef struct {
  double Etot, n_ext, eta, k, Rscale;
  double rhoNorm, pNorm, lNorm, vNorm;
  double dth, target_ar, split_AR, merge_AR;
  double t_bm_until, v_in, v_out;
  double Nalpha, Nmp, Nme;
} gamma_run_params_t;

typedef struct {
  unsigned long long c2p_calls;      /* FluidState::cons2prim calls */
  unsigned long long c2p_iters;      /* Newton iterations over those calls */
  unsigned long long c2p_fallbacks;  /* calls that hit the iteration cap */
  unsigned long long zone_updates;   /* sum over steps of active cells */
  unsigned long long splits, merges; /* regrid actions */
  int c2p_max_iters;
  int status;                        /* 0 or the first failing run's GAMMA_ERR_* */
  float device_ms;                   /* device time of the step launch(es) */
  unsigned long long c2p_guesses;    /* calls started from the learned guess (gamma_gpu_set_guess) */
  unsigned long long c2p_poor;       /* calls whose warm start was poor: the first Newton correction
                                        from the previous pressure above 3% of it */
  unsigned long long learned_steps;  /* steps that ran the step with the learned guess */
} gamma_step_stats_t;

typedef struct gamma_ctx gamma_ctx_t;

/* Allocate device state for nruns tracks of the given capacities (cells,
 * ghosts included: Grid::nde_nax = nmax + 2 ngst, 1d.cpp:60).
 * Replaces Grid::initialise (1d.cpp:53-81). */
int gamma_gpu_create(const gamma_config_t *cfg, int nruns, const int *capacity, gamma_ctx_t **out);

/* offsets[r] of each run in the pooled arrays and the total length. */
int gamma_gpu_layout(const gamma_ctx_t *ctx, long long *offsets, long long *total);

/* Problem parameters, one record per run: the BM1D module's record
 * (gamma_run_params_t), the words of its first fields. */
int gamma_gpu_set_params(gamma_ctx_t *ctx, const gamma_run_params_t *params);

/* ---- Problem modules (the reference's INITIAL files) ------------------------
 * A problem module is a set of user hooks (include/gamma_problem.h) compiled
 * into this library: the built-in "bm1d" (GAMMA_PROBLEM_BM1D), "tube"
 * (GAMMA_PROBLEM_TUBE) and "isen1d", and any named by
 * `make -C gamma_b200/csrc INITIAL=...` (the reference links one with
 * INITIAL = Tests/<name>, Makefile:1).  gamma_config_t.problem holds the id. */

/* The id of the module registered under name, or -1. */
int gamma_gpu_problem_id(const char *name);

/* The module's parameter words of every run: words[r * nwords + k], nwords <=
 * 32 (gamma_problem::PARAM_WORDS; the rest are zero).  Replaces the file-static
 * constants of an Initial file (e.g. src/Initial/Tests/isen1D.cpp:13-24). */
int gamma_gpu_set_params_words(gamma_ctx_t *ctx, const double *words, int nwords);

/* Simu::initialise of one run on the HOST (src/simu.cpp:24-38): the module's
 * loadParams, Grid::initialGeometry and Grid::initialValues, then
 * Grid::prepForRun (1d.cpp:844-856, 931-951), radiation_initGammas and the
 * first updateGhosts with the module's userBoundaries.  Outputs are host
 * arrays of cap cells (prim [nq][cap]); ntrack and t take the run's cell count
 * (ghosts included) and start time.  Needs no GPU.  GAMMA_ERR_INVALID for a
 * module whose set-up runs elsewhere (bm1d and tube are set up by
 * gamma_b200/problems.py), GAMMA_ERR_CAPACITY if nmax + 2 ngst > cap. */
int gamma_gpu_initial_state(const gamma_config_t *cfg, const double *params, int nwords, int cap, int *ntrack,
                            double *t, double *prim, double *x, double *dx, double *xI, double *dt_loc);

/* Host -> device state of every run (mpi_distribute + prepForRun leave this
 * state in the reference, 1d.cpp:956-969, grid.cpp:20-26).  t[r], it[r]:
 * Simu::t and Simu::it.  Pinned host memory makes the copies asynchronous. */
int gamma_gpu_upload(gamma_ctx_t *ctx, const int *ntrack, const double *t, const long long *it,
                     const double *prim, const double *x, const double *dx, const double *dt_loc,
                     const double *xI);

/* Advance every run by nsteps iterations of the Simu::run loop body
 * (src/simu.cpp:79-105: regrid, resetShock, updateGhosts, prepForUpdate,
 * detectShock, collect_dt, Grid::evolve (rk3.cpp:13-95, or euler.cpp:12-19
 * with GAMMA_TS_EULER), injectParticles),
 * each run with its own dt.  With stats == NULL the call only enqueues the
 * work; otherwise it waits and fills stats. */
int gamma_gpu_step(gamma_ctx_t *ctx, int nsteps, gamma_step_stats_t *stats);

/* Grid::regrid alone (1d.cpp:484-557 with the problem's checkCellForRegrid):
 * split / merge every run once, as the first phase of gamma_gpu_step does.
 * A no-op for problems without a refinement criterion (tubes). */
int gamma_gpu_regrid(gamma_ctx_t *ctx, gamma_step_stats_t *stats);

/* Device -> host state (waits for the context's stream).  Any pointer may be
 * NULL.  status[r]: 0 or GAMMA_ERR_NEG_DT for a run stopped by a negative CFL
 * candidate. */
int gamma_gpu_download(gamma_ctx_t *ctx, int *ntrack, double *t, double *dt, long long *it, int *status,
                       double *prim, double *x, double *dx, double *dt_loc, double *xI);

/* FluidState::cons2prim (rel_sph.cpp:213-320 / rel_cart.cpp:125-229) on n
 * independent states, DEVICE pointers, layout [nq][n]; prim holds the previous
 * primitives (pressure warm start) on entry, cons is rewritten by the closing
 * prim2cons as in the reference.  iters (may be NULL): Newton iterations per
 * state.  stream: a cudaStream_t, or NULL for the default stream. */
int gamma_gpu_cons2prim(const gamma_config_t *cfg, double *cons, double *prim, int n, int *iters, void *stream);

/* Per-run scalars in device memory for gamma_gpu_step_tubes_noalloc (the
 * fields a context keeps internally: Grid::ntrack, the run status, Simu::t,
 * Simu::dt and Simu::it). */
typedef struct {
  int ntrack;
  int status;    /* 0 on input; 30 after a negative CFL candidate (the reference's exit code) */
  double t;
  double dt;
  long long it;
} gamma_run_state_t;

/* No counterpart in the reference.  The batched shock-tube step
 * (cartesian + rel_cart configuration only) for callers that cannot allocate
 * device memory -- a solver embedded in a framework that owns every device
 * allocation, a memory-budgeted service, or code that must not synchronise
 * the device the way cudaMalloc/cudaFree can.  The caller passes its own
 * DEVICE arrays in the layout of this header (prim holds the nq-1 stored rows
 * -- slots 0,1,2,4,5 -- of `total` doubles each; offsets/capacity/runs have
 * nruns entries) and the call allocates nothing: the step's workspace lives
 * in one fixed 64 MiB device array inside the library (about 690,000 cells per
 * call), held by every GPU that loads the library until the process exits.
 * A call needing more returns GAMMA_ERR_CAPACITY before anything runs.  The
 * first call on a device looks up that array's address (cudaGetSymbolAddress)
 * and should come before any CUDA graph capture.  All calls on a device share
 * the workspace and it keeps the last call's contents (what must start at
 * zero is cleared on every call), so calls that overlap on the GPU race: issue
 * them one after another.  stream: a cudaStream_t or NULL; stats (host, may be
 * NULL) makes the call wait and report. */
int gamma_gpu_step_tubes_noalloc(const gamma_config_t *cfg, int nruns, long long total,
                                 const long long *offsets, const int *capacity, gamma_run_state_t *runs,
                                 double *prim, double *x, double *dx, double *dt_loc, double *xI,
                                 int nsteps, void *stream, gamma_step_stats_t *stats);

/* ---- Learned cons2prim guess ------------------------------------------------
 * No counterpart in the reference, whose cons2prim always starts its Brent
 * search from the cell's previous pressure (rel_sph.cpp:243-250).  A
 * 3 -> 64 -> 64 -> 2 SiLU network maps a conserved state to a starting
 * pressure; the Newton iteration still runs to the same tolerance, so only the
 * iteration count changes.  Parameters: gamma_mlp_param_count() floats in
 * DEVICE memory.  Inputs per state (x, [n][3] floats): log1p(|S|/D)/8,
 * log10 of the thermal part of tau/D (tau/D - sqrt(1+(S/D)^2) + 1)/10,
 * log10(D)/6.  Outputs (y, [n][2]): (ln(p/D)+14)/10 and ln(lfac)/3. */
typedef struct {
  int epochs;
  int batch;                /* samples per Adam step */
  float lr, lr_final;       /* cosine decay from lr to lr_final over all steps */
  unsigned long long seed;  /* sample order of each epoch */
} gamma_mlp_train_t;

int gamma_mlp_param_count(void);

/* Glorot-uniform weights, zero biases (device pointer). */
int gamma_mlp_init(float *params, unsigned long long seed, void *stream);

/* Training pairs: the first n_states from primitive states prim ([nq][n_states],
 * device, reference slot order), then n_uniform states drawn with
 * ln lfac ~ U(0, ln 1e3), log10 p/rho ~ U(-10, 3), log10 rho ~ U(-6, 6). */
int gamma_mlp_pairs(const gamma_config_t *cfg, const double *prim, long long n_states, long long n_uniform,
                    unsigned long long seed, float *x, float *y, void *stream);

/* Mini-batch Adam on the mean squared error (device x, y, params).
 * loss_per_epoch (host, may be NULL): mean training loss of each epoch.
 * Allocates its optimiser state for the duration of the call and waits. */
int gamma_mlp_train(float *params, const float *x, const float *y, long long n, const gamma_mlp_train_t *tc,
                    float *loss_per_epoch, void *stream);

/* The training kernel's gradient of the mean squared error over n samples
 * (device pointers; grad: gamma_mlp_param_count() floats; loss may be NULL),
 * for checking the hand-written backward pass. */
int gamma_mlp_loss_grad(const float *params, const float *x, const float *y, int n, float *grad, float *loss,
                        void *stream);

/* Network outputs for n inputs: FP32 (tensor_cores = 0) or the BF16
 * tensor-core path used inside the step (tensor_cores = 1). */
int gamma_mlp_forward(const float *params, const float *x, long long n, float *out, int tensor_cores,
                      void *stream);

/* gamma_gpu_cons2prim started from the network's pressure instead of prim's. */
int gamma_gpu_cons2prim_guess(const gamma_config_t *cfg, double *cons, double *prim, int n, int *iters,
                              const float *params, void *stream);

/* Let cons2prim in gamma_gpu_step start from the network's pressure (params:
 * device pointer that stays valid while in use), or NULL for the reference's
 * warm start alone.  With a network set, a step call runs one of two step
 * kernels, chosen on the device from the previous stepping call's statistics:
 * the plain one where poor warm starts (c2p_poor) were at most a quarter of
 * the cons2prim calls, else the one with the guess, in which the cells whose
 * warm start is poor start from the network (c2p_guesses) and the others keep
 * the warm start.  The first call after this one or after an upload takes the
 * guess.  Merges during regrid keep the warm start.  Newton converges to the
 * same tolerance from either start. */
int gamma_gpu_set_guess(gamma_ctx_t *ctx, const float *params);

/* ---- 2D runs (r, theta): NUM_D = 2, spherical, rel_sph, shock detection and
 * local synchrotron (NUM_Q = 10) --------------------------------------------
 * Replaces the 2D Grid members (src/Dimensions/2d.cpp: initialise 59-95,
 * updateGhosts 241-321, computeNeighbors 534-606, regrid 609-832,
 * movDir_ComputeLambda/updateKinematics/computeFluxes 735-839, collect_dt
 * 842-859, update 861-882) with the theta-wedge blast-wave hooks of
 * src/Initial/Tests/BM.cpp, and Grid::evolve (src/Timestep/rk3.cpp:98-194, or
 * src/Timestep/euler.cpp:12-19 with GAMMA_TS_EULER).
 *
 * A run has NJ = ntheta + 2 ngst tracks (ghost tracks included) of cap =
 * nmax + 2 ngst cells.  Per-cell arrays have NJ*cap entries, cell (j, i) at
 * j*cap + i (the reference's Cell::nde_id); per-cell [q] arrays are [NUM_Q][NJ*cap]
 * in the reference's slot order; interface (j, i) is the right edge of cell
 * (j, i).  nbr: [4][NJ*cap], the neighbour list of each cell towards track j-1
 * (first cell id, count) then towards j+1 (Cell::neigh). */
typedef struct {
  int ntheta;   /* active theta tracks (Grid::ncell[F1]) */
  int nmax;     /* active-cell capacity per track (s_par::nmax) */
  int ngst;     /* 2 */
  int nq;       /* 10 */
  int eos;      /* GAMMA_EOS_* */
  double gamma_ad, cfl, vi;
  int eos_wavespeeds;  /* as in gamma_config_t */
  int timestep;        /* as in gamma_config_t */
} gamma_2d_config_t;

/* the problem module's constants (BM.cpp userKinematics, checkCellForRegrid)
 * and the normalised synchrotron constants (constants.cpp:12-20) */
typedef struct {
  double split_DR, merge_DR;            /* lfac >= 2 */
  double split_DR_slow, merge_DR_slow;  /* lfac < 2 */
  double v_out;                         /* outer ghost-interface velocity */
  double it_hold;                       /* v_out -> 0 after it_hold steps once the flow stops */
  double Nalpha, Nmp, Nme;
} gamma_2d_params_t;

typedef struct gamma_2d gamma_2d_t;

/* theta, dtheta: centre and width of each active track (Cell::G.x[F1], dx[F1]) */
int gamma_2d_create(const gamma_2d_config_t *cfg, const double *theta, const double *dtheta, gamma_2d_t **out);
int gamma_2d_layout(const gamma_2d_t *ctx, int *ntracks, int *cap);
int gamma_2d_set_params(gamma_2d_t *ctx, const gamma_2d_params_t *params);

/* Learned cons2prim starting pressure in every cell update of the step (device
 * pointer to gamma_mlp_param_count() floats, trained with gamma_mlp_train), or
 * NULL for the reference's warm start (the cell's previous pressure).  Replaces
 * the starting point of FluidState::cons2prim (src/Hydro/rel_sph.cpp:213-320)
 * called from Cell::update and the RK3 combines (src/Timestep/rk3.cpp); the
 * root and its stopping rule are unchanged.  The pointer must stay valid while
 * steps run. */
int gamma_2d_set_guess(gamma_2d_t *ctx, const float *params);

/* Host -> device state.  grad_mv, grad_f1, nbr and dt_loc may be NULL (a new
 * grid: zero gradients, empty lists, dt_loc = 1e15).  run_ghosts = 1 runs the
 * updateGhosts that precedes Simu::run's loop (simu.cpp:74). */
int gamma_2d_upload(gamma_2d_t *ctx, const int *ntrack, const double *prim, const double *x, const double *dx,
                    const double *dt_loc, const double *xI, const double *grad_mv, const double *grad_f1,
                    const int *nbr, double t, long long it, int run_ghosts);

/* nsteps iterations of the Simu::run loop body (simu.cpp:79-105), one CUDA
 * graph launch each.  With stats == NULL the call only enqueues the work. */
int gamma_2d_step(gamma_2d_t *ctx, int nsteps, gamma_step_stats_t *stats);

/* No counterpart in the reference.  on = 1 (default): each step is one
 * replay of a captured CUDA graph; 0: the step's kernels are launched one by
 * one from the host (the plain form the benchmark compares against). */
int gamma_2d_use_graphs(gamma_2d_t *ctx, int on);

/* Device -> host state; any pointer may be NULL. */
int gamma_2d_download(gamma_2d_t *ctx, int *ntrack, double *t, double *dt, long long *it, int *status,
                      double *prim, double *x, double *dx, double *dt_loc, double *xI, double *grad_mv,
                      double *grad_f1, int *nbr, double *sd, double *pspec, unsigned char *shocked);

/* Diagnostics: the first part of one loop iteration only -- regrid,
 * resetShock, updateGhosts and prepForUpdate (simu.cpp:81-89) -- after which
 * gamma_2d_download and gamma_2d_download_fluxes return the stage-1 state:
 * interface velocity, lambda_L, lambda_R and moving-direction flux (per
 * interface), the theta fluxes flux[0][F1] / flux[1][F1] and this stage's
 * grad_f1 (per cell, [NUM_Q][NJ*cap]).  Continuing with gamma_2d_step after it
 * is not a reference step. */
int gamma_2d_prepare(gamma_2d_t *ctx);
/* The same up to stage `stage` of Grid::evolve (rk3.cpp:99-194): the stages
 * before it complete (updates and combines), then that stage's updateGhosts
 * and prepForUpdate.  stage 1 is gamma_2d_prepare. */
int gamma_2d_prepare_stage(gamma_2d_t *ctx, int stage);
int gamma_2d_download_fluxes(gamma_2d_t *ctx, double *v, double *lL, double *lR, double *flux, double *f1lo,
                             double *f1hi, double *grad_f1_stage);

void *gamma_2d_stream(gamma_2d_t *ctx);
const char *gamma_2d_last_error(const gamma_2d_t *ctx);
void gamma_2d_destroy(gamma_2d_t *ctx);

/* The context's CUDA stream (a cudaStream_t). */
void *gamma_gpu_stream(gamma_ctx_t *ctx);

/* ---- Launch shapes of the step kernel, and their autotuner ------------------
 * No counterpart in the reference (its 1D step is one thread's loop).  A
 * variant fixes the threads that advance one run (the CTA size) and the cells
 * each thread takes per sweep chunk; variant 0 is the default (128 threads,
 * one cell).  Every variant computes every cell the same way, so results are
 * identical; only the speed depends on the batch (track lengths, run count).
 * The step with the learned guess (gamma_gpu_set_guess) has every variant too;
 * the context's variant applies to whichever step runs. */
int gamma_gpu_variant_info(int variant, int *threads, int *cells_per_thread);
int gamma_gpu_set_variant(gamma_ctx_t *ctx, int variant);
int gamma_gpu_get_variant(const gamma_ctx_t *ctx);

/* Times nsteps launches of one step each with every variant on the context's
 * current state (ms[v], may be NULL; with a learned guess set, the step with
 * the guess), restores that state after each, and
 * keeps the fastest (*chosen); another variant must beat variant 0 by 3%.
 * Allocates a copy of the state for the duration of the call. */
int gamma_gpu_autotune(gamma_ctx_t *ctx, int nsteps, float *ms, int *chosen);

/* Step calls are replayed from a captured CUDA graph (the queue and statistics
 * resets and the step kernel), captured again when the step count, launch
 * shape or learned guess changes; on by default.  0 launches them directly.
 * No counterpart in the reference. */
int gamma_gpu_use_graphs(gamma_ctx_t *ctx, int on);

/* ---- Snapshots -------------------------------------------------------------
 * Text: the reference's dump columns and its resume reader, so that files move
 * between this library and the reference both ways.  The reference names a
 * dump <dir>/phys%010d.out after the iteration.  Binary: this library's exact
 * checkpoint (the text is lossy: 16 significant digits in 1D, 7 for most 2D
 * columns). */

/* Grid::printCols of the 1D build (src/IO/text1d.cpp:135-243) from host
 * arrays: one line per active cell with t, nact, i, x, dx, dl, rho, v, p, D,
 * S, tau, the first tracer, slot TR1+1 and, with local synchrotron, gamma_min
 * and gamma_max.  prim holds nq rows of `stride` doubles starting at the run's
 * cell 0 (ghosts included); slot TR1+1 must already hold what the reference
 * stores there first (isShocked, with shock detection).  D, S and tau are
 * prim2cons of each cell: what Cell::S.cons holds at a dump, since cons2prim
 * ends with prim2cons (src/Hydro/rel_sph.cpp:318). */
int gamma_text1d_write(const char *path, const gamma_config_t *cfg, int ntrack, long long it, double t,
                       const double *prim, long long stride, const double *x, const double *dx);

/* Simu::reinitialise of the 1D build (text1d.cpp:67-133, Grid::prepForRun)
 * without the problem hooks: reads a dump into `cap` cells (nmax + 2 ngst) as
 * reloadFromData, mpi_distribute and prepForRun leave them -- the file's cells
 * at ngst.., the rest default states, 3-velocities turned into 4-velocities,
 * interfaces from the cell positions.  prim is [nq][cap], xI [cap].  The
 * ghost cells are the problem's updateGhosts to fill.  `it` comes from the
 * file name, `t` from its first line. */
int gamma_text1d_read(const char *path, const gamma_config_t *cfg, int cap, int *ntrack, long long *it, double *t,
                      double *prim, double *x, double *dx, double *xI);

/* A dump of run `run` as printCols makes it: with shock detection, stores
 * isShocked in slot TR1+1 of every cell of the run on the device (the
 * reference changes the state that way too), then writes <dir>/phys%010d.out
 * from the run's state.  The directory must exist. */
int gamma_gpu_print_cols(gamma_ctx_t *ctx, int run, const char *dir);

/* Exact checkpoint of every run (the state the next step reads: primitives,
 * cells, interfaces, dt_loc, t, it, the shock fields and the run parameters).
 * Loading needs a context created with the same configuration and
 * capacities. */
int gamma_gpu_save(gamma_ctx_t *ctx, const char *path);
int gamma_gpu_load(gamma_ctx_t *ctx, const char *path);

/* Grid::printCols of the 2D build (src/IO/text2d.cpp:145-283) from host
 * arrays in the 2D layout; theta/dtheta of the active tracks.  Slot TR1+1
 * must already hold Sd (the reference's side effect). */
int gamma_text2d_write(const char *path, const gamma_2d_config_t *cfg, const int *ntrack, const double *theta,
                       const double *dtheta, long long it, double t, const double *prim, const double *x,
                       const double *dx);

/* Simu::reinitialise of the 2D build (text2d.cpp:75-143): the file's cells at
 * (j + ngst, i + ngst), default states elsewhere, v2u and
 * interfaceGeomFromCellPos on the active tracks; theta/dtheta (may be NULL)
 * receive each active track's values.  Ghost tracks and cells are the ghost
 * pass's to fill (gamma_2d_upload with run_ghosts). */
int gamma_text2d_read(const char *path, const gamma_2d_config_t *cfg, int *ntrack, long long *it, double *t,
                      double *theta, double *dtheta, double *prim, double *x, double *dx, double *xI);

/* A 2D dump as printCols makes it (Sd stored in slot TR1+1 of every cell on
 * the device first), written to <dir>/phys%010d.out. */
int gamma_2d_print_cols(gamma_2d_t *ctx, const char *dir);

/* Exact 2D checkpoint: state, gradients and neighbour lists (which the ghost
 * cells carry between stages), dt_loc, t, dt, it, shock fields, parameters. */
int gamma_2d_save(gamma_2d_t *ctx, const char *path);
int gamma_2d_load(gamma_2d_t *ctx, const char *path);

const char *gamma_gpu_strerror(int code);
const char *gamma_gpu_last_error(const gamma_ctx_t *ctx);
void gamma_gpu_destroy(gamma_ctx_t *ctx);

#ifdef __cplusplus
}
#endif

#endif
