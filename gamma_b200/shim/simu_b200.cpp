// The reference's Simu (src/simu.cpp) with its time loop on the B200 path.
//
// A GAMMA build swaps src/simu.cpp for this file and links
// gamma_b200/lib/libgamma_b200.so; every other source, the problem's Initial
// file included, stays as it is.  Simu::initialise is the reference's.
// Simu::run hands the grid that initialise built to a GPU context and runs the
// loop body of src/simu.cpp:46-76 as gamma_gpu_step calls: regrid, resetShock,
// updateGhosts, prepForUpdate, detectShock, collect_dt, Grid::evolve, t += dt,
// it++ and radiation_injectParticles all happen on the device; the output
// hooks (dataDump, runInfo, evalEnd) run on the host after each step, with the
// device state mirrored into Ctot / Itot first so that they read what the
// reference's would.
//
// The problem's hooks run on the device as the library's problem module of
// the same name (include/gamma_problem.h).  The Initial file, or a glue file
// beside it, gives the module and its parameter words by defining
//     extern "C" const char *gamma_shim_problem(double *words, int *nwords);
// (words has room for 32).
//
// Environment: GAMMA_SHIM_SYNC_EVERY=n mirrors the device state into the host
// grid every n steps only (default 1: every step, as the hooks expect);
// GAMMA_SHIM_MAX_STEPS=n stops after n steps (0: only evalEnd stops).

// the reference's headers, in src/simu.cpp's order (mpisetup.h needs Cell)
#include "simu.h"
#include "mpisetup.h"
#include "environment.h"
#include "constants.h"

#include <cstdio>
#include <cstdlib>
#include <stdexcept>
#include <string>
#include <vector>

#include "gamma_gpu.h"

extern "C" const char *gamma_shim_problem(double *words, int *nwords);

Simu::Simu() {
  stop = false;
  t = 0;
  it = 0;
}

Simu::~Simu() {}

// src/simu.cpp:24-38
void Simu::initialise() {
  loadParams(&par);
  t = par.tini;
  grid.initialise(par);
  grid.initialGeometry();
  grid.initialValues();
  mpi_distribute(&grid);
  grid.prepForRun();
#if LOCAL_SYNCHROTRON_ == ENABLED_
  grid.apply(&Cell::radiation_initGammas);
#endif
}

namespace {

struct HostTrack {  // Ctot / Itot in the C ABI's layout (one run)
  int cap = 0;
  std::vector<double> prim, x, dx, dtl, xI;
  void resize(int c) {
    cap = c;
    prim.assign((size_t)NUM_Q * c, 0.);
    x.assign(c, 0.);
    dx.assign(c, 0.);
    dtl.assign(c, 1.e15);
    xI.assign(c, 0.);
  }
};

void pack(Grid &g, HostTrack &h) {
  for (int i = 0; i < g.ntrack; ++i) {
    for (int q = 0; q < NUM_Q; ++q) h.prim[(size_t)q * h.cap + i] = g.Ctot[i].S.prim[q];
    h.x[i] = g.Ctot[i].G.x[MV];
    h.dx[i] = g.Ctot[i].G.dx[MV];
    h.dtl[i] = g.Ctot[i].dt_loc;
    if (i < g.ntrack - 1) h.xI[i] = g.Itot[i].x[MV];
  }
}

// The device state back into the host grid: cell states, geometry (with the
// derived quantities the geometry module computes), interfaces, track sizes.
void unpack(const HostTrack &h, int ntrack, Grid &g) {
  g.ntrack = ntrack;
  g.nact = ntrack - 2 * g.ngst;
  g.iRbnd = ntrack - g.ngst;
  for (int i = 0; i < ntrack; ++i) {
    Cell &c = g.Ctot[i];
    for (int q = 0; q < NUM_Q; ++q) c.S.prim[q] = h.prim[(size_t)q * h.cap + i];
    c.G.x[MV] = h.x[i];
    c.G.dx[MV] = h.dx[i];
    c.dt_loc = h.dtl[i];
    c.computeAllGeom();
    c.S.prim2cons(c.G.cen[MV]);
    if (i < ntrack - 1) {
      g.Itot[i].x[MV] = h.xI[i];
      g.Itot[i].computedA();
    }
  }
}

long env_long(const char *name, long dflt) {
  const char *v = std::getenv(name);
  return v && *v ? std::strtol(v, nullptr, 10) : dflt;
}

void check(int rc, const char *what) {
  if (rc != GAMMA_OK) throw std::runtime_error(std::string(what) + ": " + gamma_gpu_strerror(rc));
}

}  // namespace

// src/simu.cpp:41-78 on the device
void Simu::run() {
  grid.updateGhosts(it, t);
  grid.printCols(it, t);

  double words[32] = {0.};
  int nwords = 0;
  const char *module = gamma_shim_problem(words, &nwords);
  gamma_config_t cfg{};
#if SHOCK_DETECTION_ == ENABLED_ && LOCAL_SYNCHROTRON_ == ENABLED_ && NUM_Q == 10
  cfg.geometry = GAMMA_GEOM_SPHERICAL1D;  // GEOMETRY = spherical1D, HYDRO = rel_sph, RADIATION = radiation_sph
  cfg.hydro = GAMMA_HYDRO_REL_SPH;
  cfg.shock_detection = 1;
  cfg.local_synchrotron = 1;
#else
  cfg.geometry = GAMMA_GEOM_CARTESIAN;  // GEOMETRY = cartesian, HYDRO = rel_cart
  cfg.hydro = GAMMA_HYDRO_REL_CART;
#endif
  cfg.eos = EOS_ == SYNGE_EOS_ ? GAMMA_EOS_SYNGE : GAMMA_EOS_IDEAL;
  cfg.nq = NUM_Q;
  cfg.problem = gamma_gpu_problem_id(module);
  if (cfg.problem < 0) throw std::runtime_error(std::string("no problem module ") + module + " in libgamma_b200");
  cfg.ngst = grid.ngst;
  cfg.gamma_ad = GAMMA_;
  cfg.cfl = CFL_;
  cfg.vi = VI;
  cfg.timestep = GAMMA_TS_RK3;

  int cap = grid.nde_nax[MV];
  gamma_ctx_t *ctx = nullptr;
  check(gamma_gpu_create(&cfg, 1, &cap, &ctx), "gamma_gpu_create");
  check(gamma_gpu_set_params_words(ctx, words, nwords), "gamma_gpu_set_params_words");
  HostTrack h;
  h.resize(cap);
  pack(grid, h);
  long long itl = it;
  check(gamma_gpu_upload(ctx, &grid.ntrack, &t, &itl, h.prim.data(), h.x.data(), h.dx.data(), h.dtl.data(),
                         h.xI.data()),
        "gamma_gpu_upload");

  const long sync_every = env_long("GAMMA_SHIM_SYNC_EVERY", 1);
  const long max_steps = env_long("GAMMA_SHIM_MAX_STEPS", 0);
  long steps = 0;
  while (!stop) {
    gamma_step_stats_t st;
    check(gamma_gpu_step(ctx, 1, &st), "gamma_gpu_step");
    if (st.status == GAMMA_ERR_NEG_DT) exit(30);  // cell.cpp:70-73
    check(st.status, "step");
    ++steps;
    int ntrack = 0, status = 0;
    const bool sync = sync_every > 0 && steps % sync_every == 0;
    check(gamma_gpu_download(ctx, &ntrack, &t, &dt, &itl, &status, sync ? h.prim.data() : nullptr,
                             sync ? h.x.data() : nullptr, sync ? h.dx.data() : nullptr,
                             sync ? h.dtl.data() : nullptr, sync ? h.xI.data() : nullptr),
          "gamma_gpu_download");
    it = itl;
    if (sync) unpack(h, ntrack, grid);
    dataDump();
    runInfo();
    evalEnd();
    if (max_steps > 0 && steps >= max_steps) stop = true;
  }
  int ntrack = 0, status = 0;
  check(gamma_gpu_download(ctx, &ntrack, &t, &dt, &itl, &status, h.prim.data(), h.x.data(), h.dx.data(),
                           h.dtl.data(), h.xI.data()),
        "gamma_gpu_download");
  unpack(h, ntrack, grid);
  gamma_gpu_destroy(ctx);
}
