/*
 * C entry points around the compiled GAMMA reference (oracle/_ref/libref_*.so).
 * TEST INFRASTRUCTURE: only tests/, the smoke check and bench.py's CPU baseline
 * load these libraries, and only as the checker or the timed CPU reference.
 *
 * Everything that moves the solution forward is the reference's own code
 * (src/simu.cpp, src/grid.cpp, src/Dimensions/1d.cpp, src/Timestep/rk3.cpp, ...),
 * compiled unmodified.  This file only
 *   - sequences the Simu::run loop body one iteration at a time
 *     (src/simu.cpp:72-109; the loop is restated here because Simu::run only
 *     stops through the problem's evalEnd hook), and
 *   - copies the Grid state in and out as structure-of-arrays buffers.
 */
#include "simu.h"
#include "mpisetup.h"
#include "constants.h"
#include "../brent.h"

#define REF_API extern "C" __attribute__((visibility("default")))

static Simu *g_simu = nullptr;

REF_API int ref_nq(void) { return NUM_Q; }
REF_API int ref_num_d(void) { return NUM_D; }
REF_API int ref_shock_detection(void) { return SHOCK_DETECTION_ == ENABLED_; }
REF_API int ref_local_synchrotron(void) { return LOCAL_SYNCHROTRON_ == ENABLED_; }
REF_API double ref_gamma_ad(void) { return GAMMA_; }

/* Simu::initialise (src/simu.cpp:24-38) then the pre-loop part of Simu::run
 * (updateGhosts + printCols, src/simu.cpp:74-75). */
REF_API int ref_init(void) {
  int argc = 0;
  char **argv = nullptr;
  mpi_init(&argc, &argv);
  checkEnvironment();
  g_simu = new Simu();
  g_simu->initialise();
  g_simu->grid.updateGhosts(g_simu->it, g_simu->t);
  g_simu->grid.printCols(g_simu->it, g_simu->t);
  return 0;
}

/* Grid::printCols of the linked IO module (src/IO/text1d.cpp:135-243 in the *_io
 * builds): writes ../results/Last/phys%010d.out relative to the working
 * directory, which must exist.  io_none.cpp's printCols does nothing. */
REF_API void ref_print_cols(void) { g_simu->grid.printCols(g_simu->it, g_simu->t); }

/* The resume start of main.cpp (src/main.cpp:43-49 with -r): Simu::reinitialise
 * from the last phys*.out under ../results/Last, then the pre-loop part of
 * Simu::run (updateGhosts + printCols, src/simu.cpp:74-75).  *_io builds only. */
REF_API int ref_resume(void) {
  int argc = 0;
  char **argv = nullptr;
  mpi_init(&argc, &argv);
  checkEnvironment();
  DIR *dir = opendir("../results/Last");
  if (!dir) return -1;
  g_simu = new Simu();
  g_simu->reinitialise(dir);
  g_simu->grid.updateGhosts(g_simu->it, g_simu->t);
  g_simu->grid.printCols(g_simu->it, g_simu->t);
  return 0;
}

/* n iterations of the body of Simu::run's loop (src/simu.cpp:79-105). */
REF_API int ref_step(int n) {
  Simu &s = *g_simu;
  for (int k = 0; k < n; ++k) {
    s.grid.regrid();
#if SHOCK_DETECTION_ == ENABLED_
    s.grid.apply(&Cell::resetShock);
#endif
    s.grid.updateGhosts(s.it, s.t);
    s.grid.prepForUpdate(s.it, s.t);
#if SHOCK_DETECTION_ == ENABLED_
    s.grid.apply(&Cell::detectShock);
#endif
    s.dt = CFL_ * s.grid.collect_dt();
    s.grid.evolve(s.it, s.t, s.dt);
    s.t += s.dt;
    s.it++;
#if LOCAL_SYNCHROTRON_ == ENABLED_
    s.grid.apply(&Cell::radiation_injectParticles);
#endif
    s.dataDump();
    s.runInfo();
    s.evalEnd();
  }
  return 0;
}

/* Grid::regrid alone (src/Dimensions/1d.cpp:484-495). */
REF_API int ref_regrid(void) {
  g_simu->grid.regrid();
  return 0;
}

/* t, dt, it, ntrack, nact, iLbnd, iRbnd, capacity (nde_nax) */
REF_API void ref_scalars(double *out) {
  Simu &s = *g_simu;
  out[0] = s.t;
  out[1] = s.dt;
  out[2] = (double)s.it;
  out[3] = s.grid.ntrack;
  out[4] = s.grid.nact;
  out[5] = s.grid.iLbnd;
  out[6] = s.grid.iRbnd;
  out[7] = s.grid.nde_nax[MV];
}

/* Per cell i < ntrack: prim[q*cap+i], x, dx, dt_loc, Sd, pspec, isShocked.
 * Per interface i < ntrack-1: xI[i].  Any output pointer may be null. */
REF_API int ref_snapshot(double *prim, double *x, double *dx, double *dt_loc, double *sd,
                         double *pspec, double *shocked, double *xI, int cap) {
  Grid &g = g_simu->grid;
  if (g.ntrack > cap) return -1;
  for (int i = 0; i < g.ntrack; ++i) {
    Cell &c = g.Ctot[i];
    if (prim)
      for (int q = 0; q < NUM_Q; ++q) prim[q * cap + i] = c.S.prim[q];
    if (x) x[i] = c.G.x[MV];
    if (dx) dx[i] = c.G.dx[MV];
    if (dt_loc) dt_loc[i] = c.dt_loc;
#if SHOCK_DETECTION_ == ENABLED_
    if (sd) sd[i] = c.Sd;
    if (pspec) pspec[i] = c.pspec;
    if (shocked) shocked[i] = c.isShocked ? 1.0 : 0.0;
#else
    if (sd) sd[i] = 0;
    if (pspec) pspec[i] = 0;
    if (shocked) shocked[i] = 0;
#endif
  }
  if (xI)
    for (int i = 0; i < g.ntrack - 1; ++i) xI[i] = g.Itot[i].x[MV];
  return g.ntrack;
}

/* Overwrite the track with the given cells (the inverse of ref_snapshot) so a
 * regrid or a step can start from a chosen state.  Geometry is rebuilt with
 * Cell::computeAllGeom, and cons/flux with prim2cons/state2flux at G.cen, as
 * Grid::prepForRun leaves them (src/grid.cpp:20-26). */
REF_API int ref_load(int ntrack, const double *prim, const double *x, const double *dx,
                     const double *dt_loc, const double *xI, int cap, double t, long it) {
  Simu &s = *g_simu;
  Grid &g = s.grid;
  if (ntrack > g.nde_nax[MV] || ntrack > cap) return -1;
  g.ntrack = ntrack;
  g.nact = ntrack - 2 * g.ngst;
  g.iLbnd = g.ngst - 1;
  g.iRbnd = ntrack - g.ngst;
  for (int i = 0; i < ntrack; ++i) {
    Cell &c = g.Ctot[i];
    for (int q = 0; q < NUM_Q; ++q) c.S.prim[q] = prim[q * cap + i];
    c.G.x[MV] = x[i];
    c.G.dx[MV] = dx[i];
    c.computeAllGeom();
    c.dt_loc = dt_loc ? dt_loc[i] : 1.e15;
    c.S.prim2cons(c.G.cen[r_]);
    c.S.state2flux(c.G.cen[r_]);
    int ind[] = {i};
    g.assignId(ind);
  }
  for (int i = 0; i < ntrack - 1; ++i) {
    g.Itot[i].x[MV] = xI[i];
    g.Itot[i].computedA();
  }
  s.t = t;
  s.it = it;
  return 0;
}

/* FluidState::cons2prim on n independent states (src/Hydro/rel_sph.cpp:213-320 or
 * rel_cart.cpp:125-229).  prim holds the previous primitives (the pressure warm
 * start) on entry and the recovered ones on exit; cons is rewritten by the
 * closing prim2cons, as in the reference.  Layout [q*n + k]. */
REF_API void ref_cons2prim(double *cons, double *prim, const double *r, int n) {
  for (int k = 0; k < n; ++k) {
    FluidState S;
    for (int q = 0; q < NUM_Q; ++q) {
      S.cons[q] = cons[q * n + k];
      S.prim[q] = prim[q * n + k];
    }
    S.cons2prim(r ? r[k] : 1.0);
    for (int q = 0; q < NUM_Q; ++q) {
      cons[q * n + k] = S.cons[q];
      prim[q * n + k] = S.prim[q];
    }
  }
}

/* FluidState::prim2cons on n states, layout [q*n + k]. */
REF_API void ref_prim2cons(const double *prim, double *cons, const double *r, int n) {
  for (int k = 0; k < n; ++k) {
    FluidState S;
    for (int q = 0; q < NUM_Q; ++q) S.prim[q] = prim[q * n + k];
    S.prim2cons(r ? r[k] : 1.0);
    for (int q = 0; q < NUM_Q; ++q) cons[q * n + k] = S.cons[q];
  }
}

/* One moving-interface HLLC problem per k: given the left/right primitive
 * states, the interface position x and (if v_given) its velocity, compute
 * lambda_L, lambda_*, lambda_R and the flux F - vU times dA
 * (src/Hydro/rel_sph.cpp:322-450, src/Solver/hllc.cpp:12-39).  If v_given is 0
 * the interface moves at VI*lambda_* (src/Dimensions/1d.cpp:741-751).
 * out_l: [3*k + {0,1,2}]; flux: [q*n + k]. */
REF_API void ref_riemann(const double *primL, const double *primR, const double *x,
                         const double *v, int v_given, double *out_l, double *flux, int n) {
  for (int k = 0; k < n; ++k) {
    Interface I;
    I.x[MV] = x[k];
    I.computedA();
    for (int q = 0; q < NUM_Q; ++q) {
      I.SL.prim[q] = primL[q * n + k];
      I.SR.prim[q] = primR[q * n + k];
    }
    I.SL.prim2cons(I.x[MV]);
    I.SL.state2flux(I.x[MV]);
    I.SR.prim2cons(I.x[MV]);
    I.SR.state2flux(I.x[MV]);
    I.computeLambda();
    I.v = v_given ? v[k] : VI * I.lS;
    I.computeFlux();
    out_l[3 * k + 0] = I.lL;
    out_l[3 * k + 1] = I.lS;
    out_l[3 * k + 2] = I.lR;
    for (int q = 0; q < NUM_Q; ++q) flux[q * n + k] = I.flux[q];
  }
}

/* Stopping tolerance of the cons2prim root search (the reference's is 1e-13,
 * rel_sph.cpp:281 / rel_cart.cpp:193); 0 restores it. */
REF_API void ref_set_c2p_epsrel(double epsrel) { oracle_brent_override_epsrel(epsrel); }
