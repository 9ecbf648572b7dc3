/*
 * C entry points around the compiled 2D GAMMA reference (oracle/_ref/libref_jet2d.so).
 * TEST INFRASTRUCTURE: only tests/ and bench.py's CPU arms load it, as the
 * checker or the timed CPU reference.
 *
 * Everything that moves the solution is the reference's own code
 * (src/simu.cpp, src/grid.cpp, src/Dimensions/2d.cpp, src/Timestep/rk3.cpp,
 * src/Geometry/spherical.cpp, src/Hydro/rel_sph.cpp, ...) compiled unmodified
 * with NUM_D = 2.  This file sequences the Simu::run loop body
 * (src/simu.cpp:79-105) and copies the Grid out as per-track arrays, including
 * the cell fields that carry state between stages in the reference: the
 * moving-direction and transverse gradients (grad_mv, grad_f1) and the
 * neighbour lists (Cell::neigh), which cells 0 and ntrack-1 of each track keep
 * from earlier stages.
 */
#include "simu.h"
#include "mpisetup.h"
#include "constants.h"
#include "../brent.h"

#define REF_API extern "C" __attribute__((visibility("default")))

static Simu *g_simu = nullptr;

REF_API int ref_nq(void) { return NUM_Q; }
REF_API int ref_num_d(void) { return NUM_D; }
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

/* Grid::printCols of the linked IO module (src/IO/text2d.cpp:145-283 in the *_io
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

/* Grid::regrid alone (src/Dimensions/2d.cpp:609-620). */
REF_API int ref_regrid(void) {
  g_simu->grid.regrid();
  return 0;
}

/* t, dt, it, number of tracks with ghosts (nde_nax[F1]), track capacity
 * (nde_nax[MV]), jLbnd, jRbnd */
REF_API void ref_scalars(double *out) {
  Simu &s = *g_simu;
  Grid &g = s.grid;
  out[0] = s.t;
  out[1] = s.dt;
  out[2] = (double)s.it;
  out[3] = g.nde_nax[F1];
  out[4] = g.nde_nax[MV];
  out[5] = g.jLbnd;
  out[6] = g.jRbnd;
}

/* ntrack, nact, iLbnd, iRbnd of track j */
REF_API void ref_track_info(int j, int *out) {
  Grid &g = g_simu->grid;
  out[0] = g.ntrack[j];
  out[1] = g.nact[j];
  out[2] = g.iLbnd[j];
  out[3] = g.iRbnd[j];
}

/* Cells i < ntrack of track j (layout [q*cap + i]): prim, r and dr, theta and
 * dtheta, dt_loc, Sd, pspec, isShocked, grad_mv, grad_f1; interfaces
 * i < ntrack-1: xI.  nbr[(4*i + 2*side + {0,1})]: the neighbour list of cell i
 * towards track j-1 (side 0) / j+1 (side 1) as (first flat cell id, count);
 * returns -2 if a list is not a run of consecutive ids.  Any pointer may be null. */
REF_API int ref_snapshot(int j, double *prim, double *x, double *dx, double *th, double *dth, double *dt_loc,
                         double *sd, double *pspec, double *shocked, double *grad_mv, double *grad_f1,
                         double *xI, int *nbr, int cap) {
  Grid &g = g_simu->grid;
  const int n = g.ntrack[j];
  if (n > cap) return -1;
  int rc = n;
  for (int i = 0; i < n; ++i) {
    Cell &c = g.Ctot[j][i];
    for (int q = 0; q < NUM_Q; ++q) {
      if (prim) prim[q * cap + i] = c.S.prim[q];
      if (grad_mv) grad_mv[q * cap + i] = c.grad_mv[q];
      if (grad_f1) grad_f1[q * cap + i] = c.grad_f1[q];
    }
    if (x) x[i] = c.G.x[MV];
    if (dx) dx[i] = c.G.dx[MV];
    if (th) th[i] = c.G.x[F1];
    if (dth) dth[i] = c.G.dx[F1];
    if (dt_loc) dt_loc[i] = c.dt_loc;
#if SHOCK_DETECTION_ == ENABLED_
    if (sd) sd[i] = c.Sd;
    if (pspec) pspec[i] = c.pspec;
    if (shocked) shocked[i] = c.isShocked ? 1.0 : 0.0;
#endif
    if (nbr) {
      for (int side = 0; side < 2; ++side) {
        const std::vector<int> &v = c.neigh[F1][side];
        nbr[4 * i + 2 * side] = v.empty() ? -1 : v[0];
        nbr[4 * i + 2 * side + 1] = (int)v.size();
        for (size_t k = 1; k < v.size(); ++k)
          if (v[k] != v[k - 1] + 1) rc = -2;
      }
    }
  }
  if (xI)
    for (int i = 0; i < n - 1; ++i) xI[i] = g.Itot[j][i].x[MV];
  return rc;
}

/* Grid::computeNeighbors alone (src/Dimensions/2d.cpp:534-606), for tests of
 * the neighbour search on the current grid. */
REF_API void ref_compute_neighbors(void) { g_simu->grid.computeNeighbors(false); }

/* The first part of one loop iteration, for checks of intermediate results:
 * what = 1: regrid, resetShock, updateGhosts;  what = 2: ... and prepForUpdate
 * (the stage-1 fluxes);  what = 3: ... and the stage-1 update. */
REF_API int ref_partial(int what) {
  Simu &s = *g_simu;
  s.grid.regrid();
#if SHOCK_DETECTION_ == ENABLED_
  s.grid.apply(&Cell::resetShock);
#endif
  s.grid.updateGhosts(s.it, s.t);
  if (what >= 2) s.grid.prepForUpdate(s.it, s.t);
  if (what >= 3) {  // the first stage of Grid::evolve (rk3.cpp:101-105)
#if SHOCK_DETECTION_ == ENABLED_
    s.grid.apply(&Cell::detectShock);
#endif
    s.dt = CFL_ * s.grid.collect_dt();
    s.grid.copyState0();
    s.grid.update(s.dt);
  }
  // the later stages of rk3.cpp:107-192 up to their fluxes: what = 4 stops
  // after stage 2's prepForUpdate, 5 after stage 3's (the stage bodies are the
  // reference's, in its order; the combines restate its loops)
  for (int st = 2; st <= 3 && what >= st + 2; ++st) {
    Grid &g = s.grid;
    if (st == 3) {
      g.update(s.dt);
      for (int j = g.jLbnd + 1; j <= g.jRbnd - 1; ++j)
        for (int i = g.iLbnd[j] + 1; i <= g.iRbnd[j] - 1; ++i) {
          Cell *c = &g.Ctot[j][i];
          double dV = c->G.dV, dV0 = c->G0.dV;
          for (int q = 0; q < NUM_Q; ++q) c->S.cons[q] = 3. / 4. * c->S0.cons[q] * dV0 + 1. / 4. * c->S.cons[q] * dV;
        }
      for (int j = g.jLbnd + 1; j <= g.jRbnd - 1; ++j)
        for (int i = g.iLbnd[j]; i <= g.iRbnd[j] - 1; ++i) {
          Interface *I = &g.Itot[j][i];
          I->x[MV] = 3. / 4. * I->x0[MV] + 1. / 4. * I->x[MV];
          I->computedA();
        }
      g.CellGeomFromInterfacePos();
      for (int j = g.jLbnd + 1; j <= g.jRbnd - 1; ++j)
        for (int i = g.iLbnd[j] + 1; i <= g.iRbnd[j] - 1; ++i) {
          Cell *c = &g.Ctot[j][i];
          for (int q = 0; q < NUM_Q; ++q) c->S.cons[q] /= c->G.dV;
          c->S.cons2prim(c->G.x[r_]);
        }
    }
    g.updateGhosts(s.it, s.t);
    g.prepForUpdate(s.it, s.t);
  }
  return 0;
}

/* Cell::flux of the cells i < ntrack of track j: out[((s*2 + d)*NUM_Q + q)*cap + i]
 * (s: left/right side, d: MV/F1), and the interfaces' velocity, lambda_L,
 * lambda_R and flux: iface[(k*cap + i)], k = 0: v, 1: lL, 2: lR, 3+q: flux[q]. */
REF_API int ref_fluxes(int j, double *out, double *iface, int cap) {
  Grid &g = g_simu->grid;
  const int n = g.ntrack[j];
  if (n > cap) return -1;
  for (int i = 0; i < n; ++i)
    for (int s = 0; s < 2; ++s)
      for (int d = 0; d < 2; ++d)
        for (int q = 0; q < NUM_Q; ++q) out[((s * 2 + d) * NUM_Q + q) * cap + i] = g.Ctot[j][i].flux[s][d][q];
  for (int i = 0; i < n - 1; ++i) {
    Interface &I = g.Itot[j][i];
    iface[0 * cap + i] = I.v;
    iface[1 * cap + i] = I.lL;
    iface[2 * cap + i] = I.lR;
    for (int q = 0; q < NUM_Q; ++q) iface[(3 + q) * cap + i] = I.flux[q];
  }
  return n;
}

/* Stopping tolerance of the cons2prim root search (the reference's is 1e-13,
 * rel_sph.cpp:281); 0 restores it. */
REF_API void ref_set_c2p_epsrel(double epsrel) { oracle_brent_override_epsrel(epsrel); }
