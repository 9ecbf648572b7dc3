/*
 * Problem setup (an INITIAL module) for the oracle: one planar relativistic
 * shock tube on [xmin, xmax] with the discontinuity at xmid, parameters set at
 * run time through ref_set_param.  TEST INFRASTRUCTURE.
 *
 * The hooks follow src/Initial/Tests/1DST.cpp (no user kinematics, boundaries,
 * sources or regrid: 1DST.cpp:81-128).  Unlike 1DST.cpp:52,58, which write the
 * tracer into cons[TR1] where prepForRun's prim2cons overwrites it with zero,
 * the tracer is set in prim[TR1] so that it is advected.
 */
#include "environment.h"
#include "grid.h"
#include "constants.h"
#include "simu.h"

#include <cstring>

namespace {
struct TubeParams {
  double xmin = 0., xmax = 1., xmid = 0.5;
  double ncell = 1000., nmax = 1000., ngst = 2.;
  double rhoL = 10., pL = 13.33, vL = 0., trL = 1.;
  double rhoR = 1., pR = 1.e-7, vR = 0., trR = 2.;
};
TubeParams P;
}  // namespace

extern "C" __attribute__((visibility("default"))) int ref_set_param(const char *name, double v) {
#define SETP(f) \
  if (!strcmp(name, #f)) { P.f = v; return 0; }
  SETP(xmin) SETP(xmax) SETP(xmid) SETP(ncell) SETP(nmax) SETP(ngst)
  SETP(rhoL) SETP(pL) SETP(vL) SETP(trL) SETP(rhoR) SETP(pR) SETP(vR) SETP(trR)
#undef SETP
  return -1;
}

// 1DST.cpp:19-26
void loadParams(s_par *par) {
  par->tini = 0.;
  par->ncell[x_] = (int)P.ncell;
  par->nmax = (int)P.nmax;
  par->ngst = (int)P.ngst;
}

// 1DST.cpp:28-39
int Grid::initialGeometry() {
  double x = P.xmax - P.xmin;
  for (int i = 0; i < ncell[x_]; ++i) {
    Cell *c = &Cinit[i];
    c->G.x[x_] = (double)x * (i + 0.5) / ncell[x_] + P.xmin;
    c->G.dx[x_] = x / ncell[x_];
    c->computeAllGeom();
  }
  return 0;
}

// 1DST.cpp:42-78 (velocities are 3-velocities; prepForRun turns them into u = Gamma v)
int Grid::initialValues() {
  for (int i = 0; i < ncell[MV]; ++i) {
    Cell *c = &Cinit[i];
    if (c->G.x[x_] <= P.xmid) {
      c->S.prim[RHO] = P.rhoL;
      c->S.prim[VV1] = P.vL;
      c->S.prim[PPP] = P.pL;
      c->S.prim[TR1] = P.trL;
    } else {
      c->S.prim[RHO] = P.rhoR;
      c->S.prim[VV1] = P.vR;
      c->S.prim[PPP] = P.pR;
      c->S.prim[TR1] = P.trR;
    }
  }
  return 0;
}

void Grid::userKinematics(int it, double t) { UNUSED(it); UNUSED(t); }
void Cell::userSourceTerms(double dt) { UNUSED(dt); }
void Grid::userBoundaries(int it, double t) { UNUSED(it); UNUSED(t); }
int Grid::checkCellForRegrid(int j, int i) { UNUSED(j); UNUSED(i); return (skip_); }
void Cell::user_regridVal(double *res) { UNUSED(res); }
void FluidState::cons2prim_user(double *rho, double *p, double *uu) { UNUSED(rho); UNUSED(p); UNUSED(uu); }
void Simu::dataDump() {}
void Simu::runInfo() {}
void Simu::evalEnd() {}
