/*
 * Problem setup (an INITIAL module) for the oracle: a planar shock tube whose
 * every user hook does something, to pin the B200 library's hook routing
 * (tests/modules/hooked_tube.cu implements the same hooks as a problem module).
 * TEST INFRASTRUCTURE.
 *
 *   userBoundaries       a reflecting wall on the left: the left ghosts' velocity
 *                        is reversed
 *   userKinematics       left ghost interfaces fixed (v = 0), right ghost
 *                        interfaces at v_out
 *   userSourceTerms      uniform acceleration -g on the momentum
 *   cons2prim_user       a pressure floor p_floor
 *   checkCellForRegrid   split wider than split_dx, merge narrower than merge_dx
 */
#include "environment.h"
#include "grid.h"
#include "constants.h"
#include "simu.h"

#include <cstring>

namespace {
struct HookedParams {
  double g = 0.5, p_floor = 2.e-3, v_out = 0.2, split_dx = 1.6e-3, merge_dx = 0.6e-3;
  double ncell = 1000., nmax = 2000., xmin = 0.1, xmax = 1.1, xmid = 0.6;
  double rhoL = 10., pL = 13.33, vL = 0.3, rhoR = 1., pR = 1.e-3, vR = 0.;
  double reflect = 1., wall = 1.;  // 0 turns the reflecting ghosts / the fixed wall interfaces off
};
HookedParams P;
}  // namespace

extern "C" __attribute__((visibility("default"))) int ref_set_param(const char *name, double v) {
#define SETP(f) \
  if (!strcmp(name, #f)) { P.f = v; return 0; }
  SETP(g) SETP(p_floor) SETP(v_out) SETP(split_dx) SETP(merge_dx) SETP(ncell) SETP(nmax) SETP(xmin)
  SETP(xmax) SETP(xmid) SETP(rhoL) SETP(pL) SETP(vL) SETP(rhoR) SETP(pR) SETP(vR) SETP(reflect) SETP(wall)
#undef SETP
  return -1;
}

void loadParams(s_par *par) {
  par->tini = 0.;
  par->ncell[x_] = (int)P.ncell;
  par->nmax = (int)P.nmax;
  par->ngst = 2;
}

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

int Grid::initialValues() {
  for (int i = 0; i < ncell[MV]; ++i) {
    Cell *c = &Cinit[i];
    const bool left = c->G.x[x_] <= P.xmid;
    c->S.prim[RHO] = left ? P.rhoL : P.rhoR;
    c->S.prim[VV1] = left ? P.vL : P.vR;
    c->S.prim[PPP] = left ? P.pL : P.pR;
    c->S.prim[TR1] = left ? 1. : 2.;
  }
  return 0;
}

void Grid::userKinematics(int it, double t) {
  UNUSED(it);
  UNUSED(t);
  for (int n = 0; n < ngst; ++n) {
    if (P.wall != 0.) Itot[n].v = 0.;
    Itot[ntrack - 2 - n].v = P.v_out;
  }
}

void Cell::userSourceTerms(double dt) { S.cons[SS1] -= P.g * S.cons[DEN] * dt; }

void Grid::userBoundaries(int it, double t) {
  UNUSED(it);
  UNUSED(t);
  if (P.reflect != 0.)
    for (int i = 0; i <= iLbnd; ++i) Ctot[i].S.prim[UU1] = -Ctot[i].S.prim[UU1];
}

int Grid::checkCellForRegrid(int j, int i) {
  UNUSED(j);
  Cell c = Ctot[i];
  double dx = c.G.dx[x_];
  if (dx > P.split_dx) return (split_);
  if (dx < P.merge_dx) return (merge_);
  return (skip_);
}

void Cell::user_regridVal(double *res) { UNUSED(res); }

void FluidState::cons2prim_user(double *rho, double *p, double *uu) {
  UNUSED(rho);
  UNUSED(uu);
  *p = fmax(*p, P.p_floor);
}

void Simu::dataDump() {}
void Simu::runInfo() {}
void Simu::evalEnd() {}
