/*
 * Problem setup (an INITIAL module) for the oracle: a 1D spherical
 * Blandford-McKee blast wave whose parameters are set at run time through
 * ref_set_param, so one build serves both the reference's own Tests/BM1D
 * parameters and the log-spaced Gamma_shock = 100 workload.  TEST
 * INFRASTRUCTURE.
 *
 * Each hook follows src/Initial/Tests/BM1D.cpp (cited per function); the only
 * differences are that the constants are variables and that the cells may be
 * laid out log-uniformly in r.  tests/ checks this module against BM1D.cpp
 * itself (both compiled into oracle/_ref) with BM1D.cpp's parameters.
 */
#include "environment.h"
#include "grid.h"
#include "constants.h"
#include "simu.h"

#include <cstring>

namespace {
struct Bm1dParams {
  double n0 = 1.;            // CBM number density (cm^-3) -> rhoNorm = n0 mp
  double eta = 1.e-5;        // p / (rho c^2) of the ambient medium
  double Etot = 1.e53;       // erg
  double n_ext = 1.;         // external number density
  double tinit = 4.e6;       // s, start time when lorentz_mode == 0
  double lfac_shock2 = 0.;   // Gamma_shock^2 when lorentz_mode == 1
  double lorentz_mode = 0.;  // 0: BM1D.cpp LORENTZ_==0 branch; 1: Gamma_shock given
  double Rscale = 1.e17;     // cm
  double k = 0.;             // ambient density slope
  double ncell = 9900.;
  double nmax = 10000.;
  double ngst = 2.;
  double grid_log = 0.;      // 0: uniform over R(1 -+ 50/Gs^2) (BM1D.cpp); 1: log-spaced
  double r_lo = 0.9;         // log grid: [r_lo, r_hi] x R_shock
  double r_hi = 1.1;
  double dth = M_PI / 2. / 1000.;
  double target_ar = 1.;
  double split_AR = 3.;
  double merge_AR = 0.1;
  double t_bm_until = 1.e7;  // analytic inner boundary while t < this
  double v_in = 0.;          // ghost-interface velocities
  double v_out = 1.5;
};
Bm1dParams P;

// derived (BM1D.cpp:28-65)
double rho0, rhoNorm, lNorm, vNorm, pNorm;
double tstart, lfacShock2, RShock, rhoa, pa, ha, pf, lfacf, Df;

void derive() {
  rho0 = P.n0 * mp_;
  rhoNorm = rho0;
  lNorm = c_;
  vNorm = c_;
  pNorm = rhoNorm * vNorm * vNorm;
  if (P.lorentz_mode != 0.) {
    lfacShock2 = P.lfac_shock2;
    tstart = pow(P.Etot * (17.) / (8. * PI * P.n_ext * mp_ * pow(c_, 5.) * lfacShock2), 1. / 3.);
  } else {
    tstart = P.tinit;
    lfacShock2 = P.Etot * (17. - 4. * P.k) / (8. * PI * P.n_ext * mp_ * pow(tstart, 3) * pow(c_, 5));
  }
  RShock = c_ * tstart * (1. - 1. / (1. + 2. * (4. - P.k) * lfacShock2));
  rhoa = P.n_ext * mp_ * pow(RShock / P.Rscale, -P.k);
  pa = rhoa * P.eta * c_ * c_;
  ha = c_ * c_ + pa * GAMMA_ / (GAMMA_ - 1.) / rhoa;
  pf = 2. / 3. * lfacShock2 * ha * rhoa;
  lfacf = sqrt(fmax(1., .5 * lfacShock2));
  Df = 2. * lfacShock2 * rhoa;
}

// BM1D.cpp:62-86
void calcBM(double r, double t, double *rho, double *u, double *p) {
  double lfacShock2_t = P.Etot * (17. - 4. * P.k) / (8. * PI * P.n_ext * mp_ * pow(t, 3) * pow(c_, 5));
  double RShock_t = c_ * t * (1. - 1. / (1. + 2. * (4. - P.k) * lfacShock2_t));
  double rhoa_t = P.n_ext * mp_ * pow(RShock_t / P.Rscale, -P.k);
  double pa_t = rhoa_t * P.eta * c_ * c_;
  double ha_t = c_ * c_ + pa_t * GAMMA_ / (GAMMA_ - 1.) / rhoa_t;
  double pf_t = 2. / 3. * lfacShock2_t * ha_t * rhoa_t;
  double lfacf_t = sqrt(fmax(1., .5 * lfacShock2_t));
  double Df_t = 2. * lfacShock2_t * rhoa_t;
  double chi = (1. + 2. * (4. - P.k) * lfacShock2_t) * (1. - r / (c_ * t));
  *p = pf_t * pow(chi, -(17. - 4. * P.k) / (12. - 3. * P.k)) / pNorm;
  double lfac = sqrt(lfacf_t * lfacf_t / chi + 1);
  double D = Df_t * pow(chi, -(7. - 2. * P.k) / (4. - P.k));
  *rho = D / lfac / rhoNorm;
  *u = c_ * sqrt(1. - 1. / (lfac * lfac)) * lfac / vNorm;
}
}  // namespace

extern "C" __attribute__((visibility("default"))) int ref_set_param(const char *name, double v) {
#define SETP(f) \
  if (!strcmp(name, #f)) { P.f = v; return 0; }
  SETP(n0) SETP(eta) SETP(Etot) SETP(n_ext) SETP(tinit) SETP(lfac_shock2) SETP(lorentz_mode)
  SETP(Rscale) SETP(k) SETP(ncell) SETP(nmax) SETP(ngst) SETP(grid_log) SETP(r_lo) SETP(r_hi)
  SETP(dth) SETP(target_ar) SETP(split_AR) SETP(merge_AR) SETP(t_bm_until) SETP(v_in) SETP(v_out)
#undef SETP
  return -1;
}

/* Derived quantities after loadParams: tstart, RShock (code units: ls) and the
 * normalisations, so the host side can reproduce the boundary hook. */
extern "C" __attribute__((visibility("default"))) void ref_bm1d_derived(double *out) {
  derive();
  out[0] = tstart;
  out[1] = RShock / lNorm;
  out[2] = lfacShock2;
  out[3] = rhoNorm;
  out[4] = pNorm;
  out[5] = lNorm;
  out[6] = vNorm;
}

// BM1D.cpp:89-98
void loadParams(s_par *par) {
  derive();
  par->tini = tstart;
  par->ncell[x_] = (int)P.ncell;
  par->nmax = (int)P.nmax;
  par->ngst = (int)P.ngst;
  normalizeConstants(rhoNorm, vNorm, lNorm);
}

// BM1D.cpp:100-116 (uniform); the log-spaced layout places cell edges at
// r_lo R (r_hi / r_lo)^(i/N).
int Grid::initialGeometry() {
  if (P.grid_log == 0.) {
    double rmin = RShock * (1. - 50. / lfacShock2);
    double rmax = RShock * (1. + 50. / lfacShock2);
    rmin /= lNorm;
    rmax /= lNorm;
    double dr = (rmax - rmin) / ncell[x_];
    for (int i = 0; i < ncell[x_]; ++i) {
      Cell *c = &Cinit[i];
      double r = rmin + (i + 0.5) * dr;
      c->G.x[x_] = r;
      c->G.dx[x_] = dr;
      c->computeAllGeom();
    }
  } else {
    double rmin = P.r_lo * RShock / lNorm;
    double rmax = P.r_hi * RShock / lNorm;
    double lr = log(rmax / rmin);
    for (int i = 0; i < ncell[x_]; ++i) {
      Cell *c = &Cinit[i];
      double rl = rmin * exp(lr * i / ncell[x_]);
      double rr = rmin * exp(lr * (i + 1) / ncell[x_]);
      c->G.x[x_] = 0.5 * (rl + rr);
      c->G.dx[x_] = rr - rl;
      c->computeAllGeom();
    }
  }
  return 0;
}

// BM1D.cpp:118-185 (one bin per cell, as there)
int Grid::initialValues() {
  for (int i = 0; i < ncell[MV]; ++i) {
    Cell *c = &Cinit[i];
    double r = c->G.x[x_];
    double dr = c->G.dx[x_];
    double r_denorm = r * lNorm;
    double dr_denorm = dr * lNorm;
    if (r_denorm > RShock) {
      double rho = P.n_ext * mp_ * pow(r_denorm / P.Rscale, -P.k);
      c->S.prim[RHO] = rho / rhoNorm;
      c->S.prim[VV1] = 0;
      c->S.prim[PPP] = P.eta * rho * c_ * c_ / pNorm;
      c->S.prim[TR1] = 1.;
    } else {
      double xl = r_denorm - dr_denorm / 2.;
      double xr = xl + dr_denorm;
      double dV = 4. / 3. * PI * (pow(r_denorm + dr_denorm / 2., 3) - pow(r_denorm - dr_denorm / 2., 3));
      double x = (xr + xl) / 2.;
      double ddV = 4. / 3. * PI * (xr * xr * xr - xl * xl * xl);
      double chi = (1. + 2. * (4. - P.k) * lfacShock2) * (1. - x / (c_ * tstart));
      double dp = pf * pow(chi, -(17. - 4. * P.k) / (12. - 3. * P.k));
      double dlfac = sqrt(lfacf * lfacf / chi + 1);
      double dD = Df * pow(chi, -(7. - 2. * P.k) / (4. - P.k));
      double drho = dD / dlfac;
      double dv = c_ * sqrt(1. - 1. / (dlfac * dlfac));
      double rho = 0, v = 0, p = 0;
      rho += drho * ddV / dV;
      v += dv * ddV / dV;
      p += dp * ddV / dV;
      c->S.prim[RHO] = rho / rhoNorm;
      c->S.prim[VV1] = v / vNorm;
      c->S.prim[PPP] = p / pNorm;
      c->S.prim[TR1] = 2.;
    }
  }
  return 0;
}

// BM1D.cpp:188-246: the ghost interfaces move at fixed speeds (the shock scan
// there only feeds a value that is overwritten before use).
void Grid::userKinematics(int it, double t) {
  UNUSED(it);
  UNUSED(t);
  for (int n = 0; n < ngst; ++n) {
    int iL = n;
    int iR = ntrack - 2 - n;
    Itot[iL].v = P.v_in;
    Itot[iR].v = P.v_out;
  }
}

void Cell::userSourceTerms(double dt) { UNUSED(dt); }

// BM1D.cpp:254-274
void Grid::userBoundaries(int it, double t) {
  UNUSED(it);
  if (t < P.t_bm_until) {
    for (int i = 0; i <= iLbnd; ++i) {
      Cell *c = &Ctot[i];
      double rho, u, p;
      double r = c->G.x[r_] * lNorm;
      calcBM(r, t, &rho, &u, &p);
      c->S.prim[RHO] = rho;
      c->S.prim[UU1] = u;
      c->S.prim[UU2] = 0;
      c->S.prim[PPP] = p;
      c->S.prim[TR1] = 2.;
    }
  }
}

// BM1D.cpp:277-319
int Grid::checkCellForRegrid(int j, int i) {
  UNUSED(j);
  Cell c = Ctot[i];
  double dr = c.G.dx[r_];
  double rOut = Ctot[iRbnd - 1].G.x[x_];
  double ar = dr / (rOut * P.dth);
  double iS = iLbnd + 1;
  for (int ii = iRbnd - 1; ii > iLbnd; --ii) {
    double p = Ctot[ii].S.prim[PPP];
    iS = ii;
    if (p > 1.5 * P.eta) break;
  }
  double dist = i - iS;
  if (0 < dist and dist < 10) { ar *= 10; }
  double lfac = c.S.lfac();
  if (ar > P.split_AR * P.target_ar / pow(lfac, 3. / 2.)) return (split_);
  if (ar < P.merge_AR * P.target_ar / pow(lfac, 3. / 2.)) return (merge_);
  return (skip_);
}

// BM1D.cpp:322-332
void Cell::user_regridVal(double *res) {
  double r = G.x[r_];
  double dr = G.dx[r_];
  double lfac = S.lfac();
  *res = dr / (r * P.dth) * pow(lfac, 3. / 2.);
}

void FluidState::cons2prim_user(double *rho, double *p, double *uu) {
  UNUSED(rho);
  UNUSED(p);
  UNUSED(uu);
}

void Simu::dataDump() {}
void Simu::runInfo() {}
void Simu::evalEnd() {}
