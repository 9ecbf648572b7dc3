/*
 * Problem setup (an INITIAL module) for the 2D oracle build: a spherical
 * blast wave on a wedge of theta tracks, Blandford-McKee inside theta_jet and
 * cold ambient medium outside (a jet-like cap), with run-time parameters set
 * through ref_set_param.  TEST INFRASTRUCTURE.
 *
 * The hooks follow the reference's 2D problem module src/Initial/Tests/BM.cpp
 * (cited per function): the constants become variables, the theta extent and
 * the jet half-opening angle are parameters, and initialValues evaluates the
 * BM profile with `nbins` sub-samples per cell (BM.cpp uses 1000; 1 is the
 * one-point form of BM1D.cpp).
 */
#include "environment.h"
#include "grid.h"
#include "constants.h"
#include "simu.h"

#include <cstring>

namespace {
struct Jet2dParams {
  double n0 = 1.;            // CBM number density (cm^-3) -> rhoNorm = n0 mp
  double eta = 1.e-10;       // p / (rho c^2) of the ambient medium
  double Etot = 1.e53;       // erg (isotropic equivalent inside the cap)
  double n_ext = 1.;
  double lfac_shock2 = 2.e4; // Gamma_shock^2 (BM.cpp LORENTZ_ == 1 branch: 2 lfacstart^2)
  double Rscale = 1.e17;     // cm
  double k = 0.;
  double ncell = 400.;       // cells per track in r
  double ntrack = 16.;       // theta tracks
  double nmax = 800.;        // capacity per track (active cells)
  double ngst = 2.;
  double r_lo = 0.9;         // radial extent [r_lo, r_hi] x R_shock, uniform cells
  double r_hi = 1.1;
  double th_min = 0.;        // theta extent of the active tracks
  double th_max = 0.2;
  double th_jet = 0.1;       // BM profile for track centres below this angle
  double nbins = 1.;         // BM sub-samples per cell
  double split_DR = 5.;      // BM.cpp checkCellForRegrid ratios (lfac >= 2)
  double merge_DR = 0.3;
  double split_DR_slow = 20.;  // lfac < 2
  double merge_DR_slow = 1.2;
  double v_out = 1.05;       // outer ghost-interface velocity (BM.cpp userKinematics)
  double it_hold = 1000.;    // ... set to 0 once it > it_hold and the flow 10 cells in is at rest
};
Jet2dParams P;

double rhoNorm, lNorm, vNorm, pNorm;
double tstart, lfacShock2, RShock, rhoa, pa, ha, pf, lfacf, Df;

// BM.cpp:13-55 (LORENTZ_ == 1 branch)
void derive() {
  rhoNorm = P.n0 * mp_;
  lNorm = c_;
  vNorm = c_;
  pNorm = rhoNorm * vNorm * vNorm;
  lfacShock2 = P.lfac_shock2;
  tstart = pow(P.Etot * (17.) / (8. * PI * P.n_ext * mp_ * pow(c_, 5.) * lfacShock2), 1. / 3.);
  RShock = c_ * tstart * (1. - 1. / (1. + 2. * (4. - P.k) * lfacShock2));
  rhoa = P.n_ext * mp_ * pow(RShock / P.Rscale, -P.k);
  pa = rhoa * P.eta * c_ * c_;
  ha = c_ * c_ + pa * GAMMA_ / (GAMMA_ - 1.) / rhoa;
  pf = 2. / 3. * lfacShock2 * ha * rhoa;
  lfacf = sqrt(fmax(1., .5 * lfacShock2));
  Df = 2. * lfacShock2 * rhoa;
}
}  // namespace

extern "C" __attribute__((visibility("default"))) int ref_set_param(const char *name, double v) {
#define SETP(f) \
  if (!strcmp(name, #f)) { P.f = v; return 0; }
  SETP(n0) SETP(eta) SETP(Etot) SETP(n_ext) SETP(lfac_shock2) SETP(Rscale) SETP(k) SETP(ncell)
  SETP(ntrack) SETP(nmax) SETP(ngst) SETP(r_lo) SETP(r_hi) SETP(th_min) SETP(th_max) SETP(th_jet)
  SETP(nbins) SETP(split_DR) SETP(merge_DR) SETP(split_DR_slow) SETP(merge_DR_slow) SETP(v_out)
  SETP(it_hold)
#undef SETP
  return -1;
}

extern "C" __attribute__((visibility("default"))) void ref_jet2d_derived(double *out) {
  derive();
  out[0] = tstart;
  out[1] = RShock / lNorm;
  out[2] = lfacShock2;
  out[3] = rhoNorm;
  out[4] = pNorm;
  out[5] = lNorm;
  out[6] = vNorm;
}

// BM.cpp:83-93
void loadParams(s_par *par) {
  derive();
  par->tini = tstart;
  par->ncell[x_] = (int)P.ncell;
  par->ncell[y_] = (int)P.ntrack;
  par->nmax = (int)P.nmax;
  par->ngst = (int)P.ngst;
  normalizeConstants(rhoNorm, vNorm, lNorm);
}

// BM.cpp:95-126 with the radial extent [r_lo, r_hi] R_shock and theta in [th_min, th_max]
int Grid::initialGeometry() {
  double rmin = P.r_lo * RShock / lNorm;
  double rmax = P.r_hi * RShock / lNorm;
  double dr = (rmax - rmin) / ncell[x_];
  for (int j = 0; j < ncell[y_]; ++j) {
    for (int i = 0; i < ncell[x_]; ++i) {
      Cell *c = &Cinit[j][i];
      double r = rmin + (i + 0.5) * dr;
      double th = (double)P.th_min + (P.th_max - P.th_min) * (j + 0.5) / ncell[y_];
      double dth = (P.th_max - P.th_min) / ncell[y_];
      c->G.x[x_] = r;
      c->G.dx[x_] = dr;
      c->G.x[y_] = th;
      c->G.dx[y_] = dth;
      c->computeAllGeom();
    }
  }
  return 0;
}

// BM.cpp:128-195; tracks whose centre lies above th_jet hold the ambient medium only
int Grid::initialValues() {
  for (int j = 0; j < ncell[F1]; ++j) {
    for (int i = 0; i < ncell[MV]; ++i) {
      Cell *c = &Cinit[j][i];
      double r = c->G.x[x_];
      double dr = c->G.dx[x_];
      double th = c->G.x[y_];
      double r_denorm = r * lNorm;
      double dr_denorm = dr * lNorm;
      if (r_denorm > RShock || th > P.th_jet) {
        double rho = P.n_ext * mp_ * pow(r_denorm / P.Rscale, -P.k);
        c->S.prim[RHO] = rho / rhoNorm;
        c->S.prim[VV1] = 0;
        c->S.prim[VV2] = 0;
        c->S.prim[PPP] = P.eta * rho * c_ * c_ / pNorm;
        c->S.prim[TR1] = 1.;
      } else {
        int nbins = (int)P.nbins;
        double ddx = dr_denorm / nbins;
        double xl = r_denorm - dr_denorm / 2.;
        double xr = xl + ddx;
        double dV = 4. / 3. * PI * (pow(r_denorm + dr_denorm / 2., 3) - pow(r_denorm - dr_denorm / 2., 3));
        double rho = 0, v = 0, p = 0;
        for (int ix = 0; ix < nbins; ++ix) {
          double x = (xr + xl) / 2.;
          double ddV = 4. / 3. * PI * (xr * xr * xr - xl * xl * xl);
          double chi = (1. + 2. * (4. - P.k) * lfacShock2) * (1. - x / (c_ * tstart));
          double dp = pf * pow(chi, -(17. - 4. * P.k) / (12. - 3. * P.k));
          double dlfac = sqrt(lfacf * lfacf / chi + 1);
          double dD = Df * pow(chi, -(7. - 2. * P.k) / (4. - P.k));
          double drho = dD / dlfac;
          double dv = c_ * sqrt(1. - 1. / (dlfac * dlfac));
          rho += drho * ddV / dV;
          v += dv * ddV / dV;
          p += dp * ddV / dV;
          xl = xr;
          xr += ddx;
        }
        c->S.prim[RHO] = rho / rhoNorm;
        c->S.prim[VV1] = v / vNorm;
        c->S.prim[VV2] = 0;
        c->S.prim[PPP] = p / pNorm;
        c->S.prim[TR1] = 2.;
      }
    }
  }
  return 0;
}

// BM.cpp:198-218: outer ghost interfaces move at v_out until, after it_hold
// steps, the flow ten cells inside the outer edge of the first active track is
// at rest; the inner ghost interfaces keep VI * lambda*.
void Grid::userKinematics(int it, double t) {
  UNUSED(t);
  double vOut = P.v_out;
  int j = jLbnd + 1;
  int i = iRbnd[j] - 10;
  if (Ctot[j][i].S.prim[UU1] < 1.e-3 and it > P.it_hold) { vOut = 0.; }
  for (int jj = 0; jj < nde_nax[F1]; ++jj) {
    for (int n = 0; n < ngst; ++n) {
      int iR = ntrack[jj] - 2 - n;
      Itot[jj][iR].v = vOut;
    }
  }
}

void Cell::userSourceTerms(double dt) { UNUSED(dt); }

// BM.cpp:226-243: no boundary override
void Grid::userBoundaries(int it, double t) {
  UNUSED(it);
  UNUSED(t);
}

// BM.cpp:246-278: split / merge against the mean radial spacing of the first
// active track, with looser ratios where lfac < 2
int Grid::checkCellForRegrid(int j, int i) {
  Cell c = Ctot[j][i];
  double dr = c.G.dx[r_];
  int jtrk = jLbnd + 1;
  double rmin = Ctot[jtrk][iLbnd[jtrk] + 1].G.x[r_];
  double rmax = Ctot[jtrk][iRbnd[jtrk] - 1].G.x[r_];
  double delta_r = rmax - rmin;
  double target_dr = delta_r / nact[jtrk];
  double split_DR = P.split_DR;
  double merge_DR = P.merge_DR;
  if (c.S.lfac() < 2.) {
    split_DR = P.split_DR_slow;
    merge_DR = P.merge_DR_slow;
  }
  if (dr > split_DR * target_dr) return (split_);
  if (dr < merge_DR * target_dr) return (merge_);
  return (skip_);
}

// BM.cpp:281-290
void Cell::user_regridVal(double *res) {
  if (S.lfac() < 2.) { *res /= 4; }
}

void FluidState::cons2prim_user(double *rho, double *p, double *uu) {
  UNUSED(rho);
  UNUSED(p);
  UNUSED(uu);
}

void Simu::dataDump() {}
void Simu::runInfo() {}
void Simu::evalEnd() {}
