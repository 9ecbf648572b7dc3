// Device physics of the 2D (r, theta) moving-mesh step: spherical geometry,
// rel_sph hydro with both velocity components, shock detection and local
// synchrotron tracers (NUM_Q = 10, NUM_D = 2).
//
// Each function restates one member of the GAMMA reference compiled with
// NUM_D = 2 and keeps its floating-point operation order (built with
// -fmad=false), so the only differences to the CPU reference come from libm
// and from the pressure root finder.  Dimension 0 is r (the moving direction),
// dimension 1 is theta (F1).  The theta momentum is stored as S_theta * r
// (rel_sph.cpp:78): every conversion takes the radius it is made at.
#pragma once

#include "physics.cuh"

namespace gb {
namespace d2 {

constexpr int NQ = 10;
constexpr int MV = 0, F1 = 1;

// rel_sph with synchrotron tracers and shock detection, 2D
struct Cfg2 {
  static constexpr bool FAST = false;
  static constexpr bool FAST_RIEMANN = false;
  static constexpr bool FAST_ROOT = false;
  static constexpr bool CYL = false;
  static constexpr int NQ = 10;
  static constexpr bool SPH = true;
  static constexpr bool SHOCK = true;
  static constexpr bool SYNCH = true;
  static constexpr bool BM = false;
};

// FluidState::lfac (fluid.cpp:10-22)
GB_HD double lfac(const double *prim) {
  double u = 0.;
  u += prim[UU1] * prim[UU1];
  u += prim[UU2] * prim[UU2];
  u = sqrt(u);
  return sqrt(1 + u * u);
}

// FluidState::prim2cons (rel_sph.cpp:55-82) at radius r
GB_HD void prim2cons(const Phys &ph, const double *prim, double *cons, double r) {
  double rho = prim[RHO];
  double p = prim[PPP];
  double u = 0;
  double uu[2];
  for (int i = 0; i < 2; ++i) {
    uu[i] = prim[UU1 + i];
    u += uu[i] * uu[i];
  }
  u = sqrt(u);
  double lf = sqrt(1 + u * u);
  double gma = eos_gamma(ph, rho, p);
  double h = 1. + p * gma / (gma - 1.) / rho;
  double D = lf * rho;
  double tau = D * h * lf - p - D;
  cons[DEN] = D;
  cons[TAU] = tau;
  for (int i = 0; i < 2; ++i) cons[SS1 + i] = D * h * uu[i];
  cons[SS2] *= r;
#pragma unroll
  for (int t = TR1; t < NQ; ++t) cons[t] = prim[t] * D;
}

// FluidState::state2flux (rel_sph.cpp:85-113), the flux along dimension n only
GB_HD void state2flux(const double *prim, const double *cons, int n, double r, double *flux) {
  double p = prim[PPP];
  double u = 0;
  double uu[2];
  for (int i = 0; i < 2; ++i) {
    uu[i] = prim[UU1 + i];
    u += uu[i] * uu[i];
  }
  u = sqrt(u);
  double lf = sqrt(1 + u * u);
  double D = cons[DEN];
  double ss[2] = {cons[SS1], cons[SS2]};
  ss[1] = qdiv(ss[1], r);
  flux[DEN] = qdiv(D * uu[n], lf);
  for (int i = 0; i < 2; ++i) {
    if (i == n) flux[SS1 + i] = qdiv(ss[i] * uu[n], lf) + p;
    else flux[SS1 + i] = qdiv(ss[i] * uu[n], lf);
  }
  flux[SS2] *= r;
  flux[TAU] = ss[n] - qdiv(D * uu[n], lf);
#pragma unroll
  for (int t = TR1; t < NQ; ++t) flux[t] = qdiv(cons[t] * uu[n], lf);
}

// One side of a Riemann problem: the state, its flux along the interface
// normal, and the cached Lorentz factor.
struct St {
  double prim[NQ], cons[NQ], flux[NQ];
  double lfac;
};

// prim2cons + state2flux at radius r (what reconstructStates does for a
// reconstructed state; a cell state uses its own centre radius)
GB_HD void fill(const Phys &ph, St &S, int dim, double r) {
  prim2cons(ph, S.prim, S.cons, r);
  state2flux(S.prim, S.cons, dim, r, S.flux);
  S.lfac = lfac(S.prim);
}

struct Waves {
  double lL, lS, lR;
};

// Interface::wavespeedEstimates + computeLambda (rel_sph.cpp:322-394) along
// dim; d = r for the theta direction (the momentum is stored times r)
GB_HD Waves compute_lambda(const Phys &ph, const St &L, const St &R, int dim, double xr) {
  const double GL = ph.eos_ws ? eos_gamma(ph, L.prim[RHO], L.prim[PPP]) : ph.gamma_ad;
  const double GR = ph.eos_ws ? eos_gamma(ph, R.prim[RHO], R.prim[PPP]) : ph.gamma_ad;
  const int u = UU1 + dim, s = SS1 + dim;
  Waves w;
  double lfacL = L.lfac, lfacR = R.lfac;
  double vL = qdiv(L.prim[u], lfacL);
  double vR = qdiv(R.prim[u], lfacR);
  double cSL = sqrt(GL * L.prim[PPP] / (L.prim[RHO] + L.prim[PPP] * GL / (GL - 1.)));
  double cSR = sqrt(GR * R.prim[PPP] / (R.prim[RHO] + R.prim[PPP] * GR / (GR - 1.)));
  double sgSL = cSL * cSL / (lfacL * lfacL * (1. - cSL * cSL));
  double sgSR = cSR * cSR / (lfacR * lfacR * (1. - cSR * cSR));
  double l1, l2;
  l1 = (vR - sqrt(sgSR * (1. - vR * vR + sgSR))) / (1. + sgSR);
  l2 = (vL - sqrt(sgSL * (1. - vL * vL + sgSL))) / (1. + sgSL);
  w.lL = fmin(l1, l2);
  l1 = (vR + sqrt(sgSR * (1. - vR * vR + sgSR))) / (1. + sgSR);
  l2 = (vL + sqrt(sgSL * (1. - vL * vL + sgSL))) / (1. + sgSL);
  w.lR = fmax(l1, l2);

  const double d = dim == F1 ? xr : 1.;
  const double lL = w.lL, lR = w.lR;
  double mmL = qdiv(L.cons[s], d);
  double mmR = qdiv(R.cons[s], d);
  double pL = L.prim[PPP];
  double pR = R.prim[PPP];
  double EL = L.cons[TAU] + L.cons[DEN];
  double ER = R.cons[TAU] + R.cons[DEN];
  double AL = lL * EL - mmL;
  double AR = lR * ER - mmR;
  double BL = mmL * (lL - vL) - pL;
  double BR = mmR * (lR - vR) - pR;
  double FhllE = qdiv(lL * AR - lR * AL, lR - lL);
  double Ehll = (AR - AL) / (lR - lL);
  double Fhllm = (lL * BR - lR * BL) / (lR - lL);
  double mhll = qdiv(BR - BL, lR - lL);
  if (fabs(FhllE) == 0) {
    w.lS = qdiv(mhll, Ehll + Fhllm);
    return w;
  }
  // pow(x, 2.) of the C library is the correctly rounded square: x*x
  const double ef = Ehll + Fhllm;
  double delta = ef * ef - 4. * FhllE * mhll;
  w.lS = ((Ehll + Fhllm) - sqrt(delta)) / (2. * FhllE);
  return w;
}

// Interface::starState (rel_sph.cpp:397-450) along dim at radius xr
GB_HD void star_state(const St &Sin, double lbda, double lS, int dim, double xr, double *out) {
  const int u = UU1 + dim, s = SS1 + dim, so = SS1 + (1 - dim);
  double r = xr;
  double mm[2] = {Sin.cons[SS1], Sin.cons[SS2]};
  mm[1] = qdiv(mm[1], r);
  double lf = Sin.lfac;
  double v = qdiv(Sin.prim[u], lf);
  double m = mm[dim];
  double p = Sin.prim[PPP];
  double D = Sin.cons[DEN];
  double E = Sin.cons[TAU] + Sin.cons[DEN];
  double A = lbda * E - m;
  double B = m * (lbda - v) - p;
  double pS = (A * lS - B) / (1. - lbda * lS);
  double k = (lbda - v) / (lbda - lS);
  out[DEN] = D * k;
  out[s] = (m * (lbda - v) + pS - p) / (lbda - lS);
  out[so] = mm[so - SS1] * k;
  out[SS2] *= r;
  out[TAU] = (E * (lbda - v) + pS * lS - p * v) / (lbda - lS) - D * k;
#pragma unroll
  for (int t = TR1; t < NQ; ++t) out[t] = Sin.cons[t] * k;
}

// Interface::computeFlux (hllc.cpp:12-39): F - vU in the interface frame, times dA
GB_HD void hllc_flux(const St &L, const St &R, const Waves &w, double v, double dA, int dim, double xr,
                     double *flux) {
  if (v < w.lL) {
#pragma unroll
    for (int q = 0; q < NQ; ++q) flux[q] = L.flux[q] - v * L.cons[q];
  }
  if (w.lL <= v && v < w.lS) {
    double sc[NQ];
    star_state(L, w.lL, w.lS, dim, xr, sc);
#pragma unroll
    for (int q = 0; q < NQ; ++q) flux[q] = L.flux[q] + w.lL * (sc[q] - L.cons[q]) - v * sc[q];
  }
  if (w.lS <= v && v < w.lR) {
    double sc[NQ];
    star_state(R, w.lR, w.lS, dim, xr, sc);
#pragma unroll
    for (int q = 0; q < NQ; ++q) flux[q] = R.flux[q] + w.lR * (sc[q] - R.cons[q]) - v * sc[q];
  }
  if (w.lR <= v) {
#pragma unroll
    for (int q = 0; q < NQ; ++q) flux[q] = R.flux[q] - v * R.cons[q];
  }
#pragma unroll
  for (int q = 0; q < NQ; ++q) flux[q] *= dA;
}

// compute_Sd (radiation_sph.cpp:41-158) along dim, S1 upstream.  Returns false
// where the reference returns -1 before reaching the spectral index.
// What compute_Sd reads of one side along dim: pressure, density, the
// 4-velocity along dim (ux) and across it (ut), the Lorentz factor.
struct SdSide {
  double p, rho, ux, ut, lfac;
};

GB_HD SdSide sd_side(const St &S, int dim) {
  return SdSide{S.prim[PPP], S.prim[RHO], S.prim[UU1 + dim], S.prim[UU2 - dim], S.lfac};
}

GB_HD bool compute_Sd(const Phys &ph, const SdSide &S1, const SdSide &S2, bool reverse, double *Sd) {
  // with eos_ws, the upstream state's Gamma_eff throughout
  const double G = ph.eos_ws ? eos_gamma(ph, S1.rho, S1.p) : ph.gamma_ad;
  const int n_evals = 10;
  const double chi = 0.5;
  double p1 = S1.p;
  double p2 = S2.p;
  if (fabs(qdiv(p1 - p2, p1)) < 1.e-10 || p1 < p2) {
    *Sd = -1;
    return false;
  }
  double delta_p = p2 - p1;
  double dp = delta_p / (double)n_evals;
  double rho1 = S1.rho;
  double rho2 = S2.rho;
  double h1 = 1 + p1 * G / (G - 1.) / rho1;
  double h2 = 1 + p2 * G / (G - 1.) / rho2;
  double lfac2 = S2.lfac;
  double vx1 = qdiv(S1.ux, S1.lfac);
  double vx2 = qdiv(S2.ux, lfac2);
  if (reverse) {
    vx1 *= -1;
    vx2 *= -1;
  }
  double ut1 = S1.ut;
  double v12 = qdiv(vx1 - vx2, 1 - vx1 * vx2);
  double A1 = h1 * ut1;
  double I = 0;
  for (int ip = 0; ip < n_evals; ++ip) {
    double p = p1 + (ip + .5) * dp;
    double rho = rho1 * isentrope_pow(p / p1, 1. / G);
    double h = 1 + p * G / (G - 1.) / rho;
    double cs = sqrt(G * p / (rho + p * G / (G - 1.)));
    double dI = sqrt(h * h + A1 * A1 * (1. - cs * cs)) / ((h * h + A1 * A1) * rho * cs) * dp;
    I += dI;
  }
  double vSR = tanh(I);
  double rho22 = rho2 * rho2;
  double lfac22 = lfac2 * lfac2;
  double vx22 = vx2 * vx2;
  double g = G;
  double gm1 = (g - 1.);
  double gm12 = gm1 * gm1;
  double Da = 4. * g * p1 * ((g - 1) * p2 + p1) / (gm12 * (p1 - p2) * (p1 - p2));
  double Db = h2 * (p2 - p1) / rho2 - h2 * h2;
  double Dd = 1. - Da * Db;
  double h3 = (sqrt(Dd) - 1) * gm1 * (p1 - p2) / (2 * (gm1 * p2 + p1));
  double J232a = -g / gm1 * (p1 - p2);
  double J232b = h3 * (h3 - 1) / p1 - h2 * (h2 - 1) / p2;
  double J232 = J232a / J232b;
  double J23 = sqrt(J232);
  double Vsa = rho22 * lfac22 * vx2 + fabs(J23) * sqrt(J232 + rho22 * lfac22 * (1. - vx22));
  double Vsb = rho22 * lfac22 + J232;
  double Vs = Vsa / Vsb;
  double v2Sa = (p1 - p2) * (1. - vx2 * Vs);
  double v2Sb = (Vs - vx2) * (h2 * rho2 * lfac22 * (1. - vx22) + p1 - p2);
  double v2S = v2Sa / v2Sb;
  double vlim = vSR + chi * (v2S - vSR);
  *Sd = v12 - vlim;
  return true;  // spectral index: p_ (VARIABLE_PSPEC_ disabled)
}

// What the root search of cons2prim at radius r is given (rel_sph.cpp:215-250).
struct C2PInput2 {
  double D, E, ss[2], S2, S, pCand;
};

GB_HD C2PInput2 c2p_input(const double *cons, const double *prim, double r) {
  C2PInput2 in;
  in.D = cons[DEN];
  double tau = cons[TAU];
  in.E = in.D + tau;
  in.ss[0] = cons[SS1];
  in.ss[1] = qdiv(cons[SS2], r);
  double S2 = 0.;
  for (int d = 0; d < 2; ++d) S2 += in.ss[d] * in.ss[d];
  in.S2 = S2;
  in.S = sqrt(S2);
  in.pCand = fmax(1.e-13, prim[PPP]);
  return in;
}

// FluidState::cons2prim (rel_sph.cpp:213-320) at radius r: warm start from
// prim[PPP]; cons is rewritten by the closing prim2cons(r).  defer, OUTLINE:
// as in the 1D cons2prim (physics.cuh).
template <bool OUTLINE = false>
GB_HD void cons2prim(const Phys &ph, double *cons, double *prim, double r, C2PStats *st, bool defer = false) {
  const C2PInput2 in = c2p_input(cons, prim, r);
  double D = in.D;
  double E = in.E;
  double ss[2] = {in.ss[0], in.ss[1]};
  double S2 = in.S2;
  double S = in.S;
  double p = c2p_pressure<Cfg2, OUTLINE>(ph, D, S, S2, E, in.pCand, st, nullptr, defer);
  if (defer && st && st->deferred) return;
  double Ep2 = (E + p) * (E + p);
  double v2 = qdiv(S2, Ep2);
  double lf = 1. / sqrt(fabs(1. - v2));
  double rho = D / lf;
  double uu[2];
  if (fabs(S) == 0.) {
    uu[0] = uu[1] = 0;
  } else {
    double v = sqrt(1. - 1. / (lf * lf));
    for (int d = 0; d < 2; ++d) uu[d] = lf * v * qdiv(ss[d], S);
  }
  p = fmax(p, P_FLOOR);
  prim[PPP] = p;
  prim[RHO] = rho;
  prim[UU1] = uu[0];
  prim[UU2] = uu[1];
#pragma unroll
  for (int t = TR1; t < NQ; ++t) prim[t] = qdiv(cons[t], D);
  prim2cons(ph, prim, cons, r);
}

// ---------------------------------------------------------------------------
// Geometry (spherical.cpp:12-112): a cell is (r, dr) x (theta, dtheta).  Every
// cell of a track shares theta and dtheta, so the angular factors are
// evaluated once per track on the host (with the C library the reference uses)
// and the device only multiplies them in the reference's order.

struct TrackGeo {
  double th, dth;
  double cen_t;   // theta centroid (spherical.cpp:58-66)
  double sfac;    // fabs(sin(.5*dth)*sin(th))
  double s_lo;    // fabs(sin(th - dth/2))
  double s_mid;   // fabs(sin(th))
  double s_hi;    // fabs(sin(th + dth/2))
  double cos_th;  // cos(th)
};
constexpr int TG_WORDS = 8;

GB_HD TrackGeo track_geo(const double *tg) {
  TrackGeo t;
  t.th = tg[0];
  t.dth = tg[1];
  t.cen_t = tg[2];
  t.sfac = tg[3];
  t.s_lo = tg[4];
  t.s_mid = tg[5];
  t.s_hi = tg[6];
  t.cos_th = tg[7];
  return t;
}

// the host side of the per-track factors
inline void fill_track_geo(double th, double dth, double *tg) {
  double th1 = th - dth / 2.;
  double th2 = th + dth / 2.;
  tg[0] = th;
  tg[1] = dth;
  tg[2] = (th1 * cos(th1) - th2 * cos(th2) + fabs(sin(th2)) - fabs(sin(th1))) / (cos(th1) - cos(th2));
  tg[3] = fabs(sin(.5 * dth) * sin(th));
  tg[4] = fabs(sin(th - dth / 2.));
  tg[5] = fabs(sin(th));
  tg[6] = fabs(sin(th + dth / 2.));
  tg[7] = cos(th);
}

struct Geom {
  double r, dr;
  double dV, cen_r;
};

// computeAllGeom (cell.cpp:31-39 -> spherical.cpp: computedl, computedV, computeCentroid)
GB_HD Geom make_geom(double r, double dr, const TrackGeo &t) {
  Geom g;
  g.r = r;
  g.dr = dr;
  double r1 = r - dr / 2.;
  double r2 = r + dr / 2.;
  double rsq = r1 * r1 + r1 * r2 + r2 * r2;
  g.dV = 4. / 3. * PI_ * rsq * dr * t.sfac;
  double rr2 = r * r;
  double dr2 = dr * dr;
  g.cen_r = 3. * r * (rr2 + dr2) / (3 * rr2 + dr2);
  return g;
}

// Interface::computedA (spherical.cpp:81-112): a radial-direction interface at
// radius r of a track
GB_HD double dA_r(double r, const TrackGeo &t) { return 4. * PI_ * r * r * t.sfac; }

// ... and a theta-direction interface spanning dr about r, at a theta whose
// |sin| is s_abs
GB_HD double dA_t(double r, double dr, double s_abs) {
  double r1 = r - dr / 2.;
  double r2 = r + dr / 2.;
  double rsq = (r1 + r2) * dr;
  return PI_ * s_abs * rsq;
}

// Cell::sourceTerms, 2D (rel_sph.cpp:469-496)
GB_HD void source_terms(const Phys &ph, const double *prim, const Geom &G, const TrackGeo &t, double dt,
                        double *cons) {
  double rho = prim[RHO];
  double ut = prim[UU2];
  double p = prim[PPP];
  double gma = eos_gamma(ph, rho, p);
  double h = 1. + p * gma / (gma - 1.) / rho;
  double r = G.r;
  double dr = G.dr;
  double dV = G.dV;
  double r1 = r - dr / 2.;
  double r2 = r + dr / 2.;
  double rsq = (r2 * r2 + r1 * r1 + r2 * r1) / 3.;
  cons[SS1] += (rho * h * ut * ut + 2. * p) * (r / rsq) * dV * dt;
  cons[SS2] += p * t.cos_th / t.s_mid * dV * dt;
}

// ---------------------------------------------------------------------------
// Local synchrotron tracers (radiation_sph.cpp:196-300) with the 2D Lorentz factor

GB_HD double gammae2trac(double gme, const double *prim) {
  double lf = lfac(prim);
  double rho = prim[RHO];
  if (gme != 0.) return (lf * pow(rho, 4. / 3.) / gme);
  return 0;
}

// Cell::radiation_injectParticles
GB_HD void inject_particles(const Phys &ph, const SynchConst &sc, double *prim, bool shocked, double pspec) {
  double lf = lfac(prim);
  double rho = prim[RHO];
  if (shocked) {
    if (pspec > prim[PSN] || isnan(prim[PSN])) prim[PSN] = pspec;
    prim[GMX] = gammae2trac(GAMMA_MAX_INIT, prim) / (lf * rho);
    prim[GMN] = gammae2trac(gamma_min_init<Cfg2>(ph, sc, prim), prim) / (lf * rho);
  }
  if (isnan(prim[GMX]) || isnan(prim[GMN])) {  // lim only where it is used
    const double lim = lf * pow(rho, 4. / 3.) / (lf * rho);
    if (isnan(prim[GMX])) prim[GMX] = lim;
    if (isnan(prim[GMN])) prim[GMN] = lim;
  }
}

}  // namespace d2
}  // namespace gb
