/*
 * CPU restatement of GAMMA's 1D moving-mesh step -- the oracle.  TEST
 * INFRASTRUCTURE; see gamma_oracle.h.
 *
 * Expressions keep the reference's operation order (and its quirks, each noted
 * where it occurs) so that, built like the reference in oracle/_ref (no FMA
 * contraction), the two agree bit for bit.  File:line citations are to the
 * reference's src/ tree.
 */
#include "gamma_oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "brent.h"

/* src/environment.h:33-36, 70-82 */
enum { RHO = 0, PPP = 1, UU1 = 2, UU2 = 3 };
enum { DEN = 0, TAU = 1, SS1 = 2, SS2 = 3 };
enum { TR1 = 4, GMN = 6, GMX = 7, GMD = 8, PSN = 9 };
enum { SKIP = 0, MERGE = 1, SPLIT = 2 };

/* src/constants.h:6-28 */
#define P_FLOOR_ 1.e-10
#define PI M_PI
#define mp_ 1.6726219e-24
#define me_ 9.1093835e-28
#define c_ 2.99792458e10
#define alpha_ 1.29251816e-09
#define p_ 2.22
#define eps_e_ 0.1
#define eps_B_ 0.01
#define zeta_ 1.
#define GAMMA_MAX_INIT_ (1.e8)
#define DETECT_SHOCK_THRESHOLD_ 0.01

typedef struct {
  double prim[OC_NQ_MAX], cons[OC_NQ_MAX], flux[OC_NQ_MAX];
} fstate;

typedef struct {
  double dV, x, dx, dl, cen;
} geom;

typedef struct {
  double dt_loc;
  fstate S, S0;
  geom G, G0;
  double fluxL[OC_NQ_MAX], fluxR[OC_NQ_MAX];
  int isShocked;
  double Sd, pspec;
} cell;

typedef struct {
  double x, x0, v, v0, lfac, dA;
  fstate S, SL, SR;
  double lL, lS, lR;
  double flux[OC_NQ_MAX];
} iface;

struct oc_sim {
  oc_config c;
  int nq, ntr;
  int sph;  /* rel_sph hydro */
  int cap;
  cell *C;
  iface *I;
  int ntrack, nact, iLbnd, iRbnd, ngst;
  double t, dt;
  long it;
  int err;
  /* BM1D derived quantities (BM1D.cpp:28-65) and normalised constants (constants.cpp:12-20) */
  double rhoNorm, lNorm, vNorm, pNorm, tstart, lfacShock2, RShock, rhoa, pa, ha, pf, lfacf, Df;
  double Nalpha, Nmp, Nme;
};

/* ------------------------------------------------------------------------- */
/* records: FluidState ctor (rel_sph.cpp:19-32), Cell ctor (cell.cpp:4-26),  */
/* Interface ctor (interface.cpp:10-17)                                      */

static void fstate_init(fstate *S) {
  memset(S, 0, sizeof(*S));
  S->prim[RHO] = 1.;
  S->prim[PPP] = 1.;
}

static void cell_init(cell *c) {
  memset(c, 0, sizeof(*c));
  fstate_init(&c->S);
  fstate_init(&c->S0);
  c->dt_loc = 1.e15;
  c->isShocked = 0;
  c->Sd = -1.;
  c->pspec = 0;
}

static void iface_init(iface *I) {
  memset(I, 0, sizeof(*I));
  fstate_init(&I->S);
  fstate_init(&I->SL);
  fstate_init(&I->SR);
  I->lL = 0.;
  I->lS = -1.;
  I->lR = 0.;
}

/* ------------------------------------------------------------------------- */
/* EOS and state (fluid.cpp:10-22, rel_sph.cpp:37-113, rel_cart.cpp:37-95)    */

static double st_lfac(const fstate *S) {
  double u = 0;
  double uu = S->prim[UU1];
  u += uu * uu;
  u = sqrt(u);
  return sqrt(1 + u * u);
}

/* FluidState::gamma (rel_sph.cpp:37-52) */
static double eos_gamma(const oc_sim *s, double rho, double p) {
  const double G = s->c.gamma_ad;
  if (s->c.eos == OC_EOS_IDEAL) return G;
  double a = p / rho / (G - 1.);
  double e_ratio = a + sqrt(a * a + 1.);
  return G - (G - 1.) / 2. * (1. - 1. / (e_ratio * e_ratio));
}

static double st_gamma(const oc_sim *s, const fstate *S) {
  return s->sph ? eos_gamma(s, S->prim[RHO], S->prim[PPP]) : s->c.gamma_ad;
}

/* prim2cons (rel_sph.cpp:55-82; rel_cart.cpp:37-64 has no r factor) */
static void prim2cons(const oc_sim *s, fstate *S, double r) {
  double rho = S->prim[RHO];
  double p = S->prim[PPP];
  double u = 0;
  double uu = S->prim[UU1];
  u += uu * uu;
  u = sqrt(u);
  double lfac = sqrt(1 + u * u);
  double gma = st_gamma(s, S);
  double h = 1. + p * gma / (gma - 1.) / rho;
  double D = lfac * rho;
  double tau = D * h * lfac - p - D;
  double ss = D * h * uu;
  S->cons[DEN] = D;
  S->cons[TAU] = tau;
  S->cons[SS1] = ss;
  if (s->sph) S->cons[SS2] *= r;
  for (int t = 0; t < s->ntr; ++t) S->cons[TR1 + t] = S->prim[TR1 + t] * D;
}

/* state2flux (rel_sph.cpp:85-113; rel_cart.cpp:67-95).  In 1D the reference
 * also divides ss[t_] by r, one past the end of its one-element array; the
 * value is never read back. */
static void state2flux(const oc_sim *s, fstate *S, double r) {
  double p = S->prim[PPP];
  double u = 0;
  double uu = S->prim[UU1];
  u += uu * uu;
  u = sqrt(u);
  double lfac = sqrt(1 + u * u);
  double D = S->cons[DEN];
  double ss = S->cons[SS1];
  S->flux[DEN] = D * uu / lfac;
  S->flux[SS1] = ss * uu / lfac + p;
  if (s->sph) S->flux[SS2] *= r;
  S->flux[TAU] = ss - D * uu / lfac;
  for (int t = 0; t < s->ntr; ++t) S->flux[TR1 + t] = S->cons[TR1 + t] * uu / lfac;
}

typedef struct {
  const oc_sim *s;
  double D, S, E;
} fparams;

/* f(p) whose root is the pressure (rel_sph.cpp:191-210, rel_cart.cpp:108-123) */
static double c2p_f(double p, void *vp) {
  const fparams *par = (const fparams *)vp;
  double D = par->D, S = par->S, E = par->E;
  if (par->s->sph) {
    double lfac = 1. / sqrt(fabs(1. - (S * S) / ((E + p) * (E + p))));
    double gma = eos_gamma(par->s, D / lfac, p);
    return (E + p - D * lfac - (gma * p * lfac * lfac) / (gma - 1.));
  } else {
    double gamma = par->s->c.gamma_ad;
    double lfac = 1. / sqrt(1. - (S * S) / ((E + p) * (E + p)));
    return (E + p - D * lfac - (gamma * p * lfac * lfac) / (gamma - 1.));
  }
}

/* FluidState::cons2prim (rel_sph.cpp:213-320; rel_cart.cpp:125-229: guess
 * prim[PPP] without the 1e-13 lower bound and no pressure floor).  Returns the
 * number of root-finder iterations. */
static int cons2prim(const oc_sim *s, fstate *St, double r, double pin) {
  int iter = 0;
  const int max_iter = 1000;
  double res = 0;
  double D = St->cons[DEN];
  double tau = St->cons[TAU];
  double E = D + tau;
  double ss = St->cons[SS1];
  double S2 = 0.;
  S2 += ss * ss;
  double S = sqrt(S2);
  fparams params = {s, D, S, E};

  double pCand;
  if (pin != 0) pCand = pin;
  else pCand = s->sph ? fmax(1.e-13, St->prim[PPP]) : St->prim[PPP];

  double f_init = c2p_f(pCand, &params);
  if (fabs(f_init) > 0.) {
    double p_lo, p_hi;
    p_lo = fmax(0., (1. + 1e-13) * S - E);
    int find_p = 1;
    if (c2p_f(p_lo, &params) < 0) find_p = 0;
    if (f_init < 0) {
      p_hi = 1. * pCand;
    } else {
      p_hi = pCand;
      while (c2p_f(p_hi, &params) > 0) p_hi *= 10;
    }
    if (p_hi < p_lo) find_p = 0;
    if (find_p) {
      oracle_brent b;
      if (oracle_brent_set(&b, c2p_f, &params, p_lo, p_hi) != 0) abort(); /* GSL aborts too */
      int cont;
      do {
        iter++;
        oracle_brent_iterate(&b);
        res = b.b;
        p_lo = b.lower;
        p_hi = b.upper;
        cont = oracle_brent_continue(p_lo, p_hi, 0., s->c.c2p_epsrel);
      } while (cont && iter < max_iter);
      pCand = res;
    }
  }

  double p = pCand;
  double Ep2 = (E + p) * (E + p);
  double v2 = S2 / Ep2;
  double lfac = 1. / sqrt(fabs(1. - v2));
  double rho = D / lfac;
  double uu;
  if (fabs(S) == 0.) {
    uu = 0;
  } else {
    double v = sqrt(1. - 1. / (lfac * lfac));
    uu = lfac * v * (ss / S);
  }
  /* cons2prim_user: no-op for the BM1D and tube problems */
  if (s->sph) p = fmax(p, P_FLOOR_);
  St->prim[PPP] = p;
  St->prim[RHO] = rho;
  St->prim[UU1] = uu;
  for (int t = 0; t < s->ntr; ++t) St->prim[TR1 + t] = St->cons[TR1 + t] / D;
  prim2cons(s, St, r);
  return iter;
}

/* ------------------------------------------------------------------------- */
/* Riemann problem at a moving interface                                      */

/* Interface::wavespeedEstimates (rel_sph.cpp:322-350, identical in rel_cart) */
static void wavespeeds(const oc_sim *s, iface *I) {
  const int ws = s->c.eos_wavespeeds && s->sph;
  const double GL = ws ? eos_gamma(s, I->SL.prim[RHO], I->SL.prim[PPP]) : s->c.gamma_ad;
  const double GR = ws ? eos_gamma(s, I->SR.prim[RHO], I->SR.prim[PPP]) : s->c.gamma_ad;
  double lfacL = st_lfac(&I->SL);
  double lfacR = st_lfac(&I->SR);
  double vL = I->SL.prim[UU1] / lfacL;
  double vR = I->SR.prim[UU1] / lfacR;
  double cSL = sqrt(GL * I->SL.prim[PPP] / (I->SL.prim[RHO] + I->SL.prim[PPP] * GL / (GL - 1.)));
  double cSR = sqrt(GR * I->SR.prim[PPP] / (I->SR.prim[RHO] + I->SR.prim[PPP] * GR / (GR - 1.)));
  double sgSL = cSL * cSL / (lfacL * lfacL * (1. - cSL * cSL));
  double sgSR = cSR * cSR / (lfacR * lfacR * (1. - cSR * cSR));
  double l1, l2;
  l1 = (vR - sqrt(sgSR * (1. - vR * vR + sgSR))) / (1. + sgSR);
  l2 = (vL - sqrt(sgSL * (1. - vL * vL + sgSL))) / (1. + sgSL);
  I->lL = fmin(l1, l2);
  l1 = (vR + sqrt(sgSR * (1. - vR * vR + sgSR))) / (1. + sgSR);
  l2 = (vL + sqrt(sgSL * (1. - vL * vL + sgSL))) / (1. + sgSL);
  I->lR = fmax(l1, l2);
}

/* Interface::computeLambda (rel_sph.cpp:352-394; rel_cart.cpp:260-302 tests |FhllE| < 1e-15) */
static void compute_lambda(const oc_sim *s, iface *I) {
  wavespeeds(s, I);
  const double d = 1.;
  double lfacL = st_lfac(&I->SL);
  double lfacR = st_lfac(&I->SR);
  double vL = I->SL.prim[UU1] / lfacL;
  double vR = I->SR.prim[UU1] / lfacR;
  double mmL = s->sph ? I->SL.cons[SS1] / d : I->SL.cons[SS1];
  double mmR = s->sph ? I->SR.cons[SS1] / d : I->SR.cons[SS1];
  double pL = I->SL.prim[PPP];
  double pR = I->SR.prim[PPP];
  double EL = I->SL.cons[TAU] + I->SL.cons[DEN];
  double ER = I->SR.cons[TAU] + I->SR.cons[DEN];
  double lL = I->lL, lR = I->lR;
  double AL = lL * EL - mmL;
  double AR = lR * ER - mmR;
  double BL = mmL * (lL - vL) - pL;
  double BR = mmR * (lR - vR) - pR;
  double FhllE = (lL * AR - lR * AL) / (lR - lL);
  double Ehll = (AR - AL) / (lR - lL);
  double Fhllm = (lL * BR - lR * BL) / (lR - lL);
  double mhll = (BR - BL) / (lR - lL);
  int linear = s->sph ? (fabs(FhllE) == 0) : (fabs(FhllE) < 1.e-15);
  if (linear) {
    I->lS = mhll / (Ehll + Fhllm);
    return;
  }
  double delta = pow(Ehll + Fhllm, 2.) - 4. * FhllE * mhll;
  I->lS = ((Ehll + Fhllm) - sqrt(delta)) / (2. * FhllE);
}

/* Interface::starState (rel_sph.cpp:397-450; rel_cart.cpp:305-355) */
static void star_state(const oc_sim *s, const iface *I, const fstate *Sin, double lbda, fstate *Sout) {
  double r = I->x;
  double m = Sin->cons[SS1];
  double lfac = st_lfac(Sin);
  double v = Sin->prim[UU1] / lfac;
  double p = Sin->prim[PPP];
  double D = Sin->cons[DEN];
  double E = Sin->cons[TAU] + Sin->cons[DEN];
  double lS = I->lS;
  double A = lbda * E - m;
  double B = m * (lbda - v) - p;
  fstate_init(Sout);
  double pS = (A * lS - B) / (1. - lbda * lS);
  double k = (lbda - v) / (lbda - lS);
  Sout->cons[DEN] = D * k;
  Sout->cons[SS1] = (m * (lbda - v) + pS - p) / (lbda - lS);
  if (s->sph) Sout->cons[SS2] *= r;
  Sout->cons[TAU] = (E * (lbda - v) + pS * lS - p * v) / (lbda - lS) - D * k;
  for (int t = 0; t < s->ntr; ++t) Sout->cons[TR1 + t] = Sin->cons[TR1 + t] * k;
}

/* Interface::computeFlux (hllc.cpp:12-39).  The four tests are separate ifs in
 * the reference and are kept so. */
static void compute_flux(const oc_sim *s, iface *I) {
  const int nq = s->nq;
  const double v = I->v;
  if (v < I->lL) {
    I->S = I->SL;
    for (int q = 0; q < nq; ++q) I->flux[q] = I->S.flux[q] - v * I->S.cons[q];
  }
  if (I->lL <= v && v < I->lS) {
    star_state(s, I, &I->SL, I->lL, &I->S);
    for (int q = 0; q < nq; ++q)
      I->flux[q] = I->SL.flux[q] + I->lL * (I->S.cons[q] - I->SL.cons[q]) - v * I->S.cons[q];
  }
  if (I->lS <= v && v < I->lR) {
    star_state(s, I, &I->SR, I->lR, &I->S);
    for (int q = 0; q < nq; ++q)
      I->flux[q] = I->SR.flux[q] + I->lR * (I->S.cons[q] - I->SR.cons[q]) - v * I->S.cons[q];
  }
  if (I->lR <= v) {
    I->S = I->SR;
    for (int q = 0; q < nq; ++q) I->flux[q] = I->S.flux[q] - v * I->S.cons[q];
  }
  for (int q = 0; q < nq; ++q) I->flux[q] *= I->dA;
}

/* ------------------------------------------------------------------------- */
/* shock detector (radiation_sph.cpp:37-189)                                  */

/* compute_Sd (radiation_sph.cpp:41-158), forward direction in 1D.  Returns 0
 * and leaves *pspec untouched when the reference returns early (its pspec is
 * then an uninitialised local). */
static int compute_Sd(const oc_sim *s, const fstate *S1, const fstate *S2, double *Sd_out,
                      double *pspec) {
  /* with eos_wavespeeds, the upstream state's Gamma_eff throughout */
  const double G = (s->c.eos_wavespeeds && s->sph) ? eos_gamma(s, S1->prim[RHO], S1->prim[PPP]) : s->c.gamma_ad;
  const int n_evals = 10;
  const double chi = 0.5;
  double p1 = S1->prim[PPP];
  double p2 = S2->prim[PPP];
  if (fabs((p1 - p2) / p1) < 1.e-10) { *Sd_out = -1; return 0; }
  if (p1 < p2) { *Sd_out = -1; return 0; }
  double delta_p = p2 - p1;
  double dp = delta_p / (double)n_evals;
  double rho1 = S1->prim[RHO];
  double rho2 = S2->prim[RHO];
  double h1 = 1 + p1 * G / (G - 1.) / rho1;
  double h2 = 1 + p2 * G / (G - 1.) / rho2;
  double lfac2 = st_lfac(S2);
  double lfac1 = st_lfac(S1);
  double vx1 = S1->prim[UU1] / lfac1;
  double vx2 = S2->prim[UU1] / lfac2;
  double ut1 = 0;
  double v12 = (vx1 - vx2) / (1 - vx1 * vx2);
  double A1 = h1 * ut1;
  double I = 0;
  for (int ip = 0; ip < n_evals; ++ip) {
    double p = p1 + (ip + .5) * dp;
    double rho = rho1 * pow(p / p1, 1. / G);
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
  double D = 1. - Da * Db;
  double h3 = (sqrt(D) - 1) * gm1 * (p1 - p2) / (2 * (gm1 * p2 + p1));
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
  *Sd_out = v12 - vlim;
  *pspec = p_; /* spectral_p with VARIABLE_PSPEC_ disabled (radiation_sph.cpp:18-35) */
  return 1;
}

/* Interface::measureShock, moving direction: forward shocks only (radiation_sph.cpp:160-175) */
static void measure_shock(const oc_sim *s, const iface *I, cell *cL) {
  double Sd, pspec = 0;
  int have_pspec = compute_Sd(s, &I->SL, &I->SR, &Sd, &pspec);
  cL->Sd = fmax(cL->Sd, Sd);
  if (have_pspec && pspec > cL->pspec) cL->pspec = pspec;
}

/* ------------------------------------------------------------------------- */
/* local synchrotron tracers (radiation_sph.cpp:194-300)                      */

static double gammae2trac(double gme, const fstate *S) {
  double lfac = st_lfac(S);
  double rho = S->prim[RHO];
  if (gme != 0.) return (lfac * pow(rho, 4. / 3.) / gme);
  else return (0);
}

static double gamma_min_init(const oc_sim *s, const fstate *S) {
  double rho = S->prim[RHO];
  double p = S->prim[PPP];
  double psyn = S->prim[PSN];
  double gma = st_gamma(s, S);
  double h = 1. + p * gma / (gma - 1.) / rho;
  double eps = rho * (h - 1.) / gma;
  double ee = eps_e_ * eps;
  double ne = zeta_ * rho / s->Nmp;
  double lfac_av = ee / (ne * s->Nme);
  return (psyn - 2.) / (psyn - 1.) * lfac_av;
}

static void init_gammas(cell *c) {
  fstate *S = &c->S;
  double lfac = st_lfac(S);
  double rho = S->prim[RHO];
  double lim = lfac * pow(rho, 4. / 3.);
  if (S->prim[GMX] > lim / (lfac * rho) || S->prim[GMX] <= 0.) {
    S->prim[GMX] = lim / (lfac * rho);
    S->cons[GMX] = lim;
  }
  if (S->prim[GMN] > lim / (lfac * rho) || S->prim[GMN] <= 0.) {
    S->prim[GMN] = lim / (lfac * rho);
    S->cons[GMN] = lim;
  }
}

static void inject_particles(const oc_sim *s, cell *c) {
  fstate *S = &c->S;
  double lfac = st_lfac(S);
  double rho = S->prim[RHO];
  double lim = lfac * pow(rho, 4. / 3.) / (lfac * rho);
  if (c->isShocked) {
    if (c->pspec > S->prim[PSN] || isnan(S->prim[PSN])) S->prim[PSN] = c->pspec;
    S->prim[GMX] = gammae2trac(GAMMA_MAX_INIT_, S) / (lfac * rho);
    S->prim[GMN] = gammae2trac(gamma_min_init(s, S), S) / (lfac * rho);
  }
  if (isnan(S->prim[GMX])) S->prim[GMX] = lim;
  if (isnan(S->prim[GMN])) S->prim[GMN] = lim;
}

static void radiative_sources(const oc_sim *s, cell *c, double dt) {
  fstate *S = &c->S;
  double rho = S->prim[RHO];
  double p = S->prim[PPP];
  double gma = st_gamma(s, S);
  double h = 1 + p * gma / (gma - 1.) / rho;
  double eps = rho * (h - 1.) / gma;
  double eB = eps_B_ * eps;
  double B = sqrt(8. * PI * eB);
  double dgma = s->Nalpha * pow(rho, 4. / 3.) * B * B * c->G.dV * dt;
  S->cons[GMX] += dgma;
  S->cons[GMN] += dgma;
}

/* ------------------------------------------------------------------------- */
/* geometry (spherical1D.cpp:12-57,60-76; cartesian.cpp:11-43)                */

static void all_geom(const oc_sim *s, geom *g) {
  if (s->c.geometry == OC_GEOM_SPHERICAL1D) {
    double r = g->x, dr = g->dx;
    g->dl = dr;
    g->dV = 4. * PI * r * r * dr;
    double r2 = r * r;
    double dr2 = dr * dr;
    g->cen = g->x;
    g->cen = 3. * r * (r2 + dr2) / (3 * r2 + dr2);
  } else {
    g->dl = g->dx;
    g->dV = 1.;
    g->dV *= g->dx;
    g->cen = g->x;
  }
}

static void iface_dA(const oc_sim *s, iface *I) {
  if (s->c.geometry == OC_GEOM_SPHERICAL1D) {
    double r = I->x;
    I->dA = 4. * PI * r * r;
  } else {
    I->dA = 1;
  }
}

/* Cell::move (spherical1D.cpp:51-57) */
static void cell_move(const oc_sim *s, cell *c, double xL, double xR) {
  c->G.x = (xR + xL) / 2.;
  c->G.dx = (xR - xL);
  all_geom(s, &c->G);
}

/* ------------------------------------------------------------------------- */
/* cell updates (cell.cpp:47-127, rel_sph.cpp:452-466)                        */

static int update_dt(cell *c, const iface *IL, const iface *IR) {
  double a = c->G.dl;
  double l, v, dt_candL, dt_candR;
  l = IL->lR;
  v = IR->v;
  if (l > v) dt_candL = a / (l - v);
  else dt_candL = 1.e15;
  l = IR->lL;
  v = IL->v;
  if (l < v) dt_candR = a / (v - l);
  else dt_candR = 1.e15;
  double dt_cand = fmin(dt_candL, dt_candR);
  if (dt_cand < 0) return 30; /* the reference prints and exit(30)s */
  c->dt_loc = fmin(c->dt_loc, dt_cand);
  return 0;
}

static void cell_update(const oc_sim *s, cell *c, double dt, double xL, double xR) {
  const int nq = s->nq;
  for (int q = 0; q < nq; ++q) c->S.cons[q] *= c->G.dV;
  for (int q = 0; q < nq; ++q) c->S.cons[q] += (c->fluxL[q] - c->fluxR[q]) * dt;
  if (s->sph) { /* Cell::sourceTerms lives in the hydro module; rel_cart's is empty */
    double p = c->S.prim[PPP];
    double r = c->G.x;
    double dr = c->G.dx;
    double dV = c->G.dV;
    double r1 = r - dr / 2.;
    double r2 = r + dr / 2.;
    double rsq = (r2 * r2 + r1 * r1 + r2 * r1) / 3.;
    c->S.cons[SS1] += (2. * p) * (r / rsq) * dV * dt;
  }
  /* userSourceTerms: none for the BM1D and tube problems */
  if (s->c.local_synchrotron) radiative_sources(s, c, dt);
  cell_move(s, c, xL, xR);
  for (int q = 0; q < nq; ++q) c->S.cons[q] /= c->G.dV;
  cons2prim(s, &c->S, c->G.cen, 0);
}

/* ------------------------------------------------------------------------- */
/* problem hooks: BM1D (BM1D.cpp:62-332, parameterised), tube (1DST.cpp)      */

static void bm_derive(oc_sim *s) {
  const oc_config *P = &s->c;
  double rho0 = P->n0 * mp_;
  s->rhoNorm = rho0;
  s->lNorm = c_;
  s->vNorm = c_;
  s->pNorm = s->rhoNorm * s->vNorm * s->vNorm;
  if (P->lorentz_mode != 0.) {
    s->lfacShock2 = P->lfac_shock2;
    s->tstart = pow(P->Etot * (17.) / (8. * PI * P->n_ext * mp_ * pow(c_, 5.) * s->lfacShock2), 1. / 3.);
  } else {
    s->tstart = P->tinit;
    s->lfacShock2 = P->Etot * (17. - 4. * P->k) / (8. * PI * P->n_ext * mp_ * pow(s->tstart, 3) * pow(c_, 5));
  }
  const double G = P->gamma_ad;
  s->RShock = c_ * s->tstart * (1. - 1. / (1. + 2. * (4. - P->k) * s->lfacShock2));
  s->rhoa = P->n_ext * mp_ * pow(s->RShock / P->Rscale, -P->k);
  s->pa = s->rhoa * P->eta * c_ * c_;
  s->ha = c_ * c_ + s->pa * G / (G - 1.) / s->rhoa;
  s->pf = 2. / 3. * s->lfacShock2 * s->ha * s->rhoa;
  s->lfacf = sqrt(fmax(1., .5 * s->lfacShock2));
  s->Df = 2. * s->lfacShock2 * s->rhoa;
  /* normalizeConstants (constants.cpp:12-20) */
  s->Nalpha = alpha_ / (1. / (s->rhoNorm * s->vNorm * s->lNorm));
  s->Nmp = mp_ / (s->rhoNorm * pow(s->lNorm, 3));
  s->Nme = me_ / (s->rhoNorm * pow(s->lNorm, 3));
}

/* calcBM (BM1D.cpp:62-86) */
static void calc_bm(const oc_sim *s, double r, double t, double *rho, double *u, double *p) {
  const oc_config *P = &s->c;
  const double G = P->gamma_ad;
  double lfacShock2 = P->Etot * (17. - 4. * P->k) / (8. * PI * P->n_ext * mp_ * pow(t, 3) * pow(c_, 5));
  double RShock = c_ * t * (1. - 1. / (1. + 2. * (4. - P->k) * lfacShock2));
  double rhoa = P->n_ext * mp_ * pow(RShock / P->Rscale, -P->k);
  double pa = rhoa * P->eta * c_ * c_;
  double ha = c_ * c_ + pa * G / (G - 1.) / rhoa;
  double pf = 2. / 3. * lfacShock2 * ha * rhoa;
  double lfacf = sqrt(fmax(1., .5 * lfacShock2));
  double Df = 2. * lfacShock2 * rhoa;
  double chi = (1. + 2. * (4. - P->k) * lfacShock2) * (1. - r / (c_ * t));
  *p = pf * pow(chi, -(17. - 4. * P->k) / (12. - 3. * P->k)) / s->pNorm;
  double lfac = sqrt(lfacf * lfacf / chi + 1);
  double D = Df * pow(chi, -(7. - 2. * P->k) / (4. - P->k));
  *rho = D / lfac / s->rhoNorm;
  *u = c_ * sqrt(1. - 1. / (lfac * lfac)) * lfac / s->vNorm;
}

static void initial_conditions(oc_sim *s) {
  const oc_config *P = &s->c;
  const int n = P->ncell;
  cell *Cinit = s->C + s->ngst;
  if (P->problem == OC_PROBLEM_BM1D) {
    if (P->grid_log == 0.) { /* BM1D.cpp:100-116 */
      double rmin = s->RShock * (1. - 50. / s->lfacShock2);
      double rmax = s->RShock * (1. + 50. / s->lfacShock2);
      rmin /= s->lNorm;
      rmax /= s->lNorm;
      double dr = (rmax - rmin) / n;
      for (int i = 0; i < n; ++i) {
        cell *c = &Cinit[i];
        double r = rmin + (i + 0.5) * dr;
        c->G.x = r;
        c->G.dx = dr;
        all_geom(s, &c->G);
      }
    } else {
      double rmin = P->r_lo * s->RShock / s->lNorm;
      double rmax = P->r_hi * s->RShock / s->lNorm;
      double lr = log(rmax / rmin);
      for (int i = 0; i < n; ++i) {
        cell *c = &Cinit[i];
        double rl = rmin * exp(lr * i / n);
        double rr = rmin * exp(lr * (i + 1) / n);
        c->G.x = 0.5 * (rl + rr);
        c->G.dx = rr - rl;
        all_geom(s, &c->G);
      }
    }
    for (int i = 0; i < n; ++i) { /* BM1D.cpp:118-185, one bin */
      cell *c = &Cinit[i];
      double r = c->G.x;
      double dr = c->G.dx;
      double r_denorm = r * s->lNorm;
      double dr_denorm = dr * s->lNorm;
      if (r_denorm > s->RShock) {
        double rho = P->n_ext * mp_ * pow(r_denorm / P->Rscale, -P->k);
        c->S.prim[RHO] = rho / s->rhoNorm;
        c->S.prim[UU1] = 0;
        c->S.prim[PPP] = P->eta * rho * c_ * c_ / s->pNorm;
        c->S.prim[TR1] = 1.;
      } else {
        double xl = r_denorm - dr_denorm / 2.;
        double xr = xl + dr_denorm;
        double dV = 4. / 3. * PI * (pow(r_denorm + dr_denorm / 2., 3) - pow(r_denorm - dr_denorm / 2., 3));
        double x = (xr + xl) / 2.;
        double ddV = 4. / 3. * PI * (xr * xr * xr - xl * xl * xl);
        double chi = (1. + 2. * (4. - P->k) * s->lfacShock2) * (1. - x / (c_ * s->tstart));
        double dp = s->pf * pow(chi, -(17. - 4. * P->k) / (12. - 3. * P->k));
        double dlfac = sqrt(s->lfacf * s->lfacf / chi + 1);
        double dD = s->Df * pow(chi, -(7. - 2. * P->k) / (4. - P->k));
        double drho = dD / dlfac;
        double dv = c_ * sqrt(1. - 1. / (dlfac * dlfac));
        double rho = 0, v = 0, p = 0;
        rho += drho * ddV / dV;
        v += dv * ddV / dV;
        p += dp * ddV / dV;
        c->S.prim[RHO] = rho / s->rhoNorm;
        c->S.prim[UU1] = v / s->vNorm;
        c->S.prim[PPP] = p / s->pNorm;
        c->S.prim[TR1] = 2.;
      }
    }
  } else { /* 1DST.cpp:28-78 with run-time states */
    double x = P->xmax - P->xmin;
    for (int i = 0; i < n; ++i) {
      cell *c = &Cinit[i];
      c->G.x = (double)x * (i + 0.5) / n + P->xmin;
      c->G.dx = x / n;
      all_geom(s, &c->G);
    }
    for (int i = 0; i < n; ++i) {
      cell *c = &Cinit[i];
      if (c->G.x <= P->xmid) {
        c->S.prim[RHO] = P->rhoL;
        c->S.prim[UU1] = P->vL;
        c->S.prim[PPP] = P->pL;
        c->S.prim[TR1] = P->trL;
      } else {
        c->S.prim[RHO] = P->rhoR;
        c->S.prim[UU1] = P->vR;
        c->S.prim[PPP] = P->pR;
        c->S.prim[TR1] = P->trR;
      }
    }
  }
}

/* userKinematics (BM1D.cpp:188-246: fixed ghost-interface speeds; tube: none) */
static void user_kinematics(oc_sim *s) {
  if (s->c.problem != OC_PROBLEM_BM1D) return;
  for (int n = 0; n < s->ngst; ++n) {
    s->I[n].v = s->c.v_in;
    s->I[s->ntrack - 2 - n].v = s->c.v_out;
  }
}

/* userBoundaries (BM1D.cpp:254-274; tube: none) */
static void user_boundaries(oc_sim *s, double t) {
  if (s->c.problem != OC_PROBLEM_BM1D) return;
  if (t < s->c.t_bm_until) {
    for (int i = 0; i <= s->iLbnd; ++i) {
      cell *c = &s->C[i];
      double rho, u, p;
      double r = c->G.x * s->lNorm;
      calc_bm(s, r, t, &rho, &u, &p);
      c->S.prim[RHO] = rho;
      c->S.prim[UU1] = u;
      c->S.prim[UU2] = 0;
      c->S.prim[PPP] = p;
      c->S.prim[TR1] = 2.;
    }
  }
}

/* checkCellForRegrid (BM1D.cpp:277-319; tube: always skip) */
static int check_cell_for_regrid(const oc_sim *s, int i) {
  if (s->c.problem != OC_PROBLEM_BM1D) return SKIP;
  const oc_config *P = &s->c;
  const cell *c = &s->C[i];
  double dr = c->G.dx;
  double rOut = s->C[s->iRbnd - 1].G.x;
  double ar = dr / (rOut * P->dth);
  double iS = s->iLbnd + 1;
  for (int ii = s->iRbnd - 1; ii > s->iLbnd; --ii) {
    double p = s->C[ii].S.prim[PPP];
    iS = ii;
    if (p > 1.5 * P->eta) break;
  }
  double dist = i - iS;
  if (0 < dist && dist < 10) ar *= 10;
  double lfac = st_lfac(&c->S);
  if (ar > P->split_AR * P->target_ar / pow(lfac, 3. / 2.)) return SPLIT;
  if (ar < P->merge_AR * P->target_ar / pow(lfac, 3. / 2.)) return MERGE;
  return SKIP;
}

/* ------------------------------------------------------------------------- */
/* grid driver (1d.cpp)                                                       */

/* Grid::updateGhosts (1d.cpp:217-246) */
static void update_ghosts(oc_sim *s, double t) {
  cell *C = s->C;
  iface *I = s->I;
  const int iL = s->iLbnd, iR = s->iRbnd;
  for (int i = 0; i <= iL; ++i) {
    C[i] = C[iL + 1];
    C[i].G.x -= (iL - i + 1) * C[iL + 1].G.dx;
    all_geom(s, &C[i].G);
  }
  for (int i = 0; i <= iL - 1; ++i) {
    I[i] = I[iL + 1];
    I[i].x -= (iL - i + 1) * C[iL + 1].G.dx;
    iface_dA(s, &I[i]);
  }
  for (int i = iR; i < s->ntrack; ++i) {
    C[i] = C[iR - 1];
    C[i].G.x += (i - iR + 1) * C[iR - 1].G.dx;
    all_geom(s, &C[i].G);
  }
  for (int i = iR; i < s->ntrack - 1; ++i) {
    I[i] = I[iR - 1];
    I[i].x += (i - iR) * C[iR - 1].G.dx;
    iface_dA(s, &I[i]);
  }
  user_boundaries(s, t);
}

static double minmod(double a, double b) {
  if (fabs(a) < fabs(b) && a * b > 0) return a;
  if (fabs(b) < fabs(a) && a * b > 0) return b;
  return 0;
}

static void grad(const oc_sim *s, const cell *cL, const cell *cR, double *g) {
  double xL = cL->G.cen;
  double xR = cR->G.cen;
  for (int q = 0; q < s->nq; ++q) g[q] = (cR->S.prim[q] - cL->S.prim[q]) / (xR - xL);
}

/* Grid::reconstructStates, piecewise linear (1d.cpp:370-461) */
static void reconstruct(oc_sim *s, int i) {
  iface *In = &s->I[i];
  cell *C = s->C;
  const int nq = s->nq;
  if (i == 0 || i == s->ntrack - 2) {
    In->SL = C[i].S;
    In->SR = C[i + 1].S;
    return;
  }
  const cell *cL = &C[i];
  const cell *cLL = &C[i - 1 > 0 ? i - 1 : 0];
  const cell *cR = &C[i + 1];
  const cell *cRR = &C[i + 2 < s->ntrack - 1 ? i + 2 : s->ntrack - 1];
  double gL[OC_NQ_MAX], gR[OC_NQ_MAX], gN[OC_NQ_MAX];
  grad(s, cLL, cL, gL);
  grad(s, cL, cR, gN);
  grad(s, cR, cRR, gR);
  for (int q = 0; q < nq; ++q) {
    gL[q] = minmod(gL[q], gN[q]);
    gR[q] = minmod(gR[q], gN[q]);
  }
  double xI = In->x;
  for (int q = 0; q < nq; ++q) In->SL.prim[q] = cL->S.prim[q] + gL[q] * (xI - cL->G.cen);
  prim2cons(s, &In->SL, In->x);
  state2flux(s, &In->SL, In->x);
  for (int q = 0; q < nq; ++q) In->SR.prim[q] = cR->S.prim[q] + gR[q] * (xI - cR->G.cen);
  prim2cons(s, &In->SR, In->x);
  state2flux(s, &In->SR, In->x);
}

/* Grid::prepForUpdate (grid.cpp:28-37) */
static int prep_for_update(oc_sim *s) {
  cell *C = s->C;
  iface *I = s->I;
  const int n = s->ntrack;
  for (int i = 0; i < n; ++i) prim2cons(s, &C[i].S, C[i].G.cen);
  for (int i = 0; i < n; ++i) state2flux(s, &C[i].S, C[i].G.cen);
  for (int i = 0; i < n - 1; ++i) { /* movDir_ComputeLambda (1d.cpp:731-739) */
    reconstruct(s, i);
    compute_lambda(s, &I[i]);
  }
  for (int i = 0; i < n - 1; ++i) { /* updateKinematics (1d.cpp:741-751) */
    double v = s->c.vi * I[i].lS;
    double lfac = 1. / sqrt(1. - v * v);
    I[i].v = v;
    I[i].lfac = lfac;
  }
  user_kinematics(s);
  for (int i = 0; i < n - 1; ++i) { /* computeFluxes (1d.cpp:753-776) */
    compute_flux(s, &I[i]);
    if (s->c.shock_detection) measure_shock(s, &I[i], &C[i]);
  }
  for (int i = 1; i < n - 1; ++i) {
    int rc = update_dt(&C[i], &I[i - 1], &I[i]);
    if (rc) return rc;
    memcpy(C[i].fluxL, I[i - 1].flux, sizeof(C[i].fluxL));
    memcpy(C[i].fluxR, I[i].flux, sizeof(C[i].fluxR));
  }
  return 0;
}

/* Grid::collect_dt (1d.cpp:779-795) */
static double collect_dt(oc_sim *s) {
  double local_dt = 1.e15;
  for (int i = 0; i < s->ntrack; ++i) {
    local_dt = fmin(local_dt, s->C[i].dt_loc);
    s->C[i].dt_loc = 1.e15;
  }
  return local_dt;
}

/* Grid::update (1d.cpp:798-810) */
static void grid_update(oc_sim *s, double dt) {
  for (int i = 0; i < s->ntrack - 1; ++i) {
    s->I[i].x += dt * s->I[i].v;
    iface_dA(s, &s->I[i]);
  }
  for (int i = s->iLbnd + 1; i <= s->iRbnd - 1; ++i)
    cell_update(s, &s->C[i], dt, s->I[i - 1].x, s->I[i].x);
}

/* RK3 stage combination (rk3.cpp:27-55 with w0,w1 = 3/4,1/4; :63-92 with 1/3,2/3) */
static void rk_combine(oc_sim *s, double w0, double w1) {
  cell *C = s->C;
  iface *I = s->I;
  const int nq = s->nq;
  for (int i = s->iLbnd + 1; i <= s->iRbnd - 1; ++i) {
    cell *c = &C[i];
    double dV = c->G.dV;
    double dV0 = c->G0.dV;
    for (int q = 0; q < nq; ++q) {
      double Q = c->S.cons[q];
      double Q0 = c->S0.cons[q];
      c->S.cons[q] = w0 * Q0 * dV0 + w1 * Q * dV;
    }
  }
  for (int i = s->iLbnd; i <= s->iRbnd - 1; ++i) {
    double x = I[i].x;
    double x0 = I[i].x0;
    I[i].x = w0 * x0 + w1 * x;
    iface_dA(s, &I[i]);
  }
  for (int i = 1; i < s->ntrack - 1; ++i) cell_move(s, &C[i], I[i - 1].x, I[i].x); /* 1d.cpp:831-841 */
  for (int i = s->iLbnd + 1; i <= s->iRbnd - 1; ++i) {
    cell *c = &C[i];
    for (int q = 0; q < nq; ++q) c->S.cons[q] /= c->G.dV;
    cons2prim(s, &c->S, c->G.x, 0);
  }
}

/* Grid::evolve: RK3 (rk3.cpp:13-95) or Euler (euler.cpp:12-19) */
static int evolve(oc_sim *s, double t, double dt) {
  int rc;
  if (s->c.timestep == 1) {
    grid_update(s, dt);
    return 0;
  }
  for (int i = 0; i < s->ntrack; ++i) { /* copyState0 (1d.cpp:813-828) */
    s->C[i].S0 = s->C[i].S;
    s->C[i].G0 = s->C[i].G;
  }
  for (int i = 0; i < s->ntrack - 1; ++i) {
    s->I[i].x0 = s->I[i].x;
    s->I[i].v0 = s->I[i].v;
  }
  grid_update(s, dt);
  update_ghosts(s, t);
  if ((rc = prep_for_update(s))) return rc;
  grid_update(s, dt);
  rk_combine(s, 3. / 4., 1. / 4.);
  update_ghosts(s, t);
  if ((rc = prep_for_update(s))) return rc;
  grid_update(s, dt);
  rk_combine(s, 1. / 3., 2. / 3.);
  return 0;
}

/* Grid::split (1d.cpp:560-662) */
static void split(oc_sim *s, int i) {
  cell *C = s->C;
  iface *I = s->I;
  const int nq = s->nq;
  memmove(&C[i + 2], &C[i + 1], (size_t)(s->ntrack - (i + 1)) * sizeof(cell));
  memmove(&I[i + 1], &I[i], (size_t)(s->ntrack - 1 - i) * sizeof(iface));
  s->ntrack++;
  s->nact++;
  s->iRbnd++;
  cell *c = &C[i];
  cell *cR = &C[i + 1];
  cell *cL = &C[i - 1];
  cell *cR_old = &C[i + 2];
  double gL[OC_NQ_MAX], gR[OC_NQ_MAX], gN[OC_NQ_MAX], gC[OC_NQ_MAX];
  grad(s, cL, c, gL);
  grad(s, c, cR_old, gR);
  grad(s, cL, cR_old, gN);
  for (int q = 0; q < nq; ++q) {
    gL[q] = minmod(gL[q], gN[q]);
    gR[q] = minmod(gR[q], gN[q]);
    gC[q] = minmod(gL[q], gR[q]);
  }
  double x_old = c->G.x;
  double dl_old = c->G.dx;
  c->G.x = x_old - dl_old / 4.;
  cR->G.x = x_old + dl_old / 4.;
  c->G.dx = dl_old / 2.;
  cR->G.dx = dl_old / 2.;
  all_geom(s, &c->G);
  all_geom(s, &cR->G);
  double xL = c->G.cen;
  double xR = cR->G.cen;
  double xI = c->G.x + c->G.dx / 2.;
  for (int q = 0; q < nq; ++q) {
    double Sc = c->S.prim[q];
    double g = gC[q];
    c->S.prim[q] = Sc + g * (xL - xI);
    cR->S.prim[q] = Sc + g * (xR - xI);
  }
  prim2cons(s, &c->S, c->G.cen);
  state2flux(s, &c->S, c->G.cen);
  prim2cons(s, &cR->S, cR->G.cen);
  state2flux(s, &cR->S, cR->G.cen);
  I[i].x = x_old;
  iface_dA(s, &I[i]);
}

/* Grid::merge (1d.cpp:665-728) */
static void merge(oc_sim *s, int i) {
  cell *C = s->C;
  iface *I = s->I;
  const int nq = s->nq;
  cell *c = &C[i];
  cell *cL = &C[i - 1];
  cell *cR = &C[i + 1];
  cell *cVic;
  int left;
  if ((cL->G.dx < cR->G.dx && i != s->ngst) || i == s->nact + s->ngst - 1) {
    left = 1;
    cVic = cL;
  } else {
    left = 0;
    cVic = cR;
  }
  prim2cons(s, &c->S, c->G.cen);
  prim2cons(s, &cVic->S, cVic->G.cen);
  double dV_loc = c->G.dV;
  double dV_vic = cVic->G.dV;
  for (int q = 0; q < nq; ++q) {
    double Q_loc = c->S.cons[q];
    double Q_vic = cVic->S.cons[q];
    c->S.cons[q] = (Q_loc * dV_loc + Q_vic * dV_vic) / (dV_loc + dV_vic);
  }
  if (left) c->G.x = ((cVic->G.x - cVic->G.dx / 2.) + (c->G.x + c->G.dx / 2.)) / 2.;
  else c->G.x = ((cVic->G.x + cVic->G.dx / 2.) + (c->G.x - c->G.dx / 2.)) / 2.;
  c->G.dx += cVic->G.dx;
  all_geom(s, &c->G);
  cons2prim(s, &c->S, c->G.cen, 0);
  state2flux(s, &c->S, c->G.cen);
  if (left) {
    memmove(&C[i - 1], &C[i], (size_t)(s->ntrack - i) * sizeof(cell));
    memmove(&I[i - 1], &I[i], (size_t)(s->ntrack - 1 - i) * sizeof(iface));
  } else {
    memmove(&C[i + 1], &C[i + 2], (size_t)(s->ntrack - (i + 2)) * sizeof(cell));
    memmove(&I[i], &I[i + 1], (size_t)(s->ntrack - 1 - (i + 1)) * sizeof(iface));
  }
  s->ntrack--;
  s->nact--;
  s->iRbnd--;
}

/* Grid::regrid + applyRegrid (1d.cpp:484-557); targetRegridVictims only
 * matters with CIRC_REGRID_ (disabled, environment.h:61) and is omitted. */
int oc_regrid(oc_sim *s) {
  for (int i = s->iLbnd + 1; i <= s->iRbnd - 1; ++i) {
    int action = check_cell_for_regrid(s, i);
    if (action == SPLIT && s->ntrack < s->cap - 1) split(s, i);
    if (action == MERGE && s->ntrack > 2 * s->ngst + 2) merge(s, i);
  }
  return 0;
}

/* ------------------------------------------------------------------------- */
/* public API                                                                 */

void oc_config_bm1d_defaults(oc_config *c) {
  memset(c, 0, sizeof(*c));
  c->geometry = OC_GEOM_SPHERICAL1D;
  c->hydro = OC_HYDRO_REL_SPH;
  c->eos = OC_EOS_IDEAL;
  c->nq = 10;
  c->shock_detection = 1;
  c->local_synchrotron = 1;
  c->problem = OC_PROBLEM_BM1D;
  c->ngst = 2;
  c->ncell = 9900;
  c->nmax = 10000;
  c->gamma_ad = 4. / 3.;
  c->cfl = 0.2;
  c->vi = 1.;
  c->n0 = 1.;
  c->eta = 1.e-5;
  c->Etot = 1.e53;
  c->n_ext = 1.;
  c->tinit = 4.e6;
  c->lfac_shock2 = 0.;
  c->lorentz_mode = 0.;
  c->Rscale = 1.e17;
  c->k = 0.;
  c->grid_log = 0.;
  c->r_lo = 0.9;
  c->r_hi = 1.1;
  c->dth = M_PI / 2. / 1000.;
  c->target_ar = 1.;
  c->split_AR = 3.;
  c->merge_AR = 0.1;
  c->t_bm_until = 1.e7;
  c->v_in = 0.;
  c->v_out = 1.5;
  c->c2p_epsrel = 1.e-13;
}

void oc_config_tube_defaults(oc_config *c) {
  memset(c, 0, sizeof(*c));
  c->geometry = OC_GEOM_CARTESIAN;
  c->hydro = OC_HYDRO_REL_CART;
  c->eos = OC_EOS_IDEAL;
  c->nq = 6;
  c->shock_detection = 0;
  c->local_synchrotron = 0;
  c->problem = OC_PROBLEM_TUBE;
  c->ngst = 2;
  c->ncell = 1000;
  c->nmax = 1000;
  c->gamma_ad = 5. / 3.;
  c->cfl = 0.2;
  c->vi = 1.;
  c->xmin = 0.;
  c->xmax = 1.;
  c->xmid = 0.5;
  c->rhoL = 10.;
  c->pL = 13.33;
  c->vL = 0.;
  c->trL = 1.;
  c->rhoR = 1.;
  c->pR = 1.e-7;
  c->vR = 0.;
  c->trR = 2.;
  c->c2p_epsrel = 1.e-13;
}

oc_sim *oc_create(const oc_config *cfg) {
  oc_sim *s = (oc_sim *)calloc(1, sizeof(oc_sim));
  s->c = *cfg;
  s->nq = cfg->nq;
  s->ntr = cfg->nq - 4;
  s->sph = cfg->hydro == OC_HYDRO_REL_SPH;
  s->ngst = cfg->ngst;
  s->cap = cfg->nmax + 2 * cfg->ngst;
  s->C = (cell *)calloc((size_t)s->cap, sizeof(cell));
  s->I = (iface *)calloc((size_t)s->cap, sizeof(iface));
  for (int i = 0; i < s->cap; ++i) {
    cell_init(&s->C[i]);
    iface_init(&s->I[i]);
  }
  if (cfg->problem == OC_PROBLEM_BM1D) bm_derive(s);
  return s;
}

void oc_destroy(oc_sim *s) {
  if (!s) return;
  free(s->C);
  free(s->I);
  free(s);
}

int oc_init(oc_sim *s) {
  const oc_config *P = &s->c;
  s->t = (P->problem == OC_PROBLEM_BM1D) ? s->tstart : 0.;
  s->it = 0;
  s->dt = 0;
  /* Grid::initialise (1d.cpp:53-81) */
  s->nact = P->ncell;
  s->ntrack = s->nact + 2 * s->ngst;
  s->iLbnd = s->ngst - 1;
  s->iRbnd = P->ncell + s->ngst;
  initial_conditions(s);
  /* Grid::prepForRun (grid.cpp:20-26): v2u, prim2cons, interfaceGeomFromCellPos */
  for (int i = 0; i < s->ntrack; ++i) {
    double v = 0;
    double vv = s->C[i].S.prim[UU1];
    v += vv * vv;
    v = sqrt(v);
    double lfac = 1. / sqrt(1. - v * v);
    s->C[i].S.prim[UU1] *= lfac;
  }
  for (int i = 0; i < s->ntrack; ++i) prim2cons(s, &s->C[i].S, s->C[i].G.cen);
  for (int i = 0; i < s->ntrack - 1; ++i) {
    if (i != s->iLbnd) s->I[i].x = s->C[i].G.x + s->C[i].G.dx / 2.;
    else s->I[i].x = s->C[i + 1].G.x - s->C[i + 1].G.dx / 2.;
    iface_dA(s, &s->I[i]);
  }
  if (P->local_synchrotron)
    for (int i = 0; i < s->ntrack; ++i) init_gammas(&s->C[i]);
  update_ghosts(s, s->t); /* Simu::run pre-loop (simu.cpp:74) */
  return 0;
}

/* body of Simu::run's loop (simu.cpp:79-105) */
int oc_step(oc_sim *s, int n) {
  for (int k = 0; k < n; ++k) {
    oc_regrid(s);
    if (s->c.shock_detection)
      for (int i = 0; i < s->ntrack; ++i) {
        s->C[i].Sd = -1;
        s->C[i].isShocked = 0;
        s->C[i].pspec = 0;
      }
    update_ghosts(s, s->t);
    int rc = prep_for_update(s);
    if (rc) return rc;
    if (s->c.shock_detection)
      for (int i = 0; i < s->ntrack; ++i)
        if (s->C[i].Sd > DETECT_SHOCK_THRESHOLD_) s->C[i].isShocked = 1;
    s->dt = s->c.cfl * collect_dt(s);
    rc = evolve(s, s->t, s->dt);
    if (rc) return rc;
    s->t += s->dt;
    s->it++;
    if (s->c.local_synchrotron)
      for (int i = 0; i < s->ntrack; ++i) inject_particles(s, &s->C[i]);
  }
  return 0;
}

void oc_scalars(const oc_sim *s, double *out) {
  out[0] = s->t;
  out[1] = s->dt;
  out[2] = (double)s->it;
  out[3] = s->ntrack;
  out[4] = s->nact;
  out[5] = s->iLbnd;
  out[6] = s->iRbnd;
  out[7] = s->cap;
  out[8] = s->tstart;
  out[9] = s->RShock / (s->lNorm != 0 ? s->lNorm : 1.);
  out[10] = s->Nalpha;
  out[11] = s->Nmp;
  out[12] = s->Nme;
  out[13] = s->rhoNorm;
  out[14] = s->pNorm;
  out[15] = s->lNorm;
  out[16] = s->lfacShock2;
}

int oc_snapshot(const oc_sim *s, double *prim, double *x, double *dx, double *dt_loc, double *sd,
                double *pspec, double *shocked, double *xI, int cap) {
  if (s->ntrack > cap) return -1;
  for (int i = 0; i < s->ntrack; ++i) {
    const cell *c = &s->C[i];
    if (prim)
      for (int q = 0; q < s->nq; ++q) prim[q * cap + i] = c->S.prim[q];
    if (x) x[i] = c->G.x;
    if (dx) dx[i] = c->G.dx;
    if (dt_loc) dt_loc[i] = c->dt_loc;
    if (sd) sd[i] = s->c.shock_detection ? c->Sd : 0;
    if (pspec) pspec[i] = s->c.shock_detection ? c->pspec : 0;
    if (shocked) shocked[i] = (s->c.shock_detection && c->isShocked) ? 1. : 0.;
  }
  if (xI)
    for (int i = 0; i < s->ntrack - 1; ++i) xI[i] = s->I[i].x;
  return s->ntrack;
}

int oc_load(oc_sim *s, int ntrack, const double *prim, const double *x, const double *dx,
            const double *dt_loc, const double *xI, int cap, double t, long it) {
  if (ntrack > s->cap || ntrack > cap) return -1;
  s->ntrack = ntrack;
  s->nact = ntrack - 2 * s->ngst;
  s->iLbnd = s->ngst - 1;
  s->iRbnd = ntrack - s->ngst;
  for (int i = 0; i < ntrack; ++i) {
    cell *c = &s->C[i];
    for (int q = 0; q < s->nq; ++q) c->S.prim[q] = prim[q * cap + i];
    c->G.x = x[i];
    c->G.dx = dx[i];
    all_geom(s, &c->G);
    c->dt_loc = dt_loc ? dt_loc[i] : 1.e15;
    prim2cons(s, &c->S, c->G.cen);
    state2flux(s, &c->S, c->G.cen);
  }
  for (int i = 0; i < ntrack - 1; ++i) {
    s->I[i].x = xI[i];
    iface_dA(s, &s->I[i]);
  }
  s->t = t;
  s->it = it;
  return 0;
}

void oc_cons2prim(const oc_sim *s, double *cons, double *prim, const double *r, int n, int *iters) {
  for (int k = 0; k < n; ++k) {
    fstate S;
    fstate_init(&S);
    for (int q = 0; q < s->nq; ++q) {
      S.cons[q] = cons[q * n + k];
      S.prim[q] = prim[q * n + k];
    }
    int it = cons2prim(s, &S, r ? r[k] : 1.0, 0);
    if (iters) iters[k] = it;
    for (int q = 0; q < s->nq; ++q) {
      cons[q * n + k] = S.cons[q];
      prim[q * n + k] = S.prim[q];
    }
  }
}

void oc_prim2cons(const oc_sim *s, const double *prim, double *cons, const double *r, int n) {
  for (int k = 0; k < n; ++k) {
    fstate S;
    fstate_init(&S);
    for (int q = 0; q < s->nq; ++q) S.prim[q] = prim[q * n + k];
    prim2cons(s, &S, r ? r[k] : 1.0);
    for (int q = 0; q < s->nq; ++q) cons[q * n + k] = S.cons[q];
  }
}

void oc_riemann(const oc_sim *s, const double *primL, const double *primR, const double *x,
                const double *v, int v_given, double *lam, double *flux, int n) {
  for (int k = 0; k < n; ++k) {
    iface I;
    iface_init(&I);
    I.x = x[k];
    iface_dA(s, &I);
    for (int q = 0; q < s->nq; ++q) {
      I.SL.prim[q] = primL[q * n + k];
      I.SR.prim[q] = primR[q * n + k];
    }
    prim2cons(s, &I.SL, I.x);
    state2flux(s, &I.SL, I.x);
    prim2cons(s, &I.SR, I.x);
    state2flux(s, &I.SR, I.x);
    compute_lambda(s, &I);
    I.v = v_given ? v[k] : s->c.vi * I.lS;
    compute_flux(s, &I);
    lam[3 * k + 0] = I.lL;
    lam[3 * k + 1] = I.lS;
    lam[3 * k + 2] = I.lR;
    for (int q = 0; q < s->nq; ++q) flux[q * n + k] = I.flux[q];
  }
}

void oc_bm_profile(const oc_sim *s, const double *r, int n, double t, double *rho, double *u,
                   double *p) {
  for (int k = 0; k < n; ++k) calc_bm(s, r[k] * s->lNorm, t, &rho[k], &u[k], &p[k]);
}
