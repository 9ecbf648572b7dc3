// Device physics of the 1D moving-mesh relativistic hydro step (FP64).
//
// Each function restates one member of the GAMMA reference and keeps its
// floating-point operation order, so that with -fmad=false the only
// differences to the CPU reference come from libm (tanh, and pow other than
// the correctly rounded x^(3/4) of the shock detector) and from the pressure
// root finder (Newton-Raphson here, GSL Brent there).
//
// Variable slots follow src/environment.h:33-82.  Slot 3 (the theta momentum /
// 4-velocity) is identically zero in 1D: it is only ever multiplied by r
// (rel_sph.cpp:78,108,441) starting from zero, so it is neither stored nor
// computed here.
#pragma once

#include <cstdint>
#include <math.h>

#include "gamma_problem.h"

#ifndef GB_HD
#define GB_HD __device__ __forceinline__
#endif
// one out-of-line copy per kernel (see c2p_pressure)
#ifndef GB_HD_OUTLINE
#define GB_HD_OUTLINE __device__ __noinline__
#endif

namespace gb {

enum { RHO = 0, PPP = 1, UU1 = 2, UU2 = 3 };
enum { DEN = 0, TAU = 1, SS1 = 2, SS2 = 3 };
enum { TR1 = 4, GMN = 6, GMX = 7, GMD = 8, PSN = 9 };
enum { SKIP = 0, MERGE = 1, SPLIT = 2 };

// src/constants.h:6-28
constexpr double P_FLOOR = 1.e-10;
constexpr double PI_ = 3.14159265358979323846;
constexpr double MP = 1.6726219e-24;
constexpr double ME = 9.1093835e-28;
constexpr double C_LIGHT = 2.99792458e10;
constexpr double ALPHA_SYN = 1.29251816e-09;
constexpr double P_SPEC = 2.22;
constexpr double EPS_E = 0.1;
constexpr double EPS_B = 0.01;
constexpr double ZETA = 1.;
constexpr double GAMMA_MAX_INIT = 1.e8;
constexpr double DETECT_SHOCK_THRESHOLD = 0.01;
constexpr double DT_INF = 1.e15;

// ---------------------------------------------------------------------------
// Module selections (the reference's Makefile GEOMETRY/HYDRO/RADIATION slots and
// environment.h switches) as compile-time policies.

// Arithmetic form of the 1D step.
//   0: every formula in the reference's operation order, so a state, flux or
//      wave speed computed from the same inputs is bit for bit the reference's.
//   1: divisions by a shared denominator become one reciprocal and
//      multiplications (about half the FP64 instructions of the step); results
//      move at the ulp level, which the reference's own cold-gas conditioning
//      amplifies beyond the parity bars (lambda* from a near-cancelling
//      quadratic; f(p) of cons2prim cancelling to eps*E).
//   2 (default): the shared reciprocals of 1 everywhere except where the
//      reference's results hinge on exact values, which keep its order: the
//      wave speeds and the contact speed lambda*, the PLM pair gradients whose
//      minmod returns 0 on a tie (FAST_RIEMANN), and f(p) of the cons2prim
//      root search with the primitive recovery after it (FAST_ROOT).  It meets
//      every parity bar that 0 meets, with the same cell counts and regrid
//      decisions, and runs the tube step ~20% faster.
#ifndef GB_FAST_ARITH
#define GB_FAST_ARITH 2
#endif

// cartesian + rel_cart, ideal gas, no shock detection / synchrotron: NUM_Q = 6.
#ifndef GB_CART_MIN_BLOCKS
#define GB_CART_MIN_BLOCKS 5
#endif
struct CfgCart {
  static constexpr bool FAST = GB_FAST_ARITH != 0;
  static constexpr bool FAST_RIEMANN = GB_FAST_ARITH == 1;
  static constexpr bool FAST_ROOT = GB_FAST_ARITH == 1;
  static constexpr int MIN_BLOCKS = GB_CART_MIN_BLOCKS;  // 128-thread CTAs per SM (5: 96 registers)
  static constexpr int NQ = 6;
  static constexpr bool SPH = false;    // rel_sph hydro and spherical1D geometry
  static constexpr bool SHOCK = false;  // SHOCK_DETECTION_
  static constexpr bool SYNCH = false;  // LOCAL_SYNCHROTRON_
  static constexpr bool CYL = false;    // rel_cyl hydro (Hydro/rel_cyl.cpp)
};

// cartesian + rel_cyl (Hydro/rel_cyl.cpp, the HYDRO module whose GEOMETRY
// partner, Geometry/cylindrical.cpp, does not compile): rel_cart with the
// cylindrical source p/r on S_r, a root search only where |f| at the previous
// pressure exceeds 1e-13, and a zero velocity below |S| = 1e-14 (NUM_Q = 6).
struct CfgCyl : CfgCart {
  static constexpr bool CYL = true;
};

// spherical1D + rel_sph + radiation_sph: NUM_Q = 10.
#ifndef GB_SPH_MIN_BLOCKS
#define GB_SPH_MIN_BLOCKS 3
#endif
struct CfgSph {
  static constexpr bool FAST = GB_FAST_ARITH != 0;
  static constexpr bool FAST_RIEMANN = GB_FAST_ARITH == 1;
  static constexpr bool FAST_ROOT = GB_FAST_ARITH == 1;
  static constexpr int MIN_BLOCKS = GB_SPH_MIN_BLOCKS;
  static constexpr int NQ = 10;
  static constexpr bool SPH = true;
  static constexpr bool SHOCK = true;
  static constexpr bool SYNCH = true;
  static constexpr bool CYL = false;
};

// A module set with every formula in the reference's operation order, whatever
// GB_FAST_ARITH says: for results that must equal the reference's bit for bit
// (the text dump's conserved columns).
template <class Cfg>
struct RefOrder : Cfg {
  static constexpr bool FAST = false;
  static constexpr bool FAST_RIEMANN = false;
  static constexpr bool FAST_ROOT = false;
};

// Run-time constants shared by every run of a context.
struct Phys {
  double gamma_ad;  // GAMMA_
  double kgam;      // GAMMA_ / (GAMMA_ - 1), the enthalpy factor of the ideal EOS
  double cfl;       // CFL_
  double vi;        // VI
  int eos;          // 0 ideal, 1 Synge / Taub-Mathews (rel_sph.cpp:37-52)
  int ngst;
  int eos_ws;       // 1: each state's Gamma_eff in the wave speeds and the shock
                    // detector too (the reference uses GAMMA_ there)
  int euler;        // 1: Grid::evolve of Timestep/euler.cpp (one Grid::update),
                    // 0: the three SSP-RK3 stages of Timestep/rk3.cpp
};

template <class Cfg>
struct Prim {
  double v[Cfg::NQ];
};

// FluidState: primitive, conserved and physical flux of one state, with its
// Lorentz factor and 3-velocity cached (FluidState::lfac is called many times
// per interface in the reference).
template <class Cfg>
struct FState {
  double prim[Cfg::NQ];
  double cons[Cfg::NQ];
  double flux[Cfg::NQ];
  double lfac, v;
};

GB_HD double lfac_of(double uu) {
  // fluid.cpp:10-22 (u = sqrt(sum uu^2) then sqrt(1+u^2))
  double u = 0.;
  u += uu * uu;
  u = sqrt(u);
  return sqrt(1 + u * u);
}

// FluidState::gamma (rel_sph.cpp:37-52)
GB_HD double eos_gamma(const Phys &ph, double rho, double p) {
  const double G = ph.gamma_ad;
  if (ph.eos == 0) return G;
  double a = p / rho / (G - 1.);
  double e_ratio = a + sqrt(a * a + 1.);
  return G - (G - 1.) / 2. * (1. - 1. / (e_ratio * e_ratio));
}

// a / b, bit for bit, for quotients whose numerator is often zero (uniform
// tracers, flat gradients, gas at rest).  With a = +-0 the IEEE quotient is a
// signed zero (b finite or infinite, nonzero) or NaN (b zero or NaN), which is
// a * (1 / s) with s = +-1, +-0 or NaN as b's class; the divide then never
// sees a zero numerator, which sends the whole warp through the division's
// slow path.
GB_HD double qdiv(double a, double b) {
  const bool z = a == 0.;
  const double s = z ? ((b != 0. && b == b) ? copysign(1., b) : b) : b;
  const double q = (z ? 1. : a) / s;
  return z ? a * q : q;
}

// 1/x to about 2^-22, for correction terms only
GB_HD double recip_approx(double x) {
#ifdef __CUDA_ARCH__
  double r;
  asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(x));
  return r;
#else
  return 1. / x;
#endif
}

// x^(3/4) rounded to nearest: the isentrope rho1 (p/p1)^(1/GAMMA_) of the shock
// detector when 1/GAMMA_ is exactly 3/4 (GAMMA_ = 4/3), as the C library's pow
// returns it.  sqrt(x) and then x^(1/4) are carried as double-double pairs:
// the remainder of a correctly rounded square root, x - s^2, is exact as one
// FMA (Markstein 1990; Boldo & Daumas 2003), so sqrt(x) = s + (x - s^2)/(2s)
// to twice the precision, and Dekker's exact product (the FMA form) gives the
// pair s*q; it is rounded once.  The correction terms need ~20 bits, hence the
// approximate reciprocal.  Outside [2^-900, 2^900] (or NaN): pow itself.
GB_HD double pow_3_4(double x) {
  if (!(x >= 0x1p-900 && x <= 0x1p900)) return pow(x, 0.75);
  const double s = sqrt(x);
  const double sl = fma(-s, s, x) * 0.5 * recip_approx(s);  // sqrt(x) = s + sl
  const double q = sqrt(s);
  const double ql = (fma(-q, q, s) + sl) * 0.5 * recip_approx(q);  // sqrt(s + sl) = q + ql
  const double ph = s * q;
  const double lo = fma(s, q, -ph) + (s * ql + sl * q);
  return ph + lo;
}

// (p/p1)^(1/GAMMA_) of the isentrope
GB_HD double isentrope_pow(double x, double ginv) { return ginv == 0.75 ? pow_3_4(x) : pow(x, ginv); }

template <class Cfg>
GB_HD double state_gamma(const Phys &ph, const double *prim) {
  return Cfg::SPH ? eos_gamma(ph, prim[RHO], prim[PPP]) : ph.gamma_ad;
}

// gamma/(gamma-1) of a state: cached for the ideal EOS
template <class Cfg>
GB_HD double enth_k(const Phys &ph, const double *prim) {
  if (Cfg::SPH && ph.eos != 0) {
    const double g = eos_gamma(ph, prim[RHO], prim[PPP]);
    return g / (g - 1.);
  }
  return ph.kgam;
}

// prim2cons (rel_sph.cpp:55-82, rel_cart.cpp:37-64)
template <class Cfg>
GB_HD void prim2cons(const Phys &ph, const double *prim, double *cons) {
  double rho = prim[RHO];
  double p = prim[PPP];
  double uu = prim[UU1];
  double lfac = lfac_of(uu);
  double h;
  if (Cfg::FAST) {
    h = 1. + enth_k<Cfg>(ph, prim) * p / rho;
  } else {
    const double gma = state_gamma<Cfg>(ph, prim);
    h = 1. + p * gma / (gma - 1.) / rho;
  }
  double D = lfac * rho;
  double tau = D * h * lfac - p - D;
  double ss = D * h * uu;
  cons[DEN] = D;
  cons[TAU] = tau;
  cons[SS1] = ss;
  cons[SS2] = 0.;
#pragma unroll
  for (int t = TR1; t < Cfg::NQ; ++t) cons[t] = prim[t] * D;
}

// prim2cons + state2flux of a reconstructed or cell state in one pass
// (rel_sph.cpp:55-113): lfac and v = u/lfac are formed once.
template <class Cfg>
GB_HD void state2flux(const double *prim, const double *cons, double *flux);

template <class Cfg>
GB_HD void fill_state(const Phys &ph, FState<Cfg> &S) {
  if (!Cfg::FAST) {
    prim2cons<Cfg>(ph, S.prim, S.cons);
    state2flux<Cfg>(S.prim, S.cons, S.flux);
    S.lfac = lfac_of(S.prim[UU1]);
    S.v = qdiv(S.prim[UU1], S.lfac);
    return;
  }
  const double rho = S.prim[RHO], p = S.prim[PPP], uu = S.prim[UU1];
  const double lfac = sqrt(1. + uu * uu);
  const double v = uu / lfac;
  const double h = 1. + enth_k<Cfg>(ph, S.prim) * p / rho;
  const double D = lfac * rho;
  const double Dh = D * h;
  S.lfac = lfac;
  S.v = v;
  S.cons[DEN] = D;
  S.cons[TAU] = Dh * lfac - p - D;
  S.cons[SS1] = Dh * uu;
  S.cons[SS2] = 0.;
  S.flux[DEN] = D * v;
  S.flux[SS1] = S.cons[SS1] * v + p;
  S.flux[SS2] = 0.;
  S.flux[TAU] = S.cons[SS1] - D * v;
#pragma unroll
  for (int t = TR1; t < Cfg::NQ; ++t) {
    S.cons[t] = S.prim[t] * D;
    S.flux[t] = S.cons[t] * v;
  }
}

// state2flux (rel_sph.cpp:85-113, rel_cart.cpp:67-95)
template <class Cfg>
GB_HD void state2flux(const double *prim, const double *cons, double *flux) {
  double p = prim[PPP];
  double uu = prim[UU1];
  double lfac = lfac_of(uu);
  double D = cons[DEN];
  double ss = cons[SS1];
  flux[DEN] = qdiv(D * uu, lfac);
  flux[SS1] = qdiv(ss * uu, lfac) + p;
  flux[SS2] = 0.;
  flux[TAU] = ss - qdiv(D * uu, lfac);
#pragma unroll
  for (int t = TR1; t < Cfg::NQ; ++t) flux[t] = qdiv(cons[t] * uu, lfac);
}

// ---------------------------------------------------------------------------
// cons2prim: pressure root of f(p) (rel_sph.cpp:191-210 / rel_cart.cpp:108-123)
// by safeguarded Newton-Raphson on the same bracket and with the same
// no-solution semantics as the reference's Brent driver (rel_sph.cpp:243-286).

struct C2PStats {
  int iters;     // f evaluations after the bracket set-up
  int fallback;  // 1 if the iteration cap was hit (bisection-limited)
  int deferred;  // 1 if a deferring search stopped at a poor warm start (c2p_pressure_body)
  int poor;      // 1 if a search was needed and its warm start was poor (c2p_warm_start_poor)
};

// A warm start is poor where the first Newton correction from it, |f/f'|,
// exceeds this fraction of the pressure: worse than the learned guess's own
// starting error of a few per cent.  (A build may set another fraction with
// -DGB_GUESS_GATE=...)
#ifndef GB_GUESS_GATE
#define GB_GUESS_GATE 3e-2
#endif
constexpr double kGuessGate = GB_GUESS_GATE;

GB_HD bool c2p_warm_start_poor(double f, double df, double p) { return !(fabs(f) <= kGuessGate * fabs(df) * p); }

// f(p) = E + p - D lfac - k p lfac^2 with lfac = (1 - S^2/(E+p)^2)^(-1/2)
// (rel_sph.cpp:191-210 takes |1 - S^2/W^2|, rel_cart.cpp:108-123 does not).
// Returns f; with df != nullptr also df/dp and lfac^2.  For the Synge EOS the
// derivative of Gamma_eff is included through rho = D/lfac and a = p/rho/(G-1).
template <class Cfg>
GB_HD double c2p_f(const Phys &ph, double p, double D, double S2, double E, double *df = nullptr,
                   double *l2out = nullptr) {
  const double W = E + p;
  const double rW = 1. / W;
  const double x = S2 * rW * rW;
  const double arg = Cfg::SPH ? fabs(1. - x) : (1. - x);
  const double lfac = rsqrt(arg);
  const double l2 = lfac * lfac;
  double k, dk = 0.;
  if (Cfg::SPH && ph.eos != 0) {
    const double G = ph.gamma_ad;
    const double rho = D / lfac;
    const double a = p / rho / (G - 1.);
    const double sq = sqrt(a * a + 1.);
    const double e = a + sq;
    const double gma = G - (G - 1.) / 2. * (1. - 1. / (e * e));
    k = gma / (gma - 1.);
    if (df) {
      const double sgn = (1. - x) >= 0. ? 1. : -1.;
      const double dl = -sgn * lfac * l2 * x * rW;
      const double da = (lfac + p * dl) / (D * (G - 1.));
      const double dgma = -(G - 1.) / (e * e * e) * (da * (1. + a / sq));
      dk = -dgma / ((gma - 1.) * (gma - 1.));
    }
  } else {
    k = ph.kgam;
  }
  const double f = W - D * lfac - k * p * l2;
  if (df) {
    const double sgn = (1. - x) >= 0. ? 1. : -1.;
    const double dl = -sgn * lfac * l2 * x * rW;
    *df = 1. - D * dl - dk * p * l2 - k * (l2 + 2. * p * lfac * dl);
  }
  if (l2out) *l2out = l2;
  return f;
}

// f in the reference's operation order (rel_sph.cpp:198-207, rel_cart.cpp:118-120),
// with df/dp and lfac^2 on request.
template <class Cfg>
GB_HD double c2p_f_ref(const Phys &ph, double p, double D, double S, double E, double *df = nullptr,
                       double *l2out = nullptr, double *lfac_out = nullptr, bool p_may_be_zero = false) {
  const double W = E + p;
  const double x = qdiv(S * S, W * W);
  const double arg = Cfg::SPH ? fabs(1. - x) : (1. - x);
  const double lfac = 1. / sqrt(arg);
  const bool ideal = !Cfg::SPH || ph.eos == 0;
  const double gma = ideal ? ph.gamma_ad : eos_gamma(ph, D / lfac, p);
  // p = 0 at the bracket's lower end p_lo, which every search evaluates
  const double kp = gma * p * lfac * lfac;
  const double f = (E + p - D * lfac - (p_may_be_zero ? qdiv(kp, gma - 1.) : kp / (gma - 1.)));
  if (df) {
    if (!ideal) {  // Gamma_eff(p) terms: take them from the derivative form
      double dfast;
      c2p_f<Cfg>(ph, p, D, S * S, E, &dfast);
      *df = dfast;
    } else {  // d lfac/dp = -lfac^3 x / W with the same lfac and x as f
      const double sgn = (1. - x) >= 0. ? 1. : -1.;
      const double l2 = lfac * lfac;
      const double dl = qdiv(-sgn * lfac * l2 * x, W);
      // kgam is GAMMA_/(GAMMA_-1) rounded once on the host: gma/(gma-1) exactly
      *df = 1. - D * dl - ph.kgam * (l2 + 2. * p * lfac * dl);
    }
  }
  if (l2out) *l2out = lfac * lfac;
  if (lfac_out) *lfac_out = arg >= 0. ? lfac : -1.;  // -1: no lfac of fabs(1 - x) here
  return f;
}

// Pressure root of the cons2prim driver (rel_sph.cpp:243-286): the bracket,
// its no-solution tests and the warm start pCand are the reference's; the
// Brent search is replaced by safeguarded Newton-Raphson.  Returns the
// pressure the reference would go on with (pCand itself where it finds none).
//
// lfac_at (optional): the Lorentz factor 1/sqrt(|1 - S^2/(E+p)^2|) at the
// returned pressure when the search evaluated f there (the same rounding as
// f's), else -1.
//
// defer (with st): where a search is needed and the warm start is poor
// (c2p_warm_start_poor), stop before it and set st->deferred; the caller then
// starts the search again from a better pressure (the learned guess).
template <class Cfg>
GB_HD double c2p_pressure_body(const Phys &ph, double D, double S, double S2, double E, double pCand,
                               C2PStats *st, double *lfac_at, bool defer) {
  auto fval = [&](double p, double *df, double *l2, double *lf, bool p_may_be_zero = false) -> double {
    return Cfg::FAST_ROOT ? c2p_f<Cfg>(ph, p, D, S2, E, df, l2)
                     : c2p_f_ref<Cfg>(ph, p, D, S, E, df, l2, lf, p_may_be_zero);
  };
  int iters = 0, fallback = 0;
  // f at the warm start, with its slope: the search starts there when the
  // warm start lies in the bracket (f does not depend on whether df is asked for)
  double df0, l20, lf0 = -1.;
  const double f_init = fval(pCand, &df0, &l20, &lf0);
  if (lfac_at) *lfac_at = lf0;
  // rel_cyl.cpp:161 searches only where |f| exceeds 1e-13 (rel_sph, rel_cart: 0)
  int poor = 0;
  if (fabs(f_init) > (Cfg::CYL ? 1.e-13 : 0.)) {
    poor = c2p_warm_start_poor(f_init, df0, pCand);
    if (defer && st && poor) {
      st->iters = 0;
      st->fallback = 0;
      st->deferred = 1;
      st->poor = 1;
      return pCand;
    }
    double p_lo = fmax(0., (1. + 1e-13) * S - E);
    bool find_p = true;
    if (fval(p_lo, nullptr, nullptr, nullptr, true) < 0) find_p = false;
    double p_hi;
    if (f_init < 0) {
      p_hi = 1. * pCand;
    } else {
      p_hi = pCand;
      // the reference grows p_hi without bound (a zero guess would never end);
      // 400 decades reach infinity, where f is NaN and the loop stops anyway.
      // Its first test re-evaluates f(pCand), which is f_init.
      for (int g = 0; g < 400 && (g == 0 ? f_init : fval(p_hi, nullptr, nullptr, nullptr)) > 0; ++g) p_hi *= 10;
    }
    if (p_hi < p_lo) find_p = false;
    if (find_p) {
      // f(lo) >= 0 >= f(hi).  The warm start tightens one side.
      double lo = p_lo, hi = p_hi;
      if (f_init > 0.) lo = fmax(lo, pCand);
      double p = fmin(fmax(pCand, lo), hi);
      double df = df0, l2 = l20, lf = lf0;
      double f = f_init;
      if (!(p == pCand)) f = fval(p, &df, &l2, &lf);
      const int MAXIT = 100;
      const double eps = 2.220446049250313e-16;
      for (iters = 1; iters <= MAXIT; ++iters) {
        // Rounding noise of f: E, p, D lfac and k p lfac^2 cancel, and lfac
        // itself carries eps*lfac^2 relative error from 1 - S^2/W^2.  Below
        // this level the sign of f is noise and p is as good as it gets.
        const double noise = eps * (E + p + D * sqrt(l2) * (1. + l2) + 4. * p * l2 * (1. + 2. * l2));
        if (f == 0. || fabs(f) <= noise) break;
        double pn = p - f / df;
        if (!(pn > lo && pn < hi)) {
          // Newton left the bracket: bisect, geometrically once lo > 0
          pn = lo > 0. ? sqrt(lo) * sqrt(hi) : 0.5 * (lo + hi);
          if (!(pn > lo && pn < hi)) pn = 0.5 * (lo + hi);
        }
        double dfn, l2n, lfn;
        const double fn = fval(pn, &dfn, &l2n, &lfn);
        if (fn > 0.) lo = pn;
        else if (fn < 0.) hi = pn;
        const double step = fabs(pn - p);
        p = pn;
        f = fn;
        df = dfn;
        l2 = l2n;
        lf = lfn;
        if (fn == 0. || step <= 1.e-14 * pn || (hi - lo) <= 1.e-14 * hi) break;
      }
      if (iters > MAXIT) fallback = 1;
      pCand = p;
      if (lfac_at) *lfac_at = lf;
    }
  }
  if (st) {
    st->iters = iters;
    st->fallback = fallback;
    st->deferred = 0;
    st->poor = poor;
  }
  return pCand;
}

template <class Cfg>
GB_HD_OUTLINE double c2p_pressure_outline(const Phys &ph, double D, double S, double S2, double E, double pCand,
                                          C2PStats *st, double *lfac_at, bool defer) {
  return c2p_pressure_body<Cfg>(ph, D, S, S2, E, pCand, st, lfac_at, defer);
}

// The cartesian step calls the search from one out-of-line copy: inlined at
// every call site of the fused step kernel it crowds the instruction cache
// (3% slower).  The spherical kernels, the 2D passes and the batch cons2prim
// keep it inline, which is as fast or faster there.  OUTLINE forces the
// out-of-line copy (a second, rarely taken call site).
template <class Cfg, bool OUTLINE = !Cfg::SPH>
GB_HD double c2p_pressure(const Phys &ph, double D, double S, double S2, double E, double pCand, C2PStats *st,
                          double *lfac_at = nullptr, bool defer = false) {
  if (!OUTLINE) return c2p_pressure_body<Cfg>(ph, D, S, S2, E, pCand, st, lfac_at, defer);
  return c2p_pressure_outline<Cfg>(ph, D, S, S2, E, pCand, st, lfac_at, defer);
}

// What cons2prim's root search is given: D, E = D + tau, S and S^2 of the
// momentum, and the starting pressure (the previous one, floored in rel_sph).
struct C2PInput {
  double D, E, ss, S2, S, pCand;
};

template <class Cfg>
GB_HD C2PInput c2p_input(const double *cons, const double *prim) {
  C2PInput in;
  in.D = cons[DEN];
  const double tau = cons[TAU];
  in.E = in.D + tau;
  in.ss = cons[SS1];
  double S2 = 0.;
  S2 += in.ss * in.ss;
  in.S2 = S2;
  in.S = Cfg::FAST_ROOT ? fabs(in.ss) : sqrt(S2);
  in.pCand = Cfg::SPH ? fmax(1.e-13, prim[PPP]) : prim[PPP];
  return in;
}

// FluidState::cons2prim (rel_sph.cpp:213-320; rel_cart.cpp:125-229).
// On entry prim holds the previous primitives (pressure warm start); on exit
// prim holds the recovered primitives and cons is rewritten by prim2cons.
// Hooks::cons2prim_user (the problem module's FluidState::cons2prim_user,
// rel_sph.cpp:304) sees rho, p and u before the pressure floor; par is the
// run's parameter words.
// defer (with st): where the warm start is poor the search stops before it
// (st->deferred, c2p_pressure_body) and prim and cons are left as they were,
// for a second call from a better starting pressure.  OUTLINE: the search's
// out-of-line copy (c2p_pressure).
template <class Cfg, class Hooks = gamma_problem::Problem, bool OUTLINE = !Cfg::SPH>
GB_HD void cons2prim(const Phys &ph, double *cons, double *prim, C2PStats *st, const double *par = nullptr,
                     bool defer = false) {
  const C2PInput in = c2p_input<Cfg>(cons, prim);
  const double D = in.D, E = in.E, ss = in.ss, S2 = in.S2, S = in.S;
  double lf_root = -1.;
  const double pCand = c2p_pressure<Cfg, OUTLINE>(ph, D, S, S2, E, in.pCand, st, &lf_root, defer);
  if (defer && st && st->deferred) return;

  double p = pCand;
  double rho, uu;
  if (Cfg::FAST_ROOT) {  // lfac = W/sqrt(W^2-S^2), rho = D/lfac, u = lfac v S_i/S with v = S/W
    const double rW = 1. / (E + p);
    const double v2 = S2 * rW * rW;
    const double s1 = sqrt(fabs(1. - v2));  // 1/lfac
    rho = D * s1;
    uu = (fabs(S) == 0.) ? 0. : (ss * rW) / s1;
  } else {  // rel_sph.cpp:288-302
    // lfac = 1/sqrt(|1 - S2/(E+p)^2|): the root search's last f evaluation
    // formed the same quotient from S*S, which is S2 whenever S*S == S2
    double lfac = lf_root;
    if (!(lfac > 0. && S * S == S2)) {
      double Ep2 = (E + p) * (E + p);
      double v2 = qdiv(S2, Ep2);
      lfac = 1. / sqrt(fabs(1. - v2));
    }
    rho = D / lfac;
    if (Cfg::CYL ? fabs(S) < 1.e-14 : fabs(S) == 0.) {  // rel_cyl.cpp:207
      uu = 0;
    } else {
      double v = sqrt(1. - 1. / (lfac * lfac));
      // ss/S is exactly +-1 when S == |ss|
      uu = lfac * v * (fabs(ss) == S ? (ss > 0. ? 1. : -1.) : ss / S);
    }
  }
  Hooks::cons2prim_user(par, &rho, &p, &uu);
  if (Cfg::SPH) p = fmax(p, P_FLOOR);
  prim[PPP] = p;
  prim[RHO] = rho;
  prim[UU1] = uu;
  prim[UU2] = 0.;
  if (Cfg::FAST) {
    const double rD = 1. / D;
#pragma unroll
    for (int t = TR1; t < Cfg::NQ; ++t) prim[t] = cons[t] * rD;
  } else {
#pragma unroll
    for (int t = TR1; t < Cfg::NQ; ++t) prim[t] = qdiv(cons[t], D);
  }
  prim2cons<Cfg>(ph, prim, cons);
}

// ---------------------------------------------------------------------------
// Riemann problem at a moving interface

struct Waves {
  double lL, lS, lR;
};

// Interface::wavespeedEstimates + computeLambda (rel_sph.cpp:322-394;
// rel_cart.cpp:260-302 switches to the linear root when |FhllE| < 1e-15).
template <class Cfg>
GB_HD Waves compute_lambda_ref(const Phys &ph, const FState<Cfg> &L, const FState<Cfg> &R) {
  const bool ws = Cfg::SPH && ph.eos_ws;
  const double GL = ws ? eos_gamma(ph, L.prim[RHO], L.prim[PPP]) : ph.gamma_ad;
  const double GR = ws ? eos_gamma(ph, R.prim[RHO], R.prim[PPP]) : ph.gamma_ad;
  Waves w;
  double lfacL = L.lfac;
  double lfacR = R.lfac;
  double vL = L.v;
  double vR = R.v;
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

  const double lL = w.lL, lR = w.lR;
  double mmL = L.cons[SS1];
  double mmR = R.cons[SS1];
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
  bool linear = Cfg::SPH ? (fabs(FhllE) == 0) : (fabs(FhllE) < 1.e-15);
  if (linear) {
    w.lS = qdiv(mhll, Ehll + Fhllm);
  } else {
    // pow(x, 2.) of the C library is the correctly rounded square: x*x
    const double ef = Ehll + Fhllm;
    double delta = ef * ef - 4. * FhllE * mhll;
    w.lS = ((Ehll + Fhllm) - sqrt(delta)) / (2. * FhllE);
  }
  return w;
}

template <class Cfg>
GB_HD Waves compute_lambda(const Phys &ph, const FState<Cfg> &L, const FState<Cfg> &R) {
  if (!Cfg::FAST_RIEMANN || ph.eos_ws) return compute_lambda_ref<Cfg>(ph, L, R);
  const double G = ph.gamma_ad;
  const double kg = ph.kgam;
  Waves w;
  const double vL = L.v, vR = R.v;
  // relativistic sound speed (uses GAMMA_ in the reference for either EOS)
  const double cs2L = G * L.prim[PPP] / (L.prim[RHO] + L.prim[PPP] * kg);
  const double cs2R = G * R.prim[PPP] / (R.prim[RHO] + R.prim[PPP] * kg);
  const double sgSL = cs2L / (L.lfac * L.lfac * (1. - cs2L));
  const double sgSR = cs2R / (R.lfac * R.lfac * (1. - cs2R));
  const double qL = sqrt(sgSL * (1. - vL * vL + sgSL));
  const double qR = sqrt(sgSR * (1. - vR * vR + sgSR));
  const double rL = 1. / (1. + sgSL), rR = 1. / (1. + sgSR);
  w.lL = fmin((vR - qR) * rR, (vL - qL) * rL);
  w.lR = fmax((vR + qR) * rR, (vL + qL) * rL);

  const double lL = w.lL, lR = w.lR;
  const double mmL = L.cons[SS1], mmR = R.cons[SS1];
  const double pL = L.prim[PPP], pR = R.prim[PPP];
  const double EL = L.cons[TAU] + L.cons[DEN];
  const double ER = R.cons[TAU] + R.cons[DEN];
  const double AL = lL * EL - mmL;
  const double AR = lR * ER - mmR;
  const double BL = mmL * (lL - vL) - pL;
  const double BR = mmR * (lR - vR) - pR;
  const double rd = 1. / (lR - lL);
  const double FhllE = (lL * AR - lR * AL) * rd;
  const double Ehll = (AR - AL) * rd;
  const double Fhllm = (lL * BR - lR * BL) * rd;
  const double mhll = (BR - BL) * rd;
  const bool linear = Cfg::SPH ? (fabs(FhllE) == 0) : (fabs(FhllE) < 1.e-15);
  const double eh = Ehll + Fhllm;
  if (linear) {
    w.lS = mhll / eh;
  } else {
    const double delta = eh * eh - 4. * FhllE * mhll;
    w.lS = (eh - sqrt(delta)) / (2. * FhllE);
  }
  return w;
}

// HLLC flux F - vU in the frame of an interface moving at v, times dA
// (hllc.cpp:12-39 with starState rel_sph.cpp:397-450).  The four branch tests
// are independent ifs in the reference and stay so.
template <class Cfg>
GB_HD void hllc_flux(const FState<Cfg> &L, const FState<Cfg> &R, const Waves &w, double v, double dA,
                     double *flux) {
  const double lS = w.lS;
  auto star = [&](const FState<Cfg> &Sin, double lbda, double *out_cons) {
    const double m = Sin.cons[SS1];
    const double vv = Sin.v;
    const double p = Sin.prim[PPP];
    const double D = Sin.cons[DEN];
    const double E = Sin.cons[TAU] + Sin.cons[DEN];
    const double A = lbda * E - m;
    const double B = m * (lbda - vv) - p;
    const double pS = (A * lS - B) / (1. - lbda * lS);
    double k;
    if (Cfg::FAST) {
      const double rk = 1. / (lbda - lS);
      k = (lbda - vv) * rk;
      out_cons[SS1] = (m * (lbda - vv) + pS - p) * rk;
      out_cons[TAU] = (E * (lbda - vv) + pS * lS - p * vv) * rk - D * k;
    } else {  // rel_sph.cpp:433-442
      k = (lbda - vv) / (lbda - lS);
      out_cons[SS1] = (m * (lbda - vv) + pS - p) / (lbda - lS);
      out_cons[TAU] = (E * (lbda - vv) + pS * lS - p * vv) / (lbda - lS) - D * k;
    }
    out_cons[DEN] = D * k;
    out_cons[SS2] = 0.;
#pragma unroll
    for (int t = TR1; t < Cfg::NQ; ++t) out_cons[t] = Sin.cons[t] * k;
  };
  if (v < w.lL) {
#pragma unroll
    for (int q = 0; q < Cfg::NQ; ++q) flux[q] = L.flux[q] - v * L.cons[q];
  }
  if (w.lL <= v && v < lS) {
    double sc[Cfg::NQ];
    star(L, w.lL, sc);
#pragma unroll
    for (int q = 0; q < Cfg::NQ; ++q) flux[q] = L.flux[q] + w.lL * (sc[q] - L.cons[q]) - v * sc[q];
  }
  if (lS <= v && v < w.lR) {
    double sc[Cfg::NQ];
    star(R, w.lR, sc);
#pragma unroll
    for (int q = 0; q < Cfg::NQ; ++q) flux[q] = R.flux[q] + w.lR * (sc[q] - R.cons[q]) - v * sc[q];
  }
  if (w.lR <= v) {
#pragma unroll
    for (int q = 0; q < Cfg::NQ; ++q) flux[q] = R.flux[q] - v * R.cons[q];
  }
#pragma unroll
  for (int q = 0; q < Cfg::NQ; ++q) flux[q] *= dA;
}

// ---------------------------------------------------------------------------
// Shock detector (radiation_sph.cpp:41-158), forward direction.  Returns false
// (and leaves *pspec alone) where the reference returns -1 early.
template <class Cfg>
GB_HD bool compute_Sd(const Phys &ph, const FState<Cfg> &S1, const FState<Cfg> &S2, double *Sd,
                      double *pspec) {
  // with eos_ws, the upstream state's Gamma_eff throughout
  const double G = (Cfg::SPH && ph.eos_ws) ? eos_gamma(ph, S1.prim[RHO], S1.prim[PPP]) : ph.gamma_ad;
  const int n_evals = 10;
  const double chi = 0.5;
  double p1 = S1.prim[PPP];
  double p2 = S2.prim[PPP];
  if (fabs(qdiv(p1 - p2, p1)) < 1.e-10 || p1 < p2) {
    *Sd = -1;
    return false;
  }
  double delta_p = p2 - p1;
  double dp = delta_p / (double)n_evals;
  double rho1 = S1.prim[RHO];
  double rho2 = S2.prim[RHO];
  double h1 = 1 + p1 * G / (G - 1.) / rho1;
  double h2 = 1 + p2 * G / (G - 1.) / rho2;
  double lfac2 = S2.lfac;
  double vx1 = S1.v;
  double vx2 = S2.v;
  double v12 = (vx1 - vx2) / (1 - vx1 * vx2);
  double A1 = h1 * 0.;
  double I = 0;
  const double ginv = 1. / G;
#pragma unroll 2
  for (int ip = 0; ip < n_evals; ++ip) {
    double p = p1 + (ip + .5) * dp;
    double rho = rho1 * isentrope_pow(p / p1, ginv);
    double h = 1 + p * G / (G - 1.) / rho;
    double cs = sqrt(G * p / (rho + p * G / (G - 1.)));
    // with A1 = 0 (1D: no transverse velocity) the root is sqrt(h*h) = h exactly
    // (h >= 1, and sqrt of a rounded square is the number itself)
    const double num = A1 == 0. ? h : sqrt(h * h + A1 * A1 * (1. - cs * cs));
    double dI = num / ((h * h + A1 * A1) * rho * cs) * dp;
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
  *pspec = P_SPEC;  // spectral_p with VARIABLE_PSPEC_ disabled
  return true;
}

// ---------------------------------------------------------------------------
// Local synchrotron tracers (radiation_sph.cpp:196-300)

struct SynchConst {
  double Nalpha, Nmp, Nme;
};

template <class Cfg>
GB_HD double gammae2trac(double gme, const double *prim) {
  double lfac = lfac_of(prim[UU1]);
  double rho = prim[RHO];
  if (gme != 0.) return (lfac * pow(rho, 4. / 3.) / gme);
  return 0;
}

template <class Cfg>
GB_HD double gamma_min_init(const Phys &ph, const SynchConst &sc, const double *prim) {
  double rho = prim[RHO];
  double p = prim[PPP];
  double psyn = prim[PSN];
  double gma = state_gamma<Cfg>(ph, prim);
  double h = 1. + p * gma / (gma - 1.) / rho;
  double eps = rho * (h - 1.) / gma;
  double ee = EPS_E * eps;
  double ne = ZETA * rho / sc.Nmp;
  double lfac_av = ee / (ne * sc.Nme);
  return (psyn - 2.) / (psyn - 1.) * lfac_av;
}

// Cell::radiation_injectParticles
template <class Cfg>
GB_HD void inject_particles(const Phys &ph, const SynchConst &sc, double *prim, bool shocked, double pspec) {
  double lfac = lfac_of(prim[UU1]);
  double rho = prim[RHO];
  if (shocked) {
    if (pspec > prim[PSN] || isnan(prim[PSN])) prim[PSN] = pspec;
    prim[GMX] = gammae2trac<Cfg>(GAMMA_MAX_INIT, prim) / (lfac * rho);
    prim[GMN] = gammae2trac<Cfg>(gamma_min_init<Cfg>(ph, sc, prim), prim) / (lfac * rho);
  }
  if (isnan(prim[GMX]) || isnan(prim[GMN])) {  // lim only where it is used
    const double lim = lfac * pow(rho, 4. / 3.) / (lfac * rho);
    if (isnan(prim[GMX])) prim[GMX] = lim;
    if (isnan(prim[GMN])) prim[GMN] = lim;
  }
}

// Cell::radiativeSourceTerms: returns the increment of cons[GMX] and cons[GMN]
template <class Cfg>
GB_HD double radiative_source(const Phys &ph, const SynchConst &sc, const double *prim, double dV, double dt) {
  double rho = prim[RHO];
  double p = prim[PPP];
  double gma = state_gamma<Cfg>(ph, prim);
  double h = 1 + p * gma / (gma - 1.) / rho;
  double eps = rho * (h - 1.) / gma;
  double eB = EPS_B * eps;
  double B = sqrt(8. * PI_ * eB);
  return sc.Nalpha * pow(rho, 4. / 3.) * B * B * dV * dt;
}

// ---------------------------------------------------------------------------
// Geometry (spherical1D.cpp:12-76, cartesian.cpp:11-43)

struct Geom {
  double x, dx, dV, dl, cen;
};

template <class Cfg>
GB_HD Geom make_geom(double x, double dx) {
  Geom g;
  g.x = x;
  g.dx = dx;
  g.dl = dx;
  if (Cfg::SPH) {
    double r = x, dr = dx;
    g.dV = 4. * PI_ * r * r * dr;
    double r2 = r * r;
    double dr2 = dr * dr;
    g.cen = 3. * r * (r2 + dr2) / (3 * r2 + dr2);
  } else {
    g.dV = 1. * dx;
    g.cen = x;
  }
  return g;
}

// Cell::move: geometry between two interfaces
template <class Cfg>
GB_HD Geom geom_between(double xL, double xR) {
  return make_geom<Cfg>((xR + xL) / 2., (xR - xL));
}

template <class Cfg>
GB_HD double iface_area(double x) {
  if (Cfg::SPH) {
    double r = x;
    return 4. * PI_ * r * r;
  }
  return 1.;
}

GB_HD double minmod(double a, double b) {
  if (fabs(a) < fabs(b) && a * b > 0) return a;
  if (fabs(b) < fabs(a) && a * b > 0) return b;
  return 0;
}

}  // namespace gb
