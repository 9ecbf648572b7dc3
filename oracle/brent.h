/*
 * Bracketing root finder for the CPU oracle.  TEST INFRASTRUCTURE, not product.
 *
 * The GAMMA reference recovers the pressure in FluidState::cons2prim with the GNU
 * Scientific Library's Brent solver (src/Hydro/rel_sph.cpp:252-285,
 * src/Hydro/rel_cart.cpp:164-197).  GSL is not vendored and its version is not
 * pinned by the reference (no lockfile; doc/gsl_on_isambard.txt:1 only links a
 * wiki), and it is absent from this image.  This file restates the published
 * algorithm -- R. P. Brent, "Algorithms for Minimization without Derivatives"
 * (1973), ch. 4, procedure "zeroin": inverse quadratic interpolation / secant
 * steps guarded by bisection, on a bracket [b, c] with f(b) f(c) <= 0 --
 * exposed one iteration at a time like the GSL fsolver interface the reference
 * drives.  Both the oracle C restatement and the compiled reference
 * (through oracle/shim/gsl/gsl_roots.h) use this one implementation, so the two
 * oracles agree bit for bit; neither reproduces GSL's own iterates.
 */
#ifndef GAMMA_ORACLE_BRENT_H
#define GAMMA_ORACLE_BRENT_H

#ifdef __cplusplus
extern "C" {
#endif

typedef double (*oracle_fn)(double x, void *params);

typedef struct {
  oracle_fn f;
  void *params;
  double a, b, c;     /* previous iterate, best estimate, contrapoint */
  double fa, fb, fc;
  double d, e;        /* last and second-to-last step */
  double lower, upper;
} oracle_brent;

/* Returns 0 on success, -1 if f(lo), f(hi) do not straddle zero. */
int oracle_brent_set(oracle_brent *s, oracle_fn f, void *params, double lo, double hi);
/* One zeroin step.  Returns 0. */
int oracle_brent_iterate(oracle_brent *s);
/* 1 while |hi-lo| >= epsabs + epsrel*min(|lo|,|hi|) (0 if the bracket spans 0). */
int oracle_brent_continue(double lo, double hi, double epsabs, double epsrel);
/* Replace every caller's relative tolerance by epsrel (> 0), or restore them (0). */
void oracle_brent_override_epsrel(double epsrel);

#ifdef __cplusplus
}
#endif

#endif
