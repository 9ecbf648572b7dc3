/*
 * Brent's zeroin (Brent 1973, ch. 4), one step per call.  TEST INFRASTRUCTURE.
 * See brent.h for why the oracle carries its own root finder.
 */
#include "brent.h"

#include <float.h>
#include <math.h>

static int same_sign(double x, double y) { return (x > 0.0 && y > 0.0) || (x < 0.0 && y < 0.0); }

static void update_bracket(oracle_brent *s) {
  if (s->fb == 0.0) {
    s->lower = s->upper = s->b;
  } else if (s->b < s->c) {
    s->lower = s->b;
    s->upper = s->c;
  } else {
    s->lower = s->c;
    s->upper = s->b;
  }
}

int oracle_brent_set(oracle_brent *s, oracle_fn f, void *params, double lo, double hi) {
  s->f = f;
  s->params = params;
  s->a = lo;
  s->b = hi;
  s->fa = f(lo, params);
  s->fb = f(hi, params);
  if (same_sign(s->fa, s->fb)) return -1;
  s->c = s->a;
  s->fc = s->fa;
  s->d = s->b - s->a;
  s->e = s->d;
  update_bracket(s);
  return 0;
}

int oracle_brent_iterate(oracle_brent *s) {
  /* keep b the better end */
  if (fabs(s->fc) < fabs(s->fb)) {
    s->a = s->b;
    s->b = s->c;
    s->c = s->a;
    s->fa = s->fb;
    s->fb = s->fc;
    s->fc = s->fa;
  }
  const double tol = 2.0 * DBL_EPSILON * fabs(s->b);
  const double m = 0.5 * (s->c - s->b);
  if (s->fb == 0.0 || fabs(m) <= tol) {
    update_bracket(s);
    return 0;
  }

  if (fabs(s->e) < tol || fabs(s->fa) <= fabs(s->fb)) {
    s->d = m; /* bisection */
    s->e = m;
  } else {
    double p, q, r;
    const double sr = s->fb / s->fa;
    if (s->a == s->c) { /* secant */
      p = 2.0 * m * sr;
      q = 1.0 - sr;
    } else { /* inverse quadratic interpolation */
      q = s->fa / s->fc;
      r = s->fb / s->fc;
      p = sr * (2.0 * m * q * (q - r) - (s->b - s->a) * (r - 1.0));
      q = (q - 1.0) * (r - 1.0) * (sr - 1.0);
    }
    if (p > 0.0) q = -q; else p = -p;
    if (2.0 * p < 3.0 * m * q - fabs(tol * q) && p < fabs(0.5 * s->e * q)) {
      s->e = s->d;
      s->d = p / q;
    } else {
      s->d = m;
      s->e = m;
    }
  }

  s->a = s->b;
  s->fa = s->fb;
  if (fabs(s->d) > tol) s->b += s->d;
  else s->b += (m > 0.0 ? tol : -tol);
  s->fb = s->f(s->b, s->params);

  if (same_sign(s->fb, s->fc)) {
    s->c = s->a;
    s->fc = s->fa;
    s->d = s->b - s->a;
    s->e = s->d;
  }
  update_bracket(s);
  return 0;
}

/* Process-wide replacement of the callers' relative stopping tolerance (0:
 * keep theirs).  Lets the compiled reference, whose cons2prim stops at a fixed
 * 1e-13 bracket, be run to convergence so that its solver noise can be told
 * apart from differences in the rest of the step. */
static double g_epsrel_override = 0.0;

void oracle_brent_override_epsrel(double epsrel) { g_epsrel_override = epsrel; }

int oracle_brent_continue(double lo, double hi, double epsabs, double epsrel) {
  if (g_epsrel_override > 0.0) {  // converge: the relative tolerance only
    epsrel = g_epsrel_override;
    epsabs = 0.0;
  }
  double min_abs;
  if ((lo > 0.0 && hi > 0.0) || (lo < 0.0 && hi < 0.0))
    min_abs = fmin(fabs(lo), fabs(hi));
  else
    min_abs = 0.0;
  const double tolerance = epsabs + epsrel * min_abs;
  return !(fabs(hi - lo) < tolerance);
}
