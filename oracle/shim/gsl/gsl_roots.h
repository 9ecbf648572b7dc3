/*
 * The slice of the GSL root-finding interface that the GAMMA reference calls
 * (src/Hydro/rel_sph.cpp:219-283, src/Hydro/rel_cart.cpp:131-195), mapped onto
 * the oracle's own Brent solver (oracle/brent.c).  TEST INFRASTRUCTURE: it lets
 * the unmodified reference sources compile into oracle/_ref without GSL.
 */
#ifndef GAMMA_ORACLE_SHIM_GSL_ROOTS_H
#define GAMMA_ORACLE_SHIM_GSL_ROOTS_H

#include <stdio.h>
#include <stdlib.h>
#include "gsl_errno.h"
#include "../../brent.h"

typedef struct {
  double (*function)(double x, void *params);
  void *params;
} gsl_function;

typedef struct { const char *name; } gsl_root_fsolver_type;
typedef struct { oracle_brent state; } gsl_root_fsolver;

static const gsl_root_fsolver_type gamma_shim_brent_type = {"brent"};
static const gsl_root_fsolver_type *gsl_root_fsolver_brent = &gamma_shim_brent_type;

static inline gsl_root_fsolver *gsl_root_fsolver_alloc(const gsl_root_fsolver_type *T) {
  (void)T;
  return (gsl_root_fsolver *)calloc(1, sizeof(gsl_root_fsolver));
}
static inline void gsl_root_fsolver_free(gsl_root_fsolver *s) { free(s); }

/* GSL's default error handler aborts when the end points do not straddle zero. */
static inline int gsl_root_fsolver_set(gsl_root_fsolver *s, gsl_function *f, double lo, double hi) {
  if (oracle_brent_set(&s->state, f->function, f->params, lo, hi) != 0) {
    fprintf(stderr, "oracle GSL shim: endpoints do not straddle y=0\n");
    abort();
  }
  return GSL_SUCCESS;
}
static inline int gsl_root_fsolver_iterate(gsl_root_fsolver *s) { return oracle_brent_iterate(&s->state); }
static inline double gsl_root_fsolver_root(const gsl_root_fsolver *s) { return s->state.b; }
static inline double gsl_root_fsolver_x_lower(const gsl_root_fsolver *s) { return s->state.lower; }
static inline double gsl_root_fsolver_x_upper(const gsl_root_fsolver *s) { return s->state.upper; }
static inline int gsl_root_test_interval(double lo, double hi, double epsabs, double epsrel) {
  return oracle_brent_continue(lo, hi, epsabs, epsrel) ? GSL_CONTINUE : GSL_SUCCESS;
}

#endif
