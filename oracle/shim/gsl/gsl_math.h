/* The reference includes <gsl/gsl_math.h> but uses only <math.h> names from it. TEST INFRASTRUCTURE. */
#ifndef GAMMA_ORACLE_SHIM_GSL_MATH_H
#define GAMMA_ORACLE_SHIM_GSL_MATH_H
#include <math.h>
#endif
