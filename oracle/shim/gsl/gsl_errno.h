/* Status codes of the GSL root-finding shim (oracle/shim/gsl/gsl_roots.h). TEST INFRASTRUCTURE. */
#ifndef GAMMA_ORACLE_SHIM_GSL_ERRNO_H
#define GAMMA_ORACLE_SHIM_GSL_ERRNO_H
#define GSL_SUCCESS 0
#define GSL_CONTINUE (-2)
#endif
