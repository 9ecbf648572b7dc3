// Step-kernel variants of the spherical BM1D configuration (tune.h).
#define GB_TUNE_CFG CfgSph
#define GB_TUNE_CONFIGURE configure_sph
#define GB_TUNE_LAUNCH launch_sph
#include "tune_impl.cuh"
