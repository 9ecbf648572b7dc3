// Step-kernel variants of the cartesian tube configuration (tune.h).
#define GB_TUNE_CFG CfgCart
#define GB_TUNE_CONFIGURE configure_cart
#define GB_TUNE_LAUNCH launch_cart
#include "tune_impl.cuh"
