/* Oracle-only GSL-API shim: SimLoop.hpp includes this header but uses nothing from it. */
#ifndef MDG_ORACLE_GSL_QRNG_SHIM_H
#define MDG_ORACLE_GSL_QRNG_SHIM_H
#include "gsl_rng.h"
#endif
