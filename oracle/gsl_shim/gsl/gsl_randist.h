/*
 * Oracle-only GSL-API shim.  gsl_ran_dir_3d is referenced by
 * SimLoop::heatUpEveryAtom / displaceEveryAtom (mdtk/SimLoop.cxx:1257,1272),
 * which the oracle harness never calls; the shim aborts if it is reached.
 */
#ifndef MDG_ORACLE_GSL_RANDIST_SHIM_H
#define MDG_ORACLE_GSL_RANDIST_SHIM_H
#include "gsl_rng.h"
#ifdef __cplusplus
extern "C" {
#endif
void gsl_ran_dir_3d(const gsl_rng* r, double* x, double* y, double* z);
#ifdef __cplusplus
}
#endif
#endif
