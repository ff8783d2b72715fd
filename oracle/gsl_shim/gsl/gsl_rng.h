/*
 * Oracle-only GSL-API shim: random-number stubs.
 *
 * SimLoop::executeMain allocates and frees a generator it never draws from on
 * the integration path (mdtk/SimLoop.cxx:228-230, 471).  The only consumers of
 * random numbers, heatUpEveryAtom/displaceEveryAtom (SimLoop.cxx:1250-1275),
 * are never called by the oracle harness; gsl_ran_dir_3d aborts if they are.
 */
#ifndef MDG_ORACLE_GSL_RNG_SHIM_H
#define MDG_ORACLE_GSL_RNG_SHIM_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct { const char* name; } gsl_rng_type;
typedef struct { const gsl_rng_type* type; unsigned long seed; } gsl_rng;

extern const gsl_rng_type* gsl_rng_ranlxd2;

gsl_rng* gsl_rng_alloc(const gsl_rng_type* T);
void gsl_rng_set(gsl_rng* r, unsigned long seed);
void gsl_rng_free(gsl_rng* r);

#ifdef __cplusplus
}
#endif

#endif
