/*
 * Oracle-only GSL-API shim (test infrastructure; never linked into the product).
 *
 * The reference solves its spline-coefficient systems with GSL's LU routines
 * (mdtk/SplineAux.cxx:37-46, 70-92).  GSL is not installed here, so this shim
 * provides exactly the API surface those call sites use: dense row-major
 * matrices/vectors, a permutation, and an LU factorisation with partial
 * pivoting followed by forward/back substitution (the classic GSL
 * gsl_linalg_LU_decomp / gsl_linalg_LU_solve algorithm: column pivot = first
 * row holding the largest |a_ij|, row-wise elimination, unit-lower forward
 * solve, upper back solve).  The oracle's spline coefficients are therefore
 * defined by this elimination order.
 */
#ifndef MDG_ORACLE_GSL_LINALG_SHIM_H
#define MDG_ORACLE_GSL_LINALG_SHIM_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct { size_t size1, size2; double* data; } gsl_matrix;
typedef struct { size_t size; double* data; } gsl_vector;
typedef struct { size_t size; size_t* data; } gsl_permutation;

gsl_matrix* gsl_matrix_alloc(size_t n1, size_t n2);
void gsl_matrix_free(gsl_matrix* m);
void gsl_matrix_set(gsl_matrix* m, size_t i, size_t j, double x);
double gsl_matrix_get(const gsl_matrix* m, size_t i, size_t j);

gsl_vector* gsl_vector_alloc(size_t n);
void gsl_vector_free(gsl_vector* v);
void gsl_vector_set(gsl_vector* v, size_t i, double x);
double gsl_vector_get(const gsl_vector* v, size_t i);

gsl_permutation* gsl_permutation_alloc(size_t n);
void gsl_permutation_free(gsl_permutation* p);

int gsl_linalg_LU_decomp(gsl_matrix* A, gsl_permutation* p, int* signum);
int gsl_linalg_LU_solve(const gsl_matrix* LU, const gsl_permutation* p,
                        const gsl_vector* b, gsl_vector* x);

#ifdef __cplusplus
}
#endif

#endif
