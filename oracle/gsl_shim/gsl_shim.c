/*
 * Oracle-only GSL-API shim implementation (test infrastructure).
 *
 * LU with partial pivoting as used by mdtk/SplineAux.cxx:37-46:
 *   for each column j: pick the first row i >= j with the largest |A[i][j]|,
 *   swap it into place, then for every row below scale A[i][j] /= A[j][j] and
 *   subtract A[i][j] * row j from the trailing part of row i.
 * Solve: x = P b; forward substitution with the unit lower factor
 * (x[i] -= A[i][k] x[k] for k < i, in increasing k); back substitution with
 * the upper factor (x[i] -= A[i][k] x[k] for k > i, in increasing k, then
 * x[i] /= A[i][i]), walking i from the last row up.
 */
#include <stdio.h>
#include <stdlib.h>
#include <math.h>
#include "gsl/gsl_linalg.h"
#include "gsl/gsl_rng.h"
#include "gsl/gsl_randist.h"

gsl_matrix* gsl_matrix_alloc(size_t n1, size_t n2)
{
  gsl_matrix* m = (gsl_matrix*)malloc(sizeof(gsl_matrix));
  m->size1 = n1;
  m->size2 = n2;
  m->data = (double*)calloc(n1 * n2, sizeof(double));
  return m;
}
void gsl_matrix_free(gsl_matrix* m) { if (m) { free(m->data); free(m); } }
void gsl_matrix_set(gsl_matrix* m, size_t i, size_t j, double x) { m->data[i * m->size2 + j] = x; }
double gsl_matrix_get(const gsl_matrix* m, size_t i, size_t j) { return m->data[i * m->size2 + j]; }

gsl_vector* gsl_vector_alloc(size_t n)
{
  gsl_vector* v = (gsl_vector*)malloc(sizeof(gsl_vector));
  v->size = n;
  v->data = (double*)calloc(n, sizeof(double));
  return v;
}
void gsl_vector_free(gsl_vector* v) { if (v) { free(v->data); free(v); } }
void gsl_vector_set(gsl_vector* v, size_t i, double x) { v->data[i] = x; }
double gsl_vector_get(const gsl_vector* v, size_t i) { return v->data[i]; }

gsl_permutation* gsl_permutation_alloc(size_t n)
{
  gsl_permutation* p = (gsl_permutation*)malloc(sizeof(gsl_permutation));
  p->size = n;
  p->data = (size_t*)malloc(n * sizeof(size_t));
  for (size_t i = 0; i < n; i++) p->data[i] = i;
  return p;
}
void gsl_permutation_free(gsl_permutation* p) { if (p) { free(p->data); free(p); } }

int gsl_linalg_LU_decomp(gsl_matrix* A, gsl_permutation* p, int* signum)
{
  const size_t n = A->size1;
  double* a = A->data;
  for (size_t i = 0; i < n; i++) p->data[i] = i;
  *signum = 1;
  for (size_t j = 0; j + 1 < n; j++) {
    double amax = fabs(a[j * n + j]);
    size_t ipiv = j;
    for (size_t i = j + 1; i < n; i++) {
      double aij = fabs(a[i * n + j]);
      if (aij > amax) { amax = aij; ipiv = i; }
    }
    if (ipiv != j) {
      for (size_t k = 0; k < n; k++) {
        double t = a[j * n + k];
        a[j * n + k] = a[ipiv * n + k];
        a[ipiv * n + k] = t;
      }
      size_t t = p->data[j]; p->data[j] = p->data[ipiv]; p->data[ipiv] = t;
      *signum = -(*signum);
    }
    double ajj = a[j * n + j];
    if (ajj != 0.0) {
      for (size_t i = j + 1; i < n; i++) {
        double aij = a[i * n + j] / ajj;
        a[i * n + j] = aij;
        for (size_t k = j + 1; k < n; k++) a[i * n + k] -= aij * a[j * n + k];
      }
    }
  }
  return 0;
}

int gsl_linalg_LU_solve(const gsl_matrix* LU, const gsl_permutation* p,
                        const gsl_vector* b, gsl_vector* x)
{
  const size_t n = LU->size1;
  const double* a = LU->data;
  for (size_t i = 0; i < n; i++) x->data[i] = b->data[p->data[i]];
  for (size_t i = 1; i < n; i++) {
    double t = x->data[i];
    for (size_t k = 0; k < i; k++) t -= a[i * n + k] * x->data[k];
    x->data[i] = t;
  }
  x->data[n - 1] = x->data[n - 1] / a[(n - 1) * n + (n - 1)];
  for (size_t ii = n - 1; ii-- > 0;) {
    double t = x->data[ii];
    for (size_t k = ii + 1; k < n; k++) t -= a[ii * n + k] * x->data[k];
    x->data[ii] = t / a[ii * n + ii];
  }
  return 0;
}

static const gsl_rng_type ranlxd2_type = { "ranlxd2 (oracle stub)" };
const gsl_rng_type* gsl_rng_ranlxd2 = &ranlxd2_type;

gsl_rng* gsl_rng_alloc(const gsl_rng_type* T)
{
  gsl_rng* r = (gsl_rng*)malloc(sizeof(gsl_rng));
  r->type = T;
  r->seed = 0;
  return r;
}
void gsl_rng_set(gsl_rng* r, unsigned long seed) { r->seed = seed; }
void gsl_rng_free(gsl_rng* r) { free(r); }

void gsl_ran_dir_3d(const gsl_rng* r, double* x, double* y, double* z)
{
  (void)r; (void)x; (void)y; (void)z;
  fprintf(stderr, "oracle gsl shim: gsl_ran_dir_3d is not available\n");
  abort();
}
