/* GSL-API shim: dense row-major matrices (test infrastructure only). */
#ifndef HEOM_GSLSHIM_MATRIX_H
#define HEOM_GSLSHIM_MATRIX_H
#include <stddef.h>
#include "gsl_complex.h"
#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
  size_t size1, size2, tda;
  double *data;
  int owner;
} gsl_matrix_complex;

typedef struct {
  size_t size1, size2, tda;
  double *data;
  int owner;
} gsl_matrix;

gsl_matrix_complex *gsl_matrix_complex_alloc(size_t n1, size_t n2);
void gsl_matrix_complex_free(gsl_matrix_complex *m);
gsl_complex gsl_matrix_complex_get(const gsl_matrix_complex *m, size_t i, size_t j);
void gsl_matrix_complex_set(gsl_matrix_complex *m, size_t i, size_t j, gsl_complex x);
gsl_complex *gsl_matrix_complex_ptr(gsl_matrix_complex *m, size_t i, size_t j);
void gsl_matrix_complex_set_all(gsl_matrix_complex *m, gsl_complex x);
void gsl_matrix_complex_set_zero(gsl_matrix_complex *m);
int gsl_matrix_complex_memcpy(gsl_matrix_complex *dest, const gsl_matrix_complex *src);
int gsl_matrix_complex_transpose_memcpy(gsl_matrix_complex *dest, const gsl_matrix_complex *src);
int gsl_matrix_complex_add(gsl_matrix_complex *a, const gsl_matrix_complex *b);
int gsl_matrix_complex_sub(gsl_matrix_complex *a, const gsl_matrix_complex *b);
int gsl_matrix_complex_scale(gsl_matrix_complex *a, const gsl_complex x);

double gsl_matrix_get(const gsl_matrix *m, size_t i, size_t j);

#ifdef __cplusplus
}
#endif
#endif
