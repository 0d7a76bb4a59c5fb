/* GSL-API shim: the two level-1/level-3 complex BLAS routines the reference
 * path calls (test infrastructure only). */
#ifndef HEOM_GSLSHIM_BLAS_H
#define HEOM_GSLSHIM_BLAS_H
#include "gsl_matrix.h"
#include "gsl_vector.h"
#ifdef __cplusplus
extern "C" {
#endif

enum CBLAS_TRANSPOSE { CblasNoTrans = 111, CblasTrans = 112, CblasConjTrans = 113 };
typedef enum CBLAS_TRANSPOSE CBLAS_TRANSPOSE_t;

int gsl_blas_zgemm(CBLAS_TRANSPOSE_t TransA, CBLAS_TRANSPOSE_t TransB,
                   const gsl_complex alpha, const gsl_matrix_complex *A,
                   const gsl_matrix_complex *B, const gsl_complex beta,
                   gsl_matrix_complex *C);
void cblas_zaxpy(const int N, const void *alpha, const void *X, const int incX,
                 void *Y, const int incY);
void cblas_zscal(const int N, const void *alpha, void *X, const int incX);

#ifdef __cplusplus
}
#endif
#endif
