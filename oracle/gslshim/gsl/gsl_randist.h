/* GSL-API shim: the two random distributions the reference draws from
 * (test infrastructure only; stream parity with real GSL unpinned). */
#ifndef HEOM_GSLSHIM_RANDIST_H
#define HEOM_GSLSHIM_RANDIST_H
#include "gsl_rng.h"
#ifdef __cplusplus
extern "C" {
#endif

double gsl_ran_gaussian(gsl_rng *r, double sigma);
void gsl_ran_dir_3d(gsl_rng *r, double *x, double *y, double *z);

#ifdef __cplusplus
}
#endif
#endif
