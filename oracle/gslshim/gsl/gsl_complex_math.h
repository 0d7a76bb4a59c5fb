/* GSL-API shim: complex scalar arithmetic (test infrastructure only). */
#ifndef HEOM_GSLSHIM_COMPLEX_MATH_H
#define HEOM_GSLSHIM_COMPLEX_MATH_H
#include "gsl_complex.h"
#ifdef __cplusplus
extern "C" {
#endif

gsl_complex gsl_complex_rect(double x, double y);
gsl_complex gsl_complex_polar(double r, double theta);
gsl_complex gsl_complex_add(gsl_complex a, gsl_complex b);
gsl_complex gsl_complex_sub(gsl_complex a, gsl_complex b);
gsl_complex gsl_complex_mul(gsl_complex a, gsl_complex b);
gsl_complex gsl_complex_div(gsl_complex a, gsl_complex b);
gsl_complex gsl_complex_mul_real(gsl_complex a, double x);
double gsl_complex_abs(gsl_complex z);

#ifdef __cplusplus
}
#endif
#endif
