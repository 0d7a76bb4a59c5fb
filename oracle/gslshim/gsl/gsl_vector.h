/* GSL-API shim: included by the reference but no vector routine is called. */
#ifndef HEOM_GSLSHIM_VECTOR_H
#define HEOM_GSLSHIM_VECTOR_H
#include "gsl_complex.h"
#endif
