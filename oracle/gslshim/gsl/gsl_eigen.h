/* GSL-API shim: included by the reference but no eigen routine is called. */
#ifndef HEOM_GSLSHIM_EIGEN_H
#define HEOM_GSLSHIM_EIGEN_H
#include "gsl_matrix.h"
#endif
