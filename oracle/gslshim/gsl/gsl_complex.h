/* GSL-API shim (test infrastructure only).
 *
 * GSL 2.8 (the version the reference pins in INSTALL.md:16) is not installed
 * on this machine.  This header set restates the small part of the GSL API
 * that the reference CPU path (etoheom-cpu/lib/*.cpp, src/CPU_2DES.cpp) calls,
 * so that those sources compile unmodified into oracle/_ref/.  Arithmetic
 * follows the published definitions of each routine (see gslshim.c). */
#ifndef HEOM_GSLSHIM_COMPLEX_H
#define HEOM_GSLSHIM_COMPLEX_H

typedef struct { double dat[2]; } gsl_complex;

#define GSL_REAL(z) ((z).dat[0])
#define GSL_IMAG(z) ((z).dat[1])
#define GSL_SET_COMPLEX(zp, x, y) do { (zp)->dat[0] = (x); (zp)->dat[1] = (y); } while (0)

#endif
