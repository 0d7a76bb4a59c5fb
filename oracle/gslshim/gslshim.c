/* GSL-API shim implementation (test infrastructure only).
 *
 * Restates, from their published definitions, the GSL 2.8 routines that the
 * reference CPU path calls.  Only used to compile the reference's own sources
 * into oracle/_ref/; nothing in the product links it.
 *
 * Arithmetic contract (what the reference's results depend on):
 *  - complex multiply (a*b) = (ar*br - ai*bi, ar*bi + ai*br), no fused ops;
 *  - zgemm, row-major, C = alpha*A*B + beta*C in reference-BLAS loop order:
 *    C is scaled by beta first (beta == 0 clears it), then for each row i and
 *    each inner index l, temp = alpha*A[i][l] is formed once and, unless it is
 *    exactly zero, C[i][j] += temp*B[l][j] is applied for every column j;
 *  - zaxpy: y[i] += (ar*xr - ai*xi, ar*xi + ai*xr), skipped when alpha == 0;
 *  - MT19937 (Matsumoto & Nishimura 1998) with the 2002 seeding recurrence,
 *    seed 0 mapped to 4357; uniform = get / 2^32;
 *  - gaussian: Marsaglia polar method returning sigma*y*sqrt(-2 ln r2 / r2);
 *  - dir_3d: Knuth's method (x,y uniform in the unit disc, z = -1 + 2s). */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include "gsl/gsl_complex.h"
#include "gsl/gsl_complex_math.h"
#include "gsl/gsl_matrix.h"
#include "gsl/gsl_blas.h"
#include "gsl/gsl_rng.h"
#include "gsl/gsl_randist.h"

/* ---- complex scalars ---------------------------------------------------- */
gsl_complex gsl_complex_rect(double x, double y) { gsl_complex z; z.dat[0] = x; z.dat[1] = y; return z; }
gsl_complex gsl_complex_polar(double r, double theta) { return gsl_complex_rect(r * cos(theta), r * sin(theta)); }
gsl_complex gsl_complex_add(gsl_complex a, gsl_complex b) { return gsl_complex_rect(a.dat[0] + b.dat[0], a.dat[1] + b.dat[1]); }
gsl_complex gsl_complex_sub(gsl_complex a, gsl_complex b) { return gsl_complex_rect(a.dat[0] - b.dat[0], a.dat[1] - b.dat[1]); }
gsl_complex gsl_complex_mul(gsl_complex a, gsl_complex b) {
  double ar = a.dat[0], ai = a.dat[1], br = b.dat[0], bi = b.dat[1];
  return gsl_complex_rect(ar * br - ai * bi, ar * bi + ai * br);
}
gsl_complex gsl_complex_div(gsl_complex a, gsl_complex b) {
  /* Smith-free textbook form; only reachable from code the reference has commented out. */
  double d = b.dat[0] * b.dat[0] + b.dat[1] * b.dat[1];
  return gsl_complex_rect((a.dat[0] * b.dat[0] + a.dat[1] * b.dat[1]) / d,
                          (a.dat[1] * b.dat[0] - a.dat[0] * b.dat[1]) / d);
}
gsl_complex gsl_complex_mul_real(gsl_complex a, double x) { return gsl_complex_rect(x * a.dat[0], x * a.dat[1]); }
double gsl_complex_abs(gsl_complex z) { return hypot(z.dat[0], z.dat[1]); }

/* ---- matrices ----------------------------------------------------------- */
gsl_matrix_complex *gsl_matrix_complex_alloc(size_t n1, size_t n2) {
  gsl_matrix_complex *m = (gsl_matrix_complex *)malloc(sizeof *m);
  m->size1 = n1; m->size2 = n2; m->tda = n2; m->owner = 1;
  m->data = (double *)malloc(2 * n1 * n2 * sizeof(double) + 16);
  return m;
}
void gsl_matrix_complex_free(gsl_matrix_complex *m) { if (m) { free(m->data); free(m); } }
gsl_complex gsl_matrix_complex_get(const gsl_matrix_complex *m, size_t i, size_t j) {
  const double *p = m->data + 2 * (i * m->tda + j);
  return gsl_complex_rect(p[0], p[1]);
}
void gsl_matrix_complex_set(gsl_matrix_complex *m, size_t i, size_t j, gsl_complex x) {
  double *p = m->data + 2 * (i * m->tda + j);
  p[0] = x.dat[0]; p[1] = x.dat[1];
}
gsl_complex *gsl_matrix_complex_ptr(gsl_matrix_complex *m, size_t i, size_t j) {
  return (gsl_complex *)(m->data + 2 * (i * m->tda + j));
}
void gsl_matrix_complex_set_all(gsl_matrix_complex *m, gsl_complex x) {
  for (size_t i = 0; i < m->size1; i++)
    for (size_t j = 0; j < m->size2; j++) gsl_matrix_complex_set(m, i, j, x);
}
void gsl_matrix_complex_set_zero(gsl_matrix_complex *m) { gsl_matrix_complex_set_all(m, gsl_complex_rect(0.0, 0.0)); }
int gsl_matrix_complex_memcpy(gsl_matrix_complex *dest, const gsl_matrix_complex *src) {
  if (dest->size1 != src->size1 || dest->size2 != src->size2) abort();
  for (size_t i = 0; i < src->size1; i++)
    for (size_t j = 0; j < src->size2; j++) gsl_matrix_complex_set(dest, i, j, gsl_matrix_complex_get(src, i, j));
  return 0;
}
int gsl_matrix_complex_transpose_memcpy(gsl_matrix_complex *dest, const gsl_matrix_complex *src) {
  if (dest->size1 != src->size2 || dest->size2 != src->size1) abort();
  for (size_t i = 0; i < dest->size1; i++)
    for (size_t j = 0; j < dest->size2; j++) gsl_matrix_complex_set(dest, i, j, gsl_matrix_complex_get(src, j, i));
  return 0;
}
int gsl_matrix_complex_add(gsl_matrix_complex *a, const gsl_matrix_complex *b) {
  for (size_t i = 0; i < a->size1; i++)
    for (size_t j = 0; j < a->size2; j++) {
      double *p = a->data + 2 * (i * a->tda + j);
      const double *q = b->data + 2 * (i * b->tda + j);
      p[0] += q[0]; p[1] += q[1];
    }
  return 0;
}
int gsl_matrix_complex_sub(gsl_matrix_complex *a, const gsl_matrix_complex *b) {
  for (size_t i = 0; i < a->size1; i++)
    for (size_t j = 0; j < a->size2; j++) {
      double *p = a->data + 2 * (i * a->tda + j);
      const double *q = b->data + 2 * (i * b->tda + j);
      p[0] -= q[0]; p[1] -= q[1];
    }
  return 0;
}
int gsl_matrix_complex_scale(gsl_matrix_complex *a, const gsl_complex x) {
  const double xr = x.dat[0], xi = x.dat[1];
  for (size_t i = 0; i < a->size1; i++)
    for (size_t j = 0; j < a->size2; j++) {
      double *p = a->data + 2 * (i * a->tda + j);
      const double ar = p[0], ai = p[1];
      p[0] = ar * xr - ai * xi;
      p[1] = ar * xi + ai * xr;
    }
  return 0;
}
double gsl_matrix_get(const gsl_matrix *m, size_t i, size_t j) { return m->data[i * m->tda + j]; }

/* ---- BLAS --------------------------------------------------------------- */
int gsl_blas_zgemm(CBLAS_TRANSPOSE_t TransA, CBLAS_TRANSPOSE_t TransB, const gsl_complex alpha,
                   const gsl_matrix_complex *A, const gsl_matrix_complex *B, const gsl_complex beta,
                   gsl_matrix_complex *C) {
  if (TransA != CblasNoTrans || TransB != CblasNoTrans) abort(); /* the reference uses NoTrans only */
  const size_t M = C->size1, N = C->size2, K = A->size2;
  if (A->size1 != M || B->size1 != K || B->size2 != N) abort();
  const double ar = alpha.dat[0], ai = alpha.dat[1], br = beta.dat[0], bi = beta.dat[1];
  if (br == 0.0 && bi == 0.0) {
    for (size_t i = 0; i < M; i++)
      for (size_t j = 0; j < N; j++) { double *c = C->data + 2 * (i * C->tda + j); c[0] = 0.0; c[1] = 0.0; }
  } else if (!(br == 1.0 && bi == 0.0)) {
    for (size_t i = 0; i < M; i++)
      for (size_t j = 0; j < N; j++) {
        double *c = C->data + 2 * (i * C->tda + j);
        const double cr = c[0], ci = c[1];
        c[0] = br * cr - bi * ci;
        c[1] = br * ci + bi * cr;
      }
  }
  if (ar == 0.0 && ai == 0.0) return 0;
  for (size_t i = 0; i < M; i++) {
    for (size_t l = 0; l < K; l++) {
      const double *a = A->data + 2 * (i * A->tda + l);
      const double tr = ar * a[0] - ai * a[1];
      const double ti = ar * a[1] + ai * a[0];
      if (tr == 0.0 && ti == 0.0) continue;
      for (size_t j = 0; j < N; j++) {
        const double *b = B->data + 2 * (l * B->tda + j);
        double *c = C->data + 2 * (i * C->tda + j);
        c[0] += tr * b[0] - ti * b[1];
        c[1] += tr * b[1] + ti * b[0];
      }
    }
  }
  return 0;
}

void cblas_zaxpy(const int N, const void *alpha, const void *X, const int incX, void *Y, const int incY) {
  const double ar = ((const double *)alpha)[0], ai = ((const double *)alpha)[1];
  const double *x = (const double *)X;
  double *y = (double *)Y;
  if (fabs(ar) == 0 && fabs(ai) == 0) return;
  int ix = incX > 0 ? 0 : (N - 1) * -incX, iy = incY > 0 ? 0 : (N - 1) * -incY;
  for (int i = 0; i < N; i++) {
    const double xr = x[2 * ix], xi = x[2 * ix + 1];
    y[2 * iy] += (ar * xr - ai * xi);
    y[2 * iy + 1] += (ar * xi + ai * xr);
    ix += incX; iy += incY;
  }
}

void cblas_zscal(const int N, const void *alpha, void *X, const int incX) {
  const double ar = ((const double *)alpha)[0], ai = ((const double *)alpha)[1];
  double *x = (double *)X;
  if (incX <= 0) return;
  for (int i = 0, ix = 0; i < N; i++, ix += incX) {
    const double xr = x[2 * ix], xi = x[2 * ix + 1];
    x[2 * ix] = ar * xr - ai * xi;
    x[2 * ix + 1] = ar * xi + ai * xr;
  }
}

/* ---- RNG ---------------------------------------------------------------- */
static const gsl_rng_type mt_type = {"mt19937"};
const gsl_rng_type *gsl_rng_mt19937 = &mt_type;
const gsl_rng_type *gsl_rng_default = &mt_type;
unsigned long gsl_rng_default_seed = 0;

const gsl_rng_type *gsl_rng_env_setup(void) { gsl_rng_default = &mt_type; return gsl_rng_default; }

void gsl_rng_set(gsl_rng *r, unsigned long s) {
  if (s == 0) s = 4357;
  r->mt[0] = s & 0xffffffffUL;
  for (int i = 1; i < 624; i++)
    r->mt[i] = (1812433253UL * (r->mt[i - 1] ^ (r->mt[i - 1] >> 30)) + (unsigned long)i) & 0xffffffffUL;
  r->mti = 624;
}
gsl_rng *gsl_rng_alloc(const gsl_rng_type *T) {
  gsl_rng *r = (gsl_rng *)calloc(1, sizeof *r);
  r->type = T;
  gsl_rng_set(r, gsl_rng_default_seed);
  return r;
}
void gsl_rng_free(gsl_rng *r) { free(r); }

unsigned long gsl_rng_get(gsl_rng *r) {
  enum { NN = 624, MM = 397 };
  const unsigned long UPPER = 0x80000000UL, LOWER = 0x7fffffffUL;
#define SHIM_MAGIC(y) (((y) & 0x1UL) ? 0x9908b0dfUL : 0UL)
  if (r->mti >= NN) {
    int kk;
    for (kk = 0; kk < NN - MM; kk++) {
      unsigned long y = (r->mt[kk] & UPPER) | (r->mt[kk + 1] & LOWER);
      r->mt[kk] = r->mt[kk + MM] ^ (y >> 1) ^ SHIM_MAGIC(y);
    }
    for (; kk < NN - 1; kk++) {
      unsigned long y = (r->mt[kk] & UPPER) | (r->mt[kk + 1] & LOWER);
      r->mt[kk] = r->mt[kk + (MM - NN)] ^ (y >> 1) ^ SHIM_MAGIC(y);
    }
    unsigned long y = (r->mt[NN - 1] & UPPER) | (r->mt[0] & LOWER);
    r->mt[NN - 1] = r->mt[MM - 1] ^ (y >> 1) ^ SHIM_MAGIC(y);
    r->mti = 0;
  }
#undef SHIM_MAGIC
  unsigned long k = r->mt[r->mti++];
  k ^= (k >> 11);
  k ^= (k << 7) & 0x9d2c5680UL;
  k ^= (k << 15) & 0xefc60000UL;
  k ^= (k >> 18);
  return k & 0xffffffffUL;
}
double gsl_rng_uniform(gsl_rng *r) { return gsl_rng_get(r) / 4294967296.0; }
double gsl_rng_uniform_pos(gsl_rng *r) {
  double x;
  do { x = gsl_rng_uniform(r); } while (x == 0);
  return x;
}

double gsl_ran_gaussian(gsl_rng *r, double sigma) {
  double x, y, r2;
  do {
    x = -1 + 2 * gsl_rng_uniform_pos(r);
    y = -1 + 2 * gsl_rng_uniform_pos(r);
    r2 = x * x + y * y;
  } while (r2 > 1.0 || r2 == 0);
  return sigma * y * sqrt(-2.0 * log(r2) / r2);
}

void gsl_ran_dir_3d(gsl_rng *r, double *x, double *y, double *z) {
  double s, a;
  do {
    *x = -1 + 2 * gsl_rng_uniform(r);
    *y = -1 + 2 * gsl_rng_uniform(r);
    s = (*x) * (*x) + (*y) * (*y);
  } while (s > 1.0);
  *z = -1 + 2 * s;
  a = 2 * sqrt(1 - s);
  *x *= a;
  *y *= a;
}
