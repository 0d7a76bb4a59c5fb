/* GSL-API shim: random number generator (MT19937, GSL's default type).
 * Test infrastructure only.  Parity of this stream against a real GSL build
 * is unpinned: GSL is not installed here. */
#ifndef HEOM_GSLSHIM_RNG_H
#define HEOM_GSLSHIM_RNG_H
#ifdef __cplusplus
extern "C" {
#endif

typedef struct { const char *name; } gsl_rng_type;
typedef struct {
  const gsl_rng_type *type;
  unsigned long mt[624];
  int mti;
} gsl_rng;

extern const gsl_rng_type *gsl_rng_default;
extern const gsl_rng_type *gsl_rng_mt19937;
extern unsigned long gsl_rng_default_seed;

const gsl_rng_type *gsl_rng_env_setup(void);
gsl_rng *gsl_rng_alloc(const gsl_rng_type *T);
void gsl_rng_set(gsl_rng *r, unsigned long seed);
void gsl_rng_free(gsl_rng *r);
unsigned long gsl_rng_get(gsl_rng *r);
double gsl_rng_uniform(gsl_rng *r);
double gsl_rng_uniform_pos(gsl_rng *r);

#ifdef __cplusplus
}
#endif
#endif
