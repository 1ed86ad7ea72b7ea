/* Declaration-only stand-in for GSL's gsl_rng.h: src/zapping.c (birdie
 * zapping, reached only with accelsearch -zaplist) includes it; MT19937 is
 * in oracle/refshim/refshim_gsl.c.  Test infrastructure only. */
#ifndef REFSHIM_GSL_RNG_H
#define REFSHIM_GSL_RNG_H
typedef struct gsl_rng_type gsl_rng_type;
typedef struct gsl_rng gsl_rng;
extern const gsl_rng_type *gsl_rng_mt19937;
extern const gsl_rng_type *gsl_rng_default;
gsl_rng *gsl_rng_alloc(const gsl_rng_type *T);
void gsl_rng_free(gsl_rng *r);
void gsl_rng_set(const gsl_rng *r, unsigned long int seed);
unsigned long int gsl_rng_get(const gsl_rng *r);
double gsl_rng_uniform(const gsl_rng *r);
const gsl_rng_type *gsl_rng_env_setup(void);
#endif
