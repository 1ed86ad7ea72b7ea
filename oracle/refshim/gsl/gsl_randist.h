/* Declaration-only stand-in for GSL's gsl_randist.h (src/zapping.c).  Test
 * infrastructure only. */
#ifndef REFSHIM_GSL_RANDIST_H
#define REFSHIM_GSL_RANDIST_H
#include "gsl_rng.h"
double gsl_ran_gaussian(const gsl_rng *r, double sigma);
double gsl_ran_ugaussian(const gsl_rng *r);
double gsl_ran_exponential(const gsl_rng *r, double mu);
#endif
