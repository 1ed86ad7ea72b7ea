/* Stand-in for GSL's gsl_multimin.h: the derivative-free minimiser API that
 * src/maximize_rz.c drives (nmsimplex2), implemented by
 * oracle/refshim/refshim_gsl.c.  Test infrastructure only. */
#ifndef REFSHIM_GSL_MULTIMIN_H
#define REFSHIM_GSL_MULTIMIN_H
#include <stddef.h>
#include "gsl_vector.h"
typedef struct {
    double (*f)(const gsl_vector *x, void *params);
    size_t n;
    void *params;
} gsl_multimin_function;
typedef struct gsl_multimin_fminimizer_type gsl_multimin_fminimizer_type;
typedef struct {
    const gsl_multimin_fminimizer_type *type;
    gsl_multimin_function *f;
    double fval;
    gsl_vector *x;
    double size;
    void *state;
} gsl_multimin_fminimizer;
extern const gsl_multimin_fminimizer_type *gsl_multimin_fminimizer_nmsimplex2;
gsl_multimin_fminimizer *gsl_multimin_fminimizer_alloc(const gsl_multimin_fminimizer_type *T,
                                                       size_t n);
int gsl_multimin_fminimizer_set(gsl_multimin_fminimizer *s, gsl_multimin_function *f,
                                const gsl_vector *x, const gsl_vector *step_size);
int gsl_multimin_fminimizer_iterate(gsl_multimin_fminimizer *s);
double gsl_multimin_fminimizer_size(const gsl_multimin_fminimizer *s);
void gsl_multimin_fminimizer_free(gsl_multimin_fminimizer *s);
int gsl_multimin_test_size(const double size, double epsabs);
#endif
