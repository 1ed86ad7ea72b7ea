/* Stand-in for GSL's gsl_vector.h (the calls in src/maximize_rz.c),
 * implemented by oracle/refshim/refshim_gsl.c.  Test infrastructure only. */
#ifndef REFSHIM_GSL_VECTOR_H
#define REFSHIM_GSL_VECTOR_H
#include <stddef.h>
typedef struct {
    size_t size;
    size_t stride;
    double *data;
    void *block;
    int owner;
} gsl_vector;
gsl_vector *gsl_vector_alloc(size_t n);
void gsl_vector_free(gsl_vector *v);
double gsl_vector_get(const gsl_vector *v, size_t i);
void gsl_vector_set(gsl_vector *v, size_t i, double x);
void gsl_vector_set_all(gsl_vector *v, double x);
#endif
