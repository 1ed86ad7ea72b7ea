/* Stand-in for GSL's gsl_statistics_float.h (the median of src/median.c),
 * implemented by oracle/refshim/refshim_gsl.c.  Test infrastructure only. */
#ifndef REFSHIM_GSL_STATISTICS_FLOAT_H
#define REFSHIM_GSL_STATISTICS_FLOAT_H
#include <stddef.h>
double gsl_stats_float_median(float data[], const size_t stride, const size_t n);
#endif
