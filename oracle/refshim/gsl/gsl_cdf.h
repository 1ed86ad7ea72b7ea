/* Stand-in for GSL's gsl_cdf.h (src/characteristics.c), implemented by
 * oracle/refshim/refshim_gsl.c.  Test infrastructure only. */
#ifndef REFSHIM_GSL_CDF_H
#define REFSHIM_GSL_CDF_H
double gsl_cdf_chisq_Q(double x, double nu);
double gsl_cdf_chisq_Qinv(double Q, double nu);
double gsl_cdf_gaussian_Q(double x, double sigma);
double gsl_cdf_gaussian_Qinv(double Q, double sigma);
#endif
