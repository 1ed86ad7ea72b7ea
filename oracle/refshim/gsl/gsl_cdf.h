/* Declaration-only stand-in for GSL's gsl_cdf.h: src/characteristics.c
 * includes it, and the functions oracle/build_ref.sh exports from that file
 * (calc_props, calc_rzwerrs, get_localpower3d, get_derivs3d) call none of
 * these.  Test infrastructure only. */
#ifndef REFSHIM_GSL_CDF_H
#define REFSHIM_GSL_CDF_H
double gsl_cdf_chisq_Q(double x, double nu);
double gsl_cdf_chisq_Qinv(double Q, double nu);
double gsl_cdf_gaussian_Q(double x, double sigma);
double gsl_cdf_gaussian_Qinv(double Q, double sigma);
#endif
