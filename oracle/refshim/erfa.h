/* Declaration-only stand-in for ERFA's erfa.h: src/misc_utils.c and
 * src/barycenter.c include it; the functions build_ref.sh keeps from those
 * files (the angle conversions of refshim_erfa.c aside) call none of these.
 * Prototypes follow ERFA's published API.  Test infrastructure only. */
#ifndef REFSHIM_ERFA_H
#define REFSHIM_ERFA_H
int eraAf2a(char s, int ideg, int iamin, double asec, double *rad);
int eraTf2a(char s, int ihour, int imin, double sec, double *rad);
int eraCal2jd(int iy, int im, int id, double *djm0, double *djm);
int eraJd2cal(double dj1, double dj2, int *iy, int *im, int *id, double *fd);
double eraSeps(double al, double ap, double bl, double bp);
/* used by src/barycenter.c's barycentring, which the checks never keep */
#define ERFA_DJM0 (2400000.5)
#define ERFA_DAU (149597870.7e3)
#define ERFA_AULT (ERFA_DAU / 299792458.0)
#define ERFA_SRS 1.97412574336e-8
#define ERFA_WGS84 1
int eraEpv00(double date1, double date2, double pvh[2][3], double pvb[2][3]);
double eraEra00(double dj1, double dj2);
void eraPvtob(double elong, double phi, double hm, double xp, double yp, double sp, double theta,
              double pv[2][3]);
void eraTrxpv(double r[3][3], double pv[2][3], double trpv[2][3]);
double eraDtdb(double date1, double date2, double ut, double elong, double u, double v);
double eraPdp(double a[2][3], double b[2][3]);
double eraPm(double p[3]);
void eraS2c(double theta, double phi, double c[3]);
int eraGc2gd(int n, double xyz[3], double *elong, double *phi, double *height);
int eraDat(int iy, int im, int id, double fd, double *deltat);
void eraC2i06a(double date1, double date2, double rc2i[3][3]);
double eraSp00(double date1, double date2);
#endif
