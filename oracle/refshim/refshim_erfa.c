/* ERFA stand-in (declarations in oracle/refshim/erfa.h): the angle
 * conversions and the separation that src/misc_utils.c calls, from their
 * published definitions (ERFA / SOFA documentation).  Reached only for
 * observations with a telescope name.  Test infrastructure only. */
#include <math.h>
#include <stdlib.h>

#define DAS2R (4.848136811095359935899141e-6)   /* arcseconds to radians */
#define DS2R (7.272205216643039903848712e-5)    /* seconds of time to radians */

int eraAf2a(char s, int ideg, int iamin, double asec, double *rad)
{
    *rad = (s == '-' ? -1.0 : 1.0) *
           (60.0 * (60.0 * (double) abs(ideg) + (double) abs(iamin)) + fabs(asec)) * DAS2R;
    if (ideg < 0 || ideg > 359) return 1;
    if (iamin < 0 || iamin > 59) return 2;
    if (asec < 0.0 || asec >= 60.0) return 3;
    return 0;
}

int eraTf2a(char s, int ihour, int imin, double sec, double *rad)
{
    *rad = (s == '-' ? -1.0 : 1.0) *
           (60.0 * (60.0 * (double) abs(ihour) + (double) abs(imin)) + fabs(sec)) * DS2R;
    if (ihour < 0 || ihour > 23) return 1;
    if (imin < 0 || imin > 59) return 2;
    if (sec < 0.0 || sec >= 60.0) return 3;
    return 0;
}

/* angle between two directions given as (longitude, latitude) pairs */
double eraSeps(double al, double ap, double bl, double bp)
{
    const double a[3] = {cos(ap) * cos(al), cos(ap) * sin(al), sin(ap)};
    const double b[3] = {cos(bp) * cos(bl), cos(bp) * sin(bl), sin(bp)};
    const double c[3] = {a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2],
                         a[0] * b[1] - a[1] * b[0]};
    const double ss = sqrt(c[0] * c[0] + c[1] * c[1] + c[2] * c[2]);
    const double cs = a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
    return (ss != 0.0 || cs != 0.0) ? atan2(ss, cs) : 0.0;
}

