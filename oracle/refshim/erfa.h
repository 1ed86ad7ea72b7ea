/* Declaration-only stand-in for ERFA's erfa.h: src/misc_utils.c includes it;
 * the functions build_ref.sh keeps from that file call none of these.  Test
 * infrastructure only. */
#ifndef REFSHIM_ERFA_H
#define REFSHIM_ERFA_H
int eraAf2a(char s, int ideg, int iamin, double asec, double *rad);
int eraTf2a(char s, int ihour, int imin, double sec, double *rad);
int eraCal2jd(int iy, int im, int id, double *djm0, double *djm);
int eraJd2cal(double dj1, double dj2, int *iy, int *im, int *id, double *fd);
double eraSeps(double al, double ap, double bl, double bp);
#endif
