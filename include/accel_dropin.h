/*
 * accel_dropin.h -- the accelsearch hot path under the reference's own names
 * (libaccel_dropin.so).
 *
 * libaccel_dropin.so exports the functions of PRESTO's include/accel.h that
 * the accelsearch main loop calls (src/accelsearch.c:140-224), with the
 * reference's signatures, ownership rules and data layout, computed by the
 * B200 engine (libaccel_b200.so, include/accel_b200.h).  Linked ahead of
 * libpresto, or preloaded (LD_PRELOAD) into an installed accelsearch, it
 * takes those calls over; every other libpresto function (create_accelobs,
 * candidate polishing, output) stays the reference's own.
 *
 *   create_subharminfos        include/accel.h:134   src/accel_utils.c:240-305
 *   free_subharminfos          include/accel.h:135   src/accel_utils.c:308-327
 *   subharm_fderivs_vol        include/accel.h:147   src/accel_utils.c:1024-1198
 *   copy_ffdotpows             include/accel.h:150   src/accel_utils.c:1200-1217
 *   fund_to_ffdotplane         include/accel.h:151   src/accel_utils.c:1219-1233
 *   inmem_add_ffdotpows        include/accel.h:152   src/accel_utils.c:1312-1361
 *   fund_to_ffdotplane_trans   include/accel.h:154   src/accel_utils.c:1236-1250
 *   inmem_add_ffdotpows_trans  include/accel.h:155   src/accel_utils.c:1364-1409
 *   free_ffdotpows             include/accel.h:157   src/accel_utils.c:1253-1259
 *   add_ffdotpows_ptrs         include/accel.h:158   src/accel_utils.c:1284-1309
 *   add_ffdotpows              include/accel.h:160   src/accel_utils.c:1261-1282
 *   search_ffdotpows           include/accel.h:162   src/accel_utils.c:1412-1452
 *
 * The structures below repeat the reference's member order and types
 * (include/accel.h:37-130, include/ransomfft.h:13-16, glib's GSList) so that
 * objects pass between the reference's code and this library unchanged.
 *
 * Semantics kept from the reference:
 *  - subharm_fderivs_vol and copy_ffdotpows return a malloc'd ffdotpows whose
 *    powers are a three-level [numws][numzs][numrs] array over one contiguous
 *    block (gen_f3Darr's layout), valid host memory on return; free it with
 *    free_ffdotpows.  rinds / zinds point into the subharminfo, which each
 *    call on the same subharminfo overwrites (calls are not re-entrant).
 *  - add_ffdotpows / add_ffdotpows_ptrs and inmem_add_ffdotpows(_trans)
 *    update the fundamental's host powers in place.
 *  - fund_to_ffdotplane(_trans) copy the block into obs->ffdotplane (when the
 *    caller allocated it) in the reference's [z][r] (or [r][z]) layout, and
 *    into the engine's device copy of the full plane, which
 *    inmem_add_ffdotpows(_trans) read.
 *  - search_ffdotpows inserts every crossing of obs->powcut into the caller's
 *    GSList of accelcand in the reference's visit order with the reference's
 *    insertion rule, and writes the .txtcand line of every insertion that
 *    adds a candidate to obs->workfile (not for .dat input).
 *  - errors print a message and exit(1), as the reference's do.
 * Differences: kern[w][z].data of a subharminfo is NULL (the FFT'd templates
 * live on the device at the engine's transform length); the spectrum is
 * copied to the device at the first subharm_fderivs_vol after
 * create_subharminfos (later edits of obs->fft are not seen).  The engine
 * context is one per process, on device 0 or $ACCEL_B200_DEVICE; the
 * library is not thread-safe (the reference's driver calls it from one
 * thread).
 */
#ifndef ACCEL_DROPIN_H
#define ACCEL_DROPIN_H

#include <stdio.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct { float r, i; } fcomplex;

typedef struct _GSList GSList;
struct _GSList {
    void *data;
    GSList *next;
};

typedef struct accelobs {
    long long N, numbins, lobin, highestbin;
    int maxkernlen, corr_uselen, fftlen, numharmstages, numz, numw, numbetween;
    int numzap, dat_input, mmap_file, inmem, norm_type;
    double dt, T, rlo, rhi, dr, zlo, zhi, dz, wlo, whi, dw, baryv;
    float nph, sigma;
    float *powcut;              /* [numharmstages] */
    float *ffdotplane;          /* in-memory plane, [numz][(highestbin + corr_uselen) * 2] */
    double *lobins, *hibins;
    long long *numindep;        /* [numharmstages] */
    FILE *fftfile, *workfile;
    fcomplex *fft;              /* mapped or in-memory spectrum, bin lobin first */
    char *rootfilenm, *candnm, *accelnm, *workfilenm;
    int use_harmonic_polishing;
} accelobs;

typedef struct accelcand {
    float power, sigma;
    int numharm;
    double r, z, w;
    double *pows, *hirs, *hizs, *hiws;
    void *derivs;               /* rderivs[numharm] once polished */
} accelcand;

typedef struct kernel {
    int z, w, fftlen, numgoodbins, numbetween, kern_half_width;
    fcomplex *data;
} kernel;

typedef struct subharminfo {
    int numharm, harmnum, zmax, wmax, numkern_zdim, numkern_wdim, numkern;
    kernel **kern;              /* [numkern_wdim][numkern_zdim] */
    unsigned short *rinds, *zinds;
} subharminfo;

typedef struct ffdotpows {
    long long rlo;
    int zlo, wlo, numrs, numzs, numws;
    float ***powers;            /* [numws][numzs][numrs] */
    unsigned short *rinds, *zinds;
} ffdotpows;

subharminfo **create_subharminfos(accelobs *obs);
void free_subharminfos(accelobs *obs, subharminfo **shis);
ffdotpows *subharm_fderivs_vol(int numharm, int harmnum, double fullrlo, double fullrhi,
                               subharminfo *shi, accelobs *obs);
ffdotpows *copy_ffdotpows(ffdotpows *orig);
void fund_to_ffdotplane(ffdotpows *ffd, accelobs *obs);
void inmem_add_ffdotpows(ffdotpows *fundamental, accelobs *obs, int numharm, int harmnum);
void fund_to_ffdotplane_trans(ffdotpows *ffd, accelobs *obs);
void inmem_add_ffdotpows_trans(ffdotpows *fundamental, accelobs *obs, int numharm, int harmnum);
void free_ffdotpows(ffdotpows *ffd);
void add_ffdotpows_ptrs(ffdotpows *fundamental, ffdotpows *subharmonic, int numharm, int harmnum);
void add_ffdotpows(ffdotpows *fundamental, ffdotpows *subharmonic, int numharm, int harmnum);
GSList *search_ffdotpows(ffdotpows *ffdot, int numharm, accelobs *obs, GSList *cands);

#ifdef __cplusplus
}
#endif

#endif
