/* Prints the size and member offsets of the structures that cross the
 * accel.h boundary (accelobs, accelcand, kernel, subharminfo, ffdotpows,
 * fcomplex, GSList).  Compiled once against the reference's include/accel.h
 * (oracle/build_ref.sh, into oracle/_ref/accel_layout.txt) and once against
 * include/accel_dropin.h (-DDROPIN, tests/test_cpu_dropin.py): the two
 * listings must be identical for libaccel_dropin.so to exchange objects with
 * the reference's code.  Test infrastructure only. */
#include <stddef.h>
#include <stdio.h>
#ifdef DROPIN
#include "accel_dropin.h"
#else
#include "accel.h"
#endif

#define SZ(T) printf("sizeof %s %zu\n", #T, sizeof(T))
#define OFF(T, m) printf("offsetof %s.%s %zu\n", #T, #m, offsetof(T, m))

int main(void)
{
    SZ(fcomplex); OFF(fcomplex, r); OFF(fcomplex, i);
    SZ(GSList); OFF(GSList, data); OFF(GSList, next);
    SZ(accelobs);
    OFF(accelobs, N); OFF(accelobs, numbins); OFF(accelobs, lobin); OFF(accelobs, highestbin);
    OFF(accelobs, maxkernlen); OFF(accelobs, corr_uselen); OFF(accelobs, fftlen);
    OFF(accelobs, numharmstages); OFF(accelobs, numz); OFF(accelobs, numw);
    OFF(accelobs, numbetween); OFF(accelobs, numzap); OFF(accelobs, dat_input);
    OFF(accelobs, mmap_file); OFF(accelobs, inmem); OFF(accelobs, norm_type);
    OFF(accelobs, dt); OFF(accelobs, T); OFF(accelobs, rlo); OFF(accelobs, rhi);
    OFF(accelobs, dr); OFF(accelobs, zlo); OFF(accelobs, zhi); OFF(accelobs, dz);
    OFF(accelobs, wlo); OFF(accelobs, whi); OFF(accelobs, dw); OFF(accelobs, baryv);
    OFF(accelobs, nph); OFF(accelobs, sigma); OFF(accelobs, powcut); OFF(accelobs, ffdotplane);
    OFF(accelobs, lobins); OFF(accelobs, hibins); OFF(accelobs, numindep);
    OFF(accelobs, fftfile); OFF(accelobs, workfile); OFF(accelobs, fft);
    OFF(accelobs, rootfilenm); OFF(accelobs, candnm); OFF(accelobs, accelnm);
    OFF(accelobs, workfilenm); OFF(accelobs, use_harmonic_polishing);
    SZ(accelcand);
    OFF(accelcand, power); OFF(accelcand, sigma); OFF(accelcand, numharm); OFF(accelcand, r);
    OFF(accelcand, z); OFF(accelcand, w); OFF(accelcand, pows); OFF(accelcand, hirs);
    OFF(accelcand, hizs); OFF(accelcand, hiws); OFF(accelcand, derivs);
    SZ(kernel);
    OFF(kernel, z); OFF(kernel, w); OFF(kernel, fftlen); OFF(kernel, numgoodbins);
    OFF(kernel, numbetween); OFF(kernel, kern_half_width); OFF(kernel, data);
    SZ(subharminfo);
    OFF(subharminfo, numharm); OFF(subharminfo, harmnum); OFF(subharminfo, zmax);
    OFF(subharminfo, wmax); OFF(subharminfo, numkern_zdim); OFF(subharminfo, numkern_wdim);
    OFF(subharminfo, numkern); OFF(subharminfo, kern); OFF(subharminfo, rinds);
    OFF(subharminfo, zinds);
    SZ(ffdotpows);
    OFF(ffdotpows, rlo); OFF(ffdotpows, zlo); OFF(ffdotpows, wlo); OFF(ffdotpows, numrs);
    OFF(ffdotpows, numzs); OFF(ffdotpows, numws); OFF(ffdotpows, powers); OFF(ffdotpows, rinds);
    OFF(ffdotpows, zinds);
    return 0;
}
