/*
 * ab_dedisp.c -- the integer delays of prepsubband's subband dedispersion
 * (host C).
 *
 *   delay_from_dm          src/dispersion.c:30-39
 *   dedisp_delays          src/dispersion.c:54-73 (voverc = 0: doppler()
 *                          multiplies by 1.0, src/barycenter.c:5-12)
 *   subband_delays         src/dispersion.c:103-121
 *   subband_search_delays  src/dispersion.c:124-162
 *   the rounding           src/prepsubband.c:365-390 (NEAREST_LONG of the
 *                          delays in samples; DMs averaged as at :262-270)
 *
 * Channel c's delay inside its subband at the DMs' mean is
 * NEAREST_LONG(subband_search_delay[c] / dt); subband s's offset at DM d is
 * NEAREST_LONG((subband_delay_d[s] - subband_delay_d[nsub - 1]) / (dt downsamp)).
 */
#include <math.h>
#include <stdlib.h>

#include "accel_b200.h"

static double delay_from_dm(double dm, double freq)
{
    if (freq == 0.0) return 0.0;
    return dm / (0.000241 * freq * freq);
}

static long nearest_long(double x) { return (long) (x < 0 ? ceil(x - 0.5) : floor(x + 0.5)); }

/* delays of n channels from lofreq in steps of width (dedisp_delays) */
static void chan_delays(int n, double dm, double lofreq, double width, double *out)
{
    for (int i = 0; i < n; i++) out[i] = delay_from_dm(dm, (lofreq + i * width) * (1.0 + 0.0));
}

int ab_dedisp_delays(int nchan, double lofreq, double chanwidth, double dt, int nsub,
                     const double *dms, int ndm, int downsamp, int *chan_delay, int *sub_offset)
{
    if (nchan < 1 || nsub < 1 || nchan % nsub || ndm < 1 || !dms || downsamp < 1 ||
        !(dt > 0.0) || !chan_delay || !sub_offset)
        return AB_ERR_ARG;
    const int cps = nchan / nsub;
    const double subwidth = chanwidth * cps;
    const double losub_hifreq = lofreq + subwidth - chanwidth;
    double avgdm = 0.0;
    for (int d = 0; d < ndm; d++) avgdm += dms[d];
    avgdm /= ndm;
    double *cd = (double *) malloc(sizeof(double) * (size_t) nchan);
    double *sd = (double *) malloc(sizeof(double) * (size_t) nsub);
    if (!cd || !sd) {
        free(cd);
        free(sd);
        return AB_ERR_NOMEM;
    }
    /* subband_search_delays: channel delays minus their subband's top
       channel's delay */
    chan_delays(nchan, avgdm, lofreq, chanwidth, cd);
    chan_delays(nsub, avgdm, losub_hifreq, subwidth, sd);
    int rc = AB_OK;
    for (int s = 0; s < nsub; s++)
        for (int j = 0; j < cps; j++) {
            const long v = nearest_long((cd[s * cps + j] - sd[s]) / dt);
            if (v < 0 || v > (1L << 30)) rc = AB_ERR_ARG;
            chan_delay[s * cps + j] = (int) v;
        }
    const double dsdt = dt * downsamp;
    for (int d = 0; d < ndm && rc == AB_OK; d++) {
        chan_delays(nsub, dms[d], losub_hifreq, subwidth, sd);
        const double top = sd[nsub - 1];
        for (int s = 0; s < nsub; s++) {
            const long v = nearest_long((sd[s] - top) / dsdt);
            if (v < 0 || v > (1L << 30)) rc = AB_ERR_ARG;
            sub_offset[(size_t) d * nsub + s] = (int) v;
        }
    }
    free(cd);
    free(sd);
    return rc;
}
