/* Driver over the reference's own f-fdot plane generator, for plane-level
 * parity checks.  Test infrastructure only, written for this repository and
 * linked by oracle/build_ref.sh with the reference's unmodified objects into
 * oracle/_ref/libref_accel.so.
 *
 * refdrv_open parses accelsearch's options with the reference's own parser
 * (parseCmdline, src/accelsearch_cmd.c), builds the search with
 * create_accelobs (src/accel_utils.c:1455-1805, memory-mapped .fft) and the
 * template banks with create_subharminfos (:240-288), as
 * src/accelsearch.c:71-123 does.  refdrv_plane returns one
 * subharm_fderivs_vol plane (src/accel_utils.c:1024-1198) for the bank the
 * reference's main loop uses (subharminfs[stage][harm - 1],
 * src/accelsearch.c:187-206). */
#include "accel.h"
#include "accelsearch_cmd.h"

static accelobs g_obs;
static infodata g_idata;
static subharminfo **g_shis;
static int g_open;

void refdrv_close(void)
{
    if (!g_open) return;
    free_subharminfos(&g_obs, g_shis);
    free_accelobs(&g_obs);
    g_open = 0;
}

int refdrv_open(int argc, char **argv)
{
    refdrv_close();
    memset(&g_obs, 0, sizeof g_obs);
    memset(&g_idata, 0, sizeof g_idata);
    Cmdline *cmd = parseCmdline(argc, argv);
    create_accelobs(&g_obs, &g_idata, cmd, 1);
    g_shis = create_subharminfos(&g_obs);
    g_open = 1;
    return 0;
}

/* rlo, highestbin, rstep (= corr_uselen * ACCEL_DR), numharmstages, inmem */
void refdrv_geometry(double *out)
{
    out[0] = g_obs.rlo;
    out[1] = g_obs.highestbin;
    out[2] = g_obs.corr_uselen * ACCEL_DR;
    out[3] = g_obs.numharmstages;
    out[4] = g_obs.inmem;
}

/* The plane of harmonic harmnum / numharm for fundamental r in [fullrlo,
 * fullrhi]: meta = rlo, zlo, wlo, numrs, numzs, numws; the powers
 * [numws][numzs][numrs] are copied to out when they fit in cap floats.
 * Returns their count. */
long long refdrv_plane(int numharm, int harmnum, double fullrlo, double fullrhi, float *out,
                       long long cap, long long *meta)
{
    int stage = 0;
    while ((1 << stage) < numharm) stage++;
    ffdotpows *f = subharm_fderivs_vol(numharm, harmnum, fullrlo, fullrhi,
                                       &g_shis[stage][harmnum - 1], &g_obs);
    const long long n = (long long) f->numrs * f->numzs * f->numws;
    meta[0] = f->rlo;
    meta[1] = f->zlo;
    meta[2] = f->wlo;
    meta[3] = f->numrs;
    meta[4] = f->numzs;
    meta[5] = f->numws;
    if (out && n <= cap) memcpy(out, f->powers[0][0], sizeof(float) * (size_t) n);
    free_ffdotpows(f);
    return n;
}
