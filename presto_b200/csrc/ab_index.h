/*
 * ab_index.h -- exact search-geometry and index maps shared by the host C
 * code and the CUDA kernels.
 *
 * They restate the reference's FP64 formulas operation for operation, with
 * no fused multiply-add (the reference's default x86-64 build has none), so
 * the subharmonic r/z/w indices and plane offsets match bit for bit:
 *   calc_required_r/z/w      src/accel_utils.c:54-78
 *   index_from_r/z/w         src/accel_utils.c:81-102
 *   ffdot rlo/zlo/wlo/numrs  src/accel_utils.c:1034-1066
 *   in-memory r map          src/accel_utils.c:1324-1327
 */
#ifndef AB_INDEX_H
#define AB_INDEX_H

#include <math.h>

#ifdef __CUDACC__
#define AB_HD __host__ __device__ __forceinline__
#else
#define AB_HD static inline
#endif

#if defined(__CUDA_ARCH__)
#define AB_DMUL(a, b) __dmul_rn((a), (b))
#define AB_DADD(a, b) __dadd_rn((a), (b))
#else
#define AB_DMUL(a, b) ((a) * (b))
#define AB_DADD(a, b) ((a) + (b))
#endif

/* include/accel.h:19-35 */
#define AB_NUMBETWEEN 2
#define AB_DR 0.5
#define AB_RDR 2
#define AB_DZ 2
#define AB_RDZ 0.5
#define AB_DW 20
#define AB_RDW 0.05
#define AB_CLOSEST_R 15.0
#define AB_DBLCORRECT 1e-14
#define AB_NUMFINTBINS 16

AB_HD int ab_nearest_int(double x)                 /* src/accel_utils.c:36 */
{
    return (int) (x < 0 ? AB_DADD(x, -0.5) : AB_DADD(x, 0.5));
}

AB_HD double ab_calc_required_r(double f, double rfull)
{
    return AB_DMUL(rint(AB_DMUL(AB_DMUL((double) AB_RDR, rfull), f)), AB_DR);
}

AB_HD int ab_calc_required_z(double f, double zfull)
{
    return ab_nearest_int(AB_DMUL(AB_DMUL(AB_RDZ, zfull), f)) * AB_DZ;
}

AB_HD int ab_calc_required_w(double f, double wfull)
{
    return ab_nearest_int(AB_DMUL(AB_DMUL(AB_RDW, wfull), f)) * AB_DW;
}

AB_HD int ab_index_from_r(double r, double lor)
{
    return (int) AB_DADD(AB_DMUL(AB_DADD(r, -lor), (double) AB_RDR), AB_DBLCORRECT);
}

AB_HD int ab_index_from_z(double z, double loz)
{
    return (int) AB_DADD(AB_DMUL(AB_DADD(z, -loz), AB_RDZ), AB_DBLCORRECT);
}

AB_HD int ab_index_from_w(double w, double low)
{
    return (int) AB_DADD(AB_DMUL(AB_DADD(w, -low), AB_RDW), AB_DBLCORRECT);
}

/* Kernel half width in bins (src/responses.c:27-84, LOWACC). */
AB_HD int ab_resp_halfwidth(double z, double w)
{
    if (fabs(w) < 1.0e-7) return (int) (0.5 * 1.1 * fabs(z)) + AB_NUMFINTBINS;
    double r0 = 0.5 * (w / 6.0 - z);
    double r1 = 0.5 * (w / 6.0 + z);
    double maxdev = fabs(r0) > fabs(r1) ? fabs(r0) : fabs(r1);
    double u_ext = 0.5 - z / w;
    if (u_ext > 0.0 && u_ext < 1.0) {
        double z0 = z - w / 2.0;
        double r_ext = AB_DADD(AB_DADD(AB_DMUL(AB_DMUL(AB_DMUL(0.5, w), u_ext), u_ext),
                                       AB_DMUL(z0, u_ext)), r0);
        maxdev = fabs(r_ext) > maxdev ? fabs(r_ext) : maxdev;
    }
    return (int) (1.1 * maxdev) + AB_NUMFINTBINS;
}

/* Plane geometry of harmonic harmnum/numharm for the block [fullrlo,
 * fullrhi] (src/accel_utils.c:1034-1066). */
typedef struct {
    long long rlo;
    int zlo, wlo, numrs;
} ab_hgeom;

AB_HD ab_hgeom ab_harm_geom(double fullrlo, double fullrhi, int numharm, int harmnum,
                            double obs_zlo, double obs_wlo, int corr_uselen)
{
    ab_hgeom g;
    double f = (double) harmnum / (double) numharm;
    double drlo = ab_calc_required_r(f, fullrlo);
    double drhi = ab_calc_required_r(f, fullrhi);
    g.rlo = (long long) floor(drlo);
    g.zlo = ab_calc_required_z(f, obs_zlo);
    g.wlo = ab_calc_required_w(f, obs_wlo);
    g.numrs = (int) AB_DADD(AB_DMUL(AB_DADD(ceil(drhi), -floor(drlo)), (double) AB_RDR),
                            AB_DBLCORRECT) + 1;
    if (numharm == 1 && harmnum == 1) {
        g.numrs = corr_uselen;
    } else if (g.numrs % AB_RDR) {
        g.numrs = (g.numrs / AB_RDR + 1) * AB_RDR;
    }
    return g;
}

/* rinds[ii] of add_ffdotpows for fundamental r index ii
 * (src/accel_utils.c:1043-1047). */
AB_HD int ab_rind(double fullrlo, int ii, double f, long long sub_rlo)
{
    double rr = AB_DADD(fullrlo, AB_DMUL((double) ii, AB_DR));
    double subr = ab_calc_required_r(f, rr);
    return ab_index_from_r(subr, (double) sub_rlo);
}

/* zinds[ii] (src/accel_utils.c:1048-1052). */
AB_HD int ab_zind(double obs_zlo, int ii, double f, int sub_zlo)
{
    double zz = AB_DADD(obs_zlo, AB_DMUL((double) ii, (double) AB_DZ));
    int subz = ab_calc_required_z(f, zz);
    return ab_index_from_z((double) subz, (double) sub_zlo);
}

/* w index of add_ffdotpows (src/accel_utils.c:1266-1269). */
AB_HD int ab_wind(int fund_wlo, int ii, double f, int sub_wlo)
{
    int ww = fund_wlo + ii * AB_DW;
    int subw = ab_calc_required_w(f, (double) ww);
    return ab_index_from_w((double) subw, (double) sub_wlo);
}

/* In-memory r map: (int)(rrint * harm_fract + 0.5), rrint = 2*rlo + ii
 * (src/accel_utils.c:1324-1327). */
AB_HD int ab_inmem_rind(int fund_rlo, int ii, double f)
{
    int rrint = AB_RDR * fund_rlo + ii;
    return (int) AB_DADD(AB_DMUL((double) rrint, f), 0.5);
}

/* In-memory z row (src/accel_utils.c:1345-1348). */
AB_HD int ab_inmem_zind(int fund_zlo, int ii, double f)
{
    int zz = fund_zlo + ii * AB_DZ;
    int subz = ab_calc_required_z(f, (double) zz);
    return ab_index_from_z((double) subz, (double) fund_zlo);
}

#endif
