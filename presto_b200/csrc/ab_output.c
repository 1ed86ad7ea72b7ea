/*
 * ab_output.c -- accelsearch's text candidate file, <root>_ACCEL_<zmax> or
 * <root>_ACCEL_<zmax>_JERK_<wmax>: the fundamentals table (output_fundamentals,
 * src/accel_utils.c:666-841), the harmonics table (output_harmonics,
 * src/accel_utils.c:844-966), the candidate notes (compare_rzw_cands,
 * src/accel_utils.c:105-134), the value(error) number format (nice_output_1 /
 * nice_output_2, src/output.c:6-210) and the .inf appended at the end
 * (src/accel_utils.c:961-965).  The column layout, titles and number formats
 * are the file format that sifting.py and other consumers parse, so they are
 * kept exactly.  Pulsar-catalogue notes (comp_psr_to_cand, src/database.c)
 * are not made: the notes are those of a telescope "None" observation.
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "ab_host.h"
#include "ab_index.h"

#define OUT_SOL 299792458.0                       /* include/presto.h:38 */
#define OUT_TWOPI (2.0 * 3.14159265358979323846264338327950288)
#define NOTE_LEN 20

static double with_sign_of(double mag, double s)  /* COPYSIGN, src/output.c:1 */
{
    return s < 0.0 ? -fabs(mag) : fabs(mag);
}

static int finish_nice(char *out, size_t outlen, const char *t, int len)
{
    int n = len == 0 ? snprintf(out, outlen, "%s", t) : snprintf(out, outlen, "%*s", len, t);
    return (n < 0 || (size_t) n >= outlen) ? AB_ERR_ARG : n;
}

/* nice_output_1 (src/output.c:6-111): val rounded at the decimal place of
 * its one-digit error, the error in parentheses; scientific notation where
 * the reference uses it.  len == 0 left-justifies, len > 0 right-justifies. */
int ab_nice_output_1(char *out, size_t outlen, double val, double err, int len)
{
    char t[512];
    if (!out || outlen == 0) return AB_ERR_ARG;
    int e = fabs(err) == 0.0 ? 0 : (int) floor(log10(fabs(err)));
    int ev = (int) floor(fabs(err) * pow(10.0, (double) (-e)) + AB_DBLCORRECT + 0.5);
    if (ev == 10) {
        ev = 1;
        e++;
    }
    const double rv = pow(10.0, (double) e) * floor(val * pow(10.0, (double) (-e)) + 0.5);
    int nint = 1;
    if (fabs(val) != 0.0) {
        nint = (int) ceil(log10(fabs(val)));
        if (nint == 0) nint = 1;
    }
    const int nfrac = -e;
    int prec = nint + nfrac;
    const int oexp = fabs(rv) == 0.0 ? 0 : (int) floor(log10(fabs(rv)));
    const double mant = rv * pow(10.0, (double) (-oexp));
    if (fabs(1.0 - mant) < AB_DBLCORRECT || fabs(-1.0 - mant) < AB_DBLCORRECT) prec++;
    const double smant = with_sign_of(mant, rv);
    if (oexp >= 0 && e > 0 && oexp > e)
        snprintf(t, sizeof t, "% .*f(%d)x10^%d", prec - 1, smant, ev, oexp);
    else if (oexp >= 0 && e > 0 && oexp == e)
        snprintf(t, sizeof t, "% d(%d)x10^%d", (int) smant, ev, oexp);
    else if (oexp < -4 && oexp >= e)
        snprintf(t, sizeof t, "% .*f(%d)x10^%d", prec - 1, smant, ev, oexp);
    else if (oexp < e && e != 0)
        snprintf(t, sizeof t, "% d(%d)x10^%d", (int) (smant + AB_DBLCORRECT), ev, e);
    else if (nfrac == 0 && fabs(rv) < 1.0e-15)
        snprintf(t, sizeof t, "% d(%d)", (int) fabs(rv), ev);
    else if (fabs(rv) <= AB_DBLCORRECT && e < -5)
        snprintf(t, sizeof t, "0.0(%d)x10^%d", ev, e + 1);
    else
        snprintf(t, sizeof t, "% .*f(%d)", nfrac, rv, ev);
    return finish_nice(out, outlen, t, len);
}

/* nice_output_2 (src/output.c:114-210): as nice_output_1 with a two-digit
 * error.  AB_ERR_ARG where the reference exits ("undefined condition"). */
int ab_nice_output_2(char *out, size_t outlen, double val, double err, int len)
{
    char t[512];
    if (!out || outlen == 0) return AB_ERR_ARG;
    int e = fabs(err) == 0.0 ? 0 : (int) floor(log10(fabs(err)));
    int ev = (int) floor(fabs(err) * pow(10.0, (double) (-e + 1)) + AB_DBLCORRECT + 0.5);
    if (ev == 100) {
        ev = 10;
        e++;
    }
    double rv = pow(10.0, (double) (e - 1)) * floor(val * pow(10.0, (double) (-e + 1)) + 0.5);
    const int oexp = rv == 0.0 ? 0 : (int) floor(log10(fabs(rv)));
    const int vexp = val == 0.0 ? 0 : (int) floor(log10(fabs(val)));
    double mant = rv * pow(10.0, (double) (-oexp));
    const int ehi = ev / 10, elo = ev % 10;
    if (oexp < -4) {
        const int k = oexp - e + 1;
        if (k == 0)
            snprintf(t, sizeof t, "% .1f(%d.%d)x10^%d", mant / 10, ehi, elo, oexp + 1);
        else if (k < 2)
            snprintf(t, sizeof t, "% .1f(%d.%d)x10^%d", mant, ehi, elo, oexp);
        else
            snprintf(t, sizeof t, "% .*f(%.2d)x10^%d", k, mant, ev, oexp);
    } else if (e - vexp > 1 && e != 0 && e != 1) {
        snprintf(t, sizeof t, "0.0(%d.%d)x10^%d", ehi, elo, e);
    } else if (e == 0) {
        if (fabs(rv) < 0.1) rv = fabs(rv);
        snprintf(t, sizeof t, "% .1f(%d.%d)", rv, ehi, elo);
    } else if (e < 0) {
        if (fabs(rv) * pow(10.0, (double) (-e + 1)) < 0.1) rv = fabs(rv);
        if (fabs(rv) <= AB_DBLCORRECT && e < -4)
            snprintf(t, sizeof t, "0.0(%d.%d)x10^%d", ehi, elo, e);
        else
            snprintf(t, sizeof t, "% .*f(%.2d)", -e + 1, rv, ev);
    } else if (e - oexp == 0) {
        if (e == 1)
            snprintf(t, sizeof t, "% d(%.2d)", (int) rv, ev);
        else
            snprintf(t, sizeof t, "% .1f(%d.%d)x10^%d", mant, ehi, elo, e);
    } else if (e - oexp == 1) {
        if (fabs(mant) < 0.99999999999999) mant = fabs(mant);
        snprintf(t, sizeof t, "% .1f(%d.%d)x10^%d", mant / 10.0, ehi, elo, e);
    } else if (e > 1 && oexp > 1 && e - oexp <= -1) {
        snprintf(t, sizeof t, "% .*f(%.2d)x10^%d", oexp - e + 1, mant, ev, oexp);
    } else if (e == 1 && oexp > 0) {
        snprintf(t, sizeof t, "% d(%.2d)", (int) rv, ev);
    } else {
        return AB_ERR_ARG;
    }
    return finish_nice(out, outlen, t, len);
}

/* center_string (src/accel_utils.c:629-643): s centred in width columns,
 * cut to width when longer. */
static void put_centred(FILE *f, const char *s, int width, const char *tail)
{
    char b[128];
    const int len = (int) strlen(s);
    memset(b, ' ', (size_t) width);
    b[width] = '\0';
    if (len >= width) memcpy(b, s, (size_t) width);
    else memcpy(b + (width - len) / 2, s, (size_t) len);
    fputs(b, f);
    fputs(tail, f);
}

/* write_val_with_err (src/accel_utils.c:648-662) */
static int put_val_err(FILE *f, double val, double err, int digits, int width)
{
    char s[512];
    const int rc = digits == 1 ? ab_nice_output_1(s, sizeof s, val, err, 0)
                               : ab_nice_output_2(s, sizeof s, val, err, 0);
    if (rc < 0) return rc;
    put_centred(f, s, width, "  ");
    return AB_OK;
}

/* The two title lines and the dashes under them; skip[k] drops column k
 * (the jerk columns of an acceleration search). */
static void put_header(FILE *f, int ncol, const int *width, const char *const *t1,
                       const char *const *t2, const int *skip)
{
    for (int line = 0; line < 3; line++)
        for (int k = 0; k < ncol; k++) {
            if (skip[k]) continue;
            const char *tail = k == ncol - 1 ? "\n" : (line == 2 ? "--" : "  ");
            if (line < 2) {
                put_centred(f, line == 0 ? t1[k] : t2[k], width[k], tail);
            } else {
                char d[128];
                memset(d, '-', (size_t) width[k]);
                d[width[k]] = '\0';
                fputs(d, f);
                fputs(tail, f);
            }
        }
}

/* compare_rzw_cands (src/accel_utils.c:105-134): a candidate within 15 bins
 * of a stronger one at a z more than 1 away is a sidelobe ("SL? of Cand i");
 * otherwise, if its r and z divided by k (1..60) match candidate i within 3
 * and 2 of its own errors, it is "H k of Cand i".  A note, once set, stays. */
static void set_note(char *note, const char *t)   /* what "%.20s" prints of it */
{
    size_t k = strlen(t);
    if (k > NOTE_LEN) k = NOTE_LEN;
    memcpy(note, t, k);
    note[k] = '\0';
}

static void rzw_notes(const ab_fourierprops *p, long long n, char (*note)[NOTE_LEN + 1])
{
    char t[64];
    static const char blank[NOTE_LEN + 1] = "                    ";
    for (long long i = 0; i < n; i++)
        for (long long j = 0; j < n; j++) {
            if (i == j) continue;
            if (fabs(p[i].r - p[j].r) < 15.0 && fabs(p[i].z - p[j].z) > 1.0 && p[i].pow > p[j].pow) {
                if (!strncmp(note[j], blank, NOTE_LEN)) {
                    snprintf(t, sizeof t, "SL? of Cand %lld", i + 1);
                    set_note(note[j], t);
                }
                continue;
            }
            for (int k = 1; k < 61; k++) {
                const float rtol = p[j].rerr * 3, ztol = p[j].zerr * 2;
                if (fabs(p[i].r - p[j].r / k) < rtol && fabs(p[i].z - p[j].z / k) < ztol &&
                    !strncmp(note[j], blank, NOTE_LEN)) {
                    snprintf(t, sizeof t, "H %d of Cand %lld", k, i + 1);
                    set_note(note[j], t);
                    break;
                }
            }
        }
}

static int put_fundamentals(FILE *f, const ab_obs *obs, const ab_cand *c, const ab_polished *pol,
                            const ab_fourierprops *props, long long n, char (*note)[NOTE_LEN + 1])
{
    static const int width[13] = {4, 5, 6, 8, 4, 16, 15, 15, 15, 11, 11, 15, 20};
    static const char *const t1[13] = {"", "", "Summed", "Coherent", "Num", "Period",
                                       "Frequency", "FFT 'r'", "Freq Deriv", "FFT 'z'",
                                       "FFT 'w'", "Accel", ""};
    static const char *const t2[13] = {"Cand", "Sigma", "Power", "Power", "Harm", "(ms)",
                                       "(Hz)", "(bin)", "(Hz/s)", "(bins)", "(bins)",
                                       "(m/s^2)", "Notes"};
    int skip[13] = {0};
    skip[10] = obs->numw == 0;
    put_header(f, 13, width, t1, t2, skip);
    char s[64];
    for (long long i = 0; i < n; i++) {
        ab_rzwerrs er;
        int rc = ab_calc_rzwerrs(&props[i], obs->T, &er);
        if (rc) return rc;
        /* coherent sum of the harmonics, phases referred to the fundamental's
           (src/accel_utils.c:771-792) */
        double cr = 0.0, ci = 0.0;
        const double phs0 = pol[i].derivs[0].phs;
        for (int h = 0; h < c[i].numharm; h++) {
            const ab_rderivs *d = &pol[i].derivs[h];
            const double amp = obs->nph > 0.0 ? sqrt(d->pow / obs->nph) : sqrt(d->pow / d->locpow);
            const double corr = phs0 - fmod((h + 1.0) * phs0, OUT_TWOPI);
            cr += amp * cos(d->phs + corr);
            ci += amp * sin(d->phs + corr);
        }
        const double coherent = cr * cr + ci * ci;
        snprintf(s, sizeof s, "%-4lld", i + 1);
        put_centred(f, s, width[0], "  ");
        snprintf(s, sizeof s, "%.2f", c[i].sigma);
        put_centred(f, s, width[1], "  ");
        snprintf(s, sizeof s, "%.2f", c[i].power);
        put_centred(f, s, width[2], "  ");
        snprintf(s, sizeof s, "%.2f", coherent);
        put_centred(f, s, width[3], "  ");
        snprintf(s, sizeof s, "%d", c[i].numharm);
        put_centred(f, s, width[4], "  ");
        if ((rc = put_val_err(f, er.p * 1000.0, er.perr * 1000.0, 1, width[5])) ||
            (rc = put_val_err(f, er.f, er.ferr, 1, width[6])) ||
            (rc = put_val_err(f, props[i].r, props[i].rerr, 2, width[7])) ||
            (rc = put_val_err(f, er.fd, er.fderr, 1, width[8])) ||
            (rc = put_val_err(f, props[i].z, props[i].zerr, 2, width[9])) ||
            (obs->numw && (rc = put_val_err(f, props[i].w, props[i].werr, 2, width[10]))))
            return rc;
        const double accel = props[i].z * OUT_SOL / (obs->T * obs->T * er.f);
        const double accelerr = props[i].zerr * OUT_SOL / (obs->T * obs->T * er.f);
        if ((rc = put_val_err(f, accel, accelerr, 2, width[11]))) return rc;
        fprintf(f, "  %.20s\n", note[i]);
    }
    fputs("\n\n", f);
    return AB_OK;
}

static int put_harmonics(FILE *f, const ab_obs *obs, const ab_cand *c, const ab_polished *pol,
                         long long n)
{
    static const int width[15] = {5, 4, 5, 15, 11, 18, 13, 12, 9, 12, 9, 12, 10, 10, 20};
    static const char *const t1[15] = {"", "", "", "Power /", "Raw", "FFT 'r'", "Pred 'r'",
                                       "FFT 'z'", "Pred 'z'", "FFT 'w'", "Pred 'w'", "Phase",
                                       "Centroid", "Purity", ""};
    const char *t2[15] = {"Cand", "Harm", "Sigma", "Loc Pow", "Power", "(bin)", "(bin)",
                          "(bins)", "(bins)", "(bins)", "(bins)", "(rad)", "(0-1)", "<p> = 1",
                          "Notes"};
    if (obs->nph > 0.0) t2[3] = "NumPhot";
    int skip[15] = {0};
    skip[9] = skip[10] = obs->numw == 0;
    put_header(f, 15, width, t1, t2, skip);
    char s[64];
    for (long long i = 0; i < n; i++)
        for (int h = 0; h < c[i].numharm; h++) {
            ab_rderivs d = pol[i].derivs[h];
            if (obs->nph > 0.0) d.locpow = obs->nph;
            ab_fourierprops hp;
            int rc = ab_calc_props(&d, pol[i].hirs[h], pol[i].hizs[h], pol[i].hiws[h], &hp);
            if (rc) return rc;
            if (h == 0) snprintf(s, sizeof s, " %-4lld", i + 1);
            else snprintf(s, sizeof s, "     ");
            put_centred(f, s, width[0], "  ");
            snprintf(s, sizeof s, "%-4d", h + 1);
            put_centred(f, s, width[1], "  ");
            snprintf(s, sizeof s, "%.2f", ab_candidate_sigma(hp.pow, 1, 1));
            put_centred(f, s, width[2], "  ");
            if ((rc = put_val_err(f, hp.pow, hp.powerr, 2, width[3]))) return rc;
            snprintf(s, sizeof s, "%.3g", hp.rawpow);
            put_centred(f, s, width[4], "  ");
            if ((rc = put_val_err(f, hp.r, hp.rerr, 2, width[5]))) return rc;
            snprintf(s, sizeof s, "%.2f", c[i].r * (h + 1));
            put_centred(f, s, width[6], "  ");
            if ((rc = put_val_err(f, hp.z, hp.zerr, 2, width[7]))) return rc;
            snprintf(s, sizeof s, "%.2f", c[i].z * (h + 1));
            put_centred(f, s, width[8], "  ");
            if (obs->numw) {
                if ((rc = put_val_err(f, hp.w, hp.werr, 2, width[9]))) return rc;
                snprintf(s, sizeof s, "%.2f", c[i].w * (h + 1));
                put_centred(f, s, width[10], "  ");
            }
            if ((rc = put_val_err(f, hp.phs, hp.phserr, 2, width[11])) ||
                (rc = put_val_err(f, hp.cen, hp.cenerr, 2, width[12])) ||
                (rc = put_val_err(f, hp.pur, hp.purerr, 2, width[13])))
                return rc;
            fprintf(f, "  %.20s\n", "                    ");
        }
    fputs("\n\n", f);
    return AB_OK;
}

/* The whole text file (src/accel_utils.c:666-966) for n candidates in the
 * order given (sorted, harmonics removed, polished), with the .inf at
 * inf_path appended byte for byte (NULL, or a file that cannot be read:
 * nothing appended, as the reference's "cat" leaves it).  The file is
 * composed in memory and written only when every value formatted. */
int ab_write_accelfile(const char *path, const ab_obs *obs, const ab_cand *cands,
                       const ab_polished *pol, long long n, const char *inf_path)
{
    if (!path || !obs || n < 0 || (n > 0 && (!cands || !pol))) return AB_ERR_ARG;
    for (long long i = 0; i < n; i++)
        if (cands[i].numharm < 1 || cands[i].numharm > AB_POLISH_MAX_HARM) return AB_ERR_ARG;
    ab_fourierprops *props = (ab_fourierprops *) calloc((size_t) (n ? n : 1), sizeof *props);
    char (*note)[NOTE_LEN + 1] = calloc((size_t) (n ? n : 1), sizeof *note);
    char *text = NULL;
    size_t len = 0;
    FILE *m = NULL;
    int rc = AB_ERR_NOMEM;
    if (!props || !note || !(m = open_memstream(&text, &len))) goto out;
    if ((rc = ab_cand_props(cands, pol, n, props))) goto out;
    for (long long i = 0; i < n; i++) memset(note[i], ' ', NOTE_LEN);
    rzw_notes(props, n, note);
    if ((rc = put_fundamentals(m, obs, cands, pol, props, n, note))) goto out;
    if ((rc = put_harmonics(m, obs, cands, pol, n))) goto out;
    FILE *inf = inf_path ? fopen(inf_path, "rb") : NULL;
    if (inf) {
        char b[4096];
        size_t k;
        while ((k = fread(b, 1, sizeof b, inf)) > 0) fwrite(b, 1, k, m);
        fclose(inf);
    }
    fclose(m);
    m = NULL;
    FILE *f = fopen(path, "wb");
    if (!f) {
        rc = AB_ERR_ARG;
        goto out;
    }
    rc = fwrite(text, 1, len, f) == len ? AB_OK : AB_ERR_ARG;
    if (fclose(f)) rc = AB_ERR_ARG;
out:
    if (m) fclose(m);
    free(text);
    free(note);
    free(props);
    return rc;
}
