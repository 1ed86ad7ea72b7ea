/* Stand-in for FFTW's fftw3.h: the single-precision subset that the
 * reference's accelsearch sources call (src/fftcalls.c, src/fastffts.c,
 * src/accel_utils.c), implemented by oracle/refshim/refshim_fftw.c.  Flag
 * and sign values are FFTW's documented ones.  Test infrastructure only:
 * used by oracle/build_ref.sh. */
#ifndef REFSHIM_FFTW3_H
#define REFSHIM_FFTW3_H
#include <stddef.h>
#include <stdio.h>
typedef float fftwf_complex[2];
typedef double fftw_complex[2];
typedef struct fftwf_plan_s *fftwf_plan;
typedef struct fftw_plan_s *fftw_plan;
#define FFTW_FORWARD (-1)
#define FFTW_BACKWARD (+1)
#define FFTW_MEASURE (0U)
#define FFTW_DESTROY_INPUT (1U << 0)
#define FFTW_EXHAUSTIVE (1U << 3)
#define FFTW_PRESERVE_INPUT (1U << 4)
#define FFTW_PATIENT (1U << 5)
#define FFTW_ESTIMATE (1U << 6)
fftwf_plan fftwf_plan_dft_1d(int n, fftwf_complex *in, fftwf_complex *out, int sign,
                             unsigned flags);
fftwf_plan fftwf_plan_many_dft(int rank, const int *n, int howmany, fftwf_complex *in,
                               const int *inembed, int istride, int idist, fftwf_complex *out,
                               const int *onembed, int ostride, int odist, int sign,
                               unsigned flags);
typedef struct {
    int n, is, os;
} fftwf_iodim;
typedef int fftwf_r2r_kind;
fftwf_plan fftwf_plan_guru_r2r(int rank, const fftwf_iodim *dims, int howmany_rank,
                               const fftwf_iodim *howmany_dims, float *in, float *out,
                               const fftwf_r2r_kind *kind, unsigned flags);
void fftwf_execute(const fftwf_plan p);
void fftwf_execute_dft(const fftwf_plan p, fftwf_complex *in, fftwf_complex *out);
void fftwf_destroy_plan(fftwf_plan p);
void *fftwf_malloc(size_t n);
void fftwf_free(void *p);
int fftwf_import_system_wisdom(void);
int fftwf_import_wisdom_from_file(FILE *f);
int fftwf_export_wisdom_to_file(FILE *f);
int fftwf_alignment_of(float *p);
#endif
