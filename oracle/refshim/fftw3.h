/* Declaration-only stand-in for FFTW's fftw3.h, so that reference sources
 * whose headers name FFTW's types (include/vectors.h, include/ransomfft.h)
 * but whose compiled functions never call FFTW build here.  Test
 * infrastructure: used only by oracle/build_ref.sh. */
#ifndef REFSHIM_FFTW3_H
#define REFSHIM_FFTW3_H
typedef float fftwf_complex[2];
typedef double fftw_complex[2];
typedef struct fftwf_plan_s *fftwf_plan;
typedef struct fftw_plan_s *fftw_plan;
#endif
