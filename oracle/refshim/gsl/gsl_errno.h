/* Stand-in for GSL's gsl_errno.h (status codes used by src/maximize_rz.c).
 * Test infrastructure only. */
#ifndef REFSHIM_GSL_ERRNO_H
#define REFSHIM_GSL_ERRNO_H
#define GSL_SUCCESS 0
#define GSL_FAILURE (-1)
#define GSL_CONTINUE (-2)
#define GSL_EINVAL 4
#define GSL_ENOMEM 8
#define GSL_EBADFUNC 9
#define GSL_ENOPROG 27
#endif
