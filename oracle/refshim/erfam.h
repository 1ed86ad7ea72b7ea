/* Stand-in for ERFA's erfam.h (the one constant src/misc_utils.c names).
 * Test infrastructure only. */
#ifndef REFSHIM_ERFAM_H
#define REFSHIM_ERFAM_H
#define ERFA_DJM0 (2400000.5)
#endif
