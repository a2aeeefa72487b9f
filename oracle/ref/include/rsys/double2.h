/* Shim of rsys double2.h (TEST INFRASTRUCTURE ONLY) */
#ifndef REF_SHIM_DOUBLE2_H
#define REF_SHIM_DOUBLE2_H
#include "rsys.h"
static INLINE double* d2(double d[2], const double a, const double b) { d[0] = a; d[1] = b; return d; }
static INLINE double* d2_set(double d[2], const double s[2]) { d[0] = s[0]; d[1] = s[1]; return d; }
#endif
