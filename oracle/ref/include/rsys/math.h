/* Shim of rsys math.h (TEST INFRASTRUCTURE ONLY) */
#ifndef REF_SHIM_RSYS_MATH_H
#define REF_SHIM_RSYS_MATH_H
#include "rsys.h"
#include <float.h>
#include <math.h>

#define PI 3.14159265358979323846
#define INF HUGE_VAL
#define IS_INF(X) isinf(X)
#define MDEG2RAD(D) ((D) * PI / 180.0)

static INLINE int
eq_eps(const double a, const double b, const double eps)
{
  return fabs(a - b) <= eps;
}
#endif
