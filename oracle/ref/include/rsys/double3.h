/* Shim of rsys double3.h (TEST INFRASTRUCTURE ONLY): 3-vector helpers in
 * FP64, each written out from its definition. */
#ifndef REF_SHIM_DOUBLE3_H
#define REF_SHIM_DOUBLE3_H
#include "rsys.h"
#include <math.h>

static INLINE double* d3(double d[3], const double x, const double y, const double z)
{ d[0] = x; d[1] = y; d[2] = z; return d; }
static INLINE double* d3_set(double d[3], const double s[3])
{ d[0] = s[0]; d[1] = s[1]; d[2] = s[2]; return d; }
static INLINE double* d3_set_f3(double d[3], const float s[3])
{ d[0] = (double)s[0]; d[1] = (double)s[1]; d[2] = (double)s[2]; return d; }
static INLINE double d3_dot(const double a[3], const double b[3])
{ return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
static INLINE double d3_len(const double a[3]) { return sqrt(d3_dot(a, a)); }
static INLINE double* d3_minus(double d[3], const double s[3])
{ d[0] = -s[0]; d[1] = -s[1]; d[2] = -s[2]; return d; }
static INLINE double* d3_add(double d[3], const double a[3], const double b[3])
{ d[0] = a[0] + b[0]; d[1] = a[1] + b[1]; d[2] = a[2] + b[2]; return d; }
static INLINE double* d3_sub(double d[3], const double a[3], const double b[3])
{ d[0] = a[0] - b[0]; d[1] = a[1] - b[1]; d[2] = a[2] - b[2]; return d; }
static INLINE double* d3_muld(double d[3], const double a[3], const double s)
{ d[0] = a[0] * s; d[1] = a[1] * s; d[2] = a[2] * s; return d; }
static INLINE double* d3_cross(double d[3], const double a[3], const double b[3])
{
  double t[3];
  t[0] = a[1] * b[2] - a[2] * b[1];
  t[1] = a[2] * b[0] - a[0] * b[2];
  t[2] = a[0] * b[1] - a[1] * b[0];
  return d3_set(d, t);
}
/* Normalise a into d; returns the length of a (0 leaves d unspecified) */
static INLINE double d3_normalize(double d[3], const double a[3])
{
  const double len = d3_len(a);
  if(len > 0) { const double r = 1.0 / len; d[0] = a[0] * r; d[1] = a[1] * r; d[2] = a[2] * r; }
  return len;
}
static INLINE int d3_is_normalized(const double a[3]) { return fabs(d3_len(a) - 1.0) < 1.e-6; }
#endif
