/* Shim of rsys float3.h (TEST INFRASTRUCTURE ONLY) */
#ifndef REF_SHIM_FLOAT3_H
#define REF_SHIM_FLOAT3_H
#include "rsys.h"
#include <math.h>
static INLINE float* f3_set_d3(float d[3], const double s[3])
{ d[0] = (float)s[0]; d[1] = (float)s[1]; d[2] = (float)s[2]; return d; }
static INLINE float f3_dot(const float a[3], const float b[3])
{ return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
static INLINE float f3_normalize(float d[3], const float a[3])
{
  const float len = sqrtf(f3_dot(a, a));
  if(len > 0) { const float r = 1.f / len; d[0] = a[0] * r; d[1] = a[1] * r; d[2] = a[2] * r; }
  return len;
}
#endif
