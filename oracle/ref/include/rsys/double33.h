/* Shim of rsys double33.h (TEST INFRASTRUCTURE ONLY): 3x3 matrices stored
 * column by column (m[0..2] is the first column). */
#ifndef REF_SHIM_DOUBLE33_H
#define REF_SHIM_DOUBLE33_H
#include "double3.h"

/* d = m * v */
static INLINE double* d33_muld3(double d[3], const double m[9], const double v[3])
{
  double t[3];
  t[0] = m[0] * v[0] + m[3] * v[1] + m[6] * v[2];
  t[1] = m[1] * v[0] + m[4] * v[1] + m[7] * v[2];
  t[2] = m[2] * v[0] + m[5] * v[1] + m[8] * v[2];
  return d3_set(d, t);
}
static INLINE double* d33_transpose(double d[9], const double m[9])
{
  double t[9];
  int i, j;
  for(i = 0; i < 3; ++i) for(j = 0; j < 3; ++j) t[i * 3 + j] = m[j * 3 + i];
  for(i = 0; i < 9; ++i) d[i] = t[i];
  return d;
}
/* Orthonormal frame whose third column is the unit vector n; the first two
 * columns are the branchless basis of Duff et al. (JCGT 6(1), 2017), the one
 * the oracle builds its frames with, so that both turn the same local sample
 * into the same world direction. */
static INLINE double* d33_basis(double m[9], const double n[3])
{
  const double sign = copysign(1.0, n[2]);
  const double a = -1.0 / (sign + n[2]);
  const double b = n[0] * n[1] * a;
  m[0] = 1.0 + sign * n[0] * n[0] * a; m[1] = sign * b; m[2] = -sign * n[0];
  m[3] = b; m[4] = sign + n[1] * n[1] * a; m[5] = -n[1];
  m[6] = n[0]; m[7] = n[1]; m[8] = n[2];
  return m;
}
#endif
