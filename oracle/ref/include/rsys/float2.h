/* Shim of rsys float2.h (TEST INFRASTRUCTURE ONLY) */
#ifndef REF_SHIM_FLOAT2_H
#define REF_SHIM_FLOAT2_H
#include "rsys.h"
static INLINE float* f2(float d[2], const float a, const float b) { d[0] = a; d[1] = b; return d; }
#endif
