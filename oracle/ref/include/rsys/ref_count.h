/* Shim of rsys ref_count.h (TEST INFRASTRUCTURE ONLY): a plain counter;
 * the harness is single-owner so no atomics are needed. */
#ifndef REF_SHIM_REF_COUNT_H
#define REF_SHIM_REF_COUNT_H
#include "rsys.h"
#include "mem_allocator.h"

typedef int ref_T;

static INLINE void ref_init(ref_T* r) { *r = 1; }
static INLINE void ref_get(ref_T* r) { ++*r; }
static INLINE int
ref_put(ref_T* r, void (*release)(ref_T*))
{
  if(--*r == 0) { release(r); return 1; }
  return 0;
}
#endif
