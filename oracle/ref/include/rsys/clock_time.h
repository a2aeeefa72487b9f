/* Shim of rsys clock_time.h (TEST INFRASTRUCTURE ONLY).  time_current() is
 * also where the harness learns that a realisation starts (see
 * ref_harness.c): the pixel callbacks call it first thing in every
 * realisation. */
#ifndef REF_SHIM_CLOCK_TIME_H
#define REF_SHIM_CLOCK_TIME_H
#include "rsys.h"
#include <stdint.h>

struct time { int64_t nsec; };
enum time_unit { TIME_NSEC = 1, TIME_USEC = 2, TIME_MSEC = 4, TIME_SEC = 8 };

struct time* time_current(struct time* t);
static INLINE struct time*
time_sub(struct time* res, const struct time* a, const struct time* b)
{ res->nsec = a->nsec - b->nsec; return res; }
static INLINE int64_t
time_val(const struct time* t, const enum time_unit unit)
{
  switch(unit) {
    case TIME_USEC: return t->nsec / 1000;
    case TIME_MSEC: return t->nsec / 1000000;
    case TIME_SEC: return t->nsec / 1000000000;
    default: return t->nsec;
  }
}
#endif
