/* Shim of rsys algorithm.h (TEST INFRASTRUCTURE ONLY) */
#ifndef REF_SHIM_ALGORITHM_H
#define REF_SHIM_ALGORITHM_H
#include "rsys.h"
#include "math.h"

/* First element of the sorted array `base' that is not less than `key'
 * (cmp(key, elmt) <= 0); NULL when every element is less than the key. */
static INLINE void*
search_lower_bound(const void* key, const void* base, size_t nmemb, size_t size,
                   int (*cmp)(const void*, const void*))
{
  size_t lo = 0, hi = nmemb;
  while(lo < hi) {
    const size_t mid = lo + (hi - lo) / 2;
    if(cmp((const char*)base + mid * size, key) < 0) lo = mid + 1; else hi = mid;
  }
  return lo < nmemb ? (void*)((const char*)base + lo * size) : NULL;
}
#endif
