/* Shim of rsys str.h (TEST INFRASTRUCTURE ONLY): only the type is needed by
 * the structures the harness fills. */
#ifndef REF_SHIM_STR_H
#define REF_SHIM_STR_H
#include "rsys.h"
#include "mem_allocator.h"
struct str { char* cstr; size_t len; };
#endif
