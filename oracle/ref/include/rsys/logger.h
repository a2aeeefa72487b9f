/* Shim of rsys logger.h (TEST INFRASTRUCTURE ONLY) */
#ifndef REF_SHIM_LOGGER_H
#define REF_SHIM_LOGGER_H
#include "rsys.h"
#include "mem_allocator.h"
struct logger { int unused; };
#endif
