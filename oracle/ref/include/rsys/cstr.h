/* Shim of rsys cstr.h (TEST INFRASTRUCTURE ONLY) */
#ifndef REF_SHIM_CSTR_H
#define REF_SHIM_CSTR_H
#include "rsys.h"
static INLINE const char*
res_to_cstr(const res_T res)
{
  switch(res) {
    case RES_OK: return "success";
    case RES_BAD_ARG: return "invalid argument";
    case RES_MEM_ERR: return "out of memory";
    case RES_IO_ERR: return "I/O error";
    case RES_BAD_OP: return "invalid operation";
    default: return "unknown error";
  }
}
#endif
