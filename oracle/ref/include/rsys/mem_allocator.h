/* Shim of rsys mem_allocator.h (TEST INFRASTRUCTURE ONLY): every allocator
 * is the C heap. */
#ifndef REF_SHIM_MEM_ALLOCATOR_H
#define REF_SHIM_MEM_ALLOCATOR_H
#include "rsys.h"
#include <string.h>

struct mem_allocator { int unused; };

static INLINE void*
ref_shim_calloc(size_t n, size_t sz) { return calloc(n, sz); }

#define MEM_ALLOC(Allocator, Size) ((void)(Allocator), malloc(Size))
#define MEM_CALLOC(Allocator, N, Size) ((void)(Allocator), ref_shim_calloc((N), (Size)))
#define MEM_REALLOC(Allocator, Mem, Size) ((void)(Allocator), realloc((Mem), (Size)))
#define MEM_RM(Allocator, Mem) ((void)(Allocator), free(Mem))
/* Aligned block; released by MEM_RM (free) like the others */
static INLINE void*
ref_shim_aligned(size_t size, size_t align)
{
  void* p = NULL;
  if(align < sizeof(void*)) align = sizeof(void*);
  return posix_memalign(&p, align, size ? size : 1) == 0 ? p : NULL;
}
#define MEM_ALLOC_ALIGNED(Allocator, Size, Align) ((void)(Allocator), ref_shim_aligned((Size), (Align)))
#endif
