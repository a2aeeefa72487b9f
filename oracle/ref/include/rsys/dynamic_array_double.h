/* Shim of rsys dynamic_array_double.h (TEST INFRASTRUCTURE ONLY) */
#ifndef REF_SHIM_DARRAY_DOUBLE_H
#define REF_SHIM_DARRAY_DOUBLE_H
#include "mem_allocator.h"

struct darray_double { double* data; size_t size; };

static INLINE void
darray_double_init(struct mem_allocator* a, struct darray_double* d)
{ (void)a; d->data = NULL; d->size = 0; }
static INLINE void
darray_double_release(struct darray_double* d)
{ free(d->data); d->data = NULL; d->size = 0; }
static INLINE void
darray_double_clear(struct darray_double* d) { d->size = 0; }
static INLINE res_T
darray_double_resize(struct darray_double* d, const size_t n)
{
  double* p = realloc(d->data, (n ? n : 1) * sizeof(double));
  if(!p) return RES_MEM_ERR;
  if(n > d->size) memset(p + d->size, 0, (n - d->size) * sizeof(double));
  d->data = p;
  d->size = n;
  return RES_OK;
}
static INLINE double* darray_double_data_get(struct darray_double* d) { return d->data; }
static INLINE const double* darray_double_cdata_get(const struct darray_double* d) { return d->data; }
static INLINE size_t darray_double_size_get(const struct darray_double* d) { return d->size; }
#endif
