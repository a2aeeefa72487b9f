/* Shim of star-vx 0.3 (TEST INFRASTRUCTURE ONLY): the voxel and hit records
 * handed to the hit filters of htsky_trace_ray. */
#ifndef REF_SHIM_SVX_H
#define REF_SHIM_SVX_H
#include <rsys/rsys.h>
#include <float.h>

struct svx_voxel {
  const void* data; /* the traversed majorant segment (see ref_shim.c) */
  size_t depth;
  uint64_t id;
  int is_leaf;
};
#define SVX_VOXEL_NULL__ {NULL, (size_t)-1, (uint64_t)-1, 0}

struct svx_hit {
  double distance[2]; /* entry and exit distances along the ray */
  struct svx_voxel voxel;
};
#define SVX_HIT_NULL__ {{DBL_MAX, -DBL_MAX}, SVX_VOXEL_NULL__}
static const struct svx_hit SVX_HIT_NULL = SVX_HIT_NULL__;
#define SVX_HIT_NONE(Hit) ((Hit)->distance[0] >= (Hit)->distance[1])

typedef int (*svx_hit_filter_T)(const struct svx_hit* hit, const double org[3],
                                const double dir[3], const double range[2], void* context);
#endif
