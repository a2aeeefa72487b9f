/* Shim of star-3d 0.10 (TEST INFRASTRUCTURE ONLY): the hit record the
 * ground queries return. */
#ifndef REF_SHIM_S3D_H
#define REF_SHIM_S3D_H
#include <rsys/float3.h>
#include <rsys/double3.h>
#include <float.h>

struct s3d_primitive {
  unsigned prim_id, geom_id, inst_id, scene_prim_id;
  void* mesh;
};
#define S3D_PRIMITIVE_NULL__ {(unsigned)-1, (unsigned)-1, (unsigned)-1, (unsigned)-1, NULL}

struct s3d_hit {
  struct s3d_primitive prim;
  float normal[3]; /* geometric normal, not normalised */
  float uv[2];
  float distance;
};
#define S3D_HIT_NULL__ {S3D_PRIMITIVE_NULL__, {0, 0, 0}, {0, 0}, FLT_MAX}
static const struct s3d_hit S3D_HIT_NULL = S3D_HIT_NULL__;
#define S3D_HIT_NONE(Hit) ((Hit)->distance >= FLT_MAX)
#endif
