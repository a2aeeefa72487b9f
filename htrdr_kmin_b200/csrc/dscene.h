/* Device-side views of a scene and of a request (plain structs passed by
 * value to the kernels).  Shared by the host code that fills them and the
 * kernels that read them. */
#ifndef HTRDR_DSCENE_H
#define HTRDR_DSCENE_H

#include <stdint.h>

#define HG_LEAF 0xFFFFFFFFu
#define HG_MAX_DIST 1e9f          /* no collision beyond (..._sw.c:118-123) */
#define HG_TMIN_ZERO 746.0        /* exp(-Tmin) == 0.0 in FP64 from here on */
#define HG_MAX_STEPS (1u << 20)   /* voxel steps per trace before giving up */
#define HG_MAX_BOUNCES (1u << 16) /* scattering events per realisation before giving up */
#define HG_MAX_NULL (1u << 22)    /* tentative collisions per voxel before giving up */
#define HG_BVH_DEPTH_MAX 48       /* ground BVH depth bound (the traversal stack size) */

/* Register budget of the transport kernels (per thread): trades occupancy
 * against spills of the per-path state. */
#ifndef HG_PLAIN_MAXNREG
#define HG_PLAIN_MAXNREG 168
#endif
#ifndef HG_PERSIST_MAXNREG
#define HG_PERSIST_MAXNREG 255
#endif
#ifndef HG_WAVE_TRACE_MAXNREG
#define HG_WAVE_TRACE_MAXNREG 128
#endif

enum { HG_KA = 0, HG_KS = 1, HG_KEXT = 2 };
enum { HG_XWAVE_SW = 0, HG_XWAVE_LW = 1, HG_IMAGE_CIE = 2, HG_FLUX_SW = 3, HG_FLUX_LW = 4 };

/* Kernel variants: the parts of the path state machine one launch compiles.
 * A launch whose requests are all shortwave (or all longwave) leaves out the
 * other kind's states and trace filters, and a launch over plane-ground
 * scenes leaves out the mesh queries: fewer registers and spills, and less
 * code per warp.  A path of a kind its variant leaves out ends as a failed
 * realisation (never a stuck one). */
enum : uint32_t { HV_MESH = 1u, HV_SW = 2u, HV_LW = 4u, HV_ALL = 7u };

/* Internal modes of the batched radiance entry points */
#define HG_RAD_SW 5
#define HG_RAD_LW 6

/* Spectral kind of an output mode (HV_SW or HV_LW) */
static inline uint32_t
hv_kind(int mode)
{
  return (mode == HG_XWAVE_LW || mode == HG_FLUX_LW || mode == HG_RAD_LW) ? HV_LW : HV_SW;
}

/* A variant from the launch's mesh flag and kinds (no kind: both) */
static inline uint32_t
hv_make(bool mesh, uint32_t kinds)
{
  kinds &= HV_SW | HV_LW;
  return (mesh ? HV_MESH : 0u) | (kinds ? kinds : HV_SW | HV_LW);
}

/* Body of a host function returning kernel template K's instance for the
 * variant v */
#define HG_PICK_VARIANT(v, K)                                              \
  switch(hv_make(((v) & HV_MESH) != 0, (v))) {                             \
    case 2u: return K<2u>;                                                 \
    case 3u: return K<3u>;                                                 \
    case 4u: return K<4u>;                                                 \
    case 5u: return K<5u>;                                                 \
    case 6u: return K<6u>;                                                 \
    default: return K<7u>;                                                 \
  }

struct DScene {
  /* gas column */
  uint32_t nlayers;
  const float* layer_z;   /* [nlayers+1] */
  const float* layer_T;   /* [nlayers] */
  float ztop;
  const float2* gas;      /* [nq][nlayers] {ka, ks} */
  const double* layer_zd; /* [nlayers+1] layer bounds, FP64 */
  const double* gas_cum;  /* [nq][3][nlayers+1] cumulative vertical optical depth from z = 0 */
  /* spectral */
  uint32_t nbands;
  const double* band_lo;  /* [nbands] */
  const double* band_hi;  /* [nbands] */
  const uint32_t* quad_off; /* [nbands+1] */
  const double* quad_cum; /* [nq] */
  const float4* optics;   /* [nbands] {sigma_a, sigma_s, sigma_ext, g} */
  /* cloud */
  int32_t has_cloud, repeat;
  uint32_t def[3];
  float lower[3], upper[3], cell[3], inv_cell[3];
  const float* lwc;       /* [nz][ny][nx] */
  const int2* cell_layers;/* [nz] first/last gas layer overlapping the z-cell */
  uint32_t depth;
  const uint4* nodes;     /* node pool */
  const uint64_t* tree_base; /* [nq*3]: first node of the octree (q, prop) */
  /* leaf of every cell of every octree, (node index in its tree) << 5 | level:
   * grid `grid_rank[q*3+prop]' of ncell entries; null when it did not fit */
  const uint32_t* leaf_grid;
  /* or, per cell of every octree, its leaf's kmin/kmax and level (same
   * ranks); null unless built instead of leaf_grid */
  const float2* maj_grid;
  const uint8_t* lvl_grid;
  const uint32_t* grid_rank; /* [nq*3] */
  uint64_t ncell;            /* def[0] * def[1] * def[2] */
  /* ground */
  int32_t has_ground, ground_brdf;
  float ground_refl, ground_T;
  /* ground mesh (g_ntris > 0 replaces the plane ground) */
  uint32_t g_ntris, g_nmtls;
  int32_t g_repeat;
  uint32_t g_sky_mtl;         /* material of the atmosphere (~0u: none) */
  const float4* g_tri;        /* [ntris][3] v0, v1, v2 in BVH order (w unused) */
  const uint32_t* g_tri_id;   /* [ntris] BVH order -> primitive id of the caller */
  const uint32_t* g_iface_of; /* [ntris] interface of each primitive id */
  const uint4* g_iface;       /* [nifaces] {front, thin, back, 0} material (~0u: none) */
  const float4* g_bvh;        /* [nodes][2] {lo, first/left}, {hi, count (0: inner)} */
  const uint2* g_mtl;         /* [nmtls] {first brdf, nbrdf} */
  const float* g_mtl_T;       /* [nmtls] K */
  const double* g_brdf_wl;    /* [nbrdf] nm */
  const float2* g_brdf;       /* [nbrdf] {type, reflectivity} */
  double g_lower[3], g_upper[3]; /* mesh bounding box (the repeated cell) */
  /* sun */
  float sun_dir[3], sun_b1[3], sun_b2[3];
  double sun_dir_d[3];
  double sun_cos_half, sun_solid_angle, sun_T;
};

struct DRequest {
  int32_t mode;
  uint32_t width, height, spp, nreal_pp; /* nreal_pp = spp (x3 for CIE) */
  uint32_t seed;
  struct DAccum* acc;    /* [npix][channels] FP64 accumulators of this request */
  struct DAccum* tacc;   /* [npix] per-realisation time accumulators */
  unsigned long long* ndone; /* realisations finished (serving; may be null) */
  double pix_sz[2];
  double wlen_range[2];  /* nm */
  /* wavelength sampler */
  uint32_t ncdf;         /* CDF length (0: continuous/monochromatic) */
  double band_len;
  const double* cdf;     /* Planck: [ncdf]; CIE: [3][ncdf] */
  const double* pdf;     /* Planck: [ncdf] */
  const double* fbound;  /* CIE: [3][ncdf][2] fit values at each band's bounds */
  const uint32_t* guide; /* [nch][nguide+1]: first CDF entry >= b/nguide (may be null) */
  uint32_t nguide;       /* power of two */
  double rcp_integral[3];
  double ref_T;
  /* camera */
  int32_t camera_type;
  double cam_pos[3], cam_f[3], cam_r[3], cam_u[3];
  double tan_half, aspect, lens_radius, focal_dst, ortho_h;
  /* flux rectangle */
  double rect_pos[3], rect_ax[3], rect_ay[3], rect_n[3];
};

/* Per-pixel FP64 accumulators (one per channel) and per-pixel time */
struct DAccum {
  double s, s2;
  unsigned long long n, pad;
};

#endif
