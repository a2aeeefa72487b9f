/* Oracle internals.  TEST INFRASTRUCTURE ONLY (see ora.h). */
#ifndef ORA_INTERNAL_H
#define ORA_INTERNAL_H

#include "ora.h"

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

/* Beyond this traversed distance no collision is sampled
 * (src/atmosphere/htrdr_atmosphere_compute_radiance_sw.c:118-123). */
#define ORA_MAX_DIST 1e9

struct ora_tree {
  struct ora_node* nodes;
  size_t n;
};

struct ora_scene {
  uint32_t nlayers, nbands;
  size_t nq_total;
  double* layer_z;
  float* layer_T;
  double ztop;
  double* band_lo;
  double* band_hi;
  uint32_t* nquads;
  size_t* quad_off;
  double* quad_cum;
  float* gas_ka;
  float* gas_ks;
  float* gas_kext;
  float* sig; /* [nbands][3]: sigma of Ka, Ks, Kext per unit LWC */
  float* cloud_g;
  /* cloud */
  int has_cloud;
  uint32_t def[3];
  double lower[3], upper[3], cell[3];
  float* lwc;
  int* cell_layer_lo; /* per z-cell: first/last overlapping gas layer (-1: none) */
  int* cell_layer_hi;
  int repeat;
  uint32_t depth, level_force;
  double tau_thresh;
  struct ora_tree* trees; /* [nq_total][3] */
  /* ground */
  int has_ground, ground_brdf;
  double ground_reflectivity, ground_temperature;
  /* ground mesh (g_ntris > 0 replaces the plane) */
  uint32_t g_ntris, g_nmtls, g_sky_mtl;
  int g_repeat;
  float* g_v;            /* [ntris][3][3] vertices */
  uint32_t* g_iface_of;  /* [ntris] */
  uint32_t* g_iface;     /* [nifaces][3] */
  uint32_t* g_mtl_first; /* [nmtls] */
  uint32_t* g_mtl_n;     /* [nmtls] */
  float* g_mtl_T;        /* [nmtls] */
  double* g_brdf_wl;     /* [nbrdf] */
  float* g_brdf_type;    /* [nbrdf] */
  float* g_brdf_refl;    /* [nbrdf] */
  double g_lower[3], g_upper[3];
  /* sun */
  double sun_dir[3], sun_b1[3], sun_b2[3];
  double sun_cos_half, sun_solid_angle, sun_temperature;
};

/* A voxel handed to a hit filter (the svx_hit of the reference) */
struct ora_seg {
  double distance[2];
  double kmin, kmax;
  int in_cloud;
  int layer;          /* gas voxel: its layer */
  uint32_t lo[3], hi[3]; /* cloud leaf: its cell box (tile-local) */
  int64_t tile[2];
};

/* Where a collision happens: cloud cell (-1: none) and gas layer (-1: none) */
struct ora_site {
  int64_t cell;
  int layer;
};

typedef int (*ora_filter_T)(const struct ora_seg* seg, const double o[3], const double d[3],
                            void* ctx);

int ora_trace_ray(const struct ora_scene* scn, uint32_t band, uint32_t q, int prop,
                  const double o[3], const double d[3], const double range[2],
                  ora_filter_T filter, void* ctx, struct ora_counters* cnt, struct ora_seg* hit);
void ora_site_of(const struct ora_scene* scn, const struct ora_seg* seg, const double p[3],
                 struct ora_site* s);
double ora_site_k(const struct ora_scene* scn, const struct ora_site* s, uint32_t band,
                  uint32_t q, int prop, int cpnt);
void ora_onb(const double n[3], double b1[3], double b2[3]);
double ora_ground_trace(const struct ora_scene* scn, const double o[3], const double d[3],
                        double r0, double r1, int prev_ground);

/* Ground mesh (ora_ground.c) */
#define ORA_NO_PRIM 0xFFFFFFFFu
struct ora_ghit {
  float dist;    /* < 0: none */
  uint32_t prim;
  float u, v;
  float ng[3];   /* (v2 - v0) x (v1 - v0) */
};
int ora_ground_setup(struct ora_scene* scn, const struct ora_scene_desc* d);
void ora_ground_release(struct ora_scene* scn);
struct ora_ghit ora_ground_hit(const struct ora_scene* scn, const float o[3], const float d[3],
                               float r0, float r1, uint32_t from_prim, int from_edge);
int ora_on_edge(float u, float v);
uint32_t ora_hit_mtl(const struct ora_scene* scn, uint32_t prim, const float ng[3],
                     const double dir[3]);
uint32_t ora_fetch_brdf(const struct ora_scene* scn, uint32_t mtl, double wlen, double r);

#ifdef _OPENMP
#include <omp.h>
#define omp_set_num_threads_wrapper(n) omp_set_num_threads(n)
#else
#define omp_set_num_threads_wrapper(n) ((void)(n))
#endif

#endif
