/* CPU oracle for the htrdr-atmosphere null-collision path tracer.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain-C, FP64-transport restatement of
 * the reference's atmosphere hot path (AnthonyArfaux/htrdr_kmin).  It exists to
 * check the CUDA library; only the test-suite, the smoke check and the CPU
 * baseline of the benchmark may load it.  Nothing in the product links it.
 *
 * PINNED to the reference's own code: oracle/ref compiles the reference's
 * atmosphere hot-path C files unmodified (radiance routines, pixel callbacks,
 * sun, wavelength samplers, spectral routines, flux rectangle, buffer) over
 * shims of their absent dependencies (htsky 0.3, star-vx 0.3, star-sp 0.14,
 * star-sf 0.9, star-3d 0.10, star-camera 0.2, rsys 0.14), and
 * tests/test_reference_pin.py holds this restatement to it realisation by
 * realisation (relative 1e-6 at most, measured <= 5e-7) on every output mode,
 * pixel by pixel, and in the htrdr-image text.  The reference ships no test or
 * golden vector for this path; the oracle is also checked against closed-form
 * FP64 solutions (Beer-Lambert slab, isothermal absorbing slab, single
 * scattering, Planck identities) in tests/test_oracle_pins.py.
 *
 * The third-party semantics the reference relies on (htsky medium and octree,
 * star-sp samplers, star-sf phase functions and BSDFs, star-camera) are
 * restated from their published definitions; the choices made where the
 * reference leaves them to those libraries are the same ones the CUDA library
 * makes, so that both estimate the same integral. */
#ifndef ORA_H
#define ORA_H

#include <stddef.h>
#include <stdint.h>

/* res_T codes of rsys (used by every reference entry point) */
#define ORA_RES_OK 0
#define ORA_RES_BAD_ARG 1
#define ORA_RES_MEM_ERR 2
#define ORA_RES_IO_ERR 3
#define ORA_RES_UNKNOWN_ERR 4
#define ORA_RES_BAD_OP 5

/* Properties of the medium (htsky_property) */
enum { ORA_KA = 0, ORA_KS = 1, ORA_KEXT = 2 };
/* Radiance components (htrdr_atmosphere_c.h:38-44) */
enum { ORA_DIRECT = 1, ORA_DIFFUSE = 2, ORA_ALL = 3 };
/* Output modes (htrdr_atmosphere_draw_map.c:438-475) */
enum { ORA_XWAVE_SW = 0, ORA_XWAVE_LW = 1, ORA_IMAGE_CIE = 2, ORA_FLUX_SW = 3, ORA_FLUX_LW = 4 };

#define ORA_LEAF 0xFFFFFFFFu

/* One octree node: the packed 16-byte {k_min, k_max, first child, unused}
 * record shared with the CUDA library (bit-exact comparisons). */
struct ora_node {
  float kmin, kmax;
  uint32_t child; /* ORA_LEAF for a leaf, else index of the first of 8 children */
  uint32_t pad;
};

struct ora_scene_desc {
  uint32_t nlayers;
  const double* layer_z;      /* [nlayers+1] */
  const float* layer_T;       /* [nlayers] */
  uint32_t nbands;
  const double* band_lo;      /* [nbands] nm */
  const double* band_hi;      /* [nbands] nm */
  const uint32_t* nquads;     /* [nbands] */
  const double* quad_w;       /* [sum nquads] */
  const float* gas_ka;        /* [sum nquads][nlayers] */
  const float* gas_ks;        /* [sum nquads][nlayers] */
  uint32_t cloud_def[3];      /* nx, ny, nz (0 = no cloud) */
  double cloud_lower[3];
  double cloud_cell[3];
  const float* cloud_lwc;     /* [nz][ny][nx] */
  const float* cloud_sigma_ext; /* [nbands] */
  const float* cloud_ssa;     /* [nbands] */
  const float* cloud_g;       /* [nbands] */
  int32_t repeat_clouds;
  double optical_thickness;
  uint32_t grid_max_definition[3];
  int32_t has_ground;
  int32_t ground_brdf;        /* 0 Lambertian, 1 specular */
  double ground_reflectivity;
  double ground_temperature;
  double sun_azimuth, sun_elevation; /* degrees */
  uint32_t props_mask;        /* bit p: build the octrees of property p */
  /* ground mesh (replaces the plane when ground_ntris > 0); same arrays as
   * the CUDA library's scene description */
  uint32_t ground_nverts;
  const float* ground_verts;        /* [nverts][3] */
  uint32_t ground_ntris;
  const uint32_t* ground_tris;      /* [ntris][3] */
  const uint32_t* ground_tri_iface; /* [ntris] */
  uint32_t ground_nifaces;
  const uint32_t* ground_ifaces;    /* [nifaces][3] front, thin, back (UINT32_MAX: none) */
  uint32_t ground_nmtls;
  const double* ground_mtl_temperature; /* [nmtls] */
  const uint32_t* ground_mtl_nbrdf;     /* [nmtls] */
  const double* ground_mtl_brdf;        /* [sum nbrdf][3] wavelength nm, type, reflectivity */
  int32_t repeat_ground;
  uint32_t ground_sky_mtl;
};

struct ora_request {
  int32_t mode;
  uint32_t width, height, spp;
  double wlen_range[2];
  double ref_temperature;
  int32_t camera_type; /* 0 perspective, 1 orthographic */
  double cam_pos[3], cam_tgt[3], cam_up[3];
  double fov_deg, lens_radius, focal_dst, ortho_height;
  double rect_pos[3], rect_tgt[3], rect_up[3], rect_size[2];
  uint32_t seed;
};

/* ---- Counter-based random stream (Philox4x32-10, Salmon et al. SC'11) ----
 * Word j of the stream (key0, key1, ctr0, ctr1) is word (j & 3) of
 * Philox4x32-10(counter = {ctr0, ctr1, j >> 2, 0}, key = {key0, key1}).
 * Transport canonicals use one word, (w >> 8) * 2^-24; "double" canonicals
 * (film, lens, wavelength draws) use two words for 53 bits. */
struct ora_rng {
  uint32_t key[2];
  uint32_t ctr[2];
  uint32_t n;
  uint32_t blk[4];
  uint32_t blk_id;
  int blk_valid;
};

void ora_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);
void ora_rng_init(struct ora_rng* rng, uint32_t key0, uint32_t key1, uint32_t ctr0, uint32_t ctr1);
uint32_t ora_rng_u32(struct ora_rng* rng);
double ora_rng_canonical_f(struct ora_rng* rng); /* 24-bit transport canonical */
double ora_rng_canonical_d(struct ora_rng* rng); /* 53-bit canonical */

/* ---- spectral (htrdr_spectral.h / .c) ---- */
double ora_wiebelt(double v);
double ora_blackbody_fraction(double lambda0, double lambda1, double T);
double ora_planck_monochromatic(double lambda, double T);
double ora_planck_interval(double lambda_min, double lambda_max, double T);
double ora_planck(double lambda_min, double lambda_max, double T);
int ora_brightness_temperature(double lmin, double lmax, double radiance, double* T);
double ora_radiance_temperature(double lmin, double lmax, double radiance);

/* Planck wavelength sampler (htrdr_ran_wlen_planck.c) */
struct ora_planck_ran {
  double range[2];
  double band_len;
  double ref_temperature;
  size_t nbands;
  double* pdf;
  double* cdf;
};
int ora_planck_ran_init(struct ora_planck_ran* p, const double range[2], size_t nbands, double Tref);
void ora_planck_ran_release(struct ora_planck_ran* p);
double ora_planck_ran_sample(const struct ora_planck_ran* p, double r0, double r1, double* pdf);
size_t ora_planck_ran_band(const struct ora_planck_ran* p, double r0);

/* CIE XYZ sampler (htrdr_ran_wlen_cie_xyz.c) */
struct ora_cie_ran {
  double range[2];
  double band_len;
  size_t nbands;
  double* cdf[3];
  double rcp_integral[3];
};
int ora_cie_ran_init(struct ora_cie_ran* c, const double range[2], size_t nbands);
void ora_cie_ran_release(struct ora_cie_ran* c);
double ora_cie_ran_sample(const struct ora_cie_ran* c, int channel, double r0, double r1, double* pdf);
size_t ora_cie_ran_band(const struct ora_cie_ran* c, int channel, double r0);
double ora_fit_bar_1931(int channel, double lambda);

/* ---- medium (htsky restatement) ---- */
struct ora_scene;
int ora_scene_create(const struct ora_scene_desc* desc, struct ora_scene** out);
void ora_scene_release(struct ora_scene* scn);
size_t ora_scene_tree(const struct ora_scene* scn, uint32_t iband, uint32_t iquad, int prop,
                      const struct ora_node** nodes);
uint32_t ora_scene_tree_depth(const struct ora_scene* scn);
size_t ora_find_band(const struct ora_scene* scn, double wlen);
size_t ora_sample_quad(const struct ora_scene* scn, double r, size_t iband);
int ora_locate_leaf(const struct ora_scene* scn, uint32_t iband, uint32_t iquad, int prop,
                    const uint32_t cell[3], uint32_t* node, uint32_t* level);
int ora_layer_of(const struct ora_scene* scn, double z);

/* Trace counters (path segments, node fetches, tentative collisions) */
struct ora_counters {
  uint64_t nseg, nnode, ntc, nreal;
};

/* ---- radiance and drivers ---- */
double ora_radiance_sw(const struct ora_scene* scn, struct ora_rng* rng, int cpnt_mask,
                       const double pos[3], const double dir[3], double wlen, size_t iband,
                       size_t iquad, int dir_in_cone, struct ora_counters* cnt);
double ora_radiance_lw(const struct ora_scene* scn, struct ora_rng* rng, const double pos[3],
                       const double dir[3], double wlen, size_t iband, size_t iquad,
                       struct ora_counters* cnt);
/* Batched radiance, one stream per ray: key = {ray index, seed}. */
int ora_radiance_batch(const struct ora_scene* scn, int lw, size_t n, const double* pos,
                       const double* dir, const double* wlen, const uint32_t* iband,
                       const uint32_t* iquad, int cpnt_mask, uint32_t seed, double* out,
                       int nthreads);

/* htrdr_draw_map restatement: fills `buffer` (pitched rows of the reference's
 * pixel structs).  Pixels [pix_begin, pix_end) of the row-major pixel list are
 * computed (the others are left untouched) so that a bounded sample can be
 * timed. */
int ora_draw_map(const struct ora_scene* scn, const struct ora_request* req, void* buffer,
                 size_t pitch, size_t pix_begin, size_t pix_end, int nthreads,
                 struct ora_counters* cnt);

int ora_sample_wavelength(const struct ora_scene* scn, const struct ora_request* req, int channel,
                          size_t n, const double* r0, const double* r1, uint32_t* cdf_band,
                          double* wlen, double* pdf);

/* Ground-mesh queries, one per ray: rays [n][6] (origin, direction), range
 * [0, tmax), the primitive the ray leaves (UINT32_MAX: none) and whether that
 * hit lay on an edge.  prim = UINT32_MAX and dist = -1 where nothing is hit. */
int ora_ground_trace_batch(const struct ora_scene* scn, size_t n, const float* rays,
                           const float* tmax, const uint32_t* from_prim,
                           const uint8_t* from_edge, uint32_t* prim, float* dist);

/* Per-realisation weights for pixels [pix_begin, pix_end) (realisation-major
 * inside a pixel): the matched-stream comparison with the GPU. */
int ora_realisation_weights(const struct ora_scene* scn, const struct ora_request* req,
                            size_t pix_begin, size_t pix_end, double* weights, int nthreads);

#endif /* ORA_H */
