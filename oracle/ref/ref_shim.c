/* Services the reference's atmosphere hot-path files call, for the compiled
 * reference oracle (oracle/_ref).  TEST INFRASTRUCTURE ONLY.
 *
 * The reference (src/atmosphere/htrdr_atmosphere_compute_radiance_{sw,lw}.c,
 * src/atmosphere/htrdr_atmosphere_draw_map.c, src/atmosphere/htrdr_atmosphere_sun.c,
 * src/core/htrdr_ran_wlen_{planck,cie_xyz}.c, src/core/htrdr_spectral.c,
 * src/core/htrdr_rectangle.c) is compiled unmodified against the headers of
 * oracle/ref/include, and this file answers the calls those files make into
 * their dependencies, none of which is vendored:
 *
 *   - rsys (htrdr core runtime, clock) and htrdr's own runtime
 *     (src/core/htrdr.c, htrdr_log.c): allocators, thread count, logging;
 *   - star-sp: canonical numbers, exponential, cosine hemisphere and
 *     spherical-cap variates, from the oracle's Philox streams;
 *   - star-sf: HG and Rayleigh phase functions, Lambertian and specular
 *     BRDFs, restated as the oracle states them;
 *   - star-camera: the camera ray of a film/lens sample;
 *   - htsky: the medium and its majorant octrees, answered by the oracle's
 *     scene (ora_trace_ray, ora_site_of, ora_site_k);
 *   - the ground (src/atmosphere/htrdr_atmosphere_ground.c over star-3d) and
 *     htrdr_mtl_create_bsdf (src/core/htrdr_materials.c over mrumtl): the
 *     flat plane z = 0 with one BRDF and one temperature.
 *
 * Every definition here is the one the oracle (the C files of oracle/) and the CUDA
 * library use for the same service, so that the compiled reference, the
 * oracle and the GPU estimate the same integral and, where the draw order
 * allows, consume the same random stream in the same order. */
#define _POSIX_C_SOURCE 200112L
#include "ref_shim.h"

#include "../ora_internal.h"

#include <float.h>
#include <math.h>
#include <stdarg.h>
#include <string.h>
#include <time.h>

/*******************************************************************************
 * Per-thread state: the stream in use, the realisation hook, the traversal
 ******************************************************************************/
struct tls_site { double pos[3]; struct ora_site site; int valid; };

struct ref_tls {
  /* realisation hook (see time_current) */
  struct ssp_rng* rng;
  uint32_t pixel, seed;
  const uint32_t* keys; /* realisation index of each realisation of the call */
  size_t next;
  const void* start_site; /* return address of a realisation's first clock read */
  /* traversal */
  const struct ora_scene* scn;
  const struct ora_seg* seg; /* voxel handed to the filter being run */
  int trace_prop;
  struct tls_site last[3]; /* last in-trace collision candidate per property */
};
static __thread struct ref_tls tls;

/*******************************************************************************
 * htrdr runtime (src/core/htrdr.c, src/core/htrdr_log.c)
 ******************************************************************************/
static struct mem_allocator g_alloc;

struct mem_allocator* htrdr_get_allocator(struct htrdr* h) { (void)h; return &g_alloc; }
struct mem_allocator* htrdr_get_thread_allocator(struct htrdr* h, const size_t i)
{ (void)h; (void)i; return &g_alloc; }
size_t htrdr_get_threads_count(const struct htrdr* h) { return h->nthreads; }
size_t htrdr_get_procs_count(const struct htrdr* h) { (void)h; return 1; }
int htrdr_get_mpi_rank(const struct htrdr* h) { (void)h; return 0; }
void htrdr_ref_get(struct htrdr* h) { (void)h; }
void htrdr_ref_put(struct htrdr* h) { (void)h; }

static void
vlog(struct htrdr* h, const char* prefix, const char* msg, va_list ap)
{
  if(!h || !h->verbose) return;
  fputs(prefix, stderr);
  vfprintf(stderr, msg, ap);
}
void htrdr_log(struct htrdr* h, const char* msg, ...)
{ va_list ap; va_start(ap, msg); vlog(h, "", msg, ap); va_end(ap); }
void htrdr_log_err(struct htrdr* h, const char* msg, ...)
{ va_list ap; va_start(ap, msg); if(h) { fputs("error: ", stderr); vfprintf(stderr, msg, ap); } va_end(ap); }
void htrdr_log_warn(struct htrdr* h, const char* msg, ...)
{ va_list ap; va_start(ap, msg); vlog(h, "warning: ", msg, ap); va_end(ap); }

/*******************************************************************************
 * Clock and the realisation hook.  Each pixel callback of the reference reads
 * the clock first thing in every realisation (time_current(&t0),
 * src/atmosphere/htrdr_atmosphere_draw_map.c:141, 241, 357) and once more at
 * its end.  The first read of a call is a start; later reads from the same
 * call site are starts too.  At every start the thread's generator moves to
 * the stream of the next realisation: key {pixel, seed}, counter
 * {realisation, 0}, as the oracle and the CUDA kernels key theirs.
 ******************************************************************************/
void
ref_hook_begin(struct ssp_rng* rng, uint32_t pixel, uint32_t seed, const uint32_t* keys)
{
  tls.rng = rng;
  tls.pixel = pixel;
  tls.seed = seed;
  tls.keys = keys;
  tls.next = 0;
  tls.start_site = NULL;
}

void
ref_hook_end(void)
{
  tls.rng = NULL;
}

struct time*
time_current(struct time* t)
{
  struct timespec ts;
  const void* site = __builtin_return_address(0);
  if(tls.rng) {
    if(!tls.start_site) tls.start_site = site;
    if(site == tls.start_site) {
      const uint32_t ireal = tls.keys ? tls.keys[tls.next] : (uint32_t)tls.next;
      ++tls.next;
      ora_rng_init(&tls.rng->r, tls.pixel, tls.seed, ireal, 0);
    }
  }
  clock_gettime(CLOCK_MONOTONIC, &ts);
  t->nsec = (int64_t)ts.tv_sec * 1000000000 + ts.tv_nsec;
  return t;
}

/*******************************************************************************
 * star-sp
 ******************************************************************************/
double
ssp_rng_canonical(struct ssp_rng* rng)
{
  return rng->transport ? ora_rng_canonical_f(&rng->r) : ora_rng_canonical_d(&rng->r);
}

static double
transport_canonical(struct ssp_rng* rng) { return ora_rng_canonical_f(&rng->r); }

double
ssp_ran_exp(struct ssp_rng* rng, const double mu)
{
  const uint32_t m = ora_rng_u32(&rng->r) >> 9;
  const double u = (double)(2u * m + 1u) * (1.0 / 16777216.0);
  return -log(u) / mu;
}

/* Unit vector at cosine mu and azimuth phi in the frame (b1, b2, axis) */
static void
around(const double axis[3], double mu, double phi, double out[3])
{
  double b1[3], b2[3], n;
  const double s = sqrt(fmax(0.0, 1.0 - mu * mu));
  const double cp = cos(phi) * s, sp = sin(phi) * s;
  int i;
  ora_onb(axis, b1, b2);
  for(i = 0; i < 3; ++i) out[i] = b1[i] * cp + b2[i] * sp + axis[i] * mu;
  n = sqrt(out[0] * out[0] + out[1] * out[1] + out[2] * out[2]);
  for(i = 0; i < 3; ++i) out[i] /= n;
}

double*
ssp_ran_hemisphere_cos(struct ssp_rng* rng, const double up[3], double dir[3], double* pdf)
{
  const double u1 = transport_canonical(rng), u2 = transport_canonical(rng);
  const double mu = sqrt(1.0 - u2);
  around(up, mu, 2.0 * M_PI * u1, dir);
  if(pdf) *pdf = mu / M_PI;
  return dir;
}

double*
ssp_ran_sphere_cap_uniform_local(struct ssp_rng* rng, const double cos_aperture, double dir[3],
                                 double* pdf)
{
  const double u1 = transport_canonical(rng), u2 = transport_canonical(rng);
  const double mu = 1.0 - u1 * (1.0 - cos_aperture);
  const double s = sqrt(fmax(0.0, 1.0 - mu * mu));
  const double phi = 2.0 * M_PI * u2;
  dir[0] = cos(phi) * s;
  dir[1] = sin(phi) * s;
  dir[2] = mu;
  if(pdf) *pdf = 1.0 / (2.0 * M_PI * (1.0 - cos_aperture));
  return dir;
}

/*******************************************************************************
 * star-sf
 ******************************************************************************/
const struct ssf_phase_type ssf_phase_hg = {0};
const struct ssf_phase_type ssf_phase_rayleigh = {1};

struct ssf_phase { int type; double g; int ref; };

res_T
ssf_phase_create(struct mem_allocator* a, const struct ssf_phase_type* type, struct ssf_phase** out)
{
  struct ssf_phase* p = calloc(1, sizeof(*p));
  (void)a;
  if(!p) return RES_MEM_ERR;
  p->type = type->id;
  p->ref = 1;
  *out = p;
  return RES_OK;
}
res_T ssf_phase_ref_get(struct ssf_phase* p) { ++p->ref; return RES_OK; }
res_T ssf_phase_ref_put(struct ssf_phase* p) { if(--p->ref == 0) free(p); return RES_OK; }
res_T ssf_phase_hg_setup(struct ssf_phase* p, const double g) { p->g = g; return RES_OK; }

/* Henyey-Greenstein cosine by inversion of its CDF */
static double
hg_sample_mu(double g, double u)
{
  double s, mu;
  if(fabs(g) < 1e-6) return 1.0 - 2.0 * u;
  s = (1.0 - g * g) / (1.0 - g + 2.0 * g * u);
  mu = (1.0 + g * g - s * s) / (2.0 * g);
  return mu > 1.0 ? 1.0 : (mu < -1.0 ? -1.0 : mu);
}

/* Rayleigh cosine: the root of (mu^3 + 3 mu + 4) / 8 = u (Cardano) */
static double
rayleigh_sample_mu(double u)
{
  const double A = 4.0 * u - 2.0;
  const double c = cbrt(A + sqrt(A * A + 1.0));
  const double mu = c - 1.0 / c;
  return mu > 1.0 ? 1.0 : (mu < -1.0 ? -1.0 : mu);
}

void
ssf_phase_sample(struct ssf_phase* p, struct ssp_rng* rng, const double wo[3], double wi[3],
                 double* pdf)
{
  const double u1 = transport_canonical(rng), u2 = transport_canonical(rng);
  const double mu = p->type == 0 ? hg_sample_mu(p->g, u1) : rayleigh_sample_mu(u1);
  const double dir[3] = {-wo[0], -wo[1], -wo[2]};
  around(dir, mu, 2.0 * M_PI * u2, wi);
  if(pdf) *pdf = ssf_phase_eval(p, wo, wi);
}

double
ssf_phase_eval(struct ssf_phase* p, const double wo[3], const double wi[3])
{
  const double mu = -(wo[0] * wi[0] + wo[1] * wi[1] + wo[2] * wi[2]);
  if(p->type == 0) {
    const double g = p->g, d = 1.0 + g * g - 2.0 * g * mu;
    return (1.0 - g * g) / (4.0 * M_PI * d * sqrt(d));
  }
  return 3.0 / (16.0 * M_PI) * (1.0 + mu * mu);
}

struct ssf_bsdf { int specular; double reflectivity; int ref; };

res_T ssf_bsdf_ref_get(struct ssf_bsdf* b) { ++b->ref; return RES_OK; }
res_T ssf_bsdf_ref_put(struct ssf_bsdf* b) { if(--b->ref == 0) free(b); return RES_OK; }

double
ssf_bsdf_sample(struct ssf_bsdf* b, struct ssp_rng* rng, const double wo[3], const double N[3],
                double wi[3], int* type, double* pdf)
{
  if(b->specular) {
    const double c = N[0] * wo[0] + N[1] * wo[1] + N[2] * wo[2];
    double n;
    int i;
    for(i = 0; i < 3; ++i) wi[i] = 2.0 * c * N[i] - wo[i];
    n = sqrt(wi[0] * wi[0] + wi[1] * wi[1] + wi[2] * wi[2]);
    for(i = 0; i < 3; ++i) wi[i] /= n;
    if(type) *type = SSF_REFLECTION | SSF_SPECULAR;
    if(pdf) *pdf = INFINITY;
  } else {
    ssp_ran_hemisphere_cos(rng, N, wi, pdf);
    if(type) *type = SSF_REFLECTION | SSF_DIFFUSE;
  }
  return b->reflectivity;
}

double
ssf_bsdf_eval(struct ssf_bsdf* b, const double wo[3], const double N[3], const double wi[3])
{
  (void)wo;
  if(b->specular) return 0.0;
  return N[0] * wi[0] + N[1] * wi[1] + N[2] * wi[2] > 0 ? b->reflectivity / M_PI : 0.0;
}

/*******************************************************************************
 * The ground: the plane z = 0 (htrdr_atmosphere_ground_trace_ray with the
 * self-hit filter of src/core/htrdr_geometry.c:118-150) and its material
 * (htrdr_mtl_create_bsdf, src/core/htrdr_materials.c:414-463)
 ******************************************************************************/
res_T
htrdr_atmosphere_ground_trace_ray(struct htrdr_atmosphere_ground* g, const double org[3],
                                  const double dir[3], const double range[2],
                                  const struct s3d_hit* prev_hit, struct s3d_hit* hit)
{
  double t;
  *hit = S3D_HIT_NULL;
  if(!g || !g->has_ground) return RES_OK;
  if(prev_hit && !S3D_HIT_NONE(prev_hit)) return RES_OK; /* leaving the plane: no self hit */
  if(dir[2] == 0.0) return RES_OK;
  t = -org[2] / dir[2];
  if(!(t > range[0] && t < range[1])) return RES_OK;
  hit->prim.prim_id = hit->prim.geom_id = hit->prim.scene_prim_id = 0;
  hit->prim.inst_id = (unsigned)-1;
  hit->normal[0] = 0.f; hit->normal[1] = 0.f; hit->normal[2] = 1.f;
  hit->uv[0] = hit->uv[1] = 0.f;
  hit->distance = (float)t;
  if(S3D_HIT_NONE(hit)) *hit = S3D_HIT_NULL; /* beyond FLT_MAX */
  return RES_OK;
}

void
htrdr_atmosphere_ground_get_interface(struct htrdr_atmosphere_ground* g, const struct s3d_hit* hit,
                                      struct htrdr_interface* interf)
{
  (void)hit;
  /* front (the +z side): the sky; back: the ground.  A ray coming down meets
   * the front face and takes the material on the other side. */
  interf->mtl_front.name = "air";
  interf->mtl_front.mrumtl = NULL;
  interf->mtl_front.temperature = 0;
  interf->mtl_back.name = "ground";
  interf->mtl_back.mrumtl = (const struct mrumtl*)g;
  interf->mtl_back.temperature = g->temperature;
  interf->mtl_thin = HTRDR_MTL_NULL;
}

res_T
htrdr_mtl_create_bsdf(struct htrdr* h, const struct htrdr_mtl* mtl, const size_t ithread,
                      const double wavelength, struct ssp_rng* rng, struct ssf_bsdf** out)
{
  const struct htrdr_atmosphere_ground* g = (const struct htrdr_atmosphere_ground*)mtl->mrumtl;
  struct ssf_bsdf* b;
  (void)h; (void)ithread; (void)wavelength;
  /* the reference draws the canonical that picks the BRDF among the
   * material's spectral entries whatever their count */
  (void)transport_canonical(rng);
  b = calloc(1, sizeof(*b));
  if(!b) return RES_MEM_ERR;
  b->specular = g->brdf == 1;
  b->reflectivity = g->reflectivity;
  b->ref = 1;
  *out = b;
  return RES_OK;
}

/*******************************************************************************
 * star-camera
 ******************************************************************************/
res_T
scam_generate_ray(const struct scam* c, const struct scam_sample* s, struct scam_ray* ray)
{
  const double x = 2.0 * s->film[0] - 1.0, y = 2.0 * s->film[1] - 1.0;
  double n;
  int i;
  if(c->type == 1) { /* orthographic */
    const double hw = 0.5 * c->ortho_h * c->aspect, hh = 0.5 * c->ortho_h;
    for(i = 0; i < 3; ++i) {
      ray->org[i] = c->pos[i] + c->r[i] * x * hw + c->u[i] * y * hh;
      ray->dir[i] = c->f[i];
    }
    return RES_OK;
  }
  for(i = 0; i < 3; ++i)
    ray->dir[i] = c->f[i] + c->r[i] * (x * c->tan_half * c->aspect) + c->u[i] * (y * c->tan_half);
  if(c->lens_radius > 0) { /* thin lens */
    double focus[3];
    const double rho = c->lens_radius * sqrt(s->lens[0]), phi = 2.0 * M_PI * s->lens[1];
    for(i = 0; i < 3; ++i) focus[i] = c->pos[i] + ray->dir[i] * c->focal_dst;
    for(i = 0; i < 3; ++i)
      ray->org[i] = c->pos[i] + c->r[i] * rho * cos(phi) + c->u[i] * rho * sin(phi);
    for(i = 0; i < 3; ++i) ray->dir[i] = focus[i] - ray->org[i];
  } else {
    for(i = 0; i < 3; ++i) ray->org[i] = c->pos[i];
  }
  n = sqrt(ray->dir[0] * ray->dir[0] + ray->dir[1] * ray->dir[1] + ray->dir[2] * ray->dir[2]);
  for(i = 0; i < 3; ++i) ray->dir[i] /= n;
  return RES_OK;
}

/*******************************************************************************
 * htsky over the oracle's scene
 ******************************************************************************/
struct filter_adapter {
  svx_hit_filter_T filter;
  void* context;
  const double* range;
};

static int
adapt(const struct ora_seg* seg, const double o[3], const double d[3], void* c)
{
  const struct filter_adapter* a = c;
  struct svx_hit hit;
  int pursue;
  hit.distance[0] = seg->distance[0];
  hit.distance[1] = seg->distance[1];
  hit.voxel.data = seg;
  hit.voxel.depth = 0;
  hit.voxel.id = 0;
  hit.voxel.is_leaf = 1;
  tls.seg = seg;
  pursue = a->filter(&hit, o, d, a->range, a->context);
  tls.seg = NULL;
  return pursue;
}

res_T
htsky_trace_ray(struct htsky* sky, const double org[3], const double dir[3], const double range[2],
                const svx_hit_filter_T challenge, const svx_hit_filter_T filter, void* context,
                const size_t iband, const size_t iquad, struct svx_hit* hit)
{
  const struct ora_scene* scn = sky->scn;
  struct filter_adapter a;
  struct ora_seg seg;
  int prop = ref_sw_trace_prop(filter, context);
  (void)challenge;
  if(prop < 0) prop = ref_lw_trace_prop(filter, context);
  if(prop < 0) return RES_BAD_ARG;
  a.filter = filter;
  a.context = context;
  a.range = range;
  tls.scn = scn;
  tls.trace_prop = prop;
  *hit = SVX_HIT_NULL;
  if(ora_trace_ray(scn, (uint32_t)iband, (uint32_t)(scn->quad_off[iband] + iquad), prop, org, dir,
                   range, adapt, &a, NULL, &seg)) {
    hit->distance[0] = seg.distance[0];
    hit->distance[1] = seg.distance[1];
    hit->voxel.data = NULL; /* the voxel does not outlive the traversal */
    hit->voxel.depth = 0;
    hit->voxel.id = 0;
    hit->voxel.is_leaf = 1;
  }
  tls.trace_prop = -1;
  return RES_OK;
}

double
htsky_fetch_svx_voxel_property(const struct htsky* sky, const enum htsky_property prop,
                               const enum htsky_svx_op op, const int cpnt_mask, const size_t iband,
                               const size_t iquad, const struct svx_voxel* voxel)
{
  const struct ora_seg* seg = voxel->data;
  (void)sky; (void)iband; (void)iquad;
  CHK(seg && (int)prop == tls.trace_prop && cpnt_mask == HTSKY_CPNT_MASK_ALL);
  return op == HTSKY_SVX_MIN ? seg->kmin : seg->kmax;
}

/* Site of a point outside a traversal: the last collision candidate of the
 * same position, else the cell holding it and its layer */
static void
site_outside(const struct ora_scene* scn, int prop, const double pos[3], struct ora_site* s)
{
  const struct tls_site* t = &tls.last[prop];
  if(t->valid && t->pos[0] == pos[0] && t->pos[1] == pos[1] && t->pos[2] == pos[2]) {
    *s = t->site;
    return;
  }
  {
    struct ora_seg seg;
    int64_t c[3];
    int a, inside = scn->has_cloud;
    memset(&seg, 0, sizeof(seg));
    for(a = 0; a < 3 && inside; ++a) {
      double g = floor((pos[a] - scn->lower[a]) / scn->cell[a]);
      if(scn->repeat && a < 2) {
        const double n = (double)scn->def[a];
        seg.tile[a] = (int64_t)floor(g / n);
        g -= (double)seg.tile[a] * n;
      } else if(g < 0 || g >= (double)scn->def[a]) {
        inside = 0;
      }
      c[a] = (int64_t)g;
    }
    if(inside) {
      seg.in_cloud = 1;
      for(a = 0; a < 3; ++a) { seg.lo[a] = (uint32_t)c[a]; seg.hi[a] = (uint32_t)c[a] + 1u; }
    } else {
      seg.in_cloud = 0;
      seg.layer = ora_layer_of(scn, pos[2]);
    }
    ora_site_of(scn, &seg, pos, s);
  }
}

double
htsky_fetch_raw_property(const struct htsky* sky, const enum htsky_property prop,
                         const int cpnt_mask, const size_t iband, const size_t iquad,
                         const double pos[3], const double k_min, const double k_max)
{
  const struct ora_scene* scn = sky->scn;
  struct ora_site s;
  double k;
  if(tls.seg) {
    struct tls_site* t = &tls.last[tls.trace_prop];
    ora_site_of(scn, tls.seg, pos, &s);
    t->pos[0] = pos[0]; t->pos[1] = pos[1]; t->pos[2] = pos[2];
    t->site = s;
    t->valid = 1;
  } else {
    site_outside(scn, (int)prop, pos, &s);
  }
  k = ora_site_k(scn, &s, (uint32_t)iband, (uint32_t)(scn->quad_off[iband] + iquad), (int)prop,
                 cpnt_mask);
  if(k < k_min) k = k_min;
  if(k > k_max) k = k_max;
  return k;
}

double
htsky_fetch_temperature(const struct htsky* sky, const double pos[3])
{
  const struct ora_scene* scn = sky->scn;
  struct ora_site s;
  site_outside(scn, HTSKY_Kext, pos, &s);
  return (double)scn->layer_T[s.layer >= 0 ? s.layer : ora_layer_of(scn, pos[2])];
}

double
htsky_fetch_per_wavelength_particle_phase_function_asymmetry_parameter(const struct htsky* sky,
                                                                      const double wlen)
{
  const size_t b = ora_find_band(sky->scn, wlen);
  return b < sky->scn->nbands ? (double)sky->scn->cloud_g[b] : 0.0;
}

res_T
htsky_get_spectral_band_bounds(const struct htsky* sky, const size_t iband, double bounds[2])
{
  if(iband >= sky->scn->nbands) return RES_BAD_ARG;
  bounds[0] = sky->scn->band_lo[iband];
  bounds[1] = sky->scn->band_hi[iband];
  return RES_OK;
}

size_t
htsky_find_spectral_band(const struct htsky* sky, const double wlen)
{
  return ora_find_band(sky->scn, wlen);
}

size_t
htsky_spectral_band_sample_quadrature(const struct htsky* sky, const double r, const size_t iband)
{
  return ora_sample_quad(sky->scn, r, iband);
}

/*******************************************************************************
 * Entry points of the radiance routines as the pixel callbacks call them:
 * the generator switches to transport canonicals for the walk.
 ******************************************************************************/
double
ref_entry_radiance_sw(struct htrdr_atmosphere* cmd, const size_t ithread, struct ssp_rng* rng,
                      const int cpnt_mask, const double pos[3], const double dir[3],
                      const double wlen, const size_t iband, const size_t iquad)
{
  double w;
  rng->transport = 1;
  w = atmosphere_compute_radiance_sw(cmd, ithread, rng, cpnt_mask, pos, dir, wlen, iband, iquad);
  rng->transport = 0;
  return w;
}

double
ref_entry_radiance_lw(struct htrdr_atmosphere* cmd, const size_t ithread, struct ssp_rng* rng,
                      const double pos[3], const double dir[3], const double wlen,
                      const size_t iband, const size_t iquad)
{
  double w;
  rng->transport = 1;
  w = atmosphere_compute_radiance_lw(cmd, ithread, rng, pos, dir, wlen, iband, iquad);
  rng->transport = 0;
  return w;
}
