/* Oracle: per-pixel realisation callbacks and the tiled map driver.
 * TEST INFRASTRUCTURE ONLY (see ora.h).
 *
 * Restates src/atmosphere/htrdr_atmosphere_draw_map.c (draw_pixel_image,
 * draw_pixel_flux, draw_pixel_xwave, sample_rectangle_ray) and the tile loop
 * of src/core/htrdr_draw_map.c (8x8 tiles in Morton order, pixels in Morton
 * order inside a tile, OpenMP over tiles), single process. */
#include "ora_internal.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#define TILE_SIZE 8

/* htrdr_accum / htrdr_estimate (src/core/htrdr_accum.h:31-46) */
struct accum { double sum_weights, sum_weights_sqr; size_t nweights, nfailures; };
struct estimate { double E, SE; };
struct pixel_xwave { struct estimate radiance, radiance_temperature; struct accum time; };
struct pixel_flux { struct accum flux, time; };
struct pixel_image { struct estimate X, Y, Z; struct accum time; };

/* src/core/htrdr_accum.h:48-68 */
static struct estimate
get_estimation(const struct accum* a)
{
  struct estimate e = {0, 0};
  if(a->nweights) {
    const double N = (double)a->nweights;
    const double E = a->sum_weights / N;
    double V = a->sum_weights_sqr / N - E * E;
    if(V < 0) V = 0;
    e.E = E;
    e.SE = sqrt(V / N);
  }
  return e;
}

static void
accum_add(struct accum* a, double w)
{
  a->sum_weights += w;
  a->sum_weights_sqr += w * w;
  a->nweights += 1;
}

static double
now_usec(void)
{
  struct timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return (double)ts.tv_sec * 1e6 + (double)ts.tv_nsec * 1e-3;
}

static double dot3(const double a[3], const double b[3]) { return a[0]*b[0] + a[1]*b[1] + a[2]*b[2]; }
static void
cross3(double o[3], const double a[3], const double b[3])
{
  o[0] = a[1] * b[2] - a[2] * b[1];
  o[1] = a[2] * b[0] - a[0] * b[2];
  o[2] = a[0] * b[1] - a[1] * b[0];
}
static void
normalize3(double v[3])
{
  const double n = sqrt(dot3(v, v));
  v[0] /= n; v[1] /= n; v[2] /= n;
}

/* Sensors: star-camera perspective/orthographic camera and
 * src/core/htrdr_rectangle.c */
struct sensor {
  double pos[3], f[3], r[3], u[3];
  double tan_half, aspect;
  double lens_radius, focal_dst, ortho_h;
  int type;
  /* rectangle */
  double rpos[3], axis_x[3], axis_y[3], normal[3];
};

static void
setup_sensor(const struct ora_request* req, struct sensor* s)
{
  double t[3];
  int i;
  memset(s, 0, sizeof(*s));
  for(i = 0; i < 3; ++i) { s->pos[i] = req->cam_pos[i]; s->f[i] = req->cam_tgt[i] - req->cam_pos[i]; }
  normalize3(s->f);
  cross3(s->r, s->f, req->cam_up);
  normalize3(s->r);
  cross3(s->u, s->r, s->f);
  s->tan_half = tan(req->fov_deg * M_PI / 360.0);
  s->aspect = (double)req->width / (double)req->height;
  s->lens_radius = req->lens_radius;
  s->focal_dst = req->focal_dst;
  s->ortho_h = req->ortho_height;
  s->type = req->camera_type;
  /* htrdr_rectangle_create (src/core/htrdr_rectangle.c:66-135) */
  for(i = 0; i < 3; ++i) { s->normal[i] = req->rect_tgt[i] - req->rect_pos[i]; s->rpos[i] = req->rect_pos[i]; }
  normalize3(s->normal);
  cross3(s->axis_x, s->normal, req->rect_up);
  normalize3(s->axis_x);
  cross3(t, s->normal, s->axis_x);
  normalize3(t);
  for(i = 0; i < 3; ++i) {
    s->axis_y[i] = t[i] * req->rect_size[1] * 0.5;
    s->axis_x[i] *= req->rect_size[0] * 0.5;
  }
}

static void
camera_ray(const struct sensor* s, const double film[2], const double lens[2], double org[3],
           double dir[3])
{
  const double x = 2.0 * film[0] - 1.0, y = 2.0 * film[1] - 1.0;
  int i;
  if(s->type == 1) { /* orthographic */
    const double hw = 0.5 * s->ortho_h * s->aspect, hh = 0.5 * s->ortho_h;
    for(i = 0; i < 3; ++i) { org[i] = s->pos[i] + s->r[i] * x * hw + s->u[i] * y * hh; dir[i] = s->f[i]; }
    return;
  }
  for(i = 0; i < 3; ++i)
    dir[i] = s->f[i] + s->r[i] * (x * s->tan_half * s->aspect) + s->u[i] * (y * s->tan_half);
  if(s->lens_radius > 0) { /* thin lens */
    double focus[3];
    const double rho = s->lens_radius * sqrt(lens[0]), phi = 2.0 * M_PI * lens[1];
    for(i = 0; i < 3; ++i) focus[i] = s->pos[i] + dir[i] * s->focal_dst;
    for(i = 0; i < 3; ++i) org[i] = s->pos[i] + s->r[i] * rho * cos(phi) + s->u[i] * rho * sin(phi);
    for(i = 0; i < 3; ++i) dir[i] = focus[i] - org[i];
  } else {
    for(i = 0; i < 3; ++i) org[i] = s->pos[i];
  }
  normalize3(dir);
}

struct drv {
  const struct ora_scene* scn;
  const struct ora_request* req;
  struct sensor sensor;
  struct ora_planck_ran planck;
  struct ora_cie_ran cie;
  double wlen_range_m[2];
};

/* One realisation: returns 0 when the sample is rejected, the weight in *w. */
static int
realisation(const struct drv* dv, uint32_t px, uint32_t py, uint32_t ireal, double* w,
            struct ora_counters* cnt)
{
  const struct ora_request* req = dv->req;
  const struct ora_scene* scn = dv->scn;
  const double pix_sz[2] = {1.0 / (double)req->width, 1.0 / (double)req->height};
  struct ora_rng rng;
  double org[3], dir[3], r0, r1, r2, wlen, pdf;
  size_t iband, iquad;
  ora_rng_init(&rng, py * req->width + px, req->seed, ireal, 0);

  if(req->mode == ORA_FLUX_SW || req->mode == ORA_FLUX_LW) {
    /* sample_rectangle_ray (draw_map.c:51-107) */
    double s[2];
    int i;
    s[0] = ((double)px + ora_rng_canonical_d(&rng)) * pix_sz[0];
    s[1] = ((double)py + ora_rng_canonical_d(&rng)) * pix_sz[1];
    for(i = 0; i < 3; ++i)
      org[i] = dv->sensor.rpos[i] + dv->sensor.axis_x[i] * (s[0] * 2.0 - 1.0)
             + dv->sensor.axis_y[i] * (s[1] * 2.0 - 1.0);
    if(!scn->g_ntris) {
      if(scn->has_ground && org[2] < 0) return 0; /* inside the ground: rejected */
    } else { /* the upward ray must leave through the atmosphere's side (:73-99) */
      const float of[3] = {(float)org[0], (float)org[1], (float)org[2]}, up[3] = {0, 0, 1};
      const struct ora_ghit h = ora_ground_hit(scn, of, up, 0.f, FLT_MAX, ORA_NO_PRIM, 0);
      if(h.prim != ORA_NO_PRIM) {
        const uint32_t* f = scn->g_iface + 3 * (size_t)scn->g_iface_of[h.prim];
        if((h.ng[2] < 0.f ? f[0] : f[2]) != scn->g_sky_mtl) return 0; /* cos(up, N) < 0: front */
      }
    }
    {
      const double u1 = ora_rng_canonical_f(&rng), u2 = ora_rng_canonical_f(&rng);
      double b1[3], b2[3];
      const double mu = sqrt(1.0 - u2), sn = sqrt(u2), phi = 2.0 * M_PI * u1;
      ora_onb(dv->sensor.normal, b1, b2);
      for(i = 0; i < 3; ++i)
        dir[i] = b1[i] * cos(phi) * sn + b2[i] * sin(phi) * sn + dv->sensor.normal[i] * mu;
      normalize3(dir);
    }
  } else {
    double film[2], lens[2];
    film[0] = ((double)px + ora_rng_canonical_d(&rng)) * pix_sz[0];
    film[1] = ((double)py + ora_rng_canonical_d(&rng)) * pix_sz[1];
    lens[0] = ora_rng_canonical_d(&rng);
    lens[1] = ora_rng_canonical_d(&rng);
    camera_ray(&dv->sensor, film, lens, org, dir);
  }
  r0 = ora_rng_canonical_d(&rng);
  r1 = ora_rng_canonical_d(&rng);
  r2 = ora_rng_canonical_d(&rng);
  if(req->mode == ORA_IMAGE_CIE) {
    const int ch = (int)(ireal / req->spp);
    wlen = ora_cie_ran_sample(&dv->cie, ch, r0, r1, &pdf);
  } else {
    wlen = ora_planck_ran_sample(&dv->planck, r0, r1, &pdf);
  }
  pdf *= 1e9;
  iband = ora_find_band(scn, wlen);
  if(iband >= scn->nbands) return 0;
  iquad = ora_sample_quad(scn, r2, iband);
  if(cnt) cnt->nreal++;

  switch(req->mode) {
    case ORA_XWAVE_LW:
      *w = ora_radiance_lw(scn, &rng, org, dir, wlen, iband, iquad, cnt) / pdf;
      break;
    case ORA_FLUX_LW:
      *w = ora_radiance_lw(scn, &rng, org, dir, wlen, iband, iquad, cnt) * M_PI / pdf;
      break;
    case ORA_FLUX_SW: { /* draw_map.c:269-301 */
      double sun_dir[3], cosN, L_direct, L_diffuse, u1, u2, mu, sn, phi;
      int i;
      u1 = ora_rng_canonical_f(&rng); u2 = ora_rng_canonical_f(&rng);
      mu = 1.0 - u1 * (1.0 - scn->sun_cos_half);
      sn = sqrt(fmax(0.0, 1.0 - mu * mu));
      phi = 2.0 * M_PI * u2;
      for(i = 0; i < 3; ++i)
        sun_dir[i] = scn->sun_b1[i] * cos(phi) * sn + scn->sun_b2[i] * sin(phi) * sn
                   + scn->sun_dir[i] * mu;
      normalize3(sun_dir);
      cosN = dot3(dv->sensor.normal, sun_dir);
      L_direct = cosN <= 0 ? 0
        : ora_radiance_sw(scn, &rng, ORA_DIRECT, org, sun_dir, wlen, iband, iquad, 0, cnt);
      L_diffuse = ora_radiance_sw(scn, &rng, ORA_DIFFUSE, org, dir, wlen, iband, iquad, 0, cnt);
      *w = (cosN * scn->sun_solid_angle * L_direct + M_PI * L_diffuse) / pdf;
      break;
    }
    default: /* XWAVE_SW, IMAGE_CIE */
      *w = ora_radiance_sw(scn, &rng, ORA_ALL, org, dir, wlen, iband, iquad, 0, cnt) / pdf;
      break;
  }
  return 1;
}

static int
drv_init(struct drv* dv, const struct ora_scene* scn, const struct ora_request* req)
{
  int res;
  memset(dv, 0, sizeof(*dv));
  dv->scn = scn;
  dv->req = req;
  setup_sensor(req, &dv->sensor);
  dv->wlen_range_m[0] = req->wlen_range[0] * 1e-9;
  dv->wlen_range_m[1] = req->wlen_range[1] * 1e-9;
  /* compute_spectral_bands_count (src/atmosphere/htrdr_atmosphere.c:53-70) */
  {
    const size_t nb = (size_t)rint(req->wlen_range[1] - req->wlen_range[0]);
    if(req->mode == ORA_IMAGE_CIE) res = ora_cie_ran_init(&dv->cie, req->wlen_range, nb ? nb : 1);
    else res = ora_planck_ran_init(&dv->planck, req->wlen_range, nb, req->ref_temperature);
  }
  return res;
}

static void
drv_release(struct drv* dv)
{
  if(dv->req->mode == ORA_IMAGE_CIE) ora_cie_ran_release(&dv->cie);
  else ora_planck_ran_release(&dv->planck);
}

/* draw_pixel_{xwave,flux,image} (draw_map.c:109-436) */
static void
draw_pixel(const struct drv* dv, uint32_t px, uint32_t py, void* out, struct ora_counters* cnt)
{
  const struct ora_request* req = dv->req;
  struct accum acc[3], time = {0, 0, 0, 0};
  const uint32_t nch = req->mode == ORA_IMAGE_CIE ? 3 : 1;
  uint32_t ch, is;
  memset(acc, 0, sizeof(acc));
  for(ch = 0; ch < nch; ++ch) {
    for(is = 0; is < req->spp; ++is) {
      const double t0 = now_usec();
      double w = 0;
      if(!realisation(dv, px, py, ch * req->spp + is, &w, cnt)) continue;
      accum_add(&acc[ch], w);
      accum_add(&time, now_usec() - t0);
    }
  }
  switch(req->mode) {
    case ORA_FLUX_SW:
    case ORA_FLUX_LW: {
      struct pixel_flux* p = out;
      p->flux = acc[0];
      p->time = time;
      break;
    }
    case ORA_IMAGE_CIE: {
      struct pixel_image* p = out;
      p->X = get_estimation(&acc[0]);
      p->Y = get_estimation(&acc[1]);
      p->Z = get_estimation(&acc[2]);
      p->time = time;
      break;
    }
    default: {
      struct pixel_xwave* p = out;
      p->radiance = get_estimation(&acc[0]);
      p->radiance_temperature.E = 0;
      p->radiance_temperature.SE = 0;
      p->time = time;
      if(req->mode == ORA_XWAVE_LW) { /* draw_map.c:425-435 */
        const double lo = dv->wlen_range_m[0], hi = dv->wlen_range_m[1];
        double tmin, tmax;
        p->radiance_temperature.E = ora_radiance_temperature(lo, hi, p->radiance.E);
        tmin = ora_radiance_temperature(lo, hi, p->radiance.E - p->radiance.SE);
        tmax = ora_radiance_temperature(lo, hi, p->radiance.E + p->radiance.SE);
        p->radiance_temperature.SE = tmax - tmin;
      }
      break;
    }
  }
}

/* rsys morton_xy_decode_u16: x from the even bits, y from the odd bits */
static uint16_t
compact_bits(uint32_t v)
{
  v &= 0x55555555u;
  v = (v ^ (v >> 1)) & 0x33333333u;
  v = (v ^ (v >> 2)) & 0x0F0F0F0Fu;
  v = (v ^ (v >> 4)) & 0x00FF00FFu;
  v = (v ^ (v >> 8)) & 0x0000FFFFu;
  return (uint16_t)v;
}

static size_t
round_up_pow2(size_t v)
{
  size_t p = 1;
  while(p < v) p <<= 1;
  return p;
}

static size_t
pixel_size(int mode)
{
  return mode == ORA_IMAGE_CIE ? sizeof(struct pixel_image)
       : (mode == ORA_FLUX_SW || mode == ORA_FLUX_LW) ? sizeof(struct pixel_flux)
       : sizeof(struct pixel_xwave);
}

/* htrdr_draw_map / draw_map / draw_tile (src/core/htrdr_draw_map.c:270-491) */
int
ora_draw_map(const struct ora_scene* scn, const struct ora_request* req, void* buffer,
             size_t pitch, size_t pix_begin, size_t pix_end, int nthreads,
             struct ora_counters* cnt)
{
  struct drv dv;
  size_t ntx, nty, nadj;
  long long mc;
  const size_t psz = pixel_size(req->mode);
  uint64_t nseg = 0, nnode = 0, ntc = 0, nreal = 0;
  int res;
  if(!req->spp || !req->width || !req->height) return ORA_RES_BAD_ARG;
  if(pitch < req->width * psz) return ORA_RES_BAD_ARG;
  res = drv_init(&dv, scn, req);
  if(res != ORA_RES_OK) return res;
  ntx = (req->width + TILE_SIZE - 1) / TILE_SIZE;
  nty = (req->height + TILE_SIZE - 1) / TILE_SIZE;
  nadj = round_up_pow2(ntx > nty ? ntx : nty);
  nadj *= nadj;
  if(nthreads > 0) omp_set_num_threads_wrapper(nthreads);
  #pragma omp parallel for schedule(dynamic, 1) reduction(+:nseg, nnode, ntc, nreal)
  for(mc = 0; mc < (long long)nadj; ++mc) {
    const uint16_t tx = compact_bits((uint32_t)mc), ty = compact_bits((uint32_t)mc >> 1);
    size_t tsz[2], np, m;
    struct ora_counters c = {0, 0, 0, 0};
    if(tx >= ntx || ty >= nty) continue;
    tsz[0] = req->width - (size_t)tx * TILE_SIZE;
    tsz[1] = req->height - (size_t)ty * TILE_SIZE;
    if(tsz[0] > TILE_SIZE) tsz[0] = TILE_SIZE;
    if(tsz[1] > TILE_SIZE) tsz[1] = TILE_SIZE;
    np = round_up_pow2(tsz[0] > tsz[1] ? tsz[0] : tsz[1]);
    np *= np;
    for(m = 0; m < np; ++m) {
      const uint16_t ix = compact_bits((uint32_t)m), iy = compact_bits((uint32_t)m >> 1);
      const uint32_t px = (uint32_t)tx * TILE_SIZE + ix, py = (uint32_t)ty * TILE_SIZE + iy;
      const size_t lin = (size_t)py * req->width + px;
      if(ix >= tsz[0] || iy >= tsz[1]) continue;
      if(lin < pix_begin || lin >= pix_end) continue;
      draw_pixel(&dv, px, py, (char*)buffer + (size_t)py * pitch + (size_t)px * psz, &c);
    }
    nseg += c.nseg; nnode += c.nnode; ntc += c.ntc; nreal += c.nreal;
  }
  if(cnt) { cnt->nseg += nseg; cnt->nnode += nnode; cnt->ntc += ntc; cnt->nreal += nreal; }
  drv_release(&dv);
  return ORA_RES_OK;
}

/* Wavelength sampling of a request (CDF band, wavelength in nm, pdf in nm^-1) */
int
ora_sample_wavelength(const struct ora_scene* scn, const struct ora_request* req, int channel,
                      size_t n, const double* r0, const double* r1, uint32_t* cdf_band,
                      double* wlen, double* pdf)
{
  struct drv dv;
  size_t i;
  int res = drv_init(&dv, scn, req);
  if(res != ORA_RES_OK) return res;
  for(i = 0; i < n; ++i) {
    if(req->mode == ORA_IMAGE_CIE) {
      cdf_band[i] = (uint32_t)ora_cie_ran_band(&dv.cie, channel, r0[i]);
      wlen[i] = ora_cie_ran_sample(&dv.cie, channel, r0[i], r1[i], &pdf[i]);
    } else {
      cdf_band[i] = dv.planck.nbands ? (uint32_t)ora_planck_ran_band(&dv.planck, r0[i]) : 0;
      wlen[i] = ora_planck_ran_sample(&dv.planck, r0[i], r1[i], &pdf[i]);
    }
  }
  drv_release(&dv);
  return ORA_RES_OK;
}

int
ora_realisation_weights(const struct ora_scene* scn, const struct ora_request* req,
                        size_t pix_begin, size_t pix_end, double* weights, int nthreads)
{
  struct drv dv;
  const uint32_t nr = req->spp * (req->mode == ORA_IMAGE_CIE ? 3u : 1u);
  long long p;
  int res = drv_init(&dv, scn, req);
  if(res != ORA_RES_OK) return res;
  if(nthreads > 0) omp_set_num_threads_wrapper(nthreads);
  #pragma omp parallel for schedule(dynamic, 1)
  for(p = (long long)pix_begin; p < (long long)pix_end; ++p) {
    const uint32_t px = (uint32_t)(p % req->width), py = (uint32_t)(p / req->width);
    uint32_t r;
    for(r = 0; r < nr; ++r) {
      double w = 0;
      if(!realisation(&dv, px, py, r, &w, NULL)) w = NAN;
      weights[(size_t)(p - (long long)pix_begin) * nr + r] = w;
    }
  }
  drv_release(&dv);
  return ORA_RES_OK;
}
