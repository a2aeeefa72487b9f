/* Harness of the compiled reference oracle.  TEST INFRASTRUCTURE ONLY.
 *
 * src/atmosphere/htrdr_atmosphere_draw_map.c is compiled unmodified in this
 * translation unit, with its two calls into the radiance routines routed
 * through the shim's entry points (which switch the generator to transport
 * canonicals for the walk).  The harness builds the command object
 * (struct htrdr_atmosphere, src/atmosphere/htrdr_atmosphere_c.h:95-128) the
 * way htrdr_atmosphere_create does (src/atmosphere/htrdr_atmosphere.c:287-446)
 * from an oracle scene and request, runs the reference's atmosphere_draw_map,
 * and replaces only the core map driver (src/core/htrdr_draw_map.c): its
 * tiles, per-tile Threefry streams and MPI gather become a loop over pixels
 * with one stream per (pixel, realisation), the index space of the oracle
 * and of the CUDA library. */
#define atmosphere_compute_radiance_sw ref_entry_radiance_sw
#define atmosphere_compute_radiance_lw ref_entry_radiance_lw
#include "htrdr_atmosphere_draw_map.c"
#undef atmosphere_compute_radiance_sw
#undef atmosphere_compute_radiance_lw

#include "core/htrdr_buffer.h"
#include "core/htrdr_ran_wlen_cie_xyz.h"
#include "core/htrdr_ran_wlen_planck.h"
#include "core/htrdr_rectangle.h"

#include "ref.h"
#include "ref_shim.h"
#include "../ora_internal.h"

#ifdef _OPENMP
#include <omp.h>
#endif

struct ref_scene {
  struct ora_scene* scn;
  struct htsky sky;
  struct htrdr_atmosphere_ground ground;
  struct htrdr_atmosphere_sun* sun;
  struct htrdr htrdr;
};

/* What the map driver needs beyond the reference's arguments */
static struct {
  uint32_t seed;
  size_t pix_begin, pix_end;
  int nthreads;
} g_drv;

static int
max_threads(void)
{
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

static int
thread_id(void)
{
#ifdef _OPENMP
  return omp_get_thread_num();
#else
  return 0;
#endif
}

int
ref_scene_create(const struct ora_scene_desc* d, struct ref_scene** out)
{
  struct ref_scene* rs;
  int res;
  if(!d || !out) return RES_BAD_ARG;
  if(d->ground_ntris) return RES_BAD_ARG; /* the harness grounds are planes */
  rs = calloc(1, sizeof(*rs));
  if(!rs) return RES_MEM_ERR;
  res = ora_scene_create(d, &rs->scn);
  if(res != ORA_RES_OK) { free(rs); return res; }
  rs->sky.scn = rs->scn;
  rs->ground.has_ground = d->has_ground;
  rs->ground.brdf = d->ground_brdf;
  rs->ground.reflectivity = d->ground_reflectivity;
  rs->ground.temperature = d->ground_temperature;
  rs->htrdr.nthreads = (unsigned)max_threads();
  rs->htrdr.verbose = 0;
  rs->htrdr.allocator = htrdr_get_allocator(&rs->htrdr);
  ref_init(&rs->htrdr.ref);
  /* htrdr_atmosphere.c:360-364: the reference's sun, pointed at the
   * direction of the scene's azimuth and elevation */
  res = htrdr_atmosphere_sun_create(&rs->htrdr, &rs->sun);
  if(res != RES_OK) { ora_scene_release(rs->scn); free(rs); return res; }
  htrdr_atmosphere_sun_set_direction(rs->sun, rs->scn->sun_dir);
  *out = rs;
  return RES_OK;
}

void
ref_scene_release(struct ref_scene* rs)
{
  if(!rs) return;
  if(rs->sun) htrdr_atmosphere_sun_ref_put(rs->sun);
  ora_scene_release(rs->scn);
  free(rs);
}

/* atmosphere_get_pixel_format (src/atmosphere/htrdr_atmosphere.c:482-509) */
void
atmosphere_get_pixel_format(const struct htrdr_atmosphere* cmd, struct htrdr_pixel_format* fmt)
{
  if(cmd->output_type == HTRDR_ATMOSPHERE_ARGS_OUTPUT_FLUX_MAP) {
    fmt->size = sizeof(struct atmosphere_pixel_flux);
    fmt->alignment = ALIGNOF(struct atmosphere_pixel_flux);
  } else if(cmd->spectral_type == HTRDR_SPECTRAL_SW_CIE_XYZ) {
    fmt->size = sizeof(struct atmosphere_pixel_image);
    fmt->alignment = ALIGNOF(struct atmosphere_pixel_image);
  } else {
    fmt->size = sizeof(struct atmosphere_pixel_xwave);
    fmt->alignment = ALIGNOF(struct atmosphere_pixel_xwave);
  }
}

/* The core map driver in place of src/core/htrdr_draw_map.c:496-621: the
 * same argument checks (:66-79), then every pixel of [pix_begin, pix_end)
 * drawn by the callback with its own streams, OpenMP over the pixels. */
res_T
htrdr_draw_map(struct htrdr* htrdr, const struct htrdr_draw_map_args* args,
               struct htrdr_buffer* buf)
{
  const struct htrdr_buffer_layout* L;
  long long p;
  if(!args || !args->draw_pixel || !args->spp) return RES_BAD_ARG;
  if(htrdr_buffer_layout_check(&args->buffer_layout) != RES_OK) return RES_BAD_ARG;
  L = &args->buffer_layout;
  if(g_drv.nthreads > 0) omp_set_num_threads_wrapper(g_drv.nthreads);
  #pragma omp parallel for schedule(dynamic, 1)
  for(p = (long long)g_drv.pix_begin; p < (long long)g_drv.pix_end; ++p) {
    struct ssp_rng rng;
    struct htrdr_draw_pixel_args pa = HTRDR_DRAW_PIXEL_ARGS_NULL;
    const size_t x = (size_t)p % L->width, y = (size_t)p / L->width;
    memset(&rng, 0, sizeof(rng));
    pa.pixel_coord[0] = x;
    pa.pixel_coord[1] = y;
    pa.pixel_normalized_size[0] = 1.0 / (double)L->width;
    pa.pixel_normalized_size[1] = 1.0 / (double)L->height;
    pa.rng = &rng;
    pa.spp = args->spp;
    pa.ithread = (size_t)thread_id();
    pa.context = args->context;
    ref_hook_begin(&rng, (uint32_t)p, g_drv.seed, NULL);
    args->draw_pixel(htrdr, &pa, htrdr_buffer_at(buf, x, y));
    ref_hook_end();
  }
  return RES_OK;
}

/* The command object of a request: htrdr_atmosphere_create's sensor, sampler
 * and buffer set-up (src/atmosphere/htrdr_atmosphere.c:357-435) */
struct cmd_ctx {
  struct htrdr_atmosphere cmd;
  struct scam camera;
};

static void
norm3(double v[3])
{
  const double n = sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
  v[0] /= n; v[1] /= n; v[2] /= n;
}

static void
cross3(double o[3], const double a[3], const double b[3])
{
  o[0] = a[1] * b[2] - a[2] * b[1];
  o[1] = a[2] * b[0] - a[0] * b[2];
  o[2] = a[0] * b[1] - a[1] * b[0];
}

static int
cmd_setup(struct cmd_ctx* c, const struct ref_scene* rs_c, const struct ora_request* req)
{
  struct ref_scene* rs = (struct ref_scene*)rs_c;
  struct htrdr_atmosphere* cmd = &c->cmd;
  const int cie = req->mode == ORA_IMAGE_CIE;
  const int flux = req->mode == ORA_FLUX_SW || req->mode == ORA_FLUX_LW;
  const int lw = req->mode == ORA_XWAVE_LW || req->mode == ORA_FLUX_LW;
  double range_nm[2];
  size_t nintervals;
  int i, res;

  memset(c, 0, sizeof(*c));
  cmd->ground = &rs->ground;
  cmd->sun = rs->sun;
  cmd->sky = &rs->sky;
  cmd->sky_mtl_name = "air";
  cmd->htrdr = &rs->htrdr;
  cmd->spectral_type = cie ? HTRDR_SPECTRAL_SW_CIE_XYZ : (lw ? HTRDR_SPECTRAL_LW : HTRDR_SPECTRAL_SW);
  cmd->output_type = flux ? HTRDR_ATMOSPHERE_ARGS_OUTPUT_FLUX_MAP : HTRDR_ATMOSPHERE_ARGS_OUTPUT_IMAGE;
  cmd->wlen_range_m[0] = req->wlen_range[0] * 1e-9;
  cmd->wlen_range_m[1] = req->wlen_range[1] * 1e-9;
  cmd->ref_temperature = req->ref_temperature;
  cmd->spp = req->spp;
  cmd->width = req->width;
  cmd->height = req->height;
  cmd->nthreads = rs->htrdr.nthreads;

  /* compute_spectral_bands_count (src/atmosphere/htrdr_atmosphere.c:53-70) */
  range_nm[0] = cmd->wlen_range_m[0] * 1.e9;
  range_nm[1] = cmd->wlen_range_m[1] * 1.e9;
  nintervals = (size_t)rint(range_nm[1] - range_nm[0]);
  if(cie) {
    res = htrdr_ran_wlen_cie_xyz_create(&rs->htrdr, req->wlen_range, nintervals, &cmd->cie);
  } else {
    if(cmd->ref_temperature <= 0) return RES_BAD_ARG;
    res = htrdr_ran_wlen_planck_create(&rs->htrdr, req->wlen_range, nintervals,
                                       cmd->ref_temperature, &cmd->planck);
  }
  if(res != RES_OK) return res;

  if(flux) {
    res = htrdr_rectangle_create(&rs->htrdr, req->rect_size, req->rect_pos, req->rect_tgt,
                                 req->rect_up, &cmd->flux_map);
    if(res != RES_OK) return res;
  } else { /* star-camera: frame from position, target and up */
    struct scam* cam = &c->camera;
    for(i = 0; i < 3; ++i) { cam->pos[i] = req->cam_pos[i]; cam->f[i] = req->cam_tgt[i] - req->cam_pos[i]; }
    norm3(cam->f);
    cross3(cam->r, cam->f, req->cam_up);
    norm3(cam->r);
    cross3(cam->u, cam->r, cam->f);
    cam->tan_half = tan(req->fov_deg * M_PI / 360.0);
    cam->aspect = (double)req->width / (double)req->height;
    cam->lens_radius = req->lens_radius;
    cam->focal_dst = req->focal_dst;
    cam->ortho_h = req->ortho_height;
    cam->type = req->camera_type;
    cmd->camera = cam;
  }

  { /* the output buffer (htrdr_atmosphere.c:418-435) */
    struct htrdr_pixel_format fmt;
    atmosphere_get_pixel_format(cmd, &fmt);
    cmd->buf_layout.width = req->width;
    cmd->buf_layout.height = req->height;
    cmd->buf_layout.pitch = req->width * fmt.size;
    cmd->buf_layout.elmt_size = fmt.size;
    cmd->buf_layout.alignment = fmt.alignment;
    res = htrdr_buffer_create(&rs->htrdr, &cmd->buf_layout, &cmd->buf);
    if(res != RES_OK) return res;
    memset(htrdr_buffer_at(cmd->buf, 0, 0), 0, cmd->buf_layout.pitch * req->height);
  }
  return RES_OK;
}

static void
cmd_release(struct cmd_ctx* c)
{
  struct htrdr_atmosphere* cmd = &c->cmd;
  if(cmd->buf) htrdr_buffer_ref_put(cmd->buf);
  if(cmd->flux_map) htrdr_rectangle_ref_put(cmd->flux_map);
  if(cmd->cie) htrdr_ran_wlen_cie_xyz_ref_put(cmd->cie);
  if(cmd->planck) htrdr_ran_wlen_planck_ref_put(cmd->planck);
}

int
ref_draw_map(const struct ref_scene* rs, const struct ora_request* req, void* buffer, size_t pitch,
             size_t pix_begin, size_t pix_end, int nthreads, const char* dump_path)
{
  struct cmd_ctx c;
  const size_t npix = (size_t)req->width * req->height;
  size_t y;
  int res;
  if(!rs || !req || !buffer || !req->spp || !req->width || !req->height) return RES_BAD_ARG;
  res = cmd_setup(&c, rs, req);
  if(res != RES_OK) { cmd_release(&c); return res; }
  if(pitch < c.cmd.buf_layout.pitch) { cmd_release(&c); return RES_BAD_ARG; }
  g_drv.seed = req->seed;
  g_drv.pix_begin = pix_begin < npix ? pix_begin : npix;
  g_drv.pix_end = pix_end < npix ? pix_end : npix;
  g_drv.nthreads = nthreads;
  c.cmd.output = dump_path ? fopen(dump_path, "w") : tmpfile();
  if(!c.cmd.output) { cmd_release(&c); return RES_IO_ERR; }
  res = atmosphere_draw_map(&c.cmd);
  fclose(c.cmd.output);
  if(res == RES_OK) {
    for(y = 0; y < req->height; ++y)
      memcpy((char*)buffer + y * pitch, htrdr_buffer_at(c.cmd.buf, 0, y), c.cmd.buf_layout.pitch);
  }
  cmd_release(&c);
  return res;
}

int
ref_realisation_weights(const struct ref_scene* rs, const struct ora_request* req,
                        size_t pix_begin, size_t pix_end, double* weights, int nthreads)
{
  struct cmd_ctx c;
  struct htrdr_draw_map_args args;
  const int cie = req->mode == ORA_IMAGE_CIE;
  const uint32_t spp = req->spp, nr = spp * (cie ? 3u : 1u);
  long long p;
  int res;
  if(!rs || !req || !weights || !req->spp) return RES_BAD_ARG;
  res = cmd_setup(&c, rs, req);
  if(res != RES_OK) { cmd_release(&c); return res; }
  /* the reference's own choice of callback (draw_map.c:438-475) */
  if(c.cmd.output_type == HTRDR_ATMOSPHERE_ARGS_OUTPUT_FLUX_MAP)
    setup_draw_map_args_rectangle(&c.cmd, &args);
  else
    setup_draw_map_args_camera(&c.cmd, &args);
  if(nthreads > 0) omp_set_num_threads_wrapper(nthreads);
  #pragma omp parallel for schedule(dynamic, 1)
  for(p = (long long)pix_begin; p < (long long)pix_end; ++p) {
    struct ssp_rng rng;
    struct htrdr_draw_pixel_args pa = HTRDR_DRAW_PIXEL_ARGS_NULL;
    union { struct atmosphere_pixel_xwave x; struct atmosphere_pixel_flux f;
            struct atmosphere_pixel_image i; } pix;
    double* out = weights + (size_t)(p - (long long)pix_begin) * nr;
    uint32_t r;
    memset(&rng, 0, sizeof(rng));
    pa.pixel_coord[0] = (size_t)p % req->width;
    pa.pixel_coord[1] = (size_t)p / req->width;
    pa.pixel_normalized_size[0] = 1.0 / (double)req->width;
    pa.pixel_normalized_size[1] = 1.0 / (double)req->height;
    pa.rng = &rng;
    pa.spp = 1; /* one realisation per call (one per channel for CIE) */
    pa.ithread = (size_t)thread_id();
    pa.context = &c.cmd;
    for(r = 0; r < spp; ++r) {
      const uint32_t keys[3] = {r, spp + r, 2 * spp + r};
      memset(&pix, 0, sizeof(pix));
      ref_hook_begin(&rng, (uint32_t)p, req->seed, keys);
      args.draw_pixel(&((struct ref_scene*)rs)->htrdr, &pa, &pix);
      ref_hook_end();
      if(c.cmd.output_type == HTRDR_ATMOSPHERE_ARGS_OUTPUT_FLUX_MAP) {
        out[r] = pix.f.flux.nweights ? pix.f.flux.sum_weights : NAN;
      } else if(cie) {
        out[r] = pix.i.X.E;
        out[spp + r] = pix.i.Y.E;
        out[2 * spp + r] = pix.i.Z.E;
      } else {
        out[r] = pix.x.radiance.E;
      }
    }
  }
  cmd_release(&c);
  return RES_OK;
}

int
ref_radiance_batch(const struct ref_scene* rs_c, int lw, size_t n, const double* pos,
                   const double* dir, const double* wlen, const uint32_t* iband,
                   const uint32_t* iquad, int cpnt_mask, uint32_t seed, double* out, int nthreads)
{
  struct ref_scene* rs = (struct ref_scene*)rs_c;
  struct htrdr_atmosphere cmd;
  long long i;
  if(!rs || (n && (!pos || !dir || !wlen || !iband || !iquad || !out))) return RES_BAD_ARG;
  memset(&cmd, 0, sizeof(cmd));
  cmd.ground = &rs->ground;
  cmd.sun = rs->sun;
  cmd.sky = &rs->sky;
  cmd.sky_mtl_name = "air";
  cmd.htrdr = &rs->htrdr;
  cmd.spectral_type = lw ? HTRDR_SPECTRAL_LW : HTRDR_SPECTRAL_SW;
  if(nthreads > 0) omp_set_num_threads_wrapper(nthreads);
  #pragma omp parallel for schedule(dynamic, 64)
  for(i = 0; i < (long long)n; ++i) {
    struct ssp_rng rng;
    memset(&rng, 0, sizeof(rng));
    ora_rng_init(&rng.r, (uint32_t)i, seed, 0, 0); /* the oracle's batch keying */
    out[i] = lw
      ? ref_entry_radiance_lw(&cmd, (size_t)thread_id(), &rng, pos + 3 * i, dir + 3 * i, wlen[i],
                              iband[i], iquad[i])
      : ref_entry_radiance_sw(&cmd, (size_t)thread_id(), &rng, cpnt_mask, pos + 3 * i, dir + 3 * i,
                              wlen[i], iband[i], iquad[i]);
  }
  return RES_OK;
}
