/* Oracle: shortwave and longwave radiance realisations.
 * TEST INFRASTRUCTURE ONLY (see ora.h).  FP64 transport.
 *
 * Line-by-line restatement of
 *   src/atmosphere/htrdr_atmosphere_compute_radiance_sw.c (SW random walk)
 *   src/atmosphere/htrdr_atmosphere_compute_radiance_lw.c (LW random walk)
 * with the star-sp / star-sf services they call (exponential distance,
 * canonical numbers, Henyey-Greenstein and Rayleigh phase functions,
 * Lambertian and specular BRDFs, cosine hemisphere and spherical cap
 * sampling) restated from their published definitions.
 *
 * Random draw order (the CUDA kernels consume the same stream in the same
 * order so that realisations can be compared one by one):
 *   transport canonical u  = (w >> 8) 2^-24                 (1 word)
 *   exponential optical depth = -log((2 (w >> 9) + 1) 2^-24) (1 word)
 *   phase sample: u1 -> cos(theta), u2 -> phi                 (2 words)
 *   cosine hemisphere: u1 -> phi, u2 -> sin^2(theta)          (2 words)
 *   sun cap: u1 -> cos(theta), u2 -> phi                      (2 words) */
#include "ora_internal.h"

#include <float.h>
#include <math.h>
#include <string.h>

/* star-sp ssp_ran_exp(rng, 1) */
static double
ran_exp(struct ora_rng* rng)
{
  const uint32_t m = ora_rng_u32(rng) >> 9;
  const double u = (double)(2u * m + 1u) * (1.0 / 16777216.0);
  return -log(u);
}

static double
canonical(struct ora_rng* rng) { return ora_rng_canonical_f(rng); }

static double dot3(const double a[3], const double b[3]) { return a[0]*b[0] + a[1]*b[1] + a[2]*b[2]; }

static void
normalize3(double v[3])
{
  const double n = sqrt(dot3(v, v));
  v[0] /= n; v[1] /= n; v[2] /= n;
}

/* Direction at angle acos(mu) and azimuth phi around `axis' */
static void
around(const double axis[3], double mu, double phi, double out[3])
{
  double b1[3], b2[3];
  const double s = sqrt(fmax(0.0, 1.0 - mu * mu));
  const double cp = cos(phi) * s, sp = sin(phi) * s;
  int i;
  ora_onb(axis, b1, b2);
  for(i = 0; i < 3; ++i) out[i] = b1[i] * cp + b2[i] * sp + axis[i] * mu;
  normalize3(out);
}

/* Henyey-Greenstein: cosine between the propagation directions before and
 * after scattering (star-sf ssf_phase_hg) */
static double
hg_sample_mu(double g, double u)
{
  if(fabs(g) < 1e-6) return 1.0 - 2.0 * u;
  {
    const double s = (1.0 - g * g) / (1.0 - g + 2.0 * g * u);
    double mu = (1.0 + g * g - s * s) / (2.0 * g);
    if(mu > 1.0) mu = 1.0;
    if(mu < -1.0) mu = -1.0;
    return mu;
  }
}

static double
hg_eval(double g, double mu)
{
  const double d = 1.0 + g * g - 2.0 * g * mu;
  return (1.0 - g * g) / (4.0 * M_PI * d * sqrt(d));
}

/* Rayleigh: invert the CDF (mu^3 + 3 mu + 4)/8 with Cardano's formula
 * (star-sf ssf_phase_rayleigh) */
static double
rayleigh_sample_mu(double u)
{
  const double A = 4.0 * u - 2.0;
  const double c = cbrt(A + sqrt(A * A + 1.0));
  double mu = c - 1.0 / c;
  if(mu > 1.0) mu = 1.0;
  if(mu < -1.0) mu = -1.0;
  return mu;
}

static double
rayleigh_eval(double mu) { return 3.0 / (16.0 * M_PI) * (1.0 + mu * mu); }

enum { PHASE_HG, PHASE_RAYLEIGH };

static void
phase_sample(int type, double g, struct ora_rng* rng, const double dir[3], double out[3])
{
  const double u1 = canonical(rng), u2 = canonical(rng);
  const double mu = type == PHASE_HG ? hg_sample_mu(g, u1) : rayleigh_sample_mu(u1);
  around(dir, mu, 2.0 * M_PI * u2, out);
}

/* wo = -dir, wi = direction toward the light: mu = -wo.wi */
static double
phase_eval(int type, double g, const double wo[3], const double wi[3])
{
  const double mu = -dot3(wo, wi);
  return type == PHASE_HG ? hg_eval(g, mu) : rayleigh_eval(mu);
}

/* Cosine weighted hemisphere around N (ssp_ran_hemisphere_cos) */
static void
hemisphere_cos(struct ora_rng* rng, const double N[3], double out[3])
{
  const double u1 = canonical(rng), u2 = canonical(rng);
  around(N, sqrt(1.0 - u2), 2.0 * M_PI * u1, out);
}

/* Ground BRDF (htrdr_mtl_create_bsdf, src/core/htrdr_materials.c:414-463):
 * returns the reflectivity; *specular set for the specular BRDF */
static double
bsdf_sample(int brdf_specular, double refl, struct ora_rng* rng, const double wo[3],
            const double N[3], double out[3], int* specular)
{
  if(brdf_specular) {
    const double c = dot3(N, wo);
    int i;
    for(i = 0; i < 3; ++i) out[i] = 2.0 * c * N[i] - wo[i];
    normalize3(out);
    *specular = 1;
  } else {
    hemisphere_cos(rng, N, out);
    *specular = 0;
  }
  return refl;
}

static double
bsdf_eval(int brdf_specular, double refl, const double N[3], const double wi[3])
{
  if(brdf_specular) return 0.0;
  return dot3(N, wi) > 0 ? refl / M_PI : 0.0;
}

/* Ground query of the walk: the mesh when the scene has one (FP32 rays, as
 * the reference converts them for star-3d), else the plane.  `prev': the ray
 * leaves the ground at (prev_prim, prev_edge).  *h gets the mesh hit. */
static double
ground_query(const struct ora_scene* scn, const double o[3], const double d[3], double r1,
             int prev, uint32_t prev_prim, int prev_edge, struct ora_ghit* h)
{
  float of[3], df[3];
  int i;
  memset(h, 0, sizeof(*h));
  h->ng[2] = 1.f;
  if(!scn->g_ntris) return ora_ground_trace(scn, o, d, 0, r1, prev);
  for(i = 0; i < 3; ++i) { of[i] = (float)o[i]; df[i] = (float)d[i]; }
  *h = ora_ground_hit(scn, of, df, 0.f, r1 >= FLT_MAX ? FLT_MAX : (float)r1,
                      prev ? prev_prim : ORA_NO_PRIM, prev && prev_edge);
  return h->prim == ORA_NO_PRIM ? -1 : (double)h->dist;
}

/* Ground properties at a surface event: the normal, the BRDF and the
 * temperature.  Mesh: the material of the hit side (htrdr_interface_fetch_hit_mtl)
 * and its BRDF at the wavelength, chosen with one transport canonical
 * (htrdr_mtl_create_bsdf); a side without a BRDF reflects nothing.  Plane:
 * its constants; the canonical is drawn all the same, as
 * htrdr_mtl_create_bsdf draws it whatever the material's BRDF count
 * (src/core/htrdr_materials.c:428). */
struct surf {
  double N[3];
  double refl, T;
  int specular;
};

static struct surf
surface_props(const struct ora_scene* scn, struct ora_rng* rng, const double dir[3],
              const struct ora_ghit* h, double wlen)
{
  struct surf s;
  uint32_t m, b;
  double r, n;
  if(!scn->g_ntris) {
    (void)canonical(rng);
    s.N[0] = 0; s.N[1] = 0; s.N[2] = 1;
    s.refl = scn->ground_reflectivity;
    s.specular = scn->ground_brdf == 1;
    s.T = scn->ground_temperature;
    return s;
  }
  n = 1.0 / sqrt((double)h->ng[0] * h->ng[0] + (double)h->ng[1] * h->ng[1] + (double)h->ng[2] * h->ng[2]);
  s.N[0] = h->ng[0] * n; s.N[1] = h->ng[1] * n; s.N[2] = h->ng[2] * n;
  m = ora_hit_mtl(scn, h->prim, h->ng, dir);
  r = canonical(rng);
  b = m == ORA_NO_PRIM ? ORA_NO_PRIM : ora_fetch_brdf(scn, m, wlen, r);
  if(b == ORA_NO_PRIM) {
    s.refl = 0;
    s.specular = 0;
    s.T = m == ORA_NO_PRIM ? 0 : scn->g_mtl_T[m];
    return s;
  }
  s.specular = scn->g_brdf_type[b] != 0.f;
  s.refl = scn->g_brdf_refl[b];
  s.T = scn->g_mtl_T[m];
  return s;
}

/* Sun (src/atmosphere/htrdr_atmosphere_sun.c:126-166) */
static double
sun_sample(const struct ora_scene* scn, struct ora_rng* rng, double out[3])
{
  const double u1 = canonical(rng), u2 = canonical(rng);
  const double mu = 1.0 - u1 * (1.0 - scn->sun_cos_half);
  const double s = sqrt(fmax(0.0, 1.0 - mu * mu));
  const double phi = 2.0 * M_PI * u2;
  int i;
  for(i = 0; i < 3; ++i)
    out[i] = scn->sun_b1[i] * cos(phi) * s + scn->sun_b2[i] * sin(phi) * s + scn->sun_dir[i] * mu;
  normalize3(out);
  return 1.0 / scn->sun_solid_angle;
}

static int
in_solar_cone(const struct ora_scene* scn, const double d[3])
{
  return dot3(d, scn->sun_dir) >= scn->sun_cos_half;
}

/* Flat ground z = 0 (htrdr_atmosphere_ground_trace_ray with the self-hit
 * filter of src/core/htrdr_geometry.c:118-150: hits strictly inside the range
 * and not on the primitive the ray starts from).  Returns the distance or -1;
 * the distance is rounded to single precision, the precision of the star-3d
 * hit record the reference reads it from (s3d_hit.distance). */
double
ora_ground_trace(const struct ora_scene* scn, const double o[3], const double d[3],
                 double r0, double r1, int prev_ground)
{
  double t;
  if(!scn->has_ground || prev_ground || d[2] == 0.0) return -1;
  t = -o[2] / d[2];
  if(t <= r0 || t >= r1) return -1;
  return (double)(float)t;
}

/*******************************************************************************
 * Hit filters (..._sw.c:73-217, ..._lw.c:64-135)
 ******************************************************************************/
struct sctx { /* scattering_context / transmissivity_context / filter_context */
  const struct ora_scene* scn;
  struct ora_rng* rng;
  uint32_t band, q;
  int prop;
  double Ts, Tmin, traversal_dst;
  int event; /* LW: 0 absorption, 1 scattering, 2 none */
  struct ora_site site;
  struct ora_counters* cnt;
};

static int
scattering_hit_filter(const struct ora_seg* seg, const double o[3], const double d[3], void* c)
{
  struct sctx* ctx = c;
  const double ks_max = seg->kmax;
  ctx->traversal_dst = seg->distance[0];
  for(;;) {
    const double T = (seg->distance[1] - ctx->traversal_dst) * ks_max;
    double x[3], ks;
    struct ora_site s;
    if(ctx->Ts > T) {
      ctx->Ts -= T;
      ctx->traversal_dst = seg->distance[1];
      return 1;
    }
    ctx->traversal_dst += ctx->Ts / ks_max;
    if(ctx->traversal_dst > ORA_MAX_DIST) return 1;
    x[0] = o[0] + ctx->traversal_dst * d[0];
    x[1] = o[1] + ctx->traversal_dst * d[1];
    x[2] = o[2] + ctx->traversal_dst * d[2];
    ora_site_of(ctx->scn, seg, x, &s);
    ks = ora_site_k(ctx->scn, &s, ctx->band, ctx->q, ORA_KS, 3);
    if(ctx->cnt) ctx->cnt->ntc++;
    if(canonical(ctx->rng) < ks / ks_max) { ctx->site = s; return 0; }
    ctx->Ts = ran_exp(ctx->rng);
  }
}

static int
transmissivity_hit_filter(const struct ora_seg* seg, const double o[3], const double d[3], void* c)
{
  struct sctx* ctx = c;
  const double kmin = seg->kmin, kmax = seg->kmax;
  ctx->Tmin += (seg->distance[1] - seg->distance[0]) * kmin;
  /* From here on exp(-Tmin) is exactly 0.0 in FP64: the transmissivity is
   * zero whatever else happens, so stop like a real collision would. */
  if(ctx->Tmin >= 746.0) return 0;
  ctx->traversal_dst = seg->distance[0];
  for(;;) {
    const double Tdif = (seg->distance[1] - ctx->traversal_dst) * (kmax - kmin);
    double x[3], k;
    struct ora_site s;
    if(ctx->Ts > Tdif) {
      ctx->Ts -= Tdif;
      ctx->traversal_dst = seg->distance[1];
      return 1;
    }
    ctx->traversal_dst += ctx->Ts / (kmax - kmin);
    x[0] = o[0] + ctx->traversal_dst * d[0];
    x[1] = o[1] + ctx->traversal_dst * d[1];
    x[2] = o[2] + ctx->traversal_dst * d[2];
    ora_site_of(ctx->scn, seg, x, &s);
    k = ora_site_k(ctx->scn, &s, ctx->band, ctx->q, ctx->prop, 3);
    if(k < kmin) k = kmin; /* htsky_fetch_raw_property(..., k_min, k_max) */
    if(k > kmax) k = kmax;
    if(ctx->cnt) ctx->cnt->ntc++;
    if(canonical(ctx->rng) < (k - kmin) / (kmax - kmin)) return 0;
    ctx->Ts = ran_exp(ctx->rng);
  }
}

static int
lw_hit_filter(const struct ora_seg* seg, const double o[3], const double d[3], void* c)
{
  struct sctx* ctx = c;
  const double kext_max = seg->kmax;
  ctx->traversal_dst = seg->distance[0];
  for(;;) {
    const double T = (seg->distance[1] - ctx->traversal_dst) * kext_max;
    double x[3], ka, ks, r;
    struct ora_site s;
    if(ctx->Ts > T) {
      ctx->Ts -= T;
      ctx->traversal_dst = seg->distance[1];
      return 1;
    }
    ctx->traversal_dst += ctx->Ts / kext_max;
    x[0] = o[0] + ctx->traversal_dst * d[0];
    x[1] = o[1] + ctx->traversal_dst * d[1];
    x[2] = o[2] + ctx->traversal_dst * d[2];
    ora_site_of(ctx->scn, seg, x, &s);
    ka = ora_site_k(ctx->scn, &s, ctx->band, ctx->q, ORA_KA, 3);
    ks = ora_site_k(ctx->scn, &s, ctx->band, ctx->q, ORA_KS, 3);
    if(ctx->cnt) ctx->cnt->ntc++;
    r = canonical(ctx->rng);
    if(r < ka / kext_max) { ctx->event = 0; ctx->site = s; return 0; }
    if(r < ka / kext_max + ks / kext_max) { ctx->event = 1; ctx->site = s; return 0; }
    ctx->Ts = ran_exp(ctx->rng);
  }
}

/* ..._sw.c:219-251 */
static double
transmissivity(const struct ora_scene* scn, struct ora_rng* rng, int prop, uint32_t band,
               uint32_t q, const double pos[3], const double dir[3], const double range[2],
               struct ora_counters* cnt)
{
  struct sctx ctx;
  struct ora_seg hit;
  ctx.scn = scn; ctx.rng = rng; ctx.band = band; ctx.q = q; ctx.prop = prop;
  ctx.Ts = ran_exp(rng);
  ctx.Tmin = 0; ctx.traversal_dst = 0; ctx.cnt = cnt;
  if(ora_trace_ray(scn, band, q, prop, pos, dir, range, transmissivity_hit_filter, &ctx, cnt, &hit))
    return 0;
  return ctx.Tmin != 0 ? exp(-ctx.Tmin) : 1.0;
}

/*******************************************************************************
 * ..._sw.c:256-511
 ******************************************************************************/
double
ora_radiance_sw(const struct ora_scene* scn, struct ora_rng* rng, int cpnt_mask,
                const double pos_in[3], const double dir_in[3], double wlen, size_t iband,
                size_t iquad, int dir_in_cone, struct ora_counters* cnt)
{
  const uint32_t band = (uint32_t)iband;
  const uint32_t q = (uint32_t)(scn->quad_off[iband] + iquad);
  const double g = (double)scn->cloud_g[iband];
  const double L_sun = ora_planck_monochromatic(wlen * 1e-9, scn->sun_temperature);
  double pos[3], dir[3], range[2];
  double ksi = 1, w = 0;
  int prev_ground = 0, prev_edge = 0, i;
  uint32_t prev_prim = ORA_NO_PRIM;
  struct ora_ghit gh;
  for(i = 0; i < 3; ++i) { pos[i] = pos_in[i]; dir[i] = dir_in[i]; }

  if((cpnt_mask & ORA_DIRECT) && (dir_in_cone || in_solar_cone(scn, dir))) {
    range[0] = 0; range[1] = FLT_MAX;
    if(ground_query(scn, pos, dir, range[1], 0, 0, 0, &gh) < 0) {
      const double Tr = transmissivity(scn, rng, ORA_KEXT, band, q, pos, dir, range, cnt);
      w = L_sun * Tr;
    }
  }
  if(!(cpnt_mask & ORA_DIFFUSE)) return w;

  for(;;) {
    struct sctx sc;
    struct ora_seg hit;
    double pos_next[3], dir_next[3], wo[3], N[3] = {0, 0, 1}, sun_dir[3];
    double ground_dst, Tr_abs, Tr, R, sun_pdf, refl = 1;
    int surface, svx_hit, specular = 0, phase = PHASE_HG;
    struct surf sp = {{0, 0, 1}, 0, 0, 0};

    ground_dst = ground_query(scn, pos, dir, DBL_MAX, prev_ground, prev_prim, prev_edge, &gh);

    sc.scn = scn; sc.rng = rng; sc.band = band; sc.q = q; sc.prop = ORA_KS; sc.cnt = cnt;
    sc.Ts = ran_exp(rng);
    sc.traversal_dst = 0; sc.Tmin = 0;
    range[0] = 0; range[1] = ground_dst >= 0 ? ground_dst : FLT_MAX;
    svx_hit = ora_trace_ray(scn, band, q, ORA_KS, pos, dir, range, scattering_hit_filter, &sc,
                            cnt, &hit);
    if(ground_dst < 0 && !svx_hit) break;

    wo[0] = -dir[0]; wo[1] = -dir[1]; wo[2] = -dir[2];
    surface = !svx_hit;
    /* a surface event lies where the traversal ended (..._sw.c:382-385):
     * the ground distance, or the column's bottom if that is nearer */
    for(i = 0; i < 3; ++i) pos_next[i] = pos[i] + dir[i] * sc.traversal_dst;
    prev_ground = surface;
    if(surface) { prev_prim = gh.prim; prev_edge = ora_on_edge(gh.u, gh.v) && scn->g_ntris; }

    range[0] = 0; range[1] = sc.traversal_dst;
    Tr_abs = transmissivity(scn, rng, ORA_KA, band, q, pos, dir, range, cnt);
    if(Tr_abs <= 0) break;

    if(surface) {
      sp = surface_props(scn, rng, dir, &gh, wlen);
      N[0] = sp.N[0]; N[1] = sp.N[1]; N[2] = sp.N[2];
      if(dot3(N, wo) < 0) { N[0] = -N[0]; N[1] = -N[1]; N[2] = -N[2]; }
      refl = bsdf_sample(sp.specular, sp.refl, rng, wo, N, dir_next, &specular);
    } else {
      const double ks_gas = ora_site_k(scn, &sc.site, band, q, ORA_KS, 1);
      const double ks_par = ora_site_k(scn, &sc.site, band, q, ORA_KS, 2);
      const double ks = ks_par + ks_gas;
      phase = canonical(rng) < ks_gas / ks ? PHASE_RAYLEIGH : PHASE_HG;
      phase_sample(phase, g, rng, dir, dir_next);
    }

    if(surface && specular) {
      if(!in_solar_cone(scn, dir_next)) {
        R = 0;
      } else {
        for(i = 0; i < 3; ++i) sun_dir[i] = dir_next[i];
        R = dot3(N, sun_dir) < 0 ? 0 : refl;
      }
      sun_pdf = 1.0;
    } else {
      sun_pdf = sun_sample(scn, rng, sun_dir);
      if(surface) {
        R = dot3(N, sun_dir) < 0 ? 0 : bsdf_eval(sp.specular, sp.refl, N, sun_dir) * dot3(N, sun_dir);
      } else {
        R = phase_eval(phase, g, wo, sun_dir);
      }
    }

    if(R <= 0) {
      Tr = 0;
    } else {
      range[0] = 0; range[1] = FLT_MAX;
      struct ora_ghit sh;
      if(ground_query(scn, pos_next, sun_dir, range[1], prev_ground, prev_prim, prev_edge, &sh) >= 0) Tr = 0;
      else Tr = transmissivity(scn, rng, ORA_KEXT, band, q, pos_next, sun_dir, range, cnt);
    }

    ksi *= Tr_abs;
    w += ksi * L_sun * Tr * R / sun_pdf;

    if(surface && canonical(rng) >= refl) break;

    for(i = 0; i < 3; ++i) { pos[i] = pos_next[i]; dir[i] = dir_next[i]; }
  }
  return w;
}

/*******************************************************************************
 * ..._lw.c:140-279
 ******************************************************************************/
double
ora_radiance_lw(const struct ora_scene* scn, struct ora_rng* rng, const double pos_in[3],
                const double dir_in[3], double wlen, size_t iband, size_t iquad,
                struct ora_counters* cnt)
{
  const uint32_t band = (uint32_t)iband;
  const uint32_t q = (uint32_t)(scn->quad_off[iband] + iquad);
  const double g = (double)scn->cloud_g[iband];
  const double wlen_m = wlen * 1e-9;
  double pos[3], dir[3], range[2], w = 0;
  int prev_ground = 0, prev_edge = 0, i;
  uint32_t prev_prim = ORA_NO_PRIM;
  for(i = 0; i < 3; ++i) { pos[i] = pos_in[i]; dir[i] = dir_in[i]; }

  for(;;) {
    struct sctx c;
    struct ora_seg hit;
    struct ora_ghit gh;
    double pos_next[3], dir_next[3], wo[3];
    const double ground_dst = ground_query(scn, pos, dir, DBL_MAX, prev_ground, prev_prim, prev_edge,
                                           &gh);
    int svx_hit;

    c.scn = scn; c.rng = rng; c.band = band; c.q = q; c.prop = ORA_KEXT; c.cnt = cnt;
    c.Ts = ran_exp(rng);
    c.traversal_dst = 0; c.Tmin = 0; c.event = 2;
    range[0] = 0; range[1] = ground_dst >= 0 ? ground_dst : FLT_MAX;
    svx_hit = ora_trace_ray(scn, band, q, ORA_KEXT, pos, dir, range, lw_hit_filter, &c, cnt, &hit);

    if(ground_dst < 0 && !svx_hit) { w = 0; break; }
    for(i = 0; i < 3; ++i) pos_next[i] = pos[i] + dir[i] * c.traversal_dst;

    if(svx_hit && c.event == 0) { /* absorption: emission at the local temperature */
      const int l = c.site.layer >= 0 ? c.site.layer : ora_layer_of(scn, pos_next[2]);
      w = ora_planck_monochromatic(wlen_m, (double)scn->layer_T[l]);
      break;
    }
    wo[0] = -dir[0]; wo[1] = -dir[1]; wo[2] = -dir[2];
    if(svx_hit) { /* scattering */
      phase_sample(PHASE_HG, g, rng, dir, dir_next);
      prev_ground = 0;
    } else { /* surface */
      const struct surf sp = surface_props(scn, rng, dir, &gh, wlen);
      double N[3];
      int specular;
      double refl;
      N[0] = sp.N[0]; N[1] = sp.N[1]; N[2] = sp.N[2];
      if(dot3(N, wo) < 0) { N[0] = -N[0]; N[1] = -N[1]; N[2] = -N[2]; }
      refl = bsdf_sample(sp.specular, sp.refl, rng, wo, N, dir_next, &specular);
      if(canonical(rng) >= refl) {
        const double T = sp.T;
        w = T > 0 ? ora_planck_monochromatic(wlen_m, T) : 0;
        break;
      }
      prev_ground = 1;
      prev_prim = gh.prim;
      prev_edge = scn->g_ntris && ora_on_edge(gh.u, gh.v);
    }
    for(i = 0; i < 3; ++i) { pos[i] = pos_next[i]; dir[i] = dir_next[i]; }
  }
  return w;
}

int
ora_radiance_batch(const struct ora_scene* scn, int lw, size_t n, const double* pos,
                   const double* dir, const double* wlen, const uint32_t* iband,
                   const uint32_t* iquad, int cpnt_mask, uint32_t seed, double* out,
                   int nthreads)
{
  long long i;
  if(nthreads > 0) omp_set_num_threads_wrapper(nthreads);
  #pragma omp parallel for schedule(dynamic, 64)
  for(i = 0; i < (long long)n; ++i) {
    struct ora_rng rng;
    ora_rng_init(&rng, (uint32_t)i, seed, 0, 0);
    if(lw) out[i] = ora_radiance_lw(scn, &rng, pos + 3 * i, dir + 3 * i, wlen[i], iband[i], iquad[i], NULL);
    else out[i] = ora_radiance_sw(scn, &rng, cpnt_mask, pos + 3 * i, dir + 3 * i, wlen[i], iband[i], iquad[i], 0, NULL);
  }
  return ORA_RES_OK;
}
