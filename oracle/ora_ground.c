/* TEST INFRASTRUCTURE (CPU oracle). Ground mesh of the atmosphere scene:
 * ray queries against every triangle (no acceleration structure) with the
 * self-hit filter, the infinite repetition of the mesh's bounding box, and
 * the interface/material/BRDF lookups.
 *
 *   htrdr_atmosphere_ground_trace_ray   src/atmosphere/htrdr_atmosphere_ground.c:162-209
 *   self_hit / hit_on_edge              src/core/htrdr_geometry.c:96-150
 *   htrdr_slab_trace_ray                src/core/htrdr_slab.c:33-142
 *   htrdr_interface_fetch_hit_mtl       src/core/htrdr_interface.h:44-80
 *   htrdr_mtl_create_bsdf               src/core/htrdr_materials.c:414-463
 *
 * The ray/triangle test is Moller-Trumbore in FP32, evaluated operation by
 * operation (this file is compiled without floating-point contraction), the
 * same arithmetic as the CUDA library, so both find the same hits.  The
 * closest hit the filter keeps wins; ties go to the smaller primitive id.
 * mrumtl (the reference's BRDF tables) is not vendored: a material is a list
 * of BRDFs tabulated by wavelength, and the BRDF at a wavelength is one of the
 * two around it, chosen with probability linear in the wavelength. */
#include "ora_internal.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

static float f_dot(const float a[3], const float b[3])
{
  const float x = a[0] * b[0];
  const float y = a[1] * b[1];
  const float z = a[2] * b[2];
  const float s = x + y;
  return s + z;
}

static void f_cross(float r[3], const float a[3], const float b[3])
{
  float p, q;
  p = a[1] * b[2]; q = a[2] * b[1]; r[0] = p - q;
  p = a[2] * b[0]; q = a[0] * b[2]; r[1] = p - q;
  p = a[0] * b[1]; q = a[1] * b[0]; r[2] = p - q;
}

static void f_sub(float r[3], const float a[3], const float b[3])
{
  r[0] = a[0] - b[0]; r[1] = a[1] - b[1]; r[2] = a[2] - b[2];
}

int
ora_on_edge(float u, float v)
{
  const float w = (1.f - u) - v;
  const float e = 1.e-4f;
  return fabsf(u) <= e || fabsf(u - 1.f) <= e || fabsf(v) <= e || fabsf(v - 1.f) <= e
      || fabsf(w) <= e || fabsf(w - 1.f) <= e;
}

static int
intersect(const float o[3], const float d[3], const float* v, float* t, float* u, float* vv)
{
  float e1[3], e2[3], p[3], s[3], q[3], det, inv, uu, w;
  f_sub(e1, v + 3, v);
  f_sub(e2, v + 6, v);
  f_cross(p, d, e2);
  det = f_dot(e1, p);
  if(det == 0.f) return 0;
  inv = 1.f / det;
  f_sub(s, o, v);
  uu = f_dot(s, p) * inv;
  if(!(uu >= 0.f && uu <= 1.f)) return 0;
  f_cross(q, s, e1);
  w = f_dot(d, q) * inv;
  if(!(w >= 0.f && uu + w <= 1.f)) return 0;
  *t = f_dot(e2, q) * inv;
  *u = uu;
  *vv = w;
  return 1;
}

static int
self_hit(float t, uint32_t prim, float u, float v, float r0, float r1, uint32_t from_prim,
         int from_edge)
{
  if(t <= r0 || t >= r1) return 1;
  if(prim == from_prim) return 1;
  if(from_prim != ORA_NO_PRIM && fabsf(t) <= 1.e-1f && from_edge && ora_on_edge(u, v)) return 1;
  return 0;
}

static struct ora_ghit
trace_mesh(const struct ora_scene* scn, const float o[3], const float d[3], float r0, float r1,
           uint32_t from_prim, int from_edge)
{
  struct ora_ghit h;
  uint32_t i;
  float best = r1;
  memset(&h, 0, sizeof(h));
  h.dist = -1.f;
  h.prim = ORA_NO_PRIM;
  for(i = 0; i < scn->g_ntris; ++i) {
    float t, u, v;
    if(!intersect(o, d, scn->g_v + 9 * (size_t)i, &t, &u, &v)) continue;
    if(self_hit(t, i, u, v, r0, r1, from_prim, from_edge)) continue;
    if(t < best || (t == best && h.prim != ORA_NO_PRIM && i < h.prim)) {
      best = t;
      h.dist = t;
      h.prim = i;
      h.u = u;
      h.v = v;
    }
  }
  if(h.prim != ORA_NO_PRIM) {
    const float* tv = scn->g_v + 9 * (size_t)h.prim;
    float e1[3], e2[3];
    f_sub(e1, tv + 3, tv);
    f_sub(e2, tv + 6, tv);
    f_cross(h.ng, e2, e1);
  }
  return h;
}

struct ora_ghit
ora_ground_hit(const struct ora_scene* scn, const float o[3], const float d[3], float r0, float r1,
               uint32_t from_prim, int from_edge)
{
  struct ora_ghit none;
  double org[3], dir[3], tmin, tmax[3], sz[2], tdelta[2], px, py;
  int64_t xy[2];
  int incr[2], a, step;
  if(!scn->g_repeat) return trace_mesh(scn, o, d, r0, r1, from_prim, from_edge);
  memset(&none, 0, sizeof(none));
  none.dist = -1.f;
  none.prim = ORA_NO_PRIM;
  for(a = 0; a < 3; ++a) { org[a] = o[a]; dir[a] = d[a]; }
  /* htrdr_slab_trace_ray */
  tmin = (scn->g_lower[2] - org[2]) / dir[2];
  tmax[2] = (scn->g_upper[2] - org[2]) / dir[2];
  if(tmin > tmax[2]) { const double t = tmin; tmin = tmax[2]; tmax[2] = t; }
  tmin = fmax(tmin, (double)r0);
  tmax[2] = fmin(tmax[2], (double)r1);
  if(tmin > tmax[2]) return none;
  sz[0] = scn->g_upper[0] - scn->g_lower[0];
  sz[1] = scn->g_upper[1] - scn->g_lower[1];
  px = org[0] + tmin * dir[0];
  py = org[1] + tmin * dir[1];
  xy[0] = (int64_t)floor((px - scn->g_lower[0]) / sz[0]);
  xy[1] = (int64_t)floor((py - scn->g_lower[1]) / sz[1]);
  incr[0] = dir[0] < 0 ? -1 : 1;
  incr[1] = dir[1] < 0 ? -1 : 1;
  for(a = 0; a < 2; ++a) {
    const double lo = scn->g_lower[a] + (double)xy[a] * sz[a];
    tmax[a] = ((dir[a] < 0 ? lo : lo + sz[a]) - org[a]) / dir[a];
    tdelta[a] = (dir[a] < 0 ? -sz[a] : sz[a]) / dir[a];
  }
  for(step = 0; step < 32; ++step) {
    float oc[3];
    struct ora_ghit h;
    int ax;
    oc[0] = (float)(org[0] - (double)xy[0] * sz[0]);
    oc[1] = (float)(org[1] - (double)xy[1] * sz[1]);
    oc[2] = o[2];
    h = trace_mesh(scn, oc, d, r0, r1, from_prim, from_edge);
    if(h.prim != ORA_NO_PRIM) return h;
    ax = tmax[0] < tmax[1] ? (tmax[0] < tmax[2] ? 0 : 2) : (tmax[1] < tmax[2] ? 1 : 2);
    if(ax == 2) break;
    if(tmax[ax] >= (double)r1) break;
    tmax[ax] += tdelta[ax];
    xy[ax] += incr[ax];
  }
  return none;
}

uint32_t
ora_hit_mtl(const struct ora_scene* scn, uint32_t prim, const float ng[3], const double dir[3])
{
  const uint32_t* f = scn->g_iface + 3 * (size_t)scn->g_iface_of[prim];
  const double n = 1.0 / sqrt((double)ng[0] * ng[0] + (double)ng[1] * ng[1] + (double)ng[2] * ng[2]);
  int front;
  uint32_t m;
  if(f[1] != ORA_NO_PRIM) return f[1];
  front = ((double)ng[0] * dir[0] + (double)ng[1] * dir[1] + (double)ng[2] * dir[2]) * n < 0;
  m = front ? f[2] : f[0]; /* the material on the other side */
  if(m == ORA_NO_PRIM || !scn->g_mtl_n[m]) m = front ? f[0] : f[2];
  return m;
}

uint32_t
ora_fetch_brdf(const struct ora_scene* scn, uint32_t mtl, double wlen, double r)
{
  const uint32_t first = scn->g_mtl_first[mtl], n = scn->g_mtl_n[mtl];
  const double* wl = scn->g_brdf_wl + first;
  uint32_t lo = 0, hi;
  double u;
  if(!n) return ORA_NO_PRIM;
  if(wlen <= wl[0]) return first;
  if(wlen >= wl[n - 1]) return first + n - 1;
  hi = n - 1;
  while(hi - lo > 1) {
    const uint32_t mid = (lo + hi) >> 1;
    if(wl[mid] <= wlen) lo = mid; else hi = mid;
  }
  u = (wlen - wl[lo]) / (wl[hi] - wl[lo]);
  return first + (r < u ? hi : lo);
}

int
ora_ground_setup(struct ora_scene* scn, const struct ora_scene_desc* d)
{
  uint32_t i, a, nb = 0;
  scn->g_ntris = 0;
  scn->g_sky_mtl = ORA_NO_PRIM;
  if(!d->ground_ntris) return 0;
  scn->g_ntris = d->ground_ntris;
  scn->g_nmtls = d->ground_nmtls;
  scn->g_repeat = d->repeat_ground;
  scn->g_sky_mtl = d->ground_sky_mtl;
  scn->g_v = malloc(sizeof(float) * 9 * (size_t)d->ground_ntris);
  scn->g_iface_of = malloc(sizeof(uint32_t) * d->ground_ntris);
  scn->g_iface = malloc(sizeof(uint32_t) * 3 * (size_t)d->ground_nifaces);
  scn->g_mtl_first = malloc(sizeof(uint32_t) * d->ground_nmtls);
  scn->g_mtl_n = malloc(sizeof(uint32_t) * d->ground_nmtls);
  scn->g_mtl_T = malloc(sizeof(float) * d->ground_nmtls);
  for(i = 0; i < d->ground_nmtls; ++i) nb += d->ground_mtl_nbrdf[i];
  scn->g_brdf_wl = malloc(sizeof(double) * (nb ? nb : 1));
  scn->g_brdf_type = malloc(sizeof(float) * (nb ? nb : 1));
  scn->g_brdf_refl = malloc(sizeof(float) * (nb ? nb : 1));
  if(!scn->g_v || !scn->g_iface_of || !scn->g_iface || !scn->g_mtl_first || !scn->g_mtl_n
  || !scn->g_mtl_T || !scn->g_brdf_wl || !scn->g_brdf_type || !scn->g_brdf_refl)
    return -1;
  for(a = 0; a < 3; ++a) { scn->g_lower[a] = DBL_MAX; scn->g_upper[a] = -DBL_MAX; }
  for(i = 0; i < d->ground_ntris; ++i) {
    uint32_t k;
    for(k = 0; k < 3; ++k) {
      const float* p = d->ground_verts + 3 * (size_t)d->ground_tris[3 * (size_t)i + k];
      for(a = 0; a < 3; ++a) {
        scn->g_v[9 * (size_t)i + 3 * k + a] = p[a];
        scn->g_lower[a] = fmin(scn->g_lower[a], (double)p[a]);
        scn->g_upper[a] = fmax(scn->g_upper[a], (double)p[a]);
      }
    }
    scn->g_iface_of[i] = d->ground_tri_iface[i];
  }
  memcpy(scn->g_iface, d->ground_ifaces, sizeof(uint32_t) * 3 * (size_t)d->ground_nifaces);
  nb = 0;
  for(i = 0; i < d->ground_nmtls; ++i) {
    uint32_t k;
    scn->g_mtl_first[i] = nb;
    scn->g_mtl_n[i] = d->ground_mtl_nbrdf[i];
    scn->g_mtl_T[i] = (float)d->ground_mtl_temperature[i];
    for(k = 0; k < d->ground_mtl_nbrdf[i]; ++k, ++nb) {
      scn->g_brdf_wl[nb] = d->ground_mtl_brdf[3 * (size_t)nb];
      scn->g_brdf_type[nb] = (float)d->ground_mtl_brdf[3 * (size_t)nb + 1];
      scn->g_brdf_refl[nb] = (float)d->ground_mtl_brdf[3 * (size_t)nb + 2];
    }
  }
  return 0;
}

void
ora_ground_release(struct ora_scene* scn)
{
  free(scn->g_v);
  free(scn->g_iface_of);
  free(scn->g_iface);
  free(scn->g_mtl_first);
  free(scn->g_mtl_n);
  free(scn->g_mtl_T);
  free(scn->g_brdf_wl);
  free(scn->g_brdf_type);
  free(scn->g_brdf_refl);
}

int
ora_ground_trace_batch(const struct ora_scene* scn, size_t n, const float* rays, const float* tmax,
                       const uint32_t* from_prim, const uint8_t* from_edge, uint32_t* prim,
                       float* dist)
{
  size_t i;
  if(!scn || (n && (!rays || !tmax || !from_prim || !from_edge || !prim || !dist)))
    return ORA_RES_BAD_ARG;
  if(!scn->g_ntris) return ORA_RES_BAD_OP;
  for(i = 0; i < n; ++i) {
    const struct ora_ghit h = ora_ground_hit(scn, rays + 6 * i, rays + 6 * i + 3, 0.f, tmax[i],
                                             from_prim[i], from_edge[i] != 0);
    prim[i] = h.prim;
    dist[i] = h.prim == ORA_NO_PRIM ? -1.f : h.dist;
  }
  return ORA_RES_OK;
}
