/* Ground geometry on the device: ray queries against the triangle mesh of
 * the ground through its BVH, with the reference's self-hit filter, and the
 * infinite repetition of the mesh's bounding box in X and Y.
 *
 *   htrdr_atmosphere_ground_trace_ray (src/atmosphere/htrdr_atmosphere_ground.c:162-209)
 *   geometry_filter / self_hit / hit_on_edge (src/core/htrdr_geometry.c:96-173)
 *   htrdr_slab_trace_ray (src/core/htrdr_slab.c:33-142)
 *
 * The ray/triangle test is Moller-Trumbore in FP32 with every product and sum
 * rounded separately (no fused multiply-add), so that the CPU restatement,
 * compiled without contraction, finds the same hits bit for bit.  The closest
 * hit that the filter keeps wins; ties go to the smaller primitive id. */
#ifndef HTRDR_GROUND_CUH
#define HTRDR_GROUND_CUH

#include <cuda_runtime.h>
#include <float.h>
#include <stdint.h>

#include "dscene.h"

#define HG_NO_PRIM 0xFFFFFFFFu
#define HG_BVH_STACK HG_BVH_DEPTH_MAX
#define HG_SLAB_STEPS 32 /* repeated cells walked per ray (src/atmosphere/htrdr_atmosphere_ground.c:203) */

namespace {

struct GHit {
  float dist;    /* < 0: no hit */
  uint32_t prim; /* primitive id of the caller */
  float u, v;    /* barycentric coordinates of v1, v2 */
  float3 ng;     /* geometric normal (v2 - v0) x (v1 - v0), not normalised */
};

__device__ __forceinline__ float g_mul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float g_add(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float g_sub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float g_dot(float3 a, float3 b)
{
  return g_add(g_add(g_mul(a.x, b.x), g_mul(a.y, b.y)), g_mul(a.z, b.z));
}
__device__ __forceinline__ float3 g_cross(float3 a, float3 b)
{
  return make_float3(g_sub(g_mul(a.y, b.z), g_mul(a.z, b.y)),
                     g_sub(g_mul(a.z, b.x), g_mul(a.x, b.z)),
                     g_sub(g_mul(a.x, b.y), g_mul(a.y, b.x)));
}
__device__ __forceinline__ float3 g_diff(float3 a, float3 b)
{
  return make_float3(g_sub(a.x, b.x), g_sub(a.y, b.y), g_sub(a.z, b.z));
}

/* hit_on_edge: a barycentric coordinate within 1e-4 of 0 or 1 */
__device__ __forceinline__ bool
g_on_edge(float u, float v)
{
  const float w = g_sub(g_sub(1.f, u), v);
  const float e = 1.e-4f;
  return fabsf(u) <= e || fabsf(u - 1.f) <= e || fabsf(v) <= e || fabsf(v - 1.f) <= e
      || fabsf(w) <= e || fabsf(w - 1.f) <= e;
}

/* Moller-Trumbore (two-sided): distance and barycentrics, false on a miss */
__device__ __forceinline__ bool
g_intersect(float3 o, float3 d, float3 v0, float3 v1, float3 v2, float* t, float* u, float* v)
{
  const float3 e1 = g_diff(v1, v0), e2 = g_diff(v2, v0);
  const float3 p = g_cross(d, e2);
  const float det = g_dot(e1, p);
  if(det == 0.f) return false;
  const float inv = __fdiv_rn(1.f, det);
  const float3 s = g_diff(o, v0);
  const float uu = g_mul(g_dot(s, p), inv);
  if(!(uu >= 0.f && uu <= 1.f)) return false;
  const float3 q = g_cross(s, e1);
  const float vv = g_mul(g_dot(d, q), inv);
  if(!(vv >= 0.f && g_add(uu, vv) <= 1.f)) return false;
  *t = g_mul(g_dot(e2, q), inv);
  *u = uu;
  *v = vv;
  return true;
}

/* self_hit (src/core/htrdr_geometry.c:114-150): true to discard the hit */
__device__ __forceinline__ bool
g_self_hit(float t, uint32_t prim, float u, float v, float r0, float r1, uint32_t from_prim,
           bool from_edge)
{
  if(t <= r0 || t >= r1) return true;
  if(prim == from_prim) return true;
  if(from_prim != HG_NO_PRIM && fabsf(t) <= 1.e-1f && from_edge && g_on_edge(u, v)) return true;
  return false;
}

__device__ __forceinline__ bool
g_box(float3 o, float3 inv, float4 lo, float4 hi, float r0, float tbest)
{
  /* slightly widened so that rounding never culls a box whose triangle the
   * exact test accepts */
  float t0 = r0 - 1e-3f, t1 = tbest;
  float a = (lo.x - o.x) * inv.x, b = (hi.x - o.x) * inv.x;
  t0 = fmaxf(t0, fminf(a, b)); t1 = fminf(t1, fmaxf(a, b));
  a = (lo.y - o.y) * inv.y; b = (hi.y - o.y) * inv.y;
  t0 = fmaxf(t0, fminf(a, b)); t1 = fminf(t1, fmaxf(a, b));
  a = (lo.z - o.z) * inv.z; b = (hi.z - o.z) * inv.z;
  t0 = fmaxf(t0, fminf(a, b)); t1 = fminf(t1, fmaxf(a, b));
  const float pad = 1e-4f * fmaxf(fabsf(t1), 1.f);
  return t0 <= t1 + pad;
}

/* Closest kept hit of one (untranslated) copy of the mesh */
__device__ __noinline__ GHit
g_trace_mesh(const DScene& S, float3 o, float3 d, float r0, float r1, uint32_t from_prim,
             bool from_edge)
{
  GHit h;
  h.dist = -1.f;
  h.prim = HG_NO_PRIM;
  h.u = h.v = 0.f;
  h.ng = make_float3(0.f, 0.f, 0.f);
  float best = r1;
  uint32_t best_i = HG_NO_PRIM;
  const float3 inv = make_float3(1.f / d.x, 1.f / d.y, 1.f / d.z);
  uint32_t stack[HG_BVH_STACK];
  int sp = 0;
  stack[sp++] = 0;
  while(sp > 0) {
    const uint32_t ni = stack[--sp];
    const float4 a = __ldg(S.g_bvh + 2 * ni), b = __ldg(S.g_bvh + 2 * ni + 1);
    if(!g_box(o, inv, a, b, r0, best)) continue;
    const uint32_t first = __float_as_uint(a.w), count = __float_as_uint(b.w);
    if(count == 0) {
      if(sp + 2 <= HG_BVH_STACK) { stack[sp++] = first + 1; stack[sp++] = first; }
      continue;
    }
    for(uint32_t i = first; i < first + count; ++i) {
      const float4 p0 = __ldg(S.g_tri + 3 * i), p1 = __ldg(S.g_tri + 3 * i + 1),
                   p2 = __ldg(S.g_tri + 3 * i + 2);
      float t, u, v;
      if(!g_intersect(o, d, make_float3(p0.x, p0.y, p0.z), make_float3(p1.x, p1.y, p1.z),
                      make_float3(p2.x, p2.y, p2.z), &t, &u, &v))
        continue;
      const uint32_t prim = __ldg(S.g_tri_id + i);
      if(g_self_hit(t, prim, u, v, r0, r1, from_prim, from_edge)) continue;
      if(t < best || (t == best && best_i != HG_NO_PRIM && prim < h.prim)) {
        best = t;
        best_i = i;
        h.dist = t;
        h.prim = prim;
        h.u = u;
        h.v = v;
      }
    }
  }
  if(best_i != HG_NO_PRIM) {
    const float4 p0 = __ldg(S.g_tri + 3 * best_i), p1 = __ldg(S.g_tri + 3 * best_i + 1),
                 p2 = __ldg(S.g_tri + 3 * best_i + 2);
    const float3 v0 = make_float3(p0.x, p0.y, p0.z);
    h.ng = g_cross(g_diff(make_float3(p2.x, p2.y, p2.z), v0), g_diff(make_float3(p1.x, p1.y, p1.z), v0));
  }
  return h;
}

/* htrdr_atmosphere_ground_trace_ray on the mesh: one copy, or the copies of
 * the bounding box repeated in X and Y walked by htrdr_slab_trace_ray (FP64
 * cell walk, the mesh traced with the origin moved into each cell). */
__device__ __noinline__ GHit
g_trace(const DScene& S, float3 o, float3 d, float r0, float r1, uint32_t from_prim, bool from_edge)
{
  if(!S.g_repeat) return g_trace_mesh(S, o, d, r0, r1, from_prim, from_edge);
  GHit none;
  none.dist = -1.f;
  none.prim = HG_NO_PRIM;
  none.u = none.v = 0.f;
  none.ng = make_float3(0.f, 0.f, 0.f);
  const double org[3] = {o.x, o.y, o.z}, dir[3] = {d.x, d.y, d.z};
  const double rg0 = r0, rg1 = r1;
  double tmin = (S.g_lower[2] - org[2]) / dir[2];
  double tmax[3];
  tmax[2] = (S.g_upper[2] - org[2]) / dir[2];
  if(tmin > tmax[2]) { const double t = tmin; tmin = tmax[2]; tmax[2] = t; }
  tmin = fmax(tmin, rg0);
  tmax[2] = fmin(tmax[2], rg1);
  if(tmin > tmax[2]) return none;
  double sz[2] = {S.g_upper[0] - S.g_lower[0], S.g_upper[1] - S.g_lower[1]};
  const double px = org[0] + tmin * dir[0], py = org[1] + tmin * dir[1];
  long long xy[2] = {(long long)floor((px - S.g_lower[0]) / sz[0]),
                     (long long)floor((py - S.g_lower[1]) / sz[1])};
  const int incr[2] = {dir[0] < 0 ? -1 : 1, dir[1] < 0 ? -1 : 1};
  double tdelta[2];
  for(int a = 0; a < 2; ++a) {
    const double lo = S.g_lower[a] + (double)xy[a] * sz[a];
    tmax[a] = ((dir[a] < 0 ? lo : lo + sz[a]) - org[a]) / dir[a];
    tdelta[a] = (dir[a] < 0 ? -sz[a] : sz[a]) / dir[a];
  }
  for(int step = 0; step < HG_SLAB_STEPS; ++step) {
    const float3 oc = make_float3((float)(org[0] - (double)xy[0] * sz[0]),
                                  (float)(org[1] - (double)xy[1] * sz[1]), o.z);
    const GHit h = g_trace_mesh(S, oc, d, r0, r1, from_prim, from_edge);
    if(h.prim != HG_NO_PRIM) return h;
    const int ax = tmax[0] < tmax[1] ? (tmax[0] < tmax[2] ? 0 : 2) : (tmax[1] < tmax[2] ? 1 : 2);
    if(ax == 2) break;
    if(tmax[ax] >= rg1) break;
    tmax[ax] += tdelta[ax];
    xy[ax] += incr[ax];
  }
  return none;
}

/* Material of the side the ray arrives from the other side of
 * (htrdr_interface_fetch_hit_mtl, src/core/htrdr_interface.h:44-80): the
 * thin material when set, else the material opposite the hit side, else
 * the other one.  ~0u when none is defined. */
__device__ __forceinline__ uint32_t
g_hit_mtl(const DScene& S, uint32_t prim, float3 ng, float3 dir)
{
  const uint4 f = __ldg(S.g_iface + __ldg(S.g_iface_of + prim));
  if(f.y != HG_NO_PRIM) return f.y;
  const float n = rsqrtf(ng.x * ng.x + ng.y * ng.y + ng.z * ng.z);
  const bool front = (ng.x * dir.x + ng.y * dir.y + ng.z * dir.z) * n < 0.f;
  uint32_t m = front ? f.z : f.x; /* the material on the other side */
  if(m == HG_NO_PRIM || !__ldg(S.g_mtl + m).y) m = front ? f.x : f.z;
  return m;
}

/* BRDF of a material at a wavelength: the tabulated BRDF at or beside the
 * wavelength, the two around it chosen with probability linear in the
 * wavelength (r in [0, 1) decides); outside the table the nearest entry.
 * Returns the BRDF index (~0u when the material has none). */
__device__ __forceinline__ uint32_t
g_fetch_brdf(const DScene& S, uint32_t mtl, double wlen, double r)
{
  const uint2 m = __ldg(S.g_mtl + mtl);
  if(!m.y) return HG_NO_PRIM;
  const double* wl = S.g_brdf_wl + m.x;
  if(wlen <= __ldg(wl)) return m.x;
  if(wlen >= __ldg(wl + m.y - 1)) return m.x + m.y - 1;
  uint32_t lo = 0, hi = m.y - 1; /* wl[lo] < wlen < wl[hi] */
  while(hi - lo > 1) {
    const uint32_t mid = (lo + hi) >> 1;
    if(__ldg(wl + mid) <= wlen) lo = mid; else hi = mid;
  }
  const double u = (wlen - __ldg(wl + lo)) / (__ldg(wl + hi) - __ldg(wl + lo));
  return m.x + (r < u ? hi : lo);
}

}  // namespace

#endif /* HTRDR_GROUND_CUH */
