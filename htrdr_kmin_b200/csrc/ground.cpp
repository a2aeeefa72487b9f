/* Ground mesh set-up: validation of the caller's arrays (triangles,
 * interfaces, materials and their tabulated BRDFs), the BVH the device
 * traverses, and the device tables (htrdr_geometry_create and
 * htrdr_materials_create, src/core/htrdr_geometry.c:560-650 and
 * src/core/htrdr_materials.c:300-380, with the arrays in place of the
 * htrdr-obj and htrdr-materials files).
 *
 * BVH: median split of the triangle centroids along the longest axis of
 * their bounds, at most 4 triangles per leaf; the two children of a node are
 * stored side by side.  Node = 2 float4: {lower, first child or first
 * triangle}, {upper, triangle count (0: inner node)}.  Triangles are stored in
 * leaf order with the caller's primitive id beside them. */
#include "internal.h"

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstring>

namespace hg {

namespace {

struct BuildCtx {
  const std::vector<float3>* v0;
  const std::vector<float3>* v1;
  const std::vector<float3>* v2;
  std::vector<float3> cen;
  std::vector<uint32_t> order;
  std::vector<float4> nodes;
  uint32_t max_depth = 0;
};

void
bounds(const BuildCtx& c, uint32_t b, uint32_t e, float lo[3], float hi[3])
{
  for(int a = 0; a < 3; ++a) { lo[a] = FLT_MAX; hi[a] = -FLT_MAX; }
  for(uint32_t i = b; i < e; ++i) {
    const uint32_t t = c.order[i];
    const float3 p[3] = {(*c.v0)[t], (*c.v1)[t], (*c.v2)[t]};
    for(const float3& q : p) {
      lo[0] = std::min(lo[0], q.x); hi[0] = std::max(hi[0], q.x);
      lo[1] = std::min(lo[1], q.y); hi[1] = std::max(hi[1], q.y);
      lo[2] = std::min(lo[2], q.z); hi[2] = std::max(hi[2], q.z);
    }
  }
}

/* Fills node `ni' with the triangles order[b, e) */
void
build_node(BuildCtx& c, uint32_t ni, uint32_t b, uint32_t e, uint32_t depth)
{
  c.max_depth = std::max(c.max_depth, depth);
  float lo[3], hi[3];
  bounds(c, b, e, lo, hi);
  if(e - b <= 4) {
    c.nodes[2 * ni] = make_float4(lo[0], lo[1], lo[2], 0.f);
    c.nodes[2 * ni + 1] = make_float4(hi[0], hi[1], hi[2], 0.f);
    uint32_t first = b, count = e - b;
    std::memcpy(&c.nodes[2 * ni].w, &first, 4);
    std::memcpy(&c.nodes[2 * ni + 1].w, &count, 4);
    return;
  }
  float clo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, chi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
  for(uint32_t i = b; i < e; ++i) {
    const float3 q = c.cen[c.order[i]];
    clo[0] = std::min(clo[0], q.x); chi[0] = std::max(chi[0], q.x);
    clo[1] = std::min(clo[1], q.y); chi[1] = std::max(chi[1], q.y);
    clo[2] = std::min(clo[2], q.z); chi[2] = std::max(chi[2], q.z);
  }
  int ax = 0;
  for(int a = 1; a < 3; ++a) if(chi[a] - clo[a] > chi[ax] - clo[ax]) ax = a;
  auto key = [&](uint32_t t) { const float3 q = c.cen[t]; return ax == 0 ? q.x : (ax == 1 ? q.y : q.z); };
  std::sort(c.order.begin() + b, c.order.begin() + e, [&](uint32_t x, uint32_t y) {
    const float kx = key(x), ky = key(y);
    return kx < ky || (kx == ky && x < y);
  });
  const uint32_t mid = b + (e - b) / 2;
  const uint32_t child = (uint32_t)(c.nodes.size() / 2);
  c.nodes.resize(c.nodes.size() + 4);
  c.nodes[2 * ni] = make_float4(lo[0], lo[1], lo[2], 0.f);
  c.nodes[2 * ni + 1] = make_float4(hi[0], hi[1], hi[2], 0.f);
  uint32_t zero = 0;
  std::memcpy(&c.nodes[2 * ni].w, &child, 4);
  std::memcpy(&c.nodes[2 * ni + 1].w, &zero, 4);
  build_node(c, child, b, mid, depth + 1);
  build_node(c, child + 1, mid, e, depth + 1);
}

}  // namespace

htrdr_gpu_res_T
setup_ground_mesh(const htrdr_gpu_scene_desc* d, DScene& S,
                  const std::function<void*(const void*, size_t)>& upload)
{
  S.g_ntris = 0;
  S.g_repeat = 0;
  S.g_sky_mtl = 0xFFFFFFFFu;
  if(!d->ground_ntris) return HTRDR_GPU_RES_OK;
  const uint32_t nt = d->ground_ntris, nv = d->ground_nverts, nif = d->ground_nifaces,
                 nm = d->ground_nmtls;
  if(!d->ground_verts || !d->ground_tris || !d->ground_tri_iface || !nif || !d->ground_ifaces
  || !nm || !d->ground_mtl_temperature || !d->ground_mtl_nbrdf) {
    set_error("ground mesh: missing arrays");
    return HTRDR_GPU_RES_BAD_ARG;
  }
  const uint32_t NONE = 0xFFFFFFFFu;
  for(uint32_t i = 0; i < 3 * nt; ++i)
    if(d->ground_tris[i] >= nv) { set_error("ground mesh: vertex index out of range"); return HTRDR_GPU_RES_BAD_ARG; }
  for(uint32_t i = 0; i < nt; ++i)
    if(d->ground_tri_iface[i] >= nif) { set_error("ground mesh: interface index out of range"); return HTRDR_GPU_RES_BAD_ARG; }
  for(uint32_t i = 0; i < 3 * nif; ++i)
    if(d->ground_ifaces[i] != NONE && d->ground_ifaces[i] >= nm) {
      set_error("ground mesh: material index out of range");
      return HTRDR_GPU_RES_BAD_ARG;
    }
  if(d->ground_sky_mtl != NONE && d->ground_sky_mtl >= nm) {
    set_error("ground mesh: sky material out of range");
    return HTRDR_GPU_RES_BAD_ARG;
  }
  std::vector<uint2> mtl(nm);
  std::vector<float> mtl_T(nm);
  uint32_t nbrdf = 0;
  for(uint32_t m = 0; m < nm; ++m) {
    mtl[m] = make_uint2(nbrdf, d->ground_mtl_nbrdf[m]);
    mtl_T[m] = (float)d->ground_mtl_temperature[m];
    nbrdf += d->ground_mtl_nbrdf[m];
  }
  if(nbrdf && !d->ground_mtl_brdf) { set_error("ground mesh: missing BRDF table"); return HTRDR_GPU_RES_BAD_ARG; }
  std::vector<double> wl(std::max(nbrdf, 1u));
  std::vector<float2> br(std::max(nbrdf, 1u));
  for(uint32_t m = 0; m < nm; ++m) {
    for(uint32_t k = 0; k < mtl[m].y; ++k) {
      const double* e = d->ground_mtl_brdf + 3 * (size_t)(mtl[m].x + k);
      if((e[1] != 0.0 && e[1] != 1.0) || !(e[2] >= 0.0 && e[2] <= 1.0)
      || (k && !(e[0] > d->ground_mtl_brdf[3 * (size_t)(mtl[m].x + k - 1)]))) {
        set_error("ground mesh: invalid BRDF entry (type 0/1, reflectivity in [0,1], ascending wavelengths)");
        return HTRDR_GPU_RES_BAD_ARG;
      }
      wl[mtl[m].x + k] = e[0];
      br[mtl[m].x + k] = make_float2((float)e[1], (float)e[2]);
    }
  }
  std::vector<uint4> ifc(nif);
  for(uint32_t i = 0; i < nif; ++i)
    ifc[i] = make_uint4(d->ground_ifaces[3 * i], d->ground_ifaces[3 * i + 1], d->ground_ifaces[3 * i + 2], 0);

  /* BVH */
  std::vector<float3> v0(nt), v1(nt), v2(nt);
  double lo[3] = {DBL_MAX, DBL_MAX, DBL_MAX}, hi[3] = {-DBL_MAX, -DBL_MAX, -DBL_MAX};
  auto vert = [&](uint32_t i) {
    return make_float3(d->ground_verts[3 * i], d->ground_verts[3 * i + 1], d->ground_verts[3 * i + 2]);
  };
  BuildCtx c;
  c.cen.resize(nt);
  for(uint32_t t = 0; t < nt; ++t) {
    v0[t] = vert(d->ground_tris[3 * t]);
    v1[t] = vert(d->ground_tris[3 * t + 1]);
    v2[t] = vert(d->ground_tris[3 * t + 2]);
    for(const float3& q : {v0[t], v1[t], v2[t]}) {
      lo[0] = std::min(lo[0], (double)q.x); hi[0] = std::max(hi[0], (double)q.x);
      lo[1] = std::min(lo[1], (double)q.y); hi[1] = std::max(hi[1], (double)q.y);
      lo[2] = std::min(lo[2], (double)q.z); hi[2] = std::max(hi[2], (double)q.z);
    }
    c.cen[t] = make_float3((v0[t].x + v1[t].x + v2[t].x) / 3.f, (v0[t].y + v1[t].y + v2[t].y) / 3.f,
                           (v0[t].z + v1[t].z + v2[t].z) / 3.f);
  }
  c.v0 = &v0; c.v1 = &v1; c.v2 = &v2;
  c.order.resize(nt);
  for(uint32_t t = 0; t < nt; ++t) c.order[t] = t;
  c.nodes.resize(2);
  build_node(c, 0, 0, nt, 0);
  if(c.max_depth + 2 > HG_BVH_DEPTH_MAX) { set_error("ground mesh: BVH too deep"); return HTRDR_GPU_RES_BAD_ARG; }
  std::vector<float4> tri(3 * (size_t)nt);
  for(uint32_t i = 0; i < nt; ++i) {
    const uint32_t t = c.order[i];
    tri[3 * i] = make_float4(v0[t].x, v0[t].y, v0[t].z, 0.f);
    tri[3 * i + 1] = make_float4(v1[t].x, v1[t].y, v1[t].z, 0.f);
    tri[3 * i + 2] = make_float4(v2[t].x, v2[t].y, v2[t].z, 0.f);
  }
  if(d->repeat_ground && !(hi[0] > lo[0] && hi[1] > lo[1])) {
    set_error("ground mesh: a repeated ground needs a bounding box with an extent in X and Y");
    return HTRDR_GPU_RES_BAD_ARG;
  }
  if(!(S.g_tri = (const float4*)upload(tri.data(), tri.size() * sizeof(float4)))
  || !(S.g_tri_id = (const uint32_t*)upload(c.order.data(), nt * 4))
  || !(S.g_iface_of = (const uint32_t*)upload(d->ground_tri_iface, nt * 4))
  || !(S.g_iface = (const uint4*)upload(ifc.data(), nif * sizeof(uint4)))
  || !(S.g_bvh = (const float4*)upload(c.nodes.data(), c.nodes.size() * sizeof(float4)))
  || !(S.g_mtl = (const uint2*)upload(mtl.data(), nm * sizeof(uint2)))
  || !(S.g_mtl_T = (const float*)upload(mtl_T.data(), nm * 4))
  || !(S.g_brdf_wl = (const double*)upload(wl.data(), wl.size() * 8))
  || !(S.g_brdf = (const float2*)upload(br.data(), br.size() * sizeof(float2))))
    return HTRDR_GPU_RES_MEM_ERR;
  S.g_ntris = nt;
  S.g_nmtls = nm;
  S.g_repeat = d->repeat_ground ? 1 : 0;
  S.g_sky_mtl = d->ground_sky_mtl;
  for(int a = 0; a < 3; ++a) { S.g_lower[a] = lo[a]; S.g_upper[a] = hi[a]; }
  return HTRDR_GPU_RES_OK;
}

}  // namespace hg
