/* Scene upload, majorant octree construction and request set-up.
 *
 * htrdr_gpu_scene_create replaces htsky_create (called from
 * src/atmosphere/htrdr_atmosphere.c:366-382): it stores the gas column, the
 * cloud grid and the per-band optics in HBM and builds, for each (band,
 * quadrature point) and each needed property, the kmin/kmax majorant octree
 * as an array of packed 16-byte nodes.  Request set-up builds the wavelength
 * samplers of htrdr_ran_wlen_planck_create / htrdr_ran_wlen_cie_xyz_create
 * (src/atmosphere/htrdr_atmosphere.c:402-416) and the sensor frames. */
#include "internal.h"

#include <algorithm>
#include <atomic>
#include <cfloat>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <string>
#include <thread>

/* Leaf grids of the octrees (1: built when they fit; 0: never) */
#ifndef HG_LEAF_GRID
#define HG_LEAF_GRID 2
#endif

namespace hg {

static thread_local std::string g_last_error;
void set_error(const std::string& msg) { g_last_error = msg; }
const char* last_error() { return g_last_error.c_str(); }

static thread_local uint64_t g_launches = 0;
void note_launches(uint64_t n) { g_launches += n; }
uint64_t take_launches()
{
  const uint64_t n = g_launches;
  g_launches = 0;
  return n;
}

bool
cuda_ok(cudaError_t e, const char* what)
{
  if(e == cudaSuccess) return true;
  set_error(std::string(what) + ": " + cudaGetErrorString(e));
  return false;
}

DevBuf::~DevBuf() { if(ptr) cudaFree(ptr); }

bool
DevBuf::alloc(size_t n)
{
  bytes = n;
  if(!n) return true;
  return cuda_ok(cudaMalloc(&ptr, n), "cudaMalloc");
}

bool
DevBuf::upload(const void* src, size_t n)
{
  if(!alloc(n)) return false;
  if(!n) return true;
  return cuda_ok(cudaMemcpy(ptr, src, n, cudaMemcpyHostToDevice), "cudaMemcpy H2D");
}

/*******************************************************************************
 * Spectral routines (src/core/htrdr_spectral.h:56-99,
 * src/core/htrdr_ran_wlen_cie_xyz.c:57-108); same operations as the CPU
 * restatement so that the CDF tables are bit-identical.
 ******************************************************************************/
double
wiebelt(double v)
{
  const double pi = 3.14159265358979323846;
  const double c15_pi4 = 15.0 / (pi * pi * pi * pi);
  double w;
  if(v >= 2.0) {
    w = 0.0;
    for(int m = 1; m < 6; ++m) {
      const double mv = (double)m * v;
      w += std::exp(-mv) / (double)(m * m * m * m) * (((mv + 3.0) * mv + 6.0) * mv + 6.0);
    }
    w *= c15_pi4;
  } else {
    const double z0 = 1.0 / 3.0, z1 = 1.0 / 8.0, z2 = 1.0 / 60.0;
    const double z4 = 1.0 / 5040.0, z6 = 1.0 / 272160.0, z8 = 1.0 / 13305600.0;
    const double v2 = v * v, v4 = v2 * v2;
    const double poly = z0 - z1 * v + z2 * v2 - z4 * v2 * v2 + z6 * v4 * v2 - z8 * v4 * v4;
    w = 1.0 - c15_pi4 * v2 * v * poly;
  }
  return w;
}

double
blackbody_fraction(double l0, double l1, double T)
{
  const double C2 = 1.43877735e-2;
  return wiebelt(C2 / l1 / T) - wiebelt(C2 / l0 / T);
}

static double
gauss_piece(double l, double mu, double s_lo, double s_hi)
{
  const double t = (l - mu) * (l < mu ? s_lo : s_hi);
  return std::exp(-0.5 * t * t);
}

double
fit_bar_1931(int ch, double l)
{
  switch(ch) {
    case 0:
      return 0.362 * gauss_piece(l, 442.0, 0.0624, 0.0374)
           + 1.056 * gauss_piece(l, 599.8, 0.0264, 0.0323)
           - 0.065 * gauss_piece(l, 501.1, 0.0490, 0.0382);
    case 1:
      return 0.821 * gauss_piece(l, 568.8, 0.0213, 0.0247)
           + 0.286 * gauss_piece(l, 530.9, 0.0613, 0.0322);
    default:
      return 1.217 * gauss_piece(l, 437.0, 0.0845, 0.0278)
           + 0.681 * gauss_piece(l, 459.0, 0.0385, 0.0725);
  }
}

double
cie_trapezoid(double lo, double hi, int ch)
{
  const size_t n = (size_t)(hi - lo) + 1;
  const double dl = (hi - lo) / (double)n;
  double acc = 0;
  for(size_t i = 0; i < n; ++i) {
    const double f1 = fit_bar_1931(ch, lo + dl * (double)i);
    const double f2 = fit_bar_1931(ch, lo + dl * (double)(i + 1));
    acc += (f1 + f2) * dl * 0.5;
  }
  return acc;
}

/*******************************************************************************
 * Majorant octree (host build).  Definition:
 *  - level 0 = one cloud cell: k_cloud + [min, max] of k_gas over the layers
 *    that overlap the cell's z-extent (single-precision sums);
 *  - level L covers 2^L cells per axis, min/max over its valid children;
 *  - leaf iff all valid children are leaves and (L <= level_force, the -V
 *    cap) or (kmax - kmin) * 2^L * max cell size <= tau (the -T threshold);
 *  - breadth-first storage, 8 contiguous children in octant order (bit 0 x,
 *    bit 1 y, bit 2 z), children outside the grid stored as empty leaves.
 ******************************************************************************/
void
build_octree(const DScene& hs, const float* lwc, const float* sig3, const float* gas_ka,
             const float* gas_ks, const int* cl_lo, const int* cl_hi, uint32_t q, int prop,
             uint32_t D, uint32_t level_force, double tau, double cmax,
             std::vector<uint32_t>& out)
{
  struct Level { uint32_t n[3]; std::vector<float> kmin, kmax; std::vector<uint8_t> leaf; };
  std::vector<Level> lv(D + 1);
  const uint32_t nl = hs.nlayers;
  for(uint32_t L = 0; L <= D; ++L) {
    for(int a = 0; a < 3; ++a) lv[L].n[a] = (hs.def[a] + (1u << L) - 1) >> L;
    const size_t nn = (size_t)lv[L].n[0] * lv[L].n[1] * lv[L].n[2];
    lv[L].kmin.resize(nn);
    lv[L].kmax.resize(nn);
    lv[L].leaf.resize(nn);
  }
  auto gas = [&](int layer) -> float {
    const size_t i = (size_t)q * nl + (size_t)layer;
    if(prop == HG_KA) return gas_ka[i];
    if(prop == HG_KS) return gas_ks[i];
    const float a = gas_ka[i], s = gas_ks[i];
    return a + s;
  };
  const float sig = sig3[prop];
  for(uint32_t k = 0; k < hs.def[2]; ++k) {
    float gmin = 0.f, gmax = 0.f;
    if(cl_lo[k] >= 0) {
      gmin = gmax = gas(cl_lo[k]);
      for(int l = cl_lo[k] + 1; l <= cl_hi[k]; ++l) {
        const float g = gas(l);
        if(g < gmin) gmin = g;
        if(g > gmax) gmax = g;
      }
    }
    for(uint32_t j = 0; j < hs.def[1]; ++j) {
      for(uint32_t i = 0; i < hs.def[0]; ++i) {
        const size_t c = ((size_t)k * hs.def[1] + j) * hs.def[0] + i;
        const float kc = lwc[c] * sig;
        lv[0].kmin[c] = kc + gmin;
        lv[0].kmax[c] = kc + gmax;
        lv[0].leaf[c] = 1;
      }
    }
  }
  size_t n_internal = 0;
  for(uint32_t L = 1; L <= D; ++L) {
    const Level& c = lv[L - 1];
    Level& p = lv[L];
    const double size = (double)(1u << L) * cmax;
    for(uint32_t k = 0; k < p.n[2]; ++k)
    for(uint32_t j = 0; j < p.n[1]; ++j)
    for(uint32_t i = 0; i < p.n[0]; ++i) {
      const size_t pi = ((size_t)k * p.n[1] + j) * p.n[0] + i;
      float mn = FLT_MAX, mx = -FLT_MAX;
      int all_leaf = 1;
      for(int oct = 0; oct < 8; ++oct) {
        const uint32_t ci = 2 * i + (oct & 1), cj = 2 * j + ((oct >> 1) & 1), ck = 2 * k + (oct >> 2);
        if(ci >= c.n[0] || cj >= c.n[1] || ck >= c.n[2]) continue;
        const size_t cc = ((size_t)ck * c.n[1] + cj) * c.n[0] + ci;
        if(c.kmin[cc] < mn) mn = c.kmin[cc];
        if(c.kmax[cc] > mx) mx = c.kmax[cc];
        all_leaf &= c.leaf[cc];
      }
      p.kmin[pi] = mn;
      p.kmax[pi] = mx;
      p.leaf[pi] = (uint8_t)(all_leaf && (L <= level_force || ((double)mx - (double)mn) * size <= tau));
      if(!p.leaf[pi]) ++n_internal;
    }
  }
  const size_t total = 1 + 8 * n_internal;
  out.assign(total * 4, 0u);
  std::vector<uint32_t> coord(total * 4);
  auto put = [&](size_t idx, float kmin, float kmax, uint32_t child) {
    uint32_t a, b;
    std::memcpy(&a, &kmin, 4);
    std::memcpy(&b, &kmax, 4);
    out[idx * 4 + 0] = a; out[idx * 4 + 1] = b; out[idx * 4 + 2] = child; out[idx * 4 + 3] = 0;
  };
  put(0, lv[D].kmin[0], lv[D].kmax[0], HG_LEAF);
  coord[0] = D; coord[1] = coord[2] = coord[3] = 0;
  size_t count = 1;
  for(size_t idx = 0; idx < count; ++idx) {
    const uint32_t Ln = coord[idx * 4];
    if(Ln == 0xFFFFFFFFu) continue;
    const uint32_t i = coord[idx * 4 + 1], j = coord[idx * 4 + 2], k = coord[idx * 4 + 3];
    const Level& p = lv[Ln];
    if(p.leaf[((size_t)k * p.n[1] + j) * p.n[0] + i]) continue;
    out[idx * 4 + 2] = (uint32_t)count;
    const Level& c = lv[Ln - 1];
    for(int oct = 0; oct < 8; ++oct) {
      const uint32_t ci = 2 * i + (oct & 1), cj = 2 * j + ((oct >> 1) & 1), ck = 2 * k + (oct >> 2);
      if(ci >= c.n[0] || cj >= c.n[1] || ck >= c.n[2]) {
        put(count, 0.f, 0.f, HG_LEAF);
        coord[count * 4] = 0xFFFFFFFFu;
      } else {
        const size_t cc = ((size_t)ck * c.n[1] + cj) * c.n[0] + ci;
        put(count, c.kmin[cc], c.kmax[cc], HG_LEAF);
        coord[count * 4] = Ln - 1; coord[count * 4 + 1] = ci;
        coord[count * 4 + 2] = cj; coord[count * 4 + 3] = ck;
      }
      ++count;
    }
  }
}

uint32_t
pixel_size(int mode)
{
  return mode == HG_IMAGE_CIE ? 80u : 64u;
}

htrdr_gpu_res_T
check_layout(const htrdr_gpu_request* req, const htrdr_gpu_buffer_layout* layout)
{
  /* htrdr_buffer_layout_check + the pixel format of atmosphere_get_pixel_format
   * (src/atmosphere/htrdr_atmosphere.c:482-509) */
  if(!layout || !req) return HTRDR_GPU_RES_BAD_ARG;
  if(layout->width != req->width || layout->height != req->height) return HTRDR_GPU_RES_BAD_ARG;
  if(layout->elmt_size != pixel_size(req->mode)) return HTRDR_GPU_RES_BAD_ARG;
  if(layout->pitch < layout->width * layout->elmt_size) return HTRDR_GPU_RES_BAD_ARG;
  if(layout->alignment && (layout->alignment & (layout->alignment - 1))) return HTRDR_GPU_RES_BAD_ARG;
  if(layout->alignment > 16) return HTRDR_GPU_RES_BAD_ARG;
  return HTRDR_GPU_RES_OK;
}

static void
onb_d(const double n[3], double b1[3], double b2[3])
{
  const double sign = std::copysign(1.0, n[2]);
  const double a = -1.0 / (sign + n[2]);
  const double b = n[0] * n[1] * a;
  b1[0] = 1.0 + sign * n[0] * n[0] * a; b1[1] = sign * b; b1[2] = -sign * n[0];
  b2[0] = b; b2[1] = sign + n[1] * n[1] * a; b2[2] = -n[1];
}

static void
norm3(double v[3])
{
  const double n = std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
  v[0] /= n; v[1] /= n; v[2] /= n;
}

static void
cross3(double o[3], const double a[3], const double b[3])
{
  o[0] = a[1] * b[2] - a[2] * b[1];
  o[1] = a[2] * b[0] - a[0] * b[2];
  o[2] = a[0] * b[1] - a[1] * b[0];
}

/* The wavelength sampler of a request, built once per scene and spectral
 * domain (htrdr_ran_wlen_planck.c:55-134, htrdr_ran_wlen_cie_xyz.c:185-280) */
Sampler*
scene_sampler(htrdr_gpu_scene* scn, const htrdr_gpu_request* req, htrdr_gpu_res_T* res)
{
  const int cie = req->mode == HG_IMAGE_CIE;
  const auto key = std::make_tuple(cie, req->wlen_range[0], req->wlen_range[1],
                                   cie ? 0.0 : req->ref_temperature);
  std::lock_guard<std::mutex> lock(scn->mtx);
  auto it = scn->samplers.find(key);
  if(it != scn->samplers.end()) return it->second.get();
  auto s = std::make_unique<Sampler>();
  const double r0 = req->wlen_range[0], r1 = req->wlen_range[1];
  /* compute_spectral_bands_count (src/atmosphere/htrdr_atmosphere.c:53-70) */
  const size_t nb = (size_t)std::rint(r1 - r0);
  s->mode_cie = cie;
  *res = HTRDR_GPU_RES_OK;
  if(cie) {
    const size_t n = nb ? nb : 1;
    s->ncdf = (uint32_t)n;
    s->band_len = (r1 - r0) / (double)n;
    std::vector<double> cdf(3 * n), fb(3 * n * 2);
    for(int ch = 0; ch < 3; ++ch) {
      double sum = 0;
      for(size_t i = 0; i < n; ++i) {
        const double lo = r0 + (double)i * s->band_len;
        double hi = lo + s->band_len;
        if(hi > r1) hi = r1;
        cdf[ch * n + i] = cie_trapezoid(lo, hi, ch);
        sum += cdf[ch * n + i];
        fb[(ch * n + i) * 2 + 0] = fit_bar_1931(ch, lo);
        fb[(ch * n + i) * 2 + 1] = fit_bar_1931(ch, lo + s->band_len);
      }
      s->rcp_integral[ch] = 1.0 / sum;
      for(size_t i = 0; i < n; ++i) {
        cdf[ch * n + i] /= sum;
        if(i) cdf[ch * n + i] += cdf[ch * n + i - 1];
      }
      cdf[ch * n + n - 1] = 1.0;
    }
    if(!s->cdf.upload(cdf.data(), cdf.size() * 8) || !s->fbound.upload(fb.data(), fb.size() * 8)) {
      *res = HTRDR_GPU_RES_MEM_ERR;
      return nullptr;
    }
    s->host_cdf = cdf;
  } else {
    s->ncdf = (uint32_t)nb;
    if(nb) {
      s->band_len = (r1 - r0) / (double)nb;
      std::vector<double> pdf(nb), cdf(nb);
      double sum = 0;
      for(size_t i = 0; i < nb; ++i) {
        const double lo = r0 + (double)i * s->band_len;
        double hi = lo + s->band_len;
        if(hi > r1) hi = r1;
        pdf[i] = blackbody_fraction(lo * 1e-9, hi * 1e-9, req->ref_temperature);
        sum += pdf[i];
      }
      for(size_t i = 0; i < nb; ++i) {
        pdf[i] /= sum;
        cdf[i] = i == 0 ? pdf[i] : pdf[i] + cdf[i - 1];
      }
      cdf[nb - 1] = 1.0;
      if(!s->cdf.upload(cdf.data(), nb * 8) || !s->pdf.upload(pdf.data(), nb * 8)) {
        *res = HTRDR_GPU_RES_MEM_ERR;
        return nullptr;
      }
      s->host_cdf = cdf;
    }
  }
  if(s->ncdf) { /* guide table: first CDF entry >= b/G for b = 0..G */
    const uint32_t nch = cie ? 3u : 1u;
    const uint32_t G = cie ? 1024u : 16384u;
    std::vector<uint32_t> g((size_t)nch * (G + 1));
    for(uint32_t ch = 0; ch < nch; ++ch) {
      const double* c = s->host_cdf.data() + (size_t)ch * s->ncdf;
      for(uint32_t b = 0; b <= G; ++b) {
        const double key = (double)b / (double)G;
        g[(size_t)ch * (G + 1) + b] = (uint32_t)(std::lower_bound(c, c + s->ncdf, key) - c);
      }
    }
    if(!s->guide.upload(g.data(), g.size() * 4)) {
      *res = HTRDR_GPU_RES_MEM_ERR;
      return nullptr;
    }
    s->nguide = G;
  }
  Sampler* raw = s.get();
  scn->samplers.emplace(key, std::move(s));
  return raw;
}

htrdr_gpu_res_T
make_drequest(htrdr_gpu_scene* scn, const htrdr_gpu_request* req, DRequest* R)
{
  if(!req || req->mode < 0 || req->mode > 4 || !req->width || !req->height || !req->spp)
    return HTRDR_GPU_RES_BAD_ARG;
  if(req->wlen_range[0] > req->wlen_range[1]) return HTRDR_GPU_RES_BAD_ARG;
  const bool lw = req->mode == HG_XWAVE_LW || req->mode == HG_FLUX_LW;
  const uint32_t need = lw ? (1u << HG_KEXT) : 7u;
  if(scn->d.has_cloud && (scn->props_mask & need) != need) {
    set_error("the scene lacks the majorants this mode needs (props_mask)");
    return HTRDR_GPU_RES_BAD_ARG;
  }
  if(!lw && req->mode != HG_IMAGE_CIE && req->ref_temperature <= 0) return HTRDR_GPU_RES_BAD_ARG;
  if(lw && req->ref_temperature <= 0) return HTRDR_GPU_RES_BAD_ARG;
  htrdr_gpu_res_T res = HTRDR_GPU_RES_OK;
  Sampler* smp = scene_sampler(scn, req, &res);
  if(!smp) return res;
  std::memset(R, 0, sizeof(*R));
  R->mode = req->mode;
  R->width = req->width;
  R->height = req->height;
  R->spp = req->spp;
  R->nreal_pp = req->spp * (req->mode == HG_IMAGE_CIE ? 3u : 1u);
  R->seed = req->seed;
  R->acc = nullptr;
  R->tacc = nullptr;
  R->ndone = nullptr;
  R->pix_sz[0] = 1.0 / (double)req->width;
  R->pix_sz[1] = 1.0 / (double)req->height;
  R->wlen_range[0] = req->wlen_range[0];
  R->wlen_range[1] = req->wlen_range[1];
  R->ncdf = smp->ncdf;
  R->band_len = smp->band_len;
  R->cdf = (const double*)smp->cdf.ptr;
  R->pdf = (const double*)smp->pdf.ptr;
  R->fbound = (const double*)smp->fbound.ptr;
  R->guide = (const uint32_t*)smp->guide.ptr;
  R->nguide = smp->nguide;
  for(int i = 0; i < 3; ++i) R->rcp_integral[i] = smp->rcp_integral[i];
  R->ref_T = req->ref_temperature;
  /* perspective / orthographic camera (star-camera) */
  R->camera_type = req->camera_type;
  double f[3], r[3], u[3];
  for(int i = 0; i < 3; ++i) f[i] = req->cam_tgt[i] - req->cam_pos[i];
  norm3(f);
  cross3(r, f, req->cam_up);
  norm3(r);
  cross3(u, r, f);
  for(int i = 0; i < 3; ++i) {
    R->cam_pos[i] = req->cam_pos[i]; R->cam_f[i] = f[i]; R->cam_r[i] = r[i]; R->cam_u[i] = u[i];
  }
  R->tan_half = std::tan(req->fov_deg * 3.14159265358979323846 / 360.0);
  R->aspect = (double)req->width / (double)req->height;
  R->lens_radius = req->lens_radius;
  R->focal_dst = req->focal_dst;
  R->ortho_h = req->ortho_height;
  /* flux sensor (src/core/htrdr_rectangle.c:66-157) */
  double n[3], ax[3], ay[3];
  for(int i = 0; i < 3; ++i) n[i] = req->rect_tgt[i] - req->rect_pos[i];
  norm3(n);
  cross3(ax, n, req->rect_up);
  norm3(ax);
  cross3(ay, n, ax);
  norm3(ay);
  for(int i = 0; i < 3; ++i) {
    R->rect_pos[i] = req->rect_pos[i];
    R->rect_n[i] = n[i];
    R->rect_ax[i] = ax[i] * req->rect_size[0] * 0.5;
    R->rect_ay[i] = ay[i] * req->rect_size[1] * 0.5;
  }
  return HTRDR_GPU_RES_OK;
}

}  // namespace hg

using namespace hg;

extern "C" HTRDR_GPU_API const char*
htrdr_gpu_last_error(void) { return hg::last_error(); }

extern "C" HTRDR_GPU_API int
htrdr_gpu_device_count(void)
{
  int n = 0;
  if(cudaGetDeviceCount(&n) != cudaSuccess) return 0;
  return n;
}

extern "C" HTRDR_GPU_API const char*
htrdr_gpu_version(void) { return "htrdr_gpu 0.1 (sm_100a)"; }

namespace {

/* ---- majorant-octree cache (option -O) ----
 * File: a 64-byte header {magic "HGOCTREE", format 1, medium signature,
 * octree depth, quadrature points, property mask, node count}, then the
 * first node and node count of each (quad point, property) tree as u64
 * [nq][3] each, then the nodes (16 bytes each, device layout). */
constexpr char kCacheMagic[8] = {'H', 'G', 'O', 'C', 'T', 'R', 'E', 'E'};
constexpr uint64_t kCacheFormat = 1;

struct CacheHeader {
  char magic[8];
  uint64_t format;
  uint64_t signature;
  uint32_t depth, nq, props_mask, pad;
  uint64_t nodes;
  uint64_t reserved[2];
};
static_assert(sizeof(CacheHeader) == 64, "cache header layout");

/* 64-bit signature of a byte range, 8 bytes per step (FNV-1a on words
 * with a final avalanche); enough to tell two media apart */
struct Signature {
  uint64_t h = 0xcbf29ce484222325ull;
  void add(const void* data, size_t bytes)
  {
    const unsigned char* c = (const unsigned char*)data;
    size_t i = 0;
    for(; i + 8 <= bytes; i += 8) {
      uint64_t w;
      std::memcpy(&w, c + i, 8);
      h = (h ^ w) * 0x100000001b3ull;
    }
    uint64_t w = 0;
    std::memcpy(&w, c + i, bytes - i);
    h = (h ^ w ^ (uint64_t)bytes) * 0x100000001b3ull;
  }
  template <typename T> void add_val(T v) { add(&v, sizeof(v)); }
  uint64_t done() const
  {
    uint64_t x = h;
    x ^= x >> 33; x *= 0xff51afd7ed558ccdull;
    x ^= x >> 33; x *= 0xc4ceb9fe1a85ec53ull;
    return x ^ (x >> 33);
  }
};

/* The inputs the octrees depend on, but -T and -V (which the cache
 * overrides) and the options of the traversal (-r) */
uint64_t
medium_signature(const htrdr_gpu_scene_desc* d, uint32_t nq)
{
  Signature g;
  const uint32_t nl = d->nlayers, nb = d->nbands;
  g.add_val(nl);
  g.add(d->layer_z, (nl + 1) * sizeof(double));
  g.add(d->layer_T, nl * sizeof(float));
  g.add_val(nb);
  g.add(d->band_lo, nb * sizeof(double));
  g.add(d->band_hi, nb * sizeof(double));
  g.add(d->nquads, nb * sizeof(uint32_t));
  g.add(d->quad_w, nq * sizeof(double));
  g.add(d->gas_ka, (size_t)nq * nl * sizeof(float));
  g.add(d->gas_ks, (size_t)nq * nl * sizeof(float));
  g.add(d->cloud_def, sizeof(d->cloud_def));
  g.add(d->cloud_lower, sizeof(d->cloud_lower));
  g.add(d->cloud_cell, sizeof(d->cloud_cell));
  g.add(d->cloud_lwc, (size_t)d->cloud_def[0] * d->cloud_def[1] * d->cloud_def[2] * sizeof(float));
  if(d->cloud_sigma_ext) g.add(d->cloud_sigma_ext, nb * sizeof(float));
  if(d->cloud_ssa) g.add(d->cloud_ssa, nb * sizeof(float));
  if(d->cloud_g) g.add(d->cloud_g, nb * sizeof(float));
  g.add_val(d->props_mask & 7u);
  return g.done();
}

/* Reads the cache into host tables; false with the error set when the file
 * is unreadable or was written from another medium */
bool
cache_read(const char* path, uint64_t signature, uint32_t depth, uint32_t nq, uint32_t props_mask,
           std::vector<uint64_t>& base, std::vector<uint64_t>& count, std::vector<uint32_t>& nodes)
{
  std::unique_ptr<FILE, int (*)(FILE*)> f(std::fopen(path, "rb"), &std::fclose);
  CacheHeader h;
  if(!f || std::fread(&h, sizeof(h), 1, f.get()) != 1 || std::memcmp(h.magic, kCacheMagic, 8)
  || h.format != kCacheFormat) {
    set_error(std::string("octree cache `") + path + "': not an octree cache of this library");
    return false;
  }
  if(h.signature != signature || h.depth != depth || h.nq != nq || h.props_mask != (props_mask & 7u)) {
    set_error(std::string("octree cache `") + path + "' was built from other inputs");
    return false;
  }
  /* the file holds exactly what the header announces (checked before any
   * allocation sized from the header) */
  const long here = std::ftell(f.get());
  if(here < 0 || std::fseek(f.get(), 0, SEEK_END) != 0) {
    set_error(std::string("octree cache `") + path + "': not seekable");
    return false;
  }
  const long end = std::ftell(f.get());
  const uint64_t tables = (uint64_t)nq * 3 * 16;
  if(end < here || h.nodes > ((uint64_t)1 << 40) || (uint64_t)(end - here) != tables + h.nodes * 16
  || std::fseek(f.get(), here, SEEK_SET) != 0) {
    set_error(std::string("octree cache `") + path + "': size does not match its header");
    return false;
  }
  base.resize((size_t)nq * 3);
  count.resize((size_t)nq * 3);
  nodes.resize((size_t)h.nodes * 4);
  if(std::fread(base.data(), 8, base.size(), f.get()) != base.size()
  || std::fread(count.data(), 8, count.size(), f.get()) != count.size()
  || std::fread(nodes.data(), 16, h.nodes, f.get()) != h.nodes) {
    set_error(std::string("octree cache `") + path + "': truncated");
    return false;
  }
  for(size_t i = 0; i < base.size(); ++i)
    if(count[i] && (base[i] > h.nodes || count[i] > h.nodes - base[i])) {
      set_error(std::string("octree cache `") + path + "': tree out of range");
      return false;
    }
  return true;
}

/* Writes the cache (to a temporary file renamed into place) */
bool
cache_write(const char* path, uint64_t signature, uint32_t depth, uint32_t nq, uint32_t props_mask,
            const std::vector<uint64_t>& base, const std::vector<uint64_t>& count,
            const uint32_t* nodes, uint64_t nnodes)
{
  const std::string tmp = std::string(path) + ".tmp";
  CacheHeader h{};
  std::memcpy(h.magic, kCacheMagic, 8);
  h.format = kCacheFormat;
  h.signature = signature;
  h.depth = depth;
  h.nq = nq;
  h.props_mask = props_mask & 7u;
  h.nodes = nnodes;
  bool ok;
  {
    std::unique_ptr<FILE, int (*)(FILE*)> f(std::fopen(tmp.c_str(), "wb"), &std::fclose);
    ok = f && std::fwrite(&h, sizeof(h), 1, f.get()) == 1
      && std::fwrite(base.data(), 8, base.size(), f.get()) == base.size()
      && std::fwrite(count.data(), 8, count.size(), f.get()) == count.size()
      && std::fwrite(nodes, 16, nnodes, f.get()) == nnodes;
    if(f && std::fflush(f.get()) != 0) ok = false;
  }
  if(ok && std::rename(tmp.c_str(), path) != 0) ok = false;
  if(!ok) {
    std::remove(tmp.c_str());
    set_error(std::string("octree cache `") + path + "': cannot write");
  }
  return ok;
}

htrdr_gpu_res_T scene_create(int device, const htrdr_gpu_scene_desc* desc, const char* cache_path,
                             htrdr_gpu_scene** out);

}  // namespace

extern "C" HTRDR_GPU_API htrdr_gpu_res_T
htrdr_gpu_scene_create(int device, const htrdr_gpu_scene_desc* desc, htrdr_gpu_scene** out)
try {
  return scene_create(device, desc, nullptr, out);
}
HG_API_CATCH("htrdr_gpu_scene_create")

extern "C" HTRDR_GPU_API htrdr_gpu_res_T
htrdr_gpu_scene_create_cached(int device, const htrdr_gpu_scene_desc* desc, const char* cache_path,
                              htrdr_gpu_scene** out)
try {
  if(!cache_path || !*cache_path) {
    set_error("no cache path");
    return HTRDR_GPU_RES_BAD_ARG;
  }
  return scene_create(device, desc, cache_path, out);
}
HG_API_CATCH("htrdr_gpu_scene_create_cached")

namespace {

htrdr_gpu_res_T
scene_create(int device, const htrdr_gpu_scene_desc* desc, const char* cache_path, htrdr_gpu_scene** out)
{
  if(!desc || !out || !desc->nlayers || !desc->nbands || !desc->layer_z || !desc->layer_T
  || !desc->band_lo || !desc->band_hi || !desc->nquads || !desc->quad_w || !desc->gas_ka
  || !desc->gas_ks) {
    set_error("invalid scene description");
    return HTRDR_GPU_RES_BAD_ARG;
  }
  int ndev = 0;
  if(cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) {
    set_error("no CUDA device available");
    return HTRDR_GPU_RES_BAD_OP;
  }
  if(!cuda_ok(cudaSetDevice(device), "cudaSetDevice")) return HTRDR_GPU_RES_BAD_OP;

  auto scn = std::make_unique<htrdr_gpu_scene>();
  scn->device = device;
  DScene& S = scn->d;
  const uint32_t nl = desc->nlayers, nb = desc->nbands;
  uint32_t nq = 0;
  for(uint32_t b = 0; b < nb; ++b) {
    if(!desc->nquads[b]) return HTRDR_GPU_RES_BAD_ARG;
    nq += desc->nquads[b];
  }
  for(uint32_t l = 0; l < nl; ++l)
    if(!(desc->layer_z[l] < desc->layer_z[l + 1])) return HTRDR_GPU_RES_BAD_ARG;
  scn->nbands = nb; scn->nq = nq; scn->nlayers = nl; scn->props_mask = desc->props_mask;
  scn->band_lo.assign(desc->band_lo, desc->band_lo + nb);
  scn->band_hi.assign(desc->band_hi, desc->band_hi + nb);
  scn->nquads.assign(desc->nquads, desc->nquads + nb);
  scn->quad_off.assign(nb + 1, 0);
  for(uint32_t b = 0; b < nb; ++b) scn->quad_off[b + 1] = scn->quad_off[b] + desc->nquads[b];

  /* host copies in device layout */
  std::vector<float> lz(nl + 1), lT(nl);
  for(uint32_t l = 0; l <= nl; ++l) lz[l] = (float)desc->layer_z[l];
  for(uint32_t l = 0; l < nl; ++l) lT[l] = desc->layer_T[l];
  std::vector<float2> gas((size_t)nq * nl);
  for(size_t i = 0; i < (size_t)nq * nl; ++i) gas[i] = make_float2(desc->gas_ka[i], desc->gas_ks[i]);
  std::vector<double> cum(nq);
  for(uint32_t b = 0; b < nb; ++b) {
    double acc = 0;
    for(uint32_t iq = 0; iq < desc->nquads[b]; ++iq) {
      acc += desc->quad_w[scn->quad_off[b] + iq];
      cum[scn->quad_off[b] + iq] = acc;
    }
    cum[scn->quad_off[b + 1] - 1] = 1.0;
  }
  std::vector<float4> optics(nb);
  std::vector<float> sig3(nb * 3);
  for(uint32_t b = 0; b < nb; ++b) {
    const double se = desc->cloud_sigma_ext ? (double)desc->cloud_sigma_ext[b] : 0.0;
    const double ssa = desc->cloud_ssa ? (double)desc->cloud_ssa[b] : 0.0;
    const float g = desc->cloud_g ? desc->cloud_g[b] : 0.f;
    sig3[b * 3 + HG_KA] = (float)(se * (1.0 - ssa));
    sig3[b * 3 + HG_KS] = (float)(se * ssa);
    sig3[b * 3 + HG_KEXT] = (float)se;
    optics[b] = make_float4(sig3[b * 3 + 0], sig3[b * 3 + 1], sig3[b * 3 + 2], g);
  }

  auto upload = [&](const void* src, size_t bytes) -> void* {
    auto b = std::make_unique<DevBuf>();
    if(!b->upload(src, bytes)) return nullptr;
    void* p = b->ptr;
    scn->bytes += bytes;
    scn->bufs.push_back(std::move(b));
    return p;
  };

  /* cumulative vertical optical depth of the gas column per (quad, property):
   * cum[l] = sum_{i<l} k_i (z_{i+1} - z_i), with k the single-precision
   * coefficient the voxel-by-voxel traversal would use */
  std::vector<double> cum_tau((size_t)nq * 3 * (nl + 1));
  for(uint32_t q = 0; q < nq; ++q) {
    for(int p = 0; p < 3; ++p) {
      double* c = &cum_tau[((size_t)q * 3 + p) * (nl + 1)];
      c[0] = 0.0;
      for(uint32_t l = 0; l < nl; ++l) {
        const float a = desc->gas_ka[(size_t)q * nl + l], s = desc->gas_ks[(size_t)q * nl + l];
        const float k = p == HG_KA ? a : (p == HG_KS ? s : a + s);
        c[l + 1] = c[l] + (double)k * (desc->layer_z[l + 1] - desc->layer_z[l]);
      }
    }
  }
  S.nlayers = nl;
  S.ztop = lz[nl];
  S.nbands = nb;
  if(!(S.layer_zd = (const double*)upload(desc->layer_z, (nl + 1) * 8))
  || !(S.gas_cum = (const double*)upload(cum_tau.data(), cum_tau.size() * 8))
  || !(S.layer_z = (const float*)upload(lz.data(), lz.size() * 4))
  || !(S.layer_T = (const float*)upload(lT.data(), lT.size() * 4))
  || !(S.gas = (const float2*)upload(gas.data(), gas.size() * 8))
  || !(S.band_lo = (const double*)upload(desc->band_lo, nb * 8))
  || !(S.band_hi = (const double*)upload(desc->band_hi, nb * 8))
  || !(S.quad_off = (const uint32_t*)upload(scn->quad_off.data(), (nb + 1) * 4))
  || !(S.quad_cum = (const double*)upload(cum.data(), nq * 8))
  || !(S.optics = (const float4*)upload(optics.data(), nb * 16)))
    return HTRDR_GPU_RES_MEM_ERR;

  S.has_cloud = desc->cloud_def[0] && desc->cloud_def[1] && desc->cloud_def[2] && desc->cloud_lwc;
  S.repeat = desc->repeat_clouds ? 1 : 0;
  for(int a = 0; a < 3; ++a) {
    S.def[a] = S.has_cloud ? desc->cloud_def[a] : 0;
    S.lower[a] = (float)desc->cloud_lower[a];
    S.cell[a] = (float)desc->cloud_cell[a];
    S.inv_cell[a] = 1.f / S.cell[a];
    S.upper[a] = (float)(desc->cloud_lower[a] + (double)S.def[a] * desc->cloud_cell[a]);
  }
  scn->tree_base.assign((size_t)nq * 3, 0);
  scn->tree_count.assign((size_t)nq * 3, 0);
  if(S.has_cloud) {
    const uint32_t mx = std::max(S.def[0], std::max(S.def[1], S.def[2]));
    uint32_t D = 0;
    while((1u << D) < mx) ++D;
    S.depth = D;
    scn->depth = D;
    uint32_t Lf = 0;
    for(int a = 0; a < 3; ++a) {
      const uint32_t V = desc->grid_max_definition[a];
      if(V && V < S.def[a]) {
        const uint32_t need = (S.def[a] + V - 1) / V;
        uint32_t l = 0;
        while((1u << l) < need) ++l;
        Lf = std::max(Lf, l);
      }
    }
    const size_t ncell = (size_t)S.def[0] * S.def[1] * S.def[2];
    std::vector<int> cl_lo(S.def[2]), cl_hi(S.def[2]);
    std::vector<int2> cl(S.def[2]);
    for(uint32_t k = 0; k < S.def[2]; ++k) {
      const double zlo = desc->cloud_lower[2] + (double)k * desc->cloud_cell[2];
      const double zhi = zlo + desc->cloud_cell[2];
      int lo = -1, hi = -1;
      for(int l = 0; l < (int)nl; ++l) {
        if(desc->layer_z[l] < zhi && desc->layer_z[l + 1] > zlo) {
          if(lo < 0) lo = l;
          hi = l;
        }
      }
      cl_lo[k] = lo; cl_hi[k] = hi;
      cl[k] = make_int2(lo, hi);
    }
    if(!(S.lwc = (const float*)upload(desc->cloud_lwc, ncell * 4))
    || !(S.cell_layers = (const int2*)upload(cl.data(), cl.size() * sizeof(int2))))
      return HTRDR_GPU_RES_MEM_ERR;

    /* per (quad point, property) octrees, built in parallel */
    const double cmax = std::max(desc->cloud_cell[0], std::max(desc->cloud_cell[1], desc->cloud_cell[2]));
    std::vector<std::pair<uint32_t, int>> tasks;
    std::vector<uint32_t> band_of(nq);
    for(uint32_t b = 0; b < nb; ++b)
      for(uint32_t iq = scn->quad_off[b]; iq < scn->quad_off[b + 1]; ++iq) band_of[iq] = b;
    for(uint32_t q = 0; q < nq; ++q)
      for(int p = 0; p < 3; ++p)
        if(desc->props_mask & (1u << p)) tasks.emplace_back(q, p);
    const uint64_t signature = cache_path ? medium_signature(desc, nq) : 0;
    bool cached = false;
    if(cache_path) { /* an existing cache replaces the build (-O) */
      std::unique_ptr<FILE, int (*)(FILE*)> probe(std::fopen(cache_path, "rb"), &std::fclose);
      if(probe) {
        probe.reset();
        std::vector<uint32_t> nodes;
        if(!cache_read(cache_path, signature, D, nq, desc->props_mask, scn->tree_base, scn->tree_count, nodes))
          return HTRDR_GPU_RES_BAD_ARG;
        if(!(S.nodes = (const uint4*)upload(nodes.data(), std::max<size_t>(nodes.size(), 4) * 4)))
          return HTRDR_GPU_RES_MEM_ERR;
        cached = true;
      }
    }
    if(cached) {
      /* loaded */
    } else if(desc->octree_on_host) { /* host build, in parallel over the trees */
      std::vector<std::vector<uint32_t>> trees(tasks.size());
      std::atomic<size_t> next(0);
      const unsigned nth = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
      std::vector<std::thread> pool;
      for(unsigned t = 0; t < nth; ++t) {
        pool.emplace_back([&]() {
          for(;;) {
            const size_t i = next++;
            if(i >= tasks.size()) break;
            const uint32_t q = tasks[i].first;
            const int p = tasks[i].second;
            build_octree(S, desc->cloud_lwc, &sig3[band_of[q] * 3], desc->gas_ka, desc->gas_ks,
                         cl_lo.data(), cl_hi.data(), q, p, D, Lf, desc->optical_thickness, cmax,
                         trees[i]);
          }
        });
      }
      for(auto& th : pool) th.join();
      size_t total = 0;
      for(size_t i = 0; i < tasks.size(); ++i) {
        const size_t idx = (size_t)tasks[i].first * 3 + tasks[i].second;
        scn->tree_base[idx] = total / 4;
        scn->tree_count[idx] = trees[i].size() / 4;
        total += trees[i].size();
      }
      std::vector<uint32_t> pool_nodes(total);
      for(size_t i = 0; i < tasks.size(); ++i) {
        const size_t idx = (size_t)tasks[i].first * 3 + tasks[i].second;
        std::memcpy(&pool_nodes[scn->tree_base[idx] * 4], trees[i].data(), trees[i].size() * 4);
      }
      if(!(S.nodes = (const uint4*)upload(pool_nodes.data(), total * 4))) return HTRDR_GPU_RES_MEM_ERR;
      if(cache_path
      && !cache_write(cache_path, signature, D, nq, desc->props_mask, scn->tree_base, scn->tree_count,
                      pool_nodes.data(), total / 4))
        return HTRDR_GPU_RES_IO_ERR;
    } else { /* GPU build (octree_gpu.cu), same node arrays */
      DevBuf d_ka, d_ks;
      auto pool = std::make_unique<DevBuf>();
      std::vector<uint64_t> base, count;
      if(!d_ka.upload(desc->gas_ka, (size_t)nq * nl * 4) || !d_ks.upload(desc->gas_ks, (size_t)nq * nl * 4))
        return HTRDR_GPU_RES_MEM_ERR;
      if(!build_octrees_gpu(S, S.lwc, S.cell_layers, (const float*)d_ka.ptr, (const float*)d_ks.ptr, sig3,
                            band_of, tasks, Lf, desc->optical_thickness, cmax, *pool, base, count, nullptr))
        return HTRDR_GPU_RES_MEM_ERR;
      for(size_t i = 0; i < tasks.size(); ++i) {
        const size_t idx = (size_t)tasks[i].first * 3 + tasks[i].second;
        scn->tree_base[idx] = base[i];
        scn->tree_count[idx] = count[i];
      }
      S.nodes = (const uint4*)pool->ptr;
      scn->bytes += pool->bytes;
      if(cache_path) {
        uint64_t total = 0;
        for(size_t i = 0; i < base.size(); ++i) total = std::max(total, base[i] + count[i]);
        std::vector<uint32_t> host((size_t)total * 4);
        if(total && !cuda_ok(cudaMemcpy(host.data(), pool->ptr, total * 16, cudaMemcpyDeviceToHost), "D2H"))
          return HTRDR_GPU_RES_UNKNOWN_ERR;
        if(!cache_write(cache_path, signature, D, nq, desc->props_mask, scn->tree_base, scn->tree_count,
                        host.data(), total))
          return HTRDR_GPU_RES_IO_ERR;
      }
      scn->bufs.push_back(std::move(pool));
    }
    if(!(S.tree_base = (const uint64_t*)upload(scn->tree_base.data(), scn->tree_base.size() * 8)))
      return HTRDR_GPU_RES_MEM_ERR;
    S.ncell = (uint64_t)S.def[0] * S.def[1] * S.def[2];
    auto grids = std::make_unique<DevBuf>();
    std::vector<uint32_t> rank;
    /* the majorant grid (9 B per cell and tree) where it fits, else the node
     * grid (4 B), else none */
    bool maj = HG_LEAF_GRID == 2, built = false;
    if(HG_LEAF_GRID) {
      built = build_leaf_grids(S, scn->tree_base, scn->tree_count, *grids, rank, maj);
      if(!built && maj) {
        cudaGetLastError();
        grids = std::make_unique<DevBuf>();
        maj = false;
        built = build_leaf_grids(S, scn->tree_base, scn->tree_count, *grids, rank, false);
      }
    }
    if(built) {
      if(!(S.grid_rank = (const uint32_t*)upload(rank.data(), rank.size() * 4)))
        return HTRDR_GPU_RES_MEM_ERR;
      if(maj) {
        S.maj_grid = (const float2*)grids->ptr;
        S.lvl_grid = (const uint8_t*)grids->ptr + grids->bytes / 9 * 8;
      } else {
        S.leaf_grid = (const uint32_t*)grids->ptr;
      }
      scn->bytes += grids->bytes;
      scn->bufs.push_back(std::move(grids));
    } else {
      cudaGetLastError(); /* an allocation refused for the optional grids is not an error */
    }
  }

  S.has_ground = desc->has_ground ? 1 : 0;
  S.ground_brdf = desc->ground_brdf;
  S.ground_refl = (float)desc->ground_reflectivity;
  S.ground_T = (float)desc->ground_temperature;
  {
    const htrdr_gpu_res_T res = setup_ground_mesh(desc, S, upload);
    if(res != HTRDR_GPU_RES_OK) return res;
  }
  { /* sun (src/atmosphere/htrdr_atmosphere_sun.c:66-101) */
    const double pi = 3.14159265358979323846;
    const double az = desc->sun_azimuth * pi / 180.0, el = desc->sun_elevation * pi / 180.0;
    double d[3] = {std::cos(el) * std::cos(az), std::cos(el) * std::sin(az), std::sin(el)};
    double b1[3], b2[3];
    onb_d(d, b1, b2);
    for(int i = 0; i < 3; ++i) {
      S.sun_dir_d[i] = d[i];
      S.sun_dir[i] = (float)d[i];
      S.sun_b1[i] = (float)b1[i];
      S.sun_b2[i] = (float)b2[i];
    }
    S.sun_cos_half = std::cos(4.6524e-3);
    S.sun_solid_angle = 2.0 * pi * (1.0 - S.sun_cos_half);
    S.sun_T = 5778.0;
  }
  if(!cuda_ok(cudaStreamCreateWithFlags(&scn->stream, cudaStreamNonBlocking), "cudaStreamCreate"))
    return HTRDR_GPU_RES_BAD_OP;
  *out = scn.release();
  return HTRDR_GPU_RES_OK;
}

}  // namespace

extern "C" HTRDR_GPU_API void
htrdr_gpu_scene_release(htrdr_gpu_scene* scn)
{
  if(!scn) return;
  cudaSetDevice(scn->device);
  if(scn->stream) {
    cudaStreamSynchronize(scn->stream);
    cudaStreamDestroy(scn->stream);
  }
  delete scn;
}

extern "C" HTRDR_GPU_API size_t
htrdr_gpu_scene_device_bytes(const htrdr_gpu_scene* scn) { return scn ? scn->bytes : 0; }

extern "C" HTRDR_GPU_API uint32_t
htrdr_gpu_scene_tree_depth(const htrdr_gpu_scene* scn) { return scn ? scn->depth : 0; }

extern "C" HTRDR_GPU_API htrdr_gpu_res_T
htrdr_gpu_scene_get_tree(const htrdr_gpu_scene* scn, uint32_t iband, uint32_t iquad, int prop,
                         void* nodes, size_t capacity, size_t* count)
try {
  if(!scn || !count || iband >= scn->nbands || iquad >= scn->nquads[iband] || prop < 0 || prop > 2)
    return HTRDR_GPU_RES_BAD_ARG;
  const size_t idx = ((size_t)scn->quad_off[iband] + iquad) * 3 + (size_t)prop;
  *count = scn->d.has_cloud ? scn->tree_count[idx] : 0;
  if(!nodes || !*count) return HTRDR_GPU_RES_OK;
  if(capacity < *count) return HTRDR_GPU_RES_BAD_ARG;
  cudaSetDevice(scn->device);
  if(!cuda_ok(cudaMemcpy(nodes, scn->d.nodes + scn->tree_base[idx], *count * 16,
                         cudaMemcpyDeviceToHost), "cudaMemcpy D2H"))
    return HTRDR_GPU_RES_UNKNOWN_ERR;
  return HTRDR_GPU_RES_OK;
}
HG_API_CATCH("htrdr_gpu_scene_get_tree")
