/* Device transport: random streams, medium access, majorant traversal and
 * the per-realisation state machine of the atmosphere path tracer.
 *
 * A realisation is a small state machine (struct Path) advanced by
 * path_event() (sensor sampling, scattering/surface events, sun next-event
 * estimation, accumulation) and trace_step() (one voxel of a delta-tracking
 * trace).  The same code runs in the one-thread-per-realisation kernel and in
 * the persistent batched kernel, so both produce the same weight for a given
 * (pixel, realisation).
 *
 * Reference behaviour restated here:
 *   src/atmosphere/htrdr_atmosphere_compute_radiance_sw.c:73-511
 *   src/atmosphere/htrdr_atmosphere_compute_radiance_lw.c:64-279
 *   src/atmosphere/htrdr_atmosphere_draw_map.c:51-436
 *   src/atmosphere/htrdr_atmosphere_sun.c:126-166
 *   src/core/htrdr_spectral.h:101-116, src/core/htrdr_ran_wlen_planck.c:218-268,
 *   src/core/htrdr_ran_wlen_cie_xyz.c:110-183
 * Transport runs in FP32; optical depths (Ts, Tmin), weights, spectral
 * sampling and sensor sampling in FP64. */
#ifndef HTRDR_TRANSPORT_CUH
#define HTRDR_TRANSPORT_CUH

#include <cuda_runtime.h>
#include <float.h>
#include <stddef.h>
#include <stdint.h>

#include "dscene.h"
#include "ground.cuh"

#define HG_PI_D 3.14159265358979323846
#define HG_PI_F 3.14159265358979323846f

/* Internal linkage: every translation unit that includes this header gets
 * its own copy of the device code. */
namespace {

/*******************************************************************************
 * Philox4x32-10 counter-based stream (Salmon et al., SC'11).
 * Word j of the stream (k0, k1, c0, c1) is word (j & 3) of
 * Philox4x32-10({c0, c1, j >> 2, 0}, {k0, k1}).
 ******************************************************************************/
/* Out of line: one copy of the ten rounds instead of one per draw site keeps
 * the transport kernels inside the instruction cache. */
__device__ __noinline__ uint4
philox4x32_10(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3, uint32_t k0, uint32_t k1)
{
#pragma unroll
  for(int r = 0; r < 10; ++r) {
    const uint32_t hi0 = __umulhi(0xD2511F53u, c0), lo0 = 0xD2511F53u * c0;
    const uint32_t hi1 = __umulhi(0xCD9E8D57u, c2), lo1 = 0xCD9E8D57u * c2;
    c0 = hi1 ^ c1 ^ k0;
    c1 = lo1;
    c2 = hi0 ^ c3 ^ k1;
    c3 = lo0;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
  return make_uint4(c0, c1, c2, c3);
}

struct Rng {
  uint32_t k0, k1, c0, c1, n;
  uint32_t b0, b1, b2, b3;

  __device__ __forceinline__ void init(uint32_t key0, uint32_t key1, uint32_t ctr0, uint32_t ctr1)
  {
    k0 = key0; k1 = key1; c0 = ctr0; c1 = ctr1; n = 0;
  }
  __device__ __forceinline__ uint32_t u32()
  {
    const uint32_t i = n & 3u;
    if(i == 0) {
      const uint4 b = philox4x32_10(c0, c1, n >> 2, 0u, k0, k1);
      b0 = b.x; b1 = b.y; b2 = b.z; b3 = b.w;
    }
    ++n;
    return i == 0 ? b0 : (i == 1 ? b1 : (i == 2 ? b2 : b3));
  }
  /* transport canonical in [0, 1) */
  __device__ __forceinline__ float uf() { return (float)(u32() >> 8) * 0x1p-24f; }
  /* 53-bit canonical in [0, 1) */
  __device__ __forceinline__ double ud()
  {
    const uint32_t a = u32() >> 5;
    const uint32_t b = u32() >> 6;
    return ((double)a * 67108864.0 + (double)b) * 0x1p-53;
  }
  /* exponential optical depth, never 0 nor infinite */
  __device__ __forceinline__ double exp1()
  {
    const uint32_t m = u32() >> 9;
    return (double)(-logf((float)(2u * m + 1u) * 0x1p-24f));
  }
};

/*******************************************************************************
 * Small vector helpers
 ******************************************************************************/
__device__ __forceinline__ float3 mk3(float x, float y, float z) { return make_float3(x, y, z); }
__device__ __forceinline__ float3 add3(float3 a, float3 b) { return mk3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ float3 mul3(float3 a, float s) { return mk3(a.x * s, a.y * s, a.z * s); }
__device__ __forceinline__ float3 neg3(float3 a) { return mk3(-a.x, -a.y, -a.z); }
__device__ __forceinline__ float dot3(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ float3 nrm3(float3 a) { return mul3(a, rsqrtf(dot3(a, a))); }
__device__ __forceinline__ float3 madd3(float3 o, float3 d, float t)
{
  return mk3(fmaf(d.x, t, o.x), fmaf(d.y, t, o.y), fmaf(d.z, t, o.z));
}
__device__ __forceinline__ float comp(float3 v, int a) { return a == 0 ? v.x : (a == 1 ? v.y : v.z); }

/* Orthonormal basis around n (Duff et al., JCGT 6(1), 2017) */
__device__ __forceinline__ void
onb(float3 n, float3& b1, float3& b2)
{
  const float sign = copysignf(1.f, n.z);
  const float a = -1.f / (sign + n.z);
  const float b = n.x * n.y * a;
  b1 = mk3(1.f + sign * n.x * n.x * a, sign * b, -sign * n.x);
  b2 = mk3(b, sign + n.y * n.y * a, -n.y);
}

/* Direction with cosine mu to `axis' and azimuth 2 pi u */
__device__ __forceinline__ float3
around(float3 axis, float mu, float u)
{
  float3 b1, b2;
  float sp, cp;
  const float s = sqrtf(fmaxf(0.f, 1.f - mu * mu));
  onb(axis, b1, b2);
  sincospif(2.f * u, &sp, &cp);
  return nrm3(add3(add3(mul3(b1, cp * s), mul3(b2, sp * s)), mul3(axis, mu)));
}

/*******************************************************************************
 * Spectral helpers (FP64)
 ******************************************************************************/
/* B_lambda(T) in W/m^2/sr/m (src/core/htrdr_spectral.h:101-116) */
__device__ __forceinline__ double
planck_mono(double lambda, double T)
{
  const double c = 299792458.0, h = 6.62607015e-34, k = 1.380649e-23;
  const double l2 = lambda * lambda;
  const double l5 = l2 * l2 * lambda;
  return (2.0 * h * c * c / l5) / (exp(h * c / (lambda * k * T)) - 1.0);
}

__device__ __forceinline__ uint32_t
lower_bound_d(const double* a, uint32_t n, double key)
{
  uint32_t lo = 0, hi = n;
  while(lo < hi) {
    const uint32_t mid = (lo + hi) >> 1;
    if(__ldg(a + mid) < key) lo = mid + 1; else hi = mid;
  }
  return lo;
}

/* First CDF entry >= key, starting from a guide table: guide[b] is the first
 * entry >= b/G (G a power of two), so the answer lies in
 * [guide[floor(key G)], guide[floor(key G) + 1]] and a few probes finish the
 * search.  Same result as the plain lower bound, without its ~17 dependent
 * loads on a 97 000-entry Planck CDF. */
__device__ __forceinline__ uint32_t
cdf_search(const double* cdf, uint32_t n, const uint32_t* guide, uint32_t G, double key)
{
  if(!guide) return lower_bound_d(cdf, n, key);
  uint32_t b = (uint32_t)(key * (double)G);
  if(b >= G) b = G - 1;
  uint32_t lo = __ldg(guide + b), hi = __ldg(guide + b + 1);
  while(lo < hi) {
    const uint32_t mid = (lo + hi) >> 1;
    if(__ldg(cdf + mid) < key) lo = mid + 1; else hi = mid;
  }
  return lo;
}

/* htsky_find_spectral_band: lo[i] <= wlen < hi[i] (last upper bound inclusive) */
__device__ __forceinline__ uint32_t
find_band(const DScene& S, double wlen)
{
  uint32_t lo = 0, hi = S.nbands;
  while(lo < hi) {
    const uint32_t mid = (lo + hi) >> 1;
    if(__ldg(S.band_hi + mid) <= wlen) lo = mid + 1; else hi = mid;
  }
  if(lo == S.nbands) return (S.nbands && wlen == __ldg(S.band_hi + S.nbands - 1)) ? S.nbands - 1 : S.nbands;
  return wlen >= __ldg(S.band_lo + lo) ? lo : S.nbands;
}

/* htsky_spectral_band_sample_quadrature: first point whose cumulative weight > r */
__device__ __forceinline__ uint32_t
sample_quad(const DScene& S, double r, uint32_t band)
{
  const uint32_t off = __ldg(S.quad_off + band);
  const uint32_t n = __ldg(S.quad_off + band + 1) - off;
  uint32_t lo = 0, hi = n;
  while(lo < hi) {
    const uint32_t mid = (lo + hi) >> 1;
    if(__ldg(S.quad_cum + off + mid) <= r) lo = mid + 1; else hi = mid;
  }
  return lo < n ? lo : n - 1;
}

/* Black body fraction (src/core/htrdr_spectral.h:56-99), for the
 * continuous Planck sampler only */
__device__ double
wiebelt(double v)
{
  const double c15_pi4 = 15.0 / (HG_PI_D * HG_PI_D * HG_PI_D * HG_PI_D);
  double w;
  if(v >= 2.0) {
    w = 0.0;
    for(int m = 1; m < 6; ++m) {
      const double mv = (double)m * v;
      w += exp(-mv) / (double)(m * m * m * m) * (((mv + 3.0) * mv + 6.0) * mv + 6.0);
    }
    w *= c15_pi4;
  } else {
    const double v2 = v * v, v4 = v2 * v2;
    const double poly = 1.0 / 3.0 - 1.0 / 8.0 * v + 1.0 / 60.0 * v2 - 1.0 / 5040.0 * v2 * v2
                      + 1.0 / 272160.0 * v4 * v2 - 1.0 / 13305600.0 * v4 * v4;
    w = 1.0 - c15_pi4 * v2 * v * poly;
  }
  return w;
}
__device__ __forceinline__ double
bb_fraction(double l0, double l1, double T)
{
  const double C2 = 1.43877735e-2;
  return wiebelt(C2 / l1 / T) - wiebelt(C2 / l0 / T);
}
__device__ __forceinline__ double
planck_interval(double l0, double l1, double T)
{
  const double T2 = T * T;
  return bb_fraction(l0, l1, T) * 5.6696e-8 * (T2 * T2) / (HG_PI_D * (l1 - l0));
}

/* Wavelength sampling of a realisation.  Planck: 1-nm band CDF then uniform
 * in the band (htrdr_ran_wlen_planck.c:218-268), monochromatic when the
 * range is degenerate, bisection otherwise (:136-216); CIE: band CDF then the
 * quadratic inversion inside the band (htrdr_ran_wlen_cie_xyz.c:110-183).
 * *pdf in nm^-1, *cdf_band the CDF entry used. */
__device__ double
sample_wavelength(const DRequest& R, int channel, double r0, double r1, double* pdf,
                  uint32_t* cdf_band)
{
  if(R.mode == HG_IMAGE_CIE) {
    const double* cdf = R.cdf + (size_t)channel * R.ncdf;
    const uint32_t ib = cdf_search(cdf, R.ncdf, R.guide ? R.guide + (size_t)channel * (R.nguide + 1) : nullptr,
                                   R.nguide, nextafter(r0, DBL_MAX));
    const double lmin = R.wlen_range[0] + R.band_len * (double)ib;
    const double lmax = lmin + R.band_len;
    const double fmin = __ldg(R.fbound + ((size_t)channel * R.ncdf + ib) * 2 + 0);
    const double fmax = __ldg(R.fbound + ((size_t)channel * R.ncdf + ib) * 2 + 1);
    const double a = 0.5 * (fmax - fmin) / R.band_len;
    const double b = (lmax * fmin - lmin * fmax) / R.band_len;
    const double c = -lmin * fmin + lmin * lmin * a;
    const double d = 0.5 * (fmax + fmin) * R.band_len;
    double delta = b * b - 4 * a * (c - d * r1);
    if(delta < 0 && fabs(delta) <= 1e-6) delta = 0;
    const double sq = sqrt(delta);
    const double x1 = (-b - sq) / (2 * a), x2 = (-b + sq) / (2 * a);
    double l;
    if(lmin <= x1 && x1 < lmax) l = x1;
    else if(lmin <= x2 && x2 < lmax) l = x2;
    else l = (lmin + lmax) * 0.5;
    *pdf = R.rcp_integral[channel];
    *cdf_band = ib;
    return l;
  }
  if(R.ncdf) {
    const uint32_t i = cdf_search(R.cdf, R.ncdf, R.guide, R.nguide, nextafter(r0, DBL_MAX));
    const double lo = R.wlen_range[0] + (double)i * R.band_len;
    const double hi = lo + R.band_len;
    *pdf = __ldg(R.pdf + i) * (1.0 / (hi - lo));
    *cdf_band = i;
    return lo + (hi - lo) * r1;
  }
  *cdf_band = 0;
  if(fabs(R.wlen_range[0] - R.wlen_range[1]) <= 1e-6) {
    *pdf = 1.0;
    return R.wlen_range[0];
  }
  { /* continuous: bisection on the black body fraction */
    const double r0m = R.wlen_range[0] * 1e-9, r1m = R.wlen_range[1] * 1e-9;
    const double all = bb_fraction(r0m, r1m, R.ref_T);
    double lmin = r0m, lmax = r1m, l = 0, lprev = 0, bf = 0, bfprev = 0;
    for(int i = 0; i < 100; ++i) {
      l = (lmin + lmax) * 0.5;
      bf = bb_fraction(r0m, l, R.ref_T);
      if(bf / all < r0) lmin = l; else lmax = l;
      if(fabs(lprev - l) < 1e-15 || fabs(bfprev - bf) < 1e-6) break;
      lprev = l;
      bfprev = bf;
    }
    *pdf = planck_mono(l, R.ref_T) / (planck_interval(r0m, r1m, R.ref_T) * (r1m - r0m)) * 1e-9;
    return l * 1e9;
  }
}

/*******************************************************************************
 * Medium
 ******************************************************************************/
/* Layer i with z_i <= z < z_{i+1}, clamped */
__device__ __forceinline__ int
layer_of(const DScene& S, float z)
{
  uint32_t lo = 0, hi = S.nlayers + 1;
  while(lo < hi) {
    const uint32_t mid = (lo + hi) >> 1;
    if(__ldg(S.layer_z + mid) <= z) lo = mid + 1; else hi = mid;
  }
  if(lo == 0) return 0;
  if(lo > S.nlayers) return (int)S.nlayers - 1;
  return (int)lo - 1;
}

__device__ __forceinline__ float
gas_k(const DScene& S, uint32_t q, int prop, int layer)
{
  const float2 g = __ldg(S.gas + (size_t)q * S.nlayers + layer);
  return prop == HG_KA ? g.x : (prop == HG_KS ? g.y : __fadd_rn(g.x, g.y));
}

__device__ __forceinline__ float
sigma_of(const float4& o, int prop) { return prop == HG_KA ? o.x : (prop == HG_KS ? o.y : o.z); }

/* Raw k at a site: round(lwc*sigma) + k_gas in single precision, the same
 * operations as the majorant build (no contraction into an FMA). */
__device__ __forceinline__ float
site_k(const DScene& S, int cell, int layer, uint32_t band, uint32_t q, int prop, int cpnt)
{
  float kc = 0.f, kg = 0.f;
  if((cpnt & 2) && cell >= 0) kc = __fmul_rn(__ldg(S.lwc + cell), sigma_of(__ldg(S.optics + band), prop));
  if((cpnt & 1) && layer >= 0) kg = gas_k(S, q, prop, layer);
  return __fadd_rn(kc, kg);
}

/* Flat ground z = 0 with the self-hit rule of src/core/htrdr_geometry.c:118-150 */
__device__ __forceinline__ float
ground_trace(const DScene& S, float3 o, float3 d, float r0, float r1, bool prev_ground)
{
  if(!S.has_ground || prev_ground || d.z == 0.f) return -1.f;
  const float t = -o.z / d.z;
  return (t <= r0 || t >= r1) ? -1.f : t;
}

/* Ground query of the walk, on the mesh when the scene has one, else on the
 * plane: distance in [0, r1) (< 0: none), the hit primitive, whether the hit
 * lies on an edge and the geometric normal.  `prev' says the ray leaves the
 * ground at (prev_prim, prev_edge). */
template <unsigned V>
__device__ __forceinline__ float
ground_query(const DScene& S, float3 o, float3 d, float r1, bool prev, uint32_t prev_prim,
             bool prev_edge, uint32_t* prim, bool* edge, float3* ng)
{
  if(!(V & HV_MESH) || !S.g_ntris) {
    *prim = 0;
    *edge = false;
    *ng = make_float3(0.f, 0.f, 1.f);
    return ground_trace(S, o, d, 0.f, r1, prev);
  }
  const GHit h = g_trace(S, o, d, 0.f, r1, prev ? prev_prim : HG_NO_PRIM, prev && prev_edge);
  *prim = h.prim;
  *edge = h.prim != HG_NO_PRIM && g_on_edge(h.u, h.v);
  *ng = h.ng;
  return h.prim == HG_NO_PRIM ? -1.f : h.dist;
}

/* Ground properties at a surface event: the normal (unoriented), the BRDF
 * type and reflectivity and the temperature.  On the mesh, the material of
 * the hit side's interface and the BRDF tabulated at the wavelength, chosen
 * with one transport canonical as htrdr_mtl_create_bsdf does
 * (src/core/htrdr_materials.c:414-463); on the plane, its constants, the
 * canonical being drawn all the same (htrdr_mtl_create_bsdf draws it whatever
 * the material's BRDF count, :428).  A side without a BRDF reflects nothing. */
struct SurfProps {
  float3 N;
  float refl, T;
  int specular;
};

template <unsigned V>
__device__ __forceinline__ SurfProps
surface_props(const DScene& S, Rng& rng, float3 dir, uint32_t prim, float3 ng, double wlen_nm)
{
  SurfProps s;
  if(!(V & HV_MESH) || !S.g_ntris) {
    (void)rng.uf();
    s.N = make_float3(0.f, 0.f, 1.f);
    s.refl = S.ground_refl;
    s.specular = S.ground_brdf == 1;
    s.T = S.ground_T;
    return s;
  }
  const float n = rsqrtf(ng.x * ng.x + ng.y * ng.y + ng.z * ng.z);
  s.N = make_float3(ng.x * n, ng.y * n, ng.z * n);
  const uint32_t m = g_hit_mtl(S, prim, ng, dir);
  const double r = (double)rng.uf();
  const uint32_t b = m == HG_NO_PRIM ? HG_NO_PRIM : g_fetch_brdf(S, m, wlen_nm, r);
  if(b == HG_NO_PRIM) {
    s.refl = 0.f;
    s.specular = 0;
    s.T = m == HG_NO_PRIM ? 0.f : __ldg(S.g_mtl_T + m);
    return s;
  }
  const float2 br = __ldg(S.g_brdf + b);
  s.specular = br.x != 0.f;
  s.refl = br.y;
  s.T = __ldg(S.g_mtl_T + m);
  return s;
}

/*******************************************************************************
 * Trace state: one delta-tracking query through the medium
 ******************************************************************************/
enum { TK_SCATTER = 0, TK_TRANS = 1, TK_LW = 2 };

struct Trace {
  float3 o, d, inv;
  float ta, cb0, cb1, tb;  /* regions: gas [ta,cb0) | cloud [cb0,cb1) | gas [cb1,tb) */
  float t;                 /* start of the current voxel */
  float tcur;              /* traversal distance (filter context) */
  uint32_t grank;          /* leaf grid of the octree (cloud region) */
  double Ts, Tmin;
  uint64_t base;           /* first node of the octree */
  int32_t layer;           /* gas region: current layer */
  uint32_t c[3];           /* cloud region: current cell (tile-local) */
  int32_t tile[2];
  int32_t site_cell, site_layer;
  uint32_t steps;
  /* ancestor cache of the current leaf: child block and level of its parent
   * (p) and grandparent (g); `start' says where the next descent begins
   * (0 root, 1 parent, 2 grandparent) */
  uint32_t p_base, g_base;
  uint8_t p_level, g_level, start;
  uint8_t kind, prop, region, has_cloud, hit, event;
};

/*******************************************************************************
 * Path state machine
 ******************************************************************************/
enum {
  ST_IDLE = 0, ST_GEN, ST_RAD_BEGIN, ST_SW_DIRECT_END, ST_SW_WALK, ST_SW_SCAT_END,
  ST_SW_ABS_END, ST_SW_NEE_END, ST_LW_WALK, ST_LW_END, ST_RAD_END, ST_TRACE, ST_DONE
};


enum {
  PF_SURFACE = 1u << 0, PF_SPECULAR = 1u << 1, PF_PREV_GROUND = 1u << 2, PF_RAYLEIGH = 1u << 3,
  PF_DIRECT = 1u << 4, PF_DIFFUSE = 1u << 5, PF_IN_CONE = 1u << 6, PF_TRACED = 1u << 7,
  PF_REJECTED = 1u << 8, PF_STAGE2 = 1u << 9, PF_LW = 1u << 10, PF_FAILED = 1u << 11
};

struct Counters {
  unsigned long long seg, node, tc, real, fail, grid;
};

struct Path {
  /* trace part: everything trace_step reads or writes.  It comes first so
   * that the wavefront engine's trace stage moves only this prefix of a
   * stored path (HG_TRACE_WORDS). */
  Rng rng;
  uint32_t c_grid;      /* local counter of leaf-grid bytes read (the word before
                         * the 8-byte aligned Trace: no extra storage) */
  Trace tr;
  uint32_t band, q, flags;
  uint32_t si;          /* scene of the path (engines with many scenes) */
  unsigned long long t0;
  uint32_t c_seg, c_node, c_tc; /* local counters */
  uint8_t state, ret, mode, chan;
  /* walk fields the wavefront's trace stage reads or writes when it runs a
   * LW scattering itself, and the realisation's pixel and index */
  uint32_t bounces;
  float gdist;          /* ground distance along the current free path, < 0: none */
  uint32_t pix, ireal;
  /* event part */
  float3 org, rdir;     /* sensor ray */
  float3 pos, dir, pnext, dnext, sdir;
  double w, wdirect, inv_pdf, L_sun, weight, wlen_d;
  float ksi, tr_abs, R, refl, sun_ipdf, g, cosN, wlen;
  uint32_t ri;
  /* ground: the hit of the walk's last ground query, and the surface the
   * path leaves (for the self-hit rule) */
  float3 gN;
  uint32_t gprim, prev_prim;
  uint8_t gedge, prev_edge;
};

/* 32-bit words of a stored path, and of its trace part */
#define HG_PATH_WORDS ((uint32_t)(sizeof(Path) / 4))
#define HG_TRACE_WORDS ((uint32_t)(offsetof(Path, org) / 4))
static_assert(offsetof(Path, tr) == 40 && offsetof(Path, org) == 240, "trace prefix of 15 vectors");
static_assert(sizeof(Path) % 4 == 0 && offsetof(Path, org) % 4 == 0, "word-wise path storage");

__device__ __forceinline__ unsigned long long
gtimer()
{
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ void
slab(float o, float d, float inv, float lo, float hi, float& t0, float& t1)
{
  if(d != 0.f) {
    float a = (lo - o) * inv, b = (hi - o) * inv;
    if(a > b) { const float t = a; a = b; b = t; }
    t0 = fmaxf(t0, a);
    t1 = fminf(t1, b);
  } else if(o < lo || o > hi) {
    t0 = 1.f; t1 = 0.f;
  }
}

__device__ __forceinline__ int
floordiv_i(int a, int b)
{
  int q = a / b;
  if((a % b != 0) && ((a < 0) != (b < 0))) --q;
  return q;
}

/* Region r of the trace: [rstart, rend) and whether it is the cloud box */
__device__ __forceinline__ void
region_bounds(const Trace& T, int r, float& s, float& e, bool& cloud)
{
  if(!T.has_cloud) { s = T.ta; e = T.tb; cloud = false; return; }
  if(r == 0) { s = T.ta; e = T.cb0; cloud = false; }
  else if(r == 1) { s = T.cb0; e = T.cb1; cloud = true; }
  else { s = T.cb1; e = T.tb; cloud = false; }
}

/* Set up the current region (skipping empty ones) at its start */
__device__ __forceinline__ void
region_enter(Trace& T, const DScene& S)
{
  const int nreg = T.has_cloud ? 3 : 1;
  while(T.region < nreg) {
    float s, e;
    bool cloud;
    region_bounds(T, T.region, s, e, cloud);
    if(s < e) {
      T.t = s;
      const float3 p = madd3(T.o, T.d, s);
      if(!cloud) {
        int l = layer_of(S, p.z);
        if(T.d.z < 0.f && l > 0 && p.z <= __ldg(S.layer_z + l)) --l;
        T.layer = l;
      } else {
#pragma unroll
        for(int a = 0; a < 3; ++a) {
          int g = __float2int_rd((comp(p, a) - S.lower[a]) * S.inv_cell[a]);
          if(S.repeat && a < 2) {
            const int tl = floordiv_i(g, (int)S.def[a]);
            T.tile[a] = tl;
            g -= tl * (int)S.def[a];
          }
          g = max(0, min(g, (int)S.def[a] - 1));
          T.c[a] = (uint32_t)g;
        }
        if(!S.repeat) { T.tile[0] = 0; T.tile[1] = 0; }
        T.start = 0; /* descend from the root */
      }
      return;
    }
    ++T.region;
  }
}

__device__ __forceinline__ void
trace_begin(Path& p, const DScene& S, int kind, int prop, float3 o, float3 d, float t0,
            float t1, uint8_t ret)
{
  Trace& T = p.tr;
  T.kind = (uint8_t)kind;
  T.prop = (uint8_t)prop;
  T.o = o;
  T.d = d;
  T.inv = mk3(1.f / d.x, 1.f / d.y, 1.f / d.z);
  T.hit = 0;
  T.event = 2;
  T.Tmin = 0.0;
  T.tcur = 0.f;
  T.steps = 0;
  T.region = 0;
  if(kind == TK_TRANS) {
    /* a transmissivity trace sets no collision site: the site of the free
     * path before it stays for the scattering that follows (the absorption
     * transmissivity to a collision site, ..._sw.c:394-398) */
    T.Ts = p.rng.exp1(); /* ..._sw.c:239 */
  } else {
    T.site_cell = -1;
    T.site_layer = -1;
  }
  p.state = ST_TRACE;
  p.ret = ret;

  float ta = t0, tb = fminf(t1, HG_MAX_DIST);
  slab(o.z, d.z, T.inv.z, 0.f, S.ztop, ta, tb);
  T.ta = ta; T.tb = tb;
  T.has_cloud = 0;
  if(!(ta < tb)) { T.region = 3; T.ta = T.tb = 0.f; return; }
  if(S.has_cloud) {
    float c0 = ta, c1 = tb;
    if(!S.repeat) {
      slab(o.x, d.x, T.inv.x, S.lower[0], S.upper[0], c0, c1);
      slab(o.y, d.y, T.inv.y, S.lower[1], S.upper[1], c0, c1);
    }
    slab(o.z, d.z, T.inv.z, S.lower[2], S.upper[2], c0, c1);
    if(c0 < c1) {
      T.has_cloud = 1;
      T.cb0 = c0;
      T.cb1 = c1;
      T.base = S.tree_base[(size_t)p.q * 3 + prop];
      T.grank = S.grid_rank ? __ldg(S.grid_rank + (size_t)p.q * 3 + prop) : 0u;
    }
  }
  region_enter(T, S);
}

/* Collision site (cell clamped into the voxel box, gas layer clamped into the
 * layers the cell overlaps) of a point inside the current voxel. */
__device__ __forceinline__ void
site_of(const DScene& S, const Trace& T, bool cloud, const uint32_t lo[3], const uint32_t hi[3],
        float3 x, int& cell, int& layer)
{
  if(!cloud) { cell = -1; layer = T.layer; return; }
  int c[3];
#pragma unroll
  for(int a = 0; a < 3; ++a) {
    int g = __float2int_rd((comp(x, a) - S.lower[a]) * S.inv_cell[a]);
    if(a < 2) g -= T.tile[a] * (int)S.def[a];
    c[a] = max((int)lo[a], min(g, (int)hi[a] - 1));
  }
  cell = (c[2] * (int)S.def[1] + c[1]) * (int)S.def[0] + c[0];
  const int2 lr = __ldg(S.cell_layers + c[2]);
  if(lr.x < 0) { layer = -1; return; }
  layer = max(lr.x, min(layer_of(S, x.z), lr.y));
}

/* The hit filters (..._sw.c:73-217, ..._lw.c:64-135) on voxel [d0, d1].
 * Returns true when the traversal stops (real collision). */
template <unsigned V>
__device__ __forceinline__ bool
voxel_filter(Path& p, const DScene& S, float d0, float d1, float kmin, float kmax, bool cloud,
             const uint32_t lo[3], const uint32_t hi[3])
{
  Trace& T = p.tr;
  /* the kinds the variant can meet (a LW-only variant meets TK_LW alone) */
  const bool trans = (V & HV_SW) && T.kind == TK_TRANS;
  const bool scat = (V & HV_SW) && (!(V & HV_LW) || T.kind == TK_SCATTER);
  /* the traversed distance is carried in FP64 inside the voxel so that tiny
   * free paths still advance it far from the origin */
  double tc = (double)d0;
  const double e = (double)d1;
  if(trans) {
    T.Tmin += (e - tc) * (double)kmin;
    if(T.Tmin >= HG_TMIN_ZERO) return true; /* exp(-Tmin) is already 0.0 */
    const double kdif = (double)kmax - (double)kmin;
    for(uint32_t it = 0;; ++it) {
      const double Tdif = (e - tc) * kdif;
      if(T.Ts > Tdif) { T.Ts -= Tdif; T.tcur = d1; return false; }
      if(it >= HG_MAX_NULL) { p.flags |= PF_FAILED; return true; }
      tc += T.Ts / kdif;
      T.tcur = (float)tc;
      int cell, layer;
      site_of(S, T, cloud, lo, hi, madd3(T.o, T.d, T.tcur), cell, layer);
      float k = site_k(S, cell, layer, p.band, p.q, T.prop, 3);
      k = fminf(fmaxf(k, kmin), kmax);
      ++p.c_tc;
      if((double)p.rng.uf() < ((double)k - (double)kmin) / kdif) return true;
      T.Ts = p.rng.exp1();
    }
  } else {
    for(uint32_t it = 0;; ++it) {
      const double Tv = (e - tc) * (double)kmax;
      if(T.Ts > Tv) { T.Ts -= Tv; T.tcur = d1; return false; }
      if(it >= HG_MAX_NULL) { p.flags |= PF_FAILED; T.tcur = d1; return false; }
      tc += T.Ts / (double)kmax;
      T.tcur = (float)tc;
      if(tc > (double)HG_MAX_DIST) return false;
      int cell, layer;
      site_of(S, T, cloud, lo, hi, madd3(T.o, T.d, T.tcur), cell, layer);
      ++p.c_tc;
      if(scat) {
        const float ks = site_k(S, cell, layer, p.band, p.q, HG_KS, 3);
        if(p.rng.uf() < ks / kmax) { T.site_cell = cell; T.site_layer = layer; return true; }
      } else {
        const float ka = site_k(S, cell, layer, p.band, p.q, HG_KA, 3);
        const float ks = site_k(S, cell, layer, p.band, p.q, HG_KS, 3);
        const float r = p.rng.uf();
        const float pa = ka / kmax, ps = ks / kmax;
        if(r < pa) { T.event = 0; T.site_cell = cell; T.site_layer = layer; return true; }
        if(r < pa + ps) { T.event = 1; T.site_cell = cell; T.site_layer = layer; return true; }
      }
      T.Ts = p.rng.exp1();
    }
  }
}

__device__ __forceinline__ void
trace_finish(Path& p, bool hit)
{
  p.tr.hit = hit ? 1 : 0;
  p.state = p.ret;
}

/* SW walk after a free path that ended by a collision in the medium: the
 * absorption transmissivity along that free path, from its origin to the
 * collision site (..._sw.c:385-398).  It reads and writes only the trace
 * part of the path, so the wavefront's trace stage runs it in place of an
 * event-stage visit.  Returns the collision site (pos_next). */
__device__ __forceinline__ float3
sw_scat_volume(Path& p, const DScene& S)
{
  const float3 o = p.tr.o, d = p.tr.d;
  const float tdst = p.tr.tcur;
  p.flags &= ~(PF_SURFACE | PF_PREV_GROUND);
  trace_begin(p, S, TK_TRANS, HG_KA, o, d, 0.f, tdst, ST_SW_ABS_END);
  return madd3(o, d, tdst);
}

/* Vertical optical depth from z = 0 to z (clamped to the column) */
__device__ __forceinline__ double
gas_tau_at(const DScene& S, const double* cum, uint32_t q, int prop, double z)
{
  z = fmin(fmax(z, 0.0), (double)S.ztop);
  uint32_t lo = 0, hi = S.nlayers + 1; /* upper bound on the FP64 bounds */
  while(lo < hi) {
    const uint32_t mid = (lo + hi) >> 1;
    if(__ldg(S.layer_zd + mid) <= z) lo = mid + 1; else hi = mid;
  }
  const int l = lo == 0 ? 0 : min((int)lo - 1, (int)S.nlayers - 1);
  return __ldg(cum + l) + (double)gas_k(S, q, prop, l) * (z - __ldg(S.layer_zd + l));
}

/* A whole gas region [T.t, re] of a non-horizontal ray in one step.  Along
 * the ray the optical depth is the vertical one divided by |dz|, and the
 * vertical optical depth is the piecewise-linear cumulative sum over the
 * layers, so the voxel-by-voxel walk of the reference (every layer is a
 * voxel with kmin = kmax = k_gas: no null collision, no random draw except at
 * the collision) reduces to: Tmin += dtau for a transmissivity, and for a
 * free path the inversion of the cumulative depth at Ts.  The same random
 * numbers are consumed as in the layer-by-layer traversal.  Returns true when
 * the trace stops (real collision). */
template <unsigned V>
__device__ __forceinline__ bool
gas_region(Path& p, const DScene& S, float re)
{
  Trace& T = p.tr;
  const bool trans = (V & HV_SW) && T.kind == TK_TRANS;
  const bool scat = (V & HV_SW) && (!(V & HV_LW) || T.kind == TK_SCATTER);
  const double dz = (double)T.d.z, adz = fabs(dz);
  const double* cum = S.gas_cum + ((size_t)p.q * 3 + T.prop) * (S.nlayers + 1);
  double ta = (double)T.t;
  double tau_a = gas_tau_at(S, cum, p.q, T.prop, (double)T.o.z + dz * ta);
  const double tau_b = gas_tau_at(S, cum, p.q, T.prop, (double)T.o.z + dz * (double)re);
  if(trans) {
    T.Tmin += fabs(tau_b - tau_a) / adz;
    return T.Tmin >= HG_TMIN_ZERO; /* exp(-Tmin) is already 0.0 */
  }
  for(uint32_t it = 0;; ++it) {
    const double dtau = fabs(tau_b - tau_a) / adz;
    if(T.Ts > dtau) { T.Ts -= dtau; T.tcur = re; return false; }
    if(it >= HG_MAX_NULL) { p.flags |= PF_FAILED; T.tcur = re; return false; }
    /* layer where the cumulative depth reaches the target */
    const double target = tau_a + (dz > 0 ? T.Ts * adz : -T.Ts * adz);
    uint32_t lo = 0, hi = S.nlayers;
    if(dz > 0) { /* largest l with cum[l] < target */
      while(hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if(__ldg(cum + mid) < target) lo = mid; else hi = mid;
      }
    } else { /* smallest l with cum[l+1] > target */
      hi = S.nlayers - 1;
      while(lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        if(__ldg(cum + mid + 1) > target) hi = mid; else lo = mid + 1;
      }
    }
    const int l = (int)lo;
    const float k = gas_k(S, p.q, T.prop, l);
    double z = __ldg(S.layer_zd + l);
    if(k > 0.f) z += (target - __ldg(cum + l)) / (double)k;
    double t = (z - (double)T.o.z) / dz;
    t = fmin(fmax(t, ta), (double)re);
    T.tcur = (float)t;
    ++p.c_tc;
    if(scat) {
      /* k_s max of a gas voxel is k_s itself: the test always accepts */
      if(p.rng.uf() < 1.0f) { T.site_cell = -1; T.site_layer = l; return true; }
    } else {
      const float ka = site_k(S, -1, l, p.band, p.q, HG_KA, 3);
      const float ks = site_k(S, -1, l, p.band, p.q, HG_KS, 3);
      const float r = p.rng.uf();
      const float pa = ka / k, ps = ks / k;
      if(r < pa) { T.event = 0; T.site_cell = -1; T.site_layer = l; return true; }
      if(r < pa + ps) { T.event = 1; T.site_cell = -1; T.site_layer = l; return true; }
    }
    /* null collision (rounding of ka + ks): keep tracking from there */
    T.Ts = p.rng.exp1();
    tau_a = target;
    ta = t;
  }
}

/* One voxel of the current trace */
template <unsigned V>
__device__ __forceinline__ void
trace_step(Path& p, const DScene& S)
{
  Trace& T = p.tr;
  const int nreg = T.has_cloud ? 3 : 1;
  if(T.region >= nreg) { trace_finish(p, false); return; }
  if(++T.steps > HG_MAX_STEPS) { p.flags |= PF_FAILED; trace_finish(p, false); return; }
  float rs, re;
  bool cloud;
  region_bounds(T, T.region, rs, re, cloud);
  ++p.c_seg;
  if(!cloud && T.d.z != 0.f) { /* the whole gas region at once */
    if(gas_region<V>(p, S, re)) { trace_finish(p, true); return; }
    ++T.region;
    region_enter(T, S);
    return;
  }
  if(!cloud) {
    const int l = T.layer;
    float tn = FLT_MAX;
    if(T.d.z > 0.f) tn = (__ldg(S.layer_z + l + 1) - T.o.z) * T.inv.z;
    else if(T.d.z < 0.f) tn = (__ldg(S.layer_z + l) - T.o.z) * T.inv.z;
    const float t1 = fmaxf(fminf(tn, re), T.t);
    if(t1 > T.t) {
      const float k = gas_k(S, p.q, T.prop, l);
      const uint32_t z3[3] = {0, 0, 0};
      if(voxel_filter<V>(p, S, T.t, t1, k, k, false, z3, z3)) { trace_finish(p, true); return; }
    }
    if(tn >= re) { ++T.region; region_enter(T, S); return; }
    T.t = t1;
    const int ln = l + (T.d.z > 0.f ? 1 : -1);
    if(ln < 0 || ln >= (int)S.nlayers) { ++T.region; region_enter(T, S); return; }
    T.layer = ln;
    return;
  }
  /* cloud voxel: descend to the leaf holding the current cell, from the
   * deepest cached ancestor that also holds it */
  const uint4* nodes = S.nodes + T.base;
  uint32_t L, base;
  uint4 v;
  bool leaf_root = false;
  bool found = false;
  if(S.maj_grid) {
    /* the leaf's majorants and level from the cell: two independent loads,
     * no node read */
    const uint64_t gi = (uint64_t)T.grank * S.ncell
                      + ((uint64_t)T.c[2] * S.def[1] + T.c[1]) * S.def[0] + T.c[0];
    const float2 mm = __ldg(S.maj_grid + gi);
    L = __ldg(S.lvl_grid + gi);
    p.c_grid += 9;
    v.x = __float_as_uint(mm.x);
    v.y = __float_as_uint(mm.y);
    found = true;
  } else if(T.start == 1) {
    base = T.p_base; L = T.p_level;
  } else if(S.leaf_grid) {
    /* the leaf from the cell's grid entry: two dependent loads whatever the
     * depth; its parent's child block is cached for the next steps */
    const uint64_t cell = ((uint64_t)T.c[2] * S.def[1] + T.c[1]) * S.def[0] + T.c[0];
    const uint32_t e = __ldg(S.leaf_grid + (uint64_t)T.grank * S.ncell + cell);
    const uint32_t n = e >> 5;
    L = e & 31u;
    v = __ldg(nodes + n);
    ++p.c_node;
    p.c_grid += 4;
    found = true;
    if(L < S.depth) {
      const uint32_t oct = ((T.c[0] >> L) & 1u) | (((T.c[1] >> L) & 1u) << 1) | (((T.c[2] >> L) & 1u) << 2);
      T.p_base = n - oct;
      T.p_level = (uint8_t)(L + 1);
    } else {
      T.p_level = 0xFF; /* the root is the leaf: no ancestor */
    }
    T.g_level = 0xFF;
  } else if(T.start == 2) {
    base = T.g_base; L = T.g_level;
    T.p_base = base; T.p_level = (uint8_t)L; T.g_level = 0xFF;
  } else {
    v = __ldg(nodes);
    ++p.c_node;
    L = S.depth;
    base = v.z;
    T.p_base = base; T.p_level = (uint8_t)L; T.g_level = 0xFF;
    leaf_root = v.z == HG_LEAF;
  }
  if(!leaf_root && !found) {
    for(;;) {
      --L;
      const uint32_t oct = ((T.c[0] >> L) & 1u) | (((T.c[1] >> L) & 1u) << 1) | (((T.c[2] >> L) & 1u) << 2);
      v = __ldg(nodes + base + oct);
      ++p.c_node;
      if(v.z == HG_LEAF) break;
      T.g_base = T.p_base; T.g_level = T.p_level;
      T.p_base = v.z; T.p_level = (uint8_t)L;
      base = v.z;
    }
  } else if(leaf_root) {
    T.p_level = 0xFF; /* the root is the leaf: no ancestor */
  }
  uint32_t lo[3], hi[3];
  float texit = FLT_MAX;
  int axis = -1;
#pragma unroll
  for(int a = 0; a < 3; ++a) {
    lo[a] = (T.c[a] >> L) << L;
    hi[a] = min(lo[a] + (1u << L), S.def[a]);
    const float off = a < 2 ? (float)(T.tile[a] * (int)S.def[a]) : 0.f;
    const float da = comp(T.d, a);
    float ta;
    if(da > 0.f) ta = (S.lower[a] + (off + (float)hi[a]) * S.cell[a] - comp(T.o, a)) * comp(T.inv, a);
    else if(da < 0.f) ta = (S.lower[a] + (off + (float)lo[a]) * S.cell[a] - comp(T.o, a)) * comp(T.inv, a);
    else continue;
    if(ta < texit) { texit = ta; axis = a; }
  }
  const float t1 = fmaxf(fminf(texit, re), T.t);
  if(t1 > T.t) {
    if(voxel_filter<V>(p, S, T.t, t1, __uint_as_float(v.x), __uint_as_float(v.y), true, lo, hi)) {
      trace_finish(p, true);
      return;
    }
  }
  if(texit >= re || axis < 0) { ++T.region; region_enter(T, S); return; }
  /* next cell: exit face on `axis', the exit point's cell on the others */
  const float3 pe = madd3(T.o, T.d, texit);
  uint32_t nc3[3];
  bool leave = false;
#pragma unroll
  for(int a = 0; a < 3; ++a) { /* unrolled: no dynamic indexing, the path stays in registers */
    int nc;
    if(a == axis) {
      nc = comp(T.d, a) > 0.f ? (int)hi[a] : (int)lo[a] - 1;
      if(nc < 0 || nc >= (int)S.def[a]) {
        if(S.repeat && a < 2) {
          if(nc < 0) { T.tile[a] -= 1; nc = (int)S.def[a] - 1; }
          else { T.tile[a] += 1; nc = 0; }
        } else {
          leave = true;
        }
      }
    } else {
      int g = __float2int_rd((comp(pe, a) - S.lower[a]) * S.inv_cell[a]);
      if(a < 2) g -= T.tile[a] * (int)S.def[a];
      nc = max((int)lo[a], min(g, (int)hi[a] - 1));
    }
    nc3[a] = (uint32_t)nc;
  }
  if(leave) { ++T.region; region_enter(T, S); return; }
  { /* deepest cached ancestor whose cube also holds the next cell */
    const uint32_t diff = (T.c[0] ^ nc3[0]) | (T.c[1] ^ nc3[1]) | (T.c[2] ^ nc3[2]);
    if(T.p_level < 32 && (diff >> T.p_level) == 0) T.start = 1;
    else if(T.g_level < 32 && (diff >> T.g_level) == 0) T.start = 2;
    else T.start = 0;
  }
  T.c[0] = nc3[0];
  T.c[1] = nc3[1];
  T.c[2] = nc3[2];
  T.t = texit;
}

/*******************************************************************************
 * Scattering functions (star-sf), sun and ground
 ******************************************************************************/
__device__ __forceinline__ float
hg_mu(float g, float u)
{
  if(fabsf(g) < 1e-6f) return 1.f - 2.f * u;
  const float s = (1.f - g * g) / (1.f - g + 2.f * g * u);
  return fminf(1.f, fmaxf(-1.f, (1.f + g * g - s * s) / (2.f * g)));
}
__device__ __forceinline__ float
hg_eval(float g, float mu)
{
  const float d = 1.f + g * g - 2.f * g * mu;
  return (1.f - g * g) / (4.f * HG_PI_F * d * sqrtf(d));
}
__device__ __forceinline__ float
rayleigh_mu(float u)
{
  const float A = 4.f * u - 2.f;
  const float c = cbrtf(A + sqrtf(A * A + 1.f));
  return fminf(1.f, fmaxf(-1.f, c - 1.f / c));
}
__device__ __forceinline__ float
rayleigh_eval(float mu) { return 3.f / (16.f * HG_PI_F) * (1.f + mu * mu); }

/* Sun cap sample (htrdr_atmosphere_sun.c:126-136) in FP64, returns 1/pdf */
__device__ __forceinline__ float3
sun_sample(const DScene& S, Rng& rng)
{
  const double u1 = rng.uf(), u2 = rng.uf();
  const double mu = 1.0 - u1 * (1.0 - S.sun_cos_half);
  const double s = sqrt(fmax(0.0, 1.0 - mu * mu));
  double sp, cp;
  sincospi(2.0 * u2, &sp, &cp);
  double d[3];
  for(int i = 0; i < 3; ++i)
    d[i] = (double)S.sun_b1[i] * cp * s + (double)S.sun_b2[i] * sp * s + S.sun_dir_d[i] * mu;
  const double n = rsqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
  return mk3((float)(d[0] * n), (float)(d[1] * n), (float)(d[2] * n));
}

__device__ __forceinline__ bool
in_solar_cone(const DScene& S, float3 d)
{
  return (double)d.x * S.sun_dir_d[0] + (double)d.y * S.sun_dir_d[1] + (double)d.z * S.sun_dir_d[2]
      >= S.sun_cos_half;
}

/*******************************************************************************
 * Events
 ******************************************************************************/
struct GenOut {
  Rng rng;               /* stream state after the sensor and spectral draws */
  float3 org, rdir, dir; /* sensor ray; dir: direction of the first radiance call */
  double wlen, inv_pdf;
  uint32_t band, q, flags;
  float cosN;
  uint32_t chan;
};

/* The sampling part of path_generate, out of line (it runs once per
 * realisation and is large: FP64 sensor and spectral sampling). */
__device__ __noinline__ GenOut
gen_sample(const DScene& S, const DRequest& R, uint32_t pix, uint32_t ireal)
{
  GenOut g;
  Path p; /* scratch holder so that the shared helpers below keep their form */
  const uint32_t px = pix % R.width, py = pix / R.width;
  p.rng.init(pix, R.seed, ireal, 0u);
  p.flags = 0;
  p.chan = R.mode == HG_IMAGE_CIE ? (uint8_t)(ireal / R.spp) : 0;
  g.chan = p.chan;
  g.cosN = 0.f;
  g.wlen = 0;
  g.inv_pdf = 0;
  g.band = g.q = 0;
  if(R.mode == HG_FLUX_SW || R.mode == HG_FLUX_LW) {
    const double s0 = ((double)px + p.rng.ud()) * R.pix_sz[0];
    const double s1 = ((double)py + p.rng.ud()) * R.pix_sz[1];
    double o[3];
    for(int i = 0; i < 3; ++i)
      o[i] = R.rect_pos[i] + R.rect_ax[i] * (s0 * 2.0 - 1.0) + R.rect_ay[i] * (s1 * 2.0 - 1.0);
    p.org = mk3((float)o[0], (float)o[1], (float)o[2]);
    bool inside = S.g_ntris ? false : (S.has_ground && o[2] < 0);
    if(S.g_ntris) { /* the upward ray must leave through the atmosphere's side */
      const GHit h = g_trace(S, p.org, make_float3(0.f, 0.f, 1.f), 0.f, FLT_MAX, HG_NO_PRIM, false);
      if(h.prim != HG_NO_PRIM) {
        const uint4 f = __ldg(S.g_iface + __ldg(S.g_iface_of + h.prim));
        inside = (h.ng.z < 0.f ? f.x : f.z) != S.g_sky_mtl; /* cos(up, N) < 0: front */
      }
    }
    if(inside) {
      g.rng = p.rng; g.org = g.rdir = g.dir = p.org; g.flags = PF_REJECTED;
      return g;
    }
    const float u1 = p.rng.uf(), u2 = p.rng.uf();
    p.rdir = around(mk3((float)R.rect_n[0], (float)R.rect_n[1], (float)R.rect_n[2]),
                    sqrtf(1.f - u2), u1);
  } else {
    const double f0 = ((double)px + p.rng.ud()) * R.pix_sz[0];
    const double f1 = ((double)py + p.rng.ud()) * R.pix_sz[1];
    const double l0 = p.rng.ud(), l1 = p.rng.ud();
    const double x = 2.0 * f0 - 1.0, y = 2.0 * f1 - 1.0;
    double o[3], d[3];
    if(R.camera_type == 1) {
      const double hw = 0.5 * R.ortho_h * R.aspect, hh = 0.5 * R.ortho_h;
      for(int i = 0; i < 3; ++i) { o[i] = R.cam_pos[i] + R.cam_r[i] * x * hw + R.cam_u[i] * y * hh; d[i] = R.cam_f[i]; }
    } else {
      for(int i = 0; i < 3; ++i)
        d[i] = R.cam_f[i] + R.cam_r[i] * (x * R.tan_half * R.aspect) + R.cam_u[i] * (y * R.tan_half);
      if(R.lens_radius > 0) {
        const double rho = R.lens_radius * sqrt(l0);
        double sp, cp;
        sincospi(2.0 * l1, &sp, &cp);
        for(int i = 0; i < 3; ++i) {
          const double focus = R.cam_pos[i] + d[i] * R.focal_dst;
          o[i] = R.cam_pos[i] + R.cam_r[i] * rho * cp + R.cam_u[i] * rho * sp;
          d[i] = focus - o[i];
        }
      } else {
        for(int i = 0; i < 3; ++i) o[i] = R.cam_pos[i];
      }
    }
    const double n = rsqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
    p.org = mk3((float)o[0], (float)o[1], (float)o[2]);
    p.rdir = mk3((float)(d[0] * n), (float)(d[1] * n), (float)(d[2] * n));
  }
  const double r0 = p.rng.ud(), r1 = p.rng.ud(), r2 = p.rng.ud();
  double pdf;
  uint32_t cb;
  const double wlen = sample_wavelength(R, p.chan, r0, r1, &pdf, &cb);
  pdf *= 1e9;
  const uint32_t band = find_band(S, wlen);
  g.org = p.org;
  g.rdir = p.rdir;
  g.dir = p.rdir;
  if(band >= S.nbands) { g.rng = p.rng; g.flags = PF_REJECTED; return g; }
  g.wlen = wlen;
  g.band = band;
  g.q = __ldg(S.quad_off + band) + sample_quad(S, r2, band);
  g.inv_pdf = 1.0 / pdf;
  g.flags = 0;
  switch(R.mode) {
    case HG_XWAVE_LW: g.flags |= PF_LW; break;
    case HG_FLUX_LW: g.flags |= PF_LW; g.inv_pdf = HG_PI_D / pdf; break;
    case HG_FLUX_SW: {
      const float3 sd = sun_sample(S, p.rng);
      const float3 nn = mk3((float)R.rect_n[0], (float)R.rect_n[1], (float)R.rect_n[2]);
      g.cosN = dot3(nn, sd);
      if(g.cosN <= 0.f) {
        g.flags |= PF_STAGE2 | PF_DIFFUSE;
      } else {
        g.dir = sd;
        g.flags |= PF_DIRECT | PF_IN_CONE;
      }
      break;
    }
    default: g.flags |= PF_DIRECT | PF_DIFFUSE; break;
  }
  g.rng = p.rng;
  return g;
}

/* Sensor sampling of realisation (pix, ireal): camera ray or flux probe,
 * wavelength, band and quadrature point (draw_map.c:51-107, 134-177,
 * 233-263, 348-384). */
__device__ __forceinline__ void
path_generate(Path& p, const DScene& S, const DRequest& R)
{
  const GenOut g = gen_sample(S, R, p.pix, p.ireal);
  p.w = 0.0;
  p.wdirect = 0.0;
  p.c_seg = p.c_node = p.c_tc = p.c_grid = 0;
  p.t0 = gtimer();
  p.rng = g.rng;
  p.chan = (uint8_t)g.chan;
  p.flags = g.flags;
  p.org = g.org;
  p.rdir = g.rdir;
  if(g.flags & PF_REJECTED) { p.state = ST_DONE; return; }
  p.wlen = (float)g.wlen;
  p.wlen_d = g.wlen;
  p.band = g.band;
  p.q = g.q;
  p.inv_pdf = g.inv_pdf;
  p.cosN = g.cosN;
  p.pos = g.org;
  p.dir = g.dir;
  p.state = ST_RAD_BEGIN;
}

struct ScatOut {
  Rng rng;
  float3 dnext, sdir;
  float R, refl, sun_ipdf;
  uint32_t flags;
};

/* SW scattering event at the site of a collision with the scattering
 * majorant (or at the ground): the next direction and the sun direction of
 * the next-event estimate with its phase/BRDF value
 * (htrdr_atmosphere_compute_radiance_sw.c:400-490).
 * Out of line: it runs once per scattering and holds the FP64 sun sampling. */
template <unsigned V>
__device__ __noinline__ ScatOut
sw_scatter(const DScene& S, Rng rng, float3 dir, float g, uint32_t flags, float refl,
           int site_cell, int site_layer, uint32_t band, uint32_t q, uint32_t gprim, float3 gN,
           double wlen_nm)
{
  ScatOut o;
  const float3 wo = neg3(dir);
  const bool surface = (flags & PF_SURFACE) != 0;
  float3 N = mk3(0.f, 0.f, 1.f);
  bool specular = false;
  int brdf_specular = 0;
  o.refl = refl;
  o.sdir = mk3(0.f, 0.f, 0.f);
  if(surface) {
    const SurfProps sp = surface_props<V>(S, rng, dir, gprim, gN, wlen_nm);
    N = sp.N;
    brdf_specular = sp.specular;
    if(dot3(N, wo) < 0.f) N = neg3(N);
    o.refl = sp.refl;
    if(sp.specular) {
      o.dnext = nrm3(add3(mul3(N, 2.f * dot3(N, wo)), neg3(wo)));
      specular = true;
    } else {
      const float u1 = rng.uf(), u2 = rng.uf();
      o.dnext = around(N, sqrtf(1.f - u2), u1);
    }
    flags &= ~PF_RAYLEIGH;
  } else {
    const double ks_gas = (double)site_k(S, site_cell, site_layer, band, q, HG_KS, 1);
    const double ks_par = (double)site_k(S, site_cell, site_layer, band, q, HG_KS, 2);
    const double ks = ks_par + ks_gas;
    const bool ray = (double)rng.uf() < ks_gas / ks;
    if(ray) flags |= PF_RAYLEIGH; else flags &= ~PF_RAYLEIGH;
    const float u1 = rng.uf(), u2 = rng.uf();
    o.dnext = around(dir, ray ? rayleigh_mu(u1) : hg_mu(g, u1), u2);
  }
  if(specular) flags |= PF_SPECULAR; else flags &= ~PF_SPECULAR;
  if(surface && specular) {
    if(!in_solar_cone(S, o.dnext)) o.R = 0.f;
    else { o.sdir = o.dnext; o.R = dot3(N, o.sdir) < 0.f ? 0.f : o.refl; }
    o.sun_ipdf = 1.f;
  } else {
    o.sdir = sun_sample(S, rng);
    o.sun_ipdf = (float)S.sun_solid_angle;
    if(surface) {
      const float c = dot3(N, o.sdir);
      o.R = c < 0.f ? 0.f : (brdf_specular ? 0.f : (c > 0.f ? o.refl / HG_PI_F : 0.f)) * c;
    } else {
      const float mu = dot3(dir, o.sdir);
      o.R = (flags & PF_RAYLEIGH) ? rayleigh_eval(mu) : hg_eval(g, mu);
    }
  }
  o.flags = flags;
  o.rng = rng;
  return o;
}

/* A path of a kind the kernel variant leaves out: a failed realisation */
__device__ __forceinline__ void
path_variant_miss(Path& p)
{
  p.flags |= PF_FAILED;
  p.state = ST_RAD_END;
}

/* Advance the state machine until the path needs a voxel step (ST_TRACE),
 * is done (ST_DONE) or idle.  V: the kernel variant (HV_* bits); the states
 * of a spectral kind it leaves out and, without HV_MESH, the mesh queries
 * are compiled out. */
/* Whether the ground of the scene is the plane (its hit record is then the
 * same at every query: no primitive, no edge, normal +z) */
template <unsigned V>
__device__ __forceinline__ bool
lw_plane_ground(const DScene& S)
{
  return !(V & HV_MESH) || !S.g_ntris;
}

/* LW walk after a scattering in the medium, over a plane ground: the new
 * direction from the phase function (..._lw.c:235) and the next free path
 * from the collision site, the head of the walk (..._lw.c:184-205) -- the
 * steps ST_LW_END and ST_LW_WALK take there.  It reads and writes the trace
 * part of the path only (the plane's hit record, set at the walk's first
 * ground query, stays the same) and returns the walk's new position and
 * direction, which the wavefront's trace stage stores into p.pos / p.dir:
 * the stage runs it without an event-stage visit.  The caller checks that
 * the bounce limit is not reached. */
__device__ __forceinline__ void
lw_scatter_plane(Path& p, const DScene& S, float3& pos, float3& dir)
{
  pos = madd3(p.tr.o, p.tr.d, p.tr.tcur);
  const float g = __ldg(S.optics + p.band).w;
  const float u1 = p.rng.uf(), u2 = p.rng.uf();
  dir = around(p.tr.d, hg_mu(g, u1), u2);
  p.flags &= ~PF_PREV_GROUND;
  ++p.bounces;
  p.gdist = ground_trace(S, pos, dir, 0.f, FLT_MAX, false);
  p.tr.Ts = p.rng.exp1();
  trace_begin(p, S, TK_LW, HG_KEXT, pos, dir, 0.f, p.gdist >= 0.f ? p.gdist : FLT_MAX, ST_LW_END);
}

template <unsigned V>
__device__ __forceinline__ void
path_event(Path& p, const DScene& S, const DRequest& R)
{
  for(;;) {
    switch(p.state) {
      case ST_GEN: path_generate(p, S, R); break;

      case ST_RAD_BEGIN: {
        p.g = __ldg(S.optics + p.band).w;
        p.flags &= ~(PF_PREV_GROUND | PF_TRACED);
        p.w = 0.0;
        p.ksi = 1.f;
        p.bounces = 0;
        if(p.flags & PF_LW) {
          if(V & HV_LW) p.state = ST_LW_WALK;
          else path_variant_miss(p);
          break;
        }
        if constexpr(!(V & HV_SW)) { path_variant_miss(p); break; }
        else {
        p.L_sun = planck_mono(p.wlen_d * 1e-9, S.sun_T);
        if((p.flags & PF_DIRECT) && ((p.flags & PF_IN_CONE) || in_solar_cone(S, p.dir))) {
          uint32_t hp;
          bool he;
          float3 hn;
          if(ground_query<V>(S, p.pos, p.dir, FLT_MAX, false, 0u, false, &hp, &he, &hn) < 0.f) {
            p.flags |= PF_TRACED;
            trace_begin(p, S, TK_TRANS, HG_KEXT, p.pos, p.dir, 0.f, FLT_MAX, ST_SW_DIRECT_END);
            return;
          }
        }
        p.state = ST_SW_DIRECT_END;
        break;
        }
      }

      case ST_SW_DIRECT_END:
        if constexpr(!(V & HV_SW)) { path_variant_miss(p); break; }
        else {
          if(p.flags & PF_TRACED) {
            const double Tr = p.tr.hit ? 0.0 : (p.tr.Tmin != 0.0 ? exp(-p.tr.Tmin) : 1.0);
            p.w = p.L_sun * Tr;
          }
          p.state = (p.flags & PF_DIFFUSE) ? ST_SW_WALK : ST_RAD_END;
        }
        break;

      case ST_SW_WALK: if constexpr(!(V & HV_SW)) { path_variant_miss(p); break; } else {
        if(++p.bounces > HG_MAX_BOUNCES) { p.flags |= PF_FAILED; p.state = ST_RAD_END; break; }
        {
          bool e;
          p.gdist = ground_query<V>(S, p.pos, p.dir, FLT_MAX, (p.flags & PF_PREV_GROUND) != 0,
                                 p.prev_prim, p.prev_edge != 0, &p.gprim, &e, &p.gN);
          p.gedge = e;
        }
        p.tr.Ts = p.rng.exp1();
        trace_begin(p, S, TK_SCATTER, HG_KS, p.pos, p.dir, 0.f,
                    p.gdist >= 0.f ? p.gdist : FLT_MAX, ST_SW_SCAT_END);
        return;
      }

      case ST_SW_SCAT_END: if constexpr(!(V & HV_SW)) { path_variant_miss(p); break; } else {
        if(p.tr.hit) { p.pnext = sw_scat_volume(p, S); return; } /* the trace origin is p.pos */
        if(p.gdist < 0.f) { p.state = ST_RAD_END; break; }
        /* the ground: scattering at the surface */
        const float tdst = p.gdist;
        p.pnext = madd3(p.pos, p.dir, tdst);
        p.flags |= PF_SURFACE | PF_PREV_GROUND;
        p.prev_prim = p.gprim;
        p.prev_edge = p.gedge;
        trace_begin(p, S, TK_TRANS, HG_KA, p.pos, p.dir, 0.f, tdst, ST_SW_ABS_END);
        return;
      }

      case ST_SW_ABS_END: if constexpr(!(V & HV_SW)) { path_variant_miss(p); break; } else {
        p.tr_abs = p.tr.hit ? 0.f : (float)(p.tr.Tmin != 0.0 ? exp(-p.tr.Tmin) : 1.0);
        if(p.tr_abs <= 0.f) { p.state = ST_RAD_END; break; }
        /* the collision site of the free path: the absorption trace keeps it */
        const ScatOut so = sw_scatter<V>(S, p.rng, p.dir, p.g, p.flags, p.refl, p.tr.site_cell,
                                      p.tr.site_layer, p.band, p.q, p.gprim, p.gN, p.wlen_d);
        p.rng = so.rng;
        p.flags = so.flags;
        p.dnext = so.dnext;
        p.sdir = so.sdir;
        p.R = so.R;
        p.refl = so.refl;
        p.sun_ipdf = so.sun_ipdf;
        uint32_t hp;
        bool he;
        float3 hn;
        if(p.R > 0.f
        && ground_query<V>(S, p.pnext, p.sdir, FLT_MAX, (p.flags & PF_PREV_GROUND) != 0, p.prev_prim,
                        p.prev_edge != 0, &hp, &he, &hn) < 0.f) {
          p.flags |= PF_TRACED;
          trace_begin(p, S, TK_TRANS, HG_KEXT, p.pnext, p.sdir, 0.f, FLT_MAX, ST_SW_NEE_END);
          return;
        }
        p.flags &= ~PF_TRACED;
        p.state = ST_SW_NEE_END;
        break;
      }

      case ST_SW_NEE_END: if constexpr(!(V & HV_SW)) { path_variant_miss(p); break; } else {
        double Tr = 0.0;
        if(p.flags & PF_TRACED) Tr = p.tr.hit ? 0.0 : (p.tr.Tmin != 0.0 ? exp(-p.tr.Tmin) : 1.0);
        p.flags &= ~PF_TRACED;
        p.ksi *= p.tr_abs;
        p.w += (double)p.ksi * p.L_sun * Tr * (double)p.R * (double)p.sun_ipdf;
        if((p.flags & PF_SURFACE) && p.rng.uf() >= p.refl) { p.state = ST_RAD_END; break; }
        p.pos = p.pnext;
        p.dir = p.dnext;
        p.state = ST_SW_WALK;
        break;
      }

      case ST_LW_WALK: if constexpr(!(V & HV_LW)) { path_variant_miss(p); break; } else {
        if(++p.bounces > HG_MAX_BOUNCES) { p.flags |= PF_FAILED; p.state = ST_RAD_END; break; }
        {
          bool e;
          p.gdist = ground_query<V>(S, p.pos, p.dir, FLT_MAX, (p.flags & PF_PREV_GROUND) != 0,
                                 p.prev_prim, p.prev_edge != 0, &p.gprim, &e, &p.gN);
          p.gedge = e;
        }
        p.tr.Ts = p.rng.exp1();
        trace_begin(p, S, TK_LW, HG_KEXT, p.pos, p.dir, 0.f,
                    p.gdist >= 0.f ? p.gdist : FLT_MAX, ST_LW_END);
        return;
      }

      case ST_LW_END: if constexpr(!(V & HV_LW)) { path_variant_miss(p); break; } else {
        /* the free path just traced started at p.tr.o along p.tr.d (the
         * walk's position and direction, which the trace stage may have
         * moved past p.pos / p.dir) */
        const bool svx = p.tr.hit != 0;
        const double wlen_m = p.wlen_d * 1e-9;
        if(p.gdist < 0.f && !svx) { p.w = 0.0; p.state = ST_RAD_END; break; }
        const float tdst = svx ? p.tr.tcur : p.gdist;
        p.pnext = madd3(p.pos, p.dir, tdst);
        if(svx && p.tr.event == 0) {
          const int l = p.tr.site_layer >= 0 ? p.tr.site_layer : layer_of(S, p.pnext.z);
          p.w = planck_mono(wlen_m, (double)__ldg(S.layer_T + l));
          p.state = ST_RAD_END;
          break;
        }
        if(svx) {
          const float u1 = p.rng.uf(), u2 = p.rng.uf();
          p.dnext = around(p.dir, hg_mu(p.g, u1), u2);
          p.flags &= ~PF_PREV_GROUND;
        } else {
          const SurfProps sp = surface_props<V>(S, p.rng, p.dir, p.gprim, p.gN, p.wlen_d);
          float3 N = sp.N;
          const float3 wo = neg3(p.dir);
          if(dot3(N, wo) < 0.f) N = neg3(N);
          if(sp.specular) {
            p.dnext = nrm3(add3(mul3(N, 2.f * dot3(N, wo)), neg3(wo)));
          } else {
            const float u1 = p.rng.uf(), u2 = p.rng.uf();
            p.dnext = around(N, sqrtf(1.f - u2), u1);
          }
          if(p.rng.uf() >= sp.refl) {
            const double T = (double)sp.T;
            p.w = T > 0 ? planck_mono(wlen_m, T) : 0.0;
            p.state = ST_RAD_END;
            break;
          }
          p.flags |= PF_PREV_GROUND;
          p.prev_prim = p.gprim;
          p.prev_edge = p.gedge;
        }
        p.pos = p.pnext;
        p.dir = p.dnext;
        p.state = ST_LW_WALK;
        break;
      }

      case ST_RAD_END:
        if((V & HV_SW) && R.mode == HG_FLUX_SW) {
          if(!(p.flags & PF_STAGE2)) {
            p.wdirect = p.w;
            p.flags = (p.flags & ~(PF_DIRECT | PF_IN_CONE)) | PF_STAGE2 | PF_DIFFUSE;
            p.pos = p.org;
            p.dir = p.rdir;
            p.state = ST_RAD_BEGIN;
            break;
          }
          p.weight = ((double)p.cosN * S.sun_solid_angle * p.wdirect + HG_PI_D * p.w) * p.inv_pdf;
        } else {
          p.weight = p.w * p.inv_pdf;
        }
        p.state = ST_DONE;
        return;

      default: /* ST_TRACE, ST_DONE, ST_IDLE */
        return;
    }
  }
}

}  // namespace

#endif /* HTRDR_TRANSPORT_CUH */
