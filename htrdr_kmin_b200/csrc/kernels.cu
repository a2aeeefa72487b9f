/* CUDA kernels of the plain drop-in path and of the bit-exact checks.
 *
 * k_plain: one thread per realisation (the plain GPU drop-in of
 * htrdr_draw_map, src/core/htrdr_draw_map.c:270-491).  Thread i handles
 * realisation i / npix of pixel i % npix, so the 32 lanes of a warp trace
 * neighbouring pixels and accumulate into distinct FP64 accumulators. */
#include "internal.h"
#include "transport.cuh"

namespace hg {

template <unsigned V>
__device__ __forceinline__ void
run_path(Path& p, const DScene& S, const DRequest& R)
{
  for(;;) {
    if(p.state == ST_TRACE) trace_step<V>(p, S);
    else if(p.state == ST_DONE) return;
    else path_event<V>(p, S, R);
  }
}

/* Add one realisation to its pixel (src/atmosphere/htrdr_atmosphere_draw_map.c:190-198) */
__device__ __forceinline__ void
accumulate(const Path& p, const DRequest& R, DAccum* acc, DAccum* tacc)
{
  if(p.flags & PF_REJECTED) return;
  const uint32_t nch = R.mode == HG_IMAGE_CIE ? 3u : 1u;
  DAccum* a = R.acc + (size_t)p.pix * nch + p.chan;
  if(p.flags & PF_FAILED) { atomicAdd(&a->pad, 1ull); return; }
  atomicAdd(&a->s, p.weight);
  atomicAdd(&a->s2, p.weight * p.weight);
  atomicAdd(&a->n, 1ull);
  const double us = (double)(gtimer() - p.t0) * 1e-3;
  DAccum* t = R.tacc + p.pix;
  atomicAdd(&t->s, us);
  atomicAdd(&t->s2, us * us);
  atomicAdd(&t->n, 1ull);
}

__device__ __forceinline__ void
flush_counters(Counters* cnt, unsigned long long seg, unsigned long long node,
               unsigned long long tc, unsigned long long real, unsigned long long fail)
{
  if(!cnt) return;
  for(int o = 16; o > 0; o >>= 1) {
    seg += __shfl_down_sync(0xffffffffu, seg, o);
    node += __shfl_down_sync(0xffffffffu, node, o);
    tc += __shfl_down_sync(0xffffffffu, tc, o);
    real += __shfl_down_sync(0xffffffffu, real, o);
    fail += __shfl_down_sync(0xffffffffu, fail, o);
  }
  if((threadIdx.x & 31) == 0) {
    atomicAdd(&cnt->seg, seg);
    atomicAdd(&cnt->node, node);
    atomicAdd(&cnt->tc, tc);
    atomicAdd(&cnt->real, real);
    atomicAdd(&cnt->fail, fail);
  }
}

template <unsigned V>
__global__ void __maxnreg__(HG_PLAIN_MAXNREG)
k_plain(DScene S, DRequest R, DAccum* acc, DAccum* tacc, uint64_t pix_begin, uint32_t npix,
        double* weights, Counters* cnt)
{
  const uint64_t idx = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const uint64_t total = (uint64_t)npix * R.nreal_pp;
  unsigned long long seg = 0, node = 0, tc = 0, real = 0, fail = 0;
  if(idx < total) {
    Path p;
    p.ireal = (uint32_t)(idx / npix);
    p.pix = (uint32_t)(pix_begin + idx % npix);
    p.state = ST_GEN;
    p.flags = 0;
    run_path<V>(p, S, R);
    if(weights) {
      weights[(idx % npix) * R.nreal_pp + p.ireal] =
        (p.flags & (PF_REJECTED | PF_FAILED)) ? __longlong_as_double(0x7ff8000000000000ll) : p.weight;
    } else {
      accumulate(p, R, acc, tacc);
    }
    seg = p.c_seg; node = p.c_node; tc = p.c_tc;
    if(cnt && p.c_grid) atomicAdd(&cnt->grid, (unsigned long long)p.c_grid);
    real = (p.flags & (PF_REJECTED | PF_FAILED)) ? 0 : 1;
    fail = (p.flags & PF_FAILED) ? 1 : 0;
  }
  flush_counters(cnt, seg, node, tc, real, fail);
}

/*******************************************************************************
 * Pixel write-back (htrdr_accum_get_estimation, src/core/htrdr_accum.h:48-68,
 * and the brightness temperature of draw_map.c:425-435 /
 * src/core/htrdr_spectral.c:31-121)
 ******************************************************************************/
__device__ __forceinline__ void
estimate(const DAccum& a, double& E, double& SE)
{
  if(!a.n) { E = 0; SE = 0; return; }
  const double N = (double)a.n;
  E = a.s / N;
  const double V = fmax(a.s2 / N - E * E, 0.0);
  SE = sqrt(V / N);
}

__device__ double
planck_any(double l0, double l1, double T)
{
  return l0 == l1 ? planck_mono(l0, T) : planck_interval(l0, l1, T);
}

__device__ double
radiance_temperature(double l0, double l1, double radiance)
{
  double avg = radiance;
  if(l0 != l1) avg /= (l1 - l0);
  const double eps_T = 1e-4, eps_B = avg * 1e-8;
  double T = 0, T0 = 0, T1 = 0, T2 = 200, B0 = 0;
  int i;
  for(i = 0; i < 100; ++i) {
    if(planck_any(l0, l1, T2) >= avg) break;
    T2 *= 2;
  }
  if(i >= 100) return 0;
  for(i = 0; i < 100; ++i) {
    T = (T1 + T2) * 0.5;
    const double B = planck_any(l0, l1, T);
    if(B < avg) T1 = T; else T2 = T;
    if(fabs(T - T0) < eps_T || fabs(B - B0) < eps_B) break;
    T0 = T;
    B0 = B;
  }
  if(i >= 100) return 0;
  return T;
}

__global__ void
k_finalize(DRequest R, const DAccum* acc, const DAccum* tacc, char* out, size_t pitch)
{
  const uint32_t pix = blockIdx.x * blockDim.x + threadIdx.x;
  if(pix >= R.width * R.height) return;
  const uint32_t x = pix % R.width, y = pix / R.width;
  const DAccum t = R.tacc[pix];
  const DAccum* ap = R.acc;
  double* o = (double*)(out + (size_t)y * pitch + (size_t)x * (R.mode == HG_IMAGE_CIE ? 80 : 64));
  unsigned long long* ou = (unsigned long long*)o;
  if(R.mode == HG_FLUX_SW || R.mode == HG_FLUX_LW) {
    const DAccum a = ap[pix];
    o[0] = a.s; o[1] = a.s2; ou[2] = a.n; ou[3] = a.pad;
    o[4] = t.s; o[5] = t.s2; ou[6] = t.n; ou[7] = 0;
  } else if(R.mode == HG_IMAGE_CIE) {
    for(int c = 0; c < 3; ++c) estimate(ap[(size_t)pix * 3 + c], o[2 * c], o[2 * c + 1]);
    o[6] = t.s; o[7] = t.s2; ou[8] = t.n; ou[9] = 0;
  } else {
    double E, SE;
    estimate(ap[pix], E, SE);
    o[0] = E; o[1] = SE; o[2] = 0; o[3] = 0;
    if(R.mode == HG_XWAVE_LW) {
      const double l0 = R.wlen_range[0] * 1e-9, l1 = R.wlen_range[1] * 1e-9;
      o[2] = radiance_temperature(l0, l1, E);
      o[3] = radiance_temperature(l0, l1, E + SE) - radiance_temperature(l0, l1, E - SE);
    }
    o[4] = t.s; o[5] = t.s2; ou[6] = t.n; ou[7] = 0;
  }
}

/*******************************************************************************
 * Batched radiance (atmosphere_compute_radiance_sw/_lw with one stream per ray)
 ******************************************************************************/
template <unsigned V>
__global__ void __launch_bounds__(128)
k_radiance(DScene S, int lw, size_t n, const double* pos, const double* dir, const double* wlen,
           const uint32_t* band, const uint32_t* iquad, int mask, uint32_t seed, double* out)
{
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if(i >= n) return;
  DRequest R;
  R.mode = lw ? HG_RAD_LW : HG_RAD_SW;
  Path p;
  p.rng.init((uint32_t)i, seed, 0u, 0u);
  p.pos = mk3((float)pos[3 * i], (float)pos[3 * i + 1], (float)pos[3 * i + 2]);
  p.dir = mk3((float)dir[3 * i], (float)dir[3 * i + 1], (float)dir[3 * i + 2]);
  p.org = p.pos;
  p.rdir = p.dir;
  p.wlen_d = wlen[i];
  p.wlen = (float)wlen[i];
  p.band = band[i];
  p.q = S.quad_off[band[i]] + iquad[i];
  p.inv_pdf = 1.0;
  p.flags = lw ? PF_LW : (((mask & 1) ? PF_DIRECT : 0u) | ((mask & 2) ? PF_DIFFUSE : 0u));
  p.c_seg = p.c_node = p.c_tc = 0;
  p.state = ST_RAD_BEGIN;
  run_path<V>(p, S, R);
  out[i] = (p.flags & PF_FAILED) ? __longlong_as_double(0x7ff8000000000000ll) : p.weight;
}

/*******************************************************************************
 * Integer checks
 ******************************************************************************/
__global__ void
k_find_band(DScene S, size_t n, const double* wlen, uint32_t* out)
{
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if(i < n) out[i] = find_band(S, wlen[i]);
}

__global__ void
k_sample_quad(DScene S, size_t n, const double* r, const uint32_t* band, uint32_t* out)
{
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if(i < n) out[i] = band[i] < S.nbands ? sample_quad(S, r[i], band[i]) : 0xFFFFFFFFu;
}

__global__ void
k_ground_trace(DScene S, size_t n, const float* rays, const float* tmax, const uint32_t* from_prim,
               const uint8_t* from_edge, uint32_t* prim, float* dist)
{
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if(i >= n) return;
  const float3 o = make_float3(rays[6 * i], rays[6 * i + 1], rays[6 * i + 2]);
  const float3 d = make_float3(rays[6 * i + 3], rays[6 * i + 4], rays[6 * i + 5]);
  const GHit h = g_trace(S, o, d, 0.f, tmax[i], from_prim[i], from_edge[i] != 0);
  prim[i] = h.prim;
  dist[i] = h.prim == HG_NO_PRIM ? -1.f : h.dist;
}

__global__ void
k_locate_leaf(DScene S, uint32_t q, int prop, size_t n, const uint32_t* cells, uint32_t* node,
              uint32_t* level)
{
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if(i >= n) return;
  const uint32_t c0 = cells[3 * i], c1 = cells[3 * i + 1], c2 = cells[3 * i + 2];
  if(c0 >= S.def[0] || c1 >= S.def[1] || c2 >= S.def[2]) { node[i] = HG_LEAF; level[i] = HG_LEAF; return; }
  const uint4* nodes = S.nodes + S.tree_base[(size_t)q * 3 + prop];
  uint32_t nd = 0, L = S.depth;
  uint4 v = nodes[0];
  while(v.z != HG_LEAF) {
    --L;
    const uint32_t oct = ((c0 >> L) & 1u) | (((c1 >> L) & 1u) << 1) | (((c2 >> L) & 1u) << 2);
    nd = v.z + oct;
    v = nodes[nd];
  }
  node[i] = nd;
  level[i] = L;
}

__global__ void
k_sample_wavelength(DRequest R, int channel, size_t n, const double* r0, const double* r1,
                    uint32_t* cb, double* wlen, double* pdf)
{
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if(i >= n) return;
  double p;
  uint32_t b;
  wlen[i] = sample_wavelength(R, channel, r0[i], r1[i], &p, &b);
  pdf[i] = p;
  cb[i] = b;
}

/*******************************************************************************
 * Launchers
 ******************************************************************************/
static inline unsigned
nblocks(uint64_t n, unsigned bs) { return (unsigned)((n + bs - 1) / bs); }

using PlainFn = void (*)(DScene, DRequest, DAccum*, DAccum*, uint64_t, uint32_t, double*, Counters*);
static PlainFn
plain_fn(uint32_t v)
{
  HG_PICK_VARIANT(v, k_plain)
}

using RadianceFn = void (*)(DScene, int, size_t, const double*, const double*, const double*,
                            const uint32_t*, const uint32_t*, int, uint32_t, double*);
static RadianceFn
radiance_fn(uint32_t v)
{
  switch(v) {
    case HV_SW: return k_radiance<HV_SW>;
    case HV_SW | HV_MESH: return k_radiance<HV_SW | HV_MESH>;
    case HV_LW: return k_radiance<HV_LW>;
    default: return k_radiance<HV_LW | HV_MESH>;
  }
}

cudaError_t
launch_plain(const DScene& S, const DRequest& R, DAccum* acc, DAccum* tacc, uint64_t pix_begin,
             uint32_t npix, double* weights, void* counters, cudaStream_t st)
{
  const uint64_t total = (uint64_t)npix * R.nreal_pp;
  if(!total) return cudaSuccess;
  DRequest Ra = R;
  Ra.acc = acc;
  Ra.tacc = tacc;
  auto kern = plain_fn(hv_make(S.g_ntris != 0, hv_kind(R.mode)));
  kern<<<nblocks(total, 128), 128, 0, st>>>(S, Ra, acc, tacc, pix_begin, npix, weights,
                                            (Counters*)counters);
  note_launches(1);
  return cudaGetLastError();
}

cudaError_t
launch_finalize(const DRequest& R, const DAccum* acc, const DAccum* tacc, void* out, size_t pitch,
                cudaStream_t st)
{
  const uint32_t npix = R.width * R.height;
  DRequest Ra = R;
  if(acc) Ra.acc = (DAccum*)acc;
  if(tacc) Ra.tacc = (DAccum*)tacc;
  k_finalize<<<nblocks(npix, 128), 128, 0, st>>>(Ra, acc, tacc, (char*)out, pitch);
  note_launches(1);
  return cudaGetLastError();
}

cudaError_t
launch_radiance(const DScene& S, int lw, size_t n, const double* pos, const double* dir,
                const double* wlen, const uint32_t* band, const uint32_t* iquad, int mask,
                uint32_t seed, double* out, cudaStream_t st)
{
  if(!n) return cudaSuccess;
  auto kern = radiance_fn(hv_make(S.g_ntris != 0, lw ? HV_LW : HV_SW));
  kern<<<nblocks(n, 128), 128, 0, st>>>(S, lw, n, pos, dir, wlen, band, iquad, mask, seed, out);
  return cudaGetLastError();
}

cudaError_t
launch_find_band(const DScene& S, size_t n, const double* wlen, uint32_t* out, cudaStream_t st)
{
  if(!n) return cudaSuccess;
  k_find_band<<<nblocks(n, 256), 256, 0, st>>>(S, n, wlen, out);
  return cudaGetLastError();
}

cudaError_t
launch_sample_quad(const DScene& S, size_t n, const double* r, const uint32_t* band,
                   uint32_t* out, cudaStream_t st)
{
  if(!n) return cudaSuccess;
  k_sample_quad<<<nblocks(n, 256), 256, 0, st>>>(S, n, r, band, out);
  return cudaGetLastError();
}

cudaError_t
launch_ground_trace(const DScene& S, size_t n, const float* rays, const float* tmax,
                    const uint32_t* from_prim, const uint8_t* from_edge, uint32_t* prim, float* dist,
                    cudaStream_t st)
{
  if(!n) return cudaSuccess;
  k_ground_trace<<<nblocks(n, 128), 128, 0, st>>>(S, n, rays, tmax, from_prim, from_edge, prim, dist);
  return cudaGetLastError();
}

cudaError_t
launch_locate_leaf(const DScene& S, uint32_t q, int prop, size_t n, const uint32_t* cells,
                   uint32_t* node, uint32_t* level, cudaStream_t st)
{
  if(!n) return cudaSuccess;
  k_locate_leaf<<<nblocks(n, 256), 256, 0, st>>>(S, q, prop, n, cells, node, level);
  return cudaGetLastError();
}

cudaError_t
launch_sample_wavelength(const DRequest& R, int channel, size_t n, const double* r0,
                         const double* r1, uint32_t* cb, double* wlen, double* pdf,
                         cudaStream_t st)
{
  if(!n) return cudaSuccess;
  k_sample_wavelength<<<nblocks(n, 256), 256, 0, st>>>(R, channel, n, r0, r1, cb, wlen, pdf);
  return cudaGetLastError();
}

}  // namespace hg
