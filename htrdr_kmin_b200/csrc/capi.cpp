/* C ABI entry points of the drop-in draw_map path (both engines) and of the checks. */
#include "internal.h"

#include <cmath>
#include <cstring>

using namespace hg;

namespace {

struct Workspace {
  DevBuf acc, out, cnt, tables;
  size_t acc_bytes = 0, out_bytes = 0;
};

/* Grow-only device scratch of a scene (one call at a time per scene) */
Workspace&
workspace(htrdr_gpu_scene* scn)
{
  static thread_local std::map<htrdr_gpu_scene*, std::unique_ptr<Workspace>> ws;
  auto& w = ws[scn];
  if(!w) w = std::make_unique<Workspace>();
  return *w;
}

bool
ensure(DevBuf& b, size_t bytes)
{
  if(b.bytes >= bytes && b.ptr) return true;
  if(b.ptr) { cudaFree(b.ptr); b.ptr = nullptr; b.bytes = 0; }
  return b.alloc(bytes);
}

/* One map on the scene's engine.  `user_acc' (device memory) set: the FP64
 * accumulators are left there and no pixel struct is written (`layout' and
 * `buffer' unused); else they live in the scene's workspace and the map is
 * finalized into `buffer' (host or device memory). */
htrdr_gpu_res_T
draw_map_impl(htrdr_gpu_scene* scn, const htrdr_gpu_request* req,
              const htrdr_gpu_buffer_layout* layout, void* buffer, bool host,
              htrdr_gpu_stats* stats, DAccum* user_acc = nullptr)
{
  if(!scn || (!buffer && !user_acc)) return HTRDR_GPU_RES_BAD_ARG;
  htrdr_gpu_res_T res = user_acc ? HTRDR_GPU_RES_OK : check_layout(req, layout);
  if(res != HTRDR_GPU_RES_OK) return res;
  if(user_acc && (!req || req->mode < 0 || req->mode > 4 || !req->width || !req->height))
    return HTRDR_GPU_RES_BAD_ARG;
  if(!cuda_ok(cudaSetDevice(scn->device), "cudaSetDevice")) return HTRDR_GPU_RES_BAD_OP;
  DRequest R;
  res = make_drequest(scn, req, &R);
  if(res != HTRDR_GPU_RES_OK) return res;
  take_launches();
  const uint32_t npix = req->width * req->height;
  const uint32_t nch = req->mode == HG_IMAGE_CIE ? 3u : 1u;
  const size_t acc_bytes = (size_t)npix * (nch + 1) * sizeof(DAccum);
  const size_t out_bytes = user_acc ? 0 : layout->pitch * layout->height;
  Workspace& ws = workspace(scn);
  const bool plain = scn->engine_set && scn->engine == HTRDR_GPU_ENGINE_PLAIN;
  if((!user_acc && !ensure(ws.acc, acc_bytes)) || !ensure(ws.cnt, 128)) return HTRDR_GPU_RES_MEM_ERR;
  if(!plain && !ensure(ws.tables, single_tables_bytes())) return HTRDR_GPU_RES_MEM_ERR;
  if(host && !ensure(ws.out, out_bytes)) return HTRDR_GPU_RES_MEM_ERR;
  DAccum* acc = user_acc ? user_acc : (DAccum*)ws.acc.ptr;
  DAccum* tacc = acc + (size_t)npix * nch;
  void* dout = host ? ws.out.ptr : buffer;
  htrdr_gpu_tuning tun;
  if(scn->has_tuning) tun = scn->tuning;
  else htrdr_gpu_mode_tuning(req->mode, &tun);
  if(scn->engine_set && !plain) tun.engine = (uint32_t)scn->engine;
  cudaStream_t st = scn->stream;
  cudaEvent_t e0, e1, e2, e3;
  cudaEventCreate(&e0); cudaEventCreate(&e1); cudaEventCreate(&e2); cudaEventCreate(&e3);
  bool ok = true;
  cudaEventRecord(e0, st);
  ok = ok && cuda_ok(cudaMemsetAsync(acc, 0, acc_bytes, st), "cudaMemsetAsync");
  ok = ok && cuda_ok(cudaMemsetAsync(ws.cnt.ptr, 0, 128, st), "cudaMemsetAsync");
  cudaEventRecord(e1, st);
  if(plain) {
    ok = ok && cuda_ok(launch_plain(scn->d, R, acc, tacc, 0, npix, nullptr, ws.cnt.ptr, st), "k_plain");
  } else {
    R.acc = acc;
    R.tacc = tacc;
    ok = ok && cuda_ok(launch_workqueue_single(scn->d, R, ws.tables.ptr, ws.cnt.ptr, tun,
                                               &thread_wave(scn->device),
                                               scn->device, st),
                       tun.engine == HTRDR_GPU_ENGINE_WAVEFRONT ? "wavefront" : "k_persistent");
  }
  cudaEventRecord(e2, st);
  if(!user_acc)
    ok = ok && cuda_ok(launch_finalize(R, acc, tacc, dout, layout->pitch, st), "k_finalize");
  if(ok && host)
    ok = cuda_ok(cudaMemcpyAsync(buffer, dout, out_bytes, cudaMemcpyDeviceToHost, st), "D2H");
  cudaEventRecord(e3, st);
  unsigned long long c[6] = {0, 0, 0, 0, 0, 0};
  if(ok) ok = cuda_ok(cudaMemcpyAsync(c, ws.cnt.ptr, sizeof(c), cudaMemcpyDeviceToHost, st), "D2H");
  if(ok) ok = cuda_ok(cudaStreamSynchronize(st), "cudaStreamSynchronize");
  if(ok && stats) {
    float k = 0, t = 0;
    cudaEventElapsedTime(&k, e1, e2);
    cudaEventElapsedTime(&t, e0, e3);
    stats->segments = c[0]; stats->nodes = c[1]; stats->collisions = c[2];
    stats->realisations = c[3]; stats->failures = c[4]; stats->grid_bytes = c[5];
    stats->kernel_ms = k; stats->total_ms = t;
    stats->launches = take_launches();
  }
  cudaEventDestroy(e0); cudaEventDestroy(e1); cudaEventDestroy(e2); cudaEventDestroy(e3);
  return ok ? HTRDR_GPU_RES_OK : HTRDR_GPU_RES_UNKNOWN_ERR;
}

/* RAII device copy of a host array */
template<typename T>
struct DevArr {
  DevBuf b;
  bool from(const T* h, size_t n) { return b.upload(h, n * sizeof(T)); }
  bool make(size_t n) { return b.alloc(n * sizeof(T)); }
  T* p() const { return (T*)b.ptr; }
  bool to(T* h, size_t n) const { return cuda_ok(cudaMemcpy(h, b.ptr, n * sizeof(T), cudaMemcpyDeviceToHost), "D2H"); }
};

}  // namespace

extern "C" HTRDR_GPU_API htrdr_gpu_res_T
htrdr_gpu_scene_set_engine(htrdr_gpu_scene* scn, int engine, const htrdr_gpu_tuning* tuning)
try {
  if(!scn) return HTRDR_GPU_RES_BAD_ARG;
  if(engine != HTRDR_GPU_ENGINE_PERSISTENT && engine != HTRDR_GPU_ENGINE_PLAIN
  && engine != HTRDR_GPU_ENGINE_WAVEFRONT && engine != HTRDR_GPU_ENGINE_SORTED)
    return HTRDR_GPU_RES_BAD_ARG;
  if(tuning) {
    htrdr_gpu_tuning t = *tuning;
    if(engine != HTRDR_GPU_ENGINE_PLAIN) t.engine = (uint32_t)engine;
    if(!valid_tuning(t)) return HTRDR_GPU_RES_BAD_ARG;
  }
  scn->engine = engine;
  scn->engine_set = 1;
  scn->has_tuning = tuning != nullptr;
  if(tuning) scn->tuning = *tuning;
  return HTRDR_GPU_RES_OK;
}
HG_API_CATCH("htrdr_gpu_scene_set_engine")

extern "C" HTRDR_GPU_API htrdr_gpu_res_T
htrdr_gpu_draw_map(htrdr_gpu_scene* scn, const htrdr_gpu_request* req,
                   const htrdr_gpu_buffer_layout* layout, void* buffer, htrdr_gpu_stats* stats)
try {
  return draw_map_impl(scn, req, layout, buffer, true, stats);
}
HG_API_CATCH("htrdr_gpu_draw_map")

extern "C" HTRDR_GPU_API htrdr_gpu_res_T
htrdr_gpu_draw_map_device(htrdr_gpu_scene* scn, const htrdr_gpu_request* req,
                          const htrdr_gpu_buffer_layout* layout, void* device_buffer,
                          htrdr_gpu_stats* stats)
try {
  return draw_map_impl(scn, req, layout, device_buffer, false, stats);
}
HG_API_CATCH("htrdr_gpu_draw_map_device")

extern "C" HTRDR_GPU_API htrdr_gpu_res_T
htrdr_gpu_draw_map_accum_device(htrdr_gpu_scene* scn, const htrdr_gpu_request* req,
                                void* device_accum, htrdr_gpu_stats* stats)
try {
  if(!device_accum) return HTRDR_GPU_RES_BAD_ARG;
  return draw_map_impl(scn, req, nullptr, nullptr, false, stats, (DAccum*)device_accum);
}
HG_API_CATCH("htrdr_gpu_draw_map_accum_device")

extern "C" HTRDR_GPU_API htrdr_gpu_res_T
htrdr_gpu_finalize_device(htrdr_gpu_scene* scn, const htrdr_gpu_request* req,
                          const void* device_accum, const htrdr_gpu_buffer_layout* layout,
                          void* device_buffer)
try {
  if(!scn || !device_accum || !device_buffer) return HTRDR_GPU_RES_BAD_ARG;
  htrdr_gpu_res_T res = check_layout(req, layout);
  if(res != HTRDR_GPU_RES_OK) return res;
  if(!cuda_ok(cudaSetDevice(scn->device), "cudaSetDevice")) return HTRDR_GPU_RES_BAD_OP;
  DRequest R;
  res = make_drequest(scn, req, &R);
  if(res != HTRDR_GPU_RES_OK) return res;
  const uint32_t nch = req->mode == HG_IMAGE_CIE ? 3u : 1u;
  const DAccum* acc = (const DAccum*)device_accum;
  const DAccum* tacc = acc + (size_t)req->width * req->height * nch;
  cudaStream_t st = scn->stream;
  const bool ok = cuda_ok(launch_finalize(R, acc, tacc, device_buffer, layout->pitch, st), "k_finalize")
               && cuda_ok(cudaStreamSynchronize(st), "cudaStreamSynchronize");
  return ok ? HTRDR_GPU_RES_OK : HTRDR_GPU_RES_UNKNOWN_ERR;
}
HG_API_CATCH("htrdr_gpu_finalize_device")

static htrdr_gpu_res_T
radiance_impl(htrdr_gpu_scene* scn, int lw, size_t n, const double* pos, const double* dir,
              const double* wlen, const uint32_t* iband, const uint32_t* iquad, int mask,
              uint32_t seed, double* out)
{
  if(!scn || (n && (!pos || !dir || !wlen || !iband || !iquad || !out))) return HTRDR_GPU_RES_BAD_ARG;
  for(size_t i = 0; i < n; ++i)
    if(iband[i] >= scn->nbands || iquad[i] >= scn->nquads[iband[i]]) return HTRDR_GPU_RES_BAD_ARG;
  if(scn->d.has_cloud) {
    const uint32_t need = lw ? (1u << HG_KEXT) : 7u;
    if((scn->props_mask & need) != need) return HTRDR_GPU_RES_BAD_ARG;
  }
  if(!n) return HTRDR_GPU_RES_OK;
  if(!cuda_ok(cudaSetDevice(scn->device), "cudaSetDevice")) return HTRDR_GPU_RES_BAD_OP;
  DevArr<double> dp, dd, dw, dout;
  DevArr<uint32_t> db, dq;
  if(!dp.from(pos, 3 * n) || !dd.from(dir, 3 * n) || !dw.from(wlen, n) || !db.from(iband, n)
  || !dq.from(iquad, n) || !dout.make(n))
    return HTRDR_GPU_RES_MEM_ERR;
  if(!cuda_ok(launch_radiance(scn->d, lw, n, dp.p(), dd.p(), dw.p(), db.p(), dq.p(), mask, seed,
                              dout.p(), scn->stream), "k_radiance")
  || !cuda_ok(cudaStreamSynchronize(scn->stream), "sync") || !dout.to(out, n))
    return HTRDR_GPU_RES_UNKNOWN_ERR;
  return HTRDR_GPU_RES_OK;
}

extern "C" HTRDR_GPU_API htrdr_gpu_res_T
htrdr_gpu_radiance_sw(htrdr_gpu_scene* scn, size_t n, const double* pos, const double* dir,
                      const double* wlen, const uint32_t* iband, const uint32_t* iquad,
                      int cpnt_mask, uint32_t seed, double* out)
try {
  return radiance_impl(scn, 0, n, pos, dir, wlen, iband, iquad, cpnt_mask, seed, out);
}
HG_API_CATCH("htrdr_gpu_radiance_sw")

extern "C" HTRDR_GPU_API htrdr_gpu_res_T
htrdr_gpu_radiance_lw(htrdr_gpu_scene* scn, size_t n, const double* pos, const double* dir,
                      const double* wlen, const uint32_t* iband, const uint32_t* iquad,
                      uint32_t seed, double* out)
try {
  return radiance_impl(scn, 1, n, pos, dir, wlen, iband, iquad, 0, seed, out);
}
HG_API_CATCH("htrdr_gpu_radiance_lw")

extern "C" HTRDR_GPU_API htrdr_gpu_res_T
htrdr_gpu_realisation_weights(htrdr_gpu_scene* scn, const htrdr_gpu_request* req,
                              size_t pix_begin, size_t pix_end, double* weights)
try {
  if(!scn || !req || !weights || pix_end < pix_begin) return HTRDR_GPU_RES_BAD_ARG;
  if(pix_end > (size_t)req->width * req->height) return HTRDR_GPU_RES_BAD_ARG;
  if(!cuda_ok(cudaSetDevice(scn->device), "cudaSetDevice")) return HTRDR_GPU_RES_BAD_OP;
  DRequest R;
  htrdr_gpu_res_T res = make_drequest(scn, req, &R);
  if(res != HTRDR_GPU_RES_OK) return res;
  const size_t np = pix_end - pix_begin;
  if(!np) return HTRDR_GPU_RES_OK;
  DevArr<double> dw;
  if(!dw.make(np * R.nreal_pp)) return HTRDR_GPU_RES_MEM_ERR;
  if(!cuda_ok(launch_plain(scn->d, R, nullptr, nullptr, pix_begin, (uint32_t)np, dw.p(), nullptr,
                           scn->stream), "k_plain")
  || !cuda_ok(cudaStreamSynchronize(scn->stream), "sync") || !dw.to(weights, np * R.nreal_pp))
    return HTRDR_GPU_RES_UNKNOWN_ERR;
  return HTRDR_GPU_RES_OK;
}
HG_API_CATCH("htrdr_gpu_realisation_weights")

extern "C" HTRDR_GPU_API htrdr_gpu_res_T
htrdr_gpu_find_band(htrdr_gpu_scene* scn, size_t n, const double* wlen, uint32_t* out)
try {
  if(!scn || (n && (!wlen || !out))) return HTRDR_GPU_RES_BAD_ARG;
  if(!n) return HTRDR_GPU_RES_OK;
  cudaSetDevice(scn->device);
  DevArr<double> dw;
  DevArr<uint32_t> dout;
  if(!dw.from(wlen, n) || !dout.make(n)) return HTRDR_GPU_RES_MEM_ERR;
  if(!cuda_ok(launch_find_band(scn->d, n, dw.p(), dout.p(), scn->stream), "k_find_band")
  || !cuda_ok(cudaStreamSynchronize(scn->stream), "sync") || !dout.to(out, n))
    return HTRDR_GPU_RES_UNKNOWN_ERR;
  return HTRDR_GPU_RES_OK;
}
HG_API_CATCH("htrdr_gpu_find_band")

extern "C" HTRDR_GPU_API htrdr_gpu_res_T
htrdr_gpu_sample_quad(htrdr_gpu_scene* scn, size_t n, const double* r, const uint32_t* iband,
                      uint32_t* out)
try {
  if(!scn || (n && (!r || !iband || !out))) return HTRDR_GPU_RES_BAD_ARG;
  if(!n) return HTRDR_GPU_RES_OK;
  cudaSetDevice(scn->device);
  DevArr<double> dr;
  DevArr<uint32_t> db, dout;
  if(!dr.from(r, n) || !db.from(iband, n) || !dout.make(n)) return HTRDR_GPU_RES_MEM_ERR;
  if(!cuda_ok(launch_sample_quad(scn->d, n, dr.p(), db.p(), dout.p(), scn->stream), "k_sample_quad")
  || !cuda_ok(cudaStreamSynchronize(scn->stream), "sync") || !dout.to(out, n))
    return HTRDR_GPU_RES_UNKNOWN_ERR;
  return HTRDR_GPU_RES_OK;
}
HG_API_CATCH("htrdr_gpu_sample_quad")

extern "C" HTRDR_GPU_API htrdr_gpu_res_T
htrdr_gpu_locate_leaf(htrdr_gpu_scene* scn, uint32_t iband, uint32_t iquad, int prop, size_t n,
                      const uint32_t* cells, uint32_t* node, uint32_t* level)
try {
  if(!scn || !scn->d.has_cloud || iband >= scn->nbands || iquad >= scn->nquads[iband]
  || prop < 0 || prop > 2 || !(scn->props_mask & (1u << prop)))
    return HTRDR_GPU_RES_BAD_ARG;
  if(!n) return HTRDR_GPU_RES_OK;
  cudaSetDevice(scn->device);
  DevArr<uint32_t> dc, dn, dl;
  if(!dc.from(cells, 3 * n) || !dn.make(n) || !dl.make(n)) return HTRDR_GPU_RES_MEM_ERR;
  if(!cuda_ok(launch_locate_leaf(scn->d, scn->quad_off[iband] + iquad, prop, n, dc.p(), dn.p(),
                                 dl.p(), scn->stream), "k_locate_leaf")
  || !cuda_ok(cudaStreamSynchronize(scn->stream), "sync") || !dn.to(node, n) || !dl.to(level, n))
    return HTRDR_GPU_RES_UNKNOWN_ERR;
  return HTRDR_GPU_RES_OK;
}
HG_API_CATCH("htrdr_gpu_locate_leaf")

extern "C" HTRDR_GPU_API htrdr_gpu_res_T
htrdr_gpu_ground_trace(htrdr_gpu_scene* scn, size_t n, const float* rays, const float* tmax,
                       const uint32_t* from_prim, const uint8_t* from_edge, uint32_t* prim,
                       float* dist)
try {
  if(!scn || !scn->d.g_ntris) return HTRDR_GPU_RES_BAD_ARG;
  if(n && (!rays || !tmax || !from_prim || !from_edge || !prim || !dist)) return HTRDR_GPU_RES_BAD_ARG;
  if(!n) return HTRDR_GPU_RES_OK;
  if(!cuda_ok(cudaSetDevice(scn->device), "cudaSetDevice")) return HTRDR_GPU_RES_BAD_OP;
  DevArr<float> dr, dt, dd;
  DevArr<uint32_t> df, dp;
  DevArr<uint8_t> de;
  if(!dr.from(rays, 6 * n) || !dt.from(tmax, n) || !df.from(from_prim, n) || !de.from(from_edge, n)
  || !dp.make(n) || !dd.make(n))
    return HTRDR_GPU_RES_MEM_ERR;
  if(!cuda_ok(launch_ground_trace(scn->d, n, dr.p(), dt.p(), df.p(), de.p(), dp.p(), dd.p(),
                                  scn->stream), "k_ground_trace")
  || !cuda_ok(cudaStreamSynchronize(scn->stream), "sync") || !dp.to(prim, n) || !dd.to(dist, n))
    return HTRDR_GPU_RES_UNKNOWN_ERR;
  return HTRDR_GPU_RES_OK;
}
HG_API_CATCH("htrdr_gpu_ground_trace")

extern "C" HTRDR_GPU_API htrdr_gpu_res_T
htrdr_gpu_sample_wavelength(htrdr_gpu_scene* scn, const htrdr_gpu_request* req, int channel,
                            size_t n, const double* r0, const double* r1, uint32_t* cdf_band,
                            double* wlen, double* pdf)
try {
  if(!scn || !req || channel < 0 || channel > 2) return HTRDR_GPU_RES_BAD_ARG;
  cudaSetDevice(scn->device);
  DRequest R;
  htrdr_gpu_res_T res = make_drequest(scn, req, &R);
  if(res != HTRDR_GPU_RES_OK) return res;
  if(!n) return HTRDR_GPU_RES_OK;
  DevArr<double> d0, d1, dw, dp;
  DevArr<uint32_t> dc;
  if(!d0.from(r0, n) || !d1.from(r1, n) || !dw.make(n) || !dp.make(n) || !dc.make(n))
    return HTRDR_GPU_RES_MEM_ERR;
  if(!cuda_ok(launch_sample_wavelength(R, channel, n, d0.p(), d1.p(), dc.p(), dw.p(), dp.p(),
                                       scn->stream), "k_sample_wavelength")
  || !cuda_ok(cudaStreamSynchronize(scn->stream), "sync") || !dc.to(cdf_band, n)
  || !dw.to(wlen, n) || !dp.to(pdf, n))
    return HTRDR_GPU_RES_UNKNOWN_ERR;
  return HTRDR_GPU_RES_OK;
}
HG_API_CATCH("htrdr_gpu_sample_wavelength")
