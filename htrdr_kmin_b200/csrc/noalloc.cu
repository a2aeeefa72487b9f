/* Allocation-free variant of the plain drop-in draw_map.
 *
 * Some callers cannot allocate device memory while they render: a host
 * application that hands all of HBM to its own memory pool at start-up, or a
 * render loop that must not call cudaMalloc/cudaFree (cudaFree synchronises
 * the whole device).  htrdr_gpu_draw_map_noalloc serves them: the caller
 * passes the scene (created beforehand) and a device output buffer, and the
 * per-pixel FP64 accumulators, the launch counters and the wavelength-sampler
 * tables live in file-scope static device arrays of fixed size, reserved on
 * every GPU that loads the library until the process exits.
 *
 * Limits: pixels x (channels + 1) <= HG_NOALLOC_MAX_ACC accumulators
 * (65536, e.g. a 128 x 128 flux map or a 128 x 128 CIE image) and a
 * wavelength CDF of at most HG_NOALLOC_MAX_CDF entries (131072 for the Planck
 * sampler; 29127 for the CIE sampler, whose tables take 9 doubles per band).
 * Larger requests are rejected with HTRDR_GPU_RES_BAD_ARG.
 *
 * All calls share the static arrays, which keep the last call's contents:
 * the accumulators and counters are cleared at the start of every call, and
 * two calls whose GPU work overlaps (several host threads, several scenes on
 * one device) race on them; serialise such calls. */
#include "internal.h"

#include <cmath>
#include <cstring>
#include <mutex>

#define HG_NOALLOC_MAX_ACC 65536u
#define HG_NOALLOC_MAX_CDF 131072u
#define HG_NOALLOC_MAX_DEVICES 64

namespace {

__device__ __align__(256) DAccum g_noalloc_acc[HG_NOALLOC_MAX_ACC];
__device__ __align__(256) unsigned long long g_noalloc_cnt[8];
__device__ __align__(256) double g_noalloc_tab[2 * HG_NOALLOC_MAX_CDF];

/* Device addresses of the static arrays, looked up once per device with the
 * device current (a host-side reference to a __device__ symbol is only a
 * stand-in, not an address the kernels may use). */
struct SymAddr {
  DAccum* acc = nullptr;
  unsigned long long* cnt = nullptr;
  double* tab = nullptr;
  bool ready = false;
};
SymAddr g_sym[HG_NOALLOC_MAX_DEVICES];
std::mutex g_mtx;
/* host-side staging of the sampler tables (fixed size, no allocation) */
double g_host_tab[2 * HG_NOALLOC_MAX_CDF];

bool
setup_symbols(int device)
{
  SymAddr& s = g_sym[device];
  if(s.ready) return true;
  void* p = nullptr;
  if(!hg::cuda_ok(cudaGetSymbolAddress(&p, g_noalloc_acc), "cudaGetSymbolAddress(acc)")) return false;
  s.acc = (DAccum*)p;
  if(!hg::cuda_ok(cudaGetSymbolAddress(&p, g_noalloc_cnt), "cudaGetSymbolAddress(cnt)")) return false;
  s.cnt = (unsigned long long*)p;
  if(!hg::cuda_ok(cudaGetSymbolAddress(&p, g_noalloc_tab), "cudaGetSymbolAddress(tab)")) return false;
  s.tab = (double*)p;
  s.ready = true;
  return true;
}

void
norm3(double v[3])
{
  const double n = std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
  v[0] /= n; v[1] /= n; v[2] /= n;
}

void
cross3(double o[3], const double a[3], const double b[3])
{
  o[0] = a[1] * b[2] - a[2] * b[1];
  o[1] = a[2] * b[0] - a[0] * b[2];
  o[2] = a[0] * b[1] - a[1] * b[0];
}

}  // namespace

using namespace hg;

/* Draw one map like htrdr_gpu_draw_map_device, with no device allocation.
 * The first call on a device looks up the static arrays' device addresses
 * (cudaGetSymbolAddress); make that first call before any stream capture. */
extern "C" HTRDR_GPU_API htrdr_gpu_res_T
htrdr_gpu_draw_map_noalloc(htrdr_gpu_scene* scn, const htrdr_gpu_request* req,
                           const htrdr_gpu_buffer_layout* layout, void* device_buffer)
try {
  if(!scn || !req || !layout || !device_buffer) return HTRDR_GPU_RES_BAD_ARG;
  if(req->mode < 0 || req->mode > 4 || !req->width || !req->height || !req->spp)
    return HTRDR_GPU_RES_BAD_ARG;
  if(check_layout(req, layout) != HTRDR_GPU_RES_OK) return HTRDR_GPU_RES_BAD_ARG;
  if(req->wlen_range[0] > req->wlen_range[1]) return HTRDR_GPU_RES_BAD_ARG;
  const bool lw = req->mode == HG_XWAVE_LW || req->mode == HG_FLUX_LW;
  const bool cie = req->mode == HG_IMAGE_CIE;
  if(!cie && req->ref_temperature <= 0) return HTRDR_GPU_RES_BAD_ARG;
  const uint32_t need = lw ? (1u << HG_KEXT) : 7u;
  if(scn->d.has_cloud && (scn->props_mask & need) != need) return HTRDR_GPU_RES_BAD_ARG;

  const uint64_t npix = (uint64_t)req->width * req->height;
  const uint32_t nch = cie ? 3u : 1u;
  if(npix * (nch + 1) > HG_NOALLOC_MAX_ACC) {
    set_error("htrdr_gpu_draw_map_noalloc: pixels x (channels + 1) exceeds the 65536 static accumulators");
    return HTRDR_GPU_RES_BAD_ARG;
  }
  const double r0 = req->wlen_range[0], r1 = req->wlen_range[1];
  const size_t nb = (size_t)std::rint(r1 - r0);
  const size_t ncdf = cie ? (nb ? nb : 1) : nb;
  if((cie ? 9 * ncdf : 2 * ncdf) > 2 * (size_t)HG_NOALLOC_MAX_CDF) {
    set_error("htrdr_gpu_draw_map_noalloc: the wavelength CDF exceeds the static sampler tables");
    return HTRDR_GPU_RES_BAD_ARG;
  }
  if(scn->device < 0 || scn->device >= HG_NOALLOC_MAX_DEVICES) return HTRDR_GPU_RES_BAD_ARG;

  std::lock_guard<std::mutex> lock(g_mtx);
  if(!cuda_ok(cudaSetDevice(scn->device), "cudaSetDevice")) return HTRDR_GPU_RES_BAD_OP;
  if(!setup_symbols(scn->device)) return HTRDR_GPU_RES_BAD_OP;
  const SymAddr& sym = g_sym[scn->device];
  cudaStream_t st = scn->stream;

  /* Wavelength sampler tables, same definitions as the regular path
   * (htrdr_ran_wlen_planck.c:55-134, htrdr_ran_wlen_cie_xyz.c:185-280) */
  DRequest R;
  std::memset(&R, 0, sizeof(R));
  double band_len = 0;
  size_t tab_doubles = 0;
  if(cie) {
    band_len = (r1 - r0) / (double)ncdf;
    double* cdf = g_host_tab;
    double* fb = g_host_tab + 3 * ncdf;
    for(int ch = 0; ch < 3; ++ch) {
      double sum = 0;
      for(size_t i = 0; i < ncdf; ++i) {
        const double lo = r0 + (double)i * band_len;
        double hi = lo + band_len;
        if(hi > r1) hi = r1;
        cdf[ch * ncdf + i] = cie_trapezoid(lo, hi, ch);
        sum += cdf[ch * ncdf + i];
        fb[(ch * ncdf + i) * 2 + 0] = fit_bar_1931(ch, lo);
        fb[(ch * ncdf + i) * 2 + 1] = fit_bar_1931(ch, lo + band_len);
      }
      R.rcp_integral[ch] = 1.0 / sum;
      for(size_t i = 0; i < ncdf; ++i) {
        cdf[ch * ncdf + i] /= sum;
        if(i) cdf[ch * ncdf + i] += cdf[ch * ncdf + i - 1];
      }
      cdf[ch * ncdf + ncdf - 1] = 1.0;
    }
    tab_doubles = 9 * ncdf;
    R.cdf = sym.tab;
    R.fbound = sym.tab + 3 * ncdf;
  } else if(ncdf) {
    band_len = (r1 - r0) / (double)ncdf;
    double* cdf = g_host_tab;
    double* pdf = g_host_tab + ncdf;
    double sum = 0;
    for(size_t i = 0; i < ncdf; ++i) {
      const double lo = r0 + (double)i * band_len;
      double hi = lo + band_len;
      if(hi > r1) hi = r1;
      pdf[i] = blackbody_fraction(lo * 1e-9, hi * 1e-9, req->ref_temperature);
      sum += pdf[i];
    }
    for(size_t i = 0; i < ncdf; ++i) {
      pdf[i] /= sum;
      cdf[i] = i == 0 ? pdf[i] : pdf[i] + cdf[i - 1];
    }
    cdf[ncdf - 1] = 1.0;
    tab_doubles = 2 * ncdf;
    R.cdf = sym.tab;
    R.pdf = sym.tab + ncdf;
  }
  if(tab_doubles
  && !cuda_ok(cudaMemcpyAsync(sym.tab, g_host_tab, tab_doubles * sizeof(double),
                              cudaMemcpyHostToDevice, st), "cudaMemcpyAsync(tables)"))
    return HTRDR_GPU_RES_UNKNOWN_ERR;

  /* Request view (same fields as the regular path's make_drequest) */
  R.mode = req->mode;
  R.width = req->width;
  R.height = req->height;
  R.spp = req->spp;
  R.nreal_pp = req->spp * nch;
  R.seed = req->seed;
  R.acc = sym.acc;
  R.tacc = sym.acc + npix * nch;
  R.pix_sz[0] = 1.0 / (double)req->width;
  R.pix_sz[1] = 1.0 / (double)req->height;
  R.wlen_range[0] = r0;
  R.wlen_range[1] = r1;
  R.ncdf = (uint32_t)ncdf;
  R.band_len = band_len;
  R.ref_T = req->ref_temperature;
  R.camera_type = req->camera_type;
  double f[3], r[3], u[3], n[3], ax[3], ay[3];
  for(int i = 0; i < 3; ++i) f[i] = req->cam_tgt[i] - req->cam_pos[i];
  norm3(f);
  cross3(r, f, req->cam_up);
  norm3(r);
  cross3(u, r, f);
  for(int i = 0; i < 3; ++i) n[i] = req->rect_tgt[i] - req->rect_pos[i];
  norm3(n);
  cross3(ax, n, req->rect_up);
  norm3(ax);
  cross3(ay, n, ax);
  norm3(ay);
  for(int i = 0; i < 3; ++i) {
    R.cam_pos[i] = req->cam_pos[i]; R.cam_f[i] = f[i]; R.cam_r[i] = r[i]; R.cam_u[i] = u[i];
    R.rect_pos[i] = req->rect_pos[i];
    R.rect_n[i] = n[i];
    R.rect_ax[i] = ax[i] * req->rect_size[0] * 0.5;
    R.rect_ay[i] = ay[i] * req->rect_size[1] * 0.5;
  }
  R.tan_half = std::tan(req->fov_deg * 3.14159265358979323846 / 360.0);
  R.aspect = (double)req->width / (double)req->height;
  R.lens_radius = req->lens_radius;
  R.focal_dst = req->focal_dst;
  R.ortho_h = req->ortho_height;

  /* the shared scratch keeps the previous call's sums: clear what this call uses */
  bool ok = cuda_ok(cudaMemsetAsync(sym.acc, 0, npix * (nch + 1) * sizeof(DAccum), st), "cudaMemsetAsync")
         && cuda_ok(cudaMemsetAsync(sym.cnt, 0, sizeof(g_noalloc_cnt), st), "cudaMemsetAsync");
  DAccum* acc = sym.acc;
  DAccum* tacc = sym.acc + npix * nch;
  ok = ok && cuda_ok(launch_plain(scn->d, R, acc, tacc, 0, (uint32_t)npix, nullptr, sym.cnt, st), "k_plain");
  ok = ok && cuda_ok(launch_finalize(R, acc, tacc, device_buffer, layout->pitch, st), "k_finalize");
  ok = ok && cuda_ok(cudaStreamSynchronize(st), "cudaStreamSynchronize");
  return ok ? HTRDR_GPU_RES_OK : HTRDR_GPU_RES_UNKNOWN_ERR;
}
HG_API_CATCH("htrdr_gpu_draw_map_noalloc")
