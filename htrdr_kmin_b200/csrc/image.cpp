/* htrdr-image writer: a rendered map to the plain-text image format, and the
 * run summaries the reference logs after a map (time per radiative path,
 * flux density of a flux map).
 *
 * Restates dump_buffer / dump_pixel_{xwave,flux,image} / dump_accum and the
 * summaries of atmosphere_draw_map
 * (src/atmosphere/htrdr_atmosphere_draw_map.c:477-641) and the format of
 * doc/htrdr-image.5: the definition line "width height", then one line of 8
 * components per pixel, row by row from the top-left pixel, an empty line
 * after each row.  The component formats are the reference's printf formats,
 * so a map written here is byte-identical to the reference's output for the
 * same pixel values. */
#include "internal.h"

#include <cmath>
#include <cstdio>
#include <cstring>

using namespace hg;

namespace {

struct Accum {
  double s = 0, s2 = 0;
  uint64_t n = 0, nfail = 0;
};

/* htrdr_accum_get_estimation (src/core/htrdr_accum.h:48-66) */
void
estimate(const Accum& a, double* E, double* SE)
{
  if(!a.n) { *E = 0; *SE = 0; return; }
  const double N = (double)a.n;
  const double e = a.s / N;
  const double V = std::fmax(a.s2 / N - e * e, 0.0);
  *E = e;
  *SE = std::sqrt(V / N);
}

Accum
accum_at(const char* p)
{
  Accum a;
  std::memcpy(&a.s, p, 8);
  std::memcpy(&a.s2, p + 8, 8);
  std::memcpy(&a.n, p + 16, 8);
  std::memcpy(&a.nfail, p + 24, 8);
  return a;
}

/* dump_accum: the estimate, and its weights added to a run total */
void
dump_accum(const Accum& a, Accum* total, FILE* f)
{
  if(a.n == 0) {
    std::fprintf(f, "0 0 ");
    return;
  }
  double E, SE;
  estimate(a, &E, &SE);
  std::fprintf(f, "%g %g ", E, SE);
  if(total) {
    total->s += a.s;
    total->s2 += a.s2;
    total->n += a.n;
  }
}

double
d_at(const char* p)
{
  double v;
  std::memcpy(&v, p, 8);
  return v;
}

}  // namespace

extern "C" HTRDR_GPU_API htrdr_gpu_res_T
htrdr_gpu_write_image(int mode, const htrdr_gpu_buffer_layout* layout, const void* buffer,
                      const char* path, htrdr_gpu_map_summary* summary)
try {
  if(!layout || !buffer || !path) return HTRDR_GPU_RES_BAD_ARG;
  if(mode < HG_XWAVE_SW || mode > HG_FLUX_LW) return HTRDR_GPU_RES_BAD_ARG;
  if(layout->elmt_size != pixel_size(mode) || layout->pitch < layout->width * layout->elmt_size)
    return HTRDR_GPU_RES_BAD_ARG;
  const bool to_stdout = std::strcmp(path, "-") == 0;
  FILE* f = to_stdout ? stdout : std::fopen(path, "w");
  if(!f) {
    set_error(std::string("cannot open ") + path + " for writing");
    return HTRDR_GPU_RES_IO_ERR;
  }
  Accum time_total, flux_total;
  std::fprintf(f, "%lu %lu\n", (unsigned long)layout->width, (unsigned long)layout->height);
  const char* base = (const char*)buffer;
  for(uint32_t y = 0; y < layout->height; ++y) {
    for(uint32_t x = 0; x < layout->width; ++x) {
      const char* p = base + (size_t)y * layout->pitch + (size_t)x * layout->elmt_size;
      if(mode == HG_FLUX_SW || mode == HG_FLUX_LW) {
        /* atmosphere_pixel_flux {flux, time} */
        dump_accum(accum_at(p), &flux_total, f);
        std::fprintf(f, "0 0 0 0 ");
        dump_accum(accum_at(p + 32), &time_total, f);
      } else if(mode == HG_IMAGE_CIE) {
        /* atmosphere_pixel_image {X, Y, Z, time} */
        std::fprintf(f, "%g %g ", d_at(p), d_at(p + 8));
        std::fprintf(f, "%g %g ", d_at(p + 16), d_at(p + 24));
        std::fprintf(f, "%g %g ", d_at(p + 32), d_at(p + 40));
        dump_accum(accum_at(p + 48), &time_total, f);
      } else {
        /* atmosphere_pixel_xwave {radiance, radiance_temperature, time} */
        std::fprintf(f, "%g %g %f %f 0 0 ", d_at(p + 16), d_at(p + 24), d_at(p), d_at(p + 8));
        dump_accum(accum_at(p + 32), &time_total, f);
      }
      std::fprintf(f, "\n");
    }
    std::fprintf(f, "\n");
  }
  const bool io_ok = !std::ferror(f);
  if(!to_stdout) std::fclose(f);
  else std::fflush(f);
  if(!io_ok) {
    set_error(std::string("write error on ") + path);
    return HTRDR_GPU_RES_IO_ERR;
  }
  if(summary) {
    std::memset(summary, 0, sizeof(*summary));
    estimate(time_total, &summary->path_time_E, &summary->path_time_SE);
    summary->path_time_n = time_total.n;
    if(mode == HG_FLUX_SW || mode == HG_FLUX_LW) {
      estimate(flux_total, &summary->flux_E, &summary->flux_SE);
      summary->flux_n = flux_total.n;
    }
  }
  return HTRDR_GPU_RES_OK;
}
HG_API_CATCH("htrdr_gpu_write_image")
