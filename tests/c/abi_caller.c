/* A C caller of libhtrdr_gpu, written the way the reference (C) would call
 * it: the header must compile as strict C99 with every warning enabled, and
 * the calls that need no device must behave as documented.  With no device
 * visible: scene creation fails with RES_BAD_OP (no CPU fallback) and sets
 * the error text.  Always: version and tunings, argument checks, and the
 * htrdr-image writer on a 2x1 longwave flux map.
 *
 * Usage: abi_caller <output file>.  Exit status 0 on success. */
#include <stdio.h>
#include <string.h>

#include "htrdr_gpu.h"

#define CHECK(cond)                                                        \
  do {                                                                     \
    if(!(cond)) {                                                          \
      fprintf(stderr, "%s:%d: check failed: %s\n", __FILE__, __LINE__, #cond); \
      return 1;                                                            \
    }                                                                      \
  } while(0)

/* The flux pixel struct of the reference (atmosphere_pixel_flux): the
 * flux accumulator {sum, sum2, n, nfail} and the time accumulator */
struct pixel_flux {
  double sum, sum2;
  uint64_t n, nfail;
  double t_sum, t_sum2;
  uint64_t t_n, t_nfail;
};

int
main(int argc, char** argv)
{
  struct htrdr_gpu_tuning t;
  struct htrdr_gpu_scene* scene = NULL;
  struct htrdr_gpu_scene_desc desc;
  struct htrdr_gpu_buffer_layout layout;
  struct htrdr_gpu_map_summary summary;
  struct pixel_flux px[2];
  double layer_z[2] = {0.0, 1000.0}, band_lo[1] = {9000.0}, band_hi[1] = {11000.0};
  double quad_w[1] = {1.0};
  float layer_T[1] = {280.f}, ka[1] = {1e-4f}, ks[1] = {0.f};
  uint32_t nquads[1] = {1};
  FILE* f;
  char line[256];
  int ndev;

  CHECK(argc == 2);
  CHECK(htrdr_gpu_version() != NULL && strlen(htrdr_gpu_version()) > 0);
  ndev = htrdr_gpu_device_count();
  CHECK(ndev >= 0);

  htrdr_gpu_default_tuning(&t);
  CHECK(t.block_size > 0 && t.block_size % 32 == 0 && t.queue_chunk >= 1);
  CHECK(t.engine == HTRDR_GPU_ENGINE_PERSISTENT);
  htrdr_gpu_mode_tuning(HTRDR_GPU_FLUX_LW, &t);
  CHECK(t.engine == HTRDR_GPU_ENGINE_WAVEFRONT && t.wave_tail > 0);
  htrdr_gpu_mode_tuning(HTRDR_GPU_IMAGE_CIE, &t);
  CHECK(t.engine == HTRDR_GPU_ENGINE_WAVEFRONT);

  /* argument checks come before any device work */
  CHECK(htrdr_gpu_scene_create(0, NULL, &scene) == HTRDR_GPU_RES_BAD_ARG);
  CHECK(htrdr_gpu_scene_create_cached(0, NULL, "", &scene) == HTRDR_GPU_RES_BAD_ARG);

  memset(&desc, 0, sizeof(desc));
  desc.nlayers = 1; desc.layer_z = layer_z; desc.layer_T = layer_T;
  desc.nbands = 1; desc.band_lo = band_lo; desc.band_hi = band_hi;
  desc.nquads = nquads; desc.quad_w = quad_w; desc.gas_ka = ka; desc.gas_ks = ks;
  desc.has_ground = 1; desc.ground_temperature = 290.0;
  desc.props_mask = 1u << HTRDR_GPU_KEXT;
  if(ndev == 0) { /* no CPU fallback */
    CHECK(htrdr_gpu_scene_create(0, &desc, &scene) == HTRDR_GPU_RES_BAD_OP);
    CHECK(scene == NULL);
    CHECK(strlen(htrdr_gpu_last_error()) > 0);
  }

  /* the htrdr-image writer (host code) */
  memset(px, 0, sizeof(px));
  px[0].sum = 3.0; px[0].sum2 = 5.0; px[0].n = 2; px[0].t_sum = 4.0; px[0].t_sum2 = 10.0; px[0].t_n = 2;
  layout.width = 2; layout.height = 1; layout.pitch = sizeof(px); layout.elmt_size = sizeof(px[0]);
  layout.alignment = 8;
  CHECK(htrdr_gpu_write_image(HTRDR_GPU_FLUX_LW, &layout, px, argv[1], &summary) == HTRDR_GPU_RES_OK);
  CHECK(summary.flux_n == 2 && summary.path_time_n == 2);
  f = fopen(argv[1], "r");
  CHECK(f != NULL);
  CHECK(fgets(line, sizeof(line), f) != NULL);
  fclose(f);
  CHECK(strcmp(line, "2 1\n") == 0);
  layout.elmt_size = 8; /* not the flux pixel struct */
  CHECK(htrdr_gpu_write_image(HTRDR_GPU_FLUX_LW, &layout, px, argv[1], NULL) == HTRDR_GPU_RES_BAD_ARG);

  printf("abi_caller ok (%d device(s))\n", ndev);
  return 0;
}
