/* The compiled reference oracle (oracle/_ref/libhtrdr_ref.so).
 * TEST INFRASTRUCTURE ONLY: the reference's own atmosphere hot-path C files,
 * compiled unmodified, driven over the oracle's scenes; it pins the oracle
 * (the C files of oracle/) to the reference's arithmetic and draw order. */
#ifndef REF_H
#define REF_H

#include "../ora.h"

struct ref_scene;

/* The scene of `desc' (plane ground only) with the reference's sun */
int ref_scene_create(const struct ora_scene_desc* desc, struct ref_scene** out);
void ref_scene_release(struct ref_scene* scn);

/* atmosphere_draw_map of the reference (src/atmosphere/htrdr_atmosphere_draw_map.c:592-641)
 * on the request: the pixel callbacks fill the pixels [pix_begin, pix_end)
 * (row-major) of `buffer' (pitched rows of the reference's pixel structs),
 * one stream per (pixel, realisation); dump_buffer writes the htrdr-image
 * text to `dump_path' when it is not NULL.  OpenMP over the pixels. */
int ref_draw_map(const struct ref_scene* scn, const struct ora_request* req, void* buffer,
                 size_t pitch, size_t pix_begin, size_t pix_end, int nthreads,
                 const char* dump_path);

/* The weight of every realisation of the pixels [pix_begin, pix_end): the
 * pixel callbacks run one realisation per call (NaN: rejected sample), the
 * layout of ora_realisation_weights. */
int ref_realisation_weights(const struct ref_scene* scn, const struct ora_request* req,
                            size_t pix_begin, size_t pix_end, double* weights, int nthreads);

/* The radiance routines (atmosphere_compute_radiance_sw/_lw) on a batch of
 * rays, one stream per ray keyed like ora_radiance_batch's. */
int ref_radiance_batch(const struct ref_scene* scn, int lw, size_t n, const double* pos,
                       const double* dir, const double* wlen, const uint32_t* iband,
                       const uint32_t* iquad, int cpnt_mask, uint32_t seed, double* out,
                       int nthreads);

#endif
