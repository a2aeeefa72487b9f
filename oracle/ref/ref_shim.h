/* Types shared by the shim of the compiled reference oracle and its harness.
 * TEST INFRASTRUCTURE ONLY (see ref_shim.c). */
#ifndef REF_SHIM_H
#define REF_SHIM_H

#include "atmosphere/htrdr_atmosphere_c.h"
#include "atmosphere/htrdr_atmosphere_ground.h"
#include "core/htrdr_c.h"
#include "core/htrdr_interface.h"
#include "core/htrdr_materials.h"

#include <high_tune/htsky.h>
#include <rsys/clock_time.h>
#include <star/s3d.h>
#include <star/scam.h>
#include <star/ssf.h>
#include <star/ssp.h>

#include "../ora.h"

/* A generator: the oracle's stream, and whether the draws are transport
 * canonicals (inside the radiance routines) or 53-bit ones */
struct ssp_rng {
  struct ora_rng r;
  int transport;
};

struct htsky { const struct ora_scene* scn; };

struct scam {
  double pos[3], f[3], r[3], u[3];
  double tan_half, aspect, lens_radius, focal_dst, ortho_h;
  int type; /* 0 perspective (pinhole or thin lens), 1 orthographic */
};

struct htrdr_atmosphere_ground {
  int has_ground;
  int brdf; /* 0 Lambertian, 1 specular */
  double reflectivity, temperature;
};

/* Realisation hook: from the next clock read on, the calling thread's
 * realisations draw from the streams {pixel, seed} x keys[i] (keys == NULL:
 * 0, 1, 2, ...) */
void ref_hook_begin(struct ssp_rng* rng, uint32_t pixel, uint32_t seed, const uint32_t* keys);
void ref_hook_end(void);

/* Property of a traversal from its filter and context (-1: not this file's
 * filter): ref_sw.c and ref_lw.c, which see the reference's static filters */
int ref_sw_trace_prop(svx_hit_filter_T filter, void* context);
int ref_lw_trace_prop(svx_hit_filter_T filter, void* context);

/* The radiance routines entered from the pixel callbacks */
double ref_entry_radiance_sw(struct htrdr_atmosphere* cmd, const size_t ithread,
                             struct ssp_rng* rng, const int cpnt_mask, const double pos[3],
                             const double dir[3], const double wlen, const size_t iband,
                             const size_t iquad);
double ref_entry_radiance_lw(struct htrdr_atmosphere* cmd, const size_t ithread,
                             struct ssp_rng* rng, const double pos[3], const double dir[3],
                             const double wlen, const size_t iband, const size_t iquad);

/* htrdr runtime functions the reference declares in src/core/htrdr.h and
 * htrdr_log.h are defined in ref_shim.c */
#endif
