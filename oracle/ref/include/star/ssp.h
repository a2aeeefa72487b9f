/* Shim of star-sp 0.14 (TEST INFRASTRUCTURE ONLY): the random-number
 * services the reference's hot path calls, backed by the oracle's
 * counter-based Philox streams (ora_rng).  The stream a generator draws
 * from is chosen by the harness (one stream per (pixel, realisation)). */
#ifndef REF_SHIM_SSP_H
#define REF_SHIM_SSP_H
#include <rsys/rsys.h>

struct ssp_rng;

/* Canonical number in [0, 1): 24 bits from one stream word inside the
 * radiance routines (the transport canonicals), 53 bits from two words in
 * the pixel callbacks (film, lens and wavelength draws) -- the precision the
 * oracle and the CUDA kernels give each draw. */
double ssp_rng_canonical(struct ssp_rng* rng);
/* Exponential variate of rate mu from one stream word: -log(u)/mu with
 * u = (2 m + 1) 2^-24, m the word's top 23 bits (never 0 nor infinite). */
double ssp_ran_exp(struct ssp_rng* rng, const double mu);
/* Cosine-weighted direction around the unit normal `up' */
double* ssp_ran_hemisphere_cos(struct ssp_rng* rng, const double up[3], double dir[3],
                               double* pdf);
/* Uniform direction in the spherical cap of cosine `cos_aperture' around +Z */
double* ssp_ran_sphere_cap_uniform_local(struct ssp_rng* rng, const double cos_aperture,
                                         double dir[3], double* pdf);
#endif
