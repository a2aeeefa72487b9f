/* Shim of star-sf 0.9 (TEST INFRASTRUCTURE ONLY): Henyey-Greenstein and
 * Rayleigh phase functions, Lambertian and specular reflections. */
#ifndef REF_SHIM_SSF_H
#define REF_SHIM_SSF_H
#include <rsys/rsys.h>

struct mem_allocator;
struct ssp_rng;

#define SSF(Func) CHK(ssf_##Func == RES_OK)

enum ssf_bxdf_flag {
  SSF_REFLECTION = BIT(0),
  SSF_TRANSMISSION = BIT(1),
  SSF_SPECULAR = BIT(2),
  SSF_DIFFUSE = BIT(3),
  SSF_GLOSSY = BIT(4)
};

struct ssf_phase_type { int id; };
extern const struct ssf_phase_type ssf_phase_hg;
extern const struct ssf_phase_type ssf_phase_rayleigh;

struct ssf_phase;
struct ssf_bsdf;

res_T ssf_phase_create(struct mem_allocator* allocator, const struct ssf_phase_type* type,
                       struct ssf_phase** phase);
res_T ssf_phase_ref_get(struct ssf_phase* phase);
res_T ssf_phase_ref_put(struct ssf_phase* phase);
res_T ssf_phase_hg_setup(struct ssf_phase* phase, const double g);
/* wo is minus the incoming propagation direction; wi receives the new
 * propagation direction, drawn around -wo with the phase function's
 * distribution of the scattering cosine.  eval(wo, wi) takes the cosine
 * -wo.wi between the two propagation directions. */
void ssf_phase_sample(struct ssf_phase* phase, struct ssp_rng* rng, const double wo[3],
                      double wi[3], double* pdf);
double ssf_phase_eval(struct ssf_phase* phase, const double wo[3], const double wi[3]);

res_T ssf_bsdf_ref_get(struct ssf_bsdf* bsdf);
res_T ssf_bsdf_ref_put(struct ssf_bsdf* bsdf);
double ssf_bsdf_sample(struct ssf_bsdf* bsdf, struct ssp_rng* rng, const double wo[3],
                       const double N[3], double wi[3], int* type, double* pdf);
double ssf_bsdf_eval(struct ssf_bsdf* bsdf, const double wo[3], const double N[3],
                     const double wi[3]);
#endif
