/* Shim of htsky 0.3 (TEST INFRASTRUCTURE ONLY): the sky services the
 * reference's hot path calls, answered from the oracle's medium (gas layers,
 * cloud cells) and its per-(band, quadrature point, property) majorant
 * octrees. */
#ifndef REF_SHIM_HTSKY_H
#define REF_SHIM_HTSKY_H
#include <rsys/rsys.h>
#include <star/svx.h>

struct htsky;

#define HTSKY(Func) CHK(htsky_##Func == RES_OK)

enum htsky_property { HTSKY_Ka, HTSKY_Ks, HTSKY_Kext, HTSKY_PROPS_COUNT__ };
enum htsky_svx_op { HTSKY_SVX_MIN, HTSKY_SVX_MAX, HTSKY_SVX_OPS_COUNT__ };
enum htsky_component_flag {
  HTSKY_CPNT_FLAG_GAS = BIT(0),
  HTSKY_CPNT_FLAG_PARTICLES = BIT(1),
  HTSKY_CPNT_MASK_ALL = HTSKY_CPNT_FLAG_GAS | HTSKY_CPNT_FLAG_PARTICLES
};

res_T htsky_trace_ray(struct htsky* sky, const double org[3], const double dir[3],
                      const double range[2], const svx_hit_filter_T challenge,
                      const svx_hit_filter_T filter, void* context, const size_t iband,
                      const size_t iquad, struct svx_hit* hit);
double htsky_fetch_svx_voxel_property(const struct htsky* sky, const enum htsky_property prop,
                                      const enum htsky_svx_op op, const int cpnt_mask,
                                      const size_t iband, const size_t iquad,
                                      const struct svx_voxel* voxel);
double htsky_fetch_raw_property(const struct htsky* sky, const enum htsky_property prop,
                                const int cpnt_mask, const size_t iband, const size_t iquad,
                                const double pos[3], const double k_min, const double k_max);
double htsky_fetch_temperature(const struct htsky* sky, const double pos[3]);
double htsky_fetch_per_wavelength_particle_phase_function_asymmetry_parameter(
  const struct htsky* sky, const double wlen);
res_T htsky_get_spectral_band_bounds(const struct htsky* sky, const size_t iband,
                                     double bounds[2]);
size_t htsky_find_spectral_band(const struct htsky* sky, const double wlen);
size_t htsky_spectral_band_sample_quadrature(const struct htsky* sky, const double r,
                                             const size_t iband);
#endif
