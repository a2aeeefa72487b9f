/* The reference's shortwave radiance file, compiled unmodified in this
 * translation unit so that the shim can tell its two static hit filters apart
 * (TEST INFRASTRUCTURE ONLY). */
#include "htrdr_atmosphere_compute_radiance_sw.c"

int
ref_sw_trace_prop(svx_hit_filter_T filter, void* context)
{
  if(filter == scattering_hit_filter) return HTSKY_Ks;
  if(filter == transmissivity_hit_filter)
    return (int)((const struct transmissivity_context*)context)->prop;
  return -1;
}
