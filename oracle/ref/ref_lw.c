/* The reference's longwave radiance file, compiled unmodified in this
 * translation unit so that the shim can recognise its static hit filter
 * (TEST INFRASTRUCTURE ONLY). */
#include "htrdr_atmosphere_compute_radiance_lw.c"

int
ref_lw_trace_prop(svx_hit_filter_T filter, void* context)
{
  (void)context;
  return filter == hit_filter ? HTSKY_Kext : -1;
}
