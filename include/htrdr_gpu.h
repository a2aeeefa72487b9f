/* htrdr_gpu.h -- C ABI of the B200 (sm_100a) atmosphere path tracer.
 *
 * A drop-in for the hot path of htrdr-atmosphere (AnthonyArfaux/htrdr_kmin):
 * the htrdr_draw_map driver with the atmosphere per-pixel / per-probe
 * realisation callbacks, the shortwave and longwave radiance routines and
 * the per-(band, quadrature point) kmin/kmax majorant octrees of htsky.
 * Plain C types only; every buffer argument is a host pointer unless the
 * function name ends in _device.  Return codes follow rsys res_T.
 *
 * No CPU fallback: every entry point that computes runs CUDA kernels and
 * returns HTRDR_GPU_RES_BAD_OP when no usable device is present. */
#ifndef HTRDR_GPU_H
#define HTRDR_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
  #define HTRDR_GPU_API __attribute__((visibility("default")))
#else
  #define HTRDR_GPU_API
#endif

/* rsys res_T values (RES_OK, RES_BAD_ARG, RES_MEM_ERR, RES_IO_ERR,
 * RES_UNKNOWN_ERR, RES_BAD_OP) */
typedef int htrdr_gpu_res_T;
#define HTRDR_GPU_RES_OK 0
#define HTRDR_GPU_RES_BAD_ARG 1
#define HTRDR_GPU_RES_MEM_ERR 2
#define HTRDR_GPU_RES_IO_ERR 3
#define HTRDR_GPU_RES_UNKNOWN_ERR 4
#define HTRDR_GPU_RES_BAD_OP 5

/* Output/spectral mode = the atmosphere draw_pixel callback that
 * atmosphere_draw_map selects (src/atmosphere/htrdr_atmosphere_draw_map.c:438-475) */
enum htrdr_gpu_mode {
  HTRDR_GPU_XWAVE_SW = 0,  /* draw_pixel_xwave, shortwave  (:324-436) */
  HTRDR_GPU_XWAVE_LW = 1,  /* draw_pixel_xwave, longwave   (:324-436) */
  HTRDR_GPU_IMAGE_CIE = 2, /* draw_pixel_image, CIE XYZ    (:109-207) */
  HTRDR_GPU_FLUX_SW = 3,   /* draw_pixel_flux, shortwave   (:209-322) */
  HTRDR_GPU_FLUX_LW = 4    /* draw_pixel_flux, longwave    (:209-322) */
};

/* Radiance components (enum atmosphere_radiance_cpnt_flag,
 * src/atmosphere/htrdr_atmosphere_c.h:38-44) */
#define HTRDR_GPU_RADIANCE_DIRECT 1
#define HTRDR_GPU_RADIANCE_DIFFUSE 2
#define HTRDR_GPU_RADIANCE_ALL 3

/* Medium properties (enum htsky_property) */
#define HTRDR_GPU_KA 0
#define HTRDR_GPU_KS 1
#define HTRDR_GPU_KEXT 2

/* Medium, ground and sun: what htsky_create, htrdr_atmosphere_ground_create
 * and htrdr_atmosphere_sun_create set up in htrdr_atmosphere_create
 * (src/atmosphere/htrdr_atmosphere.c:353-382). */
struct htrdr_gpu_scene_desc {
  uint32_t nlayers;
  const double* layer_z;        /* [nlayers+1] layer bounds in m, ascending, from 0 */
  const float* layer_T;         /* [nlayers] temperature in K */
  uint32_t nbands;
  const double* band_lo;        /* [nbands] nm */
  const double* band_hi;        /* [nbands] nm */
  const uint32_t* nquads;       /* [nbands] quadrature points per band */
  const double* quad_w;         /* [sum nquads] quadrature weights (sum 1 per band) */
  const float* gas_ka;          /* [sum nquads][nlayers] 1/m */
  const float* gas_ks;          /* [sum nquads][nlayers] 1/m */
  uint32_t cloud_def[3];        /* nx, ny, nz; all 0 = clear sky */
  double cloud_lower[3];        /* m */
  double cloud_cell[3];         /* m */
  const float* cloud_lwc;       /* [nz][ny][nx] kg/m^3 */
  const float* cloud_sigma_ext; /* [nbands] m^2/kg */
  const float* cloud_ssa;       /* [nbands] */
  const float* cloud_g;         /* [nbands] Henyey-Greenstein asymmetry */
  int32_t repeat_clouds;        /* -r */
  double optical_thickness;     /* -T: majorant merge threshold */
  uint32_t grid_max_definition[3]; /* -V: 0 = cloud definition */
  int32_t has_ground;
  int32_t ground_brdf;          /* 0 Lambertian, 1 specular */
  double ground_reflectivity;
  double ground_temperature;    /* K */
  double sun_azimuth, sun_elevation; /* -D, degrees */
  uint32_t props_mask;          /* bit p: build the majorants of property p */
  int32_t octree_on_host;       /* 1: build the octrees on the host CPU (else on the GPU) */
  /* Ground geometry (htrdr_atmosphere_ground_create,
   * src/atmosphere/htrdr_atmosphere_ground.c:105-160): a triangle mesh that
   * replaces the plane ground above when ground_ntris > 0.  A triangle is
   * front-facing on the side from which its vertices are seen clockwise
   * (doc/htrdr-obj.5). */
  uint32_t ground_nverts;
  const float* ground_verts;        /* [nverts][3] m */
  uint32_t ground_ntris;
  const uint32_t* ground_tris;      /* [ntris][3] vertex indices */
  const uint32_t* ground_tri_iface; /* [ntris] interface of the triangle */
  uint32_t ground_nifaces;
  const uint32_t* ground_ifaces;    /* [nifaces][3] front, thin, back material
                                     * (UINT32_MAX: none; thin is used when set) */
  uint32_t ground_nmtls;
  const double* ground_mtl_temperature; /* [nmtls] K (<= 0: no emission) */
  const uint32_t* ground_mtl_nbrdf;     /* [nmtls] tabulated BRDFs (0: semi-transparent) */
  const double* ground_mtl_brdf;        /* [sum nbrdf][3]: wavelength nm (ascending per
                                         * material), type (0 Lambertian, 1 specular),
                                         * reflectivity */
  int32_t repeat_ground;            /* repeat the mesh's bounding box infinitely in X and Y */
  uint32_t ground_sky_mtl;          /* material of the atmosphere: a flux probe whose upward
                                     * ray meets the mesh from another material is rejected
                                     * (src/atmosphere/htrdr_atmosphere_draw_map.c:73-99) */
};

/* One run of the atmosphere command: sensor, spectral domain, output type
 * and spp (htrdr_atmosphere_args). */
struct htrdr_gpu_request {
  int32_t mode;                 /* enum htrdr_gpu_mode */
  uint32_t width, height, spp;
  double wlen_range[2];         /* nm */
  double ref_temperature;       /* K */
  int32_t camera_type;          /* 0 perspective, 1 orthographic */
  double cam_pos[3], cam_tgt[3], cam_up[3];
  double fov_deg, lens_radius, focal_dst, ortho_height;
  double rect_pos[3], rect_tgt[3], rect_up[3], rect_size[2];
  uint32_t seed;
};

/* struct htrdr_buffer_layout (src/core/htrdr_buffer.h:44-50) */
struct htrdr_gpu_buffer_layout {
  size_t width, height, pitch, elmt_size, alignment;
};

/* Device counters of one launch */
struct htrdr_gpu_stats {
  uint64_t realisations; /* completed realisations */
  uint64_t segments;     /* voxels (octree leaves + gas layers) visited */
  uint64_t nodes;        /* majorant nodes fetched */
  uint64_t collisions;   /* tentative collisions */
  uint64_t failures;     /* traces stopped by the step guard */
  double kernel_ms;      /* CUDA-event time of the transport kernel(s) */
  double total_ms;       /* whole call, device side */
  uint64_t launches;     /* kernels the call launched (transport, initialisation, finalize) */
  uint64_t grid_bytes;   /* bytes of leaf-grid entries read: 9 per majorant-grid
                          * lookup (a leaf's kmin/kmax and level, no node
                          * fetch), 4 per node-grid lookup (then a node) */
};

struct htrdr_gpu_scene;
struct htrdr_gpu_server;

/* ---- scene (replaces htsky_create: src/atmosphere/htrdr_atmosphere.c:366-382) ---- */
HTRDR_GPU_API htrdr_gpu_res_T
htrdr_gpu_scene_create(int device, const struct htrdr_gpu_scene_desc* desc,
                       struct htrdr_gpu_scene** scene);
/* The same with the majorant-octree cache of option -O (htsky's
 * cache_filename, src/atmosphere/htrdr_atmosphere.c:369): when `cache_path'
 * exists and was written from the same medium (layers, gas and cloud
 * coefficients, optics, spectral grid, octree properties) its octrees are
 * loaded instead of built, and optical_thickness and grid_max_definition
 * (-T, -V) are ignored; when it holds octrees of another medium the call
 * fails with RES_BAD_ARG; when it does not exist the octrees are built and
 * written to it.  The file stores 16-byte nodes in the device layout.  A
 * clear sky (no cloud grid) has no octrees: the cache is then neither read
 * nor written. */
HTRDR_GPU_API htrdr_gpu_res_T
htrdr_gpu_scene_create_cached(int device, const struct htrdr_gpu_scene_desc* desc,
                              const char* cache_path, struct htrdr_gpu_scene** scene);
HTRDR_GPU_API void htrdr_gpu_scene_release(struct htrdr_gpu_scene* scene);
/* Device bytes held by the scene (medium + octrees) */
HTRDR_GPU_API size_t htrdr_gpu_scene_device_bytes(const struct htrdr_gpu_scene* scene);
/* Copy one majorant octree to the host as 16-byte {kmin, kmax, child, 0}
 * nodes (what htsky_dump_cloud_vtk writes, src/atmosphere/htrdr_atmosphere.c:196-224).
 * With nodes == NULL only *count is set. */
HTRDR_GPU_API htrdr_gpu_res_T
htrdr_gpu_scene_get_tree(const struct htrdr_gpu_scene* scene, uint32_t iband, uint32_t iquad,
                         int prop, void* nodes, size_t capacity, size_t* count);
HTRDR_GPU_API uint32_t htrdr_gpu_scene_tree_depth(const struct htrdr_gpu_scene* scene);

/* ---- drop-in driver: htrdr_draw_map(htrdr, args, buf) with the atmosphere
 * callbacks (src/core/htrdr_draw_map.h:89-93, src/atmosphere/htrdr_atmosphere_draw_map.c:592-641).
 * Fills `buffer' (host memory, `layout') with atmosphere_pixel_{xwave,flux,image}
 * structs (src/atmosphere/htrdr_atmosphere_c.h:46-76).
 *
 * Three engines compute the same per-realisation weights (only the FP64
 * summation order of a pixel differs): the persistent megakernel with its
 * work queue, the wavefront engine (event and trace stage kernels over a
 * pool of path slots in HBM, same work queue) and the plain
 * one-thread-per-realisation kernel. ---- */
enum htrdr_gpu_engine {
  HTRDR_GPU_ENGINE_PERSISTENT = 0,
  HTRDR_GPU_ENGINE_PLAIN = 1,
  HTRDR_GPU_ENGINE_WAVEFRONT = 2,
  /* the persistent kernel with its paths in shared memory, regrouped by
   * stage across the whole block at every step */
  HTRDR_GPU_ENGINE_SORTED = 3
};
struct htrdr_gpu_tuning;
/* Engine of the scene's htrdr_gpu_draw_map(_device) calls.  `tuning' (NULL:
 * the default of the request's mode) applies to the work-queue engines;
 * `engine' overrides its engine field.  The default is the mode's tuning,
 * engine included. */
HTRDR_GPU_API htrdr_gpu_res_T
htrdr_gpu_scene_set_engine(struct htrdr_gpu_scene* scene, int engine,
                           const struct htrdr_gpu_tuning* tuning);
HTRDR_GPU_API htrdr_gpu_res_T
htrdr_gpu_draw_map(struct htrdr_gpu_scene* scene, const struct htrdr_gpu_request* req,
                   const struct htrdr_gpu_buffer_layout* layout, void* buffer,
                   struct htrdr_gpu_stats* stats);
/* Same, output written to device memory (no host copy). */
HTRDR_GPU_API htrdr_gpu_res_T
htrdr_gpu_draw_map_device(struct htrdr_gpu_scene* scene, const struct htrdr_gpu_request* req,
                          const struct htrdr_gpu_buffer_layout* layout, void* device_buffer,
                          struct htrdr_gpu_stats* stats);

/* The map's FP64 accumulators instead of its pixel structs, for callers that
 * combine maps drawn by several processes or GPUs and finalize once: the
 * reference gathers the tiles of its MPI ranks into one buffer
 * (src/core/htrdr_draw_map.c:186-268); here every rank draws the whole map on
 * its own streams, the accumulators are summed, and htrdr_gpu_finalize_device
 * turns the sum into pixel structs.  `device_accum' (device memory) receives
 * width x height x channels records, then width x height more for the time
 * per realisation, each {sum f64, sum of squares f64, count u64, failures
 * u64} (htrdr_accum, src/core/htrdr_accum.h:31-36); channels = 3 for CIE
 * images, else 1. */
HTRDR_GPU_API htrdr_gpu_res_T
htrdr_gpu_draw_map_accum_device(struct htrdr_gpu_scene* scene, const struct htrdr_gpu_request* req,
                                void* device_accum, struct htrdr_gpu_stats* stats);
/* Pixel structs of a map from its accumulators (the layout of
 * htrdr_gpu_draw_map_accum_device): the estimates and standard errors
 * (htrdr_accum_get_estimation, src/core/htrdr_accum.h:48-68) and, for
 * longwave images, the brightness temperature
 * (src/atmosphere/htrdr_atmosphere_draw_map.c:425-435). */
HTRDR_GPU_API htrdr_gpu_res_T
htrdr_gpu_finalize_device(struct htrdr_gpu_scene* scene, const struct htrdr_gpu_request* req,
                          const void* device_accum, const struct htrdr_gpu_buffer_layout* layout,
                          void* device_buffer);

/* Same as htrdr_gpu_draw_map_device without allocating device memory, for
 * callers that cannot allocate while they render (an application that owns
 * all of HBM through its own pool, a loop that must not pay for the device
 * synchronisation of cudaFree).  No counterpart in the reference.  Scratch
 * (FP64 accumulators, counters, sampler tables) lives in fixed static device
 * arrays: pixels x (channels + 1) <= 65536 and a wavelength CDF of at most
 * 131072 entries (29127 bands for CIE), else HTRDR_GPU_RES_BAD_ARG.  The
 * first call on a device looks the arrays up (make it before any stream
 * capture); calls whose GPU work overlaps race on the shared arrays. */
HTRDR_GPU_API htrdr_gpu_res_T
htrdr_gpu_draw_map_noalloc(struct htrdr_gpu_scene* scene, const struct htrdr_gpu_request* req,
                           const struct htrdr_gpu_buffer_layout* layout, void* device_buffer);

/* ---- output: the htrdr-image file of a map and the run summaries
 * (dump_buffer and atmosphere_draw_map, src/atmosphere/htrdr_atmosphere_draw_map.c:477-641;
 * format doc/htrdr-image.5).  `buffer' holds the map (host memory, `layout')
 * in the pixel structs of `mode'; `path' is a file name or "-" for stdout.
 * summary (may be NULL): the estimates of the time per radiative path (us)
 * and, for flux maps, of the flux density over all pixels' weights. ---- */
struct htrdr_gpu_map_summary {
  double path_time_E, path_time_SE;
  double flux_E, flux_SE;
  uint64_t path_time_n, flux_n;
};
HTRDR_GPU_API htrdr_gpu_res_T
htrdr_gpu_write_image(int mode, const struct htrdr_gpu_buffer_layout* layout, const void* buffer,
                      const char* path, struct htrdr_gpu_map_summary* summary);

/* ---- radiance routines, batched: atmosphere_compute_radiance_sw / _lw
 * (src/atmosphere/htrdr_atmosphere_c.h:140-163).  Ray i uses the random
 * stream keyed by (i, seed).  out[i] in W/m^2/sr/m. ---- */
HTRDR_GPU_API htrdr_gpu_res_T
htrdr_gpu_radiance_sw(struct htrdr_gpu_scene* scene, size_t n, const double* pos,
                      const double* dir, const double* wlen, const uint32_t* iband,
                      const uint32_t* iquad, int cpnt_mask, uint32_t seed, double* out);
HTRDR_GPU_API htrdr_gpu_res_T
htrdr_gpu_radiance_lw(struct htrdr_gpu_scene* scene, size_t n, const double* pos,
                      const double* dir, const double* wlen, const uint32_t* iband,
                      const uint32_t* iquad, uint32_t seed, double* out);

/* Per-realisation weights of pixels [pix_begin, pix_end) of a request
 * (NaN for rejected samples): one-to-one comparison with a CPU restatement. */
HTRDR_GPU_API htrdr_gpu_res_T
htrdr_gpu_realisation_weights(struct htrdr_gpu_scene* scene, const struct htrdr_gpu_request* req,
                              size_t pix_begin, size_t pix_end, double* weights);

/* ---- integer work, exposed for bit-exact checks ---- */
/* htsky_find_spectral_band (called at src/atmosphere/htrdr_atmosphere_draw_map.c:176) */
HTRDR_GPU_API htrdr_gpu_res_T
htrdr_gpu_find_band(struct htrdr_gpu_scene* scene, size_t n, const double* wlen, uint32_t* out);
/* htsky_spectral_band_sample_quadrature (draw_map.c:177) */
HTRDR_GPU_API htrdr_gpu_res_T
htrdr_gpu_sample_quad(struct htrdr_gpu_scene* scene, size_t n, const double* r,
                      const uint32_t* iband, uint32_t* out);
/* Octree point location: leaf node index and level of integer cells [n][3] */
HTRDR_GPU_API htrdr_gpu_res_T
htrdr_gpu_locate_leaf(struct htrdr_gpu_scene* scene, uint32_t iband, uint32_t iquad, int prop,
                      size_t n, const uint32_t* cells, uint32_t* node, uint32_t* level);
/* Ground ray queries (htrdr_atmosphere_ground_trace_ray,
 * src/atmosphere/htrdr_atmosphere_ground.c:162-209, with the self-hit filter
 * of src/core/htrdr_geometry.c:114-150): rays [n] {org[3], dir[3]} (FP32),
 * range [0, tmax[i]), from_prim[i] the primitive the ray leaves (UINT32_MAX:
 * none) and from_edge[i] whether that hit lay on an edge.  Out: the hit
 * primitive (UINT32_MAX: no hit) and distance. */
HTRDR_GPU_API htrdr_gpu_res_T
htrdr_gpu_ground_trace(struct htrdr_gpu_scene* scene, size_t n, const float* rays, const float* tmax,
                       const uint32_t* from_prim, const uint8_t* from_edge, uint32_t* prim,
                       float* dist);
/* Wavelength sampling of a request (htrdr_ran_wlen_planck_sample /
 * htrdr_ran_wlen_cie_xyz_sample_{X,Y,Z}): CDF band index, wavelength, pdf. */
HTRDR_GPU_API htrdr_gpu_res_T
htrdr_gpu_sample_wavelength(struct htrdr_gpu_scene* scene, const struct htrdr_gpu_request* req,
                            int channel, size_t n, const double* r0, const double* r1,
                            uint32_t* cdf_band, double* wlen, double* pdf);

/* ---- batched engine: many requests in one persistent kernel ---- */
struct htrdr_gpu_batch_item {
  struct htrdr_gpu_scene* scene;
  struct htrdr_gpu_request req;
  struct htrdr_gpu_buffer_layout layout;
  void* buffer; /* host */
};
struct htrdr_gpu_tuning {
  uint32_t block_size;    /* threads per block of the persistent kernel (wavefront: of its
                           * trace stage) */
  uint32_t queue_chunk;   /* realisations taken from the work queue at once (persistent) */
  uint32_t regroup_period;/* voxel steps between two regroupings of a warp's lanes (events and
                           * new realisations run together; 0 or 1: every step) (persistent, and
                           * the megakernel that finishes a wavefront run) */
  uint32_t blocks_per_sm; /* resident blocks per SM (0: occupancy maximum) */
  uint32_t engine;        /* HTRDR_GPU_ENGINE_PERSISTENT, _WAVEFRONT or _SORTED */
  uint32_t wave_slots;    /* wavefront: paths in flight (0: 2^21, at most the realisations) */
  uint32_t trace_budget;  /* wavefront: voxel steps of a trace per trace-stage visit (0: 256) */
  uint32_t wave_tail;     /* wavefront: live paths below which the remaining ones finish in one
                           * megakernel launch (0: four waves of its resident threads) */
};
/* Renders every item (each one htrdr_draw_map call of the reference) in one
 * persistent kernel; item buffers are host memory.  tuning == NULL: the
 * default of the items' modes (htrdr_gpu_mode_tuning; SW/CIE wins when mixed). */
HTRDR_GPU_API htrdr_gpu_res_T
htrdr_gpu_draw_maps_batched(struct htrdr_gpu_batch_item* items, size_t n,
                            const struct htrdr_gpu_tuning* tuning, struct htrdr_gpu_stats* stats);
/* Same, item buffers are device memory (no host copy). */
HTRDR_GPU_API htrdr_gpu_res_T
htrdr_gpu_draw_maps_batched_device(struct htrdr_gpu_batch_item* items, size_t n,
                                   const struct htrdr_gpu_tuning* tuning,
                                   struct htrdr_gpu_stats* stats);
/* Same, each item's `buffer' (device memory) receiving the request's FP64
 * accumulators in the layout of htrdr_gpu_draw_map_accum_device instead of
 * its pixel structs (its `layout' is not used): the maps of several processes
 * or GPUs are summed and finalized once with htrdr_gpu_finalize_device. */
HTRDR_GPU_API htrdr_gpu_res_T
htrdr_gpu_draw_maps_batched_accum_device(struct htrdr_gpu_batch_item* items, size_t n,
                                         const struct htrdr_gpu_tuning* tuning,
                                         struct htrdr_gpu_stats* stats);
HTRDR_GPU_API void htrdr_gpu_default_tuning(struct htrdr_gpu_tuning* tuning);
/* Default tuning of a request mode: the wavefront engine (trace-stage blocks
 * of 256, 256 voxel steps per visit, 2^21 path slots), its tail megakernel
 * taking over below 25 000 live paths for SW, 100 000 for CIE and LW. */
HTRDR_GPU_API void htrdr_gpu_mode_tuning(int mode, struct htrdr_gpu_tuning* tuning);
/* Autotuner: times the candidate tunings (persistent: block size, queue
 * chunk, regroup period; wavefront: tail threshold, regroup period) on
 * `items' (device buffers) and returns the fastest; the rendered values do
 * not depend on the tuning. */
HTRDR_GPU_API htrdr_gpu_res_T
htrdr_gpu_autotune(struct htrdr_gpu_batch_item* items, size_t n, struct htrdr_gpu_tuning* best,
                   double* best_ms);

/* Reusable batch (item buffers are device memory): the launch sequence is
 * captured once in a CUDA graph; every run replays it.  The tuning's engine
 * must be the persistent one (the wavefront's iteration count is decided on
 * the host while it runs): BAD_ARG otherwise. */
struct htrdr_gpu_batch;
HTRDR_GPU_API htrdr_gpu_res_T
htrdr_gpu_batch_create(const struct htrdr_gpu_batch_item* items, size_t n,
                       const struct htrdr_gpu_tuning* tuning, struct htrdr_gpu_batch** batch);
HTRDR_GPU_API htrdr_gpu_res_T
htrdr_gpu_batch_run(struct htrdr_gpu_batch* batch, struct htrdr_gpu_stats* stats);
HTRDR_GPU_API void htrdr_gpu_batch_release(struct htrdr_gpu_batch* batch);

/* ---- serving: a request loop with continuous batching ----
 * Requests (scene, request, layout, host buffer) are submitted at any time.
 * A scheduling thread admits them while their device memory (FP64
 * accumulators + output staging) fits in the HBM budget, keeps their
 * accumulators resident, and feeds a fair share of every admitted request's
 * remaining realisations to the engine: rounds of the persistent kernel, or
 * the wavefront's work queue, whose path slots take the realisations of newly
 * admitted requests as soon as their paths end.  Requests that arrive while
 * others render join the running work.  A request completes when all its
 * realisations are accumulated: its map is copied to its host buffer. */
struct htrdr_gpu_server_config {
  int device;
  size_t hbm_budget_bytes;       /* admission budget for per-request device memory */
  double round_target_ms;        /* rounds hold ~ this much work at the observed throughput */
  uint64_t round_realisations;   /* smallest round (0: two waves of the kernel's resident threads) */
  struct htrdr_gpu_tuning tuning;  /* persistent: rounds of the megakernel on three streams;
                                    * wavefront: one pool of path slots fed by a growing
                                    * queue (wave_slots paths, held for the server's
                                    * lifetime) */
};
struct htrdr_gpu_server_stats {
  uint64_t submitted, completed, failed, rounds, realisations;
  double p50_ms, p99_ms, mean_ms, max_ms; /* submit -> map in the host buffer */
  double busy_ms;                         /* device time of the rounds */
  double wall_ms;                         /* first submit -> last completion */
  size_t hbm_peak_bytes;
};
HTRDR_GPU_API htrdr_gpu_res_T
htrdr_gpu_server_create(const struct htrdr_gpu_server_config* config,
                        struct htrdr_gpu_server** server);
HTRDR_GPU_API htrdr_gpu_res_T
htrdr_gpu_server_submit(struct htrdr_gpu_server* server, struct htrdr_gpu_scene* scene,
                        const struct htrdr_gpu_request* req,
                        const struct htrdr_gpu_buffer_layout* layout, void* host_buffer,
                        uint64_t* ticket);
/* *done = 1 once the request's map is in its host buffer; *result its res_T */
HTRDR_GPU_API htrdr_gpu_res_T
htrdr_gpu_server_poll(struct htrdr_gpu_server* server, uint64_t ticket, int* done,
                      htrdr_gpu_res_T* result);
/* Blocks until the request completes (or timeout_s elapses: BAD_OP) */
HTRDR_GPU_API htrdr_gpu_res_T
htrdr_gpu_server_wait(struct htrdr_gpu_server* server, uint64_t ticket, double timeout_s,
                      htrdr_gpu_res_T* result);
HTRDR_GPU_API htrdr_gpu_res_T
htrdr_gpu_server_stats(struct htrdr_gpu_server* server, struct htrdr_gpu_server_stats* stats);
/* Launches of the request loop (persistent rounds or wavefront chunks,
 * numbered from 0 in launch order) that carried a request: `first', the
 * first with some of its realisations queued, and `last', the last before
 * all of them were known done.  Two requests whose ranges intersect had work
 * on the device in the same launch (continuous batching).  No counterpart in
 * the reference.  HTRDR_GPU_RES_BAD_OP: the request never reached the device. */
HTRDR_GPU_API htrdr_gpu_res_T
htrdr_gpu_server_request_launches(struct htrdr_gpu_server* server, uint64_t ticket,
                                  uint64_t* first, uint64_t* last);
/* Drains the submitted requests, then stops the scheduling thread */
HTRDR_GPU_API void htrdr_gpu_server_release(struct htrdr_gpu_server* server);

/* ---- library info ---- */
HTRDR_GPU_API const char* htrdr_gpu_version(void);
HTRDR_GPU_API int htrdr_gpu_device_count(void);
HTRDR_GPU_API const char* htrdr_gpu_last_error(void);

#ifdef __cplusplus
}
#endif

#endif /* HTRDR_GPU_H */
