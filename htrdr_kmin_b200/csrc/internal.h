/* Internal host-side declarations of the CUDA library. */
#ifndef HTRDR_INTERNAL_H
#define HTRDR_INTERNAL_H

#include <cuda_runtime.h>

#include <exception>
#include <functional>
#include <new>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

#include "../../include/htrdr_gpu.h"
#include "dscene.h"

namespace hg {

void set_error(const std::string& msg);
const char* last_error(); /* of the calling thread */
bool cuda_ok(cudaError_t e, const char* what);

/* Handler of the function-try-block of every C entry point returning a
 * res_T: no C++ exception crosses the C ABI (a host allocation that fails
 * becomes RES_MEM_ERR with the error text set). */
#define HG_API_CATCH(entry)                                                \
  catch(const std::bad_alloc&) {                                           \
    hg::set_error(std::string(entry) + ": out of host memory");            \
    return HTRDR_GPU_RES_MEM_ERR;                                          \
  } catch(const std::exception& ex) {                                      \
    hg::set_error(std::string(entry) + ": " + ex.what());                  \
    return HTRDR_GPU_RES_UNKNOWN_ERR;                                      \
  } catch(...) {                                                           \
    hg::set_error(std::string(entry) + ": unknown exception");             \
    return HTRDR_GPU_RES_UNKNOWN_ERR;                                      \
  }

/* Kernel launches of the calling thread since the last take_launches() */
void note_launches(uint64_t n);
uint64_t take_launches();

/* Device allocation owned by a scene or a request cache */
struct DevBuf {
  void* ptr = nullptr;
  size_t bytes = 0;
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  ~DevBuf();
  bool alloc(size_t n);
  bool upload(const void* src, size_t n);
};

/* Wavelength sampler tables of a request, on the device */
struct Sampler {
  int mode_cie = 0;
  uint32_t ncdf = 0;
  double band_len = 0;
  double rcp_integral[3] = {0, 0, 0};
  DevBuf cdf, pdf, fbound, guide;
  uint32_t nguide = 0;
  std::vector<double> host_cdf; /* for the host-side checks */
};

}  // namespace hg

struct htrdr_gpu_scene {
  int device = 0;
  DScene d{};
  uint32_t nbands = 0, nq = 0, nlayers = 0, props_mask = 0, depth = 0;
  std::vector<double> band_lo, band_hi;
  std::vector<uint32_t> nquads, quad_off;
  std::vector<uint64_t> tree_base, tree_count;
  std::vector<std::unique_ptr<hg::DevBuf>> bufs;
  size_t bytes = 0;
  /* Wavelength samplers keyed by (cie, range0, range1, Tref) */
  std::map<std::tuple<int, double, double, double>, std::unique_ptr<hg::Sampler>> samplers;
  std::mutex mtx;
  cudaStream_t stream = nullptr;
  /* engine of draw_map on this scene (enum htrdr_gpu_engine; engine_set == 0:
   * the mode's default) and the tuning of the work-queue engines
   * (has_tuning == 0: by mode) */
  int engine = HTRDR_GPU_ENGINE_PERSISTENT;
  int engine_set = 0;
  int has_tuning = 0;
  htrdr_gpu_tuning tuning{};
};

namespace hg {

/* Host spectral routines (same definitions as the reference's
 * src/core/htrdr_spectral.h and samplers) */
double wiebelt(double v);
double blackbody_fraction(double l0, double l1, double T);
double fit_bar_1931(int channel, double lambda);
double cie_trapezoid(double lo, double hi, int channel);

/* Sampler of a request (built on first use and cached in the scene) */
Sampler* scene_sampler(htrdr_gpu_scene* scn, const htrdr_gpu_request* req, htrdr_gpu_res_T* res);
/* Fill the device view of a request */
htrdr_gpu_res_T make_drequest(htrdr_gpu_scene* scn, const htrdr_gpu_request* req, DRequest* out);
uint32_t pixel_size(int mode);
/* Output layout of a request: the buffer checks of htrdr_buffer_layout and the
 * mode's pixel struct; every draw_map entry point applies it */
htrdr_gpu_res_T check_layout(const htrdr_gpu_request* req, const htrdr_gpu_buffer_layout* layout);

/* Octree build on the host, bit-exact definition shared with the oracle.
 * Writes nodes[4*i..] = {kmin bits, kmax bits, child, 0}. */
void build_octree(const DScene& hs, const float* lwc, const float* sig3, const float* gas_ka,
                  const float* gas_ks, const int* cl_lo, const int* cl_hi, uint32_t q, int prop,
                  uint32_t depth, uint32_t level_force, double tau, double cmax,
                  std::vector<uint32_t>& nodes);

/* Leaf of every cell of every built octree (octree_gpu.cu): false when the
 * grids do not fit or cannot be indexed (the traversal then descends).
 * `majorants': each cell holds its leaf's kmin/kmax (float2, the ntrees x
 * ncell array first) and level (u8, after it) instead of node << 5 | level. */
bool build_leaf_grids(const DScene& S, const std::vector<uint64_t>& tree_base,
                      const std::vector<uint64_t>& tree_count, DevBuf& grids, std::vector<uint32_t>& rank,
                      bool majorants);

/* Ground mesh: validation, BVH and device tables into S (ground.cpp);
 * `upload' copies a host array to a device buffer owned by the scene */
htrdr_gpu_res_T setup_ground_mesh(const htrdr_gpu_scene_desc* desc, DScene& S,
                                  const std::function<void*(const void*, size_t)>& upload);

/* Octree build on the GPU (octree_gpu.cu), node arrays identical to build_octree */
bool build_octrees_gpu(const DScene& S, const float* d_lwc, const int2* d_cl, const float* d_gka,
                       const float* d_gks, const std::vector<float>& sig3,
                       const std::vector<uint32_t>& band_of,
                       const std::vector<std::pair<uint32_t, int>>& tasks, uint32_t level_force,
                       double tau, double cmax, DevBuf& pool, std::vector<uint64_t>& base,
                       std::vector<uint64_t>& count, cudaStream_t st);

/* Kernel launchers (kernels.cu) */
struct LaunchOut {
  unsigned long long seg = 0, node = 0, tc = 0, real = 0, fail = 0;
  float kernel_ms = 0;
};
cudaError_t launch_plain(const DScene& S, const DRequest& R, DAccum* acc, DAccum* tacc,
                         uint64_t pix_begin, uint32_t npix, double* weights, void* counters,
                         cudaStream_t st);
cudaError_t launch_finalize(const DRequest& R, const DAccum* acc, const DAccum* tacc,
                            void* out, size_t pitch, cudaStream_t st);
cudaError_t launch_radiance(const DScene& S, int lw, size_t n, const double* pos,
                            const double* dir, const double* wlen, const uint32_t* band,
                            const uint32_t* iquad, int mask, uint32_t seed, double* out,
                            cudaStream_t st);
cudaError_t launch_find_band(const DScene& S, size_t n, const double* wlen, uint32_t* out,
                             cudaStream_t st);
cudaError_t launch_sample_quad(const DScene& S, size_t n, const double* r, const uint32_t* band,
                               uint32_t* out, cudaStream_t st);
cudaError_t launch_ground_trace(const DScene& S, size_t n, const float* rays, const float* tmax,
                                const uint32_t* from_prim, const uint8_t* from_edge, uint32_t* prim,
                                float* dist, cudaStream_t st);
cudaError_t launch_locate_leaf(const DScene& S, uint32_t q, int prop, size_t n,
                               const uint32_t* cells, uint32_t* node, uint32_t* level,
                               cudaStream_t st);
cudaError_t launch_sample_wavelength(const DRequest& R, int channel, size_t n, const double* r0,
                                     const double* r1, uint32_t* cb, double* wlen, double* pdf,
                                     cudaStream_t st);

/* Persistent engine (batched.cu).  A launch covers items, each a range of
 * realisations [begin, begin + count) of one request; the realisations of
 * all items form one work queue. */
struct PItem {
  uint32_t req;    /* index into reqs */
  uint32_t scene;  /* index into scenes */
  uint64_t begin;  /* first realisation (request index space) */
};
struct PTables {
  const DScene* scenes;
  const DRequest* reqs;   /* each with its own accumulators */
  const PItem* items;
  const uint64_t* offsets; /* [nitems+1] prefix sums of the items' counts */
  uint32_t nscenes, nreqs, nitems;
  uint64_t total;
  unsigned long long* next; /* queue head (zeroed before the launch) */
  void* cnt;                /* Counters (zeroed before the launch) */
  uint32_t chunk, regroup_period;
  uint32_t variant = HV_ALL; /* kernel variant (HV_* bits): the scenes' ground and the requests' kinds */
};
/* Kernel variant of a launch over these scenes and requests */
inline uint32_t
tables_variant(const std::vector<DScene>& scenes, const std::vector<DRequest>& reqs)
{
  bool mesh = false;
  uint32_t kinds = 0;
  for(const DScene& d : scenes) mesh = mesh || d.g_ntris != 0;
  for(const DRequest& r : reqs) kinds |= hv_kind(r.mode);
  return hv_make(mesh, kinds);
}
cudaError_t launch_persistent(const PTables& T, uint32_t block_size, uint32_t blocks_per_sm,
                              int device, cudaStream_t st, bool sorted = false);
bool valid_tuning(const htrdr_gpu_tuning& t);
uint64_t persistent_capacity(uint32_t block_size, uint32_t blocks_per_sm, int device);
/* One request on the persistent engine.  `tables' (device memory of
 * single_tables_bytes()) receives the launch's scene/request/item tables;
 * `cnt' (device, 128 bytes) holds the counters and the queue head and must be
 * zeroed before the launch. */
size_t single_tables_bytes();

/* Control block of a wavefront run (device) */
struct WCtl {
  uint32_t n_live[2];   /* lengths of the two live lists */
  uint32_t fetch_event; /* next entry of the event stage's input list */
  uint32_t fetch_trace; /* next entry of the trace stage's list */
  uint32_t fetch_finish;/* next entry of the live list taken by the finishing megakernel */
  uint32_t n_dead;      /* free slots on the dead list (serving) */
  uint32_t pad[2];
};

/* Wavefront engine (wavefront.cu): path slots, live lists, control block and
 * the pinned read-back of the live count, kept between runs; `dead' holds
 * the free slots of a serving pool */
struct WaveBufs {
  DevBuf paths, lists, ctl, dead;
  void* host_ctl = nullptr;
  cudaEvent_t ev[2] = {nullptr, nullptr};
  uint32_t P = 0;
  WaveBufs() = default;
  WaveBufs(const WaveBufs&) = delete;
  WaveBufs& operator=(const WaveBufs&) = delete;
  ~WaveBufs();
};
/* Device bytes of one path slot */
size_t wave_slot_bytes();
/* Path slots of the wavefront when the tuning gives none: 2^21 (940 MB).
 * Measured on a B200 (Mrealisations/s, 2^20 / 2^21 slots): full-size mix
 * 1.979 / 2.084, LW flux map 229 / 247. */
constexpr uint32_t kDefaultWaveSlots = 1u << 21;
/* Grow-only slot pool of the calling host thread on `device', for the calls
 * that run the wavefront engine to completion before they return (one call
 * at a time per thread): a call reuses the slots of the last one instead of
 * allocating and freeing some 460 MB of device memory and its pinned control
 * block. */
WaveBufs& thread_wave(int device);
cudaError_t launch_wavefront(const PTables& T, const htrdr_gpu_tuning& tun, WaveBufs& B,
                             int device, cudaStream_t st);
/* Serving pool of P slots driven chunk by chunk (the caller owns the queue):
 * reset = every slot free; revive = free slots join live list 0 (after work
 * was appended); chunk = an even number of event+trace iterations; finish =
 * the live paths complete in one megakernel launch, then reset.  The tail
 * threshold is the tuning's (or its default) for these launch shapes. */
cudaError_t wave_serve_reset(WaveBufs& B, uint32_t P, cudaStream_t st);
cudaError_t wave_serve_revive(WaveBufs& B, cudaStream_t st);
cudaError_t wave_serve_chunk(const PTables& T, const htrdr_gpu_tuning& tun, WaveBufs& B, int device,
                             uint32_t iterations, cudaStream_t st);
cudaError_t wave_serve_finish(const PTables& T, const htrdr_gpu_tuning& tun, WaveBufs& B,
                              int device, cudaStream_t st);
uint64_t wave_serve_tail(const htrdr_gpu_tuning& tun, int device);
/* One launch of a work-queue engine over T: persistent kernel or wavefront
 * (tun.engine; `wave' holds the wavefront's buffers) */
cudaError_t launch_workqueue(const PTables& T, const htrdr_gpu_tuning& tun, WaveBufs* wave,
                             int device, cudaStream_t st);
/* The same for one request; the tables are staged in `tables' */
cudaError_t launch_workqueue_single(const DScene& S, const DRequest& R, void* tables, void* cnt,
                                    const htrdr_gpu_tuning& tun, WaveBufs* wave, int device,
                                    cudaStream_t st);

}  // namespace hg

#endif
