/* Batched engine: many draw_map requests (images, flux maps, spectral
 * domains, scenes) in ONE persistent kernel fed by a device work queue.
 *
 * A launch covers items -- ranges of realisations of requests -- whose
 * realisations form one index space (item-major, realisation-major inside a
 * request).  Each resident thread owns one path slot; when its path ends it
 * takes the next realisation from its private chunk of the queue, refilled
 * `queue_chunk' realisations at a time by one warp-aggregated atomic.  Paths
 * of very different lengths therefore never leave lanes idle while work
 * remains (path regeneration), and the weight of each realisation is the same
 * as in the one-thread-per-realisation kernel because both run the same state
 * machine on the same stream.
 *
 * Lanes are regrouped by warp ballot: lanes whose trace ended (scattering
 * events, sun sampling, accumulation) and idle lanes (new realisations) wait
 * and are served together once every `regroup_period' voxel steps, or as soon
 * as no lane of the warp is tracing, so that the long sampling code runs with
 * many lanes at once while the tracing lanes keep stepping.
 *
 * Entry points: one-shot htrdr_gpu_draw_maps_batched(_device), the reusable
 * htrdr_gpu_batch_* object whose launch sequence is captured once in a CUDA
 * graph and replayed, and the autotuner.  The one-shot entry points and the
 * autotuner also run the same items on the wavefront engine (wavefront.cu)
 * when the tuning selects it. */
#include "engine.cuh"

#include <algorithm>
#include <map>
#include <memory>
#include <cstring>

namespace hg {

/* The persistent loop over one lane's path `p' (in registers or in shared
 * memory: see k_persistent) */
template <unsigned V>
__device__ __forceinline__ void
persistent_loop(PTables& T, Path& p)
{
  const unsigned lane = threadIdx.x & 31u;
  p.state = ST_IDLE;
  p.flags = 0;
  p.c_seg = p.c_node = p.c_tc = 0;
  p.ri = p.si = 0;             /* request and scene of the current path */
  uint64_t wcur = 0, wend = 0; /* private chunk of the queue */
  bool drained = false;
  unsigned long long seg = 0, node = 0, tc = 0, real = 0, fail = 0;
  const uint32_t period = T.regroup_period > 1 ? T.regroup_period : 1;

  for(uint32_t it = 0;; ++it) {
    const unsigned tmask = __ballot_sync(0xffffffffu, p.state == ST_TRACE);
    if(tmask && (it % period) != 0) { /* not a regrouping step: tracing lanes only */
      if(p.state == ST_TRACE) trace_step<V>(p, T.scenes[p.si]);
      continue;
    }
    /* refill the private chunk of lanes that are idle with nothing left */
    const bool need = p.state == ST_IDLE && wcur >= wend && !drained;
    const unsigned m = __ballot_sync(0xffffffffu, need);
    if(m) {
      const unsigned leader = __ffs(m) - 1;
      unsigned long long base = 0;
      if(lane == leader) base = atomicAdd(T.next, (unsigned long long)__popc(m) * T.chunk);
      base = __shfl_sync(0xffffffffu, base, leader);
      if(need) {
        const unsigned rank = __popc(m & ((1u << lane) - 1u));
        wcur = base + (unsigned long long)rank * T.chunk;
        wend = wcur + T.chunk;
        if(wend > T.total) wend = T.total;
        if(wcur >= T.total) { drained = true; wcur = wend = T.total; }
      }
    }
    if(p.state == ST_IDLE && wcur < wend) path_assign(p, T, wcur++);
    if(!__any_sync(0xffffffffu, p.state != ST_IDLE)) break;
    if(p.state != ST_IDLE) {
      const DRequest& R = T.reqs[p.ri];
      const DScene& S = T.scenes[p.si];
      if(p.state != ST_TRACE && p.state != ST_DONE) {
        path_event<V>(p, S, R);
        seg += p.c_seg; node += p.c_node; tc += p.c_tc;
        p.c_seg = p.c_node = p.c_tc = 0;
      }
      if(p.state == ST_TRACE) {
        trace_step<V>(p, S);
      } else if(p.state == ST_DONE) {
        accumulate_b(p, R);
        count_grid(T.cnt, p);
        real += (p.flags & (PF_REJECTED | PF_FAILED)) ? 0 : 1;
        fail += (p.flags & PF_FAILED) ? 1 : 0;
        seg += p.c_seg; node += p.c_node; tc += p.c_tc;
        p.c_seg = p.c_node = p.c_tc = 0;
        p.state = ST_IDLE;
      }
    }
  }
  seg += p.c_seg; node += p.c_node; tc += p.c_tc;
  flush_counts(T.cnt, seg, node, tc, real, fail);
}

template <unsigned V>
__global__ void __maxnreg__(HG_PERSIST_MAXNREG)
k_persistent(PTables T, int tables_in_smem)
{
  /* the scene and request views are read on every step: keep them in shared
   * memory when they fit (one copy per block), after the block's paths when
   * these live there too */
  extern __shared__ __align__(16) unsigned char smem[];
  if constexpr(persistent_smem_paths(V)) {
    PathSlot* slots = (PathSlot*)smem;
    if(tables_in_smem) tables_to_smem(T, smem + path_slots_bytes(blockDim.x));
    persistent_loop<V>(T, slots[threadIdx.x].p);
  } else {
    if(tables_in_smem) tables_to_smem(T, smem);
    Path p;
    persistent_loop<V>(T, p);
  }
}

template <unsigned V>
__global__ void __maxnreg__(HG_PERSIST_MAXNREG)
k_sorted(PTables T, int tables_in_smem)
{
  extern __shared__ __align__(16) unsigned char smem[];
  PathSlot* slots = (PathSlot*)smem;
  uint32_t* lists = (uint32_t*)(smem + path_slots_bytes(blockDim.x));
  if(tables_in_smem)
    tables_to_smem(T, smem + path_slots_bytes(blockDim.x) + sorted_lists_bytes(blockDim.x));
  sorted_loop<V>(T, slots, lists);
}

using PersistentFn = void (*)(PTables, int);
static PersistentFn
persistent_fn(uint32_t v)
{
  HG_PICK_VARIANT(v, k_persistent)
}

static PersistentFn
sorted_fn(uint32_t v)
{
  HG_PICK_VARIANT(v, k_sorted)
}

bool
valid_tuning(const htrdr_gpu_tuning& t)
{
  return t.block_size && t.block_size <= 512 && !(t.block_size & 31) && t.queue_chunk
      && (t.engine == HTRDR_GPU_ENGINE_PERSISTENT || t.engine == HTRDR_GPU_ENGINE_WAVEFRONT
          || t.engine == HTRDR_GPU_ENGINE_SORTED);
}

cudaError_t
launch_persistent(const PTables& T, uint32_t block_size, uint32_t blocks_per_sm, int device,
                  cudaStream_t st, bool sorted)
{
  static_assert(sizeof(DScene) % 4 == 0 && sizeof(DRequest) % 4 == 0, "word copies");
  if(!T.total) return cudaSuccess;
  const size_t tables = ((T.nscenes * sizeof(DScene) + 15) & ~(size_t)15) + T.nreqs * sizeof(DRequest);
  const int in_smem = tables <= 96 * 1024;
  const uint32_t v = hv_make((T.variant & HV_MESH) != 0, T.variant);
  const size_t paths = sorted ? path_slots_bytes(block_size) + sorted_lists_bytes(block_size)
                              : (persistent_smem_paths(v) ? path_slots_bytes(block_size) : 0);
  const size_t smem = (in_smem ? tables : 0) + paths;
  auto kern = sorted ? sorted_fn(v) : persistent_fn(v);
  if(smem > 227 * 1024) return cudaErrorInvalidConfiguration; /* block too large for its paths */
  if(smem > 48 * 1024) {
    const cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                               (int)smem);
    if(e != cudaSuccess) return e;
  }
  int nsm = 0, per_sm = 0;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, (int)block_size, smem);
  if(blocks_per_sm) per_sm = std::min(per_sm, (int)blocks_per_sm);
  per_sm = std::max(per_sm, 1);
  kern<<<(unsigned)(nsm * per_sm), block_size, smem, st>>>(T, in_smem);
  note_launches(1);
  return cudaGetLastError();
}

struct SingleTables {
  DScene scene;
  DRequest req;
  PItem item;
  uint64_t offsets[2];
};

size_t
single_tables_bytes()
{
  return sizeof(SingleTables);
}

cudaError_t
launch_workqueue(const PTables& T0, const htrdr_gpu_tuning& tun, WaveBufs* wave, int device,
                 cudaStream_t st)
{
  PTables T = T0;
  T.chunk = tun.queue_chunk;
  T.regroup_period = tun.regroup_period;
  if(tun.engine == HTRDR_GPU_ENGINE_WAVEFRONT) {
    if(!wave) return cudaErrorInvalidValue;
    return launch_wavefront(T, tun, *wave, device, st);
  }
  return launch_persistent(T, tun.block_size, tun.blocks_per_sm, device, st,
                           tun.engine == HTRDR_GPU_ENGINE_SORTED);
}

cudaError_t
launch_workqueue_single(const DScene& S, const DRequest& R, void* tables, void* cnt,
                        const htrdr_gpu_tuning& tun, WaveBufs* wave, int device, cudaStream_t st)
{
  SingleTables h;
  h.scene = S;
  h.req = R;
  h.item = PItem{0, 0, 0};
  h.offsets[0] = 0;
  h.offsets[1] = (uint64_t)R.width * R.height * R.nreal_pp;
  /* a pageable source is staged before the call returns: `h' may go */
  cudaError_t e = cudaMemcpyAsync(tables, &h, sizeof(h), cudaMemcpyHostToDevice, st);
  if(e != cudaSuccess) return e;
  const SingleTables* d = (const SingleTables*)tables;
  PTables T{};
  T.scenes = &d->scene;
  T.reqs = &d->req;
  T.items = &d->item;
  T.offsets = d->offsets;
  T.nscenes = 1;
  T.variant = hv_make(S.g_ntris != 0, hv_kind(R.mode));
  T.nreqs = 1;
  T.nitems = 1;
  T.total = h.offsets[1];
  T.cnt = cnt;
  T.next = (unsigned long long*)((char*)cnt + 64);
  return launch_workqueue(T, tun, wave, device, st);
}

/* Threads the persistent kernel keeps resident on the device */
uint64_t
persistent_capacity(uint32_t block_size, uint32_t blocks_per_sm, int device)
{
  int nsm = 0, per_sm = 0;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_persistent<HV_ALL>, (int)block_size, 0);
  if(blocks_per_sm) per_sm = std::min(per_sm, (int)blocks_per_sm);
  return (uint64_t)std::max(per_sm, 1) * (uint64_t)nsm * block_size;
}

/* Device buffers of a plan: tables, accumulators, counters, output staging */
struct PlanBufs {
  DevBuf d_scenes, d_reqs, d_items, d_offsets, d_acc, d_cnt, d_out;
};

/* Grow-only buffers of the one-shot calls of a host thread on a device (one
 * call at a time per thread): a call reuses those of the last one, as
 * freeing device memory after every call cost up to 0.6 s of host time */
PlanBufs&
thread_plan_bufs(int device)
{
  static thread_local std::map<int, std::unique_ptr<PlanBufs>> bufs;
  std::unique_ptr<PlanBufs>& b = bufs[device];
  if(!b) b = std::make_unique<PlanBufs>();
  return *b;
}

/* `b' holding at least `n' bytes (its contents are not kept) */
bool
reserve(DevBuf& b, size_t n)
{
  if(b.ptr && b.bytes >= n) return true;
  if(b.ptr) { cudaFree(b.ptr); b.ptr = nullptr; b.bytes = 0; }
  return b.alloc(n);
}

bool
fill(DevBuf& b, const void* src, size_t n)
{
  return reserve(b, n) && (!n || cuda_ok(cudaMemcpy(b.ptr, src, n, cudaMemcpyHostToDevice), "cudaMemcpy H2D"));
}

/* Device state of a set of items: tables, accumulators, counters */
struct Plan {
  int device = 0;
  std::vector<DRequest> reqs;
  std::vector<DScene> scenes;
  std::vector<PItem> items;
  std::vector<uint64_t> offsets;
  std::vector<size_t> out_off;
  PlanBufs own;           /* a reusable batch's buffers (its graph holds their addresses) */
  PlanBufs* B = &own;     /* the buffers in use: `own', or the thread's for a one-shot call */
  size_t acc_bytes = 0;
  bool accum_out = false; /* the items' buffers receive the accumulators */
  std::vector<size_t> item_acc_bytes;
  PTables T{};
  WaveBufs* wave = nullptr; /* path slots of the wavefront engine (the thread's pool) */
};

static htrdr_gpu_res_T
plan_build(Plan& P, const htrdr_gpu_batch_item* items, size_t n, bool host_out,
           bool accum_out = false, bool one_shot = true)
{
  const int device = items[0].scene ? items[0].scene->device : -1;
  for(size_t i = 0; i < n; ++i) {
    if(!items[i].scene || items[i].scene->device != device || !items[i].buffer)
      return HTRDR_GPU_RES_BAD_ARG;
    const htrdr_gpu_buffer_layout& L = items[i].layout;
    const htrdr_gpu_request& q = items[i].req;
    if(!accum_out && check_layout(&q, &L) != HTRDR_GPU_RES_OK) return HTRDR_GPU_RES_BAD_ARG;
    if(accum_out && (q.mode < 0 || q.mode > 4 || !q.width || !q.height)) return HTRDR_GPU_RES_BAD_ARG;
  }
  P.accum_out = accum_out;
  if(!cuda_ok(cudaSetDevice(device), "cudaSetDevice")) return HTRDR_GPU_RES_BAD_OP;
  P.device = device;
  P.wave = &thread_wave(device);
  if(one_shot) P.B = &thread_plan_bufs(device);
  PlanBufs& B = *P.B;
  P.reqs.resize(n);
  P.items.resize(n);
  P.offsets.assign(n + 1, 0);
  P.out_off.assign(n, 0);
  std::vector<htrdr_gpu_scene*> scene_ptrs;
  std::vector<uint64_t> acc_off(n);
  uint64_t acc_total = 0;
  size_t out_bytes = 0;
  for(size_t i = 0; i < n; ++i) {
    htrdr_gpu_res_T res = make_drequest(items[i].scene, &items[i].req, &P.reqs[i]);
    if(res != HTRDR_GPU_RES_OK) return res;
    auto it = std::find(scene_ptrs.begin(), scene_ptrs.end(), items[i].scene);
    uint32_t si;
    if(it == scene_ptrs.end()) {
      si = (uint32_t)scene_ptrs.size();
      scene_ptrs.push_back(items[i].scene);
      P.scenes.push_back(items[i].scene->d);
    } else {
      si = (uint32_t)(it - scene_ptrs.begin());
    }
    const uint64_t npix = (uint64_t)P.reqs[i].width * P.reqs[i].height;
    const uint32_t nch = P.reqs[i].mode == HG_IMAGE_CIE ? 3u : 1u;
    acc_off[i] = acc_total;
    acc_total += npix * (nch + 1);
    P.items[i] = PItem{(uint32_t)i, si, 0};
    P.offsets[i + 1] = P.offsets[i] + npix * P.reqs[i].nreal_pp;
    P.out_off[i] = out_bytes;
    if(host_out) out_bytes += (items[i].layout.pitch * items[i].layout.height + 255) & ~(size_t)255;
  }
  P.acc_bytes = accum_out ? 0 : acc_total * sizeof(DAccum);
  if((!accum_out && !reserve(B.d_acc, P.acc_bytes)) || !reserve(B.d_cnt, 128) || !reserve(B.d_out, out_bytes))
    return HTRDR_GPU_RES_MEM_ERR;
  P.item_acc_bytes.assign(n, 0);
  for(size_t i = 0; i < n; ++i) {
    const uint64_t npix = (uint64_t)P.reqs[i].width * P.reqs[i].height;
    const uint32_t nch = P.reqs[i].mode == HG_IMAGE_CIE ? 3u : 1u;
    P.reqs[i].acc = accum_out ? (DAccum*)items[i].buffer : (DAccum*)B.d_acc.ptr + acc_off[i];
    P.reqs[i].tacc = P.reqs[i].acc + npix * nch;
    P.item_acc_bytes[i] = npix * (nch + 1) * sizeof(DAccum);
  }
  if(!fill(B.d_scenes, P.scenes.data(), P.scenes.size() * sizeof(DScene))
  || !fill(B.d_reqs, P.reqs.data(), n * sizeof(DRequest))
  || !fill(B.d_items, P.items.data(), n * sizeof(PItem))
  || !fill(B.d_offsets, P.offsets.data(), (n + 1) * 8))
    return HTRDR_GPU_RES_MEM_ERR;
  PTables& T = P.T;
  T.scenes = (const DScene*)B.d_scenes.ptr;
  T.reqs = (const DRequest*)B.d_reqs.ptr;
  T.items = (const PItem*)B.d_items.ptr;
  T.offsets = (const uint64_t*)B.d_offsets.ptr;
  T.nscenes = (uint32_t)P.scenes.size();
  T.variant = tables_variant(P.scenes, P.reqs);
  T.nreqs = (uint32_t)n;
  T.nitems = (uint32_t)n;
  T.total = P.offsets[n];
  T.cnt = B.d_cnt.ptr;
  T.next = (unsigned long long*)((char*)B.d_cnt.ptr + 64);
  return HTRDR_GPU_RES_OK;
}

/* Launch sequence of a plan: clear, work-queue engine, finalize into the
 * items' output buffers (device) or the plan's staging (host copies after). */
static bool
plan_enqueue(Plan& P, const htrdr_gpu_batch_item* items, size_t n, const htrdr_gpu_tuning& tun,
             bool host_out, cudaStream_t st, cudaEvent_t k0, cudaEvent_t k1, bool capturing = false)
{
  bool ok = cuda_ok(cudaMemsetAsync(P.B->d_cnt.ptr, 0, 128, st), "memset");
  if(!P.accum_out)
    ok = ok && cuda_ok(cudaMemsetAsync(P.B->d_acc.ptr, 0, P.acc_bytes, st), "memset");
  for(size_t i = 0; ok && P.accum_out && i < n; ++i)
    ok = cuda_ok(cudaMemsetAsync(P.reqs[i].acc, 0, P.item_acc_bytes[i], st), "memset");
  /* inside a stream capture an event record must be an external node to time
   * the replays */
  const unsigned evf = capturing ? cudaEventRecordExternal : cudaEventRecordDefault;
  if(ok && k0) ok = cuda_ok(cudaEventRecordWithFlags(k0, st, evf), "event");
  if(ok) ok = cuda_ok(launch_workqueue(P.T, tun, P.wave, P.device, st),
                      tun.engine == HTRDR_GPU_ENGINE_WAVEFRONT ? "wavefront" : "k_persistent");
  if(ok && k1) ok = cuda_ok(cudaEventRecordWithFlags(k1, st, evf), "event");
  for(size_t i = 0; ok && !P.accum_out && i < n; ++i) {
    char* dout = host_out ? (char*)P.B->d_out.ptr + P.out_off[i] : (char*)items[i].buffer;
    ok = cuda_ok(launch_finalize(P.reqs[i], P.reqs[i].acc, P.reqs[i].tacc, dout,
                                 items[i].layout.pitch, st), "k_finalize");
    if(ok && host_out)
      ok = cuda_ok(cudaMemcpyAsync(items[i].buffer, dout, items[i].layout.pitch * items[i].layout.height,
                                   cudaMemcpyDeviceToHost, st), "D2H");
  }
  return ok;
}

static void
read_stats(const unsigned long long c[6], float kms, float tms, uint64_t launches,
           htrdr_gpu_stats* stats)
{
  if(!stats) return;
  stats->segments = c[0]; stats->nodes = c[1]; stats->collisions = c[2];
  stats->realisations = c[3]; stats->failures = c[4]; stats->grid_bytes = c[5];
  stats->kernel_ms = kms; stats->total_ms = tms;
  stats->launches = launches;
}

}  // namespace hg

using namespace hg;

extern "C" HTRDR_GPU_API void
htrdr_gpu_default_tuning(htrdr_gpu_tuning* t)
{
  if(!t) return;
  t->block_size = 128;
  t->queue_chunk = 4;
  t->regroup_period = 1;
  t->blocks_per_sm = 0;
  t->engine = HTRDR_GPU_ENGINE_PERSISTENT;
  t->wave_slots = 0;
  t->trace_budget = 0;
  t->wave_tail = 0;
}

/* Best tunings measured on a B200: the wavefront for every mode (long
 * multiple-scattering walks in the clouds; LW walks run whole in its trace
 * stage: LW flux map 232 Mrealisations/s against 135 for the persistent
 * megakernel).  The tail threshold is where iterations stop paying for their
 * launch and one trace's latency. */
extern "C" HTRDR_GPU_API void
htrdr_gpu_mode_tuning(int mode, htrdr_gpu_tuning* t)
{
  if(!t) return;
  htrdr_gpu_default_tuning(t);
  if(mode == HG_XWAVE_LW || mode == HG_FLUX_LW) {
    t->engine = HTRDR_GPU_ENGINE_WAVEFRONT;
    t->block_size = 256;
    t->queue_chunk = 1;
    t->regroup_period = 64;
    t->trace_budget = 256;
    t->wave_tail = 100000;
  } else if(mode == HG_IMAGE_CIE) {
    t->engine = HTRDR_GPU_ENGINE_WAVEFRONT;
    t->block_size = 256;
    t->queue_chunk = 1;
    t->regroup_period = 16;
    t->trace_budget = 256;
    t->wave_tail = 100000;
  } else {
    t->engine = HTRDR_GPU_ENGINE_WAVEFRONT;
    t->block_size = 256;
    t->queue_chunk = 1;
    t->regroup_period = 64;
    t->trace_budget = 256;
    t->wave_tail = 25000;
  }
}

/* `tuning' if given, else the default of the items' modes (SW/CIE if any) */
static htrdr_gpu_tuning
items_tuning(const htrdr_gpu_batch_item* items, size_t n, const htrdr_gpu_tuning* tuning)
{
  htrdr_gpu_tuning tun;
  if(tuning) return *tuning;
  int sw = 0;
  for(size_t i = 0; i < n; ++i)
    sw |= items[i].req.mode != HG_XWAVE_LW && items[i].req.mode != HG_FLUX_LW;
  htrdr_gpu_mode_tuning(sw ? HG_XWAVE_SW : HG_FLUX_LW, &tun);
  return tun;
}

static htrdr_gpu_res_T
batched_impl(htrdr_gpu_batch_item* items, size_t n, const htrdr_gpu_tuning* tuning,
             htrdr_gpu_stats* stats, bool host, bool accum = false)
{
  if(!items || !n) return HTRDR_GPU_RES_BAD_ARG;
  const htrdr_gpu_tuning tun = items_tuning(items, n, tuning);
  if(!valid_tuning(tun)) return HTRDR_GPU_RES_BAD_ARG;
  take_launches();
  Plan P;
  htrdr_gpu_res_T res = plan_build(P, items, n, host, accum);
  if(res != HTRDR_GPU_RES_OK) return res;
  cudaStream_t st = items[0].scene->stream;
  cudaEvent_t e0, e1, e2, e3;
  cudaEventCreate(&e0); cudaEventCreate(&e1); cudaEventCreate(&e2); cudaEventCreate(&e3);
  cudaEventRecord(e0, st);
  bool ok = plan_enqueue(P, items, n, tun, host, st, e1, e2);
  cudaEventRecord(e3, st);
  unsigned long long c[6] = {0, 0, 0, 0, 0, 0};
  if(ok) ok = cuda_ok(cudaMemcpyAsync(c, P.B->d_cnt.ptr, sizeof(c), cudaMemcpyDeviceToHost, st), "D2H");
  if(ok) ok = cuda_ok(cudaStreamSynchronize(st), "sync");
  if(ok) {
    float k = 0, t = 0;
    cudaEventElapsedTime(&k, e1, e2);
    cudaEventElapsedTime(&t, e0, e3);
    read_stats(c, k, t, take_launches(), stats);
  }
  cudaEventDestroy(e0); cudaEventDestroy(e1); cudaEventDestroy(e2); cudaEventDestroy(e3);
  return ok ? HTRDR_GPU_RES_OK : HTRDR_GPU_RES_UNKNOWN_ERR;
}

extern "C" HTRDR_GPU_API htrdr_gpu_res_T
htrdr_gpu_draw_maps_batched(htrdr_gpu_batch_item* items, size_t n, const htrdr_gpu_tuning* tuning,
                            htrdr_gpu_stats* stats)
try {
  return batched_impl(items, n, tuning, stats, true);
}
HG_API_CATCH("htrdr_gpu_draw_maps_batched")

extern "C" HTRDR_GPU_API htrdr_gpu_res_T
htrdr_gpu_draw_maps_batched_device(htrdr_gpu_batch_item* items, size_t n,
                                   const htrdr_gpu_tuning* tuning, htrdr_gpu_stats* stats)
try {
  return batched_impl(items, n, tuning, stats, false);
}
HG_API_CATCH("htrdr_gpu_draw_maps_batched_device")

extern "C" HTRDR_GPU_API htrdr_gpu_res_T
htrdr_gpu_draw_maps_batched_accum_device(htrdr_gpu_batch_item* items, size_t n,
                                         const htrdr_gpu_tuning* tuning, htrdr_gpu_stats* stats)
try {
  return batched_impl(items, n, tuning, stats, false, true);
}
HG_API_CATCH("htrdr_gpu_draw_maps_batched_accum_device")

/* Autotuner: times every candidate -- persistent megakernel (block size x
 * queue chunk x regroup period) and wavefront (tail threshold x regroup
 * period of its finishing megakernel) -- on the given items (device buffers)
 * with CUDA events and returns the fastest.  Results do not depend on the
 * tuning. */
extern "C" HTRDR_GPU_API htrdr_gpu_res_T
htrdr_gpu_autotune(htrdr_gpu_batch_item* items, size_t n, htrdr_gpu_tuning* best, double* best_ms)
try {
  if(!items || !n || !best) return HTRDR_GPU_RES_BAD_ARG;
  static const uint32_t blocks[] = {96, 128, 256}; /* 96: 3 blocks of 3 warps fill 9 warps at 216 registers */
  static const uint32_t chunks[] = {1, 4};
  static const uint32_t periods[] = {1, 4, 16, 64};
  static const uint32_t tails[] = {25000, 100000};
  static const uint32_t wperiods[] = {16, 64};
  htrdr_gpu_stats st;
  double best_t = 1e300;
  htrdr_gpu_tuning t;
  htrdr_gpu_default_tuning(&t);
  htrdr_gpu_res_T res = batched_impl(items, n, &t, &st, false); /* warm-up */
  if(res != HTRDR_GPU_RES_OK) return res;
  auto time_it = [&](const htrdr_gpu_tuning& c) {
    htrdr_gpu_res_T r = batched_impl(items, n, &c, &st, false);
    if(r == HTRDR_GPU_RES_OK && st.kernel_ms < best_t) { best_t = st.kernel_ms; *best = c; }
    return r;
  };
  for(uint32_t b : blocks) { /* persistent megakernel */
    for(uint32_t c : chunks)
      for(uint32_t p : periods) {
        t.block_size = b;
        t.queue_chunk = c;
        t.regroup_period = p;
        if((res = time_it(t)) != HTRDR_GPU_RES_OK) return res;
      }
  }
  htrdr_gpu_default_tuning(&t);
  t.engine = HTRDR_GPU_ENGINE_WAVEFRONT;
  t.block_size = 256;
  t.queue_chunk = 1;
  t.trace_budget = 256;
  for(uint32_t tl : tails) { /* wavefront: tail threshold x regroup period of its tail */
    for(uint32_t p : wperiods) {
      t.wave_tail = tl;
      t.regroup_period = p;
      if((res = time_it(t)) != HTRDR_GPU_RES_OK) return res;
    }
  }
  if(best_ms) *best_ms = best_t;
  return HTRDR_GPU_RES_OK;
}
HG_API_CATCH("htrdr_gpu_autotune")

/*******************************************************************************
 * Reusable batch: the whole launch sequence (clear, persistent kernel,
 * finalize of every item) captured once in a CUDA graph and replayed.
 ******************************************************************************/
struct htrdr_gpu_batch {
  Plan plan;
  std::vector<htrdr_gpu_batch_item> items;
  cudaStream_t stream = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr, e2 = nullptr, e3 = nullptr;
};

extern "C" HTRDR_GPU_API void
htrdr_gpu_batch_release(htrdr_gpu_batch* b)
{
  if(!b) return;
  cudaSetDevice(b->plan.device);
  if(b->stream) cudaStreamSynchronize(b->stream);
  if(b->exec) cudaGraphExecDestroy(b->exec);
  if(b->graph) cudaGraphDestroy(b->graph);
  if(b->e0) cudaEventDestroy(b->e0);
  if(b->e1) cudaEventDestroy(b->e1);
  if(b->e2) cudaEventDestroy(b->e2);
  if(b->e3) cudaEventDestroy(b->e3);
  if(b->stream) cudaStreamDestroy(b->stream);
  delete b;
}

extern "C" HTRDR_GPU_API htrdr_gpu_res_T
htrdr_gpu_batch_create(const htrdr_gpu_batch_item* items, size_t n, const htrdr_gpu_tuning* tuning,
                       htrdr_gpu_batch** out)
try {
  if(!items || !n || !out) return HTRDR_GPU_RES_BAD_ARG;
  htrdr_gpu_tuning tun = items_tuning(items, n, tuning);
  if(!tuning) tun.engine = HTRDR_GPU_ENGINE_PERSISTENT; /* a mode default may name the wavefront */
  if(!valid_tuning(tun)) return HTRDR_GPU_RES_BAD_ARG;
  if(tun.engine != HTRDR_GPU_ENGINE_PERSISTENT && tun.engine != HTRDR_GPU_ENGINE_SORTED) {
    set_error("graph batches run the persistent engines (the wavefront's iteration count is "
              "decided on the host)");
    return HTRDR_GPU_RES_BAD_ARG;
  }
  auto b = new htrdr_gpu_batch();
  b->items.assign(items, items + n);
  htrdr_gpu_res_T res = plan_build(b->plan, b->items.data(), n, false, false, false);
  if(res != HTRDR_GPU_RES_OK) { htrdr_gpu_batch_release(b); return res; }
  bool ok = cuda_ok(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking), "stream")
         && cuda_ok(cudaEventCreate(&b->e0), "event") && cuda_ok(cudaEventCreate(&b->e1), "event")
         && cuda_ok(cudaEventCreate(&b->e2), "event") && cuda_ok(cudaEventCreate(&b->e3), "event");
  /* the occupancy query and the smem attribute are set outside the capture */
  if(ok) ok = cuda_ok(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal), "capture");
  if(ok) {
    const bool enq = plan_enqueue(b->plan, b->items.data(), n, tun, false, b->stream, b->e1, b->e2, true);
    ok = cuda_ok(cudaStreamEndCapture(b->stream, &b->graph), "end capture") && enq;
  }
  if(ok) ok = cuda_ok(cudaGraphInstantiate(&b->exec, b->graph, 0), "graph instantiate");
  if(!ok) { htrdr_gpu_batch_release(b); return HTRDR_GPU_RES_UNKNOWN_ERR; }
  *out = b;
  return HTRDR_GPU_RES_OK;
}
HG_API_CATCH("htrdr_gpu_batch_create")

/* Replays the captured launch: the items' device buffers receive the maps. */
extern "C" HTRDR_GPU_API htrdr_gpu_res_T
htrdr_gpu_batch_run(htrdr_gpu_batch* b, htrdr_gpu_stats* stats)
try {
  if(!b) return HTRDR_GPU_RES_BAD_ARG;
  cudaSetDevice(b->plan.device);
  unsigned long long c[6] = {0, 0, 0, 0, 0, 0};
  bool ok = cuda_ok(cudaEventRecord(b->e0, b->stream), "event")
         && cuda_ok(cudaGraphLaunch(b->exec, b->stream), "graph launch")
         && cuda_ok(cudaEventRecord(b->e3, b->stream), "event")
         && cuda_ok(cudaMemcpyAsync(c, b->plan.B->d_cnt.ptr, sizeof(c), cudaMemcpyDeviceToHost, b->stream), "D2H")
         && cuda_ok(cudaStreamSynchronize(b->stream), "sync");
  if(!ok) return HTRDR_GPU_RES_UNKNOWN_ERR;
  float k = 0, t = 0;
  cudaEventElapsedTime(&k, b->e1, b->e2);
  cudaEventElapsedTime(&t, b->e0, b->e3);
  read_stats(c, k, t, 1 + b->items.size(), stats); /* persistent kernel + finalizes */
  return HTRDR_GPU_RES_OK;
}
HG_API_CATCH("htrdr_gpu_batch_run")
