/* Batched engine: many draw_map requests (images, flux maps, spectral
 * domains, scenes) in ONE persistent kernel fed by a device work queue.
 *
 * The realisations of all requests form one index space (request-major,
 * then realisation-major inside a request).  Each resident thread owns one
 * path slot; when its path ends it takes the next realisation from its
 * private chunk of the queue, refilled `queue_chunk` realisations at a time
 * by one warp-aggregated atomic.  Paths of very different lengths therefore
 * never leave lanes idle while work remains (path regeneration), and the
 * weight of each realisation is the same as in the one-thread-per-realisation
 * kernel because both run the same state machine on the same stream.
 *
 * Lanes are regrouped by warp ballot: lanes whose trace ended (scattering
 * events, sun sampling, accumulation) and idle lanes (new realisations) wait
 * and are served together once every `regroup_period' voxel steps, or as soon
 * as no lane of the warp is tracing, so that the long sampling code runs with
 * many lanes at once while the tracing lanes keep stepping. */
#include "internal.h"
#include "transport.cuh"

#include <algorithm>
#include <cstring>

namespace hg {

struct BatchTables {
  const DScene* scenes;       /* [nscenes] */
  const DRequest* reqs;       /* [nreq] */
  const uint32_t* req_scene;  /* [nreq] */
  const uint64_t* offsets;    /* [nreq+1] prefix sums of realisations */
  uint32_t nreq;
  uint64_t total;
  unsigned long long* next;   /* queue head */
  DAccum* acc;
  DAccum* tacc;
  Counters* cnt;
  uint32_t chunk;
  uint32_t regroup_period;
};

__device__ __forceinline__ uint32_t
find_request(const BatchTables& B, uint64_t g)
{
  uint32_t lo = 0, hi = B.nreq; /* last request whose offset <= g */
  while(hi - lo > 1) {
    const uint32_t mid = (lo + hi) >> 1;
    if(__ldg(B.offsets + mid) <= g) lo = mid; else hi = mid;
  }
  return lo;
}

__device__ __forceinline__ void
accumulate_b(const Path& p, const DRequest& R, DAccum* acc, DAccum* tacc)
{
  if(p.flags & PF_REJECTED) return;
  const uint32_t nch = R.mode == HG_IMAGE_CIE ? 3u : 1u;
  DAccum* a = acc + R.acc_base + (size_t)p.pix * nch + p.chan;
  if(p.flags & PF_FAILED) { atomicAdd(&a->pad, 1ull); return; }
  atomicAdd(&a->s, p.weight);
  atomicAdd(&a->s2, p.weight * p.weight);
  atomicAdd(&a->n, 1ull);
  const double us = (double)(gtimer() - p.t0) * 1e-3;
  DAccum* t = tacc + R.tacc_base + p.pix;
  atomicAdd(&t->s, us);
  atomicAdd(&t->s2, us * us);
  atomicAdd(&t->n, 1ull);
}

__global__ void __maxnreg__(HG_PERSIST_MAXNREG)
k_persistent(BatchTables B, uint32_t nscenes, int tables_in_smem)
{
  /* the scene and request views are read on every step: keep them in shared
   * memory when they fit (one copy per block) */
  extern __shared__ __align__(16) unsigned char smem[];
  if(tables_in_smem) {
    DScene* ss = (DScene*)smem;
    DRequest* sr = (DRequest*)(smem + ((nscenes * sizeof(DScene) + 15) & ~(size_t)15));
    const uint32_t* gs = (const uint32_t*)B.scenes;
    const uint32_t* gr = (const uint32_t*)B.reqs;
    for(uint32_t i = threadIdx.x; i < nscenes * sizeof(DScene) / 4; i += blockDim.x) ((uint32_t*)ss)[i] = gs[i];
    for(uint32_t i = threadIdx.x; i < B.nreq * sizeof(DRequest) / 4; i += blockDim.x) ((uint32_t*)sr)[i] = gr[i];
    __syncthreads();
    B.scenes = ss;
    B.reqs = sr;
  }
  const unsigned lane = threadIdx.x & 31u;
  Path p;
  p.state = ST_IDLE;
  p.flags = 0;
  p.c_seg = p.c_node = p.c_tc = 0;
  uint32_t ri = 0;            /* request of the current path */
  uint64_t wcur = 0, wend = 0; /* private chunk of the queue */
  bool drained = false;
  unsigned long long seg = 0, node = 0, tc = 0, real = 0, fail = 0;
  const uint32_t period = B.regroup_period > 1 ? B.regroup_period : 1;

  for(uint32_t it = 0;; ++it) {
    /* Regrouping: lanes whose trace ended (events, accumulation) and idle
     * lanes (new realisations) are served together once every `period'
     * iterations, or as soon as no lane of the warp is tracing; in between,
     * the tracing lanes advance alone, so that the long sensor-sampling and
     * scattering code runs with many lanes at once. */
    const unsigned tmask = __ballot_sync(0xffffffffu, p.state == ST_TRACE);
    if(tmask && (it % period) != 0) {
      if(p.state == ST_TRACE) trace_step(p, B.scenes[__ldg(B.req_scene + ri)]);
      continue;
    }
    /* refill the private chunk of lanes that are idle with nothing left */
    const bool need = p.state == ST_IDLE && wcur >= wend && !drained;
    const unsigned m = __ballot_sync(0xffffffffu, need);
    if(m) {
      const unsigned leader = __ffs(m) - 1;
      unsigned long long base = 0;
      if(lane == leader) base = atomicAdd(B.next, (unsigned long long)__popc(m) * B.chunk);
      base = __shfl_sync(0xffffffffu, base, leader);
      if(need) {
        const unsigned rank = __popc(m & ((1u << lane) - 1u));
        wcur = base + (unsigned long long)rank * B.chunk;
        wend = wcur + B.chunk;
        if(wend > B.total) wend = B.total;
        if(wcur >= B.total) { drained = true; wcur = wend = B.total; }
      }
    }
    if(p.state == ST_IDLE && wcur < wend) {
      const uint64_t g = wcur++;
      ri = find_request(B, g);
      const DRequest& R = B.reqs[ri];
      const uint64_t local = g - __ldg(B.offsets + ri);
      const uint32_t npix = R.width * R.height;
      p.ireal = (uint32_t)(local / npix);
      p.pix = (uint32_t)(local % npix);
      p.state = ST_GEN;
    }
    if(!__any_sync(0xffffffffu, p.state != ST_IDLE)) break;
    if(p.state != ST_IDLE) {
      const DRequest& R = B.reqs[ri];
      const DScene& S = B.scenes[__ldg(B.req_scene + ri)];
      if(p.state != ST_TRACE && p.state != ST_DONE) {
        path_event(p, S, R);
        seg += p.c_seg; node += p.c_node; tc += p.c_tc;
        p.c_seg = p.c_node = p.c_tc = 0;
      }
      if(p.state == ST_TRACE) {
        trace_step(p, S);
      } else if(p.state == ST_DONE) {
        accumulate_b(p, R, B.acc, B.tacc);
        real += (p.flags & (PF_REJECTED | PF_FAILED)) ? 0 : 1;
        fail += (p.flags & PF_FAILED) ? 1 : 0;
        seg += p.c_seg; node += p.c_node; tc += p.c_tc;
        p.c_seg = p.c_node = p.c_tc = 0;
        p.state = ST_IDLE;
      }
    }
  }
  seg += p.c_seg; node += p.c_node; tc += p.c_tc;
  for(int o = 16; o > 0; o >>= 1) {
    seg += __shfl_down_sync(0xffffffffu, seg, o);
    node += __shfl_down_sync(0xffffffffu, node, o);
    tc += __shfl_down_sync(0xffffffffu, tc, o);
    real += __shfl_down_sync(0xffffffffu, real, o);
    fail += __shfl_down_sync(0xffffffffu, fail, o);
  }
  if(lane == 0) {
    atomicAdd(&B.cnt->seg, seg);
    atomicAdd(&B.cnt->node, node);
    atomicAdd(&B.cnt->tc, tc);
    atomicAdd(&B.cnt->real, real);
    atomicAdd(&B.cnt->fail, fail);
  }
}

cudaError_t launch_finalize(const DRequest& R, const DAccum* acc, const DAccum* tacc, void* out,
                            size_t pitch, cudaStream_t st);

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
}

static htrdr_gpu_res_T
batched_impl(htrdr_gpu_batch_item* items, size_t n, const htrdr_gpu_tuning* tuning,
             htrdr_gpu_stats* stats, bool host)
{
  if(!items || !n) return HTRDR_GPU_RES_BAD_ARG;
  htrdr_gpu_tuning tun;
  htrdr_gpu_default_tuning(&tun);
  if(tuning) tun = *tuning;
  if(!tun.block_size || tun.block_size > 256 || (tun.block_size & 31) || !tun.queue_chunk)
    return HTRDR_GPU_RES_BAD_ARG;
  const int device = items[0].scene ? items[0].scene->device : -1;
  for(size_t i = 0; i < n; ++i) {
    if(!items[i].scene || items[i].scene->device != device || !items[i].buffer)
      return HTRDR_GPU_RES_BAD_ARG;
    const htrdr_gpu_buffer_layout& L = items[i].layout;
    const htrdr_gpu_request& q = items[i].req;
    if(L.width != q.width || L.height != q.height || L.elmt_size != pixel_size(q.mode)
    || L.pitch < L.width * L.elmt_size)
      return HTRDR_GPU_RES_BAD_ARG;
  }
  if(!cuda_ok(cudaSetDevice(device), "cudaSetDevice")) return HTRDR_GPU_RES_BAD_OP;

  std::vector<DRequest> reqs(n);
  std::vector<uint32_t> req_scene(n);
  std::vector<DScene> scenes;
  std::vector<htrdr_gpu_scene*> scene_ptrs;
  std::vector<uint64_t> offsets(n + 1, 0);
  uint64_t acc_total = 0, tacc_total = 0;
  size_t out_bytes = 0;
  std::vector<size_t> out_off(n);
  for(size_t i = 0; i < n; ++i) {
    htrdr_gpu_res_T res = make_drequest(items[i].scene, &items[i].req, &reqs[i]);
    if(res != HTRDR_GPU_RES_OK) return res;
    auto it = std::find(scene_ptrs.begin(), scene_ptrs.end(), items[i].scene);
    if(it == scene_ptrs.end()) {
      req_scene[i] = (uint32_t)scene_ptrs.size();
      scene_ptrs.push_back(items[i].scene);
      scenes.push_back(items[i].scene->d);
    } else {
      req_scene[i] = (uint32_t)(it - scene_ptrs.begin());
    }
    const uint64_t npix = (uint64_t)reqs[i].width * reqs[i].height;
    const uint32_t nch = reqs[i].mode == HG_IMAGE_CIE ? 3u : 1u;
    reqs[i].acc_base = acc_total;
    reqs[i].tacc_base = tacc_total;
    acc_total += npix * nch;
    tacc_total += npix;
    offsets[i + 1] = offsets[i] + npix * reqs[i].nreal_pp;
    out_off[i] = out_bytes;
    if(host) out_bytes += (items[i].layout.pitch * items[i].layout.height + 255) & ~(size_t)255;
  }
  const uint64_t total = offsets[n];

  DevBuf d_scenes, d_reqs, d_rs, d_off, d_acc, d_cnt, d_out;
  const size_t acc_bytes = (acc_total + tacc_total) * sizeof(DAccum);
  if(!d_scenes.upload(scenes.data(), scenes.size() * sizeof(DScene))
  || !d_reqs.upload(reqs.data(), n * sizeof(DRequest))
  || !d_rs.upload(req_scene.data(), n * 4)
  || !d_off.upload(offsets.data(), (n + 1) * 8)
  || !d_acc.alloc(acc_bytes) || !d_cnt.alloc(128) || !d_out.alloc(out_bytes))
    return HTRDR_GPU_RES_MEM_ERR;

  cudaStream_t st = items[0].scene->stream;
  BatchTables B;
  B.scenes = (const DScene*)d_scenes.ptr;
  B.reqs = (const DRequest*)d_reqs.ptr;
  B.req_scene = (const uint32_t*)d_rs.ptr;
  B.offsets = (const uint64_t*)d_off.ptr;
  B.nreq = (uint32_t)n;
  B.total = total;
  B.acc = (DAccum*)d_acc.ptr;
  B.tacc = B.acc + acc_total;
  B.cnt = (Counters*)d_cnt.ptr;
  B.next = (unsigned long long*)((char*)d_cnt.ptr + 64);
  B.chunk = tun.queue_chunk;
  B.regroup_period = tun.regroup_period;

  static_assert(sizeof(DScene) % 4 == 0 && sizeof(DRequest) % 4 == 0, "word copies");
  const size_t tables = ((scenes.size() * sizeof(DScene) + 15) & ~(size_t)15) + n * sizeof(DRequest);
  const int in_smem = tables <= 96 * 1024;
  const size_t smem = in_smem ? tables : 0;
  if(smem > 48 * 1024)
    cudaFuncSetAttribute(k_persistent, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  int nsm = 0, per_sm = 0;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_persistent, (int)tun.block_size, smem);
  if(tun.blocks_per_sm) per_sm = std::min(per_sm, (int)tun.blocks_per_sm);
  per_sm = std::max(per_sm, 1);
  const unsigned grid = (unsigned)(nsm * per_sm);

  cudaEvent_t e0, e1, e2, e3;
  cudaEventCreate(&e0); cudaEventCreate(&e1); cudaEventCreate(&e2); cudaEventCreate(&e3);
  bool ok = true;
  cudaEventRecord(e0, st);
  ok = ok && cuda_ok(cudaMemsetAsync(d_acc.ptr, 0, acc_bytes, st), "memset");
  ok = ok && cuda_ok(cudaMemsetAsync(d_cnt.ptr, 0, 128, st), "memset");
  cudaEventRecord(e1, st);
  if(ok) {
    k_persistent<<<grid, tun.block_size, smem, st>>>(B, (uint32_t)scenes.size(), in_smem);
    ok = cuda_ok(cudaGetLastError(), "k_persistent");
  }
  cudaEventRecord(e2, st);
  for(size_t i = 0; ok && i < n; ++i) {
    char* dout = host ? (char*)d_out.ptr + out_off[i] : (char*)items[i].buffer;
    ok = cuda_ok(launch_finalize(reqs[i], B.acc, B.tacc, dout, items[i].layout.pitch, st), "k_finalize");
    if(ok && host)
      ok = cuda_ok(cudaMemcpyAsync(items[i].buffer, dout, items[i].layout.pitch * items[i].layout.height,
                                   cudaMemcpyDeviceToHost, st), "D2H");
  }
  cudaEventRecord(e3, st);
  unsigned long long c[5] = {0, 0, 0, 0, 0};
  if(ok) ok = cuda_ok(cudaMemcpyAsync(c, d_cnt.ptr, sizeof(c), cudaMemcpyDeviceToHost, st), "D2H");
  if(ok) ok = cuda_ok(cudaStreamSynchronize(st), "sync");
  if(ok && stats) {
    float k = 0, t = 0;
    cudaEventElapsedTime(&k, e1, e2);
    cudaEventElapsedTime(&t, e0, e3);
    stats->segments = c[0]; stats->nodes = c[1]; stats->collisions = c[2];
    stats->realisations = c[3]; stats->failures = c[4];
    stats->kernel_ms = k; stats->total_ms = t;
  }
  cudaEventDestroy(e0); cudaEventDestroy(e1); cudaEventDestroy(e2); cudaEventDestroy(e3);
  return ok ? HTRDR_GPU_RES_OK : HTRDR_GPU_RES_UNKNOWN_ERR;
}

extern "C" HTRDR_GPU_API htrdr_gpu_res_T
htrdr_gpu_draw_maps_batched(htrdr_gpu_batch_item* items, size_t n, const htrdr_gpu_tuning* tuning,
                            htrdr_gpu_stats* stats)
{
  return batched_impl(items, n, tuning, stats, true);
}

extern "C" HTRDR_GPU_API htrdr_gpu_res_T
htrdr_gpu_draw_maps_batched_device(htrdr_gpu_batch_item* items, size_t n,
                                   const htrdr_gpu_tuning* tuning, htrdr_gpu_stats* stats)
{
  return batched_impl(items, n, tuning, stats, false);
}

/* Autotuner of the batched engine: times every candidate (block size x queue
 * chunk x regroup period) on the given items (device buffers) with CUDA
 * events and returns the fastest.  Results do not depend on the tuning. */
extern "C" HTRDR_GPU_API htrdr_gpu_res_T
htrdr_gpu_autotune(htrdr_gpu_batch_item* items, size_t n, htrdr_gpu_tuning* best, double* best_ms)
{
  if(!items || !n || !best) return HTRDR_GPU_RES_BAD_ARG;
  static const uint32_t blocks[] = {128, 256};
  static const uint32_t chunks[] = {1, 4};
  static const uint32_t periods[] = {1, 4, 16, 64};
  htrdr_gpu_stats st;
  double best_t = 1e300;
  htrdr_gpu_tuning t;
  htrdr_gpu_default_tuning(&t);
  htrdr_gpu_res_T res = batched_impl(items, n, &t, &st, false); /* warm-up */
  if(res != HTRDR_GPU_RES_OK) return res;
  for(uint32_t b : blocks)
    for(uint32_t c : chunks)
      for(uint32_t p : periods) {
        t.block_size = b;
        t.queue_chunk = c;
        t.regroup_period = p;
        t.blocks_per_sm = 0;
        res = batched_impl(items, n, &t, &st, false);
        if(res != HTRDR_GPU_RES_OK) return res;
        if(st.kernel_ms < best_t) { best_t = st.kernel_ms; *best = t; }
      }
  if(best_ms) *best_ms = best_t;
  return HTRDR_GPU_RES_OK;
}
