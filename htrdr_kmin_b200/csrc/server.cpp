/* Serving loop: continuous batching of draw_map requests.
 *
 * Client threads submit requests (scene, request, layout, host buffer) at any
 * time.  One scheduling thread per server:
 *   1. admits pending requests in arrival order while their device memory
 *      (FP64 accumulators + output staging) fits in the HBM budget; the
 *      accumulators stay resident until the request completes;
 *   2. launches rounds of the persistent kernel, each over a share of the
 *      not-yet-dispatched realisations of every admitted request; up to
 *      `kDepth' rounds are in flight on their own streams, so the next round
 *      fills the SMs that the slow paths of the previous one leave idle, and
 *      the round size adapts to a target device time;
 *   3. when a round ends, completes the requests whose realisations are all
 *      accumulated (finalize kernel, copy of the map to the host buffer) and
 *      frees their memory, which admits the next pending requests.
 * Requests arriving while rounds run join the next round, so their work
 * overlaps with the requests already on the GPU.  The weight of a realisation
 * does not depend on how the work is split into rounds: a request gives the
 * same map alone and in a mix (up to the FP64 summation order). */
#include "internal.h"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <thread>

using namespace hg;

namespace {

using clk = std::chrono::steady_clock;
constexpr int kDepth = 3; /* rounds in flight */

struct SReq {
  uint64_t ticket = 0;
  htrdr_gpu_scene* scene = nullptr;
  htrdr_gpu_request req{};
  htrdr_gpu_buffer_layout layout{};
  void* host = nullptr;
  DRequest dreq{};
  DevBuf acc, out;
  size_t acc_bytes = 0, out_bytes = 0;
  uint64_t total = 0;      /* realisations of the request */
  uint64_t next = 0;       /* first realisation not yet dispatched */
  uint64_t completed = 0;  /* realisations of the rounds that ended */
  int state = 0;           /* 0 pending, 1 active, 2 done */
  htrdr_gpu_res_T result = HTRDR_GPU_RES_OK;
  clk::time_point t_submit, t_done;
  /* wavefront serving: request-table slot, scene-table slot, first chunk
   * whose read-back covers the request, stream-ordered buffers, and the
   * event of the map's copy to the host */
  uint32_t rslot = 0, sslot = 0;
  uint64_t k_admit = 0;
  void* acc_a = nullptr;
  void* out_a = nullptr;
  cudaEvent_t copied = nullptr;
  bool finishing = false;
  /* launches of the loop (rounds or wavefront chunks) that carried the
   * request: the first with some of its realisations queued, and the last
   * before all of them were known done (UINT64_MAX: none yet) */
  uint64_t first_launch = UINT64_MAX, last_launch = 0;
};

/* Device resources of one round in flight */
struct Slot {
  cudaStream_t st = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  DevBuf scenes, reqs, items, offsets, cnt;
  std::vector<std::pair<SReq*, uint64_t>> parts;
  uint64_t seq = 0;
  bool busy = false;
};

double
ms_between(clk::time_point a, clk::time_point b)
{
  return std::chrono::duration<double, std::milli>(b - a).count();
}

bool
ensure(DevBuf& b, size_t bytes)
{
  if(b.ptr && b.bytes >= bytes) return true;
  if(b.ptr) { cudaFree(b.ptr); b.ptr = nullptr; b.bytes = 0; }
  return b.alloc(std::max<size_t>(bytes, 256));
}

}  // namespace

struct htrdr_gpu_server {
  htrdr_gpu_server_config cfg{};
  std::thread worker;
  std::mutex m;
  std::condition_variable cv_work, cv_done;
  bool stop = false;
  std::deque<SReq*> pending;
  std::vector<SReq*> active;
  std::map<uint64_t, std::unique_ptr<SReq>> all;
  uint64_t next_ticket = 1;
  size_t hbm_used = 0, hbm_peak = 0;
  uint64_t submitted = 0, completed = 0, failed = 0, rounds = 0, realisations = 0;
  double busy_ms = 0;
  std::vector<double> lat_ms;
  clk::time_point t_first, t_last;
  bool any = false;
  cudaStream_t io = nullptr;
  Slot slots[kDepth];
  uint64_t seq = 0;
  double round_real = 0;
  double min_round = 0;   /* two waves of resident threads */
  double rate = 0;        /* realisations/s, exponential average over rounds */
  clk::time_point prev_done;
  bool have_prev_done = false;

  void finish(SReq* r, htrdr_gpu_res_T res)
  { /* with m held */
    r->result = res;
    r->state = 2;
    r->t_done = clk::now();
    if(res == HTRDR_GPU_RES_OK) {
      ++completed;
      lat_ms.push_back(ms_between(r->t_submit, r->t_done));
    } else {
      ++failed;
    }
    t_last = r->t_done;
    cv_done.notify_all();
  }

  void loop();
  bool launch_round(Slot& s, const std::vector<SReq*>& act);

  /* wavefront serving (cfg.tuning.engine == HTRDR_GPU_ENGINE_WAVEFRONT) */
  struct Readback {
    WCtl ctl;
    unsigned long long next;
    unsigned long long ndone[1]; /* [kMaxReqs] */
  };
  static constexpr uint32_t kMaxReqs = 4096, kMaxScenes = 256;
  static constexpr uint64_t kMaxItems = 1u << 20;
  WaveBufs wave;
  uint32_t wave_P = 0;
  uint64_t wave_tail = 0;
  DevBuf w_scenes, w_reqs, w_items, w_offsets, w_cnt, w_ndone;
  void* w_rb[2] = {nullptr, nullptr}; /* pinned read-backs */
  cudaEvent_t w_ev[2] = {nullptr, nullptr}, w_ta[2] = {nullptr, nullptr}, w_tb[2] = {nullptr, nullptr};
  std::vector<htrdr_gpu_scene*> w_scene_of;   /* scene-table slots */
  std::vector<uint32_t> w_scene_refs;          /* active requests per scene-table slot */
  std::vector<uint32_t> w_free_rslots;
  uint32_t w_nreqs = 0;                        /* request-table high-water mark */
  uint32_t w_kinds = 0;                        /* spectral kinds admitted so far (HV_SW, HV_LW):
                                                * the pool may hold paths of each */
  uint64_t w_nitems = 0, w_appended = 0;       /* queue: items and realisations appended */
  std::vector<uint64_t> w_offsets_host;        /* [w_nitems + 1] */
  bool w_pool_live = false;                    /* slots hold paths (not all free) */
  void loop_wave();
  bool wave_setup();
  bool wave_admit(SReq* r);
  bool wave_append(const std::vector<SReq*>& act, uint64_t budget, uint64_t next_launch);
  PTables wave_tables_now();
};

/* Fair share of the round budget over the requests with work left, then the
 * leftovers in order; uploads the round's tables and launches it. */
bool
htrdr_gpu_server::launch_round(Slot& s, const std::vector<SReq*>& act)
{
  const uint64_t budget = (uint64_t)std::max(1.0, round_real);
  std::vector<SReq*> todo;
  for(SReq* r : act) if(r->next < r->total) todo.push_back(r);
  if(todo.empty()) return true;
  std::vector<uint64_t> counts(todo.size(), 0);
  uint64_t left = budget;
  const uint64_t share = std::max<uint64_t>(1, budget / todo.size());
  for(size_t i = 0; i < todo.size(); ++i) {
    counts[i] = std::min(todo[i]->total - todo[i]->next, std::min(share, left));
    left -= counts[i];
  }
  for(size_t i = 0; i < todo.size() && left; ++i) {
    const uint64_t c = std::min(todo[i]->total - todo[i]->next - counts[i], left);
    counts[i] += c;
    left -= c;
  }
  std::vector<DScene> scenes;
  std::vector<htrdr_gpu_scene*> sp;
  std::vector<DRequest> reqs;
  std::vector<PItem> items;
  std::vector<uint64_t> offsets(1, 0);
  s.parts.clear();
  for(size_t i = 0; i < todo.size(); ++i) {
    if(!counts[i]) continue;
    auto it = std::find(sp.begin(), sp.end(), todo[i]->scene);
    uint32_t si;
    if(it == sp.end()) { si = (uint32_t)sp.size(); sp.push_back(todo[i]->scene); scenes.push_back(todo[i]->scene->d); }
    else si = (uint32_t)(it - sp.begin());
    items.push_back(PItem{(uint32_t)reqs.size(), si, todo[i]->next});
    reqs.push_back(todo[i]->dreq);
    offsets.push_back(offsets.back() + counts[i]);
    s.parts.emplace_back(todo[i], counts[i]);
    todo[i]->next += counts[i];
    todo[i]->first_launch = std::min(todo[i]->first_launch, seq); /* this round's index */
    todo[i]->last_launch = std::max(todo[i]->last_launch, seq);
  }
  if(!ensure(s.scenes, scenes.size() * sizeof(DScene)) || !ensure(s.reqs, reqs.size() * sizeof(DRequest))
  || !ensure(s.items, items.size() * sizeof(PItem)) || !ensure(s.offsets, offsets.size() * 8)
  || !ensure(s.cnt, 128))
    return false;
  bool ok = cuda_ok(cudaMemcpyAsync(s.scenes.ptr, scenes.data(), scenes.size() * sizeof(DScene),
                                    cudaMemcpyHostToDevice, s.st), "H2D")
         && cuda_ok(cudaMemcpyAsync(s.reqs.ptr, reqs.data(), reqs.size() * sizeof(DRequest),
                                    cudaMemcpyHostToDevice, s.st), "H2D")
         && cuda_ok(cudaMemcpyAsync(s.items.ptr, items.data(), items.size() * sizeof(PItem),
                                    cudaMemcpyHostToDevice, s.st), "H2D")
         && cuda_ok(cudaMemcpyAsync(s.offsets.ptr, offsets.data(), offsets.size() * 8,
                                    cudaMemcpyHostToDevice, s.st), "H2D")
         && cuda_ok(cudaMemsetAsync(s.cnt.ptr, 0, 128, s.st), "memset");
  PTables T{};
  T.scenes = (const DScene*)s.scenes.ptr;
  T.reqs = (const DRequest*)s.reqs.ptr;
  T.items = (const PItem*)s.items.ptr;
  T.offsets = (const uint64_t*)s.offsets.ptr;
  T.nscenes = (uint32_t)scenes.size();
  T.variant = tables_variant(scenes, reqs);
  T.nreqs = (uint32_t)reqs.size();
  T.nitems = (uint32_t)items.size();
  T.total = offsets.back();
  T.cnt = s.cnt.ptr;
  T.next = (unsigned long long*)((char*)s.cnt.ptr + 64);
  T.chunk = cfg.tuning.queue_chunk;
  T.regroup_period = cfg.tuning.regroup_period;
  ok = ok && cuda_ok(cudaEventRecord(s.e0, s.st), "event")
          && cuda_ok(launch_persistent(T, cfg.tuning.block_size, cfg.tuning.blocks_per_sm, cfg.device, s.st,
                                       cfg.tuning.engine == HTRDR_GPU_ENGINE_SORTED),
                     "k_persistent")
          && cuda_ok(cudaEventRecord(s.e1, s.st), "event");
  realisations += T.total;
  s.busy = true;
  s.seq = seq++;
  return ok;
}

void
htrdr_gpu_server::loop()
{
  cudaSetDevice(cfg.device);
  for(;;) {
    std::unique_lock<std::mutex> lk(m);
    /* admission by HBM budget, in arrival order */
    while(!pending.empty()) {
      SReq* r = pending.front();
      const size_t need = r->acc_bytes + r->out_bytes;
      if(need > cfg.hbm_budget_bytes) { pending.pop_front(); finish(r, HTRDR_GPU_RES_MEM_ERR); continue; }
      if(hbm_used + need > cfg.hbm_budget_bytes) break;
      pending.pop_front();
      hbm_used += need;
      hbm_peak = std::max(hbm_peak, hbm_used);
      lk.unlock();
      const bool ok = r->acc.alloc(r->acc_bytes) && r->out.alloc(r->out_bytes)
                   && cuda_ok(cudaMemsetAsync(r->acc.ptr, 0, r->acc_bytes, io), "memset")
                   && cuda_ok(cudaStreamSynchronize(io), "sync");
      lk.lock();
      if(!ok) { hbm_used -= need; finish(r, HTRDR_GPU_RES_MEM_ERR); continue; }
      const uint32_t nch = r->dreq.mode == HG_IMAGE_CIE ? 3u : 1u;
      r->dreq.acc = (DAccum*)r->acc.ptr;
      r->dreq.tacc = r->dreq.acc + (uint64_t)r->dreq.width * r->dreq.height * nch;
      r->state = 1;
      active.push_back(r);
    }
    std::vector<SReq*> act = active;
    lk.unlock();

    /* keep up to kDepth rounds in flight */
    bool launch_failed = false;
    for(Slot& s : slots) {
      if(s.busy) continue;
      bool work = false;
      for(SReq* r : act) work |= r->next < r->total;
      if(!work) break;
      if(!launch_round(s, act)) { launch_failed = true; break; }
    }
    Slot* oldest = nullptr;
    for(Slot& s : slots) if(s.busy && (!oldest || s.seq < oldest->seq)) oldest = &s;

    if(!oldest) {
      lk.lock();
      if(launch_failed) {
        for(SReq* r : active) finish(r, HTRDR_GPU_RES_UNKNOWN_ERR);
        active.clear();
        continue;
      }
      if(stop && pending.empty() && active.empty()) break;
      if(pending.empty()) cv_work.wait(lk);
      continue;
    }

    /* wait for the oldest round, then complete the requests it finishes */
    bool ok = cuda_ok(cudaEventSynchronize(oldest->e1), "round") && !launch_failed;
    float ms = 0;
    if(ok) cudaEventElapsedTime(&ms, oldest->e0, oldest->e1);
    busy_ms += ms;
    ++rounds;
    { /* round size from the observed throughput (rounds overlap, so a
       * round's own duration overstates its cost), at least two waves of
       * the resident threads so that slow paths are amortised */
      const clk::time_point now = clk::now();
      uint64_t nreal = 0;
      for(auto& pr : oldest->parts) nreal += pr.second;
      if(have_prev_done) {
        const double dt = std::max(1e-4, ms_between(prev_done, now) * 1e-3);
        const double r = (double)nreal / dt;
        rate = rate > 0 ? 0.7 * rate + 0.3 * r : r;
        round_real = std::max(min_round, std::min(rate * cfg.round_target_ms * 1e-3, 1e12));
      }
      prev_done = now;
      have_prev_done = true;
    }
    std::vector<SReq*> done;
    for(auto& pr : oldest->parts) {
      SReq* r = pr.first;
      r->completed += pr.second;
      if(!ok || r->completed < r->total) continue;
      const bool fin = cuda_ok(launch_finalize(r->dreq, r->dreq.acc, r->dreq.tacc, r->out.ptr,
                                               r->layout.pitch, oldest->st), "k_finalize")
                    && cuda_ok(cudaMemcpyAsync(r->host, r->out.ptr, r->out_bytes, cudaMemcpyDeviceToHost,
                                               oldest->st), "D2H")
                    && cuda_ok(cudaStreamSynchronize(oldest->st), "sync");
      if(!fin) r->result = HTRDR_GPU_RES_UNKNOWN_ERR;
      done.push_back(r);
    }
    oldest->busy = false;
    oldest->parts.clear();
    lk.lock();
    if(!ok) { /* a failed round poisons every active request */
      for(Slot& s : slots) if(s.busy) { cudaStreamSynchronize(s.st); s.busy = false; s.parts.clear(); }
      done = active;
    }
    for(SReq* r : done) {
      if(r->state == 2) continue;
      const size_t need = r->acc_bytes + r->out_bytes;
      if(r->acc.ptr) { cudaFree(r->acc.ptr); r->acc.ptr = nullptr; }
      if(r->out.ptr) { cudaFree(r->out.ptr); r->out.ptr = nullptr; }
      hbm_used -= need;
      active.erase(std::find(active.begin(), active.end(), r));
      finish(r, ok ? r->result : HTRDR_GPU_RES_UNKNOWN_ERR);
    }
  }
}

/*******************************************************************************
 * Wavefront serving: one pool of path slots fed by a growing work queue.
 *
 * Admitted requests get a slot in a device request table and stay resident;
 * the scheduling thread appends fair-share slices of every admitted
 * request's remaining realisations to the queue (keeping about one pool of
 * realisations queued), and runs chunks of event+trace iterations.  Paths
 * that end take the next queued realisation in their slot, so requests that
 * arrive while others render start in the slots those free.  Per-request
 * counters of finished realisations, read back after every chunk, tell when
 * a request's map is complete (finalize, copy to the host buffer).  When no
 * work is queued and few paths are live, the megakernel finishes them and
 * the pool returns to all-free; a slot that finds the queue empty waits on
 * the dead list until work is appended.
 ******************************************************************************/
bool
htrdr_gpu_server::wave_setup()
{
  wave_P = cfg.tuning.wave_slots ? cfg.tuning.wave_slots : kDefaultWaveSlots;
  wave_tail = wave_serve_tail(cfg.tuning, cfg.device);
  const size_t rb = sizeof(Readback) + (kMaxReqs - 1) * sizeof(unsigned long long);
  bool ok = w_scenes.alloc(kMaxScenes * sizeof(DScene)) && w_reqs.alloc(kMaxReqs * sizeof(DRequest))
         && w_items.alloc(kMaxItems * sizeof(PItem)) && w_offsets.alloc((kMaxItems + 1) * 8)
         && w_cnt.alloc(128) && w_ndone.alloc(kMaxReqs * 8);
  for(int i = 0; ok && i < 2; ++i)
    ok = cuda_ok(cudaHostAlloc(&w_rb[i], rb, cudaHostAllocDefault), "cudaHostAlloc")
      && cuda_ok(cudaEventCreateWithFlags(&w_ev[i], cudaEventDisableTiming), "event")
      && cuda_ok(cudaEventCreate(&w_ta[i]), "event") && cuda_ok(cudaEventCreate(&w_tb[i]), "event");
  ok = ok && cuda_ok(cudaMemsetAsync(w_cnt.ptr, 0, 128, io), "memset")
          && cuda_ok(cudaMemsetAsync(w_ndone.ptr, 0, kMaxReqs * 8, io), "memset")
          && cuda_ok(cudaMemsetAsync(w_offsets.ptr, 0, 8, io), "memset")
          && cuda_ok(wave_serve_reset(wave, wave_P, io), "wavefront pool")
          && cuda_ok(cudaStreamSynchronize(io), "sync");
  w_offsets_host.assign(1, 0);
  for(uint32_t i = kMaxReqs; i-- > 0;) w_free_rslots.push_back(i);
  return ok;
}

/* Device memory and table entries of an admitted request (scheduling thread) */
bool
htrdr_gpu_server::wave_admit(SReq* r)
{
  uint32_t ss = 0;
  {
    auto it = std::find(w_scene_of.begin(), w_scene_of.end(), r->scene);
    if(it != w_scene_of.end()) {
      ss = (uint32_t)(it - w_scene_of.begin());
    } else { /* a table slot no active request uses, else a new one */
      ss = (uint32_t)w_scene_of.size();
      for(uint32_t i = 0; i < w_scene_of.size(); ++i)
        if(!w_scene_refs[i]) { ss = i; break; }
      if(ss == w_scene_of.size()) {
        if(ss >= kMaxScenes) { set_error("server: too many scenes in flight"); return false; }
        w_scene_of.push_back(nullptr);
        w_scene_refs.push_back(0);
      }
      w_scene_of[ss] = r->scene;
    }
  }
  const uint32_t rs = w_free_rslots.back();
  bool ok = cuda_ok(cudaMallocAsync(&r->acc_a, r->acc_bytes, io), "cudaMallocAsync")
         && cuda_ok(cudaMallocAsync(&r->out_a, r->out_bytes, io), "cudaMallocAsync")
         && cuda_ok(cudaMemsetAsync(r->acc_a, 0, r->acc_bytes, io), "memset")
         && cuda_ok(cudaEventCreateWithFlags(&r->copied, cudaEventDisableTiming), "event");
  if(!ok) {
    if(r->acc_a) cudaFreeAsync(r->acc_a, io);
    if(r->out_a) cudaFreeAsync(r->out_a, io);
    r->acc_a = r->out_a = nullptr;
    return false;
  }
  const uint32_t nch = r->dreq.mode == HG_IMAGE_CIE ? 3u : 1u;
  r->dreq.acc = (DAccum*)r->acc_a;
  r->dreq.tacc = r->dreq.acc + (uint64_t)r->dreq.width * r->dreq.height * nch;
  r->dreq.ndone = (unsigned long long*)w_ndone.ptr + rs;
  /* pageable sources are staged before the calls return */
  ok = cuda_ok(cudaMemsetAsync(r->dreq.ndone, 0, 8, io), "memset")
    && cuda_ok(cudaMemcpyAsync((DRequest*)w_reqs.ptr + rs, &r->dreq, sizeof(DRequest),
                               cudaMemcpyHostToDevice, io), "H2D")
    && cuda_ok(cudaMemcpyAsync((DScene*)w_scenes.ptr + ss, &r->scene->d, sizeof(DScene),
                               cudaMemcpyHostToDevice, io), "H2D");
  if(!ok) return false;
  w_free_rslots.pop_back();
  r->rslot = rs;
  r->sslot = ss;
  ++w_scene_refs[ss];
  w_nreqs = std::max(w_nreqs, rs + 1);
  w_kinds |= hv_kind(r->dreq.mode);
  r->next = 0;
  return true;
}

/* Fair share of `budget' realisations over the requests with work not yet
 * queued, then the leftovers in order; appends the items to the queue */
bool
htrdr_gpu_server::wave_append(const std::vector<SReq*>& act, uint64_t budget, uint64_t next_launch)
{
  std::vector<SReq*> todo;
  for(SReq* r : act) if(r->state == 1 && r->next < r->total) todo.push_back(r);
  if(todo.empty() || w_nitems + todo.size() > kMaxItems) return true;
  std::vector<uint64_t> counts(todo.size(), 0);
  uint64_t left = budget;
  const uint64_t share = std::max<uint64_t>(1, budget / todo.size());
  for(size_t i = 0; i < todo.size(); ++i) {
    counts[i] = std::min(todo[i]->total - todo[i]->next, std::min(share, left));
    left -= counts[i];
  }
  for(size_t i = 0; i < todo.size() && left; ++i) {
    const uint64_t c = std::min(todo[i]->total - todo[i]->next - counts[i], left);
    counts[i] += c;
    left -= c;
  }
  std::vector<PItem> items;
  std::vector<uint64_t> offs;
  const uint64_t begin = w_offsets_host.back();
  uint64_t end = begin;
  for(size_t i = 0; i < todo.size(); ++i) {
    if(!counts[i]) continue;
    items.push_back(PItem{todo[i]->rslot, todo[i]->sslot, todo[i]->next});
    end += counts[i];
    offs.push_back(end);
    todo[i]->next += counts[i];
    /* the next launch is the first to take these realisations */
    todo[i]->first_launch = std::min(todo[i]->first_launch, next_launch);
  }
  if(items.empty()) return true;
  const bool ok =
    cuda_ok(cudaMemcpyAsync((PItem*)w_items.ptr + w_nitems, items.data(), items.size() * sizeof(PItem),
                            cudaMemcpyHostToDevice, io), "H2D")
    && cuda_ok(cudaMemcpyAsync((uint64_t*)w_offsets.ptr + w_nitems + 1, offs.data(), offs.size() * 8,
                               cudaMemcpyHostToDevice, io), "H2D");
  w_offsets_host.insert(w_offsets_host.end(), offs.begin(), offs.end());
  w_nitems += items.size();
  w_appended = end;
  realisations += end - begin;
  return ok;
}

PTables
htrdr_gpu_server::wave_tables_now()
{
  PTables T{};
  T.scenes = (const DScene*)w_scenes.ptr;
  T.reqs = (const DRequest*)w_reqs.ptr;
  T.items = (const PItem*)w_items.ptr;
  T.offsets = (const uint64_t*)w_offsets.ptr;
  T.nscenes = (uint32_t)w_scene_of.size();
  T.variant = hv_make(std::any_of(w_scene_of.begin(), w_scene_of.end(),
                                  [](const htrdr_gpu_scene* sc) { return sc && sc->d.g_ntris != 0; }),
                      w_kinds);
  T.nreqs = w_nreqs;
  T.nitems = (uint32_t)w_nitems;
  T.total = w_appended;
  T.cnt = w_cnt.ptr;
  T.next = (unsigned long long*)((char*)w_cnt.ptr + 64);
  T.chunk = cfg.tuning.queue_chunk;
  T.regroup_period = cfg.tuning.regroup_period;
  return T;
}

void
htrdr_gpu_server::loop_wave()
{
  cudaSetDevice(cfg.device);
  bool failed_gpu = !wave_setup();
  const uint32_t C = 8;       /* iterations per chunk */
  uint64_t k = 0;             /* launches (chunks and finishes), each with a read-back */
  bool inflight[2] = {false, false};
  uint64_t rb_k[2] = {0, 0};  /* launch index of each read-back buffer */
  /* the queue restarts from zero between epochs: a read-back issued in an
   * earlier epoch holds the head of a queue that no longer exists */
  uint64_t epoch = 0, rb_epoch[2] = {0, 0};
  uint64_t dev_next = 0;      /* queue head and live paths at the last read-back */
  uint32_t dev_live = 0;

  /* read-back of one launch: queue head, live paths, finished requests */
  auto process = [&](int b) -> bool {
    if(!cuda_ok(cudaEventSynchronize(w_ev[b]), "chunk")) return false;
    inflight[b] = false;
    float ms = 0;
    if(cudaEventElapsedTime(&ms, w_ta[b], w_tb[b]) == cudaSuccess) busy_ms += ms;
    const Readback* rb = (const Readback*)w_rb[b];
    dev_next = rb_epoch[b] == epoch ? rb->next : 0; /* else: nothing known taken yet */
    dev_live = rb->ctl.n_live[0];
    for(SReq* r : active) {
      /* a read-back issued before the request was admitted holds another
       * request's count in its table slot */
      if(r->finishing || r->state != 1 || r->k_admit > rb_k[b]) continue;
      r->last_launch = std::max(r->last_launch, rb_k[b]);
      if(rb->ndone[r->rslot] < r->total) continue;
      /* every realisation accumulated: the map, on the same stream */
      const bool fin = cuda_ok(launch_finalize(r->dreq, r->dreq.acc, r->dreq.tacc, r->out_a,
                                               r->layout.pitch, io), "k_finalize")
                    && cuda_ok(cudaMemcpyAsync(r->host, r->out_a, r->out_bytes, cudaMemcpyDeviceToHost, io),
                               "D2H")
                    && cuda_ok(cudaEventRecord(r->copied, io), "event");
      if(!fin) r->result = HTRDR_GPU_RES_UNKNOWN_ERR;
      r->finishing = true;
    }
    return true;
  };
  /* requests whose map reached the host buffer leave */
  auto retire = [&](bool wait) {
    std::vector<SReq*> done;
    for(SReq* r : active) {
      if(!r->finishing) continue;
      const cudaError_t q = wait ? cudaEventSynchronize(r->copied) : cudaEventQuery(r->copied);
      if(q == cudaErrorNotReady) continue;
      if(q != cudaSuccess) r->result = HTRDR_GPU_RES_UNKNOWN_ERR;
      done.push_back(r);
    }
    for(SReq* r : done) {
      cudaFreeAsync(r->acc_a, io);
      cudaFreeAsync(r->out_a, io);
      r->acc_a = r->out_a = nullptr;
      cudaEventDestroy(r->copied);
      r->copied = nullptr;
      w_free_rslots.push_back(r->rslot);
      --w_scene_refs[r->sslot];
    }
    std::lock_guard<std::mutex> lk(m);
    for(SReq* r : done) {
      hbm_used -= r->acc_bytes + r->out_bytes;
      active.erase(std::find(active.begin(), active.end(), r));
      finish(r, r->result);
    }
  };
  /* a chunk (or the finish) into read-back buffer b */
  auto launch = [&](int b, bool finish_all) -> bool {
    Readback* rb = (Readback*)w_rb[b];
    const PTables T = wave_tables_now();
    const bool ok =
      cuda_ok(cudaEventRecord(w_ta[b], io), "event")
      && (finish_all ? cuda_ok(wave_serve_finish(T, cfg.tuning, wave, cfg.device, io), "wavefront finish")
                     : cuda_ok(wave_serve_chunk(T, cfg.tuning, wave, cfg.device, C, io), "wavefront chunk"))
      && cuda_ok(cudaEventRecord(w_tb[b], io), "event")
      && cuda_ok(cudaMemcpyAsync(&rb->ctl, wave.ctl.ptr, sizeof(WCtl), cudaMemcpyDeviceToHost, io), "D2H")
      && cuda_ok(cudaMemcpyAsync(&rb->next, (char*)w_cnt.ptr + 64, 8, cudaMemcpyDeviceToHost, io), "D2H")
      && (w_nreqs == 0
          || cuda_ok(cudaMemcpyAsync(rb->ndone, w_ndone.ptr, (size_t)w_nreqs * 8, cudaMemcpyDeviceToHost,
                                     io), "D2H"))
      && cuda_ok(cudaEventRecord(w_ev[b], io), "event");
    rb_k[b] = k;
    rb_epoch[b] = epoch;
    inflight[b] = ok;
    ++k;
    ++rounds;
    return ok;
  };

  for(;;) {
    std::unique_lock<std::mutex> lk(m);
    /* admission by HBM budget and request-table room, in arrival order */
    while(!pending.empty()) {
      SReq* r = pending.front();
      const size_t need = r->acc_bytes + r->out_bytes;
      if(failed_gpu) { pending.pop_front(); finish(r, HTRDR_GPU_RES_BAD_OP); continue; }
      if(need > cfg.hbm_budget_bytes) { pending.pop_front(); finish(r, HTRDR_GPU_RES_MEM_ERR); continue; }
      if(hbm_used + need > cfg.hbm_budget_bytes || w_free_rslots.empty()) break;
      pending.pop_front();
      hbm_used += need;
      hbm_peak = std::max(hbm_peak, hbm_used);
      lk.unlock();
      const bool ok = wave_admit(r);
      lk.lock();
      if(!ok) { hbm_used -= need; finish(r, HTRDR_GPU_RES_MEM_ERR); continue; }
      r->state = 1;
      r->k_admit = k;
      active.push_back(r);
    }
    const bool waiting = !pending.empty();
    if(failed_gpu) { /* the device failed: every request in flight fails */
      for(SReq* r : active) finish(r, HTRDR_GPU_RES_UNKNOWN_ERR);
      active.clear();
      if(stop && pending.empty()) break;
      if(pending.empty()) cv_work.wait(lk);
      continue;
    }
    lk.unlock();

    /* every queued realisation was taken (the head never passes the queued
     * total): the queue restarts from zero, which keeps the item table short.
     * Paths in flight no longer read items; the restart is ordered after the
     * launches in flight on the stream. */
    if(w_nitems && dev_next >= w_appended) {
      if(!cuda_ok(cudaMemsetAsync((char*)w_cnt.ptr + 64, 0, 8, io), "memset")) { failed_gpu = true; continue; }
      w_nitems = 0;
      w_appended = 0;
      dev_next = 0;
      w_offsets_host.assign(1, 0);
      ++epoch;
    }

    /* keep about one pool of realisations queued */
    bool unqueued = false;
    for(SReq* r : active) unqueued |= r->state == 1 && r->next < r->total;
    const uint64_t queued = w_appended > dev_next ? w_appended - dev_next : 0;
    if(unqueued && queued < wave_P) {
      const uint64_t before = w_appended;
      if(!wave_append(active, wave_P - queued, k)) { failed_gpu = true; continue; }
      if(w_appended > before) {
        if(!cuda_ok(wave_serve_revive(wave, io), "revive")) { failed_gpu = true; continue; }
        w_pool_live = true;
      }
    }

    if(w_pool_live) { /* one chunk, then the read-back of the previous launch */
      const int b = (int)(k & 1);
      if(inflight[b] && !process(b)) { failed_gpu = true; continue; }
      if(!launch(b, false)) { failed_gpu = true; continue; }
      const int pb = b ^ 1;
      if(inflight[pb] && !process(pb)) { failed_gpu = true; continue; }
      retire(false);
      /* drained: nothing queued, nothing left to queue, few live paths */
      bool more = false;
      for(SReq* r : active) more |= r->state == 1 && r->next < r->total;
      if(dev_next >= w_appended && !more && !waiting) {
        if(dev_live == 0) {
          w_pool_live = false;
        } else if(dev_live < wave_tail) { /* the tail: finish in the megakernel */
          const int nb = (int)(k & 1);
          if(inflight[nb] && !process(nb)) { failed_gpu = true; continue; }
          if(!launch(nb, true)) { failed_gpu = true; continue; }
          bool okp = true;
          for(int i = 0; i < 2; ++i)
            if(inflight[i]) okp = process(i) && okp;
          if(!okp) { failed_gpu = true; continue; }
          w_pool_live = false;
        }
      }
      continue;
    }

    /* no live path: complete what is in flight, then wait for work */
    bool okp = true;
    for(int i = 0; i < 2; ++i)
      if(inflight[i]) okp = process(i) && okp;
    if(!okp) { failed_gpu = true; continue; }
    bool finishing = false;
    for(SReq* r : active) finishing |= r->finishing;
    retire(finishing);
    if(!active.empty()) {
      if(!finishing) std::this_thread::sleep_for(std::chrono::microseconds(200));
      continue;
    }
    lk.lock();
    if(stop && pending.empty() && active.empty()) break;
    if(pending.empty()) cv_work.wait(lk);
  }
  cudaStreamSynchronize(io);
}

extern "C" HTRDR_GPU_API htrdr_gpu_res_T
htrdr_gpu_server_create(const htrdr_gpu_server_config* cfg, htrdr_gpu_server** out)
try {
  if(!cfg || !out || !cfg->hbm_budget_bytes || !valid_tuning(cfg->tuning)) return HTRDR_GPU_RES_BAD_ARG;
  int ndev = 0;
  if(cudaGetDeviceCount(&ndev) != cudaSuccess || cfg->device < 0 || cfg->device >= ndev) {
    set_error("no CUDA device available");
    return HTRDR_GPU_RES_BAD_OP;
  }
  auto s = new htrdr_gpu_server();
  s->cfg = *cfg;
  if(s->cfg.round_target_ms <= 0) s->cfg.round_target_ms = 20.0;
  cudaSetDevice(cfg->device);
  /* smallest round: the configured first size, else two waves of resident threads */
  s->min_round = cfg->round_realisations
    ? (double)cfg->round_realisations
    : 2.0 * (double)persistent_capacity(cfg->tuning.block_size, cfg->tuning.blocks_per_sm, cfg->device);
  s->round_real = s->min_round;
  bool ok = cuda_ok(cudaStreamCreateWithFlags(&s->io, cudaStreamNonBlocking), "stream");
  for(Slot& sl : s->slots)
    ok = ok && cuda_ok(cudaStreamCreateWithFlags(&sl.st, cudaStreamNonBlocking), "stream")
            && cuda_ok(cudaEventCreate(&sl.e0), "event") && cuda_ok(cudaEventCreate(&sl.e1), "event");
  if(!ok) { htrdr_gpu_server_release(s); return HTRDR_GPU_RES_BAD_OP; }
  if(cfg->tuning.engine == HTRDR_GPU_ENGINE_WAVEFRONT)
    s->worker = std::thread([s]() { s->loop_wave(); });
  else
    s->worker = std::thread([s]() { s->loop(); });
  *out = s;
  return HTRDR_GPU_RES_OK;
}
HG_API_CATCH("htrdr_gpu_server_create")

extern "C" HTRDR_GPU_API htrdr_gpu_res_T
htrdr_gpu_server_submit(htrdr_gpu_server* s, htrdr_gpu_scene* scene, const htrdr_gpu_request* req,
                        const htrdr_gpu_buffer_layout* layout, void* host_buffer, uint64_t* ticket)
try {
  if(!s || !scene || !req || !layout || !host_buffer || !ticket) return HTRDR_GPU_RES_BAD_ARG;
  if(scene->device != s->cfg.device) return HTRDR_GPU_RES_BAD_ARG;
  if(check_layout(req, layout) != HTRDR_GPU_RES_OK) return HTRDR_GPU_RES_BAD_ARG;
  auto r = std::make_unique<SReq>();
  cudaSetDevice(scene->device);
  const htrdr_gpu_res_T res = make_drequest(scene, req, &r->dreq);
  if(res != HTRDR_GPU_RES_OK) return res;
  r->scene = scene;
  r->req = *req;
  r->layout = *layout;
  r->host = host_buffer;
  const uint64_t npix = (uint64_t)req->width * req->height;
  const uint32_t nch = req->mode == HG_IMAGE_CIE ? 3u : 1u;
  r->acc_bytes = npix * (nch + 1) * sizeof(DAccum);
  r->out_bytes = layout->pitch * layout->height;
  r->total = npix * r->dreq.nreal_pp;
  r->t_submit = clk::now();
  std::lock_guard<std::mutex> lk(s->m);
  if(s->stop) return HTRDR_GPU_RES_BAD_OP;
  r->ticket = s->next_ticket++;
  *ticket = r->ticket;
  if(!s->any) { s->any = true; s->t_first = r->t_submit; }
  ++s->submitted;
  s->pending.push_back(r.get());
  s->all.emplace(r->ticket, std::move(r));
  s->cv_work.notify_one();
  return HTRDR_GPU_RES_OK;
}
HG_API_CATCH("htrdr_gpu_server_submit")

extern "C" HTRDR_GPU_API htrdr_gpu_res_T
htrdr_gpu_server_poll(htrdr_gpu_server* s, uint64_t ticket, int* done, htrdr_gpu_res_T* result)
try {
  if(!s || !done) return HTRDR_GPU_RES_BAD_ARG;
  std::lock_guard<std::mutex> lk(s->m);
  auto it = s->all.find(ticket);
  if(it == s->all.end()) return HTRDR_GPU_RES_BAD_ARG;
  *done = it->second->state == 2;
  if(result) *result = it->second->result;
  return HTRDR_GPU_RES_OK;
}
HG_API_CATCH("htrdr_gpu_server_poll")

extern "C" HTRDR_GPU_API htrdr_gpu_res_T
htrdr_gpu_server_wait(htrdr_gpu_server* s, uint64_t ticket, double timeout_s, htrdr_gpu_res_T* result)
try {
  if(!s) return HTRDR_GPU_RES_BAD_ARG;
  std::unique_lock<std::mutex> lk(s->m);
  auto it = s->all.find(ticket);
  if(it == s->all.end()) return HTRDR_GPU_RES_BAD_ARG;
  SReq* r = it->second.get();
  const bool ok = s->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s),
                                      [r]() { return r->state == 2; });
  if(!ok) return HTRDR_GPU_RES_BAD_OP;
  if(result) *result = r->result;
  return HTRDR_GPU_RES_OK;
}
HG_API_CATCH("htrdr_gpu_server_wait")

extern "C" HTRDR_GPU_API htrdr_gpu_res_T
htrdr_gpu_server_request_launches(htrdr_gpu_server* s, uint64_t ticket, uint64_t* first,
                                  uint64_t* last)
try {
  if(!s || !first || !last) return HTRDR_GPU_RES_BAD_ARG;
  std::lock_guard<std::mutex> lk(s->m);
  auto it = s->all.find(ticket);
  if(it == s->all.end()) return HTRDR_GPU_RES_BAD_ARG;
  const SReq* r = it->second.get();
  if(r->first_launch == UINT64_MAX) return HTRDR_GPU_RES_BAD_OP;
  *first = r->first_launch;
  *last = std::max(r->first_launch, r->last_launch);
  return HTRDR_GPU_RES_OK;
}
HG_API_CATCH("htrdr_gpu_server_request_launches")

extern "C" HTRDR_GPU_API htrdr_gpu_res_T
htrdr_gpu_server_stats(htrdr_gpu_server* s, struct htrdr_gpu_server_stats* st)
try {
  if(!s || !st) return HTRDR_GPU_RES_BAD_ARG;
  std::lock_guard<std::mutex> lk(s->m);
  std::memset(st, 0, sizeof(*st));
  st->submitted = s->submitted;
  st->completed = s->completed;
  st->failed = s->failed;
  st->rounds = s->rounds;
  st->realisations = s->realisations;
  st->busy_ms = s->busy_ms;
  st->hbm_peak_bytes = s->hbm_peak;
  if(s->any && (s->completed || s->failed)) st->wall_ms = ms_between(s->t_first, s->t_last);
  if(!s->lat_ms.empty()) {
    std::vector<double> v = s->lat_ms;
    std::sort(v.begin(), v.end());
    auto q = [&](double f) { return v[std::min(v.size() - 1, (size_t)std::floor(f * (double)(v.size() - 1) + 0.5))]; };
    st->p50_ms = q(0.50);
    st->p99_ms = q(0.99);
    st->max_ms = v.back();
    double acc = 0;
    for(double x : v) acc += x;
    st->mean_ms = acc / (double)v.size();
  }
  return HTRDR_GPU_RES_OK;
}
HG_API_CATCH("htrdr_gpu_server_stats")

extern "C" HTRDR_GPU_API void
htrdr_gpu_server_release(htrdr_gpu_server* s)
{
  if(!s) return;
  {
    std::lock_guard<std::mutex> lk(s->m);
    s->stop = true;
    s->cv_work.notify_all();
  }
  if(s->worker.joinable()) s->worker.join();
  cudaSetDevice(s->cfg.device);
  for(Slot& sl : s->slots) {
    if(sl.st) { cudaStreamSynchronize(sl.st); cudaStreamDestroy(sl.st); }
    if(sl.e0) cudaEventDestroy(sl.e0);
    if(sl.e1) cudaEventDestroy(sl.e1);
  }
  for(int i = 0; i < 2; ++i) {
    if(s->w_rb[i]) cudaFreeHost(s->w_rb[i]);
    if(s->w_ev[i]) cudaEventDestroy(s->w_ev[i]);
    if(s->w_ta[i]) cudaEventDestroy(s->w_ta[i]);
    if(s->w_tb[i]) cudaEventDestroy(s->w_tb[i]);
  }
  if(s->io) { cudaStreamSynchronize(s->io); cudaStreamDestroy(s->io); }
  delete s;
}
