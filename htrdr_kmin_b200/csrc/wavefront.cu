/* Wavefront engine: the path state machine split into two stage kernels
 * that run alternately over a pool of path slots in HBM.
 *
 *  - event stage (k_wave_event): for every live slot, runs path_event()
 *    (sensor sampling, scattering and surface events, sun next-event
 *    estimation) until the path needs a trace; a finished path is
 *    accumulated and the slot takes the next realisation from the work
 *    queue (path regeneration).  Slots still holding a path are compacted
 *    into the next live list with warp-aggregated atomics; slots for which
 *    the queue is empty drop out.
 *  - trace stage (k_wave_trace): every resident lane takes the next live
 *    slot, loads only the trace part of its path (a prefix of struct Path),
 *    and steps voxels until the trace ends or a step budget is spent, then
 *    stores the prefix back and takes another slot.  The stage holds no
 *    event state in registers, runs none of the event code, and so keeps
 *    more warps resident than the megakernel; lanes never wait for events.
 *
 * Both stages run the same state machine as the other engines on the same
 * Philox streams, so a realisation's weight does not depend on the engine.
 * A path is stored as contiguous 16-byte vectors per slot: the trace stage
 * visits slots in the order lanes free up, and a lane reading its own slot's
 * consecutive vectors uses every byte of the sectors it touches.
 *
 * The host drives the iterations: chunks of event+trace launches, the live
 * count read back once per chunk (pinned memory, no device wait inside a
 * kernel).  Every path is bounded in bounces and voxel steps, so the loop
 * ends. */
#include "engine.cuh"

#include <algorithm>
#include <map>
#include <memory>
#include <cstring>

namespace hg {

namespace {

constexpr uint32_t kPathV4 = (uint32_t)((sizeof(Path) + 15) / 16);
constexpr uint32_t kTraceV4 = (uint32_t)((offsetof(Path, org) + 15) / 16);
static_assert(kTraceV4 <= kPathV4, "trace part inside the path");
/* The vector holding the collision site of a SW free path (pnext), which the
 * trace stage writes when it runs the absorption trace itself.  Its last
 * word is dnext.x, dead from there until ST_SW_ABS_END sets dnext. */
constexpr uint32_t kPnextV4 = (uint32_t)(offsetof(Path, pnext) / 16);
static_assert(offsetof(Path, pnext) % 16 == 0 && offsetof(Path, dnext) == offsetof(Path, pnext) + 12,
              "pnext and dnext.x fill one 16-byte vector");
/* The vectors of the walk's position and direction, which the trace stage
 * writes when it runs a LW scattering itself: pos.x, pos.y end the first,
 * pos.z and dir fill the second */
constexpr uint32_t kPosV4 = (uint32_t)(offsetof(Path, pos) / 16);
static_assert(offsetof(Path, pos) % 16 == 8 && offsetof(Path, dir) == offsetof(Path, pos) + 12
              && offsetof(Path, dir) + 12 == (kPosV4 + 2) * 16, "pos and dir end two 16-byte vectors");

/* Gas-region batching of the trace stage (0: off).  Measured on a B200
 * (Mrealisations/s, off / batch 4 wait 8 / batch 8 wait 16): full-size mix
 * 1.876 / 1.977 / 1.973, 1/4-scale mix 3.01 / 3.22 / 3.28, SW image 12.0 /
 * 12.1 / 12.3, LW flux 227 / 230 / 227. */
#ifndef HG_GAS_BATCH
#define HG_GAS_BATCH 8
#endif
#ifndef HG_GAS_WAIT
#define HG_GAS_WAIT 16
#endif
/* Batching of the trace stage's path loads (0: off).  Measured (off /
 * batch 4 wait 8 / batch 8 wait 16, gas batching on): full-size mix 1.979 /
 * 1.966 / 1.972, 1/4-scale mix 3.28 / 3.36 / 3.43, SW image 12.26 / 12.45 /
 * 12.59, LW flux 225 / 225 / 232 Mrealisations/s. */
#ifndef HG_FETCH_BATCH
#define HG_FETCH_BATCH 8
#endif
#ifndef HG_FETCH_WAIT
#define HG_FETCH_WAIT 16
#endif

/* Whether the next step of a trace is a whole gas region (the analytic
 * column of gas_region) */
__device__ __forceinline__ bool
trace_in_gas(const Trace& T)
{
  const int nreg = T.has_cloud ? 3 : 1;
  if(T.region >= nreg) return false;
  const bool cloud = T.has_cloud && T.region == 1;
  return !cloud && T.d.z != 0.f;
}

/* Slot storage: a path is kPathV4 16-byte vectors.  HG_WAVE_SOA 0 (default)
 * keeps a slot's vectors contiguous (a lane reading its own slot uses every
 * byte of the sectors it touches, whatever slots its warp holds); 1 stores
 * vector i of every slot together (coalesced only when a warp's slots are
 * consecutive). */
#ifndef HG_WAVE_SOA
#define HG_WAVE_SOA 0
#endif

__device__ __forceinline__ size_t
vec_at(uint32_t s, uint32_t i, uint32_t P)
{
#if HG_WAVE_SOA
  return (size_t)i * P + s;
#else
  (void)P;
  return (size_t)s * kPathV4 + i;
#endif
}

__device__ __forceinline__ void
load_path(Path& p, const uint4* paths, uint32_t s, uint32_t P)
{
  uint4 v[kPathV4];
#pragma unroll
  for(uint32_t i = 0; i < kPathV4; ++i) v[i] = paths[vec_at(s, i, P)];
  memcpy(&p, v, sizeof(Path));
}

__device__ __forceinline__ void
store_path(const Path& p, uint4* paths, uint32_t s, uint32_t P)
{
  uint4 v[kPathV4];
  v[kPathV4 - 1] = make_uint4(0, 0, 0, 0);
  memcpy(v, &p, sizeof(Path));
#pragma unroll
  for(uint32_t i = 0; i < kPathV4; ++i) paths[vec_at(s, i, P)] = v[i];
}

/* The trace part and the bytes up to the next 16-byte boundary (stored back
 * unchanged) */
__device__ __forceinline__ void
load_trace(Path& p, const uint4* paths, uint32_t s, uint32_t P)
{
  uint4 v[kTraceV4];
#pragma unroll
  for(uint32_t i = 0; i < kTraceV4; ++i) v[i] = paths[vec_at(s, i, P)];
  memcpy(&p, v, kTraceV4 * 16);
}

__device__ __forceinline__ void
store_trace(const Path& p, uint4* paths, uint32_t s, uint32_t P)
{
  uint4 v[kTraceV4];
  memcpy(v, &p, kTraceV4 * 16);
#pragma unroll
  for(uint32_t i = 0; i < kTraceV4; ++i) paths[vec_at(s, i, P)] = v[i];
}

/* Whether a trace that just ended leads to a transition the trace stage runs
 * itself: the absorption trace after a SW collision in the medium, the next
 * free path after a LW scattering in the medium over a plane ground */
__device__ __forceinline__ bool
transition_here(const Path& p, const DScene& S)
{
  if(p.state == ST_SW_SCAT_END) return p.tr.hit != 0;
  return p.state == ST_LW_END && p.tr.hit && p.tr.event == 1 && p.bounces < HG_MAX_BOUNCES
      && lw_plane_ground<HV_ALL>(S);
}

/* That transition; the event-part fields it sets are stored into slot s */
__device__ __forceinline__ void
transition(Path& p, const DScene& S, uint4* paths, uint32_t s, uint32_t P)
{
  if(p.state == ST_SW_SCAT_END) {
    const float3 pn = sw_scat_volume(p, S);
    paths[vec_at(s, kPnextV4, P)] =
      make_uint4(__float_as_uint(pn.x), __float_as_uint(pn.y), __float_as_uint(pn.z), 0u);
  } else {
    float3 pos, dir;
    lw_scatter_plane(p, S, pos, dir);
    uint4* v = paths + vec_at(s, kPosV4, P);
    ((uint2*)v)[1] = make_uint2(__float_as_uint(pos.x), __float_as_uint(pos.y));
    v = paths + vec_at(s, kPosV4 + 1, P);
    *v = make_uint4(__float_as_uint(pos.z), __float_as_uint(dir.x), __float_as_uint(dir.y),
                    __float_as_uint(dir.z));
  }
}

}  // namespace

/* Control block of a wavefront run (device) */
struct WTables {
  PTables T;
  uint4* paths;     /* P slots of kPathV4 vectors (vec_at) */
  uint32_t* list0;  /* live lists, P entries each */
  uint32_t* list1;
  uint32_t* dead;   /* free slots (serving: revived when work arrives), or null */
  WCtl* ctl;
  uint32_t P;
  uint32_t budget;  /* voxel steps per trace-stage visit */
};

/* Iteration parity b: the event stage reads list b and writes list b^1; the
 * trace stage then walks list b^1. */
template <unsigned V>
__global__ void __launch_bounds__(128)
k_wave_event(WTables W, uint32_t b, int tables_in_smem)
{
  extern __shared__ __align__(16) unsigned char smem[];
  PTables T = W.T;
  if(tables_in_smem) tables_to_smem(T, smem);
  WCtl* ctl = W.ctl;
  if(blockIdx.x == 0 && threadIdx.x == 0) ctl->fetch_trace = 0;
  const uint32_t* in = b ? W.list1 : W.list0;
  uint32_t* out = b ? W.list0 : W.list1;
  const uint32_t n_in = ctl->n_live[b];
  uint32_t* n_out = &ctl->n_live[b ^ 1u];
  const unsigned lane = threadIdx.x & 31u;
  unsigned long long seg = 0, node = 0, tc = 0, real = 0, fail = 0;

  for(;;) {
    uint32_t base = 0;
    if(lane == 0) base = atomicAdd(&ctl->fetch_event, 32u);
    base = __shfl_sync(0xffffffffu, base, 0);
    if(base >= n_in) break;
    const uint32_t idx = base + lane;
    const bool active = idx < n_in;
    const uint32_t s = active ? in[idx] : 0u;
    Path p;
    p.state = ST_IDLE;
    if(active) {
      load_path(p, W.paths, s, W.P);
      p.t0 = gtimer() - p.t0; /* stored: busy time so far */
    }
    bool drained = !active;
    for(;;) {
      /* regeneration: idle lanes take the next realisations of the queue */
      const bool need = p.state == ST_IDLE && !drained;
      const unsigned m = __ballot_sync(0xffffffffu, need);
      if(m) {
        const unsigned leader = __ffs(m) - 1;
        unsigned long long g0 = 0;
        unsigned got = 0;
        if(lane == leader) g0 = queue_take(T, (unsigned)__popc(m), &got);
        g0 = __shfl_sync(0xffffffffu, g0, leader);
        got = __shfl_sync(0xffffffffu, got, leader);
        if(need) {
          const unsigned rank = __popc(m & ((1u << lane) - 1u));
          if(rank < got) path_assign(p, T, g0 + rank);
          else drained = true;
        }
      }
      const bool busy = p.state != ST_IDLE && p.state != ST_TRACE;
      if(!__any_sync(0xffffffffu, busy)) break;
      if(busy) {
        if(p.state != ST_DONE) {
          path_event<V>(p, T.scenes[p.si], T.reqs[p.ri]);
          seg += p.c_seg; node += p.c_node; tc += p.c_tc;
          p.c_seg = p.c_node = p.c_tc = 0;
        }
        if(p.state == ST_DONE) {
          accumulate_b(p, T.reqs[p.ri]);
          count_grid(T.cnt, p);
          real += (p.flags & (PF_REJECTED | PF_FAILED)) ? 0 : 1;
          fail += (p.flags & PF_FAILED) ? 1 : 0;
          p.state = ST_IDLE;
        }
      }
    }
    const bool keep = p.state == ST_TRACE;
    if(keep) {
      p.t0 = gtimer() - p.t0;
      store_path(p, W.paths, s, W.P);
    }
    const unsigned km = __ballot_sync(0xffffffffu, keep);
    if(km) {
      uint32_t pos = 0;
      if(lane == 0) pos = atomicAdd(n_out, (uint32_t)__popc(km));
      pos = __shfl_sync(0xffffffffu, pos, 0);
      if(keep) out[pos + __popc(km & ((1u << lane) - 1u))] = s;
    }
    /* serving: a slot left without work waits, idle, on the dead list */
    const bool died = active && !keep && W.dead;
    if(died) store_path(p, W.paths, s, W.P); /* p.state is ST_IDLE */
    const unsigned dm = __ballot_sync(0xffffffffu, died);
    if(dm) {
      uint32_t pos = 0;
      if(lane == 0) pos = atomicAdd(&ctl->n_dead, (uint32_t)__popc(dm));
      pos = __shfl_sync(0xffffffffu, pos, 0);
      if(died) W.dead[pos + __popc(dm & ((1u << lane) - 1u))] = s;
    }
  }
  flush_counts(T.cnt, seg, node, tc, real, fail);
}

__global__ void __maxnreg__(HG_WAVE_TRACE_MAXNREG)
k_wave_trace(WTables W, uint32_t b, int tables_in_smem)
{
  extern __shared__ __align__(16) unsigned char smem[];
  PTables T = W.T;
  if(tables_in_smem) tables_to_smem(T, smem);
  WCtl* ctl = W.ctl;
  if(blockIdx.x == 0 && threadIdx.x == 0) {
    ctl->fetch_event = 0;
    ctl->n_live[b] = 0; /* the next event stage's output */
    queue_clamp(T);     /* no stage takes work while this one runs */
  }
  const uint32_t* list = b ? W.list0 : W.list1;
  const uint32_t n = ctl->n_live[b ^ 1u];
  const unsigned lane = threadIdx.x & 31u;
  Path p;
  p.state = ST_IDLE;
  bool have = false, drained = false;
  uint32_t s = 0, left = 0;
#if HG_GAS_BATCH
  uint32_t waited = 0; /* warp-uniform */
#endif
#if HG_FETCH_BATCH
  uint32_t idle = 0; /* warp-uniform */
#endif
  for(;;) {
    const bool need = !have && !drained;
    unsigned m = __ballot_sync(0xffffffffu, need);
#if HG_FETCH_BATCH
    /* lanes whose path left wait until HG_FETCH_BATCH of them (or every
     * lane) can load a new one, or for HG_FETCH_WAIT iterations: the warp
     * then waits once on the loads of several paths */
    if(m && __popc(m) < HG_FETCH_BATCH && __any_sync(0xffffffffu, have) && idle < HG_FETCH_WAIT) {
      ++idle;
      m = 0;
    } else {
      idle = 0;
    }
#endif
    if(m) {
      const unsigned leader = __ffs(m) - 1;
      uint32_t i0 = 0;
      if(lane == leader) i0 = atomicAdd(&ctl->fetch_trace, (uint32_t)__popc(m));
      i0 = __shfl_sync(0xffffffffu, i0, leader);
      if(m & (1u << lane)) {
        const uint32_t idx = i0 + __popc(m & ((1u << lane) - 1u));
        if(idx < n) {
          s = list[idx];
          load_trace(p, W.paths, s, W.P);
          p.t0 = gtimer() - p.t0;
          have = true;
          left = W.budget;
        } else {
          drained = true;
        }
      }
    }
    if(!__any_sync(0xffffffffu, have)) break;
    bool go = have;
#if HG_GAS_BATCH
    {
      /* a gas region (an analytic column, several times a voxel step's code)
       * waits until HG_GAS_BATCH lanes of the warp want one, or for
       * HG_GAS_WAIT iterations, so that its code runs with more lanes */
      const bool gas = have && trace_in_gas(p.tr);
      const unsigned gm = __ballot_sync(0xffffffffu, gas);
      const unsigned am = __ballot_sync(0xffffffffu, have);
      if(gm && gm != am && __popc(gm) < HG_GAS_BATCH && waited < HG_GAS_WAIT) {
        ++waited;
        go = have && !gas;
      } else {
        waited = 0;
      }
    }
#endif
    if(go) {
      trace_step<HV_ALL>(p, T.scenes[p.si]);
      if(transition_here(p, T.scenes[p.si])) transition(p, T.scenes[p.si], W.paths, s, W.P);
      if(p.state != ST_TRACE || --left == 0) {
        p.t0 = gtimer() - p.t0;
        store_trace(p, W.paths, s, W.P);
        have = false;
      }
    }
  }
}

/* Live list 0 = the first n0 slots, list 1 empty, counters at zero */
__global__ void
k_wave_init(WTables W, uint32_t n0)
{
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if(i < n0) W.list0[i] = i;
  if(i == 0) {
    W.ctl->n_live[0] = n0;
    W.ctl->n_live[1] = 0;
    W.ctl->fetch_event = 0;
    W.ctl->fetch_trace = 0;
    W.ctl->fetch_finish = 0;
    W.ctl->n_dead = 0;
  }
}

/* Serving pool reset: every slot free (on the dead list), no live path */
__global__ void
k_wave_reset(WTables W)
{
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if(i < W.P) W.dead[i] = i;
  if(i == 0) {
    W.ctl->n_live[0] = 0;
    W.ctl->n_live[1] = 0;
    W.ctl->fetch_event = 0;
    W.ctl->fetch_trace = 0;
    W.ctl->fetch_finish = 0;
    W.ctl->n_dead = W.P;
  }
}

/* Serving: new work arrived, the free slots join live list 0 (idle paths
 * that the next event stage regenerates).  Between two chunks every slot is
 * either on list 0 or on the dead list, so the copy stays inside list 0. */
__global__ void
k_wave_revive(WTables W)
{
  const uint32_t n = W.ctl->n_dead, base = W.ctl->n_live[0];
  for(uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    if(base + i < W.P) W.list0[base + i] = W.dead[i];
}

__global__ void
k_wave_revive_commit(WTables W)
{
  if(threadIdx.x == 0 && blockIdx.x == 0) {
    const uint32_t n = W.ctl->n_live[0] + W.ctl->n_dead;
    W.ctl->n_live[0] = n < W.P ? n : W.P;
    W.ctl->n_dead = 0;
  }
}

/* Queue head back to the queued total after a launch that takes work */
__global__ void
k_wave_clamp(WTables W)
{
  if(threadIdx.x == 0 && blockIdx.x == 0) queue_clamp(W.T);
}

/* The tail of a run: once few paths are live, iterations would cost their
 * launch and one trace's latency each while moving almost no work, so the
 * remaining paths finish in one megakernel launch.  Lanes resume the paths of
 * live list 0 from their slots, then take any realisations left in the work
 * queue; events and traces run in the same thread, events regrouped every
 * `regroup_period' voxel steps as in the persistent engine. */
template <unsigned V>
__global__ void __maxnreg__(HG_PERSIST_MAXNREG)
k_wave_finish(WTables W, int tables_in_smem)
{
  extern __shared__ __align__(16) unsigned char smem[];
  PTables T = W.T;
  if(tables_in_smem) tables_to_smem(T, smem);
  WCtl* ctl = W.ctl;
  const uint32_t n = ctl->n_live[0];
  const unsigned lane = threadIdx.x & 31u;
  Path p;
  p.state = ST_IDLE;
  p.flags = 0;
  p.c_seg = p.c_node = p.c_tc = 0;
  p.ri = p.si = 0;
  bool list_done = false, drained = false;
  unsigned long long seg = 0, node = 0, tc = 0, real = 0, fail = 0;
  const uint32_t period = T.regroup_period > 1 ? T.regroup_period : 1;

  for(uint32_t it = 0;; ++it) {
    const unsigned tmask = __ballot_sync(0xffffffffu, p.state == ST_TRACE);
    if(tmask && (it % period) != 0) {
      if(p.state == ST_TRACE) trace_step<V>(p, T.scenes[p.si]);
      continue;
    }
    /* idle lanes: a saved path of the live list first, then the queue */
    const bool need_l = p.state == ST_IDLE && !list_done;
    const unsigned ml = __ballot_sync(0xffffffffu, need_l);
    if(ml) {
      const unsigned leader = __ffs(ml) - 1;
      uint32_t i0 = 0;
      if(lane == leader) i0 = atomicAdd(&ctl->fetch_finish, (uint32_t)__popc(ml));
      i0 = __shfl_sync(0xffffffffu, i0, leader);
      if(need_l) {
        const uint32_t idx = i0 + __popc(ml & ((1u << lane) - 1u));
        if(idx < n) {
          load_path(p, W.paths, W.list0[idx], W.P);
          p.t0 = gtimer() - p.t0;
        } else {
          list_done = true;
        }
      }
    }
    const bool need_q = p.state == ST_IDLE && list_done && !drained;
    const unsigned mq = __ballot_sync(0xffffffffu, need_q);
    if(mq) {
      const unsigned leader = __ffs(mq) - 1;
      unsigned long long g0 = 0;
      unsigned got = 0;
      if(lane == leader) g0 = queue_take(T, (unsigned)__popc(mq), &got);
      g0 = __shfl_sync(0xffffffffu, g0, leader);
      got = __shfl_sync(0xffffffffu, got, leader);
      if(need_q) {
        const unsigned rank = __popc(mq & ((1u << lane) - 1u));
        if(rank < got) path_assign(p, T, g0 + rank);
        else drained = true;
      }
    }
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

size_t
wave_slot_bytes()
{
  return (size_t)kPathV4 * 16 + 2 * sizeof(uint32_t);
}

WaveBufs::~WaveBufs()
{
  if(host_ctl) cudaFreeHost(host_ctl);
  if(ev[0]) cudaEventDestroy(ev[0]);
  if(ev[1]) cudaEventDestroy(ev[1]);
}

WaveBufs&
thread_wave(int device)
{
  static thread_local std::map<int, std::unique_ptr<WaveBufs>> pools;
  std::unique_ptr<WaveBufs>& w = pools[device];
  if(!w) w = std::make_unique<WaveBufs>();
  return *w;
}

/* Slots of a run: enough paths in flight to keep every trace lane busy
 * several times over, no more than the realisations to render */
static uint32_t
wave_slots(const htrdr_gpu_tuning& tun, uint64_t total)
{
  uint64_t P = tun.wave_slots ? tun.wave_slots : kDefaultWaveSlots;
  if(P > total) P = total;
  if(P < 1) P = 1;
  return (uint32_t)P;
}

bool
wave_reserve(WaveBufs& B, uint32_t P)
{
  if(!B.ctl.ptr && !B.ctl.alloc(sizeof(WCtl) * 2)) return false;
  if(!B.host_ctl) {
    if(!cuda_ok(cudaHostAlloc(&B.host_ctl, 2 * sizeof(WCtl), cudaHostAllocDefault), "cudaHostAlloc"))
      return false;
    if(!cuda_ok(cudaEventCreateWithFlags(&B.ev[0], cudaEventDisableTiming), "event")
    || !cuda_ok(cudaEventCreateWithFlags(&B.ev[1], cudaEventDisableTiming), "event"))
      return false;
  }
  if(B.P >= P && B.paths.ptr) return true;
  if(B.paths.ptr) { cudaFree(B.paths.ptr); B.paths.ptr = nullptr; B.paths.bytes = 0; }
  if(B.lists.ptr) { cudaFree(B.lists.ptr); B.lists.ptr = nullptr; B.lists.bytes = 0; }
  if(!B.paths.alloc((size_t)P * kPathV4 * 16) || !B.lists.alloc((size_t)P * 2 * sizeof(uint32_t)))
    return false;
  B.P = P;
  return true;
}

namespace {

using WaveEventFn = void (*)(WTables, uint32_t, int);
using WaveFinishFn = void (*)(WTables, int);
WaveEventFn
wave_event_fn(uint32_t v)
{
  HG_PICK_VARIANT(v, k_wave_event)
}
WaveFinishFn
wave_finish_fn(uint32_t v)
{
  HG_PICK_VARIANT(v, k_wave_finish)
}

/* Launch shapes of a run over the tables T */
struct WaveLaunch {
  size_t smem = 0;
  size_t fi_smem = 0; /* of the finishing kernel */
  int in_smem = 0;
  unsigned ev_grid = 0, tr_grid = 0, fi_grid = 0;
  uint32_t tb = 256;
  uint64_t tail = 0;  /* live paths below which the rest finishes in the megakernel */
  /* the event and tail kernels of the tables' scenes (with or without the
   * ground-mesh queries) */
  void (*ev)(WTables, uint32_t, int) = nullptr;
  void (*fi)(WTables, int) = nullptr;
};

cudaError_t
wave_params(const PTables& T, const htrdr_gpu_tuning& tun, int device, WaveLaunch& L)
{
  const size_t tables = ((T.nscenes * sizeof(DScene) + 15) & ~(size_t)15) + T.nreqs * sizeof(DRequest);
  L.in_smem = tables <= 96 * 1024;
  L.smem = L.in_smem ? tables : 0;
  L.ev = wave_event_fn(T.variant);
  L.fi = wave_finish_fn(T.variant);
  L.tb = tun.block_size ? tun.block_size : 256;
  L.fi_smem = L.smem;
  cudaError_t e;
  if(L.smem > 48 * 1024) {
    if((e = cudaFuncSetAttribute(L.ev, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)L.smem)))
      return e;
    if((e = cudaFuncSetAttribute(k_wave_trace, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)L.smem)))
      return e;
  }
  if(L.fi_smem > 48 * 1024
  && (e = cudaFuncSetAttribute(L.fi, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)L.fi_smem)))
    return e;
  int nsm = 0, ev_per_sm = 0, tr_per_sm = 0, fi_per_sm = 0;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&ev_per_sm, L.ev, 128, L.smem);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&tr_per_sm, k_wave_trace, (int)L.tb, L.smem);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&fi_per_sm, L.fi, (int)L.tb, L.fi_smem);
  if(tun.blocks_per_sm) tr_per_sm = std::min(tr_per_sm, (int)tun.blocks_per_sm);
  L.ev_grid = (unsigned)(nsm * std::max(ev_per_sm, 1));
  L.tr_grid = (unsigned)(nsm * std::max(tr_per_sm, 1));
  L.fi_grid = (unsigned)(nsm * std::max(fi_per_sm, 1));
  L.tail = tun.wave_tail ? tun.wave_tail : 4ull * L.fi_grid * L.tb;
  return cudaSuccess;
}

WTables
wave_tables(const PTables& T, const htrdr_gpu_tuning& tun, WaveBufs& B, bool serving)
{
  WTables W;
  W.T = T;
  W.paths = (uint4*)B.paths.ptr;
  W.list0 = (uint32_t*)B.lists.ptr;
  W.list1 = W.list0 + B.P;
  W.dead = serving ? (uint32_t*)B.dead.ptr : nullptr;
  W.ctl = (WCtl*)B.ctl.ptr;
  W.P = B.P;
  W.budget = tun.trace_budget ? tun.trace_budget : 256;
  return W;
}

/* C iterations (C even: a chunk starts and ends at parity 0, live list 0) */
cudaError_t
wave_iterations(const WTables& W, const WaveLaunch& L, uint32_t C, cudaStream_t st)
{
  for(uint32_t i = 0; i < C; ++i) {
    const uint32_t b = i & 1u;
    L.ev<<<L.ev_grid, 128, L.smem, st>>>(W, b, L.in_smem);
    k_wave_trace<<<L.tr_grid, L.tb, L.smem, st>>>(W, b, L.in_smem);
  }
  note_launches(2 * C);
  return cudaGetLastError();
}

}  // namespace

cudaError_t
launch_wavefront(const PTables& T, const htrdr_gpu_tuning& tun, WaveBufs& B, int device,
                 cudaStream_t st)
{
  if(!T.total) return cudaSuccess;
  const uint32_t P = wave_slots(tun, T.total);
  if(!wave_reserve(B, P)) return cudaErrorMemoryAllocation;
  WaveLaunch L;
  cudaError_t e = wave_params(T, tun, device, L);
  if(e) return e;
  WTables W = wave_tables(T, tun, B, false);
  W.P = P; /* the buffers may hold more slots than this run uses */

  /* a run too small to fill the stages is all tail: the megakernel takes the
   * whole queue */
  if(P < L.tail) {
    k_wave_init<<<1, 32, 0, st>>>(W, 0u);
    L.fi<<<L.fi_grid, L.tb, L.fi_smem, st>>>(W, L.in_smem);
    note_launches(2);
    return cudaGetLastError();
  }

  /* every slot starts idle (ST_IDLE is 0) */
  if((e = cudaMemsetAsync(B.paths.ptr, 0, (size_t)P * kPathV4 * 16, st))) return e;
  k_wave_init<<<(P + 255) / 256, 256, 0, st>>>(W, P);
  note_launches(1);
  if((e = cudaGetLastError())) return e;

  /* after each chunk the live count of its last event stage (list 0) is
   * copied back.  Two chunks are in flight: the host checks chunk k-1 while
   * chunk k runs. */
  const uint32_t C = 8;
  const uint64_t max_chunks = 1ull << 22;
  WCtl* hctl = (WCtl*)B.host_ctl;
  for(uint64_t k = 0;; ++k) {
    if(k >= max_chunks) return cudaErrorLaunchTimeout;
    if((e = wave_iterations(W, L, C, st))) return e;
    if((e = cudaMemcpyAsync(hctl + (k & 1), B.ctl.ptr, sizeof(WCtl), cudaMemcpyDeviceToHost, st)))
      return e;
    if((e = cudaEventRecord(B.ev[k & 1], st))) return e;
    if(k >= 1) {
      if((e = cudaEventSynchronize(B.ev[(k - 1) & 1]))) return e;
      const uint32_t live = hctl[(k - 1) & 1].n_live[0];
      if(live == 0) break;  /* chunk k runs empty stages */
      if(live < L.tail) {   /* after chunk k, the megakernel finishes list 0 */
        L.fi<<<L.fi_grid, L.tb, L.fi_smem, st>>>(W, L.in_smem);
        note_launches(1);
        return cudaGetLastError();
      }
    }
  }
  return cudaSuccess;
}

/* ---- serving: a pool of P slots driven chunk by chunk ---- */

cudaError_t
wave_serve_reset(WaveBufs& B, uint32_t P, cudaStream_t st)
{
  if(!wave_reserve(B, P)) return cudaErrorMemoryAllocation;
  if(B.dead.bytes < (size_t)B.P * sizeof(uint32_t)) {
    if(B.dead.ptr) { cudaFree(B.dead.ptr); B.dead.ptr = nullptr; B.dead.bytes = 0; }
    if(!B.dead.alloc((size_t)B.P * sizeof(uint32_t))) return cudaErrorMemoryAllocation;
  }
  htrdr_gpu_tuning t;
  htrdr_gpu_default_tuning(&t);
  const WTables W = wave_tables(PTables{}, t, B, true);
  cudaError_t e = cudaMemsetAsync(B.paths.ptr, 0, (size_t)B.P * kPathV4 * 16, st);
  if(e) return e;
  k_wave_reset<<<(B.P + 255) / 256, 256, 0, st>>>(W);
  note_launches(1);
  return cudaGetLastError();
}

cudaError_t
wave_serve_revive(WaveBufs& B, cudaStream_t st)
{
  htrdr_gpu_tuning t;
  htrdr_gpu_default_tuning(&t);
  const WTables W = wave_tables(PTables{}, t, B, true);
  k_wave_revive<<<std::max(1u, std::min(1024u, (B.P + 255) / 256)), 256, 0, st>>>(W);
  k_wave_revive_commit<<<1, 32, 0, st>>>(W);
  note_launches(2);
  return cudaGetLastError();
}

cudaError_t
wave_serve_chunk(const PTables& T, const htrdr_gpu_tuning& tun, WaveBufs& B, int device,
                 uint32_t iterations, cudaStream_t st)
{
  WaveLaunch L;
  cudaError_t e = wave_params(T, tun, device, L);
  if(e) return e;
  return wave_iterations(wave_tables(T, tun, B, true), L, iterations & ~1u, st);
}

cudaError_t
wave_serve_finish(const PTables& T, const htrdr_gpu_tuning& tun, WaveBufs& B, int device,
                  cudaStream_t st)
{
  WaveLaunch L;
  cudaError_t e = wave_params(T, tun, device, L);
  if(e) return e;
  const WTables W = wave_tables(T, tun, B, true);
  L.fi<<<L.fi_grid, L.tb, L.fi_smem, st>>>(W, L.in_smem);
  k_wave_clamp<<<1, 32, 0, st>>>(W);
  note_launches(2);
  if((e = cudaGetLastError())) return e;
  return wave_serve_reset(B, B.P, st); /* every slot is free again */
}

uint64_t
wave_serve_tail(const htrdr_gpu_tuning& tun, int device)
{
  WaveLaunch L;
  PTables T{};
  if(wave_params(T, tun, device, L)) return 0;
  return L.tail;
}

}  // namespace hg
