/* Device pieces shared by the work-queue engines (persistent megakernel and
 * wavefront): item lookup in the realisation index space and the FP64
 * accumulation of a finished realisation into its request's accumulators. */
#ifndef HTRDR_ENGINE_CUH
#define HTRDR_ENGINE_CUH

#include "internal.h"
#include "transport.cuh"

#include <cooperative_groups.h>
#include <cooperative_groups/reduce.h>

/* Order of a request's realisations in the work queue: realisation-major
 * (0: consecutive realisations are on different pixels) or pixel-major (1:
 * the realisations of a pixel are consecutive, so the lanes that take them
 * together sample the same sensor region).  Realisation-major measured
 * faster: 121.6 against 100.2 Mrealisations/s on the LW flux map with the
 * aggregation below, equal on the SW/LW mix. */
#ifndef HG_PIXEL_MAJOR
#define HG_PIXEL_MAJOR 0
#endif
/* Lanes that finish realisations of the same pixel together add their
 * weights with one set of atomics (cooperative-groups partition by pixel);
 * off by default (see above). */
#ifndef HG_AGGREGATE
#define HG_AGGREGATE 0
#endif

namespace {

/* Item holding global realisation g: the last item whose offset is <= g */
__device__ __forceinline__ uint32_t
find_item(const hg::PTables& T, uint64_t g)
{
  uint32_t lo = 0, hi = T.nitems;
  while(hi - lo > 1) {
    const uint32_t mid = (lo + hi) >> 1;
    if(__ldg(T.offsets + mid) <= g) lo = mid; else hi = mid;
  }
  return lo;
}

/* Per-pixel estimator sums (src/core/htrdr_accum.h:31-68) and the
 * realisation time, for a path in ST_DONE.  Called by the lanes of a warp
 * whose paths ended, in any subset. */
__device__ __forceinline__ void
accumulate_b(const Path& p, const DRequest& R)
{
  if(R.ndone) atomicAdd(R.ndone, 1ull); /* every realisation, rejected ones included */
  if(p.flags & PF_REJECTED) return;
  const uint32_t nch = R.mode == HG_IMAGE_CIE ? 3u : 1u;
  DAccum* a = R.acc + (size_t)p.pix * nch + p.chan;
  if(p.flags & PF_FAILED) { atomicAdd(&a->pad, 1ull); return; }
  const double us = (double)(gtimer() - p.t0) * 1e-3;
  DAccum* t = R.tacc + p.pix;
#if HG_AGGREGATE
  namespace cg = cooperative_groups;
  /* the lanes here that add to the same accumulator sum first; the time
   * accumulator of a pixel is shared by its channels, so it is grouped by
   * pixel apart */
  const cg::coalesced_group here = cg::coalesced_threads();
  const cg::coalesced_group same = cg::labeled_partition(here, (unsigned long long)(uintptr_t)a);
  const double w = cg::reduce(same, p.weight, cg::plus<double>());
  const double w2 = cg::reduce(same, p.weight * p.weight, cg::plus<double>());
  if(same.thread_rank() == 0) {
    atomicAdd(&a->s, w);
    atomicAdd(&a->s2, w2);
    atomicAdd(&a->n, (unsigned long long)same.size());
  }
  const cg::coalesced_group pix = cg::labeled_partition(here, (unsigned long long)(uintptr_t)t);
  const double ts = cg::reduce(pix, us, cg::plus<double>());
  const double ts2 = cg::reduce(pix, us * us, cg::plus<double>());
  if(pix.thread_rank() == 0) {
    atomicAdd(&t->s, ts);
    atomicAdd(&t->s2, ts2);
    atomicAdd(&t->n, (unsigned long long)pix.size());
  }
#else
  atomicAdd(&a->s, p.weight);
  atomicAdd(&a->s2, p.weight * p.weight);
  atomicAdd(&a->n, 1ull);
  atomicAdd(&t->s, us);
  atomicAdd(&t->s2, us * us);
  atomicAdd(&t->n, 1ull);
#endif
}

/* Start realisation `g' (global index) in path p: request, scene, pixel and
 * realisation of the item that holds it */
__device__ __forceinline__ void
path_assign(Path& p, const hg::PTables& T, uint64_t g)
{
  const uint32_t ii = find_item(T, g);
  const hg::PItem item = T.items[ii];
  p.ri = item.req;
  p.si = item.scene;
  const DRequest& R = T.reqs[item.req];
  const uint64_t local = g - __ldg(T.offsets + ii) + item.begin;
#if HG_PIXEL_MAJOR
  p.pix = (uint32_t)(local / R.nreal_pp);
  p.ireal = (uint32_t)(local % R.nreal_pp);
#else
  const uint32_t npix = R.width * R.height;
  p.ireal = (uint32_t)(local / npix);
  p.pix = (uint32_t)(local % npix);
#endif
  p.state = ST_GEN;
}

/* Takes up to n realisations from the work queue (one atomic per warp).
 * Returns the first index; *got is how many were taken (0: empty).  The head
 * may pass the queued total; the wavefront's trace stage, which takes no
 * work, clamps it back, so that work appended between chunks starts exactly
 * at the head. */
__device__ __forceinline__ unsigned long long
queue_take(const hg::PTables& T, unsigned n, unsigned* got)
{
  const unsigned long long old = atomicAdd(T.next, (unsigned long long)n);
  *got = old >= T.total ? 0u : (unsigned)(T.total - old < n ? T.total - old : n);
  return old;
}

/* Head back to the queued total (one thread, while no warp takes work) */
__device__ __forceinline__ void
queue_clamp(const hg::PTables& T)
{
  if(*T.next > T.total) *T.next = T.total;
}

/* Warp-wide sums of the event counters, added to the launch's totals */
__device__ __forceinline__ void
flush_counts(void* cnt, unsigned long long seg, unsigned long long node, unsigned long long tc,
             unsigned long long real, unsigned long long fail)
{
  for(int o = 16; o > 0; o >>= 1) {
    seg += __shfl_down_sync(0xffffffffu, seg, o);
    node += __shfl_down_sync(0xffffffffu, node, o);
    tc += __shfl_down_sync(0xffffffffu, tc, o);
    real += __shfl_down_sync(0xffffffffu, real, o);
    fail += __shfl_down_sync(0xffffffffu, fail, o);
  }
  if((threadIdx.x & 31u) == 0) {
    Counters* c = (Counters*)cnt;
    atomicAdd(&c->seg, seg);
    atomicAdd(&c->node, node);
    atomicAdd(&c->tc, tc);
    atomicAdd(&c->real, real);
    atomicAdd(&c->fail, fail);
  }
}

/* Leaf-grid bytes read by a completed path, added to the launch's total: one
 * atomic per realisation, so that no engine keeps another running counter */
__device__ __forceinline__ void
count_grid(void* cnt, const Path& p)
{
  if(p.c_grid) atomicAdd(&((Counters*)cnt)->grid, (unsigned long long)p.c_grid);
}

/* Copy the scene and request tables of a launch into shared memory (one
 * copy per block) and point T at them */
/* A path held in shared memory, padded to an odd number of 8-byte words
 * when the path has an even number, so that a warp's 8-byte accesses to one
 * field of 32 slots are free of bank conflicts. */
template <bool Pad> struct __align__(8) PathSlotT { Path p; uint32_t pad[2]; };
template <> struct __align__(8) PathSlotT<false> { Path p; };
using PathSlot = PathSlotT<sizeof(Path) % 16 == 0>;
static_assert(sizeof(PathSlot) % 16 == 8, "odd number of 8-byte words per slot");

/* Shared-memory bytes of the path slots of a block (16-byte rounded) */
__host__ __device__ constexpr size_t
path_slots_bytes(uint32_t threads)
{
  return ((size_t)threads * sizeof(PathSlot) + 15) & ~(size_t)15;
}

/* Where the persistent kernel keeps a lane's path.  LW-only launches keep it
 * in shared memory: with the path out of the registers the kernel needs ~156
 * of them instead of 216, so 12 warps fit on an SM instead of 8, and LW
 * walks are short enough that the shared-memory latency of each field access
 * costs less than the occupancy gains (1149 against 919 Mrealisations/s on
 * the LW flux map).  Shortwave walks are long and touch the path state
 * between every dependent load: they keep it in registers (in shared memory
 * the SW image ran 23 % slower). */
__host__ __device__ constexpr bool
persistent_smem_paths(unsigned v)
{
  return (v & HV_SW) == 0;
}

__device__ __forceinline__ void
tables_to_smem(hg::PTables& T, unsigned char* smem)
{
  DScene* ss = (DScene*)smem;
  DRequest* sr = (DRequest*)(smem + ((T.nscenes * sizeof(DScene) + 15) & ~(size_t)15));
  const uint32_t* gs = (const uint32_t*)T.scenes;
  const uint32_t* gr = (const uint32_t*)T.reqs;
  for(uint32_t i = threadIdx.x; i < T.nscenes * sizeof(DScene) / 4; i += blockDim.x) ((uint32_t*)ss)[i] = gs[i];
  for(uint32_t i = threadIdx.x; i < T.nreqs * sizeof(DRequest) / 4; i += blockDim.x) ((uint32_t*)sr)[i] = gr[i];
  __syncthreads();
  T.scenes = ss;
  T.reqs = sr;
}

/* Shared-memory bytes of the sorted kernel's stage lists (two lists of slot
 * indices and their counters) */
__host__ __device__ constexpr size_t
sorted_lists_bytes(uint32_t threads)
{
  return ((size_t)2 * threads * sizeof(uint32_t) + 4 * sizeof(uint32_t) + 15) & ~(size_t)15;
}

/* The block-sorted loop.  The block's paths live in shared-memory
 * slots that any lane may run, so every step the block sorts its slots by
 * stage -- tracing, or waiting for an event (or for new work) -- into two
 * lists, and lanes 0..n-1 take the n entries of each list in turn.  The
 * warps of each pass are therefore full of lanes in the same stage (the
 * ballot regrouping of persistent_loop only gathers the lanes a warp owns),
 * and warps past the end of a list skip it.  `regroup_period' voxel steps are
 * taken per trace visit.  Same state machine, same streams, same weights. */
template <unsigned V>
__device__ __forceinline__ void
sorted_loop(hg::PTables& T, PathSlot* slots, uint32_t* lists)
{
  const uint32_t B = blockDim.x, tid = threadIdx.x, lane = tid & 31u;
  uint32_t* trace_list = lists;
  uint32_t* event_list = lists + B;
  uint32_t* n = lists + 2 * B; /* [0] tracing, [1] events, [2] queue drained */
  unsigned long long seg = 0, node = 0, tc = 0, real = 0, fail = 0;
  const uint32_t period = T.regroup_period > 1 ? T.regroup_period : 1;
  {
    Path& own = slots[tid].p;
    own.state = ST_IDLE;
    own.flags = 0;
    own.c_seg = own.c_node = own.c_tc = 0;
    own.ri = own.si = 0;
  }
  if(tid == 0) n[2] = 0;
  for(;;) {
    if(tid == 0) { n[0] = 0; n[1] = 0; }
    __syncthreads();
    { /* sort: each thread files the slot of its own index */
      const uint8_t st = slots[tid].p.state;
      const bool tr = st == ST_TRACE;
      const bool ev = !tr && (st != ST_IDLE || !n[2]);
      const unsigned mt = __ballot_sync(0xffffffffu, tr);
      const unsigned me = __ballot_sync(0xffffffffu, ev);
      uint32_t bt = 0, be = 0;
      if(lane == 0) {
        if(mt) bt = atomicAdd(&n[0], (uint32_t)__popc(mt));
        if(me) be = atomicAdd(&n[1], (uint32_t)__popc(me));
      }
      bt = __shfl_sync(0xffffffffu, bt, 0);
      be = __shfl_sync(0xffffffffu, be, 0);
      const unsigned below = (1u << lane) - 1u;
      if(tr) trace_list[bt + __popc(mt & below)] = tid;
      if(ev) event_list[be + __popc(me & below)] = tid;
    }
    __syncthreads();
    const uint32_t ntr = n[0], nev = n[1];
    if(ntr == 0 && nev == 0) break;
    /* trace pass */
    if(tid < ntr) {
      Path& p = slots[trace_list[tid]].p;
      const DScene& S = T.scenes[p.si];
      for(uint32_t k = 0; k < period && p.state == ST_TRACE; ++k) trace_step<V>(p, S);
    }
    /* event pass: accumulate finished paths, give idle slots new work, run
     * events until the path needs a trace or ends */
    if((tid & ~31u) < nev) { /* warps with at least one entry; all their lanes vote */
      const bool act = tid < nev;
      Path& p = slots[act ? event_list[tid] : 0].p;
      if(act && p.state == ST_DONE) {
        accumulate_b(p, T.reqs[p.ri]);
        count_grid(T.cnt, p);
        real += (p.flags & (PF_REJECTED | PF_FAILED)) ? 0 : 1;
        fail += (p.flags & PF_FAILED) ? 1 : 0;
        seg += p.c_seg; node += p.c_node; tc += p.c_tc;
        p.c_seg = p.c_node = p.c_tc = 0;
        p.state = ST_IDLE;
      }
      const bool need = act && p.state == ST_IDLE && !n[2];
      const unsigned m = __ballot_sync(0xffffffffu, need);
      if(m) {
        const unsigned leader = __ffs(m) - 1;
        unsigned long long base = 0;
        if(lane == leader) base = atomicAdd(T.next, (unsigned long long)__popc(m));
        base = __shfl_sync(0xffffffffu, base, leader);
        if(need) {
          const unsigned long long g = base + (unsigned long long)__popc(m & ((1u << lane) - 1u));
          if(g < T.total) path_assign(p, T, g);
          else n[2] = 1; /* the queue is drained: idle slots stop asking */
        }
      }
      if(act && p.state != ST_IDLE && p.state != ST_TRACE && p.state != ST_DONE) {
        path_event<V>(p, T.scenes[p.si], T.reqs[p.ri]);
        seg += p.c_seg; node += p.c_node; tc += p.c_tc;
        p.c_seg = p.c_node = p.c_tc = 0;
      }
    }
    __syncthreads();
  }
  flush_counts(T.cnt, seg, node, tc, real, fail);
}

}  // namespace

#endif /* HTRDR_ENGINE_CUH */
