/* Device pieces shared by the work-queue engines (persistent megakernel and
 * wavefront): item lookup in the realisation index space and the FP64
 * accumulation of a finished realisation into its request's accumulators. */
#ifndef HTRDR_ENGINE_CUH
#define HTRDR_ENGINE_CUH

#include "internal.h"
#include "transport.cuh"

#include <cooperative_groups.h>
#include <cooperative_groups/reduce.h>

/* Order of a request's realisations in the work queue: pixel-major (the
 * realisations of a pixel are consecutive, so the lanes that take them
 * together sample the same sensor region and often finish together) or
 * realisation-major. */
#ifndef HG_PIXEL_MAJOR
#define HG_PIXEL_MAJOR 1
#endif
/* Lanes that finish realisations of the same pixel together add their
 * weights with one set of atomics (cooperative-groups partition by pixel) */
#ifndef HG_AGGREGATE
#define HG_AGGREGATE 1
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

/* Copy the scene and request tables of a launch into shared memory (one
 * copy per block) and point T at them */
/* A path held in shared memory.  8 bytes of padding give an odd number of
 * 8-byte words per slot, so a warp's 8-byte accesses to one field of 32
 * slots are free of bank conflicts. */
struct __align__(8) PathSlot {
  Path p;
  uint32_t pad[2];
};
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

}  // namespace

#endif /* HTRDR_ENGINE_CUH */
