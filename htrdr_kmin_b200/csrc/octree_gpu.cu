/* Majorant octrees built on the GPU (the htsky_create acceleration structure,
 * src/atmosphere/htrdr_atmosphere.c:366-382), node arrays byte-identical to
 * the host definition in scene.cpp:
 *
 *  - level 0: one thread per cloud cell, k_cloud = fl(lwc * sigma) plus the
 *    [min, max] of k_gas over the layers the cell overlaps (single precision,
 *    no contraction);
 *  - level L: one thread per node, min/max over its valid children and the
 *    leaf test all-children-leaves && (L <= L_force || (kmax - kmin) 2^L
 *    cmax <= tau) in FP64;
 *  - breadth-first emission, one depth at a time: the internal nodes of a
 *    depth are ranked by an exclusive scan, the node of rank r gets its 8
 *    children at base(depth + 1) + 8 r in octant order -- the same order as
 *    a queue-driven breadth-first walk.
 * A first pass counts each tree's nodes (so the node pool is allocated once,
 * exactly); a second pass recomputes the levels and emits the nodes. */
#include "internal.h"

#include <cub/cub.cuh>

#include <algorithm>
#include <cfloat>

namespace hg {

namespace {

struct LevelDims {
  uint32_t n[32][3];
  uint64_t off[33]; /* offset of level L in the concatenated level arrays */
};

__global__ void
k_level0(const float* __restrict__ lwc, uint32_t nx, uint32_t ny, uint32_t nz,
         const int2* __restrict__ cl, const float* __restrict__ gka, const float* __restrict__ gks,
         float sig, int prop, float* kmin, float* kmax, uint8_t* leaf)
{
  const uint64_t c = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const uint64_t ncell = (uint64_t)nx * ny * nz;
  if(c >= ncell) return;
  const uint32_t k = (uint32_t)(c / ((uint64_t)nx * ny));
  const int2 lr = cl[k];
  float gmin = 0.f, gmax = 0.f;
  if(lr.x >= 0) {
    for(int l = lr.x; l <= lr.y; ++l) {
      const float a = gka[l], s = gks[l];
      const float g = prop == HG_KA ? a : (prop == HG_KS ? s : __fadd_rn(a, s));
      if(l == lr.x) { gmin = gmax = g; continue; }
      if(g < gmin) gmin = g;
      if(g > gmax) gmax = g;
    }
  }
  const float kc = __fmul_rn(lwc[c], sig);
  kmin[c] = __fadd_rn(kc, gmin);
  kmax[c] = __fadd_rn(kc, gmax);
  leaf[c] = 1;
}

__global__ void
k_level(uint32_t L, LevelDims dims, float* kmin, float* kmax, uint8_t* leaf, uint32_t level_force,
        double size, double tau, unsigned long long* n_internal)
{
  const uint32_t* pn = dims.n[L];
  const uint32_t* cn = dims.n[L - 1];
  const uint64_t idx = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const uint64_t np = (uint64_t)pn[0] * pn[1] * pn[2];
  bool internal = false;
  if(idx < np) {
    const uint32_t i = (uint32_t)(idx % pn[0]);
    const uint32_t j = (uint32_t)((idx / pn[0]) % pn[1]);
    const uint32_t k = (uint32_t)(idx / ((uint64_t)pn[0] * pn[1]));
    const float* cmin = kmin + dims.off[L - 1];
    const float* cmax = kmax + dims.off[L - 1];
    const uint8_t* cleaf = leaf + dims.off[L - 1];
    float mn = FLT_MAX, mx = -FLT_MAX;
    int all_leaf = 1;
    for(int oct = 0; oct < 8; ++oct) {
      const uint32_t ci = 2 * i + (oct & 1), cj = 2 * j + ((oct >> 1) & 1), ck = 2 * k + (oct >> 2);
      if(ci >= cn[0] || cj >= cn[1] || ck >= cn[2]) continue;
      const uint64_t cc = ((uint64_t)ck * cn[1] + cj) * cn[0] + ci;
      if(cmin[cc] < mn) mn = cmin[cc];
      if(cmax[cc] > mx) mx = cmax[cc];
      all_leaf &= cleaf[cc];
    }
    const bool lf = all_leaf
      && (L <= level_force || __dmul_rn(__dsub_rn((double)mx, (double)mn), size) <= tau);
    kmin[dims.off[L] + idx] = mn;
    kmax[dims.off[L] + idx] = mx;
    leaf[dims.off[L] + idx] = lf ? 1 : 0;
    internal = !lf;
  }
  if(n_internal) {
    const unsigned m = __ballot_sync(0xffffffffu, internal);
    if((threadIdx.x & 31) == 0 && m) atomicAdd(n_internal, (unsigned long long)__popc(m));
  }
}

/* Entry of a depth list: level (0xFFFFFFFF = empty) and cell-space coordinates */
struct Entry { uint32_t L, i, j, k; };

__global__ void
k_flags(const Entry* __restrict__ list, uint32_t count, LevelDims dims, const uint8_t* __restrict__ leaf,
        uint32_t* flags)
{
  const uint32_t e = blockIdx.x * blockDim.x + threadIdx.x;
  if(e >= count) return;
  const Entry en = list[e];
  uint32_t f = 0;
  if(en.L != 0xFFFFFFFFu) {
    const uint32_t* n = dims.n[en.L];
    f = leaf[dims.off[en.L] + ((uint64_t)en.k * n[1] + en.j) * n[0] + en.i] ? 0u : 1u;
  }
  flags[e] = f;
}

__global__ void
k_emit(const Entry* __restrict__ list, uint32_t count, LevelDims dims, const float* __restrict__ kmin,
       const float* __restrict__ kmax, const uint32_t* __restrict__ flags,
       const uint32_t* __restrict__ rank, uint32_t base_d, uint32_t base_next, uint4* nodes,
       Entry* next)
{
  const uint32_t e = blockIdx.x * blockDim.x + threadIdx.x;
  if(e >= count) return;
  const Entry en = list[e];
  uint4 nd = make_uint4(0u, 0u, HG_LEAF, 0u);
  if(en.L != 0xFFFFFFFFu) {
    const uint32_t* n = dims.n[en.L];
    const uint64_t c = dims.off[en.L] + ((uint64_t)en.k * n[1] + en.j) * n[0] + en.i;
    nd.x = __float_as_uint(kmin[c]);
    nd.y = __float_as_uint(kmax[c]);
    if(flags[e]) {
      const uint32_t r = rank[e];
      nd.z = base_next + 8 * r;
      const uint32_t* cn = dims.n[en.L - 1];
      for(int oct = 0; oct < 8; ++oct) {
        const uint32_t ci = 2 * en.i + (oct & 1), cj = 2 * en.j + ((oct >> 1) & 1), ck = 2 * en.k + (oct >> 2);
        Entry ch;
        if(ci >= cn[0] || cj >= cn[1] || ck >= cn[2]) ch = Entry{0xFFFFFFFFu, 0, 0, 0};
        else ch = Entry{en.L - 1, ci, cj, ck};
        next[8 * (uint64_t)r + oct] = ch;
      }
    }
  }
  nodes[base_d + e] = nd;
}

inline unsigned
grid_of(uint64_t n, unsigned bs) { return (unsigned)((n + bs - 1) / bs); }

}  // namespace

/* Builds the trees of `tasks' ((quad, property) pairs) on the device into one
 * pool; tree_base/tree_count are filled per task index.  Returns false on a
 * CUDA error (message in the last error). */
bool
build_octrees_gpu(const DScene& S, const float* d_lwc, const int2* d_cl, const float* d_gka,
                  const float* d_gks, const std::vector<float>& sig3, const std::vector<uint32_t>& band_of,
                  const std::vector<std::pair<uint32_t, int>>& tasks, uint32_t level_force, double tau,
                  double cmax, DevBuf& pool, std::vector<uint64_t>& base, std::vector<uint64_t>& count,
                  cudaStream_t st)
{
  const uint32_t D = S.depth, nl = S.nlayers;
  LevelDims dims{};
  uint64_t total_lv = 0, max_lv = 0;
  for(uint32_t L = 0; L <= D; ++L) {
    for(int a = 0; a < 3; ++a) dims.n[L][a] = (S.def[a] + (1u << L) - 1) >> L;
    dims.off[L] = total_lv;
    const uint64_t nn = (uint64_t)dims.n[L][0] * dims.n[L][1] * dims.n[L][2];
    total_lv += nn;
    max_lv = std::max(max_lv, nn);
  }
  dims.off[D + 1] = total_lv;
  DevBuf kmin, kmax, leaf, cnt, lists[2], flags, rank, cubtmp;
  const uint64_t max_list = std::max<uint64_t>(8 * max_lv, 8);
  size_t cub_bytes = 0;
  cub::DeviceScan::ExclusiveSum(nullptr, cub_bytes, (uint32_t*)nullptr, (uint32_t*)nullptr, (int)max_list, st);
  if(!kmin.alloc(total_lv * 4) || !kmax.alloc(total_lv * 4) || !leaf.alloc(total_lv) || !cnt.alloc(8)
  || !lists[0].alloc(max_list * sizeof(Entry)) || !lists[1].alloc(max_list * sizeof(Entry))
  || !flags.alloc(max_list * 4) || !rank.alloc(max_list * 4) || !cubtmp.alloc(std::max<size_t>(cub_bytes, 16)))
    return false;
  const uint64_t ncell = (uint64_t)S.def[0] * S.def[1] * S.def[2];

  auto levels = [&](uint32_t q, int p, bool counting) -> bool {
    const float sig = sig3[band_of[q] * 3 + p];
    k_level0<<<grid_of(ncell, 256), 256, 0, st>>>(d_lwc, S.def[0], S.def[1], S.def[2], d_cl,
      d_gka + (size_t)q * nl, d_gks + (size_t)q * nl, sig, p, (float*)kmin.ptr, (float*)kmax.ptr,
      (uint8_t*)leaf.ptr);
    if(counting && cudaMemsetAsync(cnt.ptr, 0, 8, st) != cudaSuccess) return false;
    for(uint32_t L = 1; L <= D; ++L) {
      const uint64_t np = (uint64_t)dims.n[L][0] * dims.n[L][1] * dims.n[L][2];
      k_level<<<grid_of(np, 256), 256, 0, st>>>(L, dims, (float*)kmin.ptr, (float*)kmax.ptr,
        (uint8_t*)leaf.ptr, level_force, (double)(1u << L) * cmax, tau,
        counting ? (unsigned long long*)cnt.ptr : nullptr);
    }
    return cuda_ok(cudaGetLastError(), "octree levels");
  };

  /* pass 1: node counts */
  base.assign(tasks.size(), 0);
  count.assign(tasks.size(), 0);
  uint64_t total_nodes = 0;
  for(size_t t = 0; t < tasks.size(); ++t) {
    if(!levels(tasks[t].first, tasks[t].second, true)) return false;
    unsigned long long ni = 0;
    if(!cuda_ok(cudaMemcpyAsync(&ni, cnt.ptr, 8, cudaMemcpyDeviceToHost, st), "D2H")
    || !cuda_ok(cudaStreamSynchronize(st), "sync"))
      return false;
    base[t] = total_nodes;
    count[t] = 1 + 8 * ni;
    total_nodes += count[t];
  }
  if(!pool.alloc(total_nodes * 16)) return false;

  /* pass 2: emission */
  for(size_t t = 0; t < tasks.size(); ++t) {
    if(!levels(tasks[t].first, tasks[t].second, false)) return false;
    uint4* nodes = (uint4*)pool.ptr + base[t];
    const Entry root{D, 0, 0, 0};
    if(!cuda_ok(cudaMemcpyAsync(lists[0].ptr, &root, sizeof(Entry), cudaMemcpyHostToDevice, st), "H2D"))
      return false;
    uint32_t cur = 0, n_d = 1, base_d = 0;
    while(n_d) {
      k_flags<<<grid_of(n_d, 256), 256, 0, st>>>((const Entry*)lists[cur].ptr, n_d, dims,
                                                  (const uint8_t*)leaf.ptr, (uint32_t*)flags.ptr);
      size_t tb = cub_bytes;
      if(cub::DeviceScan::ExclusiveSum(cubtmp.ptr, tb, (uint32_t*)flags.ptr, (uint32_t*)rank.ptr,
                                       (int)n_d, st) != cudaSuccess)
        return cuda_ok(cudaGetLastError(), "scan");
      uint32_t last_flag = 0, last_rank = 0;
      if(!cuda_ok(cudaMemcpyAsync(&last_flag, (uint32_t*)flags.ptr + n_d - 1, 4, cudaMemcpyDeviceToHost, st), "D2H")
      || !cuda_ok(cudaMemcpyAsync(&last_rank, (uint32_t*)rank.ptr + n_d - 1, 4, cudaMemcpyDeviceToHost, st), "D2H"))
        return false;
      const uint32_t base_next = base_d + n_d;
      k_emit<<<grid_of(n_d, 256), 256, 0, st>>>((const Entry*)lists[cur].ptr, n_d, dims,
        (const float*)kmin.ptr, (const float*)kmax.ptr, (const uint32_t*)flags.ptr,
        (const uint32_t*)rank.ptr, base_d, base_next, nodes, (Entry*)lists[cur ^ 1].ptr);
      if(!cuda_ok(cudaStreamSynchronize(st), "sync")) return false;
      const uint32_t n_internal = last_rank + last_flag;
      base_d = base_next;
      n_d = 8 * n_internal;
      cur ^= 1;
    }
    if(base_d != count[t]) {
      set_error("octree emission: node count mismatch");
      return false;
    }
  }
  return true;
}

}  // namespace hg
