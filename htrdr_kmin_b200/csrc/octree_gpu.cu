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
#include <functional>
#include <memory>
#include <string>
#include <thread>

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

/* Leaf of every cell of one tree: a descent from the root by the cell's
 * coordinate bits, written as (node index in the tree) << 5 | level */
__global__ void
k_leafgrid(const uint4* __restrict__ nodes, uint32_t depth, uint32_t nx, uint32_t ny, uint32_t nz,
           uint32_t* grid)
{
  const uint64_t c = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if(c >= (uint64_t)nx * ny * nz) return;
  const uint32_t x = (uint32_t)(c % nx), y = (uint32_t)((c / nx) % ny), z = (uint32_t)(c / ((uint64_t)nx * ny));
  uint32_t n = 0, L = depth;
  uint32_t child = nodes[0].z;
  while(child != HG_LEAF && L > 0) {
    --L;
    n = child + (((x >> L) & 1u) | (((y >> L) & 1u) << 1) | (((z >> L) & 1u) << 2));
    child = nodes[n].z;
  }
  grid[c] = (n << 5) | L;
}

/* Majorants and level of the leaf of every cell of one tree (the same
 * descent): the trace reads a cell's kmin/kmax and voxel size with two
 * independent loads instead of the grid entry, then the node */
__global__ void
k_majgrid(const uint4* __restrict__ nodes, uint32_t depth, uint32_t nx, uint32_t ny, uint32_t nz,
          float2* maj, uint8_t* lvl)
{
  const uint64_t c = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if(c >= (uint64_t)nx * ny * nz) return;
  const uint32_t x = (uint32_t)(c % nx), y = (uint32_t)((c / nx) % ny), z = (uint32_t)(c / ((uint64_t)nx * ny));
  uint32_t n = 0, L = depth;
  uint32_t child = nodes[0].z;
  while(child != HG_LEAF && L > 0) {
    --L;
    n = child + (((x >> L) & 1u) | (((y >> L) & 1u) << 1) | (((z >> L) & 1u) << 2));
    child = nodes[n].z;
  }
  const uint4 v = nodes[n];
  maj[c] = make_float2(__uint_as_float(v.x), __uint_as_float(v.y));
  lvl[c] = (uint8_t)L;
}

}  // namespace

/* Leaf grids of the built trees (tree_count[i] > 0, in index order) into
 * `grids'; rank[i] is the grid of tree i.  Returns false (no grid built, no
 * error) when they would not fit in half of the free device memory or a tree
 * is too large for the 27-bit node index of an entry. */
bool
build_leaf_grids(const DScene& S, const std::vector<uint64_t>& tree_base,
                 const std::vector<uint64_t>& tree_count, DevBuf& grids, std::vector<uint32_t>& rank,
                 bool majorants)
{
  const uint64_t ncell = (uint64_t)S.def[0] * S.def[1] * S.def[2];
  rank.assign(tree_base.size(), 0);
  uint32_t ntrees = 0;
  for(size_t i = 0; i < tree_count.size(); ++i) {
    if(!tree_count[i]) continue;
    if(tree_count[i] >= (1ull << 27)) return false;
    rank[i] = ntrees++;
  }
  if(!ntrees || !ncell) return false;
  size_t free_b = 0, total_b = 0;
  if(cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) return false;
  const uint64_t bytes = (uint64_t)ntrees * ncell * (majorants ? 9 : 4);
  if(bytes > free_b / 2) return false;
  if(!grids.alloc(bytes)) return false;
  for(size_t i = 0; i < tree_count.size(); ++i) {
    if(!tree_count[i]) continue;
    const uint64_t off = (uint64_t)rank[i] * ncell;
    if(majorants) {
      float2* maj = (float2*)grids.ptr;
      uint8_t* lvl = (uint8_t*)(maj + (uint64_t)ntrees * ncell);
      k_majgrid<<<grid_of(ncell, 256), 256>>>(S.nodes + tree_base[i], S.depth, S.def[0], S.def[1],
                                               S.def[2], maj + off, lvl + off);
    } else {
      k_leafgrid<<<grid_of(ncell, 256), 256>>>(S.nodes + tree_base[i], S.depth, S.def[0], S.def[1],
                                                S.def[2], (uint32_t*)grids.ptr + off);
    }
  }
  return cuda_ok(cudaGetLastError(), "leaf grids") && cuda_ok(cudaDeviceSynchronize(), "leaf grids");
}

/* Scratch and stream of one build worker: the level arrays of one tree, the
 * depth lists of its emission and the scan's temporary storage */
struct Worker {
  cudaStream_t st = nullptr;
  DevBuf kmin, kmax, leaf, lists[2], flags, rank, cubtmp;
  size_t cub_bytes = 0;
  std::string error;
  ~Worker() { if(st) cudaStreamDestroy(st); }
};

#ifndef HG_BUILD_WORKERS
#define HG_BUILD_WORKERS 8
#endif

/* Builds the trees of `tasks' ((quad, property) pairs) on the device into one
 * pool; tree_base/tree_count are filled per task index.  The trees are
 * shared among up to 8 workers, each a host thread with its own stream and
 * scratch (as many as fit in a quarter of the free device memory, at most
 * 16 GB), so that the host round trips of one tree's emission overlap the
 * others' work.  The node arrays do not depend on the number of workers.
 * Returns false on a CUDA error (message in the last error). */
bool
build_octrees_gpu(const DScene& S, const float* d_lwc, const int2* d_cl, const float* d_gka,
                  const float* d_gks, const std::vector<float>& sig3, const std::vector<uint32_t>& band_of,
                  const std::vector<std::pair<uint32_t, int>>& tasks, uint32_t level_force, double tau,
                  double cmax, DevBuf& pool, std::vector<uint64_t>& base, std::vector<uint64_t>& count,
                  cudaStream_t st)
{
  const uint32_t D = S.depth, nl = S.nlayers;
  LevelDims dims{};
  uint64_t total_lv = 0;
  for(uint32_t L = 0; L <= D; ++L) {
    for(int a = 0; a < 3; ++a) dims.n[L][a] = (S.def[a] + (1u << L) - 1) >> L;
    dims.off[L] = total_lv;
    total_lv += (uint64_t)dims.n[L][0] * dims.n[L][1] * dims.n[L][2];
  }
  dims.off[D + 1] = total_lv;
  /* a depth list holds the 8 children of each internal node of the depth
   * above, whose level is >= 1: at most 8 x the size of level 1 */
  const uint64_t n1 = D >= 1 ? (uint64_t)dims.n[1][0] * dims.n[1][1] * dims.n[1][2] : 1;
  const uint64_t max_list = std::max<uint64_t>(8 * n1, 8);
  const uint64_t ncell = (uint64_t)S.def[0] * S.def[1] * S.def[2];
  size_t cub_bytes = 0;
  cub::DeviceScan::ExclusiveSum(nullptr, cub_bytes, (uint32_t*)nullptr, (uint32_t*)nullptr, (int)max_list, st);
  cub_bytes = std::max<size_t>(cub_bytes, 16);
  const size_t per_worker = total_lv * 9 + max_list * (2 * sizeof(Entry) + 8) + cub_bytes;

  int device = 0;
  if(!cuda_ok(cudaGetDevice(&device), "cudaGetDevice") || !cuda_ok(cudaStreamSynchronize(st), "sync"))
    return false;
  size_t free_b = 0, total_b = 0;
  if(!cuda_ok(cudaMemGetInfo(&free_b, &total_b), "cudaMemGetInfo")) return false;
  const size_t budget = std::min<size_t>(free_b / 4, (size_t)16 << 30);
  const size_t nw = std::max<size_t>(1, std::min<size_t>({(size_t)HG_BUILD_WORKERS, tasks.size(),
                                                           budget / std::max<size_t>(per_worker, 1)}));
  std::vector<std::unique_ptr<Worker>> workers;
  for(size_t w = 0; w < nw; ++w) {
    auto wk = std::make_unique<Worker>();
    wk->cub_bytes = cub_bytes;
    if(!cuda_ok(cudaStreamCreateWithFlags(&wk->st, cudaStreamNonBlocking), "stream")
    || !wk->kmin.alloc(total_lv * 4) || !wk->kmax.alloc(total_lv * 4) || !wk->leaf.alloc(total_lv)
    || !wk->lists[0].alloc(max_list * sizeof(Entry)) || !wk->lists[1].alloc(max_list * sizeof(Entry))
    || !wk->flags.alloc(max_list * 4) || !wk->rank.alloc(max_list * 4) || !wk->cubtmp.alloc(cub_bytes))
      return false;
    workers.push_back(std::move(wk));
  }
  DevBuf counts;
  if(!counts.alloc(std::max<size_t>(tasks.size(), 1) * 8)
  || !cuda_ok(cudaMemsetAsync(counts.ptr, 0, std::max<size_t>(tasks.size(), 1) * 8, st), "memset")
  || !cuda_ok(cudaStreamSynchronize(st), "sync"))
    return false;

  /* the levels of task t on worker w (counting: its internal nodes into counts[t]) */
  auto levels = [&](Worker& w, size_t t, bool counting) -> bool {
    const uint32_t q = tasks[t].first;
    const int p = tasks[t].second;
    const float sig = sig3[band_of[q] * 3 + p];
    k_level0<<<grid_of(ncell, 256), 256, 0, w.st>>>(d_lwc, S.def[0], S.def[1], S.def[2], d_cl,
      d_gka + (size_t)q * nl, d_gks + (size_t)q * nl, sig, p, (float*)w.kmin.ptr, (float*)w.kmax.ptr,
      (uint8_t*)w.leaf.ptr);
    for(uint32_t L = 1; L <= D; ++L) {
      const uint64_t np = (uint64_t)dims.n[L][0] * dims.n[L][1] * dims.n[L][2];
      k_level<<<grid_of(np, 256), 256, 0, w.st>>>(L, dims, (float*)w.kmin.ptr, (float*)w.kmax.ptr,
        (uint8_t*)w.leaf.ptr, level_force, (double)(1u << L) * cmax, tau,
        counting ? (unsigned long long*)counts.ptr + t : nullptr);
    }
    return cuda_ok(cudaGetLastError(), "octree levels");
  };

  /* the breadth-first emission of task t into the pool */
  auto emit = [&](Worker& w, size_t t) -> bool {
    uint4* nodes = (uint4*)pool.ptr + base[t];
    const Entry root{D, 0, 0, 0};
    if(!cuda_ok(cudaMemcpyAsync(w.lists[0].ptr, &root, sizeof(Entry), cudaMemcpyHostToDevice, w.st), "H2D"))
      return false;
    uint32_t cur = 0, n_d = 1, base_d = 0;
    while(n_d) {
      k_flags<<<grid_of(n_d, 256), 256, 0, w.st>>>((const Entry*)w.lists[cur].ptr, n_d, dims,
                                                    (const uint8_t*)w.leaf.ptr, (uint32_t*)w.flags.ptr);
      size_t tb = w.cub_bytes;
      if(cub::DeviceScan::ExclusiveSum(w.cubtmp.ptr, tb, (uint32_t*)w.flags.ptr, (uint32_t*)w.rank.ptr,
                                       (int)n_d, w.st) != cudaSuccess)
        return cuda_ok(cudaGetLastError(), "scan");
      uint32_t last[2] = {0, 0}; /* flag and rank of the last entry */
      if(!cuda_ok(cudaMemcpyAsync(&last[0], (uint32_t*)w.flags.ptr + n_d - 1, 4, cudaMemcpyDeviceToHost, w.st), "D2H")
      || !cuda_ok(cudaMemcpyAsync(&last[1], (uint32_t*)w.rank.ptr + n_d - 1, 4, cudaMemcpyDeviceToHost, w.st), "D2H"))
        return false;
      const uint32_t base_next = base_d + n_d;
      k_emit<<<grid_of(n_d, 256), 256, 0, w.st>>>((const Entry*)w.lists[cur].ptr, n_d, dims,
        (const float*)w.kmin.ptr, (const float*)w.kmax.ptr, (const uint32_t*)w.flags.ptr,
        (const uint32_t*)w.rank.ptr, base_d, base_next, nodes, (Entry*)w.lists[cur ^ 1].ptr);
      if(!cuda_ok(cudaStreamSynchronize(w.st), "sync")) return false;
      const uint64_t n_next = 8ull * ((uint64_t)last[1] + last[0]);
      if(n_next > max_list) { set_error("octree emission: depth list overflow"); return false; }
      base_d = base_next;
      n_d = (uint32_t)n_next;
      cur ^= 1;
    }
    if(base_d != count[t]) {
      set_error("octree emission: node count mismatch");
      return false;
    }
    return true;
  };

  /* run `job' on every task, task t on worker t % nw, one host thread per worker */
  auto run = [&](const std::function<bool(Worker&, size_t)>& job) -> bool {
    std::vector<std::thread> th;
    std::vector<int> ok(nw, 1);
    for(size_t w = 0; w < nw; ++w) {
      th.emplace_back([&, w]() {
        cudaSetDevice(device);
        for(size_t t = w; t < tasks.size() && ok[w]; t += nw)
          if(!job(*workers[w], t)) { ok[w] = 0; workers[w]->error = last_error(); }
        if(ok[w] && !cuda_ok(cudaStreamSynchronize(workers[w]->st), "sync")) {
          ok[w] = 0;
          workers[w]->error = last_error();
        }
      });
    }
    for(auto& x : th) x.join();
    for(size_t w = 0; w < nw; ++w)
      if(!ok[w]) { set_error(workers[w]->error); return false; }
    return true;
  };

  /* pass 1: node counts */
  if(!run([&](Worker& w, size_t t) { return levels(w, t, true); })) return false;
  std::vector<unsigned long long> ni(tasks.size(), 0);
  if(!tasks.empty()
  && !cuda_ok(cudaMemcpy(ni.data(), counts.ptr, tasks.size() * 8, cudaMemcpyDeviceToHost), "D2H"))
    return false;
  base.assign(tasks.size(), 0);
  count.assign(tasks.size(), 0);
  uint64_t total_nodes = 0;
  for(size_t t = 0; t < tasks.size(); ++t) {
    base[t] = total_nodes;
    count[t] = 1 + 8 * ni[t];
    total_nodes += count[t];
  }
  if(!pool.alloc(total_nodes * 16)) return false;

  /* pass 2: levels again, then emission */
  return run([&](Worker& w, size_t t) { return levels(w, t, false) && emit(w, t); });
}

}  // namespace hg
