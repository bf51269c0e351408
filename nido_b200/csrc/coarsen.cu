// coarsen.cu -- aggregation of the reference (GraphGPU::aggregation,
// graph_gpu.cpp:1382-1545) on the device.
//
// 1. Renumber: a used-flag per community id and an exclusive scan give each
//    community its rank among used ids, i.e. the reference's dense renumber
//    in ascending old-id order (sort_vertex_by_community_ids,
//    graph_gpu.cpp:1151-1222).  The clustering of the original vertices is
//    composed with it (Clustering::update_clustering, clustering.cpp:12-21).
// 2. Members: a stable radix sort of (new id, vertex) lists each coarse
//    vertex's members in ascending vertex order; a scan of member degrees
//    gives the concatenated member-adjacency positions
//    (shuffle_edge_list, graph_gpu.cpp:1088-1149).
// 3. Edges: per coarse vertex, neighbours are mapped to new ids and merged
//    with a hash; the output keeps the first-occurrence order of the
//    concatenated list (compress_edges, graph_gpu.cpp:1224-1304).
//    Coarse vertices with at most 256 member edges are handled by one warp
//    that walks the list in order and folds each weight onto its entry in
//    edge order, which is the reference's summation order.  Up to 4096 use a
//    CTA (256 threads up to 1024) with atomic first-position tracking and an
//    ordered second pass over the slots recorded in the first; larger ones
//    are cut into segments on many CTAs.  Weight sums beyond the warp tier are
//    exact for integer weights.
#include <limits.h>

#include <algorithm>

#include "common.cuh"
#include "engine.cuh"
#include "primitives.cuh"

namespace nido {
namespace {

// tiers by member-edge count D: groups of 4/8/16/32 lanes (D <= 4/8/16/32),
// warp, CTA-S, CTA-L, CTA-L without per-position slots (more than 4096
// positions but a table that fits: few coarse vertices, 2*min(D, nvp) <= 8192),
// giant
constexpr unsigned kAggTiers = 9;
constexpr int kAggWarpMaxD = 256;   // member edges handled by one warp
// CTA tiers: threads, shared-memory table slots and list positions (member
// edges) of one coarse vertex; a table holds at least twice the positions
constexpr int kAggSThreads = 256;
constexpr int kAggSCap = 2048;
constexpr int kAggSMaxD = 1024;
constexpr int kAggLThreads = 512;
constexpr int kAggLCap = 8192;
constexpr int kAggLMaxD = 4096;

struct AggArgs {
  const int64_t* __restrict__ off;
  const int32_t* __restrict__ adj;
  const double* __restrict__ w;
  const int32_t* __restrict__ newid;
  const uint32_t* __restrict__ member;  // vertices sorted by (new id, id)
  const int64_t* __restrict__ mo;       // member offsets per coarse vertex
  const int64_t* __restrict__ medge;    // concatenated-list position of each member
  int32_t* __restrict__ tadj;           // output, at the coarse vertex's list position
  double* __restrict__ tw;
  int64_t* __restrict__ degp;           // coarse degree
  int64_t nvp;                          // coarse vertex count
  unsigned long long* err;              // probe-limit failures (never expected)
  const int32_t* __restrict__ pm32;     // member holding position 32*b, for every b
};

// CTAs of a kernel resident on the whole GPU at once (at least one per SM)
template <typename K>
int agg_resident(K kernel, int threads, size_t smem) {
  int per_sm = 0, dev = 0, sms = kSMs;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, smem) != cudaSuccess ||
      cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) {
    cudaGetLastError();
    per_sm = 1;
  }
  return std::max(per_sm, 1) * sms;
}

inline unsigned grid_for(int64_t work, int per_block, int max_blocks) {
  int64_t b = (work + per_block - 1) / per_block;
  if (b < 1) b = 1;
  if (b > max_blocks) b = max_blocks;
  return (unsigned)b;
}

// A negative community drops the vertex from the coarse graph (the
// many-graph driver drops finished graphs this way; one-graph runs never do).
__global__ void k_mark_used(const int32_t* __restrict__ comm, int64_t nv, int32_t* __restrict__ used) {
  for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < nv; v += (int64_t)gridDim.x * blockDim.x) {
    const int32_t c = comm[v];
    if (c >= 0) used[c] = 1;
  }
}

__global__ void k_newid(const int32_t* __restrict__ comm, const int64_t* __restrict__ cid, int64_t nv,
                        int32_t* __restrict__ newid, uint32_t* __restrict__ keys, uint32_t* __restrict__ vals) {
  const uint32_t dropped = (uint32_t)cid[nv];  // nvp: dropped vertices sort after every member
  for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < nv; v += (int64_t)gridDim.x * blockDim.x) {
    const int32_t c = comm[v];
    const int32_t x = c >= 0 ? (int32_t)cid[c] : -1;
    newid[v] = x;
    keys[v] = c >= 0 ? (uint32_t)x : dropped;
    vals[v] = (uint32_t)v;
  }
}

// Communities never span graphs (no edge does), so the renumber keeps every
// graph's vertices contiguous and its new first vertex is cid[old first].
__global__ void k_graph_bases(const int64_t* __restrict__ gbase, int ng, const int64_t* __restrict__ cid,
                              int64_t* __restrict__ gbase2) {
  for (int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; g <= ng; g += (int64_t)gridDim.x * blockDim.x)
    gbase2[g] = cid[gbase[g]];
}

__global__ void k_compose(int32_t* __restrict__ clus, int64_t n0, const int32_t* __restrict__ newid) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n0; i += (int64_t)gridDim.x * blockDim.x) {
    const int32_t c = clus[i];
    if (c >= 0) clus[i] = newid[c];
  }
}

// member offsets from the sorted keys (every id in [0, nvp) occurs; dropped
// vertices carry key nvp and come last, with no member edges) and the member
// degrees
__global__ void k_member_bounds(const uint32_t* __restrict__ keys, const uint32_t* __restrict__ member,
                                int64_t nv, int64_t nvp, const int64_t* __restrict__ off,
                                int64_t* __restrict__ mo, int64_t* __restrict__ mdeg) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nv; i += (int64_t)gridDim.x * blockDim.x) {
    const uint32_t key = keys[i];
    if (i == 0 || key != keys[i - 1]) mo[key] = i;
    if (i == nv - 1 && key < (uint32_t)nvp) mo[nvp] = nv;
    const uint32_t v = member[i];
    mdeg[i] = key < (uint32_t)nvp ? off[v + 1] - off[v] : 0;
  }
}

// tier of each coarse vertex by its member-edge count D (counts aggregated
// per warp before the global atomics)
__global__ void k_agg_tiers(const int64_t* __restrict__ mo, const int64_t* __restrict__ medge, int64_t nvp,
                            uint32_t* __restrict__ keys, uint32_t* __restrict__ vals,
                            int64_t* __restrict__ counts) {
  const int lane = threadIdx.x & 31;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t base = blockIdx.x * (int64_t)blockDim.x; base < nvp; base += stride) {
    const int64_t c = base + threadIdx.x;
    uint32_t t = kAggTiers;
    if (c < nvp) {
      const int64_t D = medge[mo[c + 1]] - medge[mo[c]];
      const int64_t U = D < nvp ? D : nvp;
      t = D <= 4 ? 0u : D <= 8 ? 1u : D <= 16 ? 2u : D <= 32 ? 3u
        : D <= kAggWarpMaxD ? 4u : D <= kAggSMaxD ? 5u : D <= kAggLMaxD ? 6u : 2 * U <= kAggLCap ? 7u : 8u;
      keys[c] = t;
      vals[c] = (uint32_t)c;
    }
    const unsigned peers = __match_any_sync(NIDO_FULL_MASK, t);
    if (t < kAggTiers && lane == __ffs(peers) - 1)
      atomicAdd((unsigned long long*)&counts[t], (unsigned long long)__popc(peers));
  }
}

// member-edge count of the listed coarse vertices (for the segment plan)
__global__ void k_agg_sizes(const int32_t* __restrict__ list, int64_t n, const int64_t* __restrict__ mo,
                            const int64_t* __restrict__ medge, int64_t* __restrict__ out) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const int c = list[i];
    out[i] = medge[mo[c + 1]] - medge[mo[c]];
  }
}

__device__ __forceinline__ int64_t find_member(const int64_t* __restrict__ medge, int64_t lo, int64_t hi,
                                               int64_t P) {
  while (hi - lo > 1) {
    const int64_t mid = lo + (hi - lo) / 2;
    if (medge[mid] <= P) lo = mid; else hi = mid;
  }
  return lo;
}

// pm32[b] = the member whose positions include 32*b (positions run over the
// members' edge lists in member order; medge has nv+1 entries)
__global__ void k_member_blocks(const int64_t* __restrict__ medge, int64_t nv, int32_t* __restrict__ pm32) {
  const int64_t nb = (medge[nv] + 31) >> 5;
  for (int64_t b = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; b < nb; b += (int64_t)gridDim.x * blockDim.x)
    pm32[b] = (int32_t)find_member(medge, 0, nv, 32 * b);
}

// Slot of key X, inserting it if absent (*isnew reports the insert); at most
// mask+1 probes, -1 when the table is full (tables are sized to at least
// twice the number of keys, so this never happens).
__device__ __forceinline__ int find_or_insert(int* keys, unsigned mask, int X, bool* isnew) {
  unsigned h = hash_slot(X, mask);
  volatile int* vk = keys;
  *isnew = false;
  for (unsigned probe = 0; probe <= mask; ++probe) {
    const int kk = vk[h];
    if (kk == X) return (int)h;
    if (kk == -1) {
      const int old = atomicCAS(&keys[h], -1, X);
      if (old == -1) { *isnew = true; return (int)h; }
      if (old == X) return (int)h;
    }
    h = (h + 1) & mask;
  }
  return -1;
}

__device__ __forceinline__ int find_slot(const int* keys, unsigned mask, int X) {
  unsigned h = hash_slot(X, mask);
  for (unsigned probe = 0; probe <= mask; ++probe) {
    if (keys[h] == X) return (int)h;
    h = (h + 1) & mask;
  }
  return -1;
}

__device__ __forceinline__ unsigned cap_for(int64_t D, int64_t nvp) {
  const int64_t U = D < nvp ? D : nvp;
  unsigned c = 64;
  while ((int64_t)c < 2 * U) c <<= 1;
  return c;
}

// neighbour of list position P: new id and weight
// Member holding list position P: start from the member of P's 32-position
// block and step forward (a binary search over [m0, m1) only after 32 steps,
// i.e. across a run of members without edges).
__device__ __forceinline__ int64_t member_of(const AggArgs& q, int64_t m1, int64_t P) {
  int64_t i = q.pm32[P >> 5];
  for (int k = 0; k < 32 && q.medge[i + 1] <= P; ++k) ++i;
  if (q.medge[i + 1] <= P) i = find_member(q.medge, i, m1, P);
  return i;
}

__device__ __forceinline__ void load_pos(const AggArgs& q, int64_t m0, int64_t m1, int64_t P, int& X,
                                         double& wt) {
  (void)m0;
  const int64_t i = member_of(q, m1, P);
  const uint32_t v = q.member[i];
  const int64_t e = q.off[v] + (P - q.medge[i]);
  X = q.newid[q.adj[e]];
  wt = q.w[e];
}

// D <= G: a group of G lanes per coarse vertex, one list position per lane.
// Equal new ids are found with __match_any_sync (the group's index is part
// of the key), their weights folded in lane (= list) order onto the first
// lane, which is the reference's summation order, and the first lanes write
// their ids in lane order: no table.
template <int G>
__global__ void __launch_bounds__(256) k_agg_group(const int32_t* __restrict__ list, int64_t n, AggArgs q) {
  constexpr int VPW = 32 / G;
  const int lane = threadIdx.x & 31, gl = lane & (G - 1), gid = lane / G;
  const unsigned gmask = G == 32 ? NIDO_FULL_MASK : ((1u << G) - 1u) << (gid * G);
  const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t b = warp * VPW; b < n; b += nw * VPW) {
    const int64_t idx = b + gid;
    int cp = 0;
    int64_t m0 = 0, m1 = 0, P0 = 0, P1 = 0;
    if (idx < n) {
      cp = list[idx];
      m0 = q.mo[cp];
      m1 = q.mo[cp + 1];
      P0 = q.medge[m0];
      P1 = q.medge[m1];
    }
    const int64_t P = P0 + gl;
    const bool ok = idx < n && P < P1;
    int X = -1;
    double wt = 0.;
    if (ok) load_pos(q, m0, m1, P, X, wt);
    const unsigned long long key = (unsigned long long)(unsigned)gid << 32 | (unsigned)X;
    const unsigned peers = __match_any_sync(NIDO_FULL_MASK, key);
    const bool lead = ok && lane == __ffs(peers) - 1;
    double e = 0.;
    unsigned rem = ok ? peers : 0u;
    const int maxcnt = __reduce_max_sync(NIDO_FULL_MASK, (unsigned)__popc(rem));
    for (int it = 0; it < maxcnt; ++it) {
      const int src = rem ? __ffs(rem) - 1 : lane;
      const double x = __shfl_sync(NIDO_FULL_MASK, wt, src);
      if (rem) { e += x; rem &= rem - 1; }
    }
    const unsigned leaders = __ballot_sync(NIDO_FULL_MASK, lead) & gmask;
    if (lead) {
      const int o = __popc(leaders & lanemask_lt());
      q.tadj[P0 + o] = X;
      q.tw[P0 + o] = e;
    }
    if (gl == 0 && idx < n) q.degp[cp] = __popc(leaders);
  }
}

// Warp tier: one warp per coarse vertex, table in shared memory.
__global__ void __launch_bounds__(256) k_agg_warp(const int32_t* __restrict__ list, int64_t n, AggArgs q,
                                                  int capmax) {
  extern __shared__ double smem[];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  double* vals = smem + (size_t)wid * capmax;
  int* keys = reinterpret_cast<int*>(smem + (size_t)nwarps * capmax) + (size_t)wid * capmax * 2;
  int* idxs = keys + capmax;
  for (int i = lane; i < capmax; i += 32) { keys[i] = -1; vals[i] = 0.; }
  __syncwarp();
  const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t task = warp; task < n; task += nw) {
    const int cp = list[task];
    const int64_t m0 = q.mo[cp], m1 = q.mo[cp + 1];
    const int64_t P0 = q.medge[m0], P1 = q.medge[m1];
    const unsigned cap = min((unsigned)capmax, cap_for(P1 - P0, q.nvp)), mask = cap - 1;
    int running = 0;
    for (int64_t base = P0; base < P1; base += 32) {
      const int64_t P = base + lane;
      const bool ok = P < P1;
      int X = -1;
      double wt = 0.;
      if (ok) load_pos(q, m0, m1, P, X, wt);
      const unsigned peers = __match_any_sync(NIDO_FULL_MASK, X);
      const bool lead = ok && lane == __ffs(peers) - 1;
      int h = -1;
      bool isnew = false;
      if (lead) {
        h = find_or_insert(keys, mask, X, &isnew);
        if (h < 0) atomicAdd(q.err, 1ull);
      }
      const bool have = h >= 0;
      const unsigned newmask = __ballot_sync(NIDO_FULL_MASK, have && isnew);
      if (have && isnew) idxs[h] = running + __popc(newmask & lanemask_lt());
      running += __popc(newmask);
      // fold the peers' weights onto the entry in lane (= list) order
      double acc = have ? vals[h] : 0.;
      unsigned rem = ok ? peers : 0u;
      const int maxcnt = __reduce_max_sync(NIDO_FULL_MASK, (unsigned)__popc(rem));
      for (int it = 0; it < maxcnt; ++it) {
        const int src = rem ? __ffs(rem) - 1 : lane;
        const double x = __shfl_sync(NIDO_FULL_MASK, wt, src);
        if (rem) { acc += x; rem &= rem - 1; }
      }
      if (lead) vals[h] = acc;
      __syncwarp();
    }
    for (unsigned i = lane; i < cap; i += 32) {
      const int kk = keys[i];
      if (kk >= 0) {
        q.tadj[P0 + idxs[i]] = kk;
        q.tw[P0 + idxs[i]] = vals[i];
      }
    }
    if (lane == 0) q.degp[cp] = running;
    __syncwarp();
    for (unsigned i = lane; i < cap; i += 32) { keys[i] = -1; vals[i] = 0.; }
    __syncwarp();
  }
}

// CTA tiers: one CTA per coarse vertex of at most kMaxD list positions.
// Pass 1 merges with atomics, keeps the first list position of every new id
// and records the slot of every position in shared memory; pass 2 walks the
// positions in order from those slots (no second walk through members,
// offsets and the new-id gather) and emits each id at its first position.
// kMaxD == 0: any number of positions (the table still holds every id);
// pass 2 gathers each position's id again and looks its slot up.
template <int kThreads, int kCap, int kMaxD>
__global__ void __launch_bounds__(kThreads) k_agg_cta(const int32_t* __restrict__ list, int64_t n, AggArgs q) {
  extern __shared__ double smem[];
  __shared__ int wsum[2][kThreads / 32];
  double* vals = smem;
  int* keys = reinterpret_cast<int*>(smem + kCap);
  int* fpos = keys + kCap;
  int* hpos = fpos + kCap;
  for (int i = threadIdx.x; i < kCap; i += kThreads) { keys[i] = -1; vals[i] = 0.; fpos[i] = INT_MAX; }
  __syncthreads();
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  for (int64_t task = blockIdx.x; task < n; task += gridDim.x) {
    const int cp = list[task];
    const int64_t m0 = q.mo[cp], m1 = q.mo[cp + 1];
    const int64_t P0 = q.medge[m0], P1 = q.medge[m1];
    const unsigned cap = min(cap_for(P1 - P0, q.nvp), (unsigned)kCap), mask = cap - 1;
    for (int64_t base = P0 + (int64_t)wid * 32; base < P1; base += kThreads) {
      const int64_t P = base + lane;
      const bool ok = P < P1;
      int X = -1;
      double wt = 0.;
      if (ok) load_pos(q, m0, m1, P, X, wt);
      const unsigned peers = __match_any_sync(NIDO_FULL_MASK, X);
      const int leader = __ffs(peers) - 1;
      const bool lead = ok && lane == leader;
      double e = 0.;
      {
        unsigned rem = ok ? peers : 0u;
        const int maxcnt = __reduce_max_sync(NIDO_FULL_MASK, (unsigned)__popc(rem));
        for (int it = 0; it < maxcnt; ++it) {
          const int src = rem ? __ffs(rem) - 1 : lane;
          const double x = __shfl_sync(NIDO_FULL_MASK, wt, src);
          if (rem) { e += x; rem &= rem - 1; }
        }
      }
      int h = -1;
      if (lead) {
        bool isnew;
        h = find_or_insert(keys, mask, X, &isnew);
        if (h >= 0) {
          atomicAdd(&vals[h], e);
          atomicMin(&fpos[h], (int)(P - P0));
        } else {
          atomicAdd(q.err, 1ull);
        }
      }
      if (kMaxD > 0) {
        h = __shfl_sync(NIDO_FULL_MASK, h, leader);
        if (ok) hpos[P - P0] = h;
      }
    }
    // emit in list order: per kThreads positions one barrier, the warps'
    // counts double-buffered, every thread carrying the running total
    __syncthreads();
    int running = 0, par = 0;
    for (int64_t base = 0; base < P1 - P0; base += kThreads, par ^= 1) {
      const int i = (int)base + threadIdx.x;
      int h = -1;
      if (i < P1 - P0) {
        if (kMaxD > 0) {
          h = hpos[i];
        } else {
          int X;
          double wt;
          load_pos(q, m0, m1, P0 + i, X, wt);
          h = find_slot(keys, mask, X);
        }
      }
      const bool first = h >= 0 && fpos[h] == i;
      const unsigned bal = __ballot_sync(NIDO_FULL_MASK, first);
      if (lane == 0) wsum[par][wid] = __popc(bal);
      __syncthreads();
      int pre = running, tot = 0;
#pragma unroll
      for (int k = 0; k < kThreads / 32; ++k) {
        const int c = wsum[par][k];
        if (k < wid) pre += c;
        tot += c;
      }
      running += tot;
      if (first) {
        const int idx = pre + __popc(bal & lanemask_lt());
        q.tadj[P0 + idx] = keys[h];
        q.tw[P0 + idx] = vals[h];
      }
    }
    if (threadIdx.x == 0) q.degp[cp] = running;
    __syncthreads();  // every warp is done reading the table before it is cleared
    for (unsigned i = threadIdx.x; i < cap; i += kThreads) { keys[i] = -1; vals[i] = 0.; fpos[i] = INT_MAX; }
    __syncthreads();
  }
}

template <int kThreads, int kCap, int kMaxD>
constexpr size_t agg_cta_smem() {
  return (size_t)kCap * (sizeof(double) + 2 * sizeof(int)) + (size_t)kMaxD * sizeof(int);
}

// ---- giant coarse vertices: kAggSeg-position segments on many CTAs ----------
// Segment items (coarse vertex index in the list, segment) are processed in
// three passes over per-vertex tables in global memory: insert (atomic sums,
// first list position per id), count first occurrences per segment, and, after
// a scan of the counts, emit every id at its first-occurrence rank.
constexpr int kAggSeg = 4096;
// table slots of one wave of giant coarse vertices (4M slots of key, first
// position and value: 64 MB, L2 resident); one larger table is a wave alone
constexpr int64_t kAggWaveSlots = (int64_t)4 << 20;

struct SegArgs {
  const int2* __restrict__ items;
  const int32_t* __restrict__ cids;     // coarse vertex of each list entry
  const int64_t* __restrict__ toff;     // table offset of each list entry
  const int32_t* __restrict__ caps;     // table size of each list entry
  const int64_t* __restrict__ first;    // first item of each list entry
  int32_t* keys;
  double* vals;
  int32_t* fpos;
};

__device__ __forceinline__ void seg_range(const AggArgs& q, const SegArgs& a, int2 item, int& cp, int64_t& m0,
                                          int64_t& m1, int64_t& P0, int64_t& s0, int64_t& s1) {
  cp = a.cids[item.x];
  m0 = q.mo[cp];
  m1 = q.mo[cp + 1];
  P0 = q.medge[m0];
  const int64_t P1 = q.medge[m1];
  s0 = P0 + (int64_t)item.y * kAggSeg;
  s1 = min(P1, s0 + kAggSeg);
}

// items [it0, it0 + n) of the list (one wave)
__global__ void __launch_bounds__(256) k_agg_seg_insert(int64_t it0, int64_t n, AggArgs q, SegArgs a) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  for (int64_t it = it0 + blockIdx.x; it < it0 + n; it += gridDim.x) {
    const int2 item = a.items[it];
    int cp;
    int64_t m0, m1, P0, s0, s1;
    seg_range(q, a, item, cp, m0, m1, P0, s0, s1);
    int* keys = a.keys + a.toff[item.x];
    double* vals = a.vals + a.toff[item.x];
    int* fpos = a.fpos + a.toff[item.x];
    const unsigned mask = (unsigned)a.caps[item.x] - 1;
    for (int64_t base = s0 + (int64_t)wid * 32; base < s1; base += blockDim.x) {
      const int64_t P = base + lane;
      const bool ok = P < s1;
      int X = -1;
      double wt = 0.;
      if (ok) load_pos(q, m0, m1, P, X, wt);
      const unsigned peers = __match_any_sync(NIDO_FULL_MASK, X);
      const bool lead = ok && lane == __ffs(peers) - 1;
      double e = 0.;
      unsigned rem = ok ? peers : 0u;
      const int maxcnt = __reduce_max_sync(NIDO_FULL_MASK, (unsigned)__popc(rem));
      for (int k = 0; k < maxcnt; ++k) {
        const int src = rem ? __ffs(rem) - 1 : lane;
        const double x = __shfl_sync(NIDO_FULL_MASK, wt, src);
        if (rem) { e += x; rem &= rem - 1; }
      }
      if (lead) {
        bool isnew;
        const int h = find_or_insert(keys, mask, X, &isnew);
        if (h >= 0) {
          atomicAdd(&vals[h], e);
          atomicMin(&fpos[h], (int)(P - P0));
        } else {
          atomicAdd(q.err, 1ull);
        }
      }
    }
  }
}

// Giants of a wave hold the table slots [toff[i], toff[i] + caps[i]) of the
// wave's region, in giant order: the giant holding slot h.
__device__ __forceinline__ int64_t giant_of_slot(const int64_t* __restrict__ toff, int64_t g0, int64_t g1,
                                                 int64_t h) {
  int64_t lo = g0, hi = g1;
  while (hi - lo > 1) {
    const int64_t mid = lo + (hi - lo) / 2;
    if (toff[mid] <= h) lo = mid; else hi = mid;
  }
  return lo;
}

constexpr int kSegWords = kAggSeg / 32;  // bitmap words of one segment item

// After the inserts of a wave: every occupied slot sets the bit of its id's
// first list position in the bitmap of the segment item holding it.
__global__ void k_agg_mark(int64_t g0, int64_t g1, int64_t ws, int64_t i0, SegArgs a, uint32_t* __restrict__ bm) {
  for (int64_t h = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; h < ws; h += (int64_t)gridDim.x * blockDim.x) {
    if (a.keys[h] < 0) continue;
    const int64_t i = giant_of_slot(a.toff, g0, g1, h);
    const int f = a.fpos[h];
    const int64_t li = a.first[i] + f / kAggSeg - i0;
    const int b = f % kAggSeg;
    atomicOr(&bm[li * kSegWords + (b >> 5)], 1u << (b & 31));
  }
}

// Per segment item of a wave (one warp each): its count of first
// occurrences and the exclusive prefix count of every bitmap word.
__global__ void k_agg_seg_count(int64_t i0, int64_t n, const uint32_t* __restrict__ bm, int32_t* __restrict__ wpre,
                                int64_t* __restrict__ segcnt) {
  static_assert(kSegWords == 128, "four bitmap words per lane");
  const int lane = threadIdx.x & 31;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t li = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; li < n; li += nw) {
    const uint4 w4 = reinterpret_cast<const uint4*>(bm + li * kSegWords)[lane];
    const int c0 = __popc(w4.x), c1 = __popc(w4.y), c2 = __popc(w4.z), c3 = __popc(w4.w);
    const int tot = c0 + c1 + c2 + c3;
    int inc = tot;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(NIDO_FULL_MASK, inc, o);
      if (lane >= o) inc += y;
    }
    const int ex = inc - tot;
    reinterpret_cast<int4*>(wpre + li * kSegWords)[lane] = make_int4(ex, ex + c0, ex + c0 + c1, ex + c0 + c1 + c2);
    if (lane == 31) segcnt[i0 + li] = inc;
  }
}

// After the scan of the wave's counts: every occupied slot writes its id and
// summed weight at its rank among the first occurrences of its giant's list.
__global__ void k_agg_emit(int64_t g0, int64_t g1, int64_t ws, int64_t i0, AggArgs q, SegArgs a,
                           const uint32_t* __restrict__ bm, const int32_t* __restrict__ wpre,
                           const int64_t* __restrict__ segcnt) {
  for (int64_t h = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; h < ws; h += (int64_t)gridDim.x * blockDim.x) {
    const int key = a.keys[h];
    if (key < 0) continue;
    const int64_t i = giant_of_slot(a.toff, g0, g1, h);
    const int f = a.fpos[h];
    const int64_t it = a.first[i] + f / kAggSeg, li = it - i0;
    const int b = f % kAggSeg, w = b >> 5;
    const int64_t idx = (segcnt[it] - segcnt[a.first[i]]) + wpre[li * kSegWords + w] +
                        __popc(bm[li * kSegWords + w] & ((1u << (b & 31)) - 1u));
    const int64_t P0 = q.medge[q.mo[a.cids[i]]];
    q.tadj[P0 + idx] = key;
    q.tw[P0 + idx] = a.vals[h];
  }
}

// degree of each giant coarse vertex from the scanned segment counts
__global__ void k_agg_seg_deg(int64_t nlist, const int32_t* __restrict__ cids, const int64_t* __restrict__ first,
                              const int64_t* __restrict__ segoff, int64_t* __restrict__ degp) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nlist; i += (int64_t)gridDim.x * blockDim.x)
    degp[cids[i]] = segoff[first[i + 1]] - segoff[first[i]];
}

// Copy each coarse vertex's entries to its final offset.  A warp takes 32
// consecutive coarse vertices and copies their entries as one run: each
// lane finds its entry's vertex by a search over the lanes' prefix counts,
// four entries in flight per lane.  Vertices of more than kCompactBig
// entries are left out of the runs and listed for k_compact_big.
constexpr int kCompactBig = 4096;

__global__ void k_compact(int64_t nvp, const int64_t* __restrict__ mo, const int64_t* __restrict__ medge,
                          const int64_t* __restrict__ coff, const int32_t* __restrict__ tadj,
                          const double* __restrict__ tw, int32_t* __restrict__ adj, double* __restrict__ w,
                          int32_t* __restrict__ big, unsigned long long* __restrict__ nbig) {
  const int lane = threadIdx.x & 31;
  const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t c0 = warp * 32; c0 < nvp; c0 += nw * 32) {
    const int64_t c = c0 + lane;
    int64_t src = 0, dst = 0, len = 0;
    if (c < nvp) {
      dst = coff[c];
      len = coff[c + 1] - dst;
      src = medge[mo[c]];
      if (len > kCompactBig) {
        big[atomicAdd(nbig, 1ull)] = (int32_t)c;
        len = 0;
      }
    }
    int64_t inc = len;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int64_t y = __shfl_up_sync(NIDO_FULL_MASK, inc, o);
      if (lane >= o) inc += y;
    }
    const int64_t pre = inc - len;
    const int64_t T = __shfl_sync(NIDO_FULL_MASK, inc, 31);
    for (int64_t b = 0; b < T; b += 4 * 32) {
      int64_t sp[4], dp[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const int64_t i = b + u * 32 + lane;
        int k = 0;  // the last lane whose run starts at or before i
#pragma unroll
        for (int step = 16; step >= 1; step >>= 1) {
          const int64_t pk = __shfl_sync(NIDO_FULL_MASK, pre, k + step);
          if (pk <= i) k += step;
        }
        const int64_t pk = __shfl_sync(NIDO_FULL_MASK, pre, k);
        const int64_t sk = __shfl_sync(NIDO_FULL_MASK, src, k);
        const int64_t dk = __shfl_sync(NIDO_FULL_MASK, dst, k);
        sp[u] = i < T ? sk + (i - pk) : -1;
        dp[u] = dk + (i - pk);
      }
      int32_t a[4];
      double x[4];
#pragma unroll
      for (int u = 0; u < 4; ++u)
        if (sp[u] >= 0) { a[u] = tadj[sp[u]]; x[u] = tw[sp[u]]; }
#pragma unroll
      for (int u = 0; u < 4; ++u)
        if (sp[u] >= 0) { adj[dp[u]] = a[u]; w[dp[u]] = x[u]; }
    }
  }
}

// Entries of the listed large coarse vertices, one CTA per vertex, eight
// entries in flight per thread.
__global__ void __launch_bounds__(256) k_compact_big(const int32_t* __restrict__ big,
                                                     const unsigned long long* __restrict__ nbig,
                                                     const int64_t* __restrict__ mo,
                                                     const int64_t* __restrict__ medge,
                                                     const int64_t* __restrict__ coff,
                                                     const int32_t* __restrict__ tadj,
                                                     const double* __restrict__ tw, int32_t* __restrict__ adj,
                                                     double* __restrict__ w) {
  const int64_t n = (int64_t)*nbig;
  for (int64_t t = blockIdx.x; t < n; t += gridDim.x) {
    const int c = big[t];
    const int64_t dst = coff[c], len = coff[c + 1] - dst, src = medge[mo[c]];
    for (int64_t b = 0; b < len; b += 8 * 256) {
      int32_t a[8];
      double x[8];
#pragma unroll
      for (int u = 0; u < 8; ++u) {
        const int64_t i = b + u * 256 + threadIdx.x;
        if (i < len) { a[u] = tadj[src + i]; x[u] = tw[src + i]; }
      }
#pragma unroll
      for (int u = 0; u < 8; ++u) {
        const int64_t i = b + u * 256 + threadIdx.x;
        if (i < len) { adj[dst + i] = a[u]; w[dst + i] = x[u]; }
      }
    }
  }
}

}  // namespace

int launch_aggregation(nido_graph_s* g, int* done) {
  cudaStream_t s = g->ctx->stream;
  const int64_t nv = g->nv;
  *done = 1;
  if (nv == 0) return NIDO_OK;
  Arena ar(g->scratch, g->scratch_bytes);
  int32_t* used = ar.take<int32_t>(nv);
  int64_t* cid = ar.take<int64_t>(nv + 1);
  int32_t* newid = ar.take<int32_t>(nv);
  uint32_t* rk = ar.take<uint32_t>(nv);
  uint32_t* rv = ar.take<uint32_t>(nv);
  uint32_t* rk2 = ar.take<uint32_t>(nv);
  uint32_t* rv2 = ar.take<uint32_t>(nv);
  int64_t* mo = ar.take<int64_t>(nv + 1);
  int64_t* medge = ar.take<int64_t>(nv + 1);
  int64_t* degp = ar.take<int64_t>(nv + 1);
  int64_t* counts = ar.take<int64_t>(kAggTiers);
  int64_t* temp = ar.take<int64_t>(std::max(radix_temp_elems(nv), scan_temp_elems(nv + 1)));
  if (!temp) return nido_set_error(NIDO_E_NOMEM, "scratch arena too small (aggregation)");
  const unsigned gv = grid_for(nv, 256, kSMs * 16);
  NIDO_CUDA_TRY(cudaMemsetAsync(used, 0, sizeof(int32_t) * nv, s));
  k_mark_used<<<gv, 256, 0, s>>>(g->comm, nv, used);
  NIDO_LAUNCH_CHECK();
  NIDO_TRY(scan_exclusive_i32(used, cid, nv, temp, s));
  k_newid<<<gv, 256, 0, s>>>(g->comm, cid, nv, newid, rk, rv);
  NIDO_LAUNCH_CHECK();
  k_compose<<<grid_for(g->nv0, 256, kSMs * 16), 256, 0, s>>>(g->clus, g->nv0, newid);
  NIDO_LAUNCH_CHECK();
  if (g->gid) {  // many graphs: each graph's first coarse vertex
    k_graph_bases<<<grid_for(g->ngraphs + 1, 256, kSMs), 256, 0, s>>>(g->gbase, g->ngraphs, cid, g->gbase2);
    NIDO_LAUNCH_CHECK();
  }
  int64_t nvp = 0;
  NIDO_CUDA_TRY(cudaMemcpyAsync(&nvp, cid + nv, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
  NIDO_CUDA_TRY(cudaStreamSynchronize(s));
  if (nvp == nv || nvp == 1) return NIDO_OK;  // graph_gpu.cpp:1391-1392
  *done = 0;
  int bits = 0;
  while (((int64_t)1 << bits) < nvp + 1) ++bits;  // keys run to nvp (dropped vertices)
  NIDO_TRY(radix_sort_pairs(rk, rv, rk2, rv2, nv, bits, temp, s));
  k_member_bounds<<<gv, 256, 0, s>>>(rk, rv, nv, nvp, g->off, mo, medge);
  NIDO_LAUNCH_CHECK();
  NIDO_TRY(scan_exclusive_i64(medge, medge, nv, temp, s));
  {  // member of every 32-position block of the member-edge lists
    const int64_t nblk = (g->ne + 31) / 32 + 1;
    if (nblk > g->pm32_cap) {
      NIDO_CUDA_TRY(cudaStreamSynchronize(s));
      raw_free(g->ctx, g->pm32);
      g->pm32 = nullptr;
      g->pm32_cap = 0;
      NIDO_CUDA_TRY(raw_alloc(g->ctx, (void**)&g->pm32, sizeof(int32_t) * (size_t)nblk));
      g->pm32_cap = nblk;
    }
    k_member_blocks<<<grid_for(nblk, 256, kSMs * 16), 256, 0, s>>>(medge, nv, g->pm32);
    NIDO_LAUNCH_CHECK();
  }
  NIDO_CUDA_TRY(cudaMemsetAsync(counts, 0, sizeof(int64_t) * kAggTiers, s));
  // coarse-vertex tiers (rk2/rv2 are free after the member sort)
  uint32_t* tk = rk2;
  uint32_t* tv = rv2;
  uint32_t* tk2 = reinterpret_cast<uint32_t*>(used);
  uint32_t* tv2 = reinterpret_cast<uint32_t*>(degp);  // degp is written only after the tier sort
  k_agg_tiers<<<grid_for(nvp, 256, kSMs * 16), 256, 0, s>>>(mo, medge, nvp, tk, tv, counts);
  NIDO_LAUNCH_CHECK();
  NIDO_TRY(radix_sort_pairs(tk, tv, tk2, tv2, nvp, 4, temp, s));
  int64_t cnt[kAggTiers] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  NIDO_CUDA_TRY(cudaMemcpyAsync(cnt, counts, sizeof(cnt), cudaMemcpyDeviceToHost, s));
  NIDO_CUDA_TRY(cudaStreamSynchronize(s));
  int64_t at[kAggTiers + 1] = {0};  // first list entry of every tier
  for (unsigned t = 0; t < kAggTiers; ++t) at[t + 1] = at[t] + cnt[t];

  AggArgs q{g->off, g->adj, g->w, newid, rv, mo, medge, g->adj2, g->w2, degp, nvp,
            reinterpret_cast<unsigned long long*>(g->dcount + 1), g->pm32};
  const int32_t* list = reinterpret_cast<const int32_t*>(tv);
  // the tiers write disjoint coarse vertices: the lane-group and warp tiers
  // run on one side stream, the CTA tiers on the other, while the giant path
  // (which plans on the host) runs on the context's stream; all join before
  // the offsets are scanned
  nido_ctx_s* ctx = g->ctx;
  NIDO_CUDA_TRY(cudaEventRecord(ctx->fork_ev, s));
  for (int i = 0; i < 2; ++i) NIDO_CUDA_TRY(cudaStreamWaitEvent(ctx->aux[i], ctx->fork_ev, 0));
  if (cnt[0] > 0) k_agg_group<4><<<grid_for(cnt[0], 64, kSMs * 16), 256, 0, ctx->aux[0]>>>(list + at[0], cnt[0], q);
  if (cnt[1] > 0) k_agg_group<8><<<grid_for(cnt[1], 32, kSMs * 16), 256, 0, ctx->aux[0]>>>(list + at[1], cnt[1], q);
  if (cnt[2] > 0) k_agg_group<16><<<grid_for(cnt[2], 16, kSMs * 16), 256, 0, ctx->aux[0]>>>(list + at[2], cnt[2], q);
  if (cnt[3] > 0) k_agg_group<32><<<grid_for(cnt[3], 8, kSMs * 16), 256, 0, ctx->aux[0]>>>(list + at[3], cnt[3], q);
  NIDO_LAUNCH_CHECK();
  if (cnt[4] > 0) {
    const int capmax = 2 * kAggWarpMaxD;
    const size_t sm = (size_t)8 * capmax * (sizeof(double) + 2 * sizeof(int));
    NIDO_CUDA_TRY(cudaFuncSetAttribute(k_agg_warp, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    k_agg_warp<<<grid_for(cnt[4], 8, kSMs * 8), 256, sm, ctx->aux[0]>>>(list + at[4], cnt[4], q, capmax);
    NIDO_LAUNCH_CHECK();
  }
  if (cnt[5] > 0) {
    constexpr size_t sm = agg_cta_smem<kAggSThreads, kAggSCap, kAggSMaxD>();
    auto k = k_agg_cta<kAggSThreads, kAggSCap, kAggSMaxD>;
    NIDO_CUDA_TRY(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    k<<<grid_for(cnt[5], 1, agg_resident(k, kAggSThreads, sm)), kAggSThreads, sm, ctx->aux[1]>>>(list + at[5],
                                                                                             cnt[5], q);
    NIDO_LAUNCH_CHECK();
  }
  if (cnt[6] > 0) {
    constexpr size_t sm = agg_cta_smem<kAggLThreads, kAggLCap, kAggLMaxD>();
    auto k = k_agg_cta<kAggLThreads, kAggLCap, kAggLMaxD>;
    NIDO_CUDA_TRY(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    k<<<grid_for(cnt[6], 1, agg_resident(k, kAggLThreads, sm)), kAggLThreads, sm, ctx->aux[1]>>>(list + at[6],
                                                                                             cnt[6], q);
    NIDO_LAUNCH_CHECK();
  }
  if (cnt[7] > 0) {
    constexpr size_t sm = agg_cta_smem<kAggLThreads, kAggLCap, 0>();
    auto k = k_agg_cta<kAggLThreads, kAggLCap, 0>;
    NIDO_CUDA_TRY(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    k<<<grid_for(cnt[7], 1, agg_resident(k, kAggLThreads, sm)), kAggLThreads, sm, ctx->aux[1]>>>(list + at[7],
                                                                                             cnt[7], q);
    NIDO_LAUNCH_CHECK();
  }
  if (cnt[8] > 0) {
    // plan: per giant coarse vertex a table of >= 2*min(D, nvp) slots and
    // ceil(D / kAggSeg) segment items; giants go in waves whose tables share
    // one region of at most kAggWaveSlots slots (or one larger table)
    const int64_t n2 = cnt[8];
    const int32_t* list2 = list + at[8];
    int64_t* dsz = ar.take<int64_t>(n2);
    if (!dsz) return nido_set_error(NIDO_E_NOMEM, "scratch arena too small (aggregation plan)");
    k_agg_sizes<<<grid_for(n2, 256, kSMs * 4), 256, 0, s>>>(list2, n2, mo, medge, dsz);
    NIDO_LAUNCH_CHECK();
    std::vector<int64_t> D(n2);
    std::vector<int32_t> cids(n2), caps(n2);
    NIDO_CUDA_TRY(cudaMemcpyAsync(D.data(), dsz, sizeof(int64_t) * n2, cudaMemcpyDeviceToHost, s));
    NIDO_CUDA_TRY(cudaMemcpyAsync(cids.data(), list2, sizeof(int32_t) * n2, cudaMemcpyDeviceToHost, s));
    NIDO_CUDA_TRY(cudaStreamSynchronize(s));
    std::vector<int64_t> toff(n2), first(n2 + 1);
    std::vector<int64_t> wave_g{0};  // first giant of every wave, then n2
    std::vector<int2> items;
    int64_t slots = 0, wslots = 0;
    for (int64_t i = 0; i < n2; ++i) {
      const int64_t u = std::min<int64_t>(D[i], nvp);
      int64_t cap = 64;
      while (cap < 2 * u) cap <<= 1;
      caps[i] = (int32_t)cap;
      if (i > 0 && wslots + cap > kAggWaveSlots) {
        wave_g.push_back(i);
        wslots = 0;
      }
      toff[i] = wslots;
      wslots += cap;
      slots = std::max(slots, wslots);
      first[i] = (int64_t)items.size();
      for (int64_t sg = 0; sg * kAggSeg < D[i]; ++sg) items.push_back(make_int2((int)i, (int)sg));
    }
    wave_g.push_back(n2);
    first[n2] = (int64_t)items.size();
    const int64_t ni = (int64_t)items.size();
    int64_t wave_items = 0;  // most segment items in one wave
    for (size_t wv = 0; wv + 1 < wave_g.size(); ++wv)
      wave_items = std::max(wave_items, first[wave_g[wv + 1]] - first[wave_g[wv]]);
    const size_t bytes = sizeof(int2) * ni + sizeof(int32_t) * 2 * n2 + sizeof(int64_t) * (2 * n2 + 1) +
                         sizeof(int64_t) * (ni + 1) + sizeof(int64_t) * scan_temp_elems(ni) +
                         (sizeof(int32_t) * 2 + sizeof(double)) * slots +
                         2 * sizeof(uint32_t) * kSegWords * wave_items + 16 * 256;
    if (bytes > g->agg_buf_bytes) {
      NIDO_CUDA_TRY(cudaStreamSynchronize(s));
      raw_free(g->ctx, g->agg_buf);
      g->agg_buf = nullptr;
      g->agg_buf_bytes = 0;
      const size_t want = bytes + bytes / 4;
      NIDO_CUDA_TRY(raw_alloc(g->ctx, (void**)&g->agg_buf, want));
      g->agg_buf_bytes = want;
    }
    Arena pa(g->agg_buf, g->agg_buf_bytes);
    int2* ditems = pa.take<int2>(ni);
    int32_t* dcids = pa.take<int32_t>(n2);
    int32_t* dcaps = pa.take<int32_t>(n2);
    int64_t* dtoff = pa.take<int64_t>(n2);
    int64_t* dfirst = pa.take<int64_t>(n2 + 1);
    int64_t* segcnt = pa.take<int64_t>(ni + 1);
    int64_t* stemp = pa.take<int64_t>(scan_temp_elems(ni));
    int32_t* tkeys = pa.take<int32_t>(slots);
    int32_t* tfpos = pa.take<int32_t>(slots);
    double* tvals = pa.take<double>(slots);
    uint32_t* bm = pa.take<uint32_t>(kSegWords * wave_items);
    int32_t* wpre = pa.take<int32_t>(kSegWords * wave_items);
    NIDO_CUDA_TRY(cudaMemcpyAsync(ditems, items.data(), sizeof(int2) * ni, cudaMemcpyHostToDevice, s));
    NIDO_CUDA_TRY(cudaMemcpyAsync(dcids, cids.data(), sizeof(int32_t) * n2, cudaMemcpyHostToDevice, s));
    NIDO_CUDA_TRY(cudaMemcpyAsync(dcaps, caps.data(), sizeof(int32_t) * n2, cudaMemcpyHostToDevice, s));
    NIDO_CUDA_TRY(cudaMemcpyAsync(dtoff, toff.data(), sizeof(int64_t) * n2, cudaMemcpyHostToDevice, s));
    NIDO_CUDA_TRY(cudaMemcpyAsync(dfirst, first.data(), sizeof(int64_t) * (n2 + 1), cudaMemcpyHostToDevice, s));
    SegArgs sa{ditems, dcids, dtoff, dcaps, dfirst, tkeys, tvals, tfpos};
    for (size_t wv = 0; wv + 1 < wave_g.size(); ++wv) {
      const int64_t g0 = wave_g[wv], g1 = wave_g[wv + 1];
      const int64_t i0 = first[g0], nw = first[g1] - i0;
      const int64_t ws = toff[g1 - 1] + caps[g1 - 1];
      NIDO_CUDA_TRY(cudaMemsetAsync(tkeys, 0xff, sizeof(int32_t) * ws, s));
      NIDO_CUDA_TRY(cudaMemsetAsync(tfpos, 0x7f, sizeof(int32_t) * ws, s));
      NIDO_CUDA_TRY(cudaMemsetAsync(tvals, 0, sizeof(double) * ws, s));
      NIDO_CUDA_TRY(cudaMemsetAsync(bm, 0, sizeof(uint32_t) * kSegWords * nw, s));
      const unsigned gi = grid_for(nw, 1, kSMs * 8);
      k_agg_seg_insert<<<gi, 256, 0, s>>>(i0, nw, q, sa);
      NIDO_LAUNCH_CHECK();
      const unsigned gs = grid_for(ws, 256, kSMs * 8);
      k_agg_mark<<<gs, 256, 0, s>>>(g0, g1, ws, i0, sa, bm);
      NIDO_LAUNCH_CHECK();
      k_agg_seg_count<<<grid_for(nw * 32, 256, kSMs * 8), 256, 0, s>>>(i0, nw, bm, wpre, segcnt);
      NIDO_LAUNCH_CHECK();
      // within the wave: each giant's output offsets need only differences
      // of this scan (segcnt[i0 + nw] is overwritten by the next wave)
      NIDO_TRY(scan_exclusive_i64(segcnt + i0, segcnt + i0, nw, stemp, s));
      k_agg_emit<<<gs, 256, 0, s>>>(g0, g1, ws, i0, q, sa, bm, wpre, segcnt);
      NIDO_LAUNCH_CHECK();
      k_agg_seg_deg<<<grid_for(g1 - g0, 256, kSMs * 4), 256, 0, s>>>(g1 - g0, dcids + g0, dfirst + g0, segcnt, degp);
      NIDO_LAUNCH_CHECK();
    }
    NIDO_CUDA_TRY(cudaStreamSynchronize(s));  // the host plan vectors go out of scope
  }
  for (int i = 0; i < 2; ++i) {
    NIDO_CUDA_TRY(cudaEventRecord(ctx->join_ev[i], ctx->aux[i]));
    NIDO_CUDA_TRY(cudaStreamWaitEvent(s, ctx->join_ev[i], 0));
  }
  // coarse offsets into off2, then the entries into the work CSR (when the
  // current graph is the work CSR, its lists are dead once pass 1 is done)
  NIDO_TRY(scan_exclusive_i64(degp, g->off2, nvp, temp, s));
  {
    // large coarse vertices are listed in the member-key buffer (free once
    // the member bounds are known), their count in the tier counters (read)
    int32_t* big = reinterpret_cast<int32_t*>(rk);
    unsigned long long* nbig = reinterpret_cast<unsigned long long*>(counts);
    NIDO_CUDA_TRY(cudaMemsetAsync(nbig, 0, sizeof(unsigned long long), s));
    k_compact<<<grid_for(nvp, 256, kSMs * 16), 256, 0, s>>>(nvp, mo, medge, g->off2, g->adj2, g->w2, g->adjA,
                                                             g->wA, big, nbig);
    NIDO_LAUNCH_CHECK();
    k_compact_big<<<kSMs * 2, 256, 0, s>>>(big, nbig, mo, medge, g->off2, g->adj2, g->w2, g->adjA, g->wA);
    NIDO_LAUNCH_CHECK();
  }
  int64_t nep = 0, nerr = 0;
  NIDO_CUDA_TRY(cudaMemcpyAsync(&nep, g->off2 + nvp, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
  NIDO_CUDA_TRY(cudaMemcpyAsync(&nerr, g->dcount + 1, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
  NIDO_CUDA_TRY(cudaStreamSynchronize(s));
  if (nerr) return nido_set_error(NIDO_E_CUDA, "hash table overflow in %lld probes", (long long)nerr);
  std::swap(g->offA, g->off2);
  g->off = g->offA;
  g->adj = g->adjA;
  g->w = g->wA;
  g->coarsened = true;
  g->nv = nvp;
  g->ne = nep;
  g->bins_valid = false;
  return NIDO_OK;
}

}  // namespace nido
