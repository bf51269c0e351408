// phase.cu -- per-phase and per-iteration kernels around the move phase:
// vertex weights k_v, mass m, singleton start, community-degree commit and
// restore (FP64 atomics), modularity, and the -b batch cuts with the degree
// tier lists.
//
// k_v, m and Q are reduced in exactly the order of the reference kernels
// (cited below), so they are bit-identical to the reference given the same
// inputs; the per-vertex in-community sums inside Q use a fixed order of this
// engine, which equals the reference's wherever the sums are exact (integer
// weights).
#include <string.h>

#include <algorithm>

#include "common.cuh"
#include "cuts.cuh"
#include "engine.cuh"
#include "primitives.cuh"

namespace nido {
namespace {

constexpr int kThreads = 256;

inline unsigned grid_for(int64_t work, int per_block, int max_blocks = 148 * 16) {
  int64_t b = (work + per_block - 1) / per_block;
  if (b < 1) b = 1;
  if (b > max_blocks) b = max_blocks;
  return (unsigned)b;
}

// k_v: one warp per vertex, lane l sums edges l, l+32, ... then a shuffle-down
// tree (sum_vertex_weights_kernel, graph_cuda.cu:302-346).  Alongside, for
// the move kernels' choice of integer tables: flags[0] becomes nonzero when a
// weight is not a finite integer and flags[1] keeps the largest sum of |w| of
// a vertex (as the bits of a non-negative double, which order like the
// values).  One lane per warp writes each, and only while the value would
// change, so the flags cost no queue of same-address atomics.
__global__ void k_vertex_weights(const int64_t* __restrict__ off, const double* __restrict__ w,
                                 int64_t nv, double* __restrict__ k, unsigned long long* __restrict__ flags) {
  const int lane = threadIdx.x & 31;
  const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  unsigned long long bad = 0;
  double amax = 0.;
  for (int64_t v = warp; v < nv; v += nw) {
    const int64_t s = off[v], e = off[v + 1];
    double x = 0., ax = 0.;
    for (int64_t j = s + lane; j < e; j += 32) {
      const double y = w[j];
      x += y;
      ax += fabs(y);
      if (!(fabs(y) < 9.0e15) || y != trunc(y)) ++bad;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      x += __shfl_down_sync(NIDO_FULL_MASK, x, o);
      ax += __shfl_down_sync(NIDO_FULL_MASK, ax, o);
    }
    if (lane == 0) {
      k[v] = x;
      amax = fmax(amax, ax);
    }
  }
  const bool anybad = __any_sync(NIDO_FULL_MASK, bad != 0);
  if (lane == 0) {
    volatile unsigned long long* vf = flags;
    if (anybad && vf[0] == 0) atomicExch(&flags[0], 1ull);
    const unsigned long long ab = (unsigned long long)__double_as_longlong(amax);
    if (amax > 0. && vf[1] < ab) atomicMax(&flags[1], ab);
  }
}

// m, first stage: compute_mass_reduce_kernel<32><<<4096,32>>>
// (graph_cuda.cu:1786-1804).
__global__ void k_mass_blocks(const double* __restrict__ k, int64_t nv, double* __restrict__ part) {
  double x = 0.;
  for (int64_t i = threadIdx.x + 32 * (int64_t)blockIdx.x; i < nv; i += 32 * (int64_t)gridDim.x) x += k[i];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(NIDO_FULL_MASK, x, o);
  if (threadIdx.x == 0) part[blockIdx.x] = x;
}

// reduce_vector_kernel<32><<<1,1024>>> (graph_cuda.cu:1806-1835); writes
// scale * sum to *out.
__global__ void __launch_bounds__(1024) k_reduce_1024(const double* __restrict__ x, int64_t n,
                                                      double scale, double* __restrict__ out) {
  __shared__ double ws[32];
  double s = 0.;
  for (int64_t i = threadIdx.x; i < n; i += 1024) s += x[i];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(NIDO_FULL_MASK, s, o);
  if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x < 32) {
    s = ws[threadIdx.x];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(NIDO_FULL_MASK, s, o);
    if (threadIdx.x == 0) *out = scale * s;
  }
}

// singleton_partition_kernel (graph_cuda.cu:410-429)
__global__ void k_singleton(int64_t nv, const double* __restrict__ k, int32_t* __restrict__ comm,
                            int32_t* __restrict__ newc, double* __restrict__ a) {
  for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < nv;
       v += (int64_t)gridDim.x * blockDim.x) {
    comm[v] = (int32_t)v;
    newc[v] = (int32_t)v;
    a[v] = k[v];
  }
}

// compute_community_weights_kernel (graph_cuda.cu:370-390)
__global__ void k_comm_weights(int64_t nv, const int32_t* __restrict__ comm,
                               const double* __restrict__ k, double* __restrict__ a) {
  for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < nv;
       v += (int64_t)gridDim.x * blockDim.x)
    atomicAdd(&a[comm[v]], k[v]);
}

// update_community_weights_kernel + exchange_vector_kernel fused
// (graph_cuda.cu:1234-1250, 1191-1196): movers subtract k_v from the old
// community and add it to the new one; then ids swap so newc keeps the old
// id for restore_community.  Movers of a warp with the same old (new)
// community add their k_v first (in lane order) and issue one atomic per
// community, which takes the contention off communities many vertices join.
// The atomics' order is not fixed (as in the reference); on integer weights
// every sum is exact.
__device__ __forceinline__ void warp_community_add(double* a, int c, double x, bool on) {
  const int lane = threadIdx.x & 31;
  const unsigned peers = __match_any_sync(NIDO_FULL_MASK, on ? c : -1);
  double s = 0.;
  unsigned rem = on ? peers : 0u;
  const int maxcnt = __reduce_max_sync(NIDO_FULL_MASK, (unsigned)__popc(rem));
  for (int it = 0; it < maxcnt; ++it) {
    const int src = rem ? __ffs(rem) - 1 : lane;
    const double y = __shfl_sync(NIDO_FULL_MASK, x, src);
    if (rem) { s += y; rem &= rem - 1; }
  }
  if (on && lane == __ffs(peers) - 1) atomicAdd(&a[c], s);
}

__global__ void k_commit(int64_t v0, int64_t v1, const double* __restrict__ k,
                         int32_t* __restrict__ comm, int32_t* __restrict__ newc,
                         double* __restrict__ a, int64_t* __restrict__ moved,
                         const int32_t* __restrict__ gate) {
  if (gate && *gate == 0) return;  // the device-resident loop's restore, when not needed
  int64_t cnt = 0;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  // the loop runs warp-uniformly (the warp's first lane decides)
  for (int64_t base = v0 + blockIdx.x * (int64_t)blockDim.x + (threadIdx.x & ~31); base < v1; base += stride) {
    const int64_t v = base + (threadIdx.x & 31);
    int32_t src = 0, dst = 0;
    double kv = 0.;
    const bool in = v < v1;
    if (in) {
      src = comm[v];
      dst = newc[v];
    }
    const bool mv = in && src != dst;
    if (mv) {
      kv = k[v];
      ++cnt;
    }
    if (__any_sync(NIDO_FULL_MASK, mv)) {
      warp_community_add(a, src, -kv, mv);
      warp_community_add(a, dst, kv, mv);
    }
    if (in) {
      comm[v] = dst;
      newc[v] = src;
    }
  }
  if (moved) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) cnt += __shfl_down_sync(NIDO_FULL_MASK, cnt, o);
    if ((threadIdx.x & 31) == 0 && cnt) atomicAdd((unsigned long long*)moved, (unsigned long long)cnt);
  }
}

// The vertices of one batch as ranges of perm (one per degree tier).
struct PermSpans {
  int64_t start[kNumTiers];
  int64_t pre[kNumTiers + 1];  // prefix of the range lengths
};

// k_commit over the vertices of PermSpans (a colour-class batch); movers of a
// warp with the same old (new) community add their k_v first, as k_commit does
__global__ void k_commit_spans(PermSpans r, const int32_t* __restrict__ perm, const double* __restrict__ k,
                               int32_t* __restrict__ comm, int32_t* __restrict__ newc, double* __restrict__ a) {
  const int64_t total = r.pre[kNumTiers];
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t base = blockIdx.x * (int64_t)blockDim.x + (threadIdx.x & ~31); base < total; base += stride) {
    const int64_t x = base + (threadIdx.x & 31);
    const bool in = x < total;
    int v = 0;
    int32_t src = 0, dst = 0;
    double kv = 0.;
    if (in) {
      int t = 0;
      while (r.pre[t + 1] <= x) ++t;
      v = perm[r.start[t] + (x - r.pre[t])];
      src = comm[v];
      dst = newc[v];
    }
    const bool mv = in && src != dst;
    if (mv) kv = k[v];
    if (__any_sync(NIDO_FULL_MASK, mv)) {
      warp_community_add(a, src, -kv, mv);
      warp_community_add(a, dst, kv, mv);
    }
    if (in) {
      comm[v] = dst;
      newc[v] = src;
    }
  }
}

// ---- modularity -------------------------------------------------------------------
// Sum of w[j] over j = j0, j0+step, ... < e with comm[adj[j]] == own, added in
// that order; four edges' loads (bounds-guarded) are issued before any is
// added, so four dependent gathers are in flight per lane at every degree.
__device__ __forceinline__ double own_weight(const int32_t* __restrict__ adj, const double* __restrict__ w,
                                             const int32_t* __restrict__ comm, int32_t own, int64_t j0,
                                             int64_t e, int step) {
  double x = 0.;
  for (int64_t j = j0; j < e; j += 4 * (int64_t)step) {
    int u[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const int64_t jk = j + k * (int64_t)step;
      u[k] = jk < e ? adj[jk] : -1;
    }
    int c[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) c[k] = u[k] >= 0 ? comm[u[k]] : 0;
    // only in-community edges load their weight: a warp's 32-byte weight
    // sectors with no such edge are never fetched (most of them while the
    // communities are small); the sum and its order are unchanged
    bool in[4];
    double wt[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      in[k] = u[k] >= 0 && c[k] == own;
      wt[k] = in[k] ? w[j + k * (int64_t)step] : 0.;
    }
#pragma unroll
    for (int k = 0; k < 4; ++k)
      if (in[k]) x += wt[k];
  }
  return x;
}

// Stage 1: per-vertex in-community weight (self-loops included), one group of
// G lanes per vertex; lane l sums edges l, l+G, ... then a fixed tree.
template <int G>
__global__ void k_q_self_group(const int32_t* __restrict__ list, int64_t n,
                               const int64_t* __restrict__ off, const int32_t* __restrict__ adj,
                               const double* __restrict__ w, const int32_t* __restrict__ comm,
                               double* __restrict__ selfv) {
  constexpr int VPW = 32 / G;
  const int lane = threadIdx.x & 31, gl = lane & (G - 1), gid = lane / G;
  const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t b = warp * VPW; b < n; b += nw * VPW) {
    const int64_t idx = b + gid;
    double x = 0.;
    int v = 0;
    if (idx < n) {
      v = list[idx];
      x = own_weight(adj, w, comm, comm[v], off[v] + gl, off[v + 1], G);
    }
#pragma unroll
    for (int o = G / 2; o > 0; o >>= 1) x += __shfl_down_sync(NIDO_FULL_MASK, x, o, G);
    if (gl == 0 && idx < n) selfv[v] = x;
  }
}

template <int T>
__global__ void __launch_bounds__(T) k_q_self_cta(const int32_t* __restrict__ list, int64_t n,
                                                  const int64_t* __restrict__ off,
                                                  const int32_t* __restrict__ adj,
                                                  const double* __restrict__ w,
                                                  const int32_t* __restrict__ comm,
                                                  double* __restrict__ selfv) {
  __shared__ double ws[T / 32];
  for (int64_t idx = blockIdx.x; idx < n; idx += gridDim.x) {
    const int v = list[idx];
    double x = own_weight(adj, w, comm, comm[v], off[v] + threadIdx.x, off[v + 1], T);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(NIDO_FULL_MASK, x, o);
    if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = x;
    __syncthreads();
    if (threadIdx.x == 0) {
      double s = 0.;
      for (int i = 0; i < T / 32; ++i) s += ws[i];
      selfv[v] = s;
    }
    __syncthreads();
  }
}

// Hub tier: one CTA per kHubSeg-edge segment of the hub plan (a partial sum
// per item), then one warp per hub adds its items' partials (lane-strided,
// then a fixed tree), so a hub's sum is spread over many CTAs instead of
// running its whole edge list on one.
__global__ void __launch_bounds__(256) k_q_self_seg(const int2* __restrict__ items, int64_t n,
                                                    const int32_t* __restrict__ hub_v,
                                                    const int64_t* __restrict__ off,
                                                    const int32_t* __restrict__ adj,
                                                    const double* __restrict__ w,
                                                    const int32_t* __restrict__ comm,
                                                    double* __restrict__ part) {
  __shared__ double ws[8];
  for (int64_t idx = blockIdx.x; idx < n; idx += gridDim.x) {
    const int2 it = items[idx];
    const int v = hub_v[it.x];
    const int64_t e0 = off[v] + (int64_t)it.y * kHubSeg;
    const int64_t e1 = min(off[v + 1], e0 + kHubSeg);
    double x = own_weight(adj, w, comm, comm[v], e0 + threadIdx.x, e1, 256);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(NIDO_FULL_MASK, x, o);
    if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = x;
    __syncthreads();
    if (threadIdx.x == 0) {
      double s = 0.;
      for (int i = 0; i < 8; ++i) s += ws[i];
      part[idx] = s;
    }
    __syncthreads();
  }
}

__global__ void k_q_hub_sum(int64_t nh, const int32_t* __restrict__ hub_v, const int64_t* __restrict__ first,
                            const double* __restrict__ part, double* __restrict__ selfv) {
  const int lane = threadIdx.x & 31;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t h = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; h < nh; h += nw) {
    double x = 0.;
    for (int64_t i = first[h] + lane; i < first[h + 1]; i += 32) x += part[i];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(NIDO_FULL_MASK, x, o);
    if (lane == 0) selfv[hub_v[h]] = x;
  }
}

// Stage 2: the reference's thread slots and 16-lane groups
// (compute_modularity_reduce_kernel<128,16>, graph_cuda.cu:2096-2134, grid
// min(ceil(nv/8), 65535)): slot t takes vertices t, t+S, ...; ac folds
// fma(a_v, a_v, ac) as nvcc contracts "ac += w*w"; lane 0 of each group
// writes self/(2m) - ac/(4m*m).
__global__ void k_q_groups(int64_t nv, int64_t S, int64_t ngroups, const double* __restrict__ selfv,
                           const double* __restrict__ a, const double* __restrict__ dm,
                           double* __restrict__ modv) {
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const int64_t g = t >> 4;
  double s = 0., ac = 0.;
  if (g < ngroups) {
    for (int64_t v = t; v < nv; v += S) {
      s += selfv[v];
      ac = fma(a[v], a[v], ac);
    }
  }
#pragma unroll
  for (int o = 8; o > 0; o >>= 1) {
    s += __shfl_down_sync(NIDO_FULL_MASK, s, o, 16);
    ac += __shfl_down_sync(NIDO_FULL_MASK, ac, o, 16);
  }
  if ((t & 15) == 0 && g < ngroups) {
    const double m = dm[0];
    double x = __ddiv_rn(s, __dmul_rn(2., m));
    x = __dsub_rn(x, __ddiv_rn(ac, __dmul_rn(__dmul_rn(4., m), m)));
    modv[g] = __dadd_rn(0., x);
  }
}

// Batch cuts of partition_graph_edge_batch (graph_gpu.cpp:303-339) on one
// thread.
__global__ void k_batch_cuts(const int64_t* __restrict__ off, int64_t nv, int nb,
                             int64_t* __restrict__ cuts, int64_t* __restrict__ parts) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  batch_cuts(off, nv, nb, cuts, parts);
}

// maximum degrees of the warp, CTA-S, CTA-M, CTA-L and CTA-XL tiers
struct TierThresholds {
  int warp, ctas, ctam, ctal, ctax;
};

__device__ __forceinline__ int tier_of(int64_t d, const TierThresholds& thr) {
  if (d <= 4) return kTierG4;
  if (d <= 8) return kTierG8;
  if (d <= 16) return kTierG16;
  if (d <= 32) return kTierG32;
  if (d <= thr.warp) return kTierWarp;
  if (d <= thr.ctas) return kTierCtaS;
  if (d <= thr.ctam) return kTierCtaM;
  if (d <= thr.ctal) return kTierCtaL;
  if (d <= thr.ctax && d <= kCtaXAMaxDeg) return kTierCtaXA;  // two 512-thread CTAs an SM
  if (d <= thr.ctax) return kTierCtaX;
  return kTierHub;
}

// key = tier * nb + batch, so every (tier, batch) range and every tier over
// all batches is contiguous after the stable sort.  Counts and the maximum
// degree are aggregated per warp before the global atomics.
// Many-graph mode (gid non-null): the batch is found in the vertex's own
// graph's cuts (gcuts, nb+1 per graph, relative to gbase), vertices of graphs
// that are not iterating get the key past all tiers, and every vertex's batch
// is stored in vbatch.
__global__ void k_tier_keys(const int64_t* __restrict__ off, int64_t nv, const int64_t* __restrict__ cuts,
                            int nb, uint32_t* __restrict__ keys, uint32_t* __restrict__ vals,
                            int64_t* __restrict__ counts, unsigned long long* __restrict__ maxdeg,
                            const int32_t* __restrict__ gid, const int64_t* __restrict__ gbase,
                            const int64_t* __restrict__ gcuts, const int32_t* __restrict__ gactive,
                            int32_t* __restrict__ vbatch, const int32_t* __restrict__ vcolor, TierThresholds thr) {
  const int lane = threadIdx.x & 31;
  const uint32_t skip = (uint32_t)(kNumTiers * nb);
  unsigned long long md = 0;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t base = blockIdx.x * (int64_t)blockDim.x; base < nv; base += stride) {
    const int64_t v = base + threadIdx.x;
    uint32_t key = 0xffffffffu;
    if (v < nv) {
      const int64_t* c = cuts;
      int64_t x = v;
      bool active = true;
      if (gid) {
        const int g = gid[v];
        c = gcuts + (int64_t)g * (nb + 1);
        x = v - gbase[g];
        active = gactive[g] != 0;
      }
      int lo = 0, hi = nb;  // batch b with c[b] <= x < c[b+1]
      if (vcolor) {
        lo = vcolor[v];  // colour-class batches
      } else {
        while (hi - lo > 1) {
          const int mid = (lo + hi) / 2;
          if (c[mid] <= x) lo = mid; else hi = mid;
        }
      }
      if (vbatch) vbatch[v] = lo;
      const int64_t d = off[v + 1] - off[v];
      // vertices without edges never move (no neighbour community; their
      // target stays their own community), so no tier lists them
      key = (active && d > 0) ? (uint32_t)(tier_of(d, thr) * nb + lo) : skip;
      keys[v] = key;
      vals[v] = (uint32_t)v;
      if (active) md = md > (unsigned long long)d ? md : (unsigned long long)d;
    }
    const unsigned peers = __match_any_sync(NIDO_FULL_MASK, key);
    if (key != 0xffffffffu && lane == __ffs(peers) - 1)
      atomicAdd((unsigned long long*)&counts[key], (unsigned long long)__popc(peers));
  }
  md = __reduce_max_sync(NIDO_FULL_MASK, (unsigned)md);
  if (lane == 0 && md) atomicMax(maxdeg, md);
}

// Keep flags of the listed vertices whose graph still iterates (pos[i] = 1)
// and, after the scan, their scatter in list order.
__global__ void k_keep_flags(const int32_t* __restrict__ perm, int64_t n, const int32_t* __restrict__ gid,
                             const int32_t* __restrict__ gactive, int64_t* __restrict__ pos) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    pos[i] = gactive[gid[perm[i]]] != 0 ? 1 : 0;
}

__global__ void k_scatter_kept(const int32_t* __restrict__ perm, int64_t n, const int32_t* __restrict__ gid,
                               const int32_t* __restrict__ gactive, const int64_t* __restrict__ pos,
                               int32_t* __restrict__ out) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const int32_t v = perm[i];
    if (gactive[gid[v]] != 0) out[pos[i]] = v;
  }
}

// new segment offsets: the scanned positions at the old segment starts
__global__ void k_gather_offsets(const int64_t* __restrict__ old_off, int64_t nseg, const int64_t* __restrict__ pos,
                                 int64_t* __restrict__ new_off) {
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k <= nseg; k += (int64_t)gridDim.x * blockDim.x)
    new_off[k] = pos[old_off[k]];
}

}  // namespace

// k_v of the current phase; its weight flags (dcount[2..3]) are read back by
// build_batches, which every phase runs after it
int launch_vertex_weights(nido_graph_s* g) {
  if (g->nv == 0) return NIDO_OK;
  cudaStream_t s = g->ctx->stream;
  unsigned long long* flags = reinterpret_cast<unsigned long long*>(g->dcount + 2);
  NIDO_CUDA_TRY(cudaMemsetAsync(flags, 0, 2 * sizeof(unsigned long long), s));
  k_vertex_weights<<<grid_for(g->nv * 32, kThreads, 148 * 64), kThreads, 0, s>>>(g->off, g->w, g->nv, g->k, flags);
  NIDO_LAUNCH_CHECK();
  return NIDO_OK;
}

int launch_mass(nido_graph_s* g) {
  Arena ar(g->scratch, g->scratch_bytes);
  double* part = ar.take<double>(4096);
  if (!part) return nido_set_error(NIDO_E_NOMEM, "scratch arena too small (mass)");
  k_mass_blocks<<<4096, 32, 0, g->ctx->stream>>>(g->k, g->nv, part);
  NIDO_LAUNCH_CHECK();
  k_reduce_1024<<<1, 1024, 0, g->ctx->stream>>>(part, 4096, 0.5, g->dm);
  NIDO_LAUNCH_CHECK();
  NIDO_CUDA_TRY(cudaMemcpyAsync(&g->m, g->dm, sizeof(double), cudaMemcpyDeviceToHost, g->ctx->stream));
  NIDO_CUDA_TRY(cudaStreamSynchronize(g->ctx->stream));
  return NIDO_OK;
}

int launch_singleton(nido_graph_s* g) {
  if (g->nv == 0) return NIDO_OK;
  k_singleton<<<grid_for(g->nv, kThreads), kThreads, 0, g->ctx->stream>>>(g->nv, g->k, g->comm,
                                                                          g->newc, g->a);
  NIDO_LAUNCH_CHECK();
  return NIDO_OK;
}

int launch_set_comm(nido_graph_s* g) {
  NIDO_CUDA_TRY(cudaMemsetAsync(g->a, 0, sizeof(double) * g->nv, g->ctx->stream));
  if (g->nv == 0) return NIDO_OK;
  k_comm_weights<<<grid_for(g->nv, kThreads), kThreads, 0, g->ctx->stream>>>(g->nv, g->comm, g->k, g->a);
  NIDO_LAUNCH_CHECK();
  return NIDO_OK;
}

int launch_commit(nido_graph_s* g, int64_t v0, int64_t v1) {
  if (v1 <= v0) return NIDO_OK;
  k_commit<<<grid_for(v1 - v0, kThreads), kThreads, 0, g->ctx->stream>>>(v0, v1, g->k, g->comm,
                                                                         g->newc, g->a, nullptr, nullptr);
  NIDO_LAUNCH_CHECK();
  return NIDO_OK;
}

int launch_commit_batch(nido_graph_s* g, int b) {
  if (b < 0 || b >= g->nbatches) return nido_set_error(NIDO_E_INVALID, "batch %d out of range", b);
  if (!g->color_mode || g->gid) return launch_commit(g, g->cuts[b], g->cuts[b + 1]);
  // a colour class is not a vertex range: commit the batch's vertices from
  // the tier lists, every (tier, batch) range of perm
  PermSpans r{};
  int64_t tot = 0;
  const int nb = g->nbatches;
  for (int t = 0; t < kNumTiers; ++t) {
    r.start[t] = g->tier_off[(size_t)t * nb + b];
    r.pre[t] = tot;
    tot += g->tier_off[(size_t)t * nb + b + 1] - r.start[t];
  }
  r.pre[kNumTiers] = tot;
  if (tot == 0) return NIDO_OK;
  k_commit_spans<<<grid_for(tot, kThreads), kThreads, 0, g->ctx->stream>>>(r, g->perm, g->k, g->comm, g->newc, g->a);
  NIDO_LAUNCH_CHECK();
  return NIDO_OK;
}

// the commit of [v0, v1) only when *gate is non-zero (read on the device)
int launch_commit_gated(nido_graph_s* g, int64_t v0, int64_t v1, const int32_t* gate) {
  if (v1 <= v0) return NIDO_OK;
  k_commit<<<grid_for(v1 - v0, kThreads), kThreads, 0, g->ctx->stream>>>(v0, v1, g->k, g->comm,
                                                                         g->newc, g->a, nullptr, gate);
  NIDO_LAUNCH_CHECK();
  return NIDO_OK;
}

// Per-vertex in-community weight (self-loops included) of every listed
// vertex, over all tiers of the current tier lists.
// CTAs of the self-sum kernels resident on the GPU at once (grids are capped
// there: grid-stride kernels launched with more leave a partial last wave)
struct QResident {
  int g4 = 148 * 8, g8 = 148 * 8, g16 = 148 * 8, g32 = 148 * 8, cta = 148 * 8, seg = 148 * 8;
};

template <typename K>
int q_resident(K kernel, int threads, int sms) {
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, 0) != cudaSuccess) {
    cudaGetLastError();
    per_sm = 1;
  }
  return std::max(per_sm, 1) * sms;
}

QResident q_resident_all() {
  QResident r;
  int dev = 0, sms = 148;
  if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) {
    cudaGetLastError();
    return r;
  }
  r.g4 = q_resident(k_q_self_group<4>, kThreads, sms);
  r.g8 = q_resident(k_q_self_group<8>, kThreads, sms);
  r.g16 = q_resident(k_q_self_group<16>, kThreads, sms);
  r.g32 = q_resident(k_q_self_group<32>, kThreads, sms);
  r.cta = q_resident(k_q_self_cta<256>, 256, sms);
  r.seg = q_resident(k_q_self_seg, 256, sms);
  return r;
}

// The tiers' self-sums touch disjoint vertices: the large-degree tiers run
// on the context's side streams beside the small ones (joined on return).
int launch_q_self(nido_graph_s* g, double* selfv) {
  nido_ctx_s* ctx = g->ctx;
  static const QResident g_qres = q_resident_all();  // once per process (thread-safe)
  const cudaStream_t main_s = ctx->stream;
  // vertices in no tier list (no edges) have no in-community weight
  NIDO_CUDA_TRY(cudaMemsetAsync(selfv, 0, sizeof(double) * (size_t)g->nv, main_s));
  NIDO_CUDA_TRY(cudaEventRecord(ctx->fork_ev, main_s));
  for (int i = 0; i < 2; ++i) NIDO_CUDA_TRY(cudaStreamWaitEvent(ctx->aux[i], ctx->fork_ev, 0));
  const int nb = g->nbatches;
  for (int t = kNumTiers - 1; t >= 0; --t) {
    const int64_t b0 = g->tier_off[(size_t)t * nb], b1 = g->tier_off[(size_t)(t + 1) * nb];
    const int64_t n = b1 - b0;
    if (n == 0) continue;
    const int32_t* list = g->perm + b0;
    const cudaStream_t s = t >= kTierCtaL ? ctx->aux[0] : (t >= kTierG32 ? ctx->aux[1] : main_s);
    switch (t) {
      case kTierG4:
        k_q_self_group<4><<<grid_for(n, kThreads / 4 * 8, g_qres.g4), kThreads, 0, s>>>(list, n, g->off, g->adj, g->w,
                                                                                       g->comm, selfv);
        break;
      case kTierG8:
        k_q_self_group<8><<<grid_for(n, kThreads / 8 * 4, g_qres.g8), kThreads, 0, s>>>(list, n, g->off, g->adj, g->w,
                                                                                       g->comm, selfv);
        break;
      case kTierG16:
        k_q_self_group<16><<<grid_for(n, kThreads / 16 * 2, g_qres.g16), kThreads, 0, s>>>(list, n, g->off, g->adj,
                                                                                           g->w, g->comm, selfv);
        break;
      case kTierG32:
      case kTierWarp:
      case kTierCtaS:
      case kTierCtaM:
        k_q_self_group<32><<<grid_for(n, kThreads / 32, g_qres.g32), kThreads, 0, s>>>(list, n, g->off, g->adj, g->w,
                                                                                      g->comm, selfv);
        break;
      case kTierHub:
        if (g->nhubs == n && g->hub_nitems > 0) {  // the hub plan covers this list
          k_q_self_seg<<<grid_for(g->hub_nitems, 1, g_qres.seg), 256, 0, s>>>(
              g->hub_items, g->hub_nitems, g->hub_v, g->off, g->adj, g->w, g->comm, g->hub_part);
          NIDO_LAUNCH_CHECK();
          k_q_hub_sum<<<grid_for(n * 32, 256, kSMs * 8), 256, 0, s>>>(n, g->hub_v, g->hub_item_first, g->hub_part,
                                                                     selfv);
          break;
        }
        k_q_self_cta<256><<<grid_for(n, 1, g_qres.cta), 256, 0, s>>>(list, n, g->off, g->adj, g->w, g->comm, selfv);
        break;
      default:
        k_q_self_cta<256><<<grid_for(n, 1, g_qres.cta), 256, 0, s>>>(list, n, g->off, g->adj, g->w, g->comm, selfv);
        break;
    }
    NIDO_LAUNCH_CHECK();
  }
  for (int i = 0; i < 2; ++i) {
    NIDO_CUDA_TRY(cudaEventRecord(ctx->join_ev[i], ctx->aux[i]));
    NIDO_CUDA_TRY(cudaStreamWaitEvent(main_s, ctx->join_ev[i], 0));
  }
  return NIDO_OK;
}

int launch_modularity(nido_graph_s* g, double* q) {
  cudaStream_t s = g->ctx->stream;
  if (g->nv == 0) { *q = 0.; return NIDO_OK; }
  NIDO_TRY(launch_modularity_dev(g));
  NIDO_CUDA_TRY(cudaMemcpyAsync(q, g->dm + 1, sizeof(double), cudaMemcpyDeviceToHost, s));
  NIDO_CUDA_TRY(cudaStreamSynchronize(s));
  return NIDO_OK;
}

// Q of the current partition into g->dm[1], enqueued only (no host
// synchronisation), so it can be captured into the device-resident loop.
// The tier lists must be valid (build_batches) before a capture.
int launch_modularity_dev(nido_graph_s* g) {
  cudaStream_t s = g->ctx->stream;
  const int64_t nv = g->nv;
  if (nv == 0) {
    NIDO_CUDA_TRY(cudaMemsetAsync(g->dm + 1, 0, sizeof(double), s));
    return NIDO_OK;
  }
  if (!g->bins_valid) NIDO_TRY(build_batches(g));
  Arena ar(g->scratch, g->scratch_bytes);
  double* selfv = ar.take<double>(nv);
  int64_t grid = (nv + 7) / 8;
  if (grid > 65535) grid = 65535;
  const int64_t S = 128 * grid;
  const int64_t nslots = std::min<int64_t>(S, nv);
  const int64_t ngroups = (nslots + 15) / 16;
  double* modv = ar.take<double>(ngroups);
  if (!selfv || !modv) return nido_set_error(NIDO_E_NOMEM, "scratch arena too small (modularity)");
  NIDO_TRY(launch_q_self(g, selfv));
  const int64_t threads = ngroups * 16;
  k_q_groups<<<(unsigned)((threads + 255) / 256), 256, 0, s>>>(nv, S, ngroups, selfv, g->a, g->dm, modv);
  NIDO_LAUNCH_CHECK();
  k_reduce_1024<<<1, 1024, 0, s>>>(modv, ngroups, 1.0, g->dm + 1);
  NIDO_LAUNCH_CHECK();
  return NIDO_OK;
}

int build_batches(nido_graph_s* g) {
  cudaStream_t s = g->ctx->stream;
  const bool multi = g->gid != nullptr;  // many graphs: per-graph cuts in g->gcuts
  const bool colored = g->color_mode && !multi;
  if (colored) {
    // conflict-free batches: the colour classes of the current graph
    if (g->cap_vcolor < g->nv) {
      raw_free(g->ctx, g->vcolor);
      g->vcolor = nullptr;
      g->cap_vcolor = 0;
      NIDO_CUDA_TRY(raw_alloc(g->ctx, (void**)&g->vcolor, sizeof(int32_t) * (size_t)std::max<int64_t>(g->nv, 1)));
      g->cap_vcolor = std::max<int64_t>(g->nv, 1);
    }
    int64_t nc = 0;
    NIDO_TRY(color_current_graph(g, kColorBatchSeed, g->vcolor, &nc));
    g->nbatches = (int)std::max<int64_t>(nc, 1);
  } else if (!multi) {
    g->nbatches = g->nb_user;
  }
  const int nb = g->nbatches;
  const int64_t nv = g->nv;
  Arena ar(g->scratch, g->scratch_bytes);
  int64_t* dcuts = ar.take<int64_t>(nb + 1);
  int64_t* dparts = ar.take<int64_t>(nb + 2);
  const int64_t nkeys = (int64_t)kNumTiers * nb;
  int64_t* counts = ar.take<int64_t>(nkeys + 1);
  unsigned long long* maxdeg = ar.take<unsigned long long>(1);
  uint32_t* keys = ar.take<uint32_t>(nv);
  uint32_t* keys2 = ar.take<uint32_t>(nv);
  uint32_t* vals2 = ar.take<uint32_t>(nv);
  int64_t* rtemp = ar.take<int64_t>(std::max(radix_temp_elems(nv), scan_temp_elems(nkeys)));
  if (!rtemp) return nido_set_error(NIDO_E_NOMEM, "scratch arena too small (batches)");
  if (!multi && !colored) {
    k_batch_cuts<<<1, 1, 0, s>>>(g->off, nv, nb, dcuts, dparts);
    NIDO_LAUNCH_CHECK();
  }
  NIDO_CUDA_TRY(cudaMemsetAsync(counts, 0, sizeof(int64_t) * (nkeys + 1), s));
  NIDO_CUDA_TRY(cudaMemsetAsync(maxdeg, 0, sizeof(unsigned long long), s));
  if (nv > 0) {
    k_tier_keys<<<grid_for(nv, kThreads), kThreads, 0, s>>>(g->off, nv, dcuts, nb, keys, (uint32_t*)g->perm,
                                                           counts, maxdeg, g->gid, g->gbase, g->gcuts,
                                                           g->gactive, g->vbatch, colored ? g->vcolor : nullptr,
                                                           TierThresholds{g->cfg.warp_max, g->cfg.ctas_max,
                                                                          g->cfg.ctam_max, g->cfg.ctal_max,
                                                                          g->cfg.ctax_max});
    NIDO_LAUNCH_CHECK();
    int bits = 0;
    while (((int64_t)1 << bits) < nkeys + 1) ++bits;
    NIDO_TRY(radix_sort_pairs(keys, (uint32_t*)g->perm, keys2, vals2, nv, bits, rtemp, s));
  }
  NIDO_TRY(scan_exclusive_i64(counts, counts, nkeys, rtemp, s));
  g->cuts.assign(nb + 1, 0);
  g->tier_off.assign(nkeys + 1, 0);
  unsigned long long md = 0;
  if (!multi && !colored)
    NIDO_CUDA_TRY(cudaMemcpyAsync(g->cuts.data(), dcuts, sizeof(int64_t) * (nb + 1), cudaMemcpyDeviceToHost, s));
  NIDO_CUDA_TRY(cudaMemcpyAsync(g->tier_off.data(), counts, sizeof(int64_t) * (nkeys + 1), cudaMemcpyDeviceToHost, s));
  NIDO_CUDA_TRY(cudaMemcpyAsync(&md, maxdeg, sizeof(md), cudaMemcpyDeviceToHost, s));
  unsigned long long wf[2] = {1, 0};  // weight flags of the last k_v
  if (nv > 0) NIDO_CUDA_TRY(cudaMemcpyAsync(wf, g->dcount + 2, sizeof(wf), cudaMemcpyDeviceToHost, s));
  NIDO_CUDA_TRY(cudaStreamSynchronize(s));
  {
    double amax = 0.;
    memcpy(&amax, &wf[1], sizeof(amax));
    // int32 table sums are exact when no vertex's sum of |w| reaches 2^31
    g->int_weights = wf[0] == 0 && amax < 2147483648.0;
  }
  g->max_degree = (int64_t)md;
  g->bins_valid = true;
  ++g->plan_epoch;
  return plan_hubs(g);
}

// Many-graph mode: drop the vertices of graphs that stopped iterating
// (gactive 0) from the current tier lists.  A stable compaction of the
// listed vertices (flags, scan, scatter) keeps every (tier, batch) list in its
// order, so the lists equal what build_batches would list for the same
// graphs, at the cost of one pass over the listed vertices instead of a key
// pass over every vertex and a sort.  The largest degree stays the old one
// (an upper bound).
int compact_batches(nido_graph_s* g) {
  if (!g->gid || !g->bins_valid || g->color_mode) {
    g->bins_valid = false;
    return build_batches(g);
  }
  cudaStream_t s = g->ctx->stream;
  const int64_t nseg = (int64_t)kNumTiers * g->nbatches;
  const int64_t n = g->tier_off[(size_t)nseg];
  if (n == 0) return NIDO_OK;
  Arena ar(g->scratch, g->scratch_bytes);
  int64_t* pos = ar.take<int64_t>(n + 1);
  int32_t* out = ar.take<int32_t>(n);
  int64_t* segs = ar.take<int64_t>(2 * (nseg + 1));
  int64_t* rtemp = ar.take<int64_t>(scan_temp_elems(n));
  if (!pos || !out || !segs || !rtemp) return nido_set_error(NIDO_E_NOMEM, "scratch arena too small (list compaction)");
  int32_t* perm = reinterpret_cast<int32_t*>(g->perm);
  k_keep_flags<<<grid_for(n, kThreads), kThreads, 0, s>>>(perm, n, g->gid, g->gactive, pos);
  NIDO_LAUNCH_CHECK();
  NIDO_TRY(scan_exclusive_i64(pos, pos, n, rtemp, s));
  k_scatter_kept<<<grid_for(n, kThreads), kThreads, 0, s>>>(perm, n, g->gid, g->gactive, pos, out);
  NIDO_LAUNCH_CHECK();
  NIDO_CUDA_TRY(cudaMemcpyAsync(segs, g->tier_off.data(), sizeof(int64_t) * (nseg + 1), cudaMemcpyHostToDevice, s));
  k_gather_offsets<<<grid_for(nseg + 1, 128), 128, 0, s>>>(segs, nseg, pos, segs + nseg + 1);
  NIDO_LAUNCH_CHECK();
  std::vector<int64_t> off(nseg + 1);
  NIDO_CUDA_TRY(cudaMemcpyAsync(off.data(), segs + nseg + 1, sizeof(int64_t) * (nseg + 1), cudaMemcpyDeviceToHost, s));
  NIDO_CUDA_TRY(cudaStreamSynchronize(s));
  if (off[nseg] > 0)
    NIDO_CUDA_TRY(cudaMemcpyAsync(perm, out, sizeof(int32_t) * off[nseg], cudaMemcpyDeviceToDevice, s));
  g->tier_off = off;
  ++g->plan_epoch;
  return plan_hubs(g);
}

}  // namespace nido
