// move.cu -- the Louvain move phase for one -b batch.
//
// Replaces the reference's sort-based move (graph_gpu.cpp:457-517 +
// louvain_update_kernel, graph_cuda.cu:1450-1540): instead of building
// (vertex, community) keys for every edge and sorting them, each vertex's
// neighbour-community weights e_vc are accumulated on chip:
//   degree <= 32       a group of 4/8/16/32 lanes holds one edge per lane;
//                      equal communities are found with __match_any_sync and
//                      their weights folded in edge order (registers only)
//   degree <= warp_max one warp, open-addressing hash in shared memory
//   degree <= cta_max  one CTA, hash in shared memory
//   larger             one CTA, hash in an L2-resident global-memory slab
// Gains and the final decision use the reference's operation order
// (graph_cuda.cu:1505-1506, 1530-1533):
//   gain_c = (e_vc - ki*a_c/(2m)) / m,  self = (e_own - ki*(a_own-ki)/(2m)) / m,
//   move to the best c when gain_best - self > 0.
// Self-loops contribute weight 0 but their community still counts as a
// neighbour community (copy_weights_exclude_self_loops_kernel,
// graph_cuda.cu:2306-2316).  Equal gains go to the smallest community id, or,
// with NIDO_TIE_NIDO, to the entry the reference's 8-lane strided scan and
// shuffle tree picks: among tied entries of rank r in the id-sorted list of
// the vertex's neighbour communities, the smallest (bitrev3(r mod 8), r).
#include <algorithm>

#include "common.cuh"
#include "engine.cuh"

namespace nido {
namespace {

struct MoveArgs {
  const int64_t* __restrict__ off;
  const int32_t* __restrict__ adj;
  const double* __restrict__ w;
  const int32_t* __restrict__ comm;
  const double* __restrict__ k;
  const double* __restrict__ a;
  int32_t* __restrict__ newc;
  double m;
  int tie;
  unsigned long long* err;  // probe-limit failures (never expected)
};

constexpr unsigned long long kNoKey = ~0ull;

__device__ __forceinline__ double gain_of(double e, double ki, double ac, double m) {
  const double t = __ddiv_rn(__dmul_rn(ki, ac), __dmul_rn(2.0, m));
  return __ddiv_rn(__dsub_rn(e, t), m);
}

__device__ __forceinline__ double self_of(double eown, double ki, double aown, double m) {
  const double t = __ddiv_rn(__dmul_rn(ki, __dsub_rn(aown, ki)), __dmul_rn(2.0, m));
  return __ddiv_rn(__dsub_rn(eown, t), m);
}

__device__ __forceinline__ unsigned long long nido_key(unsigned rank) {
  return ((unsigned long long)bitrev3(rank & 7u) << 32) | rank;
}

// Sum of `wt` over the lanes in `peers`, in ascending lane order (a left fold
// in edge order).  Every lane of the warp must call it.
__device__ __forceinline__ double fold_peers(unsigned peers, bool ok, double wt) {
  const int lane = threadIdx.x & 31;
  unsigned rem = ok ? peers : 0u;
  const int maxcnt = __reduce_max_sync(NIDO_FULL_MASK, (unsigned)__popc(rem));
  double e = 0.;
  for (int i = 0; i < maxcnt; ++i) {
    const int src = rem ? __ffs(rem) - 1 : lane;
    const double x = __shfl_sync(NIDO_FULL_MASK, wt, src);
    if (rem) {
      e += x;
      rem &= rem - 1;
    }
  }
  return e;
}

// Butterfly argmax over groups of G lanes (every lane ends with the result).
template <int G>
__device__ __forceinline__ void group_best(double& g, unsigned long long& tk, int& cand) {
#pragma unroll
  for (int o = G / 2; o > 0; o >>= 1) {
    const double g2 = __shfl_xor_sync(NIDO_FULL_MASK, g, o, G);
    const unsigned long long t2 = __shfl_xor_sync(NIDO_FULL_MASK, tk, o, G);
    const int c2 = __shfl_xor_sync(NIDO_FULL_MASK, cand, o, G);
    if (better(g2, t2, g, tk)) { g = g2; tk = t2; cand = c2; }
  }
}

template <int G>
__device__ __forceinline__ double group_max(double g) {
#pragma unroll
  for (int o = G / 2; o > 0; o >>= 1) g = fmax(g, __shfl_xor_sync(NIDO_FULL_MASK, g, o, G));
  return g;
}

template <int G>
__device__ __forceinline__ double group_sum(double x) {
#pragma unroll
  for (int o = G / 2; o > 0; o >>= 1) x += __shfl_xor_sync(NIDO_FULL_MASK, x, o, G);
  return x;
}

// ---- degree <= 32: registers ---------------------------------------------------
template <int G>
__global__ void __launch_bounds__(256) k_move_group(const int32_t* __restrict__ list, int64_t n,
                                                    MoveArgs p) {
  constexpr int VPW = 32 / G;
  const int lane = threadIdx.x & 31, gl = lane & (G - 1), gid = lane / G;
  const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t b = warp * VPW; b < n; b += nw * VPW) {
    const int64_t idx = b + gid;
    const bool vok = idx < n;
    int v = 0, own = -1;
    int64_t s = 0, d = 0;
    double ki = 0., aown = 0.;
    if (vok) {
      v = list[idx];
      s = p.off[v];
      d = p.off[v + 1] - s;
      own = p.comm[v];
      ki = p.k[v];
      aown = p.a[own];
    }
    const bool ok = gl < d;
    int c = -1;
    double wt = 0.;
    if (ok) {
      const int u = p.adj[s + gl];
      c = p.comm[u];
      wt = (u == v) ? 0. : p.w[s + gl];
    }
    const unsigned long long mkey = ((unsigned long long)(unsigned)gid << 32) | (unsigned)c;
    const unsigned peers = __match_any_sync(NIDO_FULL_MASK, mkey);
    const bool lead = ok && lane == __ffs(peers) - 1;
    const double e = fold_peers(peers, ok, wt);
    double g = -NIDO_MAX_FLOAT, eown = 0.;
    unsigned long long tk = kNoKey;
    int cand = -1;
    if (lead) {
      if (c == own) {
        eown = e;
      } else {
        g = gain_of(e, ki, p.a[c], p.m);
        tk = (unsigned)c;
        cand = c;
      }
    }
    eown = group_sum<G>(eown);
    if (p.tie == NIDO_TIE_NIDO) {
      const double gm = group_max<G>(g);
      unsigned rank = 0;
      const int gbase = gid * G;
      for (int j = 0; j < G; ++j) {
        const int cj = __shfl_sync(NIDO_FULL_MASK, c, gbase + j);
        const int lj = __shfl_sync(NIDO_FULL_MASK, (int)lead, gbase + j);
        rank += (lj && cj < c) ? 1u : 0u;
      }
      tk = (cand >= 0 && g == gm) ? nido_key(rank) : kNoKey;
      if (tk == kNoKey) { g = -NIDO_MAX_FLOAT; cand = -1; }
    }
    group_best<G>(g, tk, cand);
    if (gl == 0 && vok) {
      const double self = self_of(eown, ki, aown, p.m);
      const double tot = __dsub_rn(g, self);
      p.newc[v] = (cand >= 0 && tot > 0.) ? cand : own;
    }
  }
}

// Insert (c, e) into an open-addressing table.  Tables owned by one warp
// (kAtomicVals false) see distinct keys from the warp's leaders, so the value
// update needs no atomic.  Tables hold at least twice as many slots as the
// vertex has edges, so a free slot always exists; the probe count is still
// bounded by the table size, and a full table is reported through *err.
template <bool kAtomicVals>
__device__ __forceinline__ void table_add(int* keys, double* vals, unsigned mask, int c, double e,
                                          unsigned long long* err) {
  unsigned h = hash_slot(c, mask);
  volatile int* vk = keys;
  for (unsigned probe = 0; probe <= mask; ++probe) {
    const int kk = vk[h];
    bool hit = kk == c;
    if (!hit && kk == -1) {
      const int old = atomicCAS(&keys[h], -1, c);
      hit = (old == -1 || old == c);
    }
    if (hit) {
      if (kAtomicVals) atomicAdd(&vals[h], e);
      else vals[h] += e;
      return;
    }
    h = (h + 1) & mask;
  }
  atomicAdd(err, 1ull);
}

__device__ __forceinline__ unsigned next_pow2_cap(int64_t d) {
  unsigned c = 64;
  while ((int64_t)c < 2 * d) c <<= 1;
  return c;
}

// ---- degree <= warp_max: one warp per vertex, shared-memory hash ---------------
__global__ void __launch_bounds__(256) k_move_warp(const int32_t* __restrict__ list, int64_t n,
                                                   MoveArgs p, int capmax) {
  extern __shared__ double smem[];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  double* vals = smem + (size_t)wid * capmax;
  int* keys = reinterpret_cast<int*>(smem + (size_t)nwarps * capmax) + (size_t)wid * capmax;
  for (int i = lane; i < capmax; i += 32) { keys[i] = -1; vals[i] = 0.; }
  __syncwarp();
  const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t task = warp; task < n; task += nw) {
    const int v = list[task];
    const int64_t s = p.off[v], eend = p.off[v + 1];
    const unsigned cap = min((unsigned)capmax, next_pow2_cap(eend - s)), mask = cap - 1;
    const int own = p.comm[v];
    const double ki = p.k[v], aown = p.a[own];
    for (int64_t base = s; base < eend; base += 32) {
      const int64_t j = base + lane;
      const bool ok = j < eend;
      int c = -1;
      double wt = 0.;
      if (ok) {
        const int u = p.adj[j];
        c = p.comm[u];
        wt = (u == v) ? 0. : p.w[j];
      }
      const unsigned peers = __match_any_sync(NIDO_FULL_MASK, c);
      const bool lead = ok && lane == __ffs(peers) - 1;
      const double e = fold_peers(peers, ok, wt);
      if (lead) table_add<false>(keys, vals, mask, c, e, p.err);
      __syncwarp();
    }
    double g = -NIDO_MAX_FLOAT, eown = 0.;
    unsigned long long tk = kNoKey;
    int cand = -1;
    for (unsigned i = lane; i < cap; i += 32) {
      const int cc = keys[i];
      if (cc < 0) continue;
      if (cc == own) {
        eown = vals[i];
      } else {
        const double gg = gain_of(vals[i], ki, p.a[cc], p.m);
        if (better(gg, (unsigned)cc, g, tk)) { g = gg; tk = (unsigned)cc; cand = cc; }
      }
    }
    eown = group_sum<32>(eown);
    if (p.tie == NIDO_TIE_NIDO) {
      const double gm = group_max<32>(g);
      g = -NIDO_MAX_FLOAT; tk = kNoKey; cand = -1;
      for (unsigned i = lane; i < cap; i += 32) {
        const int cc = keys[i];
        if (cc < 0 || cc == own) continue;
        if (gain_of(vals[i], ki, p.a[cc], p.m) != gm) continue;
        unsigned rank = 0;
        for (unsigned q = 0; q < cap; ++q) {
          const int kq = keys[q];
          rank += (kq >= 0 && kq < cc) ? 1u : 0u;
        }
        const unsigned long long key = nido_key(rank);
        if (key < tk) { tk = key; cand = cc; g = gm; }
      }
    }
    group_best<32>(g, tk, cand);
    if (lane == 0) {
      const double self = self_of(eown, ki, aown, p.m);
      const double tot = __dsub_rn(g, self);
      p.newc[v] = (cand >= 0 && tot > 0.) ? cand : own;
    }
    __syncwarp();
    for (unsigned i = lane; i < cap; i += 32) { keys[i] = -1; vals[i] = 0.; }
    __syncwarp();
  }
}

// Block-wide argmax: every thread gets the result.
__device__ void block_best(double& g, unsigned long long& tk, int& cand, double* sg,
                           unsigned long long* stk, int* sc) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  group_best<32>(g, tk, cand);
  if (lane == 0) { sg[wid] = g; stk[wid] = tk; sc[wid] = cand; }
  __syncthreads();
  if (wid == 0) {
    g = lane < nw ? sg[lane] : -NIDO_MAX_FLOAT;
    tk = lane < nw ? stk[lane] : kNoKey;
    cand = lane < nw ? sc[lane] : -1;
    group_best<32>(g, tk, cand);
    if (lane == 0) { sg[0] = g; stk[0] = tk; sc[0] = cand; }
  }
  __syncthreads();
  g = sg[0]; tk = stk[0]; cand = sc[0];
  __syncthreads();
}

__device__ double block_sum(double x, double* sx) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  x = group_sum<32>(x);
  if (lane == 0) sx[wid] = x;
  __syncthreads();
  double t = 0.;
  for (int i = 0; i < nw; ++i) t += sx[i];
  __syncthreads();
  return t;
}

__device__ double block_max(double x, double* sx) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  x = group_max<32>(x);
  if (lane == 0) sx[wid] = x;
  __syncthreads();
  double t = -NIDO_MAX_FLOAT;
  for (int i = 0; i < nw; ++i) t = fmax(t, sx[i]);
  __syncthreads();
  return t;
}

// ---- larger degrees: one CTA per vertex; table in shared memory or in a
// per-CTA global-memory slab (kept cleared between vertices) -------------------
template <bool kGlobal>
__global__ void __launch_bounds__(512) k_move_cta(const int32_t* __restrict__ list, int64_t n, MoveArgs p,
                                                  int capmax, int32_t* gkeys, double* gvals,
                                                  int64_t gslab) {
  extern __shared__ double smem[];
  __shared__ double sg[32];
  __shared__ unsigned long long stk[32];
  __shared__ int sc[32];
  int* keys;
  double* vals;
  if (kGlobal) {
    keys = gkeys + (size_t)blockIdx.x * gslab;
    vals = gvals + (size_t)blockIdx.x * gslab;
  } else {
    vals = smem;
    keys = reinterpret_cast<int*>(smem + capmax);
    for (int i = threadIdx.x; i < capmax; i += blockDim.x) { keys[i] = -1; vals[i] = 0.; }
    __syncthreads();
  }
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  for (int64_t task = blockIdx.x; task < n; task += gridDim.x) {
    const int v = list[task];
    const int64_t s = p.off[v], eend = p.off[v + 1];
    unsigned cap = next_pow2_cap(eend - s);
    if (!kGlobal) cap = min(cap, (unsigned)capmax);
    const unsigned mask = cap - 1;
    const int own = p.comm[v];
    const double ki = p.k[v], aown = p.a[own];
    for (int64_t base = s + (int64_t)wid * 32; base < eend; base += blockDim.x) {
      const int64_t j = base + lane;
      const bool ok = j < eend;
      int c = -1;
      double wt = 0.;
      if (ok) {
        const int u = p.adj[j];
        c = p.comm[u];
        wt = (u == v) ? 0. : p.w[j];
      }
      const unsigned peers = __match_any_sync(NIDO_FULL_MASK, c);
      const bool lead = ok && lane == __ffs(peers) - 1;
      const double e = fold_peers(peers, ok, wt);
      if (lead) table_add<true>(keys, vals, mask, c, e, p.err);
    }
    __syncthreads();
    double g = -NIDO_MAX_FLOAT, eown = 0.;
    unsigned long long tk = kNoKey;
    int cand = -1;
    for (unsigned i = threadIdx.x; i < cap; i += blockDim.x) {
      const int cc = keys[i];
      if (cc < 0) continue;
      if (cc == own) {
        eown = vals[i];
      } else {
        const double gg = gain_of(vals[i], ki, p.a[cc], p.m);
        if (better(gg, (unsigned)cc, g, tk)) { g = gg; tk = (unsigned)cc; cand = cc; }
      }
    }
    eown = block_sum(eown, sg);
    if (p.tie == NIDO_TIE_NIDO) {
      const double gm = block_max(g, sg);
      g = -NIDO_MAX_FLOAT; tk = kNoKey; cand = -1;
      for (unsigned i = threadIdx.x; i < cap; i += blockDim.x) {
        const int cc = keys[i];
        if (cc < 0 || cc == own) continue;
        if (gain_of(vals[i], ki, p.a[cc], p.m) != gm) continue;
        unsigned rank = 0;
        for (unsigned q = 0; q < cap; ++q) {
          const int kq = keys[q];
          rank += (kq >= 0 && kq < cc) ? 1u : 0u;
        }
        const unsigned long long key = nido_key(rank);
        if (key < tk) { tk = key; cand = cc; g = gm; }
      }
    }
    block_best(g, tk, cand, sg, stk, sc);
    if (threadIdx.x == 0) {
      const double self = self_of(eown, ki, aown, p.m);
      const double tot = __dsub_rn(g, self);
      p.newc[v] = (cand >= 0 && tot > 0.) ? cand : own;
    }
    for (unsigned i = threadIdx.x; i < cap; i += blockDim.x) { keys[i] = -1; vals[i] = 0.; }
    __syncthreads();
  }
}

inline unsigned grid_cap(int64_t blocks, int64_t cap) {
  if (blocks < 1) blocks = 1;
  return (unsigned)std::min<int64_t>(blocks, cap);
}

unsigned pow2_at_least(int64_t x) {
  unsigned c = 64;
  while ((int64_t)c < x) c <<= 1;
  return c;
}

}  // namespace

int launch_move(nido_graph_s* g, int batch, int tie, cudaEvent_t ev_start, cudaEvent_t ev_end) {
  if (batch < 0 || batch >= g->nbatches)
    return nido_set_error(NIDO_E_INVALID, "louvain_update: batch %d out of range [0,%d)", batch, g->nbatches);
  if (!g->bins_valid) NIDO_TRY(build_batches(g));
  cudaStream_t s = g->ctx->stream;
  const TierConfig& tc = g->ctx->tiers;
  MoveArgs p{g->off, g->adj, g->w, g->comm, g->k, g->a, g->newc, g->m, tie,
             reinterpret_cast<unsigned long long*>(g->dcount + 1)};
  const int nb = g->nbatches;
  if (ev_start) NIDO_CUDA_TRY(cudaEventRecord(ev_start, s));
  for (int t = 0; t < kNumTiers; ++t) {
    const int64_t b0 = g->tier_off[(size_t)t * nb + batch], b1 = g->tier_off[(size_t)t * nb + batch + 1];
    const int64_t n = b1 - b0;
    if (n <= 0) continue;
    const int32_t* list = g->perm + b0;
    switch (t) {
      case kTierG4:
        k_move_group<4><<<grid_cap((n + 63) / 64, kSMs * 16), 256, 0, s>>>(list, n, p);
        break;
      case kTierG8:
        k_move_group<8><<<grid_cap((n + 31) / 32, kSMs * 16), 256, 0, s>>>(list, n, p);
        break;
      case kTierG16:
        k_move_group<16><<<grid_cap((n + 15) / 16, kSMs * 16), 256, 0, s>>>(list, n, p);
        break;
      case kTierG32:
        k_move_group<32><<<grid_cap((n + 7) / 8, kSMs * 16), 256, 0, s>>>(list, n, p);
        break;
      case kTierWarp: {
        const int capmax = (int)pow2_at_least(2 * (int64_t)tc.warp_max);
        const int threads = 32 * tc.warps_per_cta;
        const size_t sm = (size_t)tc.warps_per_cta * capmax * (sizeof(double) + sizeof(int));
        NIDO_CUDA_TRY(cudaFuncSetAttribute(k_move_warp, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
        k_move_warp<<<grid_cap((n + tc.warps_per_cta - 1) / tc.warps_per_cta, kSMs * 8), threads, sm, s>>>(
            list, n, p, capmax);
        break;
      }
      case kTierCta: {
        const int capmax = (int)pow2_at_least(2 * (int64_t)tc.cta_max);
        const size_t sm = (size_t)capmax * (sizeof(double) + sizeof(int));
        NIDO_CUDA_TRY(cudaFuncSetAttribute(k_move_cta<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
        k_move_cta<false><<<grid_cap(n, kSMs * 2), tc.cta_threads, sm, s>>>(list, n, p, capmax, nullptr,
                                                                            nullptr, 0);
        break;
      }
      default: {
        if (g->gslabs <= 0 || (int64_t)pow2_at_least(2 * g->max_degree) > g->gslab)
          return nido_set_error(NIDO_E_INVALID, "global hash slabs not sized for degree %lld",
                                (long long)g->max_degree);
        k_move_cta<true><<<grid_cap(n, g->gslabs), tc.cta_threads, 0, s>>>(list, n, p, 0, g->gkeys,
                                                                          g->gvals, g->gslab);
        break;
      }
    }
    NIDO_LAUNCH_CHECK();
  }
  if (ev_end) NIDO_CUDA_TRY(cudaEventRecord(ev_end, s));
  return NIDO_OK;
}

}  // namespace nido
