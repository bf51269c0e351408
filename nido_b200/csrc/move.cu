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
#include <cooperative_groups.h>

#include <algorithm>
#include <mutex>

#include "common.cuh"
#include "engine.cuh"

namespace nido {
namespace {

namespace cg = cooperative_groups;

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
  // many-graph mode: graph of every vertex and mass of every graph (null for
  // one graph, whose mass is m)
  const int32_t* __restrict__ gid;
  const double* __restrict__ mg;
  // every weight integral and every vertex's sum of |w| below 2^31: the
  // shared-memory tables then add int32 (a native shared-memory atomic; the
  // FP64 one is several times slower) and every partial sum is exact, so
  // the e_vc read back are the FP64 sums bit for bit
  int ints;
  int64_t nv;  // vertices of the current graph (all graphs in many-graph mode)
};

// The mass of v's graph (kernels are instantiated per mode, so the
// one-graph kernels carry no graph-id lookup).
template <bool kMulti>
__device__ __forceinline__ double vertex_mass(const MoveArgs& p, int v) {
  return kMulti ? p.mg[p.gid[v]] : p.m;
}

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

// Warp argmax of (gain, smallest id) under the smallest-id rule (tk is the
// community id, kNoKey without a candidate) with three 32-bit warp
// reductions instead of a shuffle tree: the gain as an order-preserving
// 64-bit key (+0 for -0, which compares equal to it), then the smallest id
// among the lanes holding the largest gain.  The result is group_best<32>'s.
// Every lane of the warp must call it; all end with the result.
__device__ __forceinline__ void warp_best_id(double& g, unsigned long long& tk, int& cand) {
  const long long b = __double_as_longlong(g + 0.0);
  const unsigned long long key = b < 0 ? ~(unsigned long long)b : ((unsigned long long)b | 0x8000000000000000ull);
  const unsigned hi = (unsigned)(key >> 32), lo = (unsigned)key;
  const unsigned mh = __reduce_max_sync(NIDO_FULL_MASK, hi);
  const unsigned ml = __reduce_max_sync(NIDO_FULL_MASK, hi == mh ? lo : 0u);
  const bool top = hi == mh && lo == ml;
  const unsigned id = tk == kNoKey ? 0xFFFFFFFFu : (unsigned)tk;
  const unsigned mid = __reduce_min_sync(NIDO_FULL_MASK, top ? id : 0xFFFFFFFFu);
  const int src = __ffs(__ballot_sync(NIDO_FULL_MASK, top && id == mid)) - 1;
  g = __shfl_sync(NIDO_FULL_MASK, g, src);
  tk = __shfl_sync(NIDO_FULL_MASK, tk, src);
  cand = __shfl_sync(NIDO_FULL_MASK, cand, src);
}

// ---- degree <= 32: registers ---------------------------------------------------
// Six 256-thread blocks an SM (at most 40 registers a thread): the tier waits
// on its gathers, and more resident warps hide more of them.
template <int G, bool kMulti>
__global__ void __launch_bounds__(256, 6) k_move_group(const int32_t* __restrict__ list, int64_t n,
                                                    MoveArgs p) {
  constexpr int VPW = 32 / G;
  __shared__ int fold[256];  // integer phases: per-lane group sums
  const int lane = threadIdx.x & 31, gl = lane & (G - 1), gid = lane / G;
  const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t b = warp * VPW; b < n; b += nw * VPW) {
    const int64_t idx = b + gid;
    const bool vok = idx < n;
    int v = 0, own = -1;
    int64_t s = 0, d = 0;
    double ki = 0., aown = 0., m = p.m;
    if (vok) {
      v = list[idx];
      s = p.off[v];
      d = p.off[v + 1] - s;
      own = p.comm[v];
      ki = p.k[v];
      aown = p.a[own];
      m = vertex_mass<kMulti>(p, v);
    }
    const bool ok = gl < d;
    int c = -1;
    double wt = 0.;
    if (ok) {
      const int u = p.adj[s + gl];
      c = p.comm[u];
      wt = (u == v) ? 0. : p.w[s + gl];
    }
    // lanes of one vertex with equal communities: a 32-bit match where the
    // group index fits above the ids (invalid lanes, c = -1, may match across
    // groups; they add nothing), else a 64-bit one
    unsigned peers;
    if constexpr (G == 32) {
      peers = __match_any_sync(NIDO_FULL_MASK, (unsigned)c);
    } else if (p.nv <= (int64_t)1 << 29) {
      peers = __match_any_sync(NIDO_FULL_MASK, (unsigned)c | ((unsigned)gid << 29));
    } else {
      peers = __match_any_sync(NIDO_FULL_MASK, ((unsigned long long)(unsigned)gid << 32) | (unsigned)c);
    }
    const int leader = __ffs(peers) - 1;
    const bool lead = ok && lane == leader;
    double e;
    if (p.ints) {
      // integer weights: every lane adds its weight into its group leader's
      // shared-memory slot (int32 adds, exact in any order; equal addresses
      // are serialised by the atomic unit, not by instructions)
      fold[threadIdx.x] = 0;
      __syncwarp();
      if (ok) atomicAdd(&fold[(threadIdx.x & ~31) + leader], __double2int_rn(wt));
      __syncwarp();
      e = (double)fold[threadIdx.x];
    } else {
      e = fold_peers(peers, ok, wt);
    }
    double g = -NIDO_MAX_FLOAT, eown = 0.;
    unsigned long long tk = kNoKey;
    int cand = -1;
    if (lead) {
      if (c == own) {
        eown = e;
      } else {
        g = gain_of(e, ki, p.a[c], m);
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
    if (G == 32 && p.tie != NIDO_TIE_NIDO) warp_best_id(g, tk, cand);
    else group_best<G>(g, tk, cand);
    if (gl == 0 && vok) {
      const double self = self_of(eown, ki, aown, m);
      const double tot = __dsub_rn(g, self);
      p.newc[v] = (cand >= 0 && tot > 0.) ? cand : own;
    }
  }
}


// ---- hash tables --------------------------------------------------------------
// Open addressing over a power-of-two slot array.  New keys are appended to an
// occupied-slot list so that evaluation and clearing cost O(unique keys).
// Tables hold at least twice as many slots as the vertex has edges, so a free
// slot always exists; probing is still bounded by the table size, and a full
// table is reported through *err.
struct Table {
  int* keys;
  double* vals;  // FP64 values, or with ints the int32 sum in each slot's low word
  int* occ;
  int* nocc;
  unsigned mask;
  bool ints = false;  // shared-memory tables of integer-weight phases
  // integer-weight phases in shared memory: one 64-bit word a slot, the
  // community id in the high half (-1: empty) and the int32 sum in the low
  // half, so an insert and its first add are one compare-and-swap (keys and
  // vals are unused then)
  unsigned long long* slots = nullptr;
};

constexpr unsigned long long kEmptySlot = 0xFFFFFFFF00000000ull;
__device__ __forceinline__ int slot_key(unsigned long long x) { return (int)(x >> 32); }
__device__ __forceinline__ int slot_sum(unsigned long long x) { return (int)(unsigned)x; }

__device__ __forceinline__ int* int_slot(const Table& t, unsigned h) { return reinterpret_cast<int*>(t.vals + h); }

// e_vc of a slot of a shared-memory table
__device__ __forceinline__ double table_val(const Table& t, int slot) {
  if (t.slots) return (double)slot_sum(t.slots[slot]);
  return t.ints ? (double)*int_slot(t, (unsigned)slot) : t.vals[slot];
}

__device__ __forceinline__ int table_key(const Table& t, int slot) {
  return t.slots ? slot_key(t.slots[slot]) : t.keys[slot];
}

// Adds the integer w to key c's sum in a packed table, inserting c when
// absent (the insert carries w); returns the slot.  Sums are int32 adds on
// the slot's low half, exact in any order (integer weights, every vertex's
// sum of |w| below 2^31).
__device__ __forceinline__ int table_add_packed(const Table& t, int c, int w, bool& isnew, unsigned long long* err) {
  unsigned h = hash_slot(c, t.mask);
  volatile unsigned long long* vs = t.slots;
  isnew = false;
  for (unsigned probe = 0; probe <= t.mask; ++probe) {
    int k = slot_key(vs[h]);
    if (k == -1) {
      const unsigned long long mine = ((unsigned long long)(unsigned)c << 32) | (unsigned)w;
      const unsigned long long old = atomicCAS(&t.slots[h], kEmptySlot, mine);
      if (old == kEmptySlot) {
        isnew = true;
        return (int)h;
      }
      k = slot_key(old);
    }
    if (k == c) {
      atomicAdd(reinterpret_cast<int*>(&t.slots[h]), w);
      return (int)h;
    }
    h = (h + probe + 1) & t.mask;  // triangular steps: every slot once
  }
  atomicAdd(err, 1ull);
  return -1;
}

// Adds e to key c's value, inserting c when absent; returns the slot and
// whether this call inserted it.  Tables in global memory (kGlobal) go
// straight to the compare-and-swap, one L2 round trip per probe; shared-memory
// tables read the key first.
template <bool kAtomicVals, bool kGlobal = false>
__device__ __forceinline__ int table_add(const Table& t, int c, double e, bool& isnew, unsigned long long* err) {
  unsigned h = hash_slot(c, t.mask);
  volatile int* vk = t.keys;
  isnew = false;
  for (unsigned probe = 0; probe <= t.mask; ++probe) {
    if constexpr (kGlobal) {
      const int old = atomicCAS(&t.keys[h], -1, c);
      if (old == -1 || old == c) {
        isnew = old == -1;
        atomicAdd(&t.vals[h], e);
        return (int)h;
      }
      h = (h + 1) & t.mask;
      continue;
    }
    const int kk = vk[h];
    bool hit = kk == c;
    if (!hit && kk == -1) {
      const int old = atomicCAS(&t.keys[h], -1, c);
      isnew = old == -1;
      hit = isnew || old == c;
    }
    if (hit) {
      if (t.ints) {
        if (kAtomicVals) atomicAdd(int_slot(t, h), __double2int_rn(e));
        else *int_slot(t, h) += __double2int_rn(e);
      } else {
        if (kAtomicVals) atomicAdd(&t.vals[h], e);
        else t.vals[h] += e;
      }
      return (int)h;
    }
    h = (h + probe + 1) & t.mask;  // triangular steps: every slot once
  }
  atomicAdd(err, 1ull);
  return -1;
}

// Appends the slots this warp inserted to the occupied list with one atomic
// per warp.  Every lane of the warp must call it.
__device__ __forceinline__ void occ_append(const Table& t, bool isnew, int slot) {
  const unsigned nb = __ballot_sync(NIDO_FULL_MASK, isnew);
  if (nb == 0u || t.occ == nullptr) return;
  const int lane = threadIdx.x & 31, leader = __ffs(nb) - 1;
  int base = 0;
  if (lane == leader) base = atomicAdd(t.nocc, __popc(nb));
  base = __shfl_sync(NIDO_FULL_MASK, base, leader);
  if (isnew) t.occ[base + __popc(nb & lanemask_lt())] = slot;
}

// Edge ids and weights are read once per sweep: loaded without allocating in
// L1, which keeps L1 for the comm[u] and a[c] gathers (-2% on the move phase).
__device__ __forceinline__ int ld_stream(const int* q) {
  int v;
  asm("ld.global.L1::no_allocate.s32 %0, [%1];" : "=r"(v) : "l"(q));
  return v;
}
__device__ __forceinline__ double ld_stream(const double* q) {
  double v;
  asm("ld.global.L1::no_allocate.f64 %0, [%1];" : "=d"(v) : "l"(q));
  return v;
}

// smallest power of two >= max(64, 2d) (shared-memory tiers: d <= 2^30)
__device__ __forceinline__ unsigned next_pow2_cap(int64_t d) {
  const unsigned x = (unsigned)max((int64_t)64, 2 * min(d, (int64_t)1 << 30));
  return 1u << (32 - __clz(x - 1));
}

// Accumulate the edges [first, eend) of vertex v: the warp takes 32-edge
// chunks at first, first+stride, ...  kUnroll chunks are loaded (ids, weights,
// then the communities) before any is merged, so each warp keeps several
// dependent gathers in flight.  Chunks are merged in order.  Every lane of the
// warp takes part.
// The edges come from global memory, or (sadj non-null) from a copy of the
// vertex's ranges in shared memory: edge j at sadj[j - a0] and sw[j - w0].
template <bool kAtomicVals, int kUnroll, bool kGlobal = false>
__device__ __forceinline__ void accumulate_edges(const MoveArgs& p, int v, int64_t first, int64_t eend,
                                                 int64_t stride, const Table& t, const int32_t* sadj = nullptr,
                                                 const double* sw = nullptr, int64_t a0 = 0, int64_t w0 = 0) {
  const int lane = threadIdx.x & 31;
  for (int64_t base = first; base < eend; base += kUnroll * stride) {
    int u[kUnroll], c[kUnroll];
    double wt[kUnroll];
#pragma unroll
    for (int k = 0; k < kUnroll; ++k) {
      const int64_t j = base + k * stride + lane;
      u[k] = -1;
      wt[k] = 0.;
      if (j < eend) {
        if (sadj) {
          u[k] = sadj[j - a0];
          wt[k] = sw[j - w0];
        } else {
          u[k] = ld_stream(p.adj + j);
          wt[k] = ld_stream(p.w + j);
        }
      }
    }
#pragma unroll
    for (int k = 0; k < kUnroll; ++k) {
      c[k] = u[k] >= 0 ? p.comm[u[k]] : -1;
      if (u[k] == v) wt[k] = 0.;
    }
    if (!kGlobal && t.slots) {
      // packed integer table: every lane adds its own edge (native 32-bit
      // shared-memory atomics, exact in any order), no fold across lanes
#pragma unroll
      for (int k = 0; k < kUnroll; ++k) {
        const bool ok = u[k] >= 0;
        if (!__any_sync(NIDO_FULL_MASK, ok)) break;
        bool isnew = false;
        int slot = -1;
        if (ok) slot = table_add_packed(t, c[k], __double2int_rn(wt[k]), isnew, p.err);
        occ_append(t, isnew, slot);
        __syncwarp();
      }
      continue;
    }
#pragma unroll
    for (int k = 0; k < kUnroll; ++k) {
      const bool ok = u[k] >= 0;
      if (!__any_sync(NIDO_FULL_MASK, ok)) break;
      const unsigned peers = __match_any_sync(NIDO_FULL_MASK, c[k]);
      const bool lead = ok && lane == __ffs(peers) - 1;
      const double e = fold_peers(peers, ok, wt[k]);
      bool isnew = false;
      int slot = -1;
      if (lead) slot = table_add<kAtomicVals, kGlobal>(t, c[k], e, isnew, p.err);
      occ_append(t, isnew, slot);
      if (!kAtomicVals) __syncwarp();
    }
  }
}

// Hub segments (smallest-id rule): like accumulate_edges into a global
// table, but every lane keeps the compare-and-swaps of its kUnroll chunks in
// flight together instead of finishing one chunk's probe before the next.
// Equal communities within a chunk are still folded onto one lane first.
template <int kUnroll>
__device__ __forceinline__ void merge_edges_global(const MoveArgs& p, int v, int64_t first, int64_t eend,
                                                   int64_t stride, int* keys, double* vals, unsigned mask) {
  const int lane = threadIdx.x & 31;
  for (int64_t base = first; base < eend; base += kUnroll * stride) {
    int u[kUnroll], c[kUnroll];
    double wt[kUnroll];
    unsigned h[kUnroll];
#pragma unroll
    for (int k = 0; k < kUnroll; ++k) {
      const int64_t j = base + k * stride + lane;
      u[k] = -1;
      wt[k] = 0.;
      if (j < eend) {
        u[k] = p.adj[j];
        wt[k] = p.w[j];
      }
    }
#pragma unroll
    for (int k = 0; k < kUnroll; ++k) {
      c[k] = u[k] >= 0 ? p.comm[u[k]] : -1;
      if (u[k] == v) wt[k] = 0.;
    }
    unsigned pending = 0u;
#pragma unroll
    for (int k = 0; k < kUnroll; ++k) {
      const bool ok = u[k] >= 0;
      const unsigned peers = __match_any_sync(NIDO_FULL_MASK, c[k]);
      wt[k] = fold_peers(peers, ok, wt[k]);
      if (ok && lane == __ffs(peers) - 1) pending |= 1u << k;
      h[k] = ok ? hash_slot(c[k], mask) : 0u;
    }
    for (unsigned probe = 0; pending != 0u && probe <= mask; ++probe) {
      int old[kUnroll];
#pragma unroll
      for (int k = 0; k < kUnroll; ++k) old[k] = (pending >> k & 1u) ? atomicCAS(&keys[h[k]], -1, c[k]) : 0;
#pragma unroll
      for (int k = 0; k < kUnroll; ++k) {
        if (!(pending >> k & 1u)) continue;
        if (old[k] == -1 || old[k] == c[k]) {
          atomicAdd(&vals[h[k]], wt[k]);
          pending &= ~(1u << k);
        } else {
          h[k] = (h[k] + 1) & mask;
        }
      }
    }
    if (pending != 0u) atomicAdd(p.err, 1ull);
  }
}

// merge_edges_global for packed integer tables (integer-weight phases): one
// 64-bit slot per community (id, int32 sum), so a new community is one
// compare-and-swap that also carries its first sum, an existing one one
// 32-bit add.  Equal communities within a chunk are still folded onto one
// lane first (fewer L2 atomics).
template <int kUnroll>
__device__ __forceinline__ void merge_edges_packed(const MoveArgs& p, int v, int64_t first, int64_t eend,
                                                   int64_t stride, unsigned long long* slots, unsigned mask) {
  const int lane = threadIdx.x & 31;
  for (int64_t base = first; base < eend; base += kUnroll * stride) {
    int u[kUnroll], c[kUnroll], x[kUnroll];
    double wt[kUnroll];
    unsigned h[kUnroll];
#pragma unroll
    for (int k = 0; k < kUnroll; ++k) {
      const int64_t j = base + k * stride + lane;
      u[k] = -1;
      wt[k] = 0.;
      if (j < eend) {
        u[k] = p.adj[j];
        wt[k] = p.w[j];
      }
    }
#pragma unroll
    for (int k = 0; k < kUnroll; ++k) {
      c[k] = u[k] >= 0 ? p.comm[u[k]] : -1;
      if (u[k] == v) wt[k] = 0.;
    }
    unsigned pending = 0u;
#pragma unroll
    for (int k = 0; k < kUnroll; ++k) {
      const bool ok = u[k] >= 0;
      const unsigned peers = __match_any_sync(NIDO_FULL_MASK, c[k]);
      x[k] = __double2int_rn(fold_peers(peers, ok, wt[k]));
      if (ok && lane == __ffs(peers) - 1) pending |= 1u << k;
      h[k] = ok ? hash_slot(c[k], mask) : 0u;
    }
    for (unsigned probe = 0; pending != 0u && probe <= mask; ++probe) {
      unsigned long long old[kUnroll];
#pragma unroll
      for (int k = 0; k < kUnroll; ++k)
        old[k] = (pending >> k & 1u)
                     ? atomicCAS(&slots[h[k]], kEmptySlot, ((unsigned long long)(unsigned)c[k] << 32) | (unsigned)x[k])
                     : 0ull;
#pragma unroll
      for (int k = 0; k < kUnroll; ++k) {
        if (!(pending >> k & 1u)) continue;
        if (old[k] == kEmptySlot) {
          pending &= ~(1u << k);
        } else if (slot_key(old[k]) == c[k]) {
          atomicAdd(reinterpret_cast<int*>(&slots[h[k]]), x[k]);
          pending &= ~(1u << k);
        } else {
          h[k] = (h[k] + 1) & mask;
        }
      }
    }
    if (pending != 0u) atomicAdd(p.err, 1ull);
  }
}

// Scan entries i = t0, t0+step, ... of the occupied list (or of all slots when
// occ is null): e_own and the best (gain, tie key, community) of this thread.
// Entries are taken four at a time so that their a_c gathers are in flight
// together.
__device__ __forceinline__ void scan_entries(const MoveArgs& p, double m, const Table& t, int n, int t0, int step,
                                             int own, double ki, bool cg, double& eown, double& g,
                                             unsigned long long& tk, int& cand) {
  constexpr int U = 4;
  for (int i = t0; i < n; i += U * step) {
    int cc[U];
    double val[U], ac[U];
#pragma unroll
    for (int k = 0; k < U; ++k) {
      const int ii = i + k * step;
      cc[k] = -1;
      if (ii < n) {
        const int slot = t.occ ? t.occ[ii] : ii;
        if (t.slots) {
          const unsigned long long x = t.slots[slot];
          cc[k] = slot_key(x);
          val[k] = (double)slot_sum(x);
        } else {
          cc[k] = cg ? __ldcg(&t.keys[slot]) : t.keys[slot];
          val[k] = cg ? __ldcg(&t.vals[slot]) : table_val(t, slot);
        }
      }
    }
#pragma unroll
    for (int k = 0; k < U; ++k) ac[k] = (cc[k] >= 0 && cc[k] != own) ? p.a[cc[k]] : 0.;
#pragma unroll
    for (int k = 0; k < U; ++k) {
      if (cc[k] < 0) continue;
      if (cc[k] == own) {
        eown = val[k];
      } else {
        const double gg = gain_of(val[k], ki, ac[k], m);
        if (better(gg, (unsigned)cc[k], g, tk)) { g = gg; tk = (unsigned)cc[k]; cand = cc[k]; }
      }
    }
  }
}


// The reference's tie rule over the same entries: among communities whose
// gain equals gm, the smallest (bitrev3(rank mod 8), rank), where rank counts
// the vertex's neighbour communities with a smaller id.
__device__ __forceinline__ void nido_tie_entries(const MoveArgs& p, double m, const Table& t, int n, int t0, int step,
                                                 int own, double ki, double gm, bool cg, double& g,
                                                 unsigned long long& tk, int& cand) {
  g = -NIDO_MAX_FLOAT; tk = kNoKey; cand = -1;
  for (int i = t0; i < n; i += step) {
    const int slot = t.occ ? t.occ[i] : i;
    const int cc = cg ? __ldcg(&t.keys[slot]) : table_key(t, slot);
    if (cc < 0 || cc == own) continue;
    const double val = cg ? __ldcg(&t.vals[slot]) : table_val(t, slot);
    if (gain_of(val, ki, p.a[cc], m) != gm) continue;
    unsigned rank = 0;
    for (int q = 0; q < n; ++q) {
      const int sq = t.occ ? t.occ[q] : q;
      const int kq = cg ? __ldcg(&t.keys[sq]) : table_key(t, sq);
      rank += (kq >= 0 && kq < cc) ? 1u : 0u;
    }
    const unsigned long long key = nido_key(rank);
    if (key < tk) { tk = key; cand = cc; g = gm; }
  }
}

__device__ __forceinline__ void decide(const MoveArgs& p, double m, int v, int own, double ki, double aown, double eown,
                                       double g, int cand) {
  const double self = self_of(eown, ki, aown, m);
  const double tot = __dsub_rn(g, self);
  p.newc[v] = (cand >= 0 && tot > 0.) ? cand : own;
}

// ---- 32 < degree <= 256: one warp per vertex, table in shared memory -----------
// Shared memory of the tables: FP64 tables hold 8-byte values, 4-byte keys
// and a 4-byte occupied list (16 bytes a slot); packed integer tables 8-byte
// slots and the occupied list (12 bytes a slot).
constexpr size_t table_bytes(int slots, bool ints) { return (size_t)slots * (ints ? 12 : 16); }

// Five 256-thread blocks an SM (at most 48 registers a thread; a few spill).
template <int kCap, bool kMulti, bool kInts>
__global__ void __launch_bounds__(256, 5) k_move_warp(const int32_t* __restrict__ list, int64_t n, MoveArgs p) {
  extern __shared__ double smem[];
  __shared__ int nocc_s[8];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  Table t;
  if constexpr (kInts) {
    t.slots = reinterpret_cast<unsigned long long*>(smem) + (size_t)wid * kCap;
    t.keys = nullptr;
    t.vals = nullptr;
    t.occ = reinterpret_cast<int*>(smem + 8 * kCap) + (size_t)wid * kCap;
    for (int i = lane; i < kCap; i += 32) t.slots[i] = kEmptySlot;
  } else {
    t.vals = smem + (size_t)wid * kCap;
    t.keys = reinterpret_cast<int*>(smem + 8 * kCap) + (size_t)wid * 2 * kCap;
    t.occ = t.keys + kCap;
    for (int i = lane; i < kCap; i += 32) { t.keys[i] = -1; t.vals[i] = 0.; }
  }
  t.nocc = &nocc_s[wid];
  t.ints = kInts;
  if (lane == 0) *t.nocc = 0;
  __syncwarp();
  const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t task = warp; task < n; task += nw) {
    const int v = list[task];
    const int64_t s = p.off[v], eend = p.off[v + 1];
    t.mask = min((unsigned)kCap, next_pow2_cap(eend - s)) - 1;
    const int own = p.comm[v];
    const double ki = p.k[v], aown = p.a[own];
    accumulate_edges<false, 4>(p, v, s, eend, 32, t);
    const int nu = *t.nocc;
    double g = -NIDO_MAX_FLOAT, eown = 0.;
    unsigned long long tk = kNoKey;
    int cand = -1;
    const double m = vertex_mass<kMulti>(p, v);
    scan_entries(p, m, t, nu, lane, 32, own, ki, false, eown, g, tk, cand);
    eown = group_sum<32>(eown);
    if (p.tie == NIDO_TIE_NIDO) {
      const double gm = group_max<32>(g);
      nido_tie_entries(p, m, t, nu, lane, 32, own, ki, gm, false, g, tk, cand);
      group_best<32>(g, tk, cand);
    } else {
      warp_best_id(g, tk, cand);
    }
    if (lane == 0) decide(p, m, v, own, ki, aown, eown, g, cand);
    __syncwarp();
    for (int i = lane; i < nu; i += 32) {
      const int slot = t.occ[i];
      if constexpr (kInts) {
        t.slots[slot] = kEmptySlot;
      } else {
        t.keys[slot] = -1;
        t.vals[slot] = 0.;
      }
    }
    if (lane == 0) *t.nocc = 0;
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

// Evaluate a filled table with the whole block and write newc[v].
__device__ __forceinline__ void block_evaluate(const MoveArgs& p, double m, const Table& t, int n, bool cg, int v, int own,
                                               double ki, double aown, double* sg, unsigned long long* stk,
                                               int* sc) {
  double g = -NIDO_MAX_FLOAT, eown = 0.;
  unsigned long long tk = kNoKey;
  int cand = -1;
  scan_entries(p, m, t, n, threadIdx.x, blockDim.x, own, ki, cg, eown, g, tk, cand);
  if (p.tie == NIDO_TIE_NIDO) {
    eown = block_sum(eown, sg);
    const double gm = block_max(g, sg);
    nido_tie_entries(p, m, t, n, threadIdx.x, blockDim.x, own, ki, gm, cg, g, tk, cand);
  }
  // one reduction for the best entry and e_own (e_own is nonzero in one
  // thread at most, so its sum is exact in any order)
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  if (p.tie != NIDO_TIE_NIDO) {
    eown = group_sum<32>(eown);
    warp_best_id(g, tk, cand);
  } else {
    group_best<32>(g, tk, cand);
  }
  __shared__ double se[32];
  if (lane == 0) { sg[wid] = g; stk[wid] = tk; sc[wid] = cand; se[wid] = eown; }
  __syncthreads();
  if (wid == 0) {
    g = lane < nw ? sg[lane] : -NIDO_MAX_FLOAT;
    tk = lane < nw ? stk[lane] : kNoKey;
    cand = lane < nw ? sc[lane] : -1;
    double e2 = lane < nw ? se[lane] : 0.;
    if (p.tie != NIDO_TIE_NIDO) warp_best_id(g, tk, cand);
    else group_best<32>(g, tk, cand);
    e2 = group_sum<32>(e2);
    if (lane == 0) decide(p, m, v, own, ki, aown, p.tie == NIDO_TIE_NIDO ? eown : e2, g, cand);
  }
}

// ---- staged adjacency: 1-D bulk copies (TMA) of a vertex's edge ranges --------
// One thread copies the next vertex's ids and weights from this GPU's global
// memory into shared memory with cp.async.bulk, completed on an mbarrier,
// while the block still evaluates the current vertex; the block then reads
// the edges from shared memory.  Copies start and end on 16-byte boundaries:
// the id range is widened to multiples of 4 ids and the weight range to
// multiples of 2 weights (the edge arrays carry 4 spare entries so the widened
// end stays inside them).  No multicast.
__device__ __forceinline__ unsigned smem_u32(const void* ptr) { return (unsigned)__cvta_generic_to_shared(ptr); }

__device__ __forceinline__ void mbar_init(unsigned long long* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(unsigned long long* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(unsigned long long* bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred P;\n mbarrier.try_wait.parity.shared::cta.b64 P, [%1], %2;\n selp.u32 %0, 1, 0, P;\n}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

__device__ __forceinline__ unsigned long long gtimer_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// bounded wait: gives up (false) after kMbarTries attempts or about a second,
// whichever comes first, instead of spinning forever; the caller counts the
// failure in p.err
constexpr int kMbarTries = 1 << 20;
constexpr unsigned long long kMbarWaitNs = 1000000000ull;
__device__ __forceinline__ bool mbar_wait(unsigned long long* bar, unsigned parity) {
  const unsigned long long t0 = gtimer_ns();
  for (int i = 0; i < kMbarTries; ++i) {
    if (mbar_try_wait(bar, parity)) return true;
    if ((i & 255) == 255 && gtimer_ns() - t0 > kMbarWaitNs) return false;
  }
  return false;
}

// Self-check of the bounded waits: one thread waits on an mbarrier that
// expects an arrival nobody makes.  The wait must give up and the kernel
// report it (out[0] = 1, out[1] = milliseconds waited), leaving the context
// usable.
__global__ void k_check_bounded_wait(int32_t* out) {
  __shared__ unsigned long long bar;
  if (threadIdx.x != 0) return;
  mbar_init(&bar, 1);
  const unsigned long long t0 = gtimer_ns();
  const bool done = mbar_wait(&bar, 0);
  out[0] = done ? 0 : 1;
  out[1] = (int32_t)min((gtimer_ns() - t0) / 1000000ull, 1ull << 30);
}

__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, unsigned bytes, unsigned long long* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}

// shared memory of one staged vertex of degree <= kDeg: ids then weights
template <int kDeg>
struct Stage {
  static constexpr int kIds = kDeg + 8;     // widened by up to 3 ids each side
  static constexpr int kWts = kDeg + 4;     // widened by up to 1 weight each side
  static constexpr size_t kBytes = (size_t)kIds * 4 + (size_t)kWts * 8;
};

// Thread 0: copy the edges [s, e) into the stage (ids at sadj, weights at
// sw) on bar; *a0 / *w0 receive the first id / weight index held.
__device__ __forceinline__ void stage_edges(const MoveArgs& p, int64_t s, int64_t e, int32_t* sadj, double* sw,
                                            unsigned long long* bar, int64_t* a0, int64_t* w0) {
  const int64_t ia = s & ~(int64_t)3, ib = (e + 3) & ~(int64_t)3;
  const int64_t wa = s & ~(int64_t)1, wb = (e + 1) & ~(int64_t)1;
  const unsigned bi = (unsigned)(4 * (ib - ia)), bw = (unsigned)(8 * (wb - wa));
  *a0 = ia;
  *w0 = wa;
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // earlier reads of the stage come first
  mbar_arrive_expect_tx(bar, bi + bw);
  if (bi) bulk_g2s(sadj, p.adj + ia, bi, bar);
  if (bw) bulk_g2s(sw, p.w + wa, bw, bar);
}

// ---- 256 < degree <= 2048: one CTA per vertex, table in shared memory ----------
// kOcc: keep a list of occupied slots (16 bytes a slot) so evaluation and
// clearing touch only used slots; without it (12 bytes a slot, for the
// largest FP64 table) both walk the vertex's whole table.  Packed integer
// tables (kInts) always keep the list: 12 bytes a slot with it.
// kStageDeg > 0: the tier's vertices (degree <= kStageDeg) have their edges
// staged in shared memory behind the table (see stage_edges), one vertex
// ahead: the copy of vertex i+1 runs while vertex i is evaluated.
// Resident CTAs an SM: ten of 128 threads or five of 256 (at most 48 registers
// a thread), else the 64-register fill of 1024 threads.
template <int kThreads, int kCap, bool kMulti, bool kInts, bool kOcc = true, int kStageDeg = 0>
__global__ void __launch_bounds__(kThreads, kThreads == 128 ? 10 : (kThreads == 256 ? 5 : 1024 / kThreads)) k_move_cta(const int32_t* __restrict__ list, int64_t n, MoveArgs p) {
  constexpr bool kList = kOcc || kInts;
  constexpr bool kStaged = kStageDeg > 0;
  extern __shared__ __align__(128) double smem[];
  __shared__ double sg[32];
  __shared__ unsigned long long stk[32];
  __shared__ int sc[32];
  __shared__ int nocc_s;
  __shared__ unsigned long long stage_bar;
  __shared__ long long stage_off[2];  // first id and weight index held by the stage
  int32_t* sadj = nullptr;
  double* sw = nullptr;
  if constexpr (kStaged) {
    char* st = reinterpret_cast<char*>(smem) + table_bytes(kCap, kInts);
    sadj = reinterpret_cast<int32_t*>(st);
    sw = reinterpret_cast<double*>(st + (size_t)Stage<kStageDeg>::kIds * 4);
    if (threadIdx.x == 0) {
      mbar_init(&stage_bar, 1);
      if (blockIdx.x < n) {  // the first vertex's edges start on their way at once
        const int v0 = list[blockIdx.x];
        int64_t a0, w0;
        stage_edges(p, p.off[v0], p.off[v0 + 1], sadj, sw, &stage_bar, &a0, &w0);
        stage_off[0] = a0;
        stage_off[1] = w0;
      }
    }
  }
  unsigned stage_parity = 0;
  Table t;
  if constexpr (kInts) {
    t.slots = reinterpret_cast<unsigned long long*>(smem);
    t.keys = nullptr;
    t.vals = nullptr;
    t.occ = reinterpret_cast<int*>(smem + kCap);
    for (int i = threadIdx.x; i < kCap; i += kThreads) t.slots[i] = kEmptySlot;
  } else {
    t.vals = smem;
    t.keys = reinterpret_cast<int*>(smem + kCap);
    t.occ = kOcc ? t.keys + kCap : nullptr;
    for (int i = threadIdx.x; i < kCap; i += kThreads) { t.keys[i] = -1; t.vals[i] = 0.; }
  }
  t.nocc = &nocc_s;
  t.ints = kInts;
  if (threadIdx.x == 0) nocc_s = 0;
  __syncthreads();
  const int wid = threadIdx.x >> 5;
  // The next vertex's header (id, offsets, community, k, a_own) is loaded
  // while the current one is evaluated, so its dependent round trips overlap.
  int64_t task = blockIdx.x;
  int v = 0, own = 0;
  int64_t s = 0, eend = 0;
  double ki = 0., aown = 0.;
  if (task < n) {
    v = list[task];
    s = p.off[v];
    eend = p.off[v + 1];
    own = p.comm[v];
    ki = p.k[v];
    aown = p.a[own];
  }
  for (; task < n; task += gridDim.x) {
    const int64_t nt = task + gridDim.x;
    const int vn = nt < n ? list[nt] : 0;
    int64_t sn = 0, en = 0;
    if (nt < n) {
      sn = p.off[vn];
      en = p.off[vn + 1];
    }
    t.mask = min((unsigned)kCap, next_pow2_cap(eend - s)) - 1;
    if constexpr (kStaged) {
      if (!mbar_wait(&stage_bar, stage_parity)) atomicAdd(p.err, 1ull);
      stage_parity ^= 1u;
      accumulate_edges<true, 4>(p, v, s + (int64_t)wid * 32, eend, kThreads, t, sadj, sw, stage_off[0],
                                stage_off[1]);
    } else {
      accumulate_edges<true, 4>(p, v, s + (int64_t)wid * 32, eend, kThreads, t);
    }
    __syncthreads();
    if constexpr (kStaged) {
      // every thread has read the stage (and stage_off): the next vertex's
      // edges go into it while this one is evaluated
      if (threadIdx.x == 0 && nt < n) {
        int64_t a0, w0;
        stage_edges(p, sn, en, sadj, sw, &stage_bar, &a0, &w0);
        stage_off[0] = a0;
        stage_off[1] = w0;
      }
    }
    const int nu = kList ? nocc_s : (int)(t.mask + 1);
    int ownn = 0;
    double kin = 0.;
    if (nt < n) {
      ownn = p.comm[vn];
      kin = p.k[vn];
    }
    // block_evaluate ends with a barrier that every thread reaches after
    // reading nu, so the count can be reset right after it
    block_evaluate(p, vertex_mass<kMulti>(p, v), t, nu, false, v, own, ki, aown, sg, stk, sc);
    if (threadIdx.x == 0) nocc_s = 0;
    const double aownn = nt < n ? p.a[ownn] : 0.;
    for (int i = threadIdx.x; i < nu; i += kThreads) {
      const int slot = kList ? t.occ[i] : i;
      if constexpr (kInts) {
        t.slots[slot] = kEmptySlot;
      } else {
        t.keys[slot] = -1;
        t.vals[slot] = 0.;
      }
    }
    __syncthreads();
    v = vn;
    s = sn;
    eend = en;
    own = ownn;
    ki = kin;
    aown = aownn;
  }
}

// ---- degree > 2048: hub vertices split into segments of kHubSeg edges ----------
// Each CTA takes one (hub, segment) item and merges its edges into the hub's
// table in global memory (L2-resident); the CTA that finishes a hub's last
// segment (an atomic ticket; nobody waits) evaluates and clears the table.
constexpr int kHubThreads = 256;

template <bool kMulti>
__global__ void __launch_bounds__(kHubThreads) k_move_hub(const int2* __restrict__ items, int64_t n,
                                                          const int32_t* __restrict__ hub_v,
                                                          const int64_t* __restrict__ hub_toff,
                                                          const int32_t* __restrict__ hub_cap,
                                                          const int32_t* __restrict__ hub_nseg,
                                                          int32_t* __restrict__ hub_done, int32_t* gkeys,
                                                          double* gvals, MoveArgs p) {
  __shared__ double sg[32];
  __shared__ unsigned long long stk[32];
  __shared__ int sc[32];
  __shared__ int last_s;
  const int wid = threadIdx.x >> 5;
  for (int64_t it = blockIdx.x; it < n; it += gridDim.x) {
    const int2 item = items[it];
    const int h = item.x;
    const int v = hub_v[h];
    Table t;
    t.keys = gkeys + hub_toff[h];
    t.vals = gvals + hub_toff[h];
    t.occ = nullptr;
    t.nocc = nullptr;
    t.mask = (unsigned)hub_cap[h] - 1;
    const int64_t s = p.off[v], eend = p.off[v + 1];
    const int64_t s0 = s + (int64_t)item.y * kHubSeg;
    const int64_t s1 = min(eend, s0 + kHubSeg);
    accumulate_edges<true, 2, true>(p, v, s0 + (int64_t)wid * 32, s1, kHubThreads, t);
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) last_s = atomicAdd(&hub_done[h], 1) == hub_nseg[h] - 1;
    __syncthreads();
    if (last_s) {
      __threadfence();
      const int own = p.comm[v];
      const double ki = p.k[v], aown = p.a[own];
      block_evaluate(p, vertex_mass<kMulti>(p, v), t, (int)(t.mask + 1), true, v, own, ki, aown, sg, stk, sc);
      for (unsigned i = threadIdx.x; i <= t.mask; i += kHubThreads) {
        t.keys[i] = -1;
        t.vals[i] = 0.;
      }
      if (threadIdx.x == 0) hub_done[h] = 0;
    }
    __syncthreads();
  }
}

// Fast path for the smallest-id rule: segments only merge (k_hub_insert),
// then every kHubSlice-slot slice of a table is scanned and cleared by its
// own CTA (k_hub_slices), and one warp per hub combines the slice results
// (k_hub_combine).  The reference's tie rule needs ranks over the whole
// table and uses k_move_hub instead.
constexpr int kHubSlice = 4096;
// The table slots of one wave of hubs come from the graph's tier
// configuration (default 4M slots: 48 MB of keys and values, which leaves
// room in the 126 MB L2 for the streamed adjacency and the gathers).

__global__ void __launch_bounds__(kHubThreads) k_hub_insert(const int2* __restrict__ items, int64_t n,
                                                            const int32_t* __restrict__ hub_v,
                                                            const int64_t* __restrict__ hub_toff,
                                                            const int32_t* __restrict__ hub_cap, int32_t* gkeys,
                                                            double* gvals, MoveArgs p) {
  const int wid = threadIdx.x >> 5;
  for (int64_t it = blockIdx.x; it < n; it += gridDim.x) {
    const int2 item = items[it];
    const int h = item.x;
    const int v = hub_v[h];
    const int64_t s = p.off[v], eend = p.off[v + 1];
    const int64_t s0 = s + (int64_t)item.y * kHubSeg;
    merge_edges_global<4>(p, v, s0 + (int64_t)wid * 32, min(eend, s0 + kHubSeg), kHubThreads, gkeys + hub_toff[h],
                          gvals + hub_toff[h], (unsigned)hub_cap[h] - 1);
  }
}

struct SliceResult {
  double g;
  double eown;
  unsigned long long tk;
  int cand;
  int pad;
};

// Slice y of hub x covers slots [y*kHubSlice, (y+1)*kHubSlice) of the hub's
// table, read and cleared in order.  (A per-hub list of occupied slots,
// appended during the merge, measured twice as slow on R-MAT scale 22: the
// hub tables are mostly full and the list's counter is one contended
// address per hub.)
template <bool kMulti>
__global__ void __launch_bounds__(kHubThreads) k_hub_slices(const int2* __restrict__ slices, int64_t n,
                                                            const int32_t* __restrict__ hub_v,
                                                            const int64_t* __restrict__ hub_toff,
                                                            const int32_t* __restrict__ hub_cap, int32_t* gkeys,
                                                            double* gvals, MoveArgs p,
                                                            SliceResult* __restrict__ res) {
  __shared__ double sg[32];
  __shared__ unsigned long long stk[32];
  __shared__ int sc[32];
  for (int64_t it = blockIdx.x; it < n; it += gridDim.x) {
    const int2 sl = slices[it];
    const int len = min(kHubSlice, hub_cap[sl.x] - sl.y * kHubSlice);
    const int v = hub_v[sl.x];
    int* keys = gkeys + hub_toff[sl.x] + (int64_t)sl.y * kHubSlice;
    double* vals = gvals + hub_toff[sl.x] + (int64_t)sl.y * kHubSlice;
    const int own = p.comm[v];
    const double ki = p.k[v];
    const double m = vertex_mass<kMulti>(p, v);
    double g = -NIDO_MAX_FLOAT, eown = 0.;
    unsigned long long tk = kNoKey;
    int cand = -1;
    // four slots per thread at a time, so their a_c gathers are in flight together
    constexpr int U = 4;
    for (int i0 = threadIdx.x; i0 < len; i0 += U * kHubThreads) {
      int cc[U];
      double val[U], ac[U];
#pragma unroll
      for (int k = 0; k < U; ++k) {
        const int i = i0 + k * kHubThreads;
        cc[k] = -1;
        if (i < len) {
          cc[k] = keys[i];
          val[k] = vals[i];
        }
      }
#pragma unroll
      for (int k = 0; k < U; ++k) ac[k] = (cc[k] >= 0 && cc[k] != own) ? p.a[cc[k]] : 0.;
#pragma unroll
      for (int k = 0; k < U; ++k) {
        if (cc[k] < 0) continue;
        const int i = i0 + k * kHubThreads;
        keys[i] = -1;
        vals[i] = 0.;
        if (cc[k] == own) {
          eown = val[k];
        } else {
          const double gg = gain_of(val[k], ki, ac[k], m);
          if (better(gg, (unsigned)cc[k], g, tk)) { g = gg; tk = (unsigned)cc[k]; cand = cc[k]; }
        }
      }
    }
    eown = block_sum(eown, sg);
    block_best(g, tk, cand, sg, stk, sc);
    if (threadIdx.x == 0) res[it] = SliceResult{g, eown, tk, cand, 0};
  }
}

// k_hub_insert / k_hub_slices on packed integer tables
__global__ void __launch_bounds__(kHubThreads) k_hub_insert_packed(const int2* __restrict__ items, int64_t n,
                                                                   const int32_t* __restrict__ hub_v,
                                                                   const int64_t* __restrict__ hub_toff,
                                                                   const int32_t* __restrict__ hub_cap,
                                                                   unsigned long long* gslots, MoveArgs p) {
  const int wid = threadIdx.x >> 5;
  for (int64_t it = blockIdx.x; it < n; it += gridDim.x) {
    const int2 item = items[it];
    const int h = item.x;
    const int v = hub_v[h];
    const int64_t s = p.off[v], eend = p.off[v + 1];
    const int64_t s0 = s + (int64_t)item.y * kHubSeg;
    merge_edges_packed<4>(p, v, s0 + (int64_t)wid * 32, min(eend, s0 + kHubSeg), kHubThreads, gslots + hub_toff[h],
                          (unsigned)hub_cap[h] - 1);
  }
}

template <bool kMulti>
__global__ void __launch_bounds__(kHubThreads) k_hub_slices_packed(const int2* __restrict__ slices, int64_t n,
                                                                   const int32_t* __restrict__ hub_v,
                                                                   const int64_t* __restrict__ hub_toff,
                                                                   const int32_t* __restrict__ hub_cap,
                                                                   unsigned long long* gslots, MoveArgs p,
                                                                   SliceResult* __restrict__ res) {
  __shared__ double sg[32];
  __shared__ unsigned long long stk[32];
  __shared__ int sc[32];
  for (int64_t it = blockIdx.x; it < n; it += gridDim.x) {
    const int2 sl = slices[it];
    const int len = min(kHubSlice, hub_cap[sl.x] - sl.y * kHubSlice);
    const int v = hub_v[sl.x];
    unsigned long long* slots = gslots + hub_toff[sl.x] + (int64_t)sl.y * kHubSlice;
    const int own = p.comm[v];
    const double ki = p.k[v];
    const double m = vertex_mass<kMulti>(p, v);
    double g = -NIDO_MAX_FLOAT, eown = 0.;
    unsigned long long tk = kNoKey;
    int cand = -1;
    constexpr int U = 4;
    for (int i0 = threadIdx.x; i0 < len; i0 += U * kHubThreads) {
      int cc[U];
      double val[U], ac[U];
#pragma unroll
      for (int k = 0; k < U; ++k) {
        const int i = i0 + k * kHubThreads;
        cc[k] = -1;
        if (i < len) {
          const unsigned long long x = __ldcg(&slots[i]);
          cc[k] = slot_key(x);
          val[k] = (double)slot_sum(x);
        }
      }
#pragma unroll
      for (int k = 0; k < U; ++k) ac[k] = (cc[k] >= 0 && cc[k] != own) ? p.a[cc[k]] : 0.;
#pragma unroll
      for (int k = 0; k < U; ++k) {
        if (cc[k] < 0) continue;
        slots[i0 + k * kHubThreads] = kEmptySlot;
        if (cc[k] == own) {
          eown = val[k];
        } else {
          const double gg = gain_of(val[k], ki, ac[k], m);
          if (better(gg, (unsigned)cc[k], g, tk)) { g = gg; tk = (unsigned)cc[k]; cand = cc[k]; }
        }
      }
    }
    eown = block_sum(eown, sg);
    block_best(g, tk, cand, sg, stk, sc);
    if (threadIdx.x == 0) res[it] = SliceResult{g, eown, tk, cand, 0};
  }
}

__global__ void k_fill_u64(unsigned long long* __restrict__ x, int64_t n, unsigned long long val) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    x[i] = val;
}

template <bool kMulti>
__global__ void k_hub_combine(int64_t nh, const int32_t* __restrict__ hub_v, const int64_t* __restrict__ slice_first,
                              const SliceResult* __restrict__ res, MoveArgs p) {
  const int lane = threadIdx.x & 31;
  const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t h = warp; h < nh; h += nw) {
    const int64_t r0 = slice_first[h], r1 = slice_first[h + 1];
    if (r1 == r0) continue;  // hub of another batch
    double g = -NIDO_MAX_FLOAT, eown = 0.;
    unsigned long long tk = kNoKey;
    int cand = -1;
    for (int64_t r = r0 + lane; r < r1; r += 32) {
      const SliceResult x = res[r];
      eown += x.eown;
      if (better(x.g, x.tk, g, tk)) { g = x.g; tk = x.tk; cand = x.cand; }
    }
    eown = group_sum<32>(eown);
    group_best<32>(g, tk, cand);
    if (lane == 0) {
      const int v = hub_v[h];
      const int own = p.comm[v];
      decide(p, vertex_mass<kMulti>(p, v), v, own, p.k[v], p.a[own], eown, g, cand);
    }
  }
}

// ---- hubs in thread-block clusters (integer-weight phases) ---------------------
// One cluster of kCtas CTAs per hub: the hub's table spans the clusters'
// shared memory, kClSlots slots in each CTA, so every insert is a
// distributed-shared-memory access instead of an L2 round trip.  The edges
// are spread over all warps of the cluster; after a cluster barrier each CTA
// evaluates (and clears) its own slots, the per-CTA bests meet in rank 0's
// shared memory, and after a second barrier rank 0 decides.  Sums are int32
// (integer weights, every vertex's sum of |w| below 2^31), so the shared
// atomics are native 32-bit ones and exact; the smallest-id tie rule picks
// the same entry in any order of evaluation.
constexpr int kClThreads = 1024;
constexpr int kClSlots = 16384;   // 192 KB of keys and values per CTA
constexpr int kClusterBins = 4;   // clusters of 2, 4, 8 and 16 CTAs

constexpr int64_t cluster_max_degree(int bin) { return (int64_t)(2 << bin) * kClSlots * 3 / 4; }

// cluster size bin of a hub of degree d (-1: more than a 16-CTA table holds)
inline int cluster_bin(int64_t d) {
  for (int b = 0; b < kClusterBins; ++b)
    if (d <= cluster_max_degree(b)) return b;
  return -1;
}

// whether clusters of each size can be resident on this GPU (set once per
// process by move_init_attributes; unlaunchable bins keep hubs on the
// global-memory path)
bool g_cluster_ok[kClusterBins] = {false, false, false, false};
inline bool cluster_launchable(int bin) { return bin >= 0 && g_cluster_ok[bin]; }

__device__ __forceinline__ void cluster_add(cg::cluster_group& cl, int* keys, double* vals, unsigned mask, int c,
                                            int x, unsigned long long* err) {
  unsigned h = hash_slot(c, mask);
  for (unsigned probe = 0; probe <= mask; ++probe) {
    const unsigned owner = h / kClSlots, loc = h % kClSlots;
    int* kp = cl.map_shared_rank(keys, owner) + loc;
    const int kk = *reinterpret_cast<volatile int*>(kp);
    bool hit = kk == c;
    if (!hit && kk == -1) {
      const int old = atomicCAS(kp, -1, c);
      hit = old == -1 || old == c;
    }
    if (hit) {
      atomicAdd(reinterpret_cast<int*>(cl.map_shared_rank(vals, owner) + loc), x);
      return;
    }
    h = (h + 1) & mask;
  }
  atomicAdd(err, 1ull);
}

template <int kCtas, bool kMulti>
__global__ void __launch_bounds__(kClThreads, 1) k_move_cluster(const int32_t* __restrict__ list, int64_t n,
                                                                MoveArgs p) {
  cg::cluster_group cluster = cg::this_cluster();
  extern __shared__ double smem[];
  double* vals = smem;                                    // int32 sums in the low words
  int* keys = reinterpret_cast<int*>(smem + kClSlots);
  __shared__ double sg[32], se[32];
  __shared__ unsigned long long stk[32];
  __shared__ int sc[32];
  __shared__ double rg[kCtas], re[kCtas];                 // the ranks' bests, in rank 0
  __shared__ unsigned long long rtk[kCtas];
  __shared__ int rc[kCtas];
  constexpr unsigned kMask = (unsigned)kCtas * kClSlots - 1;
  constexpr int kWarps = kCtas * (kClThreads / 32);
  const unsigned rank = cluster.block_rank();
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int gw = (int)rank * (kClThreads / 32) + wid;
  for (int i = threadIdx.x; i < kClSlots; i += kClThreads) { keys[i] = -1; vals[i] = 0.; }
  cluster.sync();
  const int64_t ncl = gridDim.x / kCtas;
  for (int64_t task = blockIdx.x / kCtas; task < n; task += ncl) {
    const int v = list[task];
    const int64_t s = p.off[v], e = p.off[v + 1];
    for (int64_t base = s + (int64_t)gw * 32; base < e; base += (int64_t)4 * kWarps * 32) {
      int u[4], c[4];
      double wt[4];
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        const int64_t j = base + (int64_t)k * kWarps * 32 + lane;
        u[k] = -1;
        wt[k] = 0.;
        if (j < e) {
          u[k] = p.adj[j];
          wt[k] = p.w[j];
        }
      }
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        c[k] = u[k] >= 0 ? p.comm[u[k]] : -1;
        if (u[k] == v) wt[k] = 0.;
      }
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        const bool ok = u[k] >= 0;
        if (!__any_sync(NIDO_FULL_MASK, ok)) break;
        const unsigned peers = __match_any_sync(NIDO_FULL_MASK, c[k]);
        const double x = fold_peers(peers, ok, wt[k]);
        if (ok && lane == __ffs(peers) - 1) cluster_add(cluster, keys, vals, kMask, c[k], __double2int_rn(x), p.err);
      }
    }
    cluster.sync();  // every insert of this hub is in place
    const int own = p.comm[v];
    const double ki = p.k[v], aown = p.a[own], m = vertex_mass<kMulti>(p, v);
    double g = -NIDO_MAX_FLOAT, eown = 0.;
    unsigned long long tk = kNoKey;
    int cand = -1;
    for (int i0 = threadIdx.x; i0 < kClSlots; i0 += 4 * kClThreads) {
      int cc[4];
      double val[4], ac[4];
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        const int i = i0 + k * kClThreads;
        cc[k] = keys[i];
        val[k] = (double)*reinterpret_cast<const int*>(vals + i);
        if (cc[k] >= 0) {  // this thread is the slot's only reader
          keys[i] = -1;
          vals[i] = 0.;
        }
      }
#pragma unroll
      for (int k = 0; k < 4; ++k) ac[k] = (cc[k] >= 0 && cc[k] != own) ? p.a[cc[k]] : 0.;
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        if (cc[k] < 0) continue;
        if (cc[k] == own) {
          eown = val[k];
        } else {
          const double gg = gain_of(val[k], ki, ac[k], m);
          if (better(gg, (unsigned)cc[k], g, tk)) { g = gg; tk = (unsigned)cc[k]; cand = cc[k]; }
        }
      }
    }
    eown = group_sum<32>(eown);  // nonzero in one lane of the cluster at most: exact
    group_best<32>(g, tk, cand);
    if (lane == 0) { sg[wid] = g; stk[wid] = tk; sc[wid] = cand; se[wid] = eown; }
    __syncthreads();
    if (wid == 0) {
      g = sg[lane];
      tk = stk[lane];
      cand = sc[lane];
      double e2 = se[lane];
      group_best<32>(g, tk, cand);
      e2 = group_sum<32>(e2);
      if (lane == 0) {
        *cluster.map_shared_rank(&rg[rank], 0) = g;
        *cluster.map_shared_rank(&rtk[rank], 0) = tk;
        *cluster.map_shared_rank(&rc[rank], 0) = cand;
        *cluster.map_shared_rank(&re[rank], 0) = e2;
      }
    }
    cluster.sync();  // the ranks' bests are in rank 0; every slot is clear again
    if (rank == 0 && threadIdx.x == 0) {
      double bg = -NIDO_MAX_FLOAT, be = 0.;
      unsigned long long bt = kNoKey;
      int bc = -1;
      for (int r = 0; r < kCtas; ++r) {
        be += re[r];
        if (better(rg[r], rtk[r], bg, bt)) { bg = rg[r]; bt = rtk[r]; bc = rc[r]; }
      }
      decide(p, m, v, own, ki, aown, be, bg, bc);
    }
  }
}

__global__ void k_hub_degrees(const int32_t* __restrict__ list, int64_t n, const int64_t* __restrict__ off,
                              int64_t* __restrict__ out) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const int v = list[i];
    out[2 * i] = v;
    out[2 * i + 1] = off[v + 1] - off[v];
  }
}

inline unsigned grid_cap(int64_t blocks, int64_t cap) {
  if (blocks < 1) blocks = 1;
  return (unsigned)std::min<int64_t>(blocks, cap);
}

template <typename T>
int ensure(nido_graph_s* g, T** p, int64_t* cap, int64_t n) {
  if (n <= *cap) return NIDO_OK;
  raw_free(g->ctx, *p);
  *p = nullptr;
  *cap = 0;
  const int64_t m = std::max<int64_t>(n, 1024);
  NIDO_CUDA_TRY(raw_alloc(g->ctx, (void**)p, sizeof(T) * (size_t)m));
  *cap = m;
  return NIDO_OK;
}

}  // namespace

// Per-phase plan of the hub tier: table offsets, segment items per batch.
int plan_hubs(nido_graph_s* g) {
  const int nb = g->nbatches;
  const int64_t h0 = g->tier_off[(size_t)kTierHub * nb], h1 = g->tier_off[(size_t)(kTierHub + 1) * nb];
  const int64_t nh = h1 - h0;
  g->hub_waves.clear();
  g->hub_wave_off.assign(nb + 1, 0);
  g->nhubs = nh;
  g->hub_nitems = 0;
  g->hub_cl_ok = false;
  g->hub_cl_off.assign((size_t)nb * kClusterBins + 1, 0);
  if (nh == 0) return NIDO_OK;
  cudaStream_t s = g->ctx->stream;
  Arena ar(g->scratch, g->scratch_bytes);
  int64_t* vd = ar.take<int64_t>(2 * nh);
  if (!vd) return nido_set_error(NIDO_E_NOMEM, "scratch arena too small (hubs)");
  k_hub_degrees<<<grid_cap((nh + 255) / 256, kSMs * 4), 256, 0, s>>>(g->perm + h0, nh, g->off, vd);
  NIDO_LAUNCH_CHECK();
  std::vector<int64_t> h(2 * nh);
  NIDO_CUDA_TRY(cudaMemcpyAsync(h.data(), vd, sizeof(int64_t) * 2 * nh, cudaMemcpyDeviceToHost, s));
  NIDO_CUDA_TRY(cudaStreamSynchronize(s));
  std::vector<int32_t> hv(nh), hcap(nh), hseg(nh);
  std::vector<int64_t> htoff(nh);
  std::vector<int2> items;
  for (int64_t i = 0; i < nh; ++i) {
    const int64_t d = h[2 * i + 1];
    const int64_t u = std::min<int64_t>(d, g->nv);
    int64_t cap = 64;
    while (cap < 2 * u) cap <<= 1;
    hv[i] = (int32_t)h[2 * i];
    hcap[i] = (int32_t)cap;
    hseg[i] = (int32_t)((d + kHubSeg - 1) / kHubSeg);
  }
  // Hubs are listed by batch within the tier.  Each batch's hubs are cut into
  // waves whose tables together hold at most cfg.hub_wave_slots slots (so they stay
  // in L2); table offsets are relative to the wave, and every wave reuses the
  // same region because its slice scan clears the tables.  Items and table
  // slices of a hub follow one another.
  std::vector<int2> slices;
  std::vector<int64_t> sfirst(nh + 1, 0);
  std::vector<int64_t> ifirst(nh + 1, 0);
  g->hub_waves.clear();
  g->hub_wave_off.assign(nb + 1, 0);
  int64_t maxslots = 0;
  for (int b = 0; b < nb; ++b) {
    const int64_t a0 = g->tier_off[(size_t)kTierHub * nb + b] - h0;
    const int64_t a1 = g->tier_off[(size_t)kTierHub * nb + b + 1] - h0;
    int64_t wslots = 0;
    for (int64_t i = a0; i < a1; ++i) {
      if (i == a0 || wslots + hcap[i] > g->cfg.hub_wave_slots) {
        g->hub_waves.push_back({(int64_t)items.size(), 0, (int64_t)slices.size(), 0, i, 0});
        wslots = 0;
      }
      htoff[i] = wslots;
      wslots += hcap[i];
      maxslots = std::max(maxslots, wslots);
      ifirst[i] = (int64_t)items.size();
      for (int sgi = 0; sgi < hseg[i]; ++sgi) items.push_back(make_int2((int)i, sgi));
      sfirst[i] = (int64_t)slices.size();
      for (int sl = 0; sl * kHubSlice < hcap[i]; ++sl) slices.push_back(make_int2((int)i, sl));
      sfirst[i + 1] = (int64_t)slices.size();
      nido_graph_s::HubWave& w = g->hub_waves.back();
      w.i1 = (int64_t)items.size();
      w.s1 = (int64_t)slices.size();
      w.h1 = i + 1;
    }
    g->hub_wave_off[b + 1] = (int64_t)g->hub_waves.size();
  }
  ifirst[nh] = (int64_t)items.size();
  g->hub_nitems = (int64_t)items.size();
  const int64_t toff = maxslots;
  g->gslab_need = toff;
  NIDO_TRY(ensure(g, &g->hub_v, &g->hub_cap_hubs_v, nh));
  NIDO_TRY(ensure(g, &g->hub_capv, &g->hub_cap_hubs_c, nh));
  NIDO_TRY(ensure(g, &g->hub_nseg, &g->hub_cap_hubs_s, nh));
  NIDO_TRY(ensure(g, &g->hub_toff, &g->hub_cap_hubs_t, nh));
  NIDO_TRY(ensure(g, &g->hub_done, &g->hub_cap_hubs_d, nh));
  NIDO_TRY(ensure(g, &g->hub_items, &g->hub_cap_items, (int64_t)items.size()));
  NIDO_TRY(ensure(g, &g->hub_slices, &g->hub_cap_slices, (int64_t)slices.size()));
  NIDO_TRY(ensure(g, &g->hub_slice_first, &g->hub_cap_first, nh + 1));
  NIDO_TRY(ensure(g, &g->hub_res, &g->hub_cap_res, (int64_t)(slices.size() * sizeof(SliceResult))));
  NIDO_TRY(ensure(g, &g->hub_item_first, &g->hub_cap_ifirst, nh + 1));
  NIDO_TRY(ensure(g, &g->hub_part, &g->hub_cap_part, (int64_t)items.size()));
  NIDO_CUDA_TRY(cudaMemcpyAsync(g->hub_item_first, ifirst.data(), sizeof(int64_t) * (nh + 1), cudaMemcpyHostToDevice, s));
  NIDO_CUDA_TRY(cudaMemcpyAsync(g->hub_slices, slices.data(), sizeof(int2) * slices.size(), cudaMemcpyHostToDevice, s));
  NIDO_CUDA_TRY(cudaMemcpyAsync(g->hub_slice_first, sfirst.data(), sizeof(int64_t) * (nh + 1), cudaMemcpyHostToDevice, s));
  if (toff > g->gslab) {
    raw_free(g->ctx, g->gkeys);
    raw_free(g->ctx, g->gvals);
    g->gkeys = nullptr;
    g->gvals = nullptr;
    g->gslab = 0;
    NIDO_CUDA_TRY(raw_alloc(g->ctx, (void**)&g->gkeys, sizeof(int32_t) * (size_t)toff));
    NIDO_CUDA_TRY(raw_alloc(g->ctx, (void**)&g->gvals, sizeof(double) * (size_t)toff));
    NIDO_CUDA_TRY(cudaMemsetAsync(g->gkeys, 0xff, sizeof(int32_t) * (size_t)toff, s));
    NIDO_CUDA_TRY(cudaMemsetAsync(g->gvals, 0, sizeof(double) * (size_t)toff, s));
    g->gslab = toff;
  }
  // packed tables for integer-weight phases (smallest-id rule), kept empty
  // between waves by the slice scans like the FP64 ones
  if (g->int_weights && toff > g->gslab_packed) {
    raw_free(g->ctx, g->gpacked);
    g->gpacked = nullptr;
    g->gslab_packed = 0;
    NIDO_CUDA_TRY(raw_alloc(g->ctx, (void**)&g->gpacked, sizeof(unsigned long long) * (size_t)toff));
    k_fill_u64<<<grid_cap((toff + 255) / 256, kSMs * 8), 256, 0, s>>>(g->gpacked, toff, kEmptySlot);
    NIDO_LAUNCH_CHECK();
    g->gslab_packed = toff;
  }
  NIDO_CUDA_TRY(cudaMemcpyAsync(g->hub_v, hv.data(), sizeof(int32_t) * nh, cudaMemcpyHostToDevice, s));
  NIDO_CUDA_TRY(cudaMemcpyAsync(g->hub_capv, hcap.data(), sizeof(int32_t) * nh, cudaMemcpyHostToDevice, s));
  NIDO_CUDA_TRY(cudaMemcpyAsync(g->hub_nseg, hseg.data(), sizeof(int32_t) * nh, cudaMemcpyHostToDevice, s));
  NIDO_CUDA_TRY(cudaMemcpyAsync(g->hub_toff, htoff.data(), sizeof(int64_t) * nh, cudaMemcpyHostToDevice, s));
  NIDO_CUDA_TRY(cudaMemsetAsync(g->hub_done, 0, sizeof(int32_t) * nh, s));
  NIDO_CUDA_TRY(cudaMemcpyAsync(g->hub_items, items.data(), sizeof(int2) * items.size(), cudaMemcpyHostToDevice, s));
  // cluster bins of every batch's hubs (the tier is used when all fit)
  std::vector<int32_t> clv;
  clv.reserve((size_t)nh);
  bool cl_ok = g->cfg.hub_clusters;
  for (int b = 0; b < nb && cl_ok; ++b) {
    const int64_t a0 = g->tier_off[(size_t)kTierHub * nb + b] - h0;
    const int64_t a1 = g->tier_off[(size_t)kTierHub * nb + b + 1] - h0;
    for (int bin = 0; bin < kClusterBins; ++bin) {
      g->hub_cl_off[(size_t)b * kClusterBins + bin] = (int64_t)clv.size();
      for (int64_t i = a0; i < a1; ++i)
        if (cluster_bin(h[2 * i + 1]) == bin) clv.push_back(hv[i]);
    }
    for (int64_t i = a0; i < a1; ++i)
      if (cluster_bin(h[2 * i + 1]) < 0 || !cluster_launchable(cluster_bin(h[2 * i + 1]))) cl_ok = false;
  }
  g->hub_cl_off[(size_t)nb * kClusterBins] = (int64_t)clv.size();
  if (cl_ok && !clv.empty()) {
    NIDO_TRY(ensure(g, &g->hub_cl_v, &g->hub_cap_cl, (int64_t)clv.size()));
    NIDO_CUDA_TRY(cudaMemcpyAsync(g->hub_cl_v, clv.data(), sizeof(int32_t) * clv.size(), cudaMemcpyHostToDevice, s));
    g->hub_cl_ok = true;
  }
  NIDO_CUDA_TRY(cudaStreamSynchronize(s));  // the host vectors go out of scope
  return NIDO_OK;
}

namespace {
constexpr int kWarpCap = 256;     // warp tier: degree <= 128
// threads per CTA and table slots of the CTA tiers
constexpr int kCtaSThreads = 128;
constexpr int kCtaMThreads = 256;
constexpr int kCtaLThreads = 256;
constexpr int kCtaSCap = 1024;
constexpr int kCtaMCap = 2048;
constexpr int kCtaLCap = 4096;
// CTA-S and CTA-M with staged edges: table plus one vertex's widened ranges
constexpr size_t smem_s_staged(bool ints) { return table_bytes(kCtaSCap, ints) + Stage<kCtaSMaxDeg>::kBytes; }
constexpr size_t smem_m_staged(bool ints) { return table_bytes(kCtaMCap, ints) + Stage<kCtaMMaxDeg>::kBytes; }
constexpr int kCtaXAThreads = 512;
constexpr int kCtaXACap = 8192;   // 512-thread CTA-XA tier, two CTAs an SM (occupied list in integer phases)
constexpr int kCtaXCap = 16384;   // 1024-thread CTA-XL tier (occupied list in integer phases)

template <typename K>
int set_smem(K kernel, size_t bytes) {
  NIDO_CUDA_TRY(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
  return NIDO_OK;
}
}  // namespace

namespace {
// CTAs of every move kernel that fit on the GPU at once (SMs x resident CTAs
// per SM, from the occupancy calculator): grid-stride kernels launched with
// more would leave a partial wave at the end.
struct Resident {
  int64_t g4 = kSMs, g8 = kSMs, g16 = kSMs, g32 = kSMs, warp = kSMs, ctas = kSMs, ctam = kSMs, ctal = kSMs,
          ctaxa = kSMs, ctax = kSMs, hubmv = kSMs, hubins = kSMs, hubsl = kSMs, ctas_st = kSMs, ctam_st = kSMs;
};
Resident g_resident[2][2];  // [many graphs][integer tables]

template <typename K>
int64_t resident(K kernel, int threads, size_t smem, int sms) {
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, smem) != cudaSuccess) {
    cudaGetLastError();
    per_sm = 1;
  }
  return (int64_t)std::max(per_sm, 1) * sms;
}

template <bool kMulti, bool kInts>
int set_smem_mode() {
  NIDO_TRY(set_smem(k_move_warp<kWarpCap, kMulti, kInts>, 8 * table_bytes(kWarpCap, kInts)));
  NIDO_TRY(set_smem(k_move_cta<kCtaSThreads, kCtaSCap, kMulti, kInts>, table_bytes(kCtaSCap, kInts)));
  NIDO_TRY(set_smem(k_move_cta<kCtaMThreads, kCtaMCap, kMulti, kInts>, table_bytes(kCtaMCap, kInts)));
  NIDO_TRY(set_smem(k_move_cta<kCtaSThreads, kCtaSCap, kMulti, kInts, true, kCtaSMaxDeg>, smem_s_staged(kInts)));
  NIDO_TRY(set_smem(k_move_cta<kCtaMThreads, kCtaMCap, kMulti, kInts, true, kCtaMMaxDeg>, smem_m_staged(kInts)));
  NIDO_TRY(set_smem(k_move_cta<kCtaLThreads, kCtaLCap, kMulti, kInts>, table_bytes(kCtaLCap, kInts)));
  NIDO_TRY(set_smem(k_move_cta<kCtaXAThreads, kCtaXACap, kMulti, kInts, false>, (size_t)kCtaXACap * 12));
  NIDO_TRY(set_smem(k_move_cta<1024, kCtaXCap, kMulti, kInts, false>, (size_t)kCtaXCap * 12));
  int dev = 0, sms = kSMs;
  NIDO_CUDA_TRY(cudaGetDevice(&dev));
  NIDO_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  static std::mutex mu;  // contexts may be created from several threads
  std::lock_guard<std::mutex> lk(mu);
  Resident& R = g_resident[kMulti ? 1 : 0][kInts ? 1 : 0];
  R.g4 = resident(k_move_group<4, kMulti>, 256, 0, sms);
  R.g8 = resident(k_move_group<8, kMulti>, 256, 0, sms);
  R.g16 = resident(k_move_group<16, kMulti>, 256, 0, sms);
  R.g32 = resident(k_move_group<32, kMulti>, 256, 0, sms);
  R.warp = resident(k_move_warp<kWarpCap, kMulti, kInts>, 256, 8 * table_bytes(kWarpCap, kInts), sms);
  R.ctas = resident(k_move_cta<kCtaSThreads, kCtaSCap, kMulti, kInts>, kCtaSThreads, table_bytes(kCtaSCap, kInts), sms);
  R.ctam = resident(k_move_cta<kCtaMThreads, kCtaMCap, kMulti, kInts>, kCtaMThreads, table_bytes(kCtaMCap, kInts), sms);
  R.ctas_st = resident(k_move_cta<kCtaSThreads, kCtaSCap, kMulti, kInts, true, kCtaSMaxDeg>, kCtaSThreads,
                       smem_s_staged(kInts), sms);
  R.ctam_st = resident(k_move_cta<kCtaMThreads, kCtaMCap, kMulti, kInts, true, kCtaMMaxDeg>, kCtaMThreads,
                       smem_m_staged(kInts), sms);
  R.ctal = resident(k_move_cta<kCtaLThreads, kCtaLCap, kMulti, kInts>, kCtaLThreads, table_bytes(kCtaLCap, kInts), sms);
  R.ctaxa = resident(k_move_cta<kCtaXAThreads, kCtaXACap, kMulti, kInts, false>, kCtaXAThreads,
                     (size_t)kCtaXACap * 12, sms);
  R.ctax = resident(k_move_cta<1024, kCtaXCap, kMulti, kInts, false>, 1024, (size_t)kCtaXCap * 12, sms);
  R.hubmv = resident(k_move_hub<kMulti>, kHubThreads, 0, sms);
  R.hubins = resident(k_hub_insert, kHubThreads, 0, sms);
  R.hubsl = resident(k_hub_slices<kMulti>, kHubThreads, 0, sms);
  return NIDO_OK;
}

int64_t g_cluster_max[kClusterBins] = {0, 0, 0, 0};  // clusters resident on the GPU at once

template <int kCtas>
cudaLaunchConfig_t cluster_config(int64_t clusters, cudaStream_t s, cudaLaunchAttribute* attr) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)(clusters * kCtas), 1, 1);
  cfg.blockDim = dim3(kClThreads, 1, 1);
  cfg.dynamicSmemBytes = (size_t)kClSlots * 12;
  cfg.stream = s;
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = kCtas;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cfg;
}

// shared memory and cluster-size attributes of one cluster kernel, and how
// many of its clusters fit on the GPU (0: none, the bin stays off)
template <int kCtas, bool kMulti>
int64_t cluster_setup() {
  auto k = k_move_cluster<kCtas, kMulti>;
  if (cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, kClSlots * 12) != cudaSuccess ||
      (kCtas > 8 && cudaFuncSetAttribute(k, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess)) {
    cudaGetLastError();
    return 0;
  }
  cudaLaunchAttribute attr[1];
  cudaLaunchConfig_t cfg = cluster_config<kCtas>(1, nullptr, attr);
  int n = 0;
  if (cudaOccupancyMaxActiveClusters(&n, k, &cfg) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return n;
}

int cluster_init() {
  const int64_t m[kClusterBins] = {std::min(cluster_setup<2, false>(), cluster_setup<2, true>()),
                                   std::min(cluster_setup<4, false>(), cluster_setup<4, true>()),
                                   std::min(cluster_setup<8, false>(), cluster_setup<8, true>()),
                                   std::min(cluster_setup<16, false>(), cluster_setup<16, true>())};
  for (int b = 0; b < kClusterBins; ++b) {
    g_cluster_max[b] = m[b];
    g_cluster_ok[b] = m[b] > 0;
  }
  return NIDO_OK;
}

template <int kCtas, bool kMulti>
int launch_cluster_bin(int bin, const int32_t* list, int64_t n, const MoveArgs& p, cudaStream_t s) {
  cudaLaunchAttribute attr[1];
  cudaLaunchConfig_t cfg = cluster_config<kCtas>(std::min<int64_t>(n, g_cluster_max[bin]), s, attr);
  NIDO_CUDA_TRY(cudaLaunchKernelEx(&cfg, k_move_cluster<kCtas, kMulti>, list, n, p));
  return NIDO_OK;
}

// the hubs of one batch on clusters of 2, 4, 8 and 16 CTAs by degree
template <bool kMulti>
int launch_clusters(nido_graph_s* g, int batch, const MoveArgs& p, cudaStream_t s) {
  for (int bin = 0; bin < kClusterBins; ++bin) {
    const int64_t c0 = g->hub_cl_off[(size_t)batch * kClusterBins + bin];
    const int64_t c1 = g->hub_cl_off[(size_t)batch * kClusterBins + bin + 1];
    if (c1 <= c0) continue;
    const int32_t* list = g->hub_cl_v + c0;
    switch (bin) {
      case 0: NIDO_TRY((launch_cluster_bin<2, kMulti>(bin, list, c1 - c0, p, s))); break;
      case 1: NIDO_TRY((launch_cluster_bin<4, kMulti>(bin, list, c1 - c0, p, s))); break;
      case 2: NIDO_TRY((launch_cluster_bin<8, kMulti>(bin, list, c1 - c0, p, s))); break;
      default: NIDO_TRY((launch_cluster_bin<16, kMulti>(bin, list, c1 - c0, p, s))); break;
    }
  }
  return NIDO_OK;
}

// the tier kernels of one batch; kMulti: many graphs (per-vertex mass).  The
// tiers cover disjoint vertices and only read comm and a, so they run on
// three streams: the hub chain and the CTA tiers on the context's side
// streams, the rest on its stream, joined before the function returns.
template <bool kMulti, bool kInts>
int launch_tiers(nido_graph_s* g, int batch, int tie, const MoveArgs& p) {
  nido_ctx_s* ctx = g->ctx;
  const Resident& R = g_resident[kMulti ? 1 : 0][kInts ? 1 : 0];
  const cudaStream_t main_s = ctx->stream;
  NIDO_CUDA_TRY(cudaEventRecord(ctx->fork_ev, main_s));
  for (int i = 0; i < 2; ++i) NIDO_CUDA_TRY(cudaStreamWaitEvent(ctx->aux[i], ctx->fork_ev, 0));
  const int nb = g->nbatches;
  // edges staged in shared memory by bulk copies from this GPU's memory (a
  // tier option; never for edges kept in mapped host memory)
  const bool staged = g->cfg.staged_edges && !g->host_edges;
  for (int t = kNumTiers - 1; t >= 0; --t) {  // longest chains first
    const cudaStream_t s = t == kTierHub ? ctx->aux[0] : (t >= kTierCtaS ? ctx->aux[1] : main_s);
    const int64_t b0 = g->tier_off[(size_t)t * nb + batch], b1 = g->tier_off[(size_t)t * nb + batch + 1];
    const int64_t n = b1 - b0;
    if (n <= 0) continue;
    const int32_t* list = g->perm + b0;
    switch (t) {
      case kTierG4:
        k_move_group<4, kMulti><<<grid_cap((n + 63) / 64, R.g4), 256, 0, s>>>(list, n, p);
        break;
      case kTierG8:
        k_move_group<8, kMulti><<<grid_cap((n + 31) / 32, R.g8), 256, 0, s>>>(list, n, p);
        break;
      case kTierG16:
        k_move_group<16, kMulti><<<grid_cap((n + 15) / 16, R.g16), 256, 0, s>>>(list, n, p);
        break;
      case kTierG32:
        k_move_group<32, kMulti><<<grid_cap((n + 7) / 8, R.g32), 256, 0, s>>>(list, n, p);
        break;
      case kTierWarp:
        k_move_warp<kWarpCap, kMulti, kInts><<<grid_cap((n + 7) / 8, R.warp), 256, 8 * table_bytes(kWarpCap, kInts), s>>>(
            list, n, p);
        break;
      case kTierCtaS:
        if (staged)
          k_move_cta<kCtaSThreads, kCtaSCap, kMulti, kInts, true, kCtaSMaxDeg>
              <<<grid_cap(n, R.ctas_st), kCtaSThreads, smem_s_staged(kInts), s>>>(list, n, p);
        else
          k_move_cta<kCtaSThreads, kCtaSCap, kMulti, kInts>
              <<<grid_cap(n, R.ctas), kCtaSThreads, table_bytes(kCtaSCap, kInts), s>>>(list, n, p);
        break;
      case kTierCtaM:
        if (staged)
          k_move_cta<kCtaMThreads, kCtaMCap, kMulti, kInts, true, kCtaMMaxDeg>
              <<<grid_cap(n, R.ctam_st), kCtaMThreads, smem_m_staged(kInts), s>>>(list, n, p);
        else
          k_move_cta<kCtaMThreads, kCtaMCap, kMulti, kInts>
              <<<grid_cap(n, R.ctam), kCtaMThreads, table_bytes(kCtaMCap, kInts), s>>>(list, n, p);
        break;
      case kTierCtaL:
        k_move_cta<kCtaLThreads, kCtaLCap, kMulti, kInts><<<grid_cap(n, R.ctal), kCtaLThreads, table_bytes(kCtaLCap, kInts), s>>>(list, n, p);
        break;
      case kTierCtaXA:
        k_move_cta<kCtaXAThreads, kCtaXACap, kMulti, kInts, false>
            <<<grid_cap(n, R.ctaxa), kCtaXAThreads, (size_t)kCtaXACap * 12, s>>>(list, n, p);
        break;
      case kTierCtaX:
        k_move_cta<1024, kCtaXCap, kMulti, kInts, false><<<grid_cap(n, R.ctax), 1024, (size_t)kCtaXCap * 12, s>>>(list, n, p);
        break;
      default: {
        if constexpr (kInts) {
          // integer-weight phases with the smallest-id rule: hubs on
          // thread-block clusters when every hub of the phase fits one
          if (tie != NIDO_TIE_NIDO && g->cfg.hub_clusters && g->hub_cl_ok) {
            NIDO_TRY(launch_clusters<kMulti>(g, batch, p, s));
            break;
          }
        }
        SliceResult* res = reinterpret_cast<SliceResult*>(g->hub_res);
        for (int64_t wv = g->hub_wave_off[batch]; wv < g->hub_wave_off[batch + 1]; ++wv) {
          const nido_graph_s::HubWave& w = g->hub_waves[wv];
          const int2* items = g->hub_items + w.i0;
          if (tie == NIDO_TIE_NIDO) {
            k_move_hub<kMulti><<<grid_cap(w.i1 - w.i0, R.hubmv), kHubThreads, 0, s>>>(
                items, w.i1 - w.i0, g->hub_v, g->hub_toff, g->hub_capv, g->hub_nseg, g->hub_done, g->gkeys,
                g->gvals, p);
            NIDO_LAUNCH_CHECK();
            continue;
          }
          if (kInts && g->gpacked && g->gslab_packed >= g->gslab_need) {
            k_hub_insert_packed<<<grid_cap(w.i1 - w.i0, R.hubins), kHubThreads, 0, s>>>(
                items, w.i1 - w.i0, g->hub_v, g->hub_toff, g->hub_capv, g->gpacked, p);
            NIDO_LAUNCH_CHECK();
            k_hub_slices_packed<kMulti><<<grid_cap(w.s1 - w.s0, R.hubsl), kHubThreads, 0, s>>>(
                g->hub_slices + w.s0, w.s1 - w.s0, g->hub_v, g->hub_toff, g->hub_capv, g->gpacked, p, res + w.s0);
            NIDO_LAUNCH_CHECK();
          } else {
            k_hub_insert<<<grid_cap(w.i1 - w.i0, R.hubins), kHubThreads, 0, s>>>(
                items, w.i1 - w.i0, g->hub_v, g->hub_toff, g->hub_capv, g->gkeys, g->gvals, p);
            NIDO_LAUNCH_CHECK();
            k_hub_slices<kMulti><<<grid_cap(w.s1 - w.s0, R.hubsl), kHubThreads, 0, s>>>(
                g->hub_slices + w.s0, w.s1 - w.s0, g->hub_v, g->hub_toff, g->hub_capv, g->gkeys, g->gvals, p,
                res + w.s0);
            NIDO_LAUNCH_CHECK();
          }
          k_hub_combine<kMulti><<<grid_cap((w.h1 - w.h0 + 7) / 8, kSMs * 4), 256, 0, s>>>(
              w.h1 - w.h0, g->hub_v + w.h0, g->hub_slice_first + w.h0, res, p);
          NIDO_LAUNCH_CHECK();
        }
        continue;
      }
    }
    NIDO_LAUNCH_CHECK();
  }
  for (int i = 0; i < 2; ++i) {
    NIDO_CUDA_TRY(cudaEventRecord(ctx->join_ev[i], ctx->aux[i]));
    NIDO_CUDA_TRY(cudaStreamWaitEvent(main_s, ctx->join_ev[i], 0));
  }
  return NIDO_OK;
}
}  // namespace

int move_init_attributes() {
  NIDO_TRY(cluster_init());
  NIDO_TRY((set_smem_mode<false, false>()));
  NIDO_TRY((set_smem_mode<false, true>()));
  NIDO_TRY((set_smem_mode<true, false>()));
  return set_smem_mode<true, true>();
}

namespace {
MoveArgs move_args(nido_graph_s* g, int tie) {
  return MoveArgs{g->off, g->adj, g->w, g->comm, g->k, g->a, g->newc, g->m, tie,
                  reinterpret_cast<unsigned long long*>(g->dcount + 1), g->gid, g->mg, g->int_weights ? 1 : 0, g->nv};
}

int tiers_direct(nido_graph_s* g, int batch, int tie, const MoveArgs& p) {
  if (g->gid) return p.ints ? launch_tiers<true, true>(g, batch, tie, p) : launch_tiers<true, false>(g, batch, tie, p);
  return p.ints ? launch_tiers<false, true>(g, batch, tie, p) : launch_tiers<false, false>(g, batch, tie, p);
}
}  // namespace

// The tier kernels of one batch, enqueued directly (no events, no per-batch
// graph): what the device-resident loop captures.  The plan (tier lists, hub
// plan) must be valid.
int launch_move_tiers(nido_graph_s* g, int batch, int tie) {
  if (batch < 0 || batch >= g->nbatches)
    return nido_set_error(NIDO_E_INVALID, "louvain_update: batch %d out of range [0,%d)", batch, g->nbatches);
  return tiers_direct(g, batch, tie, move_args(g, tie));
}

int check_bounded_wait(nido_ctx_s* ctx, int32_t* gave_up, int32_t* waited_ms) {
  int32_t* d = nullptr;
  NIDO_CUDA_TRY(cudaMalloc((void**)&d, 2 * sizeof(int32_t)));
  int32_t h[2] = {0, 0};
  k_check_bounded_wait<<<1, 32, 0, ctx->stream>>>(d);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpyAsync(h, d, sizeof(h), cudaMemcpyDeviceToHost, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  cudaFree(d);
  if (e != cudaSuccess) return nido_set_error(NIDO_E_CUDA, "bounded-wait check: %s", cudaGetErrorString(e));
  nido_count_launches(1);
  if (gave_up) *gave_up = h[0];
  if (waited_ms) *waited_ms = h[1];
  return NIDO_OK;
}

int launch_move(nido_graph_s* g, int batch, int tie, cudaEvent_t ev_start, cudaEvent_t ev_end) {
  if (batch < 0 || batch >= g->nbatches)
    return nido_set_error(NIDO_E_INVALID, "louvain_update: batch %d out of range [0,%d)", batch, g->nbatches);
  if (!g->bins_valid) NIDO_TRY(build_batches(g));
  cudaStream_t s = g->ctx->stream;
  const MoveArgs p = move_args(g, tie);
  if (ev_start) NIDO_CUDA_TRY(cudaEventRecord(ev_start, s));
  auto direct = [&]() { return tiers_direct(g, batch, tie, p); };
  if (!g->use_graphs) {
    NIDO_TRY(direct());
  } else {
    // The launches of a batch are fixed for a phase: the first sweep runs them
    // directly, the second captures them into a CUDA graph, later sweeps
    // replay it (the arguments are all device pointers that live for the
    // phase).
    if (g->move_graphs.size() < (size_t)g->nbatches) g->move_graphs.resize(g->nbatches);
    nido_graph_s::MoveGraph& mg = g->move_graphs[batch];
    if (mg.epoch != g->plan_epoch || mg.tie != tie) {
      if (mg.exec) cudaGraphExecDestroy(mg.exec);
      mg = nido_graph_s::MoveGraph();
      mg.epoch = g->plan_epoch;
      mg.tie = tie;
    }
    if (mg.exec) {
      NIDO_CUDA_TRY(cudaGraphLaunch(mg.exec, s));
      nido_count_launches(mg.kernels);
    } else if (mg.uses++ == 0) {
      NIDO_TRY(direct());
    } else {
      const uint64_t l0 = nido_launch_count();
      cudaGraph_t graph = nullptr;
      NIDO_CUDA_TRY(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
      const int st = direct();
      const cudaError_t ce = cudaStreamEndCapture(s, &graph);
      if (st != NIDO_OK) {
        if (graph) cudaGraphDestroy(graph);
        return st;
      }
      if (ce != cudaSuccess) return nido_set_error(NIDO_E_CUDA, "move-sweep capture failed: %s", cudaGetErrorString(ce));
      mg.kernels = nido_launch_count() - l0;
      const cudaError_t ie = cudaGraphInstantiate(&mg.exec, graph, 0);
      cudaGraphDestroy(graph);
      if (ie != cudaSuccess) {
        mg.exec = nullptr;
        return nido_set_error(NIDO_E_CUDA, "move-sweep graph instantiation failed: %s", cudaGetErrorString(ie));
      }
      NIDO_CUDA_TRY(cudaGraphLaunch(mg.exec, s));
    }
  }
  if (ev_end) NIDO_CUDA_TRY(cudaEventRecord(ev_end, s));
  return NIDO_OK;
}

}  // namespace nido
