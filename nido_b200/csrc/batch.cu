// batch.cu -- many independent graphs in one run.
//
// The reference runs one graph per process (louvain_gpu.cpp:6-139).  Here
// any number of graphs are packed into one CSR over all their vertices (a
// disjoint union: graph i owns vertices [vbase[i], vbase[i+1]) and every edge
// stays inside its graph), and one phase loop drives all of them: each move
// sweep, commit, modularity and coarsening pass covers every graph still
// running with the same kernels the one-graph run uses.  What is per graph:
//   - the mass m (looked up per vertex through the graph id gid[v]);
//   - the -b cuts (the reference's rule applied to the graph's own CSR);
//   - Q, reduced in the reference's shape for the graph alone, so it is the
//     same value a run on that graph by itself computes;
//   - the loop control: per-graph dQ, loop counters and convergence flags
//     live on the device; graphs that stop iterating are no longer committed
//     and drop out of the degree-tier lists once enough of them stopped;
//     a graph that finishes has its clustering written out at once and its
//     vertices dropped from the union at the next coarsening, so later
//     phases carry only the graphs still running.
// Given integer weights (exact FP64 sums) every graph's clustering equals the
// one nido_run produces for that graph alone.
#include <string.h>

#include <algorithm>
#include <chrono>
#include <new>
#include <numeric>
#include <type_traits>
#include <vector>

#include "common.cuh"
#include "cuts.cuh"
#include "engine.cuh"

using nido::Arena;

struct nido_batch_s {
  nido_graph_s* g = nullptr;  // the union graph
  int32_t ng = 0;
  int nb = 1;
  std::vector<int64_t> vbase;  // original vertex bases (host)
  // per graph (device)
  int64_t* gbase0 = nullptr;   // original bases, ng+1
  int64_t* gbA = nullptr;      // current / next bases (ng+1 each)
  int64_t* gbB = nullptr;
  int64_t* gcuts = nullptr;    // ng*(nb+1)
  int64_t* gparts = nullptr;   // ng*(nb+2)
  int64_t* gedges = nullptr;   // ng: edges of the current phase's graphs
  int32_t* gactive = nullptr;  // in the degree-tier lists
  int32_t* giter = nullptr;    // iterating in this loop
  int32_t* grest = nullptr;    // undo this loop's moves
  int32_t* gagg = nullptr;     // aggregates at the end of this phase
  int32_t* gfin = nullptr;     // finished
  int32_t* loops_phase = nullptr;
  int64_t* loops_total = nullptr;
  int64_t* phases = nullptr;
  double* Q = nullptr;
  double* Qold = nullptr;
  double* qnew = nullptr;
  double* mg = nullptr;
  // work lists (graph ids and value offsets) and reduction buffers
  int32_t* plist = nullptr;    // graphs of the phase
  int32_t* llist = nullptr;    // graphs in the tier lists
  int64_t* moff = nullptr;     // mass partial blocks over plist (ng+1)
  int64_t* qoff = nullptr;     // modularity groups over llist (ng+1)
  double* part = nullptr;
  double* modv = nullptr;
  double* selfv = nullptr;
  int64_t* counters = nullptr; // [0] iterating graphs [1] restoring [2] iterating vertices [3] aggregating
  int64_t* bctl = nullptr;     // control block of the device-resident sweep loop (BatchCtl)
  int32_t* gid = nullptr;
  int64_t* outc = nullptr;     // final clustering of every original vertex (ids within its graph)
  int32_t* elist = nullptr;    // graphs whose clustering is written out now
  int64_t cap_part = 0, cap_modv = 0;
  size_t bytes = 0;            // budgeted bytes of the arrays above
};

namespace nido {
namespace {

constexpr int kThreads = 256;

inline unsigned grid_for(int64_t work, int per_block, int max_blocks = kSMs * 16) {
  int64_t b = (work + per_block - 1) / per_block;
  if (b < 1) b = 1;
  if (b > max_blocks) b = max_blocks;
  return (unsigned)b;
}

// largest i in [0, n) with offs[i] <= x (offs non-decreasing, offs[0] <= x);
// empty ranges are skipped toward the later item
__device__ __forceinline__ int find_item(const int64_t* __restrict__ offs, int n, int64_t x) {
  int lo = 0, hi = n;
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (offs[mid] <= x) lo = mid; else hi = mid;
  }
  return lo;
}

__global__ void k_gid(const int64_t* __restrict__ gbase, int ng, int64_t nv, int32_t* __restrict__ gid) {
  for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < nv; v += (int64_t)gridDim.x * blockDim.x)
    gid[v] = find_item(gbase, ng, v);
}

// every edge of a vertex must end inside the vertex's graph
__global__ void k_check_edges(const int64_t* __restrict__ off, const int32_t* __restrict__ adj, int64_t nv,
                              const int32_t* __restrict__ gid, const int64_t* __restrict__ gbase,
                              unsigned long long* __restrict__ bad) {
  const int lane = threadIdx.x & 31;
  const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  unsigned long long b = 0;
  for (int64_t v = warp; v < nv; v += nw) {
    const int g = gid[v];
    const int64_t lo = gbase[g], hi = gbase[g + 1];
    for (int64_t j = off[v] + lane; j < off[v + 1]; j += 32)
      if (adj[j] < lo || adj[j] >= hi) ++b;
  }
  if (b) atomicAdd(bad, b);
}

__global__ void k_graph_edges(const int64_t* __restrict__ off, const int64_t* __restrict__ gbase, int ng,
                              int64_t* __restrict__ gedges) {
  for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < ng; g += gridDim.x * blockDim.x)
    gedges[g] = off[gbase[g + 1]] - off[gbase[g]];
}

__global__ void k_set_flags(const int32_t* __restrict__ list, int n, int32_t* __restrict__ flags) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) flags[list[i]] = 1;
}

// m, first stage, per graph: the partial of block b of the reference's
// compute_mass_reduce_kernel<32><<<4096,32>>> (graph_cuda.cu:1786-1804) run
// on the graph alone; one warp per (graph, block) item.
__global__ void k_mass_parts(const int32_t* __restrict__ gl, const int64_t* __restrict__ moff, int n,
                             const int64_t* __restrict__ gbase, const double* __restrict__ k,
                             double* __restrict__ part) {
  const int lane = threadIdx.x & 31;
  const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  const int64_t total = moff[n];
  for (int64_t it = warp; it < total; it += nw) {
    const int i = find_item(moff, n, it);
    const int g = gl[i];
    const int64_t b = it - moff[i];
    const int64_t base = gbase[g], nvg = gbase[g + 1] - base;
    double x = 0.;
    for (int64_t j = lane + 32 * b; j < nvg; j += 32 * 4096) x += k[base + j];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(NIDO_FULL_MASK, x, o);
    if (lane == 0) part[it] = x;
  }
}

// reduce_vector_kernel<32><<<1,1024>>> (graph_cuda.cu:1806-1835) once per
// listed graph: item i reduces vals[offs[i], offs[i+1]) into out[gl[i]].
__global__ void __launch_bounds__(1024) k_reduce_block(const int32_t* __restrict__ gl, const int64_t* __restrict__ offs,
                                                       const double* __restrict__ vals, double scale,
                                                       double* __restrict__ out) {
  __shared__ double ws[32];
  const int i = blockIdx.x;
  const double* x = vals + offs[i];
  const int64_t n = offs[i + 1] - offs[i];
  double s = 0.;
  for (int64_t j = threadIdx.x; j < n; j += 1024) s += x[j];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(NIDO_FULL_MASK, s, o);
  if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x < 32) {
    s = ws[threadIdx.x];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(NIDO_FULL_MASK, s, o);
    if (threadIdx.x == 0) out[gl[i]] = scale * s;
  }
}

// The same reduction for items of at most 1024 values on one warp: virtual
// thread t of the 1024 holds 0 + x[t]; the warp replays each virtual warp's
// shuffle tree, then the tree over the 32 warp sums, so the result is the
// block kernel's bit for bit.
__global__ void k_reduce_warp(const int32_t* __restrict__ gl, const int64_t* __restrict__ offs, int i0, int n,
                              const double* __restrict__ vals, double scale, double* __restrict__ out) {
  const int lane = threadIdx.x & 31;
  const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t i = i0 + warp; i < n; i += nw) {
    const double* x = vals + offs[i];
    const int64_t cnt = offs[i + 1] - offs[i];
    double mine = 0.;
    for (int w = 0; 32 * w < cnt; ++w) {
      double s = 0.;
      const int64_t j = 32 * w + lane;
      if (j < cnt) s += x[j];
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(NIDO_FULL_MASK, s, o);
      const double r = __shfl_sync(NIDO_FULL_MASK, s, 0);
      if (lane == w) mine = r;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) mine += __shfl_down_sync(NIDO_FULL_MASK, mine, o);
    if (lane == 0) out[gl[i]] = scale * mine;
  }
}

__global__ void k_cuts_multi(const int32_t* __restrict__ gl, int n, const int64_t* __restrict__ off,
                             const int64_t* __restrict__ gbase, int nb, int64_t* __restrict__ gcuts,
                             int64_t* __restrict__ gparts) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int g = gl[i];
    const int64_t base = gbase[g];
    batch_cuts(off + base, gbase[g + 1] - base, nb, gcuts + (int64_t)g * (nb + 1), gparts + (int64_t)g * (nb + 2));
  }
}

// Modularity, second stage, per graph: the thread slots and 16-lane groups of
// compute_modularity_reduce_kernel<128,16> (graph_cuda.cu:2096-2134) on the
// graph alone (S = 128 * min(ceil(nv/8), 65535) slots), one 16-lane group per
// (graph, group) item.
__global__ void k_q_groups_multi(const int32_t* __restrict__ gl, const int64_t* __restrict__ qoff, int n,
                                 const int64_t* __restrict__ gbase, const double* __restrict__ selfv,
                                 const double* __restrict__ a, const double* __restrict__ mg,
                                 double* __restrict__ modv) {
  const int64_t total = qoff[n] * 16;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t t0 = blockIdx.x * (int64_t)blockDim.x; t0 < total; t0 += stride) {
    const int64_t t = t0 + threadIdx.x;
    const int64_t G = t >> 4;
    double s = 0., ac = 0., m = 0.;
    if (t < total) {
      const int i = find_item(qoff, n, G);
      const int g = gl[i];
      const int64_t base = gbase[g], nvg = gbase[g + 1] - base;
      int64_t grid = (nvg + 7) / 8;
      if (grid > 65535) grid = 65535;
      const int64_t S = 128 * grid;
      for (int64_t v = (G - qoff[i]) * 16 + (t & 15); v < nvg; v += S) {
        s += selfv[base + v];
        ac = fma(a[base + v], a[base + v], ac);
      }
      m = mg[g];
    }
#pragma unroll
    for (int o = 8; o > 0; o >>= 1) {
      s += __shfl_down_sync(NIDO_FULL_MASK, s, o, 16);
      ac += __shfl_down_sync(NIDO_FULL_MASK, ac, o, 16);
    }
    if ((t & 15) == 0 && t < total) {
      double x = __ddiv_rn(s, __dmul_rn(2., m));
      x = __dsub_rn(x, __ddiv_rn(ac, __dmul_rn(__dmul_rn(4., m), m)));
      modv[G] = __dadd_rn(0., x);
    }
  }
}

// Per-graph loop control after a sweep (louvain_gpu.cpp:74-98): dQ, undo on
// dQ < 0, and whether the graph goes on (tau < dQ and loops < max_iter).
__global__ void k_control(const int32_t* __restrict__ gl, int n, const double* __restrict__ qnew,
                          double* __restrict__ Q, int32_t* __restrict__ loops_phase,
                          int64_t* __restrict__ loops_total, int32_t* __restrict__ giter,
                          int32_t* __restrict__ grest, double tau, int64_t max_iter,
                          const int64_t* __restrict__ gbase, unsigned long long* __restrict__ counters) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int g = gl[i];
    if (!giter[g]) continue;
    const double qt = qnew[g];
    const double dQ = qt - Q[g];
    const int lp = ++loops_phase[g];
    loops_total[g] += 1;
    if (dQ < 0) {
      grest[g] = 1;
      atomicAdd(&counters[1], 1ull);
    } else {
      Q[g] = qt;
    }
    const bool go = tau < dQ && lp < max_iter;
    giter[g] = go ? 1 : 0;
    if (go) {
      atomicAdd(&counters[0], 1ull);
      atomicAdd(&counters[2], (unsigned long long)(gbase[g + 1] - gbase[g]));
    }
  }
}

// The listed vertices of one batch: the perm ranges of its (tier, batch)
// keys, which are not contiguous (the keys are tier-major).
struct PermRanges {
  int64_t start[kNumTiers];
  int64_t pre[kNumTiers + 1];  // prefix of the range lengths
};

// k_commit of the one-graph driver for the listed vertices of a batch (or,
// for restore, for every listed vertex: one range) of the graphs whose flag
// is set.
__global__ void k_commit_listed(PermRanges r, int nr, const int32_t* __restrict__ perm,
                                const int32_t* __restrict__ gid, const int32_t* __restrict__ flag,
                                const double* __restrict__ k, int32_t* __restrict__ comm,
                                int32_t* __restrict__ newc, double* __restrict__ a,
                                const int64_t* __restrict__ gate) {
  if (gate && *gate == 0) return;  // the device-resident loop's restore, when no graph needs it
  const int64_t total = r.pre[nr];
  for (int64_t x = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; x < total; x += (int64_t)gridDim.x * blockDim.x) {
    int t = 0;
    while (r.pre[t + 1] <= x) ++t;
    const int v = perm[r.start[t] + (x - r.pre[t])];
    if (!flag[gid[v]]) continue;
    const int32_t src = comm[v], dst = newc[v];
    if (src != dst) {
      const double kv = k[v];
      atomicAdd(&a[src], -kv);
      atomicAdd(&a[dst], kv);
    }
    comm[v] = dst;
    newc[v] = src;
  }
}

// Control block of the device-resident sweep loop: stamps and device times
// of the move kernels and of the modularity, sweeps run, and the counters of
// the last sweep.
struct BatchCtl {
  unsigned long long t_move, move_ns, t_q, q_ns;
  long long sweeps;
  long long cnt[4];
};

// After k_control: go on while some graph iterates and the graphs still
// iterating hold at least 3/4 of the listed vertices (below that the host
// rebuilds the tier lists without the stopped graphs).
__global__ void k_batch_cond(const unsigned long long* __restrict__ counters, BatchCtl* c, int64_t listed_v,
                             cudaGraphConditionalHandle h) {
  c->sweeps += 1;
  for (int i = 0; i < 4; ++i) c->cnt[i] = (long long)counters[i];
  const bool any = counters[0] > 0;
  const bool keep = 4 * (long long)counters[2] >= 3 * listed_v;
  cudaGraphSetConditional(h, any && keep ? 1u : 0u);
}

__global__ void k_batch_ctl_reset(BatchCtl* c) {
  c->move_ns = 0;
  c->q_ns = 0;
  c->sweeps = 0;
}

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
__global__ void k_bstamp(unsigned long long* t) { *t = global_ns(); }
__global__ void k_blap(const unsigned long long* t0, unsigned long long* acc) { *acc += global_ns() - *t0; }

struct LoopGraph {  // destroyed on every return
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  ~LoopGraph() {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
  }
};

// end of a phase (louvain_gpu.cpp:100-118): aggregate if Q - Q_old > tau,
// else the graph is finished
__global__ void k_phase_end(const int32_t* __restrict__ gl, int n, const double* __restrict__ Q,
                            const double* __restrict__ Qold, double tau, int32_t* __restrict__ gagg,
                            int32_t* __restrict__ gfin, int64_t* __restrict__ phases,
                            unsigned long long* __restrict__ counters) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int g = gl[i];
    phases[g] += 1;
    if (Q[g] - Qold[g] > tau) {
      gagg[g] = 1;
      atomicAdd(&counters[3], 1ull);
    } else {
      gfin[g] = 1;
    }
  }
}

// graphs that do not aggregate are finished (their clustering is written
// out already): community -1 drops their vertices from the coarse union
__global__ void k_drop(int64_t nv, const int32_t* __restrict__ gid, const int32_t* __restrict__ gagg,
                       int32_t* __restrict__ comm) {
  for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < nv; v += (int64_t)gridDim.x * blockDim.x)
    if (!gagg[gid[v]]) comm[v] = -1;
}

// final clustering of the listed graphs: clus of their original vertices,
// renumbered within each graph (one block per graph)
__global__ void k_emit(const int32_t* __restrict__ gl, int n, const int64_t* __restrict__ gbase0,
                       const int64_t* __restrict__ gbase, const int32_t* __restrict__ clus, int64_t* __restrict__ outc) {
  for (int i = blockIdx.x; i < n; i += gridDim.x) {
    const int g = gl[i];
    const int64_t b = gbase[g];
    for (int64_t v = gbase0[g] + threadIdx.x; v < gbase0[g + 1]; v += blockDim.x) outc[v] = (int64_t)clus[v] - b;
  }
}

// a graph whose coarsening kept its vertex count or left one vertex is
// finished (graph_gpu.cpp:1391-1392)
__global__ void k_post_agg(const int32_t* __restrict__ gl, int n, const int64_t* __restrict__ gold,
                           const int64_t* __restrict__ gnew, const int32_t* __restrict__ gagg,
                           int32_t* __restrict__ gfin) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int g = gl[i];
    if (!gagg[g]) continue;
    const int64_t nvo = gold[g + 1] - gold[g], nvp = gnew[g + 1] - gnew[g];
    if (nvp == nvo || nvp == 1) gfin[g] = 1;
  }
}

__global__ void k_iota32(int32_t* __restrict__ x, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    x[i] = (int32_t)i;
}

// ---- host side ------------------------------------------------------------------

// per-graph sizes of the reductions (the reference's shapes for one graph)
inline int64_t mass_blocks(int64_t nvg) { return std::min<int64_t>(4096, (nvg + 31) / 32); }
inline int64_t q_groups(int64_t nvg) {
  const int64_t grid = std::min<int64_t>((nvg + 7) / 8, 65535);
  return (std::min<int64_t>(128 * grid, nvg) + 15) / 16;
}

struct Lists {
  std::vector<int32_t> ids;  // graph ids, larger graphs first
  std::vector<int64_t> off;  // value offsets (ids.size()+1)
  int nbig = 0;              // items reduced by a whole block (more than 1024 values)
};

Lists make_list(const std::vector<int32_t>& ids, const std::vector<int64_t>& base, int64_t (*count)(int64_t)) {
  Lists L;
  L.ids = ids;
  std::stable_sort(L.ids.begin(), L.ids.end(), [&](int32_t x, int32_t y) {
    return base[x + 1] - base[x] > base[y + 1] - base[y];
  });
  L.off.assign(L.ids.size() + 1, 0);
  for (size_t i = 0; i < L.ids.size(); ++i) {
    const int64_t c = count(base[L.ids[i] + 1] - base[L.ids[i]]);
    L.off[i + 1] = L.off[i] + c;
    if (c > 1024) L.nbig = (int)i + 1;
  }
  return L;
}

int upload_list(cudaStream_t s, const Lists& L, int32_t* ids, int64_t* off) {
  if (L.ids.empty()) return NIDO_OK;
  NIDO_CUDA_TRY(cudaMemcpyAsync(ids, L.ids.data(), sizeof(int32_t) * L.ids.size(), cudaMemcpyHostToDevice, s));
  NIDO_CUDA_TRY(cudaMemcpyAsync(off, L.off.data(), sizeof(int64_t) * L.off.size(), cudaMemcpyHostToDevice, s));
  return NIDO_OK;
}

int reduce_lists(cudaStream_t s, const Lists& L, const int32_t* ids, const int64_t* off, const double* vals,
                 double scale, double* out) {
  const int n = (int)L.ids.size();
  if (L.nbig > 0) {
    k_reduce_block<<<L.nbig, 1024, 0, s>>>(ids, off, vals, scale, out);
    NIDO_LAUNCH_CHECK();
  }
  if (n > L.nbig) {
    k_reduce_warp<<<grid_for((int64_t)(n - L.nbig) * 32, kThreads), kThreads, 0, s>>>(ids, off, L.nbig, n, vals,
                                                                                     scale, out);
    NIDO_LAUNCH_CHECK();
  }
  return NIDO_OK;
}

// per-graph Q of the listed graphs into out (the tier lists cover exactly them)
int batch_modularity(nido_batch_s* B, const Lists& ql, double* out) {
  nido_graph_s* g = B->g;
  cudaStream_t s = g->ctx->stream;
  if (ql.ids.empty()) return NIDO_OK;
  NIDO_TRY(launch_q_self(g, B->selfv));
  const int n = (int)ql.ids.size();
  const int64_t threads = ql.off[n] * 16;
  k_q_groups_multi<<<grid_for(threads, kThreads, kSMs * 32), kThreads, 0, s>>>(B->llist, B->qoff, n, g->gbase,
                                                                               B->selfv, g->a, B->mg, B->modv);
  NIDO_LAUNCH_CHECK();
  return reduce_lists(s, ql, B->llist, B->qoff, B->modv, 1.0, out);
}

// (re)build the degree-tier lists and the modularity layout over the graphs
// in ids, which become the listed (gactive) graphs
// The graphs ids are listed: modularity groups, active flags and the tier
// lists of their vertices.  relist: ids is a subset of the graphs listed so
// far in this phase, so the tier lists are compacted instead of rebuilt.
int batch_list(nido_batch_s* B, const std::vector<int32_t>& ids, const std::vector<int64_t>& base, Lists* ql,
               bool relist = false) {
  nido_graph_s* g = B->g;
  cudaStream_t s = g->ctx->stream;
  NIDO_CUDA_TRY(cudaMemsetAsync(B->gactive, 0, sizeof(int32_t) * B->ng, s));
  *ql = make_list(ids, base, q_groups);
  NIDO_TRY(upload_list(s, *ql, B->llist, B->qoff));
  if (!ids.empty()) {
    k_set_flags<<<grid_for((int64_t)ids.size(), kThreads), kThreads, 0, s>>>(B->llist, (int)ids.size(), B->gactive);
    NIDO_LAUNCH_CHECK();
  }
  if (ql->off.back() > B->cap_modv) return nido_set_error(NIDO_E_NOMEM, "modularity buffer too small");
  if (relist && g->bins_valid) return compact_batches(g);
  g->bins_valid = false;
  return build_batches(g);
}

int batch_reset(nido_batch_s* B) {
  nido_graph_s* g = B->g;
  cudaStream_t s = g->ctx->stream;
  g->off = g->off0;
  g->adj = g->adj0;
  g->w = g->w0;
  g->nv = g->nv0;
  g->ne = g->ne0;
  g->coarsened = false;
  g->bins_valid = false;
  k_iota32<<<grid_for(g->nv0, kThreads), kThreads, 0, s>>>(g->clus, g->nv0);
  NIDO_LAUNCH_CHECK();
  g->gbase = B->gbA;
  g->gbase2 = B->gbB;
  const size_t n1 = sizeof(int64_t) * (B->ng + 1);
  NIDO_CUDA_TRY(cudaMemcpyAsync(g->gbase, B->gbase0, n1, cudaMemcpyDeviceToDevice, s));
  NIDO_CUDA_TRY(cudaMemsetAsync(B->gfin, 0, sizeof(int32_t) * B->ng, s));
  NIDO_CUDA_TRY(cudaMemsetAsync(B->grest, 0, sizeof(int32_t) * B->ng, s));
  NIDO_CUDA_TRY(cudaMemsetAsync(B->loops_total, 0, sizeof(int64_t) * B->ng, s));
  NIDO_CUDA_TRY(cudaMemsetAsync(B->phases, 0, sizeof(int64_t) * B->ng, s));
  NIDO_CUDA_TRY(cudaMemsetAsync(B->Q, 0, sizeof(double) * B->ng, s));
  return NIDO_OK;
}

}  // namespace
}  // namespace nido

using namespace nido;

extern "C" int nido_batch_free(nido_batch B) {
  if (!B) return NIDO_OK;
  nido_ctx ctx = B->g ? B->g->ctx : nullptr;
  if (ctx) {
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    for (void* p : {(void*)B->gbase0, (void*)B->gbA, (void*)B->gbB, (void*)B->gcuts, (void*)B->gparts,
                    (void*)B->gedges, (void*)B->gactive, (void*)B->giter, (void*)B->grest, (void*)B->gagg,
                    (void*)B->gfin, (void*)B->loops_phase, (void*)B->loops_total, (void*)B->phases, (void*)B->Q,
                    (void*)B->Qold, (void*)B->qnew, (void*)B->mg, (void*)B->plist, (void*)B->llist,
                    (void*)B->moff, (void*)B->qoff, (void*)B->part, (void*)B->modv, (void*)B->selfv,
                    (void*)B->counters, (void*)B->bctl, (void*)B->gid, (void*)B->outc,
                    (void*)B->elist})
      raw_free(ctx, p);
    ctx->used -= std::min(ctx->used, B->bytes);
    nido_graph_free(B->g);
  }
  delete B;
  return NIDO_OK;
}

extern "C" int nido_batch_upload(nido_ctx ctx, int32_t ngraphs, const int64_t* vbase, int64_t nv, int64_t ne,
                                 const int64_t* off, const int64_t* adj, const double* w, int32_t nbatches,
                                 nido_batch* out) {
  if (!ctx || !out || !vbase) return nido_set_error(NIDO_E_INVALID, "nido_batch_upload: null argument");
  *out = nullptr;
  if (ngraphs < 1) return nido_set_error(NIDO_E_INVALID, "ngraphs must be >= 1 (got %d)", ngraphs);
  if (vbase[0] != 0 || vbase[ngraphs] != nv)
    return nido_set_error(NIDO_E_INVALID, "vertex bases must run from 0 to nv");
  for (int32_t i = 0; i < ngraphs; ++i)
    if (vbase[i + 1] < vbase[i]) return nido_set_error(NIDO_E_INVALID, "vertex bases must not decrease");
  nido_graph g = nullptr;
  NIDO_TRY(nido_graph_upload(ctx, nv, ne, off, adj, w, nbatches, &g));
  nido_batch B = new (std::nothrow) nido_batch_s();
  if (!B) { nido_graph_free(g); return nido_set_error(NIDO_E_NOMEM, "host allocation failed"); }
  B->g = g;
  B->ng = ngraphs;
  B->nb = nbatches;
  B->vbase.assign(vbase, vbase + ngraphs + 1);
  const int64_t G = ngraphs, V = nv;
  B->cap_part = V / 32 + 2 * G + 16;
  B->cap_modv = V / 16 + 2 * G + 16;
  int st = NIDO_OK;
  auto take = [&](auto** p, int64_t n) {
    if (st != NIDO_OK) return;
    const size_t bytes = sizeof(**p) * (size_t)std::max<int64_t>(n, 1);
    void* q = nullptr;
    st = device_alloc(ctx, &q, bytes);
    *p = static_cast<std::remove_reference_t<decltype(*p)>>(q);
    if (st == NIDO_OK) B->bytes += bytes;
  };
  take(&B->gbase0, G + 1); take(&B->gbA, G + 1); take(&B->gbB, G + 1);
  take(&B->gcuts, G * (nbatches + 1)); take(&B->gparts, G * (nbatches + 2)); take(&B->gedges, G);
  take(&B->gactive, G); take(&B->giter, G); take(&B->grest, G); take(&B->gagg, G); take(&B->gfin, G);
  take(&B->loops_phase, G); take(&B->loops_total, G); take(&B->phases, G);
  take(&B->Q, G); take(&B->Qold, G); take(&B->qnew, G); take(&B->mg, G);
  take(&B->plist, G); take(&B->llist, G); take(&B->moff, G + 1); take(&B->qoff, G + 1);
  take(&B->part, B->cap_part); take(&B->modv, B->cap_modv); take(&B->selfv, V);
  take(&B->counters, 4); take(&B->bctl, 16); take(&B->gid, V);
  take(&B->outc, V); take(&B->elist, G);
  if (st != NIDO_OK) {
    // device_alloc counted only what it allocated; nido_batch_free subtracts B->bytes
    nido_batch_free(B);
    return st;
  }
  cudaStream_t s = ctx->stream;
  NIDO_CUDA_TRY(cudaMemcpyAsync(B->gbase0, vbase, sizeof(int64_t) * (G + 1), cudaMemcpyHostToDevice, s));
  NIDO_CUDA_TRY(cudaMemsetAsync(B->gcuts, 0, sizeof(int64_t) * G * (nbatches + 1), s));
  k_gid<<<grid_for(V, kThreads), kThreads, 0, s>>>(B->gbase0, ngraphs, V, B->gid);
  NIDO_LAUNCH_CHECK();
  unsigned long long* bad = reinterpret_cast<unsigned long long*>(B->counters);
  NIDO_CUDA_TRY(cudaMemsetAsync(bad, 0, sizeof(unsigned long long), s));
  k_check_edges<<<grid_for(V * 32, kThreads), kThreads, 0, s>>>(g->off0, g->adj0, V, B->gid, B->gbase0, bad);
  NIDO_LAUNCH_CHECK();
  unsigned long long nbad = 0;
  NIDO_CUDA_TRY(cudaMemcpyAsync(&nbad, bad, sizeof(nbad), cudaMemcpyDeviceToHost, s));
  NIDO_CUDA_TRY(cudaStreamSynchronize(s));
  if (nbad) {
    nido_batch_free(B);
    return nido_set_error(NIDO_E_INVALID, "%llu edges leave their graph", nbad);
  }
  g->gid = B->gid;
  g->mg = B->mg;
  g->gcuts = B->gcuts;
  g->gactive = B->gactive;
  g->gbase = B->gbA;
  g->gbase2 = B->gbB;
  g->ngraphs = ngraphs;
  g->bins_valid = false;
  *out = B;
  return NIDO_OK;
}

// Phase loop of LouvainGPU::run (louvain_gpu.cpp:28-124) over all graphs at
// once; see the file comment.
extern "C" int nido_batch_run(nido_batch B, const nido_params* p, int64_t* out_comm, double* out_q,
                              int64_t* out_phases, int64_t* out_loops, nido_run_stats* stats) {
  if (!B || !p) return nido_set_error(NIDO_E_INVALID, "null argument");
  nido_graph_s* g = B->g;
  if (p->nbatches != g->nbatches)
    return nido_set_error(NIDO_E_INVALID, "params.nbatches (%d) differs from the batch's (%d)", p->nbatches, g->nbatches);
  if (p->color_batches)
    return nido_set_error(NIDO_E_INVALID, "colour-class batches are for one-graph runs (nido_run)");
  if (p->host_loop < 0 || p->host_loop > 2)
    return nido_set_error(NIDO_E_INVALID, "host_loop must be 0, 1 or 2 (got %d)", p->host_loop);
  if (p->tie_mode != NIDO_TIE_SMALLEST_ID && p->tie_mode != NIDO_TIE_NIDO)
    return nido_set_error(NIDO_E_INVALID, "unknown tie mode %d", p->tie_mode);
  NIDO_CUDA_TRY(cudaSetDevice(g->ctx->device));
  cudaStream_t s = g->ctx->stream;
  nido_run_stats st;
  memset(&st, 0, sizeof(st));
  const uint64_t launches0 = nido_launch_count();
  struct RunEvents {  // destroyed on every return, early ones included
    cudaEvent_t t0 = nullptr, t1 = nullptr, a0 = nullptr, a1 = nullptr;
    ~RunEvents() {
      for (cudaEvent_t e : {t0, t1, a0, a1})
        if (e) cudaEventDestroy(e);
    }
  } re;
  NIDO_CUDA_TRY(cudaEventCreate(&re.t0));
  NIDO_CUDA_TRY(cudaEventCreate(&re.t1));
  NIDO_CUDA_TRY(cudaEventCreate(&re.a0));
  NIDO_CUDA_TRY(cudaEventCreate(&re.a1));
  cudaEvent_t t0 = re.t0, t1 = re.t1;
  std::vector<cudaEvent_t>& ev = g->ctx->move_ev;
  while (ev.size() < 4) {
    cudaEvent_t e;
    NIDO_CUDA_TRY(cudaEventCreate(&e));
    ev.push_back(e);
  }
  // host wall time per section (the slots of nido_run_stats.host_ms for
  // batched runs); the sections end with a stream synchronisation, so each
  // includes the device work it waits for
  auto now_ms = [] {
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now().time_since_epoch()).count();
  };
  double tm = now_ms();
  auto lap = [&](int slot) {
    const double t = now_ms();
    st.host_ms[slot] += t - tm;
    tm = t;
  };
  NIDO_CUDA_TRY(cudaEventRecord(t0, s));
  NIDO_TRY(batch_reset(B));
  lap(0);
  const int ng = B->ng, nb = g->nbatches;
  const double tau = p->tau;
  const double tau_phase = p->tau_phase_set ? p->tau_phase : p->tau;
  std::vector<int64_t> base(B->vbase), edges(ng);
  std::vector<int32_t> fin(ng, 0), flags(ng);
  // graphs whose final clustering is written to outc (empty graphs have none)
  std::vector<char> emitted(ng, 0);
  for (int32_t i = 0; i < ng; ++i) emitted[i] = B->vbase[i + 1] == B->vbase[i];
  auto emit = [&](const std::vector<int32_t>& em) -> int {
    if (em.empty()) return NIDO_OK;
    NIDO_CUDA_TRY(cudaMemcpyAsync(B->elist, em.data(), sizeof(int32_t) * em.size(), cudaMemcpyHostToDevice, s));
    k_emit<<<grid_for((int64_t)em.size(), 1, kSMs * 8), 256, 0, s>>>(B->elist, (int)em.size(), B->gbase0, g->gbase,
                                                                 g->clus, B->outc);
    NIDO_LAUNCH_CHECK();
    NIDO_CUDA_TRY(cudaStreamSynchronize(s));  // em is a local vector
    return NIDO_OK;
  };
  unsigned long long cnt[4];
  int64_t phase = 0;
  bool first = true;
  while (phase < 200) {
    if (!first) {
      NIDO_CUDA_TRY(cudaMemcpyAsync(base.data(), g->gbase, sizeof(int64_t) * (ng + 1), cudaMemcpyDeviceToHost, s));
      NIDO_CUDA_TRY(cudaMemcpyAsync(fin.data(), B->gfin, sizeof(int32_t) * ng, cudaMemcpyDeviceToHost, s));
      NIDO_CUDA_TRY(cudaStreamSynchronize(s));
    }
    std::vector<int32_t> act;
    for (int32_t i = 0; i < ng; ++i)
      if (!fin[i] && base[i + 1] > base[i]) act.push_back(i);
    if (act.empty()) break;
    // phase set-up: graph ids, k, per-graph m and cuts, tier lists
    k_gid<<<grid_for(g->nv, kThreads), kThreads, 0, s>>>(g->gbase, ng, g->nv, B->gid);
    NIDO_LAUNCH_CHECK();
    first = false;
    const int np = (int)act.size();
    NIDO_TRY(launch_vertex_weights(g));
    Lists ml = make_list(act, base, mass_blocks);
    NIDO_TRY(upload_list(s, ml, B->plist, B->moff));
    k_mass_parts<<<grid_for(ml.off[np] * 32, kThreads, kSMs * 32), kThreads, 0, s>>>(B->plist, B->moff, np,
                                                                                    g->gbase, g->k, B->part);
    NIDO_LAUNCH_CHECK();
    NIDO_TRY(reduce_lists(s, ml, B->plist, B->moff, B->part, 0.5, B->mg));
    k_cuts_multi<<<grid_for(np, 128), 128, 0, s>>>(B->plist, np, g->off, g->gbase, nb, B->gcuts, B->gparts);
    NIDO_LAUNCH_CHECK();
    k_graph_edges<<<grid_for(ng, kThreads), kThreads, 0, s>>>(g->off, g->gbase, ng, B->gedges);
    NIDO_LAUNCH_CHECK();
    NIDO_CUDA_TRY(cudaMemcpyAsync(edges.data(), B->gedges, sizeof(int64_t) * ng, cudaMemcpyDeviceToHost, s));
    Lists ql;
    NIDO_TRY(batch_list(B, act, base, &ql));  // synchronizes
    int64_t listed_v = 0, listed_e = 0;
    for (int32_t i : act) { listed_v += base[i + 1] - base[i]; listed_e += edges[i]; }
    // singleton start and Q_old (the tier autotuner, when asked, times move
    // sweeps of the first phase and leaves the tier lists rebuilt)
    NIDO_TRY(launch_singleton(g));
    if (p->tune && !g->tuned && phase == 0) {
      NIDO_TRY(tune_tiers(g, p->tie_mode, 2, nullptr));
      NIDO_TRY(launch_singleton(g));
    }
    NIDO_CUDA_TRY(cudaMemsetAsync(B->gagg, 0, sizeof(int32_t) * ng, s));
    NIDO_CUDA_TRY(cudaMemsetAsync(B->giter, 0, sizeof(int32_t) * ng, s));
    NIDO_CUDA_TRY(cudaMemsetAsync(B->loops_phase, 0, sizeof(int32_t) * ng, s));
    if (p->max_iter > 0) {
      k_set_flags<<<grid_for(np, kThreads), kThreads, 0, s>>>(B->plist, np, B->giter);
      NIDO_LAUNCH_CHECK();
    }
    NIDO_TRY(batch_modularity(B, ql, B->Q));
    NIDO_CUDA_TRY(cudaMemcpyAsync(B->Qold, B->Q, sizeof(double) * ng, cudaMemcpyDeviceToDevice, s));
    NIDO_CUDA_TRY(cudaStreamSynchronize(s));
    lap(4);
    int64_t n_iter = p->max_iter > 0 ? np : 0;
    // the commit of every batch's listed vertices of the iterating graphs
    auto commit_batch = [&](int b) -> int {
      PermRanges r{};
      int64_t tot = 0;
      for (int t = 0; t < kNumTiers; ++t) {
        r.start[t] = g->tier_off[(size_t)t * nb + b];
        r.pre[t] = tot;
        tot += g->tier_off[(size_t)t * nb + b + 1] - r.start[t];
      }
      r.pre[kNumTiers] = tot;
      if (tot > 0) {
        k_commit_listed<<<grid_for(tot, kThreads), kThreads, 0, s>>>(r, kNumTiers, g->perm, B->gid, B->giter, g->k,
                                                                      g->comm, g->newc, g->a, nullptr);
        NIDO_LAUNCH_CHECK();
      }
      return NIDO_OK;
    };
    // the undo of the graphs whose last sweep lowered Q (gate: only when the
    // device counter of such graphs is non-zero)
    auto restore_listed = [&](const int64_t* gate) -> int {
      PermRanges r{};
      r.start[0] = 0;
      r.pre[0] = 0;
      r.pre[1] = g->tier_off[(size_t)kNumTiers * nb];  // every listed vertex
      if (r.pre[1] > 0) {
        k_commit_listed<<<grid_for(r.pre[1], kThreads), kThreads, 0, s>>>(r, 1, g->perm, B->gid, B->grest, g->k,
                                                                           g->comm, g->newc, g->a, gate);
        NIDO_LAUNCH_CHECK();
      }
      NIDO_CUDA_TRY(cudaMemsetAsync(B->grest, 0, sizeof(int32_t) * ng, s));
      return NIDO_OK;
    };
    // Sweeps on the device: one CUDA graph whose conditional while node runs
    // move + commit of every batch, the per-graph modularity and the per-graph
    // loop control, until no graph iterates or the iterating graphs hold less
    // than 3/4 of the listed vertices.  One readback at the end.
    auto device_sweeps = [&](bool* unsupported) -> int {
      *unsupported = false;
      BatchCtl* ctl = reinterpret_cast<BatchCtl*>(B->bctl);
      k_batch_ctl_reset<<<1, 1, 0, s>>>(ctl);
      NIDO_LAUNCH_CHECK();
      LoopGraph lg;
      NIDO_CUDA_TRY(cudaGraphCreate(&lg.graph, 0));
      cudaGraphConditionalHandle h;
      if (cudaGraphConditionalHandleCreate(&h, lg.graph, 1, cudaGraphCondAssignDefault) != cudaSuccess) {
        cudaGetLastError();
        *unsupported = true;
        return NIDO_OK;
      }
      cudaGraphNodeParams cp = {cudaGraphNodeTypeConditional};
      cp.conditional.handle = h;
      cp.conditional.type = cudaGraphCondTypeWhile;
      cp.conditional.size = 1;
      cudaGraphNode_t node;
      if (cudaGraphAddNode(&node, lg.graph, nullptr, 0, &cp) != cudaSuccess) {
        cudaGetLastError();
        *unsupported = true;
        return NIDO_OK;
      }
      const uint64_t l0 = nido_launch_count();
      const auto tb0 = std::chrono::steady_clock::now();
      NIDO_CUDA_TRY(cudaStreamBeginCaptureToGraph(s, cp.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                                  cudaStreamCaptureModeThreadLocal));
      auto body = [&]() -> int {
        for (int b = 0; b < nb; ++b) {
          k_bstamp<<<1, 1, 0, s>>>(&ctl->t_move);
          NIDO_LAUNCH_CHECK();
          NIDO_TRY(launch_move_tiers(g, b, p->tie_mode));
          k_blap<<<1, 1, 0, s>>>(&ctl->t_move, &ctl->move_ns);
          NIDO_LAUNCH_CHECK();
          NIDO_TRY(commit_batch(b));
        }
        k_bstamp<<<1, 1, 0, s>>>(&ctl->t_q);
        NIDO_LAUNCH_CHECK();
        NIDO_TRY(batch_modularity(B, ql, B->qnew));
        k_blap<<<1, 1, 0, s>>>(&ctl->t_q, &ctl->q_ns);
        NIDO_LAUNCH_CHECK();
        NIDO_CUDA_TRY(cudaMemsetAsync(B->counters, 0, sizeof(int64_t) * 4, s));
        k_control<<<grid_for((int64_t)ql.ids.size(), 128), 128, 0, s>>>(
            B->llist, (int)ql.ids.size(), B->qnew, B->Q, B->loops_phase, B->loops_total, B->giter, B->grest, tau,
            p->max_iter, g->gbase, reinterpret_cast<unsigned long long*>(B->counters));
        NIDO_LAUNCH_CHECK();
        k_batch_cond<<<1, 1, 0, s>>>(reinterpret_cast<unsigned long long*>(B->counters), ctl, listed_v, h);
        NIDO_LAUNCH_CHECK();
        return restore_listed(B->counters + 1);
      };
      const int bst = body();
      cudaGraph_t captured = nullptr;
      const cudaError_t ce = cudaStreamEndCapture(s, &captured);
      if (bst != NIDO_OK) return bst;
      if (ce != cudaSuccess) return nido_set_error(NIDO_E_CUDA, "sweep-loop capture failed: %s", cudaGetErrorString(ce));
      const uint64_t body_kernels = nido_launch_count() - l0;
      const cudaError_t ie = cudaGraphInstantiate(&lg.exec, lg.graph, 0);
      if (ie != cudaSuccess) {
        lg.exec = nullptr;
        return nido_set_error(NIDO_E_CUDA, "sweep-loop graph instantiation failed: %s", cudaGetErrorString(ie));
      }
      st.host_ms[7] += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - tb0).count();
      NIDO_CUDA_TRY(cudaGraphLaunch(lg.exec, s));
      BatchCtl hc;
      NIDO_CUDA_TRY(cudaMemcpyAsync(&hc, ctl, sizeof(hc), cudaMemcpyDeviceToHost, s));
      NIDO_CUDA_TRY(cudaStreamSynchronize(s));
      if (hc.sweeps > 1) nido_count_launches(body_kernels * (uint64_t)(hc.sweeps - 1));
      st.move_launches += (int64_t)nb * hc.sweeps;
      st.edges_scanned += (double)listed_e * (double)hc.sweeps;
      st.move_bytes += (16.0 * (double)listed_e + 32.0 * (double)listed_vertices(g)) * (double)hc.sweeps;
      st.total_loops += hc.sweeps;
      st.move_ms += hc.move_ns * 1e-6;
      st.q_ms += hc.q_ns * 1e-6;
      for (int i = 0; i < 4; ++i) cnt[i] = (unsigned long long)hc.cnt[i];
      return NIDO_OK;
    };
    while (n_iter > 0) {
      bool ran_on_device = false;
      const bool want_device = p->host_loop == 2;
      if (want_device && g->ctx->device_loop) {
        bool unsupported = false;
        NIDO_TRY(device_sweeps(&unsupported));
        if (unsupported) g->ctx->device_loop = false;
        ran_on_device = !unsupported;
      }
      if (ran_on_device) {
        n_iter = (int64_t)cnt[0];
      } else {
      NIDO_CUDA_TRY(cudaEventRecord(ev[0], s));
      for (int b = 0; b < nb; ++b) {
        NIDO_TRY(launch_move(g, b, p->tie_mode, nullptr, nullptr));
        NIDO_TRY(commit_batch(b));
      }
      NIDO_CUDA_TRY(cudaEventRecord(ev[1], s));
      st.move_launches += nb;
      st.edges_scanned += (double)listed_e;
      st.move_bytes += 16.0 * (double)listed_e + 32.0 * (double)listed_vertices(g);
      ++st.total_loops;
      NIDO_CUDA_TRY(cudaEventRecord(ev[2], s));
      NIDO_TRY(batch_modularity(B, ql, B->qnew));
      NIDO_CUDA_TRY(cudaEventRecord(ev[3], s));
      NIDO_CUDA_TRY(cudaMemsetAsync(B->counters, 0, sizeof(int64_t) * 4, s));
      k_control<<<grid_for((int64_t)ql.ids.size(), 128), 128, 0, s>>>(
          B->llist, (int)ql.ids.size(), B->qnew, B->Q, B->loops_phase, B->loops_total, B->giter, B->grest, tau,
          p->max_iter, g->gbase, reinterpret_cast<unsigned long long*>(B->counters));
      NIDO_LAUNCH_CHECK();
      NIDO_CUDA_TRY(cudaMemcpyAsync(cnt, B->counters, sizeof(cnt), cudaMemcpyDeviceToHost, s));
      NIDO_CUDA_TRY(cudaStreamSynchronize(s));
      float ms = 0.f;
      NIDO_CUDA_TRY(cudaEventElapsedTime(&ms, ev[0], ev[1]));
      st.move_ms += ms;
      NIDO_CUDA_TRY(cudaEventElapsedTime(&ms, ev[2], ev[3]));
      st.q_ms += ms;
      if (cnt[1]) NIDO_TRY(restore_listed(nullptr));
      n_iter = (int64_t)cnt[0];
      }
      lap(1);
      // drop stopped graphs from the tier lists once a quarter of the listed
      // vertices belong to them
      if (n_iter > 0 && 4 * (int64_t)cnt[2] < 3 * listed_v) {
        NIDO_CUDA_TRY(cudaMemcpyAsync(flags.data(), B->giter, sizeof(int32_t) * ng, cudaMemcpyDeviceToHost, s));
        NIDO_CUDA_TRY(cudaStreamSynchronize(s));
        std::vector<int32_t> it;
        listed_v = listed_e = 0;
        for (int32_t i : act)
          if (flags[i]) { it.push_back(i); listed_v += base[i + 1] - base[i]; listed_e += edges[i]; }
        NIDO_TRY(batch_list(B, it, base, &ql, true));
        lap(2);
      }
    }
    // phase end: aggregate the graphs that gained more than tau
    NIDO_CUDA_TRY(cudaMemsetAsync(B->counters, 0, sizeof(int64_t) * 4, s));
    k_phase_end<<<grid_for(np, 128), 128, 0, s>>>(B->plist, np, B->Q, B->Qold, tau_phase, B->gagg, B->gfin, B->phases,
                                                  reinterpret_cast<unsigned long long*>(B->counters));
    NIDO_LAUNCH_CHECK();
    NIDO_CUDA_TRY(cudaMemcpyAsync(cnt, B->counters, sizeof(cnt), cudaMemcpyDeviceToHost, s));
    NIDO_CUDA_TRY(cudaStreamSynchronize(s));
    ++phase;
    if (phase - 1 < 200) {
      st.nv_phase[phase - 1] = listed_v;
      st.ne_phase[phase - 1] = g->ne;
    }
    // graphs that do not aggregate are finished: their clustering is final
    NIDO_CUDA_TRY(cudaMemcpyAsync(flags.data(), B->gagg, sizeof(int32_t) * ng, cudaMemcpyDeviceToHost, s));
    NIDO_CUDA_TRY(cudaStreamSynchronize(s));
    {
      std::vector<int32_t> em;
      for (int32_t i = 0; i < ng; ++i)
        if (!emitted[i] && !flags[i]) { em.push_back(i); emitted[i] = 1; }
      NIDO_TRY(emit(em));
    }
    if (cnt[3] == 0) {
      lap(3);
      break;
    }
    k_drop<<<grid_for(g->nv, kThreads), kThreads, 0, s>>>(g->nv, B->gid, B->gagg, g->comm);
    NIDO_LAUNCH_CHECK();
    int done = 0;
    NIDO_CUDA_TRY(cudaEventRecord(re.a0, s));
    NIDO_TRY(launch_aggregation(g, &done));
    NIDO_CUDA_TRY(cudaEventRecord(re.a1, s));
    std::swap(g->gbase, g->gbase2);  // the clustering is in the new numbering either way
    k_post_agg<<<grid_for(np, 128), 128, 0, s>>>(B->plist, np, g->gbase2, g->gbase, B->gagg, B->gfin);
    NIDO_LAUNCH_CHECK();
    // graphs whose coarsening kept their size or left one vertex are
    // finished too (their vertices leave the union at the next coarsening)
    NIDO_CUDA_TRY(cudaMemcpyAsync(flags.data(), B->gfin, sizeof(int32_t) * ng, cudaMemcpyDeviceToHost, s));
    NIDO_CUDA_TRY(cudaStreamSynchronize(s));
    {
      float ams = 0.f;
      NIDO_CUDA_TRY(cudaEventElapsedTime(&ams, re.a0, re.a1));
      st.agg_ms += ams;
    }
    {
      std::vector<int32_t> em;
      for (int32_t i = 0; i < ng; ++i)
        if (!emitted[i] && flags[i]) { em.push_back(i); emitted[i] = 1; }
      NIDO_TRY(emit(em));
    }
    lap(3);
    if (done) break;  // every graph kept its size or collapsed: all finished
  }
  {  // graphs still running when the phase cap ended the loop
    std::vector<int32_t> em;
    for (int32_t i = 0; i < ng; ++i)
      if (!emitted[i]) { em.push_back(i); emitted[i] = 1; }
    NIDO_TRY(emit(em));
  }
  lap(3);
  NIDO_CUDA_TRY(cudaEventRecord(t1, s));
  NIDO_CUDA_TRY(cudaEventSynchronize(t1));
  float tot = 0.f;
  NIDO_CUDA_TRY(cudaEventElapsedTime(&tot, t0, t1));
  int64_t nerr = 0;
  NIDO_CUDA_TRY(cudaMemcpyAsync(&nerr, g->dcount + 1, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
  NIDO_CUDA_TRY(cudaStreamSynchronize(s));
  if (nerr)
    return nido_set_error(NIDO_E_CUDA, "a move kernel gave up %lld times (hash-table probe limit or bounded wait)",
                          (long long)nerr);
  st.total_ms = tot;
  st.phases = phase;
  if (out_comm) NIDO_CUDA_TRY(cudaMemcpyAsync(out_comm, B->outc, sizeof(int64_t) * g->nv0, cudaMemcpyDeviceToHost, s));
  if (out_q) NIDO_CUDA_TRY(cudaMemcpyAsync(out_q, B->Q, sizeof(double) * ng, cudaMemcpyDeviceToHost, s));
  if (out_phases) NIDO_CUDA_TRY(cudaMemcpyAsync(out_phases, B->phases, sizeof(int64_t) * ng, cudaMemcpyDeviceToHost, s));
  if (out_loops) NIDO_CUDA_TRY(cudaMemcpyAsync(out_loops, B->loops_total, sizeof(int64_t) * ng, cudaMemcpyDeviceToHost, s));
  NIDO_CUDA_TRY(cudaStreamSynchronize(s));
  lap(5);
  st.kernel_launches = (int64_t)(nido_launch_count() - launches0);
  if (stats) *stats = st;
  return NIDO_OK;
}

extern "C" int nido_batch_size(nido_batch B, int32_t* ngraphs, int64_t* nv, int64_t* ne) {
  if (!B) return nido_set_error(NIDO_E_INVALID, "null batch");
  if (ngraphs) *ngraphs = B->ng;
  if (nv) *nv = B->g->nv0;
  if (ne) *ne = B->g->ne0;
  return NIDO_OK;
}
