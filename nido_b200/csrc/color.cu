// color.cu -- colouring for -c (Graph::coloring, graph.cpp:548-694).
//
// The reference colours with one racy parallel greedy pass over random
// priorities (graph.cpp:572-606) and then relabels the CSR so colour classes
// are contiguous, ordered by (colour, vertex id) (graph.cpp:611-693).  Here
// the colouring is Jones-Plassmann-Luby on the device: in every round each
// uncoloured vertex whose (hashed priority, id) beats all uncoloured
// neighbours takes the smallest colour unused by its neighbours.  The result
// is a proper colouring and depends only on the graph and the seed.  The
// relabel follows the reference's contract exactly.
#include <algorithm>
#include <vector>

#include "common.cuh"
#include "engine.cuh"
#include "primitives.cuh"

namespace nido {
namespace {

__device__ __forceinline__ unsigned long long prio(uint64_t seed, int v) {
  unsigned long long z = seed + 0x9E3779B97F4A7C15ull * (unsigned long long)(v + 1);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

// one JPL round, one warp per vertex
__global__ void k_jpl_round(const int64_t* __restrict__ off, const int32_t* __restrict__ adj, int64_t nv,
                            uint64_t seed, const int32_t* __restrict__ cin, int32_t* __restrict__ cout,
                            unsigned long long* __restrict__ remaining) {
  const int lane = threadIdx.x & 31;
  const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t v = warp; v < nv; v += nw) {
    if (cin[v] >= 0) continue;  // warp-uniform
    const unsigned long long pv = prio(seed, (int)v);
    const int64_t s = off[v], e = off[v + 1];
    bool beaten = false;
    for (int64_t j = s + lane; j < e; j += 32) {
      const int u = adj[j];
      if (u == v || cin[u] >= 0) continue;
      const unsigned long long pu = prio(seed, u);
      if (pu > pv || (pu == pv && u > v)) beaten = true;
    }
    if (__any_sync(NIDO_FULL_MASK, beaten)) {
      if (lane == 0) atomicAdd(remaining, 1ull);
      continue;
    }
    // smallest colour not used by a coloured neighbour, 64 colours per window
    for (int base = 0;; base += 64) {
      unsigned long long used = 0;
      for (int64_t j = s + lane; j < e; j += 32) {
        const int c = cin[adj[j]];
        if (c >= base && c < base + 64) used |= 1ull << (c - base);
      }
      const unsigned lo = __reduce_or_sync(NIDO_FULL_MASK, (unsigned)used);
      const unsigned hi = __reduce_or_sync(NIDO_FULL_MASK, (unsigned)(used >> 32));
      const unsigned long long all = ((unsigned long long)hi << 32) | lo;
      if (all != ~0ull) {
        if (lane == 0) cout[v] = base + __ffsll((long long)~all) - 1;
        break;
      }
    }
  }
}

// largest colour + 1 (rem zeroed by the caller's last round, which found none left)
__global__ void k_max_color(const int32_t* __restrict__ c, int64_t n, unsigned long long* __restrict__ out) {
  unsigned long long m = 0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    m = max(m, (unsigned long long)(c[i] + 1));
  m = __reduce_max_sync(NIDO_FULL_MASK, (unsigned)m);
  if ((threadIdx.x & 31) == 0 && m) atomicMax(out, m);
}

__global__ void k_copy_i32(const int32_t* __restrict__ x, int32_t* __restrict__ y, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    y[i] = x[i];
}

__global__ void k_narrow_ids(const int64_t* __restrict__ x, int32_t* __restrict__ y, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    y[i] = (int32_t)x[i];
}

__global__ void k_color_keys(const int64_t* __restrict__ colors, int64_t nv, uint32_t* __restrict__ keys,
                             uint32_t* __restrict__ vals) {
  for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < nv; v += (int64_t)gridDim.x * blockDim.x) {
    keys[v] = (uint32_t)colors[v];
    vals[v] = (uint32_t)v;
  }
}

__global__ void k_relabel_prep(const uint32_t* __restrict__ order, const int64_t* __restrict__ off, int64_t nv,
                               int64_t* __restrict__ orders, int64_t* __restrict__ ndeg,
                               int64_t* __restrict__ new_orders) {
  for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < nv; p += (int64_t)gridDim.x * blockDim.x) {
    const uint32_t v = order[p];
    orders[v] = p;
    new_orders[p] = v;
    ndeg[p] = off[v + 1] - off[v];
  }
}

__global__ void k_relabel_edges(const uint32_t* __restrict__ order, const int64_t* __restrict__ off,
                                const int64_t* __restrict__ adj, const double* __restrict__ w,
                                const int64_t* __restrict__ orders, const int64_t* __restrict__ noff,
                                int64_t nv, int64_t* __restrict__ nadj, double* __restrict__ nw) {
  const int lane = threadIdx.x & 31;
  const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nws = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t p = warp; p < nv; p += nws) {
    const uint32_t v = order[p];
    const int64_t s = off[v], d = off[v + 1] - s, t = noff[p];
    for (int64_t j = lane; j < d; j += 32) {
      nadj[t + j] = orders[adj[s + j]];
      nw[t + j] = w[s + j];
    }
  }
}

struct DevBuf {
  void* p = nullptr;
  cudaStream_t s = nullptr;
  ~DevBuf() { if (p) cudaFreeAsync(p, s); }
};

template <typename T>
int take(DevBuf& b, cudaStream_t s, T** out, int64_t n) {
  b.s = s;
  NIDO_CUDA_TRY(cudaMallocAsync(&b.p, sizeof(T) * (size_t)(n > 0 ? n : 1), s));
  *out = (T*)b.p;
  return NIDO_OK;
}

int check_csr(const nido_csr* in) {
  if (!in || !in->off || (in->ne > 0 && (!in->adj || !in->w)))
    return nido_set_error(NIDO_E_INVALID, "colouring: null graph");
  if (in->nv >= ((int64_t)1 << 31) - 1) return nido_set_error(NIDO_E_TOO_LARGE, "too many vertices");
  for (int64_t i = 0; i < in->ne; ++i)
    if (in->adj[i] < 0 || in->adj[i] >= in->nv)
      return nido_set_error(NIDO_E_INVALID, "neighbour id out of range at %lld", (long long)i);
  return NIDO_OK;
}

}  // namespace

// JPL colouring of the graph's current (possibly coarse) CSR into colors
// (device, nv entries); *ncolors = largest colour + 1.  Temporaries come from
// the scratch arena, which is free again on return.
int color_current_graph(nido_graph_s* g, uint64_t seed, int32_t* colors, int64_t* ncolors) {
  cudaStream_t s = g->ctx->stream;
  const int64_t nv = g->nv;
  *ncolors = 0;
  if (nv == 0) return NIDO_OK;
  Arena ar(g->scratch, g->scratch_bytes);
  int32_t* c1 = ar.take<int32_t>(nv);
  unsigned long long* rem = ar.take<unsigned long long>(1);
  if (!c1 || !rem) return nido_set_error(NIDO_E_NOMEM, "scratch arena too small (colouring)");
  NIDO_CUDA_TRY(cudaMemsetAsync(colors, 0xff, 4 * nv, s));
  NIDO_CUDA_TRY(cudaMemsetAsync(c1, 0xff, 4 * nv, s));
  // every round colours at least the uncoloured vertex of largest (priority,
  // id), so nv rounds always suffice
  for (int64_t round = 0; round <= nv; ++round) {
    NIDO_CUDA_TRY(cudaMemsetAsync(rem, 0, 8, s));
    k_jpl_round<<<kSMs * 16, 256, 0, s>>>(g->off, g->adj, nv, seed, colors, c1, rem);
    NIDO_LAUNCH_CHECK();
    k_copy_i32<<<kSMs * 8, 256, 0, s>>>(c1, colors, nv);
    NIDO_LAUNCH_CHECK();
    unsigned long long r = 0;
    NIDO_CUDA_TRY(cudaMemcpyAsync(&r, rem, 8, cudaMemcpyDeviceToHost, s));
    NIDO_CUDA_TRY(cudaStreamSynchronize(s));
    if (r == 0) break;
  }
  NIDO_CUDA_TRY(cudaMemsetAsync(rem, 0, 8, s));
  k_max_color<<<kSMs * 4, 256, 0, s>>>(colors, nv, rem);
  NIDO_LAUNCH_CHECK();
  unsigned long long mx = 0;
  NIDO_CUDA_TRY(cudaMemcpyAsync(&mx, rem, 8, cudaMemcpyDeviceToHost, s));
  NIDO_CUDA_TRY(cudaStreamSynchronize(s));
  *ncolors = (int64_t)mx;
  return NIDO_OK;
}
}  // namespace nido

using namespace nido;

extern "C" int nido_color(nido_ctx ctx, const nido_csr* in, uint64_t seed, int64_t* colors, int64_t* ncolors) {
  if (!ctx || !colors) return nido_set_error(NIDO_E_INVALID, "nido_color: null argument");
  NIDO_TRY(check_csr(in));
  NIDO_CUDA_TRY(cudaSetDevice(ctx->device));
  cudaStream_t s = ctx->stream;
  const int64_t nv = in->nv, ne = in->ne;
  DevBuf b0, b1, b2, b3, b4, b5;
  int64_t *off, *adj64;
  int32_t *adj, *c0, *c1;
  unsigned long long* rem;
  NIDO_TRY(take(b0, s, &off, nv + 1));
  NIDO_TRY(take(b1, s, &adj64, ne));
  NIDO_TRY(take(b2, s, &adj, ne));
  NIDO_TRY(take(b3, s, &c0, nv));
  NIDO_TRY(take(b4, s, &c1, nv));
  NIDO_TRY(take(b5, s, &rem, 1));
  NIDO_CUDA_TRY(cudaMemcpyAsync(off, in->off, 8 * (nv + 1), cudaMemcpyHostToDevice, s));
  if (ne) NIDO_CUDA_TRY(cudaMemcpyAsync(adj64, in->adj, 8 * ne, cudaMemcpyHostToDevice, s));
  k_narrow_ids<<<kSMs * 8, 256, 0, s>>>(adj64, adj, ne);
  NIDO_LAUNCH_CHECK();
  NIDO_CUDA_TRY(cudaMemsetAsync(c0, 0xff, 4 * nv, s));
  NIDO_CUDA_TRY(cudaMemsetAsync(c1, 0xff, 4 * nv, s));
  for (int round = 0; round < 1 << 20; ++round) {
    NIDO_CUDA_TRY(cudaMemsetAsync(rem, 0, 8, s));
    k_jpl_round<<<kSMs * 16, 256, 0, s>>>(off, adj, nv, seed, c0, c1, rem);
    NIDO_LAUNCH_CHECK();
    k_copy_i32<<<kSMs * 8, 256, 0, s>>>(c1, c0, nv);
    NIDO_LAUNCH_CHECK();
    unsigned long long r = 0;
    NIDO_CUDA_TRY(cudaMemcpyAsync(&r, rem, 8, cudaMemcpyDeviceToHost, s));
    NIDO_CUDA_TRY(cudaStreamSynchronize(s));
    if (r == 0) break;
  }
  std::vector<int32_t> h(nv);
  NIDO_CUDA_TRY(cudaMemcpyAsync(h.data(), c0, 4 * nv, cudaMemcpyDeviceToHost, s));
  NIDO_CUDA_TRY(cudaStreamSynchronize(s));
  int64_t nc = 0;
  for (int64_t v = 0; v < nv; ++v) {
    colors[v] = h[v];
    nc = std::max<int64_t>(nc, (int64_t)h[v] + 1);
  }
  if (ncolors) *ncolors = nc;
  return NIDO_OK;
}

extern "C" int nido_color_relabel(nido_ctx ctx, const nido_csr* in, const int64_t* colors, nido_csr* out,
                                  int64_t* new_orders) {
  if (!ctx || !colors || !out || !out->off || !new_orders || (in && in->ne > 0 && (!out->adj || !out->w)))
    return nido_set_error(NIDO_E_INVALID, "nido_color_relabel: null argument");
  NIDO_TRY(check_csr(in));
  const int64_t nv = in->nv, ne = in->ne;
  int64_t maxc = 0;
  for (int64_t v = 0; v < nv; ++v) {
    if (colors[v] < 0 || colors[v] >= ((int64_t)1 << 31))
      return nido_set_error(NIDO_E_INVALID, "colour out of range at vertex %lld", (long long)v);
    maxc = std::max(maxc, colors[v]);
  }
  NIDO_CUDA_TRY(cudaSetDevice(ctx->device));
  cudaStream_t s = ctx->stream;
  DevBuf b[12];
  int64_t *off, *adj, *col, *orders, *noff, *nadj, *nord, *temp;
  double *w, *nw;
  uint32_t *k0, *v0, *k1, *v1;
  const int64_t tmpn = std::max(radix_temp_elems(nv), scan_temp_elems(nv + 1));
  NIDO_TRY(take(b[0], s, &off, nv + 1));
  NIDO_TRY(take(b[1], s, &adj, ne));
  NIDO_TRY(take(b[2], s, &w, ne));
  NIDO_TRY(take(b[3], s, &col, nv));
  NIDO_TRY(take(b[4], s, &orders, nv));
  NIDO_TRY(take(b[5], s, &noff, nv + 1));
  NIDO_TRY(take(b[6], s, &nadj, ne));
  NIDO_TRY(take(b[7], s, &nw, ne));
  NIDO_TRY(take(b[8], s, &nord, nv));
  NIDO_TRY(take(b[9], s, &temp, tmpn));
  NIDO_TRY(take(b[10], s, &k0, 4 * nv));
  v0 = k0 + nv; k1 = v0 + nv; v1 = k1 + nv;
  NIDO_CUDA_TRY(cudaMemcpyAsync(off, in->off, 8 * (nv + 1), cudaMemcpyHostToDevice, s));
  if (ne) {
    NIDO_CUDA_TRY(cudaMemcpyAsync(adj, in->adj, 8 * ne, cudaMemcpyHostToDevice, s));
    NIDO_CUDA_TRY(cudaMemcpyAsync(w, in->w, 8 * ne, cudaMemcpyHostToDevice, s));
  }
  NIDO_CUDA_TRY(cudaMemcpyAsync(col, colors, 8 * nv, cudaMemcpyHostToDevice, s));
  k_color_keys<<<kSMs * 8, 256, 0, s>>>(col, nv, k0, v0);
  NIDO_LAUNCH_CHECK();
  int bits = 0;
  while (((int64_t)1 << bits) <= maxc) ++bits;
  NIDO_TRY(radix_sort_pairs(k0, v0, k1, v1, nv, bits, temp, s));
  k_relabel_prep<<<kSMs * 8, 256, 0, s>>>(v0, off, nv, orders, noff, nord);
  NIDO_LAUNCH_CHECK();
  NIDO_TRY(scan_exclusive_i64(noff, noff, nv, temp, s));
  k_relabel_edges<<<kSMs * 16, 256, 0, s>>>(v0, off, adj, w, orders, noff, nv, nadj, nw);
  NIDO_LAUNCH_CHECK();
  out->nv = nv;
  out->ne = ne;
  NIDO_CUDA_TRY(cudaMemcpyAsync(out->off, noff, 8 * (nv + 1), cudaMemcpyDeviceToHost, s));
  if (ne) {
    NIDO_CUDA_TRY(cudaMemcpyAsync(out->adj, nadj, 8 * ne, cudaMemcpyDeviceToHost, s));
    NIDO_CUDA_TRY(cudaMemcpyAsync(out->w, nw, 8 * ne, cudaMemcpyDeviceToHost, s));
  }
  NIDO_CUDA_TRY(cudaMemcpyAsync(new_orders, nord, 8 * nv, cudaMemcpyDeviceToHost, s));
  NIDO_CUDA_TRY(cudaStreamSynchronize(s));
  return NIDO_OK;
}
