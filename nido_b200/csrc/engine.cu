// engine.cu -- C ABI of the engine: contexts, graph upload, the step-level
// operators of the reference's GraphGPU (graph_gpu.hpp:168-247) and the
// whole-run driver LouvainGPU::run (louvain_gpu.cpp:6-139).
#include <fcntl.h>
#include <omp.h>
#include <stdio.h>
#include <string.h>
#include <unistd.h>

#include <algorithm>
#include <chrono>
#include <new>
#include <vector>

#include "common.cuh"
#include "engine.cuh"
#include "primitives.cuh"

using nido::Arena;

namespace nido {
// Blocks of a context that is not stream-ordered: cudaMalloc maps new memory
// (tens to hundreds of ms for the few GB of a large graph) and cudaFree waits
// for the whole device, so freed blocks stay with the context and later
// requests reuse them: the smallest free block of at least the request and at
// most twice it.  Sizes are rounded (512 B; 2 MiB from 1 MiB up).  Every use
// of a block is on the context's stream or on side streams joined back to it,
// so a reused block's new work is ordered after its old work.  When cudaMalloc
// fails the free blocks are released and the call retried; destroying the
// context releases them.
namespace {
size_t block_size(size_t bytes) {
  const size_t g = bytes >= ((size_t)1 << 20) ? ((size_t)2 << 20) : (size_t)512;
  return (std::max<size_t>(bytes, 1) + g - 1) / g * g;
}
}  // namespace

cudaError_t raw_alloc(nido_ctx_s* ctx, void** p, size_t bytes) {
  if (ctx->async_alloc)
    return ctx->pool ? cudaMallocFromPoolAsync(p, bytes, ctx->pool, ctx->stream)
                     : cudaMallocAsync(p, bytes, ctx->stream);
  const size_t b = block_size(bytes);
  auto it = ctx->free_blocks.lower_bound(b);
  if (it != ctx->free_blocks.end() && it->first <= 2 * b) {
    *p = it->second;
    ctx->live_blocks[it->second] = it->first;
    ctx->cached_bytes -= it->first;
    ctx->free_blocks.erase(it);
    return cudaSuccess;
  }
  cudaError_t e = cudaMalloc(p, b);
  if (e == cudaErrorMemoryAllocation && !ctx->free_blocks.empty()) {
    cudaGetLastError();
    release_cached(ctx);
    e = cudaMalloc(p, b);
  }
  if (e == cudaSuccess) ctx->live_blocks[*p] = b;
  return e;
}

void raw_free(nido_ctx_s* ctx, void* p) {
  if (!p) return;
  if (ctx->async_alloc) {
    cudaFreeAsync(p, ctx->stream);
    return;
  }
  auto it = ctx->live_blocks.find(p);
  if (it == ctx->live_blocks.end()) {  // not from raw_alloc
    cudaFree(p);
    return;
  }
  ctx->free_blocks.emplace(it->second, p);
  ctx->cached_bytes += it->second;
  ctx->live_blocks.erase(it);
}

cudaError_t pinned_buffer(nido_ctx_s* ctx, size_t bytes, void** p) {
  if (bytes > ctx->pinned_bytes) {
    if (ctx->pinned) cudaFreeHost(ctx->pinned);
    ctx->pinned = nullptr;
    ctx->pinned_bytes = 0;
    const cudaError_t e = cudaHostAlloc(&ctx->pinned, bytes, cudaHostAllocDefault);
    if (e != cudaSuccess) return e;
    ctx->pinned_bytes = bytes;
  }
  *p = ctx->pinned;
  return cudaSuccess;
}

void release_cached(nido_ctx_s* ctx) {
  if (ctx->free_blocks.empty()) return;
  cudaStreamSynchronize(ctx->stream);
  for (auto& kv : ctx->free_blocks) cudaFree(kv.second);
  ctx->free_blocks.clear();
  ctx->cached_bytes = 0;
}
}  // namespace nido

namespace {

template <typename T>
int dev_alloc(nido_ctx ctx, T** p, int64_t n) {
  const size_t bytes = sizeof(T) * (size_t)(n > 0 ? n : 1);
  if (ctx->budget && ctx->used + bytes > ctx->budget)
    return nido_set_error(NIDO_E_NOMEM, "HBM budget of %zu bytes exceeded", ctx->budget);
  cudaError_t e = nido::raw_alloc(ctx, (void**)p, bytes);
  if (e != cudaSuccess) {
    *p = nullptr;
    cudaGetLastError();
    return nido_set_error(NIDO_E_NOMEM, "cudaMalloc(%zu) failed: %s", bytes, cudaGetErrorString(e));
  }
  ctx->used += bytes;
  return NIDO_OK;
}

// Page-locked host memory mapped into the device's address space (with
// unified addressing the host pointer is also the device pointer).
template <typename T>
int host_alloc(T** p, int64_t n) {
  const size_t bytes = sizeof(T) * (size_t)(n > 0 ? n : 1);
  void* h = nullptr;
  const cudaError_t e = cudaHostAlloc(&h, bytes, cudaHostAllocMapped | cudaHostAllocPortable);
  if (e != cudaSuccess) {
    *p = nullptr;
    cudaGetLastError();
    return nido_set_error(NIDO_E_NOMEM, "cudaHostAlloc(%zu) failed: %s", bytes, cudaGetErrorString(e));
  }
  void* d = nullptr;
  const cudaError_t e2 = cudaHostGetDevicePointer(&d, h, 0);
  if (e2 != cudaSuccess || d != h) {
    cudaFreeHost(h);
    *p = nullptr;
    return nido_set_error(NIDO_E_CUDA, "mapped host memory is not addressable at its host address");
  }
  *p = static_cast<T*>(h);
  return NIDO_OK;
}

void dev_free(nido_ctx ctx, void* p, size_t bytes) {
  if (p) {
    nido::raw_free(ctx, p);
    ctx->used -= std::min(ctx->used, bytes);
  }
}

// Narrow int64 neighbour ids to int32 while checking 0 <= id < nv; offsets
// must be non-decreasing and start at 0.
__global__ void k_narrow(const int64_t* __restrict__ adj64, int64_t ne, int64_t nv,
                         int32_t* __restrict__ adj, const int64_t* __restrict__ off,
                         unsigned long long* __restrict__ bad) {
  unsigned long long b = 0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < ne;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t x = adj64[i];
    if (x < 0 || x >= nv) ++b;
    adj[i] = (int32_t)x;
  }
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nv;
       i += (int64_t)gridDim.x * blockDim.x)
    if (off[i + 1] < off[i]) ++b;
  if (b) atomicAdd(bad, b);
}

__global__ void k_iota(int32_t* __restrict__ x, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    x[i] = (int32_t)i;
}

__global__ void k_widen(const int32_t* __restrict__ x, int64_t n, int64_t* __restrict__ y) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    y[i] = x[i];
}

// comm ids from int64 with range check; newc gets the same ids
__global__ void k_set_ids(const int64_t* __restrict__ c64, int64_t nv, int32_t* __restrict__ comm,
                          int32_t* __restrict__ newc, unsigned long long* __restrict__ bad) {
  unsigned long long b = 0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nv;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t c = c64[i];
    if (c < 0 || c >= nv) ++b;
    const int32_t ci = (c < 0 || c >= nv) ? 0 : (int32_t)c;
    comm[i] = ci;
    newc[i] = ci;
  }
  if (b) atomicAdd(bad, b);
}

constexpr unsigned kGrid = 148 * 8;

int prepare_phase(nido_graph g) {
  NIDO_TRY(nido::launch_vertex_weights(g));
  NIDO_TRY(nido::launch_mass(g));
  g->bins_valid = false;
  NIDO_TRY(nido::build_batches(g));
  return NIDO_OK;
}

}  // namespace

namespace nido {
int graph_prepare_phase(nido_graph g) { return prepare_phase(g); }
int device_alloc(nido_ctx ctx, void** p, size_t bytes) {
  char* q = nullptr;
  const int st = dev_alloc(ctx, &q, (int64_t)bytes);
  *p = q;
  return st;
}
void device_free(nido_ctx ctx, void* p, size_t bytes) { dev_free(ctx, p, bytes); }
}

extern "C" int nido_ctx_create(int device, size_t hbm_budget_bytes, nido_ctx* out) {
  if (!out) return nido_set_error(NIDO_E_INVALID, "nido_ctx_create: null output");
  *out = nullptr;
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
    cudaGetLastError();
    return nido_set_error(NIDO_E_NODEVICE, "no CUDA device available");
  }
  if (device < 0 || device >= n) return nido_set_error(NIDO_E_INVALID, "device %d out of range", device);
  NIDO_CUDA_TRY(cudaSetDevice(device));
  cudaDeviceProp prop;
  NIDO_CUDA_TRY(cudaGetDeviceProperties(&prop, device));
  if (prop.major != 10)
    return nido_set_error(NIDO_E_NODEVICE, "device %d is sm_%d%d; this build targets sm_100a", device,
                          prop.major, prop.minor);
  NIDO_TRY(nido::move_init_attributes());
  nido_ctx ctx = new (std::nothrow) nido_ctx_s();
  if (!ctx) return nido_set_error(NIDO_E_NOMEM, "host allocation failed");
  ctx->device = device;
  ctx->budget = hbm_budget_bytes;
  NIDO_CUDA_TRY(cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking));
  NIDO_CUDA_TRY(cudaEventCreate(&ctx->ev0));
  NIDO_CUDA_TRY(cudaEventCreate(&ctx->ev1));
  for (int i = 0; i < 2; ++i) {
    NIDO_CUDA_TRY(cudaStreamCreateWithFlags(&ctx->aux[i], cudaStreamNonBlocking));
    NIDO_CUDA_TRY(cudaEventCreateWithFlags(&ctx->join_ev[i], cudaEventDisableTiming));
  }
  NIDO_CUDA_TRY(cudaEventCreateWithFlags(&ctx->fork_ev, cudaEventDisableTiming));
  *out = ctx;
  return NIDO_OK;
}

extern "C" int nido_ctx_destroy(nido_ctx ctx) {
  if (!ctx) return NIDO_OK;
  cudaSetDevice(ctx->device);
  cudaStreamSynchronize(ctx->stream);
  cudaEventDestroy(ctx->ev0);
  cudaEventDestroy(ctx->ev1);
  for (cudaEvent_t e : ctx->move_ev) cudaEventDestroy(e);
  for (int i = 0; i < 2; ++i) {
    if (ctx->aux[i]) {
      cudaStreamSynchronize(ctx->aux[i]);
      cudaStreamDestroy(ctx->aux[i]);
    }
    if (ctx->join_ev[i]) cudaEventDestroy(ctx->join_ev[i]);
  }
  if (ctx->fork_ev) cudaEventDestroy(ctx->fork_ev);
  nido::release_cached(ctx);
  if (ctx->pinned) cudaFreeHost(ctx->pinned);
  cudaStreamDestroy(ctx->stream);
  delete ctx;
  return NIDO_OK;
}

extern "C" int nido_ctx_trim(nido_ctx ctx, size_t* released_bytes) {
  if (!ctx) return nido_set_error(NIDO_E_INVALID, "null context");
  NIDO_CUDA_TRY(cudaSetDevice(ctx->device));
  if (released_bytes) *released_bytes = ctx->cached_bytes;
  nido::release_cached(ctx);
  return NIDO_OK;
}

extern "C" int nido_check_bounded_wait(nido_ctx ctx, int32_t* gave_up, int32_t* waited_ms) {
  if (!ctx) return nido_set_error(NIDO_E_INVALID, "null context");
  NIDO_CUDA_TRY(cudaSetDevice(ctx->device));
  return nido::check_bounded_wait(ctx, gave_up, waited_ms);
}

extern "C" int nido_ctx_sync(nido_ctx ctx) {
  if (!ctx) return nido_set_error(NIDO_E_INVALID, "null context");
  NIDO_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  return NIDO_OK;
}

extern "C" int nido_ctx_stream(nido_ctx ctx, void** stream) {
  if (!ctx || !stream) return nido_set_error(NIDO_E_INVALID, "null argument");
  *stream = (void*)ctx->stream;
  return NIDO_OK;
}

extern "C" int nido_graph_free(nido_graph g) {
  if (!g) return NIDO_OK;
  nido_ctx ctx = g->ctx;
  cudaSetDevice(ctx->device);
  cudaStreamSynchronize(ctx->stream);
  const int64_t V = g->cap_v, E = g->cap_e;
  dev_free(ctx, g->off0, 8 * (V + 1)); dev_free(ctx, g->offA, 8 * (V + 1));
  dev_free(ctx, g->off2, 8 * (V + 1));
  if (g->host_edges) {
    for (void* p : {(void*)g->adj0, (void*)g->adjA, (void*)g->adj2, (void*)g->w0, (void*)g->wA, (void*)g->w2})
      if (p) cudaFreeHost(p);
  } else {
    dev_free(ctx, g->adj0, 4 * (E + 4)); dev_free(ctx, g->adjA, 4 * (E + 4)); dev_free(ctx, g->adj2, 4 * (E + 4));
    dev_free(ctx, g->w0, 8 * (E + 4)); dev_free(ctx, g->wA, 8 * (E + 4)); dev_free(ctx, g->w2, 8 * (E + 4));
  }
  dev_free(ctx, g->k, 8 * V); dev_free(ctx, g->a, 8 * V);
  dev_free(ctx, g->comm, 4 * V); dev_free(ctx, g->newc, 4 * V);
  dev_free(ctx, g->clus, 4 * g->nv0); dev_free(ctx, g->perm, 4 * V);
  dev_free(ctx, g->dm, 64); dev_free(ctx, g->dcount, 64);
  dev_free(ctx, g->scratch, g->scratch_bytes);
  // hub-tier buffers are sized per phase outside the budget accounting
  for (void* p : {(void*)g->gkeys, (void*)g->gvals, (void*)g->gpacked, (void*)g->hub_items, (void*)g->hub_v, (void*)g->hub_capv,
                  (void*)g->hub_nseg, (void*)g->hub_toff, (void*)g->hub_done, (void*)g->hub_slices,
                  (void*)g->hub_slice_first, (void*)g->hub_res, (void*)g->hub_item_first,
                  (void*)g->hub_part, (void*)g->hub_cl_v, (void*)g->agg_buf, (void*)g->pm32,
                  (void*)g->loop_buf, (void*)g->vcolor})
    nido::raw_free(ctx, p);
  for (nido_graph_s::MoveGraph& mg : g->move_graphs)
    if (mg.exec) cudaGraphExecDestroy(mg.exec);
  delete g;
  return NIDO_OK;
}

namespace {
// Every device array of a graph of nv vertices and ne edges; the caller
// fills g->off, the int64 ids (in the w2 buffer, narrowed by graph_finish)
// and g->w.
int graph_create(nido_ctx ctx, int64_t nv, int64_t ne, int32_t nbatches, nido_graph* out) {
  *out = nullptr;
  if (nv < 0 || ne < 0) return nido_set_error(NIDO_E_INVALID, "negative graph size");
  if (nv >= ((int64_t)1 << 31) - 1) return nido_set_error(NIDO_E_TOO_LARGE, "%lld vertices exceed 2^31-1", (long long)nv);
  if (nbatches < 1) return nido_set_error(NIDO_E_INVALID, "nbatches must be >= 1 (got %d)", nbatches);
  NIDO_CUDA_TRY(cudaSetDevice(ctx->device));
  nido_graph g = new (std::nothrow) nido_graph_s();
  if (!g) return nido_set_error(NIDO_E_NOMEM, "host allocation failed");
  g->ctx = ctx;
  g->nv0 = g->nv = g->cap_v = nv;
  g->ne = g->ne0 = g->cap_e = ne;
  g->nbatches = nbatches;
  g->nb_user = nbatches;
  const int64_t V = nv, E = ne;
  int st = NIDO_OK;
  // Over the context's budget, the graph keeps its edge arrays in mapped
  // page-locked host memory when what is left (vertex state, offsets,
  // scratch) fits: every kernel then reads the edges over the host link.
  {
    const size_t edge_bytes = 36 * (size_t)std::max<int64_t>(E, 1);
    const size_t vert_bytes = (size_t)nido_graph_footprint_streamed(nv, ne, nbatches);
    g->host_edges = ctx->budget && ctx->used + edge_bytes + vert_bytes > ctx->budget &&
                    ctx->used + vert_bytes <= ctx->budget;
  }
#define ALLOC(p, n) if (st == NIDO_OK) st = dev_alloc(ctx, &g->p, (n))
#define EALLOC(p, n) if (st == NIDO_OK) st = g->host_edges ? host_alloc(&g->p, (n)) : dev_alloc(ctx, &g->p, (n))
  ALLOC(off0, V + 1); ALLOC(offA, V + 1); ALLOC(off2, V + 1);
  // 4 spare entries: the move kernels' bulk copies widen an edge range to
  // 16-byte boundaries and may read up to 3 ids and 1 weight past its end
  EALLOC(adj0, E + 4); EALLOC(adjA, E + 4); EALLOC(adj2, E + 4);
  EALLOC(w0, E + 4); EALLOC(wA, E + 4); EALLOC(w2, E + 4);
#undef EALLOC
  ALLOC(k, V); ALLOC(a, V);
  ALLOC(comm, V); ALLOC(newc, V);
  ALLOC(clus, V); ALLOC(perm, V);
  ALLOC(dm, 8); ALLOC(dcount, 8);
#undef ALLOC
  // scratch: radix sort / modularity / coarsening temporaries
  g->scratch_bytes = (size_t)64 * (V + 1) + (size_t)(1 << 20) +
                     sizeof(int64_t) * (size_t)(nido::radix_temp_elems(V) + nido::scan_temp_elems(E + 1));
  if (st == NIDO_OK) st = dev_alloc(ctx, &g->scratch, (int64_t)g->scratch_bytes);
  if (st != NIDO_OK) { nido_graph_free(g); return st; }
  g->off = g->off0;
  g->adj = g->adj0;
  g->w = g->w0;
  *out = g;
  return NIDO_OK;
}

// The int64 ids travel in the (not yet used) w2 buffer.
int64_t* staged_ids(nido_graph g) { return reinterpret_cast<int64_t*>(g->w2); }

// After the CSR is on the device: narrow and check the ids and offsets, then
// k_v, m, the batches and the singleton partition of the first phase.
int graph_finish(nido_graph g) {
  cudaStream_t s = g->ctx->stream;
  const int64_t V = g->nv, E = g->ne;
  unsigned long long* bad = reinterpret_cast<unsigned long long*>(g->dcount);
  NIDO_CUDA_TRY(cudaMemsetAsync(g->dcount, 0, 8 * sizeof(int64_t), s));
  k_narrow<<<kGrid, 256, 0, s>>>(staged_ids(g), E, V, g->adj, g->off, bad);
  NIDO_LAUNCH_CHECK();
  k_iota<<<kGrid, 256, 0, s>>>(g->clus, V);
  NIDO_LAUNCH_CHECK();
  unsigned long long nbad = 0;
  NIDO_CUDA_TRY(cudaMemcpyAsync(&nbad, bad, 8, cudaMemcpyDeviceToHost, s));
  NIDO_CUDA_TRY(cudaStreamSynchronize(s));
  if (nbad) return nido_set_error(NIDO_E_INVALID, "%llu neighbour ids out of range or decreasing offsets", nbad);
  NIDO_TRY(prepare_phase(g));
  return nido::launch_singleton(g);
}

// Frees a graph whose construction failed (after its stream is idle) and
// passes the status on.
int fail_graph(nido_graph g, int st) {
  cudaStreamSynchronize(g->ctx->stream);
  nido_graph_free(g);
  return st;
}

// Vite edge records {int64 tail; double weight} to ids and weights.
__global__ void k_split_records(const longlong2* __restrict__ rec, int64_t n, int64_t* __restrict__ adj64,
                                double* __restrict__ w) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const longlong2 r = rec[i];
    adj64[i] = r.x;
    w[i] = __longlong_as_double(r.y);
  }
}

// Reads bytes [pos, pos + n) of fd into dst with `threads` concurrent
// preads; false on a short file or a read error.
bool pread_all(int fd, char* dst, int64_t n, int64_t pos, int threads) {
  bool ok = true;
  const int64_t per = (n + threads - 1) / threads;
#pragma omp parallel for num_threads(threads) schedule(static) reduction(&& : ok)
  for (int t = 0; t < threads; ++t) {
    int64_t lo = (int64_t)t * per, hi = std::min(n, lo + per);
    while (lo < hi) {
      const ssize_t r = pread(fd, dst + lo, (size_t)(hi - lo), (off_t)(pos + lo));
      if (r <= 0) { ok = false; break; }
      lo += r;
    }
  }
  return ok;
}
}  // namespace

extern "C" int nido_graph_upload(nido_ctx ctx, int64_t nv, int64_t ne, const int64_t* off,
                                 const int64_t* adj, const double* w, int32_t nbatches,
                                 nido_graph* out) {
  if (!ctx || !out || !off || (ne > 0 && (!adj || !w)))
    return nido_set_error(NIDO_E_INVALID, "nido_graph_upload: null argument");
  *out = nullptr;
  if (nv >= 0 && ne >= 0 && nv < ((int64_t)1 << 31) - 1 && (off[0] != 0 || off[nv] != ne))
    return nido_set_error(NIDO_E_INVALID, "offsets must run from 0 to ne");
  nido_graph g = nullptr;
  NIDO_TRY(graph_create(ctx, nv, ne, nbatches, &g));
  cudaStream_t s = ctx->stream;
  cudaError_t e = cudaMemcpyAsync(g->off, off, 8 * (nv + 1), cudaMemcpyHostToDevice, s);
  // cudaMemcpyDefault: the edge arrays are device or mapped host memory
  if (e == cudaSuccess && ne > 0) e = cudaMemcpyAsync(staged_ids(g), adj, 8 * ne, cudaMemcpyDefault, s);
  if (e == cudaSuccess && ne > 0) e = cudaMemcpyAsync(g->w, w, 8 * ne, cudaMemcpyDefault, s);
  if (e != cudaSuccess) return fail_graph(g, nido_set_error(NIDO_E_CUDA, "upload: %s", cudaGetErrorString(e)));
  const int st = graph_finish(g);
  if (st != NIDO_OK) return fail_graph(g, st);
  *out = g;
  return NIDO_OK;
}

// Vite binary straight to the device (graph.cpp:322-495 for the format and
// its checks): the header and offsets are read on the host; the edge records
// stream through two pinned buffers, each filled by parallel preads while the
// other is copied, and are split into ids and weights by a kernel.
extern "C" int nido_graph_upload_vite(nido_ctx ctx, const char* path, int32_t nbatches, nido_graph* out) {
  if (!ctx || !path || !out) return nido_set_error(NIDO_E_INVALID, "nido_graph_upload_vite: null argument");
  *out = nullptr;
  const int fd = open(path, O_RDONLY);
  if (fd < 0) return nido_set_error(NIDO_E_IO, " Error opening file! (%s)", path);
  struct FdGuard {
    int fd;
    ~FdGuard() { close(fd); }
  } guard{fd};
  int64_t hdr[2];
  if (!pread_all(fd, reinterpret_cast<char*>(hdr), 16, 0, 1) || hdr[0] < 0)
    return nido_set_error(NIDO_E_IO, "%s: truncated header", path);
  const int64_t nv = hdr[0];
  if (nv >= ((int64_t)1 << 31) - 1) return nido_set_error(NIDO_E_TOO_LARGE, "%lld vertices exceed 2^31-1", (long long)nv);
  const int threads = std::max(1, std::min(16, omp_get_max_threads()));
  std::vector<int64_t> off((size_t)nv + 1);
  if (!pread_all(fd, reinterpret_cast<char*>(off.data()), 8 * (nv + 1), 16, threads))
    return nido_set_error(NIDO_E_IO, "%s: truncated offsets", path);
  const int64_t ne = off[nv] - off[0];
  if (ne < 0) return nido_set_error(NIDO_E_IO, "%s: decreasing offsets", path);
  if (ne != hdr[1]) {
    printf("!!! The graph has been modified in edges\n");
    printf("Original edges: %lld\nNew edges: %lld\n", (long long)hdr[1], (long long)ne);
  }
  const int64_t base = off[0];
  for (int64_t& o : off) o -= base;
  nido_graph g = nullptr;
  NIDO_TRY(graph_create(ctx, nv, ne, nbatches, &g));
  cudaStream_t s = ctx->stream;
  const int64_t rec0 = 16 + 8 * (nv + 1);  // file position of the first record
  const int64_t chunk = std::min<int64_t>(std::max<int64_t>(ne, 1), (int64_t)1 << 22);
  int st = NIDO_OK;
  cudaError_t e = cudaMemcpyAsync(g->off, off.data(), 8 * (nv + 1), cudaMemcpyHostToDevice, s);
  char* host = nullptr;
  longlong2* dev = nullptr;
  cudaEvent_t ev[2] = {nullptr, nullptr};
  if (e == cudaSuccess) e = nido::pinned_buffer(ctx, (size_t)2 * 16 * chunk, reinterpret_cast<void**>(&host));
  if (e == cudaSuccess) e = nido::raw_alloc(ctx, reinterpret_cast<void**>(&dev), (size_t)2 * 16 * chunk);
  for (int b = 0; b < 2 && e == cudaSuccess; ++b) e = cudaEventCreateWithFlags(&ev[b], cudaEventDisableTiming);
  for (int64_t done = 0, i = 0; e == cudaSuccess && st == NIDO_OK && done < ne; ++i) {
    const int b = (int)(i & 1);
    const int64_t n = std::min(chunk, ne - done);
    if (i >= 2 && (e = cudaEventSynchronize(ev[b])) != cudaSuccess) break;  // buffer b is free again
    char* hb = host + (size_t)b * 16 * chunk;
    if (!pread_all(fd, hb, 16 * n, rec0 + 16 * done, threads)) {
      st = nido_set_error(NIDO_E_IO, "%s: truncated edge records", path);
      break;
    }
    e = cudaMemcpyAsync(dev + (size_t)b * chunk, hb, 16 * n, cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) break;
    k_split_records<<<kGrid, 256, 0, s>>>(dev + (size_t)b * chunk, n, staged_ids(g) + done, g->w + done);
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaEventRecord(ev[b], s);
    done += n;
  }
  cudaStreamSynchronize(s);
  for (cudaEvent_t x : ev)
    if (x) cudaEventDestroy(x);
  nido::raw_free(ctx, dev);
  if (st == NIDO_OK && e != cudaSuccess) st = nido_set_error(NIDO_E_CUDA, "upload_vite: %s", cudaGetErrorString(e));
  if (st == NIDO_OK) st = graph_finish(g);
  if (st != NIDO_OK) return fail_graph(g, st);
  *out = g;
  return NIDO_OK;
}

extern "C" int nido_graph_device_bytes(nido_graph g, int64_t* bytes) {
  if (!g || !bytes) return nido_set_error(NIDO_E_INVALID, "null argument");
  const int64_t V = g->cap_v, E = g->host_edges ? 0 : g->cap_e;  // mapped host edges hold no HBM
  int64_t b = 24 * (V + 1) + 36 * E + 28 * V + 4 * g->nv0 + 128 + (int64_t)g->scratch_bytes;
  b += 12 * g->gslab + 8 * g->gslab_packed + 8 * g->hub_cap_items + 4 * (g->hub_cap_hubs_v + g->hub_cap_hubs_c + g->hub_cap_hubs_s +
                                                   g->hub_cap_hubs_d) +
       8 * (g->hub_cap_hubs_t + g->hub_cap_slices + g->hub_cap_first) + g->hub_cap_res + (int64_t)g->agg_buf_bytes + 4 * g->pm32_cap;
  *bytes = b;
  return NIDO_OK;
}

extern "C" int nido_graph_host_edges(nido_graph g, int32_t* host_edges) {
  if (!g || !host_edges) return nido_set_error(NIDO_E_INVALID, "null argument");
  *host_edges = g->host_edges ? 1 : 0;
  return NIDO_OK;
}

extern "C" int nido_graph_size(nido_graph g, int64_t* nv, int64_t* ne) {
  if (!g) return nido_set_error(NIDO_E_INVALID, "null graph");
  if (nv) *nv = g->nv;
  if (ne) *ne = g->ne;
  return NIDO_OK;
}

extern "C" int nido_graph_download(nido_graph g, int64_t* off, int64_t* adj, double* w) {
  if (!g) return nido_set_error(NIDO_E_INVALID, "null graph");
  cudaStream_t s = g->ctx->stream;
  NIDO_CUDA_TRY(cudaSetDevice(g->ctx->device));
  if (off) NIDO_CUDA_TRY(cudaMemcpyAsync(off, g->off, 8 * (g->nv + 1), cudaMemcpyDeviceToHost, s));
  if (w && g->ne) NIDO_CUDA_TRY(cudaMemcpyAsync(w, g->w, 8 * g->ne, cudaMemcpyDefault, s));
  if (adj && g->ne) {
    int64_t* tmp = reinterpret_cast<int64_t*>(g->w2);  // ne doubles, free outside coarsening
    k_widen<<<kGrid, 256, 0, s>>>(g->adj, g->ne, tmp);
    NIDO_LAUNCH_CHECK();
    NIDO_CUDA_TRY(cudaMemcpyAsync(adj, tmp, 8 * g->ne, cudaMemcpyDefault, s));
  }
  NIDO_CUDA_TRY(cudaStreamSynchronize(s));
  return NIDO_OK;
}

extern "C" int nido_graph_batches(nido_graph g, int64_t* cuts) {
  if (g && g->color_mode)
    return nido_set_error(NIDO_E_INVALID, "colour-class batches are not vertex ranges: no cut points");
  if (!g || !cuts) return nido_set_error(NIDO_E_INVALID, "null argument");
  if (!g->bins_valid) NIDO_TRY(nido::build_batches(g));
  std::copy(g->cuts.begin(), g->cuts.end(), cuts);
  return NIDO_OK;
}

extern "C" int nido_graph_vertex_weights(nido_graph g, double* k, double* m) {
  if (!g) return nido_set_error(NIDO_E_INVALID, "null graph");
  if (k) {
    NIDO_CUDA_TRY(cudaMemcpyAsync(k, g->k, 8 * g->nv, cudaMemcpyDeviceToHost, g->ctx->stream));
    NIDO_CUDA_TRY(cudaStreamSynchronize(g->ctx->stream));
  }
  if (m) *m = g->m;
  return NIDO_OK;
}

namespace {
int reset_graph(nido_graph g) {
  cudaStream_t s = g->ctx->stream;
  k_iota<<<kGrid, 256, 0, s>>>(g->clus, g->nv0);
  NIDO_LAUNCH_CHECK();
  if (!g->coarsened) return NIDO_OK;
  g->off = g->off0;
  g->adj = g->adj0;
  g->w = g->w0;
  g->nv = g->nv0;
  g->ne = g->ne0;
  g->coarsened = false;
  return prepare_phase(g);
}
}  // namespace

extern "C" int nido_graph_reset(nido_graph g) {
  if (!g) return nido_set_error(NIDO_E_INVALID, "null graph");
  NIDO_CUDA_TRY(cudaSetDevice(g->ctx->device));
  NIDO_TRY(reset_graph(g));
  return nido::launch_singleton(g);
}

extern "C" int nido_host_register(void* ptr, size_t bytes) {
  if (!ptr || !bytes) return nido_set_error(NIDO_E_INVALID, "nido_host_register: empty range");
  NIDO_CUDA_TRY(cudaHostRegister(ptr, bytes, cudaHostRegisterDefault));
  return NIDO_OK;
}

extern "C" int nido_host_unregister(void* ptr) {
  if (!ptr) return nido_set_error(NIDO_E_INVALID, "nido_host_unregister: null pointer");
  NIDO_CUDA_TRY(cudaHostUnregister(ptr));
  return NIDO_OK;
}

extern "C" int nido_singleton_partition(nido_graph g) {
  if (!g) return nido_set_error(NIDO_E_INVALID, "null graph");
  return nido::launch_singleton(g);
}

extern "C" int nido_set_community_ids(nido_graph g, const int64_t* comm) {
  if (!g || !comm) return nido_set_error(NIDO_E_INVALID, "null argument");
  cudaStream_t s = g->ctx->stream;
  Arena ar(g->scratch, g->scratch_bytes);
  int64_t* c64 = ar.take<int64_t>(g->nv);
  if (!c64) return nido_set_error(NIDO_E_NOMEM, "scratch arena too small");
  NIDO_CUDA_TRY(cudaMemcpyAsync(c64, comm, 8 * g->nv, cudaMemcpyHostToDevice, s));
  unsigned long long* bad = reinterpret_cast<unsigned long long*>(g->dcount);
  NIDO_CUDA_TRY(cudaMemsetAsync(bad, 0, 8, s));
  k_set_ids<<<kGrid, 256, 0, s>>>(c64, g->nv, g->comm, g->newc, bad);
  NIDO_LAUNCH_CHECK();
  NIDO_TRY(nido::launch_set_comm(g));
  unsigned long long nbad = 0;
  NIDO_CUDA_TRY(cudaMemcpyAsync(&nbad, bad, 8, cudaMemcpyDeviceToHost, s));
  NIDO_CUDA_TRY(cudaStreamSynchronize(s));
  if (nbad) return nido_set_error(NIDO_E_INVALID, "%llu community ids outside [0, nv)", nbad);
  return NIDO_OK;
}

extern "C" int nido_compute_community_weights(nido_graph g) {
  if (!g) return nido_set_error(NIDO_E_INVALID, "null graph");
  NIDO_CUDA_TRY(cudaSetDevice(g->ctx->device));
  return nido::launch_set_comm(g);
}

extern "C" int nido_compute_modularity(nido_graph g, double* q) {
  if (!g || !q) return nido_set_error(NIDO_E_INVALID, "null argument");
  return nido::launch_modularity(g, q);
}

extern "C" int nido_louvain_update(nido_graph g, int32_t batch, int32_t tie_mode) {
  if (!g) return nido_set_error(NIDO_E_INVALID, "null graph");
  if (tie_mode != NIDO_TIE_SMALLEST_ID && tie_mode != NIDO_TIE_NIDO)
    return nido_set_error(NIDO_E_INVALID, "unknown tie mode %d", tie_mode);
  return nido::launch_move(g, batch, tie_mode, nullptr, nullptr);
}

// The reference updates community degrees and then swaps ids as two calls
// (graph_gpu.cpp:779-820); the engine fuses them into one kernel, so the
// degree update performs both and the id update is a no-op kept for API
// parity.  Calling them in the reference's order gives the reference's state.
extern "C" int nido_update_community_weights(nido_graph g, int32_t batch) {
  if (!g) return nido_set_error(NIDO_E_INVALID, "null graph");
  if (batch < 0 || batch >= g->nbatches) return nido_set_error(NIDO_E_INVALID, "batch out of range");
  if (!g->bins_valid) NIDO_TRY(nido::build_batches(g));
  return nido::launch_commit_batch(g, batch);
}

extern "C" int nido_update_community_ids(nido_graph g, int32_t batch) {
  if (!g) return nido_set_error(NIDO_E_INVALID, "null graph");
  if (batch < 0 || batch >= g->nbatches) return nido_set_error(NIDO_E_INVALID, "batch out of range");
  return NIDO_OK;
}

extern "C" int nido_restore_community(nido_graph g) {
  if (!g) return nido_set_error(NIDO_E_INVALID, "null graph");
  return nido::launch_commit(g, 0, g->nv);
}

extern "C" int nido_aggregation(nido_graph g, int32_t* done) {
  if (!g || !done) return nido_set_error(NIDO_E_INVALID, "null argument");
  int d = 0;
  NIDO_TRY(nido::launch_aggregation(g, &d));
  *done = d;
  if (!d) NIDO_TRY(prepare_phase(g));
  return NIDO_OK;
}

extern "C" int nido_get_state(nido_graph g, int64_t* comm, int64_t* newcomm, double* a) {
  if (!g) return nido_set_error(NIDO_E_INVALID, "null graph");
  cudaStream_t s = g->ctx->stream;
  Arena ar(g->scratch, g->scratch_bytes);
  int64_t* tmp = ar.take<int64_t>(g->nv);
  if (!tmp) return nido_set_error(NIDO_E_NOMEM, "scratch arena too small");
  if (comm) {
    k_widen<<<kGrid, 256, 0, s>>>(g->comm, g->nv, tmp);
    NIDO_LAUNCH_CHECK();
    NIDO_CUDA_TRY(cudaMemcpyAsync(comm, tmp, 8 * g->nv, cudaMemcpyDeviceToHost, s));
    NIDO_CUDA_TRY(cudaStreamSynchronize(s));
  }
  if (newcomm) {
    k_widen<<<kGrid, 256, 0, s>>>(g->newc, g->nv, tmp);
    NIDO_LAUNCH_CHECK();
    NIDO_CUDA_TRY(cudaMemcpyAsync(newcomm, tmp, 8 * g->nv, cudaMemcpyDeviceToHost, s));
    NIDO_CUDA_TRY(cudaStreamSynchronize(s));
  }
  if (a) NIDO_CUDA_TRY(cudaMemcpyAsync(a, g->a, 8 * g->nv, cudaMemcpyDeviceToHost, s));
  NIDO_CUDA_TRY(cudaStreamSynchronize(s));
  return NIDO_OK;
}

extern "C" int nido_get_clustering(nido_graph g, int64_t* clustering) {
  if (!g || !clustering) return nido_set_error(NIDO_E_INVALID, "null argument");
  cudaStream_t s = g->ctx->stream;
  Arena ar(g->scratch, g->scratch_bytes);
  int64_t* tmp = ar.take<int64_t>(g->nv0);
  if (!tmp) return nido_set_error(NIDO_E_NOMEM, "scratch arena too small");
  k_widen<<<kGrid, 256, 0, s>>>(g->clus, g->nv0, tmp);
  NIDO_LAUNCH_CHECK();
  // A pageable destination (a fresh host array, say) is copied to at a
  // fraction of the link's speed and faults its pages in one at a time; such
  // copies go through the context's pinned buffer and are spread over the
  // host threads.
  const size_t bytes = 8 * (size_t)g->nv0;
  cudaPointerAttributes pa{};
  bool pinned = cudaPointerGetAttributes(&pa, clustering) == cudaSuccess && pa.type == cudaMemoryTypeHost;
  if (!pinned) cudaGetLastError();
  void* stage = nullptr;
  if (!pinned && bytes >= ((size_t)1 << 20) && nido::pinned_buffer(g->ctx, bytes, &stage) == cudaSuccess) {
    NIDO_CUDA_TRY(cudaMemcpyAsync(stage, tmp, bytes, cudaMemcpyDeviceToHost, s));
    NIDO_CUDA_TRY(cudaStreamSynchronize(s));
    const int T = std::max(1, std::min(16, omp_get_max_threads()));
    const int64_t n = g->nv0, per = (n + T - 1) / T;
    const int64_t* src = static_cast<const int64_t*>(stage);
#pragma omp parallel for num_threads(T) schedule(static)
    for (int t = 0; t < T; ++t) {
      const int64_t lo = std::min(n, (int64_t)t * per), hi = std::min(n, lo + per);
      if (hi > lo) memcpy(clustering + lo, src + lo, sizeof(int64_t) * (size_t)(hi - lo));
    }
    return NIDO_OK;
  }
  cudaGetLastError();
  NIDO_CUDA_TRY(cudaMemcpyAsync(clustering, tmp, bytes, cudaMemcpyDeviceToHost, s));
  NIDO_CUDA_TRY(cudaStreamSynchronize(s));
  return NIDO_OK;
}

namespace {
// "%lld\n" of x at p; returns the end
char* put_line(char* p, int64_t x) {
  char tmp[20];
  unsigned long long u = x < 0 ? 0ull - (unsigned long long)x : (unsigned long long)x;
  int k = 0;
  do {
    tmp[k++] = (char)('0' + u % 10);
    u /= 10;
  } while (u);
  if (x < 0) *p++ = '-';
  while (k) *p++ = tmp[--k];
  *p++ = '\n';
  return p;
}
}  // namespace

// Clustering::dump_partition (clustering.cpp:23-46): one "%lld\n" line per
// original vertex, un-permuted through new_orders when given; the lines are
// formatted by host threads in slices and written in order.
extern "C" int nido_dump_partition(nido_graph g, const char* path, const int64_t* new_orders) {
  if (!g || !path) return nido_set_error(NIDO_E_INVALID, "null argument");
  const int64_t n = g->nv0;
  std::vector<int64_t> c((size_t)n);
  NIDO_TRY(nido_get_clustering(g, c.data()));
  if (new_orders) {
    std::vector<int64_t> t((size_t)n);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) t[new_orders[i]] = c[i];
    c.swap(t);
  }
  FILE* f = fopen(path, "wt");
  if (!f) return nido_set_error(NIDO_E_IO, "cannot open %s", path);
  const int T = std::max(1, std::min(16, omp_get_max_threads()));
  const int64_t per = (n + T - 1) / T;
  std::vector<std::vector<char>> parts((size_t)T);
#pragma omp parallel for num_threads(T) schedule(static)
  for (int t = 0; t < T; ++t) {
    const int64_t lo = std::min(n, (int64_t)t * per), hi = std::min(n, lo + per);
    std::vector<char>& b = parts[(size_t)t];
    b.resize((size_t)(hi - lo) * 21);
    char* p = b.data();
    for (int64_t i = lo; i < hi; ++i) p = put_line(p, c[(size_t)i]);
    b.resize((size_t)(p - b.data()));
  }
  bool ok = true;
  for (const std::vector<char>& b : parts) ok = ok && fwrite(b.data(), 1, b.size(), f) == b.size();
  if (fclose(f) != 0 || !ok) return nido_set_error(NIDO_E_IO, "short write to %s", path);
  return NIDO_OK;
}

// ---- degree-tier autotuner ------------------------------------------------------

namespace nido {
namespace {
bool config_ok(const TierConfig& c) {
  return c.warp_max >= 32 && c.warp_max <= kWarpMaxDeg && c.ctas_max >= c.warp_max && c.ctas_max <= kCtaSMaxDeg &&
         c.ctam_max >= c.ctas_max && c.ctam_max <= kCtaMMaxDeg && c.ctal_max >= c.ctam_max &&
         c.ctal_max <= kCtaLMaxDeg && c.ctax_max >= c.ctal_max && c.ctax_max <= kCtaXMaxDeg &&
         c.hub_wave_slots >= 4096;
}

// one move sweep over every batch, timed on the device (ms)
int time_sweeps(nido_graph_s* g, int tie, int sweeps, double* ms) {
  cudaStream_t s = g->ctx->stream;
  g->bins_valid = false;
  NIDO_TRY(build_batches(g));
  for (int b = 0; b < g->nbatches; ++b) NIDO_TRY(launch_move(g, b, tie, nullptr, nullptr));  // warm
  NIDO_CUDA_TRY(cudaEventRecord(g->ctx->ev0, s));
  for (int i = 0; i < sweeps; ++i)
    for (int b = 0; b < g->nbatches; ++b) NIDO_TRY(launch_move(g, b, tie, nullptr, nullptr));
  NIDO_CUDA_TRY(cudaEventRecord(g->ctx->ev1, s));
  NIDO_CUDA_TRY(cudaEventSynchronize(g->ctx->ev1));
  float t = 0.f;
  NIDO_CUDA_TRY(cudaEventElapsedTime(&t, g->ctx->ev0, g->ctx->ev1));
  *ms = t / sweeps;
  return NIDO_OK;
}
}  // namespace

int tune_tiers(nido_graph_s* g, int tie, int sweeps, double* best_ms) {
  if (sweeps < 1) sweeps = 1;
  TierConfig best = g->cfg;
  double bt = 0.;
  NIDO_TRY(time_sweeps(g, tie, sweeps, &bt));
  // coordinate descent: each knob in turn, a candidate kept when 2% faster
  auto try_cfg = [&](const TierConfig& c) -> int {
    if (!config_ok(c)) return NIDO_OK;
    g->cfg = c;
    double t = 0.;
    NIDO_TRY(time_sweeps(g, tie, sweeps, &t));
    if (t < 0.98 * bt) { bt = t; best = c; }
    g->cfg = best;
    return NIDO_OK;
  };
  for (int32_t v : {8192, 4096}) { TierConfig c = best; c.ctax_max = v; NIDO_TRY(try_cfg(c)); }
  for (int32_t v : {3072, 1536}) { TierConfig c = best; c.ctal_max = v; NIDO_TRY(try_cfg(c)); }
  for (int32_t v : {1024, 768}) { TierConfig c = best; c.ctam_max = v; NIDO_TRY(try_cfg(c)); }
  for (int32_t v : {512, 384}) { TierConfig c = best; c.ctas_max = v; NIDO_TRY(try_cfg(c)); }
  for (int32_t v : {128, 64}) { TierConfig c = best; c.warp_max = v; NIDO_TRY(try_cfg(c)); }
  { TierConfig c = best; c.staged_edges = !c.staged_edges; NIDO_TRY(try_cfg(c)); }
  if (g->max_degree > best.ctax_max) {
    for (int64_t v : {(int64_t)2 << 20, (int64_t)8 << 20}) { TierConfig c = best; c.hub_wave_slots = v; NIDO_TRY(try_cfg(c)); }
    if (g->int_weights && tie != NIDO_TIE_NIDO) { TierConfig c = best; c.hub_clusters = true; NIDO_TRY(try_cfg(c)); }
  }
  g->cfg = best;
  g->bins_valid = false;
  NIDO_TRY(build_batches(g));
  g->tuned = true;
  if (best_ms) *best_ms = bt;
  return NIDO_OK;
}
}  // namespace nido

extern "C" int nido_get_tier_config(nido_graph g, nido_tier_config* c) {
  if (!g || !c) return nido_set_error(NIDO_E_INVALID, "null argument");
  *c = nido_tier_config{g->cfg.warp_max, g->cfg.ctas_max, g->cfg.ctam_max, g->cfg.ctal_max, g->cfg.ctax_max,
                        g->cfg.hub_clusters ? 1 : 0, g->cfg.hub_wave_slots, g->cfg.staged_edges ? 1 : 0, 0};
  return NIDO_OK;
}

extern "C" int nido_set_tier_config(nido_graph g, const nido_tier_config* c) {
  if (!g || !c) return nido_set_error(NIDO_E_INVALID, "null argument");
  TierConfig t;
  t.warp_max = c->warp_max_degree;
  t.ctas_max = c->cta_s_max_degree;
  t.ctam_max = c->cta_m_max_degree;
  t.ctal_max = c->cta_l_max_degree;
  t.ctax_max = c->cta_x_max_degree;
  t.hub_wave_slots = c->hub_wave_slots;
  if (c->hub_clusters != 0 && c->hub_clusters != 1)
    return nido_set_error(NIDO_E_INVALID, "hub_clusters must be 0 or 1 (got %d)", c->hub_clusters);
  t.hub_clusters = c->hub_clusters != 0;
  if (c->staged_edges != 0 && c->staged_edges != 1)
    return nido_set_error(NIDO_E_INVALID, "staged_edges must be 0 or 1 (got %d)", c->staged_edges);
  t.staged_edges = c->staged_edges != 0;
  if (!nido::config_ok(t)) return nido_set_error(NIDO_E_INVALID, "tier thresholds out of range or decreasing");
  g->cfg = t;
  g->bins_valid = false;
  return nido::build_batches(g);
}

extern "C" int nido_tune(nido_graph g, int32_t tie_mode, int32_t sweeps, nido_tier_config* best, double* best_ms) {
  if (!g) return nido_set_error(NIDO_E_INVALID, "null graph");
  if (tie_mode != NIDO_TIE_SMALLEST_ID && tie_mode != NIDO_TIE_NIDO)
    return nido_set_error(NIDO_E_INVALID, "unknown tie mode %d", tie_mode);
  NIDO_CUDA_TRY(cudaSetDevice(g->ctx->device));
  NIDO_TRY(nido::tune_tiers(g, tie_mode, sweeps, best_ms));
  if (best) NIDO_TRY(nido_get_tier_config(g, best));
  return NIDO_OK;
}

namespace {
// Device time of a section that runs many times per run (modularity,
// aggregation): event pairs in two slots, each pair read back once a later
// stream synchronisation has certainly passed it, so timing adds no wait.
struct SectionTimer {
  cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
  bool pending[2] = {false, false};
  int slot = 0;
  double ms = 0.;
  int init() {
    for (cudaEvent_t& e : ev) NIDO_CUDA_TRY(cudaEventCreate(&e));
    return NIDO_OK;
  }
  ~SectionTimer() {
    for (cudaEvent_t e : ev)
      if (e) cudaEventDestroy(e);
  }
  int begin(cudaStream_t s) {
    if (pending[slot]) NIDO_TRY(harvest(slot));
    NIDO_CUDA_TRY(cudaEventRecord(ev[2 * slot], s));
    return NIDO_OK;
  }
  int end(cudaStream_t s) {
    NIDO_CUDA_TRY(cudaEventRecord(ev[2 * slot + 1], s));
    pending[slot] = true;
    slot ^= 1;
    return NIDO_OK;
  }
  // after a synchronisation of the stream: read the other slot's pair
  int synced() { return pending[slot] ? harvest(slot) : NIDO_OK; }
  int harvest(int i) {
    float t = 0.f;
    NIDO_CUDA_TRY(cudaEventElapsedTime(&t, ev[2 * i], ev[2 * i + 1]));
    ms += t;
    pending[i] = false;
    return NIDO_OK;
  }
  int finish() {  // the stream is idle
    for (int i = 0; i < 2; ++i)
      if (pending[i]) NIDO_TRY(harvest(i));
    return NIDO_OK;
  }
};
}  // namespace

// LouvainGPU::run (louvain_gpu.cpp:28-124): phases of singleton start,
// iterations of batched moves until dQ <= tau or max_iter, undo of an
// iteration that lowered Q, and aggregation when the phase gained more
// than tau.
extern "C" int nido_run(nido_graph g, const nido_params* p, int64_t* out_comm, nido_run_stats* stats) {
  if (!g || !p) return nido_set_error(NIDO_E_INVALID, "null argument");
  if (p->nbatches != g->nb_user)
    return nido_set_error(NIDO_E_INVALID, "params.nbatches (%d) differs from the graph's (%d)", p->nbatches, g->nb_user);
  if (p->host_loop < 0 || p->host_loop > 2)
    return nido_set_error(NIDO_E_INVALID, "host_loop must be 0, 1 or 2 (got %d)", p->host_loop);
  if (p->color_batches != 0 && p->color_batches != 1)
    return nido_set_error(NIDO_E_INVALID, "color_batches must be 0 or 1 (got %d)", p->color_batches);
  if ((p->color_batches != 0) != g->color_mode) {
    g->color_mode = p->color_batches != 0;  // the batches of every phase follow this run's choice
    g->bins_valid = false;
  }
  if (p->tie_mode != NIDO_TIE_SMALLEST_ID && p->tie_mode != NIDO_TIE_NIDO)
    return nido_set_error(NIDO_E_INVALID, "unknown tie mode %d", p->tie_mode);
  NIDO_CUDA_TRY(cudaSetDevice(g->ctx->device));
  nido_run_stats st;
  memset(&st, 0, sizeof(st));
  cudaStream_t s = g->ctx->stream;
  struct RunEvents {  // destroyed on every return, early ones included
    cudaEvent_t t0 = nullptr, t1 = nullptr;
    ~RunEvents() {
      if (t0) cudaEventDestroy(t0);
      if (t1) cudaEventDestroy(t1);
    }
  } re;
  NIDO_CUDA_TRY(cudaEventCreate(&re.t0));
  NIDO_CUDA_TRY(cudaEventCreate(&re.t1));
  cudaEvent_t t0 = re.t0, t1 = re.t1;
  auto now_ms = [] {
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now().time_since_epoch()).count();
  };
  SectionTimer qt, at;  // modularity and aggregation device time
  NIDO_TRY(qt.init());
  NIDO_TRY(at.init());
  auto modularity = [&](double* q) -> int {
    NIDO_TRY(qt.begin(s));
    NIDO_TRY(nido::launch_modularity(g, q));  // ends with a stream synchronisation
    NIDO_TRY(qt.end(s));
    NIDO_TRY(qt.synced());
    return at.synced();
  };
  const uint64_t launches0 = nido_launch_count();
  double tm = now_ms();
  auto lap = [&](int slot) {
    const double t = now_ms();
    st.host_ms[slot] += t - tm;
    tm = t;
  };
  NIDO_CUDA_TRY(cudaEventRecord(t0, s));
  // every run starts from the uploaded graph, as on a fresh GraphGPU
  NIDO_TRY(reset_graph(g));
  lap(0);
  const double tau = p->tau;
  const double tau_phase = p->tau_phase_set ? p->tau_phase : p->tau;
  bool done = false;
  int64_t phases = 0;
  while (!done && phases < 200) {
    if (p->verbose) printf("PHASE #%lld: \n", (long long)phases);
    if (p->tune && !g->tuned && phases == 0) {
      NIDO_TRY(nido::launch_singleton(g));
      NIDO_TRY(nido::tune_tiers(g, p->tie_mode, 2, nullptr));
      lap(6);
    }
    NIDO_TRY(nido::launch_singleton(g));
    double Q = 0., Q_old = 0.;
    int64_t loops = 0;
    const bool want_device = p->host_loop == 2;
    bool host_loop = !want_device || !g->ctx->device_loop || (p->verbose && p->max_iter > nido::kLoopLogCap);
    if (!host_loop) {
      // the phase's iteration loop as one device-resident CUDA graph
      nido::PhaseLoop r;
      bool unsupported = false;
      NIDO_TRY(nido::device_phase_loop(g, p->tie_mode, tau, p->max_iter, p->verbose != 0, &r, &unsupported));
      if (unsupported) {
        g->ctx->device_loop = false;  // this driver has no conditional graph nodes
        host_loop = true;
      } else {
        Q_old = r.q_old;
        Q = r.q;
        loops = r.loops;
        st.move_ms += r.move_ms;
        st.q_ms += r.q_ms;
        st.host_ms[7] += r.build_ms;
        st.move_launches += g->nbatches * loops;
        st.edges_scanned += (double)g->ne * (double)loops;
        st.move_bytes += (16.0 * (double)g->ne + 32.0 * (double)nido::listed_vertices(g)) * (double)loops;
        if (p->verbose) {
          printf("LOOP# \tQ \t\tdQ\n----------------------------------------\n0 \t%g \t0\n", Q_old);
          for (size_t i = 0; 2 * i + 1 < r.log.size(); ++i)
            printf("%lld \t%g \t%g\n", (long long)(i + 1), r.log[2 * i], r.log[2 * i + 1]);
        }
        lap(1);
      }
    }
    if (host_loop) {
    NIDO_TRY(modularity(&Q));
    lap(2);
    Q_old = Q;
    if (p->verbose) printf("LOOP# \tQ \t\tdQ\n----------------------------------------\n0 \t%g \t0\n", Q);
    double dQ = NIDO_MAX_FLOAT;
    while (tau < dQ && loops < p->max_iter) {
      std::vector<cudaEvent_t>& ev = g->ctx->move_ev;
      while (ev.size() < 2 * (size_t)g->nbatches) {
        cudaEvent_t e;
        NIDO_CUDA_TRY(cudaEventCreate(&e));
        ev.push_back(e);
      }
      for (int b = 0; b < g->nbatches; ++b) {
        NIDO_TRY(nido::launch_move(g, b, p->tie_mode, ev[2 * b], ev[2 * b + 1]));
        NIDO_TRY(nido::launch_commit_batch(g, b));
      }
      st.move_launches += g->nbatches;
      st.edges_scanned += (double)g->ne;
      st.move_bytes += 16.0 * (double)g->ne + 32.0 * (double)nido::listed_vertices(g);
      lap(1);
      double Qtmp;
      NIDO_TRY(modularity(&Qtmp));
      lap(2);
      dQ = Qtmp - Q;
      ++loops;
      for (int b = 0; b < g->nbatches; ++b) {  // complete: the Q readback synchronized the stream
        float ms = 0.f;
        NIDO_CUDA_TRY(cudaEventElapsedTime(&ms, ev[2 * b], ev[2 * b + 1]));
        st.move_ms += ms;
      }
      if (dQ < 0) NIDO_TRY(nido::launch_commit(g, 0, g->nv));
      else Q = Qtmp;
      if (p->verbose) printf("%lld \t%g \t%g\n", (long long)loops, Qtmp, dQ);
    }
    }
    if (phases < 200) {
      st.q_phase[phases] = Q;
      st.loops_phase[phases] = loops;
      st.nv_phase[phases] = g->nv;
      st.ne_phase[phases] = g->ne;
    }
    st.total_loops += loops;
    st.final_q = Q;
    if (p->verbose) {
      if (loops >= p->max_iter) printf("Exceed maximum loop number\n");
      printf("Final Q: %g\n", Q);
    }
    if (Q - Q_old > tau_phase) {
      int d = 0;
      lap(1);
      NIDO_TRY(at.begin(s));
      NIDO_TRY(nido::launch_aggregation(g, &d));
      NIDO_TRY(at.end(s));
      lap(3);
      done = d != 0;
      if (!done) NIDO_TRY(prepare_phase(g));
      lap(4);
    } else {
      done = true;
    }
    if (p->verbose) printf("----------------------------------------\n");
    ++phases;
  }
  NIDO_CUDA_TRY(cudaEventRecord(t1, s));
  NIDO_CUDA_TRY(cudaEventSynchronize(t1));
  float tot = 0.f;
  NIDO_CUDA_TRY(cudaEventElapsedTime(&tot, t0, t1));
  st.total_ms = tot;
  st.phases = phases;
  NIDO_TRY(qt.finish());
  NIDO_TRY(at.finish());
  st.q_ms += qt.ms;
  st.agg_ms = at.ms;
  int64_t nerr = 0;
  NIDO_CUDA_TRY(cudaMemcpyAsync(&nerr, g->dcount + 1, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
  NIDO_CUDA_TRY(cudaStreamSynchronize(s));
  if (nerr)
    return nido_set_error(NIDO_E_CUDA, "a move kernel gave up %lld times (hash-table probe limit or bounded wait)",
                          (long long)nerr);
  lap(1);
  if (out_comm) NIDO_TRY(nido_get_clustering(g, out_comm));
  lap(5);
  st.kernel_launches = (int64_t)(nido_launch_count() - launches0);
  if (stats) *stats = st;
  if (p->verbose) fflush(stdout);
  return NIDO_OK;
}
