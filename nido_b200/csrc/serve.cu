// serve.cu -- a request loop on one GPU: continuous batching of Louvain
// requests of different sizes (no reference counterpart; nido runs one graph
// per process).
//
// Requests queue in arrival order.  A pool of worker threads, each owning a
// context (its own stream, stream-ordered allocation), takes the request at
// the head of the queue as soon as a worker is free and the request's device
// footprint fits in what the HBM budget has left; requests that arrive while
// others run are admitted the moment slots and memory free up, and their
// kernels overlap on the device through the workers' streams.  Every request
// keeps its CSR and state resident on the device across all its phases and
// runs the one-graph engine unchanged, so its result does not depend on what
// else is running (bit-identical on integer weights).
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <mutex>
#include <new>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "common.cuh"
#include "engine.cuh"
#include "primitives.cuh"

namespace {

double now_ms() {
  return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

struct Request {
  int64_t id = 0;
  nido_csr g{};
  nido_params p{};
  int64_t* out = nullptr;
  int64_t bytes = 0;
  int state = 0;  // 0 queued, 1 running, 2 finished
  bool claimed = false;  // a nido_server_wait is blocked on it
  bool streamed = false; // admitted over budget: edges in mapped host memory
  nido_request_info info{};
  std::string err;
  double t_submit = 0, t_start = 0;
};

}  // namespace

struct nido_server_s {
  int device = 0;
  int64_t budget = 0;
  int64_t reserved = 0;
  std::vector<nido_ctx> ctxs;
  std::vector<std::thread> workers;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<Request*> queue;
  std::unordered_map<int64_t, Request*> live;
  int64_t next_id = 1;
  int running = 0;
  bool stop = false;
  // the workers' stream-ordered allocations come from this pool, whose
  // release threshold keeps freed blocks for the next request; the device's
  // default pool (and every other allocator in the process) is untouched
  cudaMemPool_t pool = nullptr;
};

namespace {

void worker_loop(nido_server_s* S, int wid) {
  nido_ctx ctx = S->ctxs[wid];
  cudaSetDevice(S->device);
  for (;;) {
    Request* r = nullptr;
    {
      std::unique_lock<std::mutex> lk(S->mu);
      S->cv_work.wait(lk, [&] {
        return (S->stop && S->queue.empty()) ||
               (!S->queue.empty() && S->reserved + S->queue.front()->bytes <= S->budget);
      });
      if (S->queue.empty()) return;
      r = S->queue.front();
      S->queue.pop_front();
      S->reserved += r->bytes;
      S->running += 1;
      r->state = 1;
      r->t_start = now_ms();
    }
    nido_graph g = nullptr;
    nido_run_stats st;
    memset(&st, 0, sizeof(st));
    // a streamed request's context budget is its reservation, which leaves
    // the edge arrays to mapped host memory
    if (r->streamed) ctx->budget = (size_t)r->bytes;
    int rc = nido_graph_upload(ctx, r->g.nv, r->g.ne, r->g.off, r->g.adj, r->g.w, r->p.nbatches, &g);
    ctx->budget = 0;
    if (rc == NIDO_OK) rc = nido_run(g, &r->p, r->out, &st);
    std::string err = rc == NIDO_OK ? std::string() : std::string(nido_last_error());
    nido_graph_free(g);
    const double t_end = now_ms();
    {
      std::lock_guard<std::mutex> lk(S->mu);
      S->reserved -= r->bytes;
      S->running -= 1;
      r->state = 2;
      r->err = err;
      nido_request_info& in = r->info;
      in.status = rc;
      in.final_q = st.final_q;
      in.phases = st.phases;
      in.total_loops = st.total_loops;
      in.queue_ms = r->t_start - r->t_submit;
      in.run_ms = t_end - r->t_start;
      in.latency_ms = t_end - r->t_submit;
      in.device_ms = st.total_ms;
      in.hbm_bytes = r->bytes;
      in.worker = wid;
      in.host_edges = r->streamed ? 1 : 0;
    }
    S->cv_work.notify_all();  // memory came back: the head may fit now
    S->cv_done.notify_all();
  }
}

}  // namespace

// Upload (three CSR copies, per-vertex state, scratch as nido_graph_upload
// sizes them); the hub-table region, one wave of tables at 12 bytes a slot
// plus its packed 8-byte copy for integer phases (at most 8M slots, or one
// table of up to 4*nv slots); the coarsening
// plan's region for giant communities, one wave at 16 bytes a slot (at most
// 4M slots or one table of up to 4*nv), grown by a quarter, plus its
// per-vertex and per-segment lists; and the hub work lists.
// The same with the edge arrays (three CSR copies of 12 bytes an edge) in
// mapped host memory, as over-budget graphs keep them.
extern "C" int64_t nido_graph_footprint_streamed(int64_t nv, int64_t ne, int32_t nbatches) {
  return nido_graph_footprint(nv, ne, nbatches) - 36 * std::max<int64_t>(ne, 1);
}

extern "C" int64_t nido_graph_footprint(int64_t nv, int64_t ne, int32_t nbatches) {
  (void)nbatches;
  const int64_t V = std::max<int64_t>(nv, 1), E = std::max<int64_t>(ne, 1);
  int64_t b = 24 * (V + 1) + 36 * E + 32 * V + 128;
  b += 64 * (V + 1) + (1 << 20) + 8 * (nido::radix_temp_elems(V) + nido::scan_temp_elems(E + 1));
  b += 20 * std::max<int64_t>((int64_t)8 << 20, 4 * V);  // FP64 and packed hub tables
  b += 20 * std::max<int64_t>((int64_t)4 << 20, 4 * V) + 40 * V + E / 32;
  b += 4 * (E / 32 + 2);  // member index of the coarsening's 32-position blocks
  b += E;  // first-position bitmaps and word prefixes of the giant segments
  b += (int64_t)32 << 20;
  return b;
}

extern "C" int nido_server_create(int device, size_t hbm_budget_bytes, int32_t nworkers, nido_server* out) {
  if (!out) return nido_set_error(NIDO_E_INVALID, "nido_server_create: null output");
  *out = nullptr;
  if (nworkers < 1 || nworkers > 64) return nido_set_error(NIDO_E_INVALID, "nworkers must be in [1, 64]");
  NIDO_CUDA_TRY(cudaSetDevice(device));
  size_t freeb = 0, totalb = 0;
  NIDO_CUDA_TRY(cudaMemGetInfo(&freeb, &totalb));
  // freed blocks stay in the server's own pool for the next request instead
  // of going back to the driver at every synchronization
  cudaMemPoolProps props = {};
  props.allocType = cudaMemAllocationTypePinned;
  props.handleTypes = cudaMemHandleTypeNone;
  props.location.type = cudaMemLocationTypeDevice;
  props.location.id = device;
  cudaMemPool_t pool = nullptr;
  NIDO_CUDA_TRY(cudaMemPoolCreate(&pool, &props));
  uint64_t keep = UINT64_MAX;
  const cudaError_t pe = cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
  if (pe != cudaSuccess) {
    cudaMemPoolDestroy(pool);
    return nido_set_error(NIDO_E_CUDA, "cudaMemPoolSetAttribute failed: %s", cudaGetErrorString(pe));
  }
  nido_server S = new (std::nothrow) nido_server_s();
  if (!S) {
    cudaMemPoolDestroy(pool);
    return nido_set_error(NIDO_E_NOMEM, "host allocation failed");
  }
  S->device = device;
  S->pool = pool;
  const int64_t cap = (int64_t)freeb - ((int64_t)1 << 30);  // keep 1 GiB for the runtime
  S->budget = hbm_budget_bytes ? std::min<int64_t>((int64_t)hbm_budget_bytes, cap) : cap;
  for (int i = 0; i < nworkers; ++i) {
    nido_ctx c = nullptr;
    const int st = nido_ctx_create(device, 0, &c);
    if (st != NIDO_OK) {
      for (nido_ctx x : S->ctxs) nido_ctx_destroy(x);
      cudaMemPoolDestroy(S->pool);
      delete S;
      return st;
    }
    c->async_alloc = true;
    c->pool = S->pool;
    S->ctxs.push_back(c);
  }
  for (int i = 0; i < nworkers; ++i) S->workers.emplace_back(worker_loop, S, i);
  *out = S;
  return NIDO_OK;
}

extern "C" int nido_server_budget(nido_server S, int64_t* budget, int64_t* reserved, int32_t* running,
                                  int32_t* queued) {
  if (!S) return nido_set_error(NIDO_E_INVALID, "null server");
  std::lock_guard<std::mutex> lk(S->mu);
  if (budget) *budget = S->budget;
  if (reserved) *reserved = S->reserved;
  if (running) *running = S->running;
  if (queued) *queued = (int32_t)S->queue.size();
  return NIDO_OK;
}

extern "C" int nido_server_submit(nido_server S, const nido_csr* g, const nido_params* p, int64_t* out_comm,
                                  int64_t* ticket) {
  if (!S || !g || !p || !ticket) return nido_set_error(NIDO_E_INVALID, "nido_server_submit: null argument");
  if (p->nbatches < 1) return nido_set_error(NIDO_E_INVALID, "nbatches must be >= 1");
  const int64_t bytes = nido_graph_footprint(g->nv, g->ne, p->nbatches);
  const int64_t bytes_streamed = nido_graph_footprint_streamed(g->nv, g->ne, p->nbatches);
  Request* r = new (std::nothrow) Request();
  if (!r) return nido_set_error(NIDO_E_NOMEM, "host allocation failed");
  r->g = *g;
  r->p = *p;
  r->p.verbose = 0;
  r->out = out_comm;
  r->bytes = bytes;
  r->t_submit = now_ms();
  {
    std::lock_guard<std::mutex> lk(S->mu);
    if (bytes > S->budget) {
      // over the budget in HBM: admitted with its edges in mapped host memory
      // when the rest fits, refused otherwise
      if (bytes_streamed > S->budget) {
        delete r;
        return nido_set_error(NIDO_E_TOO_LARGE, "request needs %lld bytes (%lld with its edges on the host); "
                              "the HBM budget is %lld", (long long)bytes, (long long)bytes_streamed,
                              (long long)S->budget);
      }
      r->bytes = bytes_streamed;
      r->streamed = true;
    }
    if (S->stop) {
      delete r;
      return nido_set_error(NIDO_E_BUSY, "server is shutting down");
    }
    r->id = S->next_id++;
    S->live[r->id] = r;
    S->queue.push_back(r);
  }
  *ticket = r->id;
  S->cv_work.notify_all();
  return NIDO_OK;
}

extern "C" int nido_server_poll(nido_server S, int64_t ticket, int32_t* state) {
  if (!S || !state) return nido_set_error(NIDO_E_INVALID, "null argument");
  std::lock_guard<std::mutex> lk(S->mu);
  auto it = S->live.find(ticket);
  if (it == S->live.end()) return nido_set_error(NIDO_E_INVALID, "unknown ticket %lld", (long long)ticket);
  *state = it->second->state;
  return NIDO_OK;
}

extern "C" int nido_server_wait(nido_server S, int64_t ticket, double timeout_s, nido_request_info* info) {
  if (!S) return nido_set_error(NIDO_E_INVALID, "null server");
  std::unique_lock<std::mutex> lk(S->mu);
  auto it = S->live.find(ticket);
  if (it == S->live.end()) return nido_set_error(NIDO_E_INVALID, "unknown ticket %lld", (long long)ticket);
  Request* r = it->second;
  // one waiter per ticket: the waiter that returns frees the request, so a
  // second one would be left reading freed memory
  if (r->claimed)
    return nido_set_error(NIDO_E_INVALID, "ticket %lld is already being waited on", (long long)ticket);
  r->claimed = true;
  const auto pred = [&] { return r->state == 2; };
  if (timeout_s < 0) {
    S->cv_done.wait(lk, pred);
  } else if (!S->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s), pred)) {
    r->claimed = false;
    return nido_set_error(NIDO_E_TIMEOUT, "request %lld still running", (long long)ticket);
  }
  // submissions made while this thread waited may have rehashed the map:
  // erase by key, not through the iterator taken before the wait
  S->live.erase(ticket);
  lk.unlock();
  if (info) *info = r->info;
  const int rc = r->info.status;
  if (rc != NIDO_OK) nido_set_error(rc, "%s", r->err.c_str());
  delete r;
  return rc;
}

extern "C" int nido_server_destroy(nido_server S) {
  if (!S) return NIDO_OK;
  {
    std::lock_guard<std::mutex> lk(S->mu);
    S->stop = true;
  }
  S->cv_work.notify_all();
  for (std::thread& t : S->workers) t.join();
  for (auto& kv : S->live) delete kv.second;
  for (nido_ctx c : S->ctxs) nido_ctx_destroy(c);
  if (S->pool) {
    cudaSetDevice(S->device);
    cudaMemPoolDestroy(S->pool);
  }
  delete S;
  return NIDO_OK;
}
