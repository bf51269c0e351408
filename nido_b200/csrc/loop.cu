// loop.cu -- the iteration loop of a Louvain phase on the device.
//
// The reference runs the loop of louvain_gpu.cpp:53-90 on the host: after
// every iteration it reads Q back, computes dQ, restores the communities when
// Q fell and tests `tau < dQ && loops < maxLoops`.  Here one phase's loop is
// one CUDA graph whose body is a conditional WHILE node: every batch's move
// kernels and commit, the modularity, a one-thread control kernel that does
// the reference's bookkeeping and sets the loop condition, and the restore
// commit gated on the control kernel's flag.  The host launches the graph
// once per phase and reads the loop's state back once, at the end.
//
// CUDA events cannot be recorded inside a conditional body, so the time spent
// in the move kernels and in the modularity is taken with %globaltimer stamps
// written by one-thread kernels around those sections (stream-ordered: a stamp
// runs after everything before it has finished).
#include <string.h>

#include <chrono>
#include <vector>

#include "common.cuh"
#include "engine.cuh"

namespace nido {
namespace {

struct LoopCtl {
  double q;       // Q of the phase so far (the last accepted iteration)
  double q_old;   // Q at the start of the phase
  double q_tmp;   // Q after the last iteration
  double dq;      // its gain
  int64_t loops;
  int32_t restore;  // the last iteration lowered Q: undo it
  int32_t pad;
  unsigned long long t_move, t_q;    // stamps at the start of the current section
  unsigned long long move_ns, q_ns;  // time inside the move kernels / the modularity
};

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__global__ void k_loop_reset(LoopCtl* c) {
  c->dq = 0.;
  c->loops = 0;
  c->restore = 0;
  c->move_ns = 0;
  c->q_ns = 0;
}

__global__ void k_loop_start(LoopCtl* c, const double* __restrict__ q) {
  c->q = *q;
  c->q_old = *q;
  c->q_tmp = *q;
}

__global__ void k_stamp(unsigned long long* t) { *t = global_ns(); }

__global__ void k_lap(const unsigned long long* t0, unsigned long long* acc) { *acc += global_ns() - *t0; }

// louvain_gpu.cpp:76-90: dQ = Qtmp - Q, loops++, undo when dQ < 0 else accept,
// go on while tau < dQ and loops < maxLoops.  log (when given) keeps Qtmp and
// dQ of every iteration for the reference's per-loop lines.
__global__ void k_loop_control(LoopCtl* c, const double* __restrict__ qtmp, double tau, int64_t max_iter,
                               double* __restrict__ log, int64_t log_cap, cudaGraphConditionalHandle h) {
  const double qt = *qtmp;
  const double dq = __dsub_rn(qt, c->q);
  const int64_t loops = c->loops + 1;
  c->loops = loops;
  c->q_tmp = qt;
  c->dq = dq;
  c->restore = dq < 0 ? 1 : 0;
  if (!(dq < 0)) c->q = qt;
  if (log && loops <= log_cap) {
    log[2 * (loops - 1)] = qt;
    log[2 * (loops - 1) + 1] = dq;
  }
  cudaGraphSetConditional(h, (tau < dq && loops < max_iter) ? 1u : 0u);
}

int ensure_loop_buf(nido_graph_s* g, int64_t log_cap) {
  const size_t need = sizeof(LoopCtl) + sizeof(double) * 2 * (size_t)log_cap;
  if (need <= g->loop_bytes) return NIDO_OK;
  raw_free(g->ctx, g->loop_buf);
  g->loop_buf = nullptr;
  g->loop_bytes = 0;
  NIDO_CUDA_TRY(raw_alloc(g->ctx, (void**)&g->loop_buf, need));
  g->loop_bytes = need;
  return NIDO_OK;
}

struct GraphHolder {  // destroyed on every return
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  ~GraphHolder() {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
  }
};

}  // namespace

// One phase's iteration loop on the device (see the file comment).  The phase
// must be prepared (singleton partition, tier lists and hub plan valid).
// On return r holds Q at the start and end of the phase, the loop count, the
// device time of the move kernels and of the modularity evaluations, and,
// with want_log, Qtmp and dQ of every iteration.  *unsupported is set (and
// NIDO_OK returned) when this device or driver cannot run conditional graph
// nodes; the caller then runs the host loop.
int device_phase_loop(nido_graph_s* g, int tie, double tau, int64_t max_iter, bool want_log, PhaseLoop* r,
                      bool* unsupported) {
  *unsupported = false;
  cudaStream_t s = g->ctx->stream;
  const int64_t log_cap = want_log ? std::min<int64_t>(max_iter, kLoopLogCap) : 0;
  NIDO_TRY(ensure_loop_buf(g, log_cap));
  LoopCtl* ctl = reinterpret_cast<LoopCtl*>(g->loop_buf);
  double* log = log_cap ? reinterpret_cast<double*>(g->loop_buf + sizeof(LoopCtl)) : nullptr;
  if (!g->bins_valid) NIDO_TRY(build_batches(g));
  k_loop_reset<<<1, 1, 0, s>>>(ctl);
  NIDO_LAUNCH_CHECK();
  k_stamp<<<1, 1, 0, s>>>(&ctl->t_q);
  NIDO_LAUNCH_CHECK();
  NIDO_TRY(launch_modularity_dev(g));
  k_lap<<<1, 1, 0, s>>>(&ctl->t_q, &ctl->q_ns);
  NIDO_LAUNCH_CHECK();
  k_loop_start<<<1, 1, 0, s>>>(ctl, g->dm + 1);
  NIDO_LAUNCH_CHECK();
  uint64_t body_kernels = 0;
  GraphHolder gh;
  const auto tb0 = std::chrono::steady_clock::now();
  if (max_iter > 0) {
    NIDO_CUDA_TRY(cudaGraphCreate(&gh.graph, 0));
    cudaGraphConditionalHandle h;
    if (cudaGraphConditionalHandleCreate(&h, gh.graph, 1, cudaGraphCondAssignDefault) != cudaSuccess) {
      cudaGetLastError();
      *unsupported = true;
      return NIDO_OK;
    }
    cudaGraphNodeParams cp = {cudaGraphNodeTypeConditional};
    cp.conditional.handle = h;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    cudaGraphNode_t node;
    if (cudaGraphAddNode(&node, gh.graph, nullptr, 0, &cp) != cudaSuccess) {
      cudaGetLastError();
      *unsupported = true;
      return NIDO_OK;
    }
    cudaGraph_t body = cp.conditional.phGraph_out[0];
    const uint64_t l0 = nido_launch_count();
    NIDO_CUDA_TRY(cudaStreamBeginCaptureToGraph(s, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
    auto enqueue_body = [&]() -> int {
      for (int b = 0; b < g->nbatches; ++b) {
        k_stamp<<<1, 1, 0, s>>>(&ctl->t_move);
        NIDO_LAUNCH_CHECK();
        NIDO_TRY(launch_move_tiers(g, b, tie));
        k_lap<<<1, 1, 0, s>>>(&ctl->t_move, &ctl->move_ns);
        NIDO_LAUNCH_CHECK();
        NIDO_TRY(launch_commit_batch(g, b));
      }
      k_stamp<<<1, 1, 0, s>>>(&ctl->t_q);
      NIDO_LAUNCH_CHECK();
      NIDO_TRY(launch_modularity_dev(g));
      k_lap<<<1, 1, 0, s>>>(&ctl->t_q, &ctl->q_ns);
      NIDO_LAUNCH_CHECK();
      k_loop_control<<<1, 1, 0, s>>>(ctl, g->dm + 1, tau, max_iter, log, log_cap, h);
      NIDO_LAUNCH_CHECK();
      return launch_commit_gated(g, 0, g->nv, &ctl->restore);
    };
    const int st = enqueue_body();
    cudaGraph_t captured = nullptr;
    const cudaError_t ce = cudaStreamEndCapture(s, &captured);
    if (st != NIDO_OK) return st;
    if (ce != cudaSuccess)
      return nido_set_error(NIDO_E_CUDA, "phase-loop capture failed: %s", cudaGetErrorString(ce));
    body_kernels = nido_launch_count() - l0;
    const cudaError_t ie = cudaGraphInstantiate(&gh.exec, gh.graph, 0);
    if (ie != cudaSuccess) {
      gh.exec = nullptr;
      return nido_set_error(NIDO_E_CUDA, "phase-loop graph instantiation failed: %s", cudaGetErrorString(ie));
    }
    r->build_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - tb0).count();
    NIDO_CUDA_TRY(cudaGraphLaunch(gh.exec, s));
  }
  LoopCtl hc;
  NIDO_CUDA_TRY(cudaMemcpyAsync(&hc, ctl, sizeof(hc), cudaMemcpyDeviceToHost, s));
  r->log.clear();
  if (log_cap) r->log.resize(2 * (size_t)log_cap);
  if (log_cap) NIDO_CUDA_TRY(cudaMemcpyAsync(r->log.data(), log, sizeof(double) * r->log.size(), cudaMemcpyDeviceToHost, s));
  NIDO_CUDA_TRY(cudaStreamSynchronize(s));
  r->q_old = hc.q_old;
  r->q = hc.q;
  r->loops = hc.loops;
  r->move_ms = hc.move_ns * 1e-6;
  r->q_ms = hc.q_ns * 1e-6;
  // the capture counted one iteration's kernels; the graph ran `loops` of them
  if (hc.loops > 1) nido_count_launches(body_kernels * (uint64_t)(hc.loops - 1));
  if (log_cap) r->log.resize(2 * (size_t)std::min<int64_t>(hc.loops, log_cap));
  return NIDO_OK;
}

}  // namespace nido
