/*
 * nido_b200.h -- C ABI of the B200-native Louvain engine (libnido_b200.so).
 *
 * The reference (sg0/nido) is a monolithic program whose internal operator
 * API is the GraphGPU class (graph_gpu.hpp:168-247) over the *_cuda launchers
 * of graph_cuda.hpp.  Each entry point below names the reference interface it
 * replaces.  Plain pointers and sizes only; every function returns an int
 * status (NIDO_OK or a negative NIDO_E_* code) and never throws; the message of
 * the last failure on the calling thread is available from nido_last_error().
 *
 * Host buffers are owned by the caller; device buffers are owned by the engine.
 * Ids crossing the ABI are int64 and weights FP64, as in the reference
 * (types.hpp:14-22).  On the device, vertex and community ids are int32
 * (graphs must have fewer than 2^31 vertices; larger ones are rejected with
 * NIDO_E_TOO_LARGE) and edge offsets int64.
 */
#ifndef NIDO_B200_H_
#define NIDO_B200_H_
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes -------------------------------------------------------- */
#define NIDO_OK 0
#define NIDO_E_INVALID -1   /* bad argument */
#define NIDO_E_CUDA -2      /* CUDA runtime error (message has the CUDA text) */
#define NIDO_E_NOMEM -3     /* device or host allocation failed / over budget */
#define NIDO_E_IO -4        /* file could not be opened, read or written */
#define NIDO_E_TOO_LARGE -5 /* more than 2^31-1 vertices */
#define NIDO_E_TIMEOUT -6   /* a bounded device wait gave up */
#define NIDO_E_NODEVICE -7  /* no CUDA device / not an sm_100 device */
#define NIDO_E_BUSY -8      /* queue full (serving) */

/* tie rules for the best-move argmax */
#define NIDO_TIE_SMALLEST_ID 0 /* equal gains: smallest community id (default) */
#define NIDO_TIE_NIDO 1        /* reference rule: 8-lane strided scan + shuffle tree
                                  (graph_cuda.cu:1493-1526), for parity runs */

typedef struct nido_ctx_s* nido_ctx;
typedef struct nido_graph_s* nido_graph;

/* Host CSR in the reference's layout (graph.hpp:23-26). */
typedef struct {
  int64_t nv;
  int64_t ne;
  int64_t* off; /* nv+1 */
  int64_t* adj; /* ne   */
  double* w;    /* ne   */
} nido_csr;

/* Run parameters: the reference's -b/-t/-i options (main.cpp:38-79, defaults
 * types.hpp:24-38) plus the tie rule. */
typedef struct {
  int32_t nbatches;  /* -b, default 2 */
  int32_t tie_mode;  /* NIDO_TIE_* */
  double tau;        /* -t, default 1e-6 */
  int64_t max_iter;  /* -i, default 500 */
  int32_t verbose;   /* print the reference's per-loop lines to stdout */
  int32_t tune;      /* 1: autotune the degree tiers on the first phase of the
                        first run of this graph (nido_tune), then keep them */
  double tau_phase;  /* LouvainGPU's tol_phase (louvain_gpu.hpp:20-21): a phase
                        is coarsened when it gained more than this; used only
                        when tau_phase_set, otherwise tau (the reference's
                        three-argument LouvainGPU) */
  int32_t tau_phase_set;
  int32_t host_loop; /* who drives each phase's iteration loop.  2: the device,
                        one CUDA graph per phase with a conditional while node,
                        read back once per phase; 1 or 0 (default): the host,
                        one Q readback per iteration, as the reference does.
                        Measured on B200 (driver 580) the host loop is the
                        faster: building the loop graphs costs more than the
                        round trips they save, for small and large graphs and
                        for graph sets alike */
  int32_t color_batches; /* 1: conflict-free batches instead of the -b cuts:
                        every phase colours its graph (Jones-Plassmann-Luby,
                        seed 1) and sweeps the colour classes in colour order,
                        one class per batch, so no two neighbours move in the
                        same batch (one-graph runs only) */
  int32_t reserved;  /* must be 0 */
} nido_params;

/* Per-run statistics (the reference prints these, louvain_gpu.cpp:43-131). */
typedef struct {
  int64_t phases;
  int64_t total_loops;
  double final_q;      /* "Final Q" of the last phase */
  double total_ms;     /* device-event time of the whole run */
  double move_ms;      /* time inside move-phase kernels */
  double move_bytes;   /* algorithmic bytes of all move sweeps (16E + 32V per sweep) */
  double edges_scanned;/* edges visited by move sweeps */
  int64_t move_launches;
  int64_t kernel_launches;
  /* host wall time per section (ms): [0] restart from the uploaded graph,
   * [1] enqueueing moves and commits, [2] modularity including the wait for
   * the device, [3] aggregation, [4] per-phase preparation after
   * aggregation, [5] download of the clustering, [6] autotuning, [7] capture
   * and instantiation of the device-resident loop graphs.  Batched runs
   * (nido_batch_run): [0] reset, [1] sweeps (moves, commits, modularity,
   * loop control and their readbacks; [7] is part of it), [2] tier-list
   * rebuilds after graphs stop iterating, [3] phase end, aggregation and
   * emits, [4] phase set-up (graph ids, masses, cuts, lists, singleton
   * start, Q_old), [5] download of the results */
  double host_ms[8];
  double q_phase[200];
  int64_t loops_phase[200];
  int64_t nv_phase[200];
  int64_t ne_phase[200];
  double q_ms;         /* device time of the modularity evaluations */
  double agg_ms;       /* device time of the aggregations (coarsening) */
} nido_run_stats;

/* ---- library ---------------------------------------------------------------- */
const char* nido_last_error(void);
const char* nido_version(void);
/* number of kernels this library has launched in the process (all contexts) */
uint64_t nido_launch_count(void);

/* ---- context: one CUDA device + one stream; one per host thread ----------- */
/* Replaces GraphGPU's per-device setup (graph_gpu.cpp:33-100). */
int nido_ctx_create(int device, size_t hbm_budget_bytes, nido_ctx* out);
int nido_ctx_destroy(nido_ctx ctx);
int nido_ctx_sync(nido_ctx ctx);
/* the ctx's cudaStream_t, for callers that order their own work with it */
int nido_ctx_stream(nido_ctx ctx, void** stream);
/* Device blocks freed by this context's graphs stay with the context and are
 * reused by its later uploads and runs (no cudaMalloc / cudaFree between
 * graphs).  This returns the free ones to the driver; released_bytes (may be
 * null) receives their size.  Destroying the context does the same. */
int nido_ctx_trim(nido_ctx ctx, size_t* released_bytes);
/* Self-check of the bounded device waits (no reference counterpart): a kernel
 * waits on a barrier nothing arrives at, with the wait the move kernels use
 * (an attempt count and about one second of %globaltimer); it must give up.
 * *gave_up = 1 when it did, *waited_ms the time it waited; the context stays
 * usable.  Kernels whose bounded waits give up count it in the run's error
 * counter, which nido_run / nido_batch_run report as a failure. */
int nido_check_bounded_wait(nido_ctx ctx, int32_t* gave_up, int32_t* waited_ms);

/* ---- graphs ----------------------------------------------------------------- */
/* Upload a CSR and compute k_v and m.  Replaces the GraphGPU constructor
 * (graph_gpu.cpp:19-185: H2D copies, sum_vertex_weights, compute_mass,
 * partition_graph_edge_batch).  nbatches sets the -b cuts. */
int nido_graph_upload(nido_ctx ctx, int64_t nv, int64_t ne, const int64_t* off,
                      const int64_t* adj, const double* w, int32_t nbatches,
                      nido_graph* out);
/* Read a Vite binary straight into device memory: the reference's Graph(file)
 * (graph.cpp:322-495) followed by the GraphGPU upload, without the host CSR.
 * Header and offsets are read on the host (offsets not starting at 0 are
 * rebased; a header edge count that differs from the offsets prints the
 * reference's warning); the 16-byte edge records stream through pinned
 * buffers, read by parallel preads while the previous chunk is copied, and
 * are split into ids and weights on the device.  Same checks and result as
 * nido_read_vite + nido_graph_upload; NIDO_E_IO for a missing or truncated
 * file. */
int nido_graph_upload_vite(nido_ctx ctx, const char* path, int32_t nbatches, nido_graph* out);
int nido_graph_free(nido_graph g);
/* sizes of the current (possibly coarsened) graph */
int nido_graph_size(nido_graph g, int64_t* nv, int64_t* ne);
/* download the current CSR (caller sizes from nido_graph_size) */
int nido_graph_download(nido_graph g, int64_t* off, int64_t* adj, double* w);
/* batch cut points of the current graph, nbatches+1 entries
 * (GraphGPU::vertex_per_batch_, graph_gpu.cpp:280-359); NIDO_E_INVALID after a
 * run with colour-class batches, whose batches are not vertex ranges */
int nido_graph_batches(nido_graph g, int64_t* cuts);
/* k_v (vertexWeights_) and m (mass_) of the current graph */
int nido_graph_vertex_weights(nido_graph g, double* k, double* m);
/* Return to the uploaded graph (undo coarsening) with a singleton partition,
 * from the device-resident original CSR.  The reference has no counterpart:
 * it re-reads and re-uploads the file (graph_gpu.cpp:19-185). */
int nido_graph_reset(nido_graph g);

/* Page-lock a caller's host buffer so uploads and downloads run at full
 * link bandwidth (cudaHostRegister); the reference uses pinned buffers via
 * CudaMallocHost (cuda_wrapper.hpp:22-25). */
int nido_host_register(void* ptr, size_t bytes);
int nido_host_unregister(void* ptr);

/* ---- step-level operators: GraphGPU's public methods (graph_gpu.hpp:172-241) */
int nido_singleton_partition(nido_graph g);                  /* graph_gpu.cpp:519-536 */
int nido_set_community_ids(nido_graph g, const int64_t* comm);/* graph_gpu.cpp:433-448 */
int nido_compute_community_weights(nido_graph g);            /* graph_gpu.cpp:450-455 */
int nido_compute_modularity(nido_graph g, double* q);        /* graph_gpu.cpp:862-905 */
int nido_louvain_update(nido_graph g, int32_t batch, int32_t tie_mode); /* graph_gpu.cpp:602-624 */
int nido_update_community_weights(nido_graph g, int32_t batch);/* graph_gpu.cpp:779-791 */
int nido_update_community_ids(nido_graph g, int32_t batch);  /* graph_gpu.cpp:808-820 */
int nido_restore_community(nido_graph g);                    /* graph_gpu.cpp:822-842 */
/* aggregation (graph_gpu.cpp:1382-1545): renumber, compose the clustering,
 * coarsen in place; *done = 1 when the reference would stop (no merge, or one
 * community left). */
int nido_aggregation(nido_graph g, int32_t* done);
/* state download: commIds_, newCommIds_, commWeights_ (any may be NULL) */
int nido_get_state(nido_graph g, int64_t* comm, int64_t* newcomm, double* a);
/* clustering of the ORIGINAL vertices (Clustering::commIds_, clustering.hpp:7-41) */
int nido_get_clustering(nido_graph g, int64_t* clustering);
/* Clustering::dump_partition (clustering.cpp:23-46); new_orders may be NULL */
int nido_dump_partition(nido_graph g, const char* path, const int64_t* new_orders);

/* Modularity of a partition from caller-owned DEVICE arrays, allocating no
 * memory: for code that cannot call cudaMalloc (a stream being captured
 * into a CUDA graph, an allocator or memory-pool callback, a process whose
 * device memory is all handed to a fixed pool).  No counterpart in the
 * reference, whose modularity cudaMallocs a partials buffer on every call.
 * Layout as in the reference: d_off[nv+1] and d_adj (int64), d_w (FP64),
 * all non-null when nv > 0 (a graph without edges may pass any non-null
 * d_adj and d_w; they are not read), d_comm[nv] (int64 community ids in
 * [0, nv)), d_a[nv] community degrees
 * a_c indexed by community id, m the mass; Q is written to d_q (device) on
 * `stream` (a cudaStream_t, NULL for the legacy default stream), without a
 * host synchronisation.  The reduction follows the reference's order, so Q
 * matches nido_compute_modularity bit for bit on integer weights.
 * Scratch: a fixed 4 MiB array (524,280 FP64 group partials, the
 * reference's own maximum) inside the library, held by every GPU that loads
 * it until exit; it covers any nv up to the limit of 2^31-2 vertices, and
 * larger nv is rejected with NIDO_E_TOO_LARGE.  The first call on a device
 * looks up the array's device address (cudaGetSymbolAddress), so make that
 * first call before any stream capture.  All calls on a device share the
 * array: calls that overlap on the GPU race and return wrong values. */
int nido_modularity_noalloc(void* stream, int64_t nv, const int64_t* d_off, const int64_t* d_adj,
                            const double* d_w, const int64_t* d_comm, const double* d_a, double m,
                            double* d_q);

/* ---- degree tiers and their autotuner (no reference counterpart: the reference
 * bins by fixed degree bounds, graph_gpu.cpp:602-624) -------------------------- */
typedef struct {
  int32_t warp_max_degree;   /* one warp, 256-slot shared table; <= 192 */
  int32_t cta_s_max_degree;  /* 128-thread CTA, 1024 slots; <= 768 */
  int32_t cta_m_max_degree;  /* 256-thread CTA, 2048 slots; <= 1536 */
  int32_t cta_l_max_degree;  /* 256-thread CTA, 4096 slots; <= 3072 (default 2048) */
  int32_t cta_x_max_degree;  /* <= 12288; above: hub tier.  Degrees up to 6144 of this
                                range run on 512-thread CTAs with 8192 slots (two an
                                SM), the rest on 1024-thread CTAs with 16384 slots */
  int32_t hub_clusters;      /* 1: in integer-weight phases with the smallest-id rule,
                                hubs run on thread-block clusters of 2..16 CTAs whose
                                distributed shared memory holds the hub's table (when
                                every hub of the phase fits: degree <= 196,608);
                                0 (default): hub tables in global memory */
  int64_t hub_wave_slots;    /* hub-table slots processed together (L2 residency) */
  int32_t staged_edges;      /* 1: the CTA-S and CTA-M tiers copy the next vertex's ids and
                                weights into shared memory with 1-D bulk copies (TMA) while
                                the current vertex is evaluated; 0 (default): they read
                                them from global memory (faster on R-MAT scale 22) */
  int32_t reserved;          /* must be 0 */
} nido_tier_config;
/* Thresholds must be non-decreasing, at least 32 and within the capacities
 * above; results on integer weights do not depend on them. */
int nido_get_tier_config(nido_graph g, nido_tier_config* c);
int nido_set_tier_config(nido_graph g, const nido_tier_config* c);
/* Times `sweeps` move sweeps of every -b batch (no commit) on the graph's
 * current state for candidate configurations (coordinate descent over the
 * thresholds and the hub wave size), keeps the fastest and returns it with
 * its sweep time.  Overwrites the move targets: call it before a run
 * (nido_run starts from a fresh singleton partition). */
int nido_tune(nido_graph g, int32_t tie_mode, int32_t sweeps, nido_tier_config* best, double* best_ms);

/* ---- whole run: LouvainGPU::run (louvain_gpu.cpp:6-139) ------------------------ */
/* Starts from the uploaded graph (any earlier coarsening is undone first).
 * out_comm (nv entries, may be NULL) receives the clustering of the original
 * vertices; stats may be NULL. */
int nido_run(nido_graph g, const nido_params* p, int64_t* out_comm, nido_run_stats* stats);

/* ---- many graphs in one run (no reference counterpart: nido runs one graph per
 * process, louvain_gpu.cpp:6-139) ---------------------------------------------- */
typedef struct nido_batch_s* nido_batch;
/* Packs ngraphs independent graphs as one CSR over all their vertices: graph i
 * owns vertices [vbase[i], vbase[i+1]) (vbase has ngraphs+1 entries from 0 to
 * nv), neighbour ids are global, and every edge must stay inside its graph
 * (NIDO_E_INVALID otherwise).  nbatches is the -b of every graph. */
int nido_batch_upload(nido_ctx ctx, int32_t ngraphs, const int64_t* vbase, int64_t nv, int64_t ne,
                      const int64_t* off, const int64_t* adj, const double* w, int32_t nbatches,
                      nido_batch* out);
/* Runs every graph to completion in one phase loop.  Each graph's result is
 * the one nido_run gives for it alone (identical on integer weights).
 * out_comm (nv entries): each vertex's community, numbered within its graph;
 * out_q, out_phases, out_loops (ngraphs entries): final Q, phases and total
 * loops of every graph.  Any output may be NULL. */
int nido_batch_run(nido_batch b, const nido_params* p, int64_t* out_comm, double* out_q,
                   int64_t* out_phases, int64_t* out_loops, nido_run_stats* stats);
int nido_batch_size(nido_batch b, int32_t* ngraphs, int64_t* nv, int64_t* ne);
int nido_batch_free(nido_batch b);

/* ---- serving: a request loop with continuous batching on one GPU (no reference
 * counterpart) ------------------------------------------------------------------ */
typedef struct nido_server_s* nido_server;
typedef struct {
  int32_t status;      /* NIDO_OK or the run's error code */
  int32_t worker;      /* worker (stream) that ran it */
  double final_q;
  int64_t phases;
  int64_t total_loops;
  double queue_ms;     /* submit -> admitted on a worker */
  double run_ms;       /* admitted -> result in host memory */
  double latency_ms;   /* submit -> result in host memory */
  double device_ms;    /* device-event time of the run */
  int64_t hbm_bytes;   /* reservation held against the budget while it ran */
  int32_t host_edges;  /* 1: admitted over budget, edges in mapped host memory */
  int32_t pad;
} nido_request_info;
/* Device bytes reserved for a graph of this size while it runs: the upload,
 * work buffers and scratch, plus the hub-table and coarsening-plan regions,
 * which are processed in waves and so bounded by max(8M, 4*nv) and
 * max(4M, 4*nv) slots. */
int64_t nido_graph_footprint(int64_t nv, int64_t ne, int32_t nbatches);
/* Over-budget graphs (no reference counterpart in this form; the reference
 * streams edge windows per batch, graph_gpu.cpp:362-417, 967-1042): when a
 * context with a budget cannot hold a graph's edges in HBM but can hold the
 * rest, the upload keeps the three CSR copies' edge arrays (12 bytes an edge
 * each) in page-locked host memory mapped into the device's address space,
 * and every kernel streams them over the host link as it reads them.  Results
 * are the in-HBM run's.  This is the HBM such a graph reserves. */
int64_t nido_graph_footprint_streamed(int64_t nv, int64_t ne, int32_t nbatches);
/* 1 when the graph's edges are in mapped host memory (see above) */
int nido_graph_host_edges(nido_graph g, int32_t* host_edges);
/* Device bytes a graph holds now (upload, scratch, hub tables, plan). */
int nido_graph_device_bytes(nido_graph g, int64_t* bytes);
/* nworkers threads, each with its own stream; requests are admitted in
 * arrival order while their footprints fit in the budget (0: all free HBM
 * less 1 GiB; never more than that).  A request whose footprint exceeds the
 * whole budget runs with its edges in mapped host memory when its streamed
 * footprint fits (nido_request_info.host_edges). */
int nido_server_create(int device, size_t hbm_budget_bytes, int32_t nworkers, nido_server* out);
/* Queues a run of g with p.  g's arrays and out_comm (nv entries, may be
 * NULL) must stay valid until nido_server_wait returns for *ticket.  A
 * request whose streamed footprint exceeds the whole budget is refused
 * (NIDO_E_TOO_LARGE). */
int nido_server_submit(nido_server s, const nido_csr* g, const nido_params* p, int64_t* out_comm,
                       int64_t* ticket);
/* *state: 0 queued, 1 running, 2 finished */
int nido_server_poll(nido_server s, int64_t ticket, int32_t* state);
/* Blocks until the request finishes (timeout_s < 0: no limit); NIDO_E_TIMEOUT
 * leaves the ticket valid.  Returns the request's own status and releases
 * the ticket.  One waiter per ticket: a wait on a ticket that another thread
 * is already waiting on returns NIDO_E_INVALID at once.  Submissions and
 * waits on other tickets may proceed from any thread meanwhile. */
int nido_server_wait(nido_server s, int64_t ticket, double timeout_s, nido_request_info* info);
/* budget, bytes reserved by running requests, running and queued counts */
int nido_server_budget(nido_server s, int64_t* budget, int64_t* reserved, int32_t* running,
                       int32_t* queued);
/* Finishes every queued request, then stops the workers. */
int nido_server_destroy(nido_server s);

/* ---- colouring for -c (Graph::coloring, graph.cpp:548-694) ---------------------- */
/* Jones-Plassmann-Luby colouring on the device; colors has nv entries;
 * returns the number of colours in *ncolors. Proper (no two neighbours share a
 * colour) and deterministic for a given seed. */
int nido_color(nido_ctx ctx, const nido_csr* in, uint64_t seed, int64_t* colors,
               int64_t* ncolors);
/* relabel by (colour, id) as graph.cpp:611-693: out gets the permuted CSR (its
 * arrays caller-allocated with the input sizes), new_orders[p] = old id */
int nido_color_relabel(nido_ctx ctx, const nido_csr* in, const int64_t* colors,
                       nido_csr* out, int64_t* new_orders);

/* ---- Vite binary files (graph.cpp:322-495) -------------------------------------- */
int nido_read_vite(const char* path, nido_csr* out); /* arrays malloc'ed */
int nido_write_vite(const char* path, const nido_csr* g);
void nido_csr_free(nido_csr* g);

/* ---- seeded synthetic generators (test and benchmark inputs) -------------------- */
/* weight modes */
#define NIDO_W_ONE 0       /* all 1.0; duplicate edges dropped */
#define NIDO_W_UNIFORM 1   /* U[0.5, 1.5]; duplicates merged by summing */
#define NIDO_W_LOGNORMAL 2 /* lognormal(0, 0.5); duplicates summed */
#define NIDO_W_INT8 3      /* integers uniform in {1..8}; duplicates summed */
int nido_gen_planted(int64_t nblocks, int64_t block_size, double avg_degree,
                     double p_intra, int32_t wmode, uint64_t seed, nido_csr* out);
int nido_gen_rmat(int64_t nv, int64_t npairs, double a, double b, double c,
                  int32_t wmode, uint64_t seed, nido_csr* out);
int nido_gen_sbm(int64_t nv, double alpha, int64_t cmin, int64_t cmax,
                 double avg_degree, double p_intra, int32_t wmode, int32_t permute,
                 uint64_t seed, nido_csr* out);

#ifdef __cplusplus
}
#endif
#endif /* NIDO_B200_H_ */
