// engine.cuh -- device state of one graph and the kernel launchers that
// operate on it.
//
// HBM layout of a graph (all arrays resident for the whole run):
//   off   int64[nv+1]   CSR offsets            adj  int32[ne]  neighbour ids
//   w     f64[ne]       edge weights           k    f64[nv]    vertex weights k_v
//   comm  int32[nv]     community ids          newc int32[nv]  move targets / undo ids
//   a     f64[nv]       community degrees a_c (indexed by community id)
//   clus  int32[nv0]    clustering of the original vertices
//   perm  int32[nv]     vertex list ordered by (batch, degree tier, id)
// plus ping-pong CSR buffers for coarsening and a scratch arena.
#ifndef NIDO_ENGINE_CUH_
#define NIDO_ENGINE_CUH_
#include <cuda_runtime.h>
#include <stdint.h>

#include <map>
#include <unordered_map>
#include <vector>

#include "common.cuh"

// degree tiers of the move / modularity kernels
enum Tier {
  kTierG4 = 0,  // d <= 4   : 4-lane group per vertex, registers
  kTierG8,      // d <= 8   : 8-lane group
  kTierG16,     // d <= 16  : 16-lane group
  kTierG32,     // d <= 32  : one warp, registers
  kTierWarp,    // d <= 192  : one warp, shared-memory hash (256 slots)
  kTierCtaS,    // d <= 768  : one 128-thread CTA, shared-memory hash (1024 slots)
  kTierCtaM,    // d <= 1536 : one 256-thread CTA, shared-memory hash (2048 slots)
  kTierCtaL,    // d <= 3072 : one 256-thread CTA, shared-memory hash (4096 slots)
  kTierCtaXA,   // d <= 6144 : one 512-thread CTA, shared-memory hash (8192 slots, 96 KB: two CTAs an SM)
  kTierCtaX,    // d <= 12288: one 1024-thread CTA, shared-memory hash (16384 slots, 192 KB, load <= 3/4)
  kTierHub,     // larger    : 2048-edge segments on many CTAs, hash in global memory (L2)
  kNumTiers
};

// largest degree each shared-memory tier accepts: its table (256 / 1024 /
// 2048 / 4096 / 16384 slots) filled to at most 3/4
constexpr int kWarpMaxDeg = 192;
constexpr int kCtaSMaxDeg = 768;
constexpr int kCtaMMaxDeg = 1536;
constexpr int kCtaLMaxDeg = 3072;
constexpr int kCtaXAMaxDeg = 6144;  // table load up to 3/4 in the 8192 slots
constexpr int kCtaXMaxDeg = 12288;  // table load up to 3/4 in the 16384 slots
constexpr int kHubSeg = 2048;        // edges of one hub segment (move and modularity)

// Degree thresholds of the shared-memory tiers, the hub wave size and the
// hub-cluster option.  The defaults are the kernels' capacities except for
// CTA-L (measured below); the tuner (engine.cu) may move the thresholds (a
// tier takes any degree up to its capacity), pick the wave and the option.
struct TierConfig {
  int32_t warp_max = kWarpMaxDeg;
  int32_t ctas_max = kCtaSMaxDeg;
  int32_t ctam_max = kCtaMMaxDeg;
  // degree 2049..3072 runs faster on the 1024-thread tier since the tables
  // sum in int32 (R-MAT scale 22: 113.4 -> 110.3 ms of move phase)
  int32_t ctal_max = 2048;
  int32_t ctax_max = kCtaXMaxDeg;
  int64_t hub_wave_slots = (int64_t)4 << 20;
  bool hub_clusters = false;  // hubs on thread-block clusters where they fit
  // CTA-S / CTA-M vertices' edges staged in shared memory by bulk copies
  // (move.cu); off by default: slower on R-MAT scale 22 with a warm L2
  bool staged_edges = false;
};

struct nido_ctx_s {
  int device = 0;
  cudaStream_t stream = nullptr;
  size_t budget = 0;
  size_t used = 0;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  std::vector<cudaEvent_t> move_ev;  // 2 per batch, for per-iteration move timing
  // side streams of the move sweep: the degree tiers of one batch touch
  // disjoint vertices, so the hub chain and the CTA tiers run beside the
  // small-degree tiers (fork and join events on the context's stream)
  cudaStream_t aux[2] = {nullptr, nullptr};
  cudaEvent_t fork_ev = nullptr;
  cudaEvent_t join_ev[2] = {nullptr, nullptr};
  // stream-ordered allocation (cudaMallocFromPoolAsync / cudaFreeAsync on the
  // context's stream): allocating or freeing then does not wait for the work
  // of other contexts on the same GPU.  The pool is the owner's (the serving
  // loop creates one for its workers), so the device's default pool and its
  // settings are left alone.
  bool async_alloc = false;
  cudaMemPool_t pool = nullptr;
  // device-resident phase loops (loop.cu, params.host_loop = 2) are possible
  // until the CUDA driver turns out to lack conditional graph nodes
  bool device_loop = true;
  // otherwise blocks come from cudaMalloc and are kept for reuse when freed
  // (raw_alloc / raw_free): free blocks by size, the size of every block in
  // use, and the bytes held in free blocks
  std::multimap<size_t, void*> free_blocks;
  std::unordered_map<void*, size_t> live_blocks;
  size_t cached_bytes = 0;
  // pinned host staging of nido_graph_upload_vite (grows, kept until destroy)
  void* pinned = nullptr;
  size_t pinned_bytes = 0;
};

struct nido_graph_s {
  nido_ctx ctx = nullptr;
  int64_t nv0 = 0;           // original vertex count
  int64_t nv = 0, ne = 0;    // current phase
  int64_t cap_v = 0, cap_e = 0;
  int nbatches = 1;          // batches of the current phase
  int nb_user = 1;           // the -b the graph was uploaded with
  // conflict-free batches: every phase colours the current graph (JPL, seed
  // kColorBatchSeed) and its colour classes are the batches, in colour order
  bool color_mode = false;
  int32_t* vcolor = nullptr; // colour of every current vertex (color_mode)
  int64_t cap_vcolor = 0;
  // every weight of the current phase integral and every vertex's sum of |w|
  // below 2^31 (set with k_v each phase; the move phase then sums in int32)
  bool int_weights = false;
  double m = 0.0;            // host copy of the mass

  int64_t ne0 = 0;           // original edge count
  bool coarsened = false;    // current CSR is a coarse graph
  // current CSR (points at the original or at the work buffers)
  int64_t* off = nullptr;
  int32_t* adj = nullptr;
  double* w = nullptr;
  // original CSR, never modified: runs restart from it without a host copy
  int64_t* off0 = nullptr;
  int32_t* adj0 = nullptr;
  double* w0 = nullptr;
  // work CSR that holds coarse graphs
  int64_t* offA = nullptr;
  int32_t* adjA = nullptr;
  double* wA = nullptr;
  // coarsening temporaries (per-coarse-vertex lists before compaction)
  int64_t* off2 = nullptr;
  int32_t* adj2 = nullptr;
  double* w2 = nullptr;
  double* k = nullptr;
  double* a = nullptr;
  int32_t* comm = nullptr;
  int32_t* newc = nullptr;
  int32_t* clus = nullptr;
  int32_t* perm = nullptr;
  double* dm = nullptr;      // device scalars: [0] m, [1] Q, [2..] spare
  int64_t* dcount = nullptr; // device counters
  // scratch arena (bytes), carved per operation
  char* scratch = nullptr;
  size_t scratch_bytes = 0;
  // hub tier of the move phase: per-hub tables in global memory (gslab slots
  // in all) and (hub, segment) work items, planned once per phase
  int32_t* gkeys = nullptr;
  double* gvals = nullptr;
  int64_t gslab = 0;
  // the same region as packed 64-bit slots (id, int32 sum) for integer-weight
  // phases; gslab_need is the current plan's size
  unsigned long long* gpacked = nullptr;
  int64_t gslab_packed = 0, gslab_need = 0;
  int2* hub_items = nullptr;
  int32_t* hub_v = nullptr;
  int32_t* hub_capv = nullptr;
  int32_t* hub_nseg = nullptr;
  int64_t* hub_toff = nullptr;
  int32_t* hub_done = nullptr;
  int64_t hub_cap_items = 0, hub_cap_hubs_v = 0, hub_cap_hubs_c = 0, hub_cap_hubs_s = 0,
          hub_cap_hubs_t = 0, hub_cap_hubs_d = 0;
  int64_t nhubs = 0;
  // waves of hubs whose tables fit in L2 together: item, slice and hub ranges
  struct HubWave {
    int64_t i0, i1, s0, s1, h0, h1;
  };
  std::vector<HubWave> hub_waves;
  std::vector<int64_t> hub_wave_off;  // waves of each batch
  // table slices scanned in parallel, their per-slice results, and the hub
  // index range of every batch
  int2* hub_slices = nullptr;
  int64_t* hub_slice_first = nullptr;
  char* hub_res = nullptr;
  int64_t hub_cap_slices = 0, hub_cap_first = 0, hub_cap_res = 0;
  // first segment item of every hub (nhubs + 1; items run in hub order) and
  // the per-item partial in-community sums of the modularity
  int64_t* hub_item_first = nullptr;
  double* hub_part = nullptr;
  int64_t hub_cap_ifirst = 0, hub_cap_part = 0, hub_nitems = 0;
  // hub vertices of every batch by cluster size (2, 4, 8, 16 CTAs sharing
  // one table in their distributed shared memory): hub_cl_off[batch * 4 +
  // bin] is the first list entry; hub_cl_ok when every hub of the phase fits
  int32_t* hub_cl_v = nullptr;
  int64_t hub_cap_cl = 0;
  std::vector<int64_t> hub_cl_off;
  bool hub_cl_ok = false;
  // coarsening plan and tables of giant coarse vertices (grows, never shrinks,
  // so runs after the first allocate nothing)
  char* agg_buf = nullptr;
  size_t agg_buf_bytes = 0;
  int32_t* pm32 = nullptr;   // member of every 32-position block of the member-edge lists
  int64_t pm32_cap = 0;

  // many-graph mode (null / empty for one graph): the graph of every current
  // vertex and the mass of every graph; vbatch (optional) receives every
  // vertex's batch relative to its own graph's -b cuts
  int32_t* gid = nullptr;
  double* mg = nullptr;
  int32_t* vbatch = nullptr;
  int64_t* gbase = nullptr;   // first vertex of every graph (ngraphs+1)
  int64_t* gcuts = nullptr;   // -b cuts of every graph, relative (ngraphs*(nbatches+1))
  int32_t* gactive = nullptr; // graph iterating in the current phase
  int64_t* gbase2 = nullptr;  // first vertex of every graph after coarsening
  int32_t ngraphs = 1;

  std::vector<int64_t> cuts;     // host batch cuts (nbatches+1)
  std::vector<int64_t> tier_off; // host: nbatches*kNumTiers+1 offsets into perm
  bool bins_valid = false;
  int64_t max_degree = 0;
  TierConfig cfg;
  bool tuned = false;
  // the move sweep of every batch captured as a CUDA graph, replayed for the
  // later sweeps of a phase (plan_epoch changes whenever the tier lists or
  // the hub plan are rebuilt)
  struct MoveGraph {
    cudaGraphExec_t exec = nullptr;
    int tie = -1;
    int64_t epoch = -1;
    int uses = 0;
    uint64_t kernels = 0;
  };
  std::vector<MoveGraph> move_graphs;
  int64_t plan_epoch = 0;
  bool use_graphs = true;
  // over-budget graphs: the edge arrays (adj0/w0, adjA/wA, adj2/w2) live in
  // page-locked host memory mapped into the device's address space, and the
  // kernels stream them over the host link as they read them
  bool host_edges = false;
  // device-resident iteration loop (loop.cu): its control block and per-loop log
  char* loop_buf = nullptr;
  size_t loop_bytes = 0;
  double host_pinned_dummy = 0;
};

namespace nido {

// bump allocation inside the graph's scratch arena
struct Arena {
  char* base;
  size_t size;
  size_t used = 0;
  Arena(char* b, size_t s) : base(b), size(s) {}
  template <typename T>
  T* take(int64_t n) {
    size_t off = (used + 255) & ~(size_t)255;
    size_t bytes = sizeof(T) * (size_t)(n > 0 ? n : 1);
    if (off + bytes > size) return nullptr;
    used = off + bytes;
    return reinterpret_cast<T*>(base + off);
  }
};

// phase-level kernels (phase.cu)
int launch_vertex_weights(nido_graph_s* g);             // k_v, nido order
int launch_mass(nido_graph_s* g);                       // g->m (host) and dm[0]
int launch_singleton(nido_graph_s* g);
int launch_set_comm(nido_graph_s* g);                   // a from comm
int launch_commit(nido_graph_s* g, int64_t v0, int64_t v1);
int launch_modularity(nido_graph_s* g, double* q);      // host value
int launch_modularity_dev(nido_graph_s* g);             // into g->dm[1], no host sync
int launch_commit_gated(nido_graph_s* g, int64_t v0, int64_t v1, const int32_t* gate);
int launch_q_self(nido_graph_s* g, double* selfv);      // per-vertex in-community weight
int graph_prepare_phase(nido_graph_s* g);               // k, m, tier lists (engine.cu)
// device memory of a context: stream-ordered when ctx->async_alloc (engine.cu)
cudaError_t raw_alloc(nido_ctx_s* ctx, void** p, size_t bytes);
void raw_free(nido_ctx_s* ctx, void* p);  // null is a no-op
void release_cached(nido_ctx_s* ctx);     // cudaFree every cached free block
// the context's pinned host staging buffer, grown to at least `bytes`
cudaError_t pinned_buffer(nido_ctx_s* ctx, size_t bytes, void** p);
// device memory counted against the context's HBM budget (engine.cu)
int device_alloc(nido_ctx_s* ctx, void** p, size_t bytes);
void device_free(nido_ctx_s* ctx, void* p, size_t bytes);
int build_batches(nido_graph_s* g);                     // cuts (host) + tier lists
int compact_batches(nido_graph_s* g);                   // many graphs: drop stopped graphs' vertices
// vertices in the tier lists (vertices with at least one edge)
inline int64_t listed_vertices(const nido_graph_s* g) {
  return g->tier_off.empty() ? g->nv : g->tier_off[(size_t)kNumTiers * g->nbatches];
}
// the commit of batch b: the vertex range [cuts[b], cuts[b+1]), or with
// colour-class batches the batch's vertices in the tier lists
int launch_commit_batch(nido_graph_s* g, int b);
constexpr uint64_t kColorBatchSeed = 1;
int color_current_graph(nido_graph_s* g, uint64_t seed, int32_t* colors, int64_t* ncolors);  // color.cu
// move phase (move.cu)
// ev_start / ev_end (may be null) are recorded around the tier kernels
int launch_move(nido_graph_s* g, int batch, int tie, cudaEvent_t ev_start, cudaEvent_t ev_end);
int launch_move_tiers(nido_graph_s* g, int batch, int tie);  // enqueue only (capturable)
int check_bounded_wait(nido_ctx_s* ctx, int32_t* gave_up, int32_t* waited_ms);  // move.cu
int plan_hubs(nido_graph_s* g);          // per phase, after the tier lists
int move_init_attributes();              // once per device
// times `sweeps` move sweeps (no commit) for candidate tier configurations
// and keeps the fastest in g->cfg (engine.cu); clobbers newc
int tune_tiers(nido_graph_s* g, int tie, int sweeps, double* best_ms);
// the iteration loop of one phase on the device (loop.cu)
constexpr int64_t kLoopLogCap = 65536;  // per-loop (Qtmp, dQ) entries kept for printing
struct PhaseLoop {
  double q_old = 0., q = 0.;
  int64_t loops = 0;
  double move_ms = 0., q_ms = 0.;
  double build_ms = 0.;     // host time to capture and instantiate the loop graph
  std::vector<double> log;  // Qtmp, dQ of every iteration (with want_log)
};
int device_phase_loop(nido_graph_s* g, int tie, double tau, int64_t max_iter, bool want_log, PhaseLoop* r,
                      bool* unsupported);
// coarsening (coarsen.cu)
int launch_aggregation(nido_graph_s* g, int* done);

}  // namespace nido
#endif
