// nido_host.hpp -- the reference's host classes as C++ over the C ABI of
// libnido_b200.so, with the reference's names, signatures and meanings:
//   Graph       graph.hpp:14-102       Vite reader, CSR accessors, print_stats, coloring
//   Clustering  clustering.hpp:7-41    composed community ids, dump_partition
//   GraphGPU    graph_gpu.hpp:168-247  device graph and its step operators
//   LouvainGPU  louvain_gpu.hpp:6-24   the phase / iteration driver
// A program written against the reference's classes compiles unchanged
// against this header (the reference's own header names are provided by
// include/nido_compat/, each of which includes this file).  Everything runs on
// one B200: the multi-GPU arguments keep their meaning for one device
// (host_id 0, part_on_device/part_on_batch 1) and other values are refused.
// Failures print the library's message and exit, as the reference does on a
// file it cannot open (graph.cpp:334-338).
#ifndef NIDO_HOST_HPP_
#define NIDO_HOST_HPP_
#include <stdio.h>
#include <stdlib.h>

#include <algorithm>
#include <cmath>
#include <numeric>
#include <string>
#include <vector>

#include "nido_b200.h"

// types.hpp:14-38 (64-bit build: int64 ids, FP64 weights)
using GraphElem = int64_t;
using GraphWeight = double;
using Int = int64_t;
using Float = double;
using UInt = uint64_t;
#ifndef MAX_PHASES
#define MAX_PHASES (200)
#endif
#ifndef DEFAULT_ITERATIONS
#define DEFAULT_ITERATIONS (500)
#endif
#ifndef DEFAULT_BATCHES
#define DEFAULT_BATCHES (2)
#endif
#ifndef DEFAULT_THRESHOLD
#define DEFAULT_THRESHOLD (1.0E-06)
#endif
#ifndef NGPU
#define NGPU 1
#endif

inline void nido_check(int st, const char* what) {
  if (st != NIDO_OK) {
    fprintf(stderr, "%s failed (%d): %s\n", what, st, nido_last_error());
    exit(EXIT_FAILURE);
  }
}

// Graph::print_stats (graph.cpp:280-320): degree statistics from the offsets.
inline void print_graph_stats(const GraphElem* off, GraphElem nv, GraphElem ne) {
  std::vector<GraphElem> pdeg(nv);
  for (GraphElem v = 0; v < nv; ++v) pdeg[v] = off[v + 1] - off[v];
  std::sort(pdeg.begin(), pdeg.end());
  GraphElem median = 0, mx = 0;
  double sum = 0., sq = 0.;
  if (nv > 0) {
    median = nv % 2 ? pdeg[nv / 2] : (pdeg[nv / 2 - 1] + pdeg[nv / 2]) / 2;
    mx = pdeg.back();
    for (GraphElem d : pdeg) { sum += (double)d; sq += (double)d * (double)d; }
  }
  const double avg = nv ? sum / nv : 0., avg_sq = nv ? sq / nv : 0.;
  const double var = std::abs(avg_sq - avg * avg);
  printf("\n--------------------------------------\nGraph characteristics\n");
  printf("--------------------------------------\n");
  printf("Number of vertices: %lld\nNumber of edges: %lld\n", (long long)nv, (long long)ne);
  printf("Maximum number of edges: %lld\nMedian number of edges: %lld\n", (long long)mx, (long long)median);
  printf("Expected value of X^2: %g\nVariance: %g\nStandard deviation: %g\n", avg_sq, var, std::sqrt(var));
  printf("--------------------------------------\n");
}

// One context for the duration of a host-class call that needs a device but
// was given none (the reference's classes take no device handle).
class ScopedContext {
 public:
  ScopedContext() { nido_check(nido_ctx_create(0, 0, &ctx_), "nido_ctx_create"); }
  ~ScopedContext() { nido_ctx_destroy(ctx_); }
  ScopedContext(const ScopedContext&) = delete;
  ScopedContext& operator=(const ScopedContext&) = delete;
  nido_ctx get() const { return ctx_; }

 private:
  nido_ctx ctx_ = nullptr;
};

class Graph {
 public:
  explicit Graph(const std::string& binfile) {
    int st = nido_read_vite(binfile.c_str(), &g_);
    if (st == NIDO_E_IO && g_.off == nullptr) {
      printf(" Error opening file! \n");
      fflush(stdout);
      abort();
    }
    nido_check(st, "Graph(binfile)");
    print_stats();
  }
  // Graph(totalVertices, m0): the reference's random Barabasi-Albert graph
  // (graph.cpp:137-160, the -r option), which this build does not provide.
  Graph(const GraphElem&, const GraphElem&) {
    fprintf(stderr, "-r (random graph) is not supported; generate a Vite binary and use -f\n");
    exit(EXIT_FAILURE);
  }
  ~Graph() { nido_csr_free(&g_); }
  Graph(const Graph&) = delete;
  Graph& operator=(const Graph&) = delete;

  GraphElem get_num_vertices() const { return g_.nv; }
  GraphElem get_num_edges() const { return g_.ne; }
  GraphElem get_num_adjacent_vertices(const GraphElem& i) const { return g_.off[i + 1] - g_.off[i]; }
  GraphElem* get_adjacent_vertices(const GraphElem& i) { return g_.adj + g_.off[i]; }
  GraphWeight* get_adjacent_weights(const GraphElem& i) { return g_.w + g_.off[i]; }
  GraphElem* get_index_ranges() { return g_.off; }
  GraphElem* get_edges() { return g_.adj; }
  GraphWeight* get_edge_weights() { return g_.w; }
  GraphElem get_max_order() const {
    GraphElem m = 0;
    for (GraphElem v = 0; v < g_.nv; ++v) m = std::max(m, g_.off[v + 1] - g_.off[v]);
    return m;
  }
  // degrees and weighted degrees of every vertex (neigh_scan, graph.cpp:190-213)
  GraphElem* get_orders() {
    orders_.resize(g_.nv);
    for (GraphElem v = 0; v < g_.nv; ++v) orders_[v] = g_.off[v + 1] - g_.off[v];
    return orders_.data();
  }
  GraphWeight* get_weighted_orders() {
    worders_.assign(g_.nv, 0.);
    for (GraphElem v = 0; v < g_.nv; ++v)
      for (GraphElem e = g_.off[v]; e < g_.off[v + 1]; ++e) worders_[v] += g_.w[e];
    return worders_.data();
  }
  const nido_csr& csr() const { return g_; }

  // graph.cpp:280-320 (degree statistics)
  void print_stats() const { print_graph_stats(g_.off, g_.nv, g_.ne); }

  // Graph::coloring (graph.cpp:548-694): colour the vertices, relabel the CSR
  // in place so that colour classes are contiguous in (colour, id) order and
  // return new_orders (new position -> old id), released with delete[].  The
  // colouring runs on the device (Jones-Plassmann-Luby); num_colors() and
  // color_offsets() then describe the classes of the relabelled CSR.
  GraphElem* coloring() {
    ScopedContext ctx;
    return coloring(ctx.get());
  }
  GraphElem* coloring(nido_ctx ctx, uint64_t seed = 1) {
    std::vector<int64_t> colors(g_.nv);
    int64_t ncolors = 0;
    nido_check(nido_color(ctx, &g_, seed, colors.data(), &ncolors), "coloring");
    nido_csr out;
    out.nv = g_.nv;
    out.ne = g_.ne;
    out.off = (int64_t*)malloc(8 * (g_.nv + 1));
    out.adj = (int64_t*)malloc(8 * (g_.ne > 0 ? g_.ne : 1));
    out.w = (double*)malloc(8 * (g_.ne > 0 ? g_.ne : 1));
    GraphElem* new_orders = new GraphElem[g_.nv > 0 ? g_.nv : 1];
    nido_check(nido_color_relabel(ctx, &g_, colors.data(), &out, new_orders), "coloring relabel");
    // colour classes of the relabelled graph: class c holds new ids
    // [color_off_[c], color_off_[c+1])
    color_off_.assign((size_t)ncolors + 1, 0);
    for (GraphElem v = 0; v < g_.nv; ++v) color_off_[(size_t)colors[v] + 1] += 1;
    std::partial_sum(color_off_.begin(), color_off_.end(), color_off_.begin());
    nido_csr_free(&g_);
    g_ = out;
    num_colors_ = ncolors;
    return new_orders;
  }
  GraphElem num_colors() const { return num_colors_; }
  const std::vector<GraphElem>& color_offsets() const { return color_off_; }

 private:
  nido_csr g_{};
  GraphElem num_colors_ = 0;
  std::vector<GraphElem> color_off_;
  std::vector<GraphElem> orders_;
  std::vector<GraphWeight> worders_;
};

// Clustering (clustering.hpp:7-41, clustering.cpp:1-46): the community of
// every original vertex, composed phase by phase.
class Clustering {
 public:
  explicit Clustering(const GraphElem& nv) : ids_((size_t)std::max<GraphElem>(nv, 0)) {
    std::iota(ids_.begin(), ids_.end(), (GraphElem)0);
  }
  // every original vertex i moves to commIdsHost[commIds[i]] (clustering.cpp:12-21)
  void update_clustering(GraphElem* commIdsHost) {
    for (GraphElem& c : ids_) c = commIdsHost[c];
  }
  // one "%lld\n" line per vertex; with new_orders (a colouring relabel) entry
  // i belongs to original vertex new_orders[i] (clustering.cpp:23-46)
  void dump_partition(const std::string& filename, GraphElem* new_orders) {
    if (new_orders) {
      std::vector<GraphElem> tmp(ids_.size());
      for (size_t i = 0; i < ids_.size(); ++i) tmp[(size_t)new_orders[i]] = ids_[i];
      ids_.swap(tmp);
    }
    FILE* f = fopen(filename.c_str(), "wt");
    if (!f) return;
    for (GraphElem c : ids_) fprintf(f, "%lld\n", (long long)c);
    fclose(f);
  }
  GraphElem get_num_vertices() const { return (GraphElem)ids_.size(); }
  GraphElem* get_community_ids() { return ids_.data(); }

 private:
  std::vector<GraphElem> ids_;
};

class GraphGPU {
 public:
  // GraphGPU(Graph*, nbatches, part_on_device, part_on_batch)
  // (graph_gpu.hpp:169, graph_gpu.cpp:19-185): uploads the graph, computes
  // k_v and m and cuts the -b batches.  One B200 holds the whole graph, so
  // the partitioning switches keep their default 1, 1 (other values are
  // refused, as the command line's -p is).  The device context is owned.
  GraphGPU(Graph* graph, const int& nbatches, const int& part_on_device, const int& part_on_batch)
      : nv0_(graph->get_num_vertices()) {
    if (part_on_device != 1 || part_on_batch != 1) {
      fprintf(stderr, "GraphGPU: only the default partitioning (1, 1) is supported on one GPU\n");
      exit(EXIT_FAILURE);
    }
    nido_check(nido_ctx_create(0, 0, &owned_), "nido_ctx_create");
    upload(graph, nbatches, owned_);
  }
  // the same on a caller's context
  GraphGPU(Graph* graph, const int& nbatches, nido_ctx ctx) : nv0_(graph->get_num_vertices()) {
    upload(graph, nbatches, ctx);
  }
  // Graph(file) + GraphGPU in one step: the Vite file streams to the device
  // (nido_graph_upload_vite) and only the offsets come back for the
  // statistics the reference prints while reading.
  GraphGPU(const std::string& binfile, const int& nbatches, nido_ctx ctx) : nbatches_(nbatches) {
    FILE* f = fopen(binfile.c_str(), "rb");
    if (!f) {
      printf(" Error opening file! \n");
      fflush(stdout);
      abort();
    }
    fclose(f);
    nido_check(nido_graph_upload_vite(ctx, binfile.c_str(), nbatches, &g_), "GraphGPU(binfile)");
    int64_t nv = 0, ne = 0;
    nido_check(nido_graph_size(g_, &nv, &ne), "GraphGPU(binfile)");
    std::vector<int64_t> off((size_t)nv + 1);
    nido_check(nido_graph_download(g_, off.data(), nullptr, nullptr), "GraphGPU(binfile)");
    nv0_ = nv;
    print_graph_stats(off.data(), nv, ne);
  }
  ~GraphGPU() {
    nido_graph_free(g_);
    if (owned_) nido_ctx_destroy(owned_);
  }
  GraphGPU(const GraphGPU&) = delete;
  GraphGPU& operator=(const GraphGPU&) = delete;

  // graph_gpu.cpp:433-448: community ids from the host, then a_c
  void set_community_ids(const GraphElem* commIds) {
    nido_check(nido_set_community_ids(g_, commIds), "set_community_ids");
  }
  void singleton_partition() { nido_check(nido_singleton_partition(g_), "singleton_partition"); }
  // graph_gpu.cpp:450-455: a_c = sum of k_v over the community's members
  void compute_community_weights(const int& host_id) {
    check_host(host_id, "compute_community_weights");
    nido_check(nido_compute_community_weights(g_), "compute_community_weights");
  }
  GraphWeight compute_modularity() {
    double q = 0.;
    nido_check(nido_compute_modularity(g_, &q), "compute_modularity");
    return q;
  }
  // graph_gpu.cpp:602-624: best moves of one -b batch, under the tie rule
  // set with set_tie_rule (smallest community id unless changed)
  void louvain_update(const int& batch, const int& host_id) {
    check_host(host_id, "louvain_update");
    nido_check(nido_louvain_update(g_, batch, tie_), "louvain_update");
  }
  // graph_gpu.cpp:779-791 and 808-820 (the engine fuses the degree update and
  // the id swap into the first call; the second only checks its arguments)
  void update_community_weights(const int& batch, const int& host_id) {
    check_host(host_id, "update_community_weights");
    nido_check(nido_update_community_weights(g_, batch), "update_community_weights");
  }
  void update_community_ids(const int& batch, const int& host_id) {
    check_host(host_id, "update_community_ids");
    nido_check(nido_update_community_ids(g_, batch), "update_community_ids");
  }
  void restore_community() { nido_check(nido_restore_community(g_), "restore_community"); }
  // graph_gpu.cpp:1382-1545: true when the reference would stop
  bool aggregation() {
    int32_t done = 0;
    nido_check(nido_aggregation(g_, &done), "aggregation");
    return done != 0;
  }
  void dump_partition(const std::string& file, GraphElem* new_orders) {
    nido_check(nido_dump_partition(g_, file.c_str(), new_orders), "dump_partition");
  }
  // Equal gains: NIDO_TIE_SMALLEST_ID (default) or NIDO_TIE_NIDO, the
  // reference's 8-lane strided rule, for louvain_update and LouvainGPU::run.
  void set_tie_rule(int tie) { tie_ = tie; }
  int tie_rule() const { return tie_; }
  // Conflict-free batches for LouvainGPU::run: every phase's colour classes
  // (device colouring of the phase's graph) are its batches, in colour order,
  // instead of the -b cuts.
  void set_color_batches(bool on) { color_batches_ = on; }
  bool color_batches() const { return color_batches_; }
  int nbatches() const { return nbatches_; }
  nido_graph handle() const { return g_; }
  GraphElem original_vertices() const { return nv0_; }

 private:
  void upload(Graph* graph, int nbatches, nido_ctx ctx) {
    const nido_csr& c = graph->csr();
    nbatches_ = nbatches;
    nido_check(nido_graph_upload(ctx, c.nv, c.ne, c.off, c.adj, c.w, nbatches, &g_), "GraphGPU");
  }
  static void check_host(int host_id, const char* what) {
    if (host_id != 0) {
      fprintf(stderr, "%s: host_id %d: this build runs on one GPU (host_id 0)\n", what, host_id);
      exit(EXIT_FAILURE);
    }
  }
  nido_graph g_ = nullptr;
  nido_ctx owned_ = nullptr;
  GraphElem nv0_ = 0;
  int nbatches_ = 1;
  int tie_ = NIDO_TIE_SMALLEST_ID;
  bool color_batches_ = false;
};

class LouvainGPU {
 public:
  // louvain_gpu.hpp:17-21: the loop stops when an iteration gains at most
  // tol; a phase is coarsened when it gained more than tol_phase (= tol
  // unless given)
  LouvainGPU(const Int& maxLoops, const Float& tol, const int& nbatches)
      : maxLoops_(maxLoops), tol_(tol), tol_phase_(tol), nbatches_(nbatches) {}
  LouvainGPU(const Int& maxLoops, const Float& tol, const Float& tol_phase, const int& nbatches)
      : maxLoops_(maxLoops), tol_(tol), tol_phase_(tol_phase), nbatches_(nbatches) {}

  // louvain_gpu.cpp:6-139, printing the reference's per-loop and summary lines
  nido_run_stats run(GraphGPU* graph, bool verbose = true) {
    nido_params p{};
    p.nbatches = nbatches_;
    p.tie_mode = graph->tie_rule();
    p.color_batches = graph->color_batches() ? 1 : 0;
    p.tau = tol_;
    p.tau_phase = tol_phase_;
    p.tau_phase_set = 1;
    p.max_iter = maxLoops_;
    p.verbose = verbose ? 1 : 0;
    nido_run_stats st{};
    nido_check(nido_run(graph->handle(), &p, nullptr, &st), "LouvainGPU::run");
    if (verbose) {
      const double total = st.total_ms / 1e3, agg = st.agg_ms / 1e3;
      printf("Total time elapse: %g s\n", total);
      printf("Total Loops: %lld\n", (long long)st.total_loops);
      printf("Time per loop: %g s/loop\n", st.total_loops ? (total - agg) / st.total_loops : 0.);
      printf("Aggregation time: %g s\n", agg);
      printf("Aggregation time: %g s\n", agg);
    }
    return st;
  }

 private:
  Int maxLoops_;
  Float tol_;
  Float tol_phase_;
  int nbatches_;
};

#endif
