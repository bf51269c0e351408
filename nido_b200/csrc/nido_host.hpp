// nido_host.hpp -- the reference's host classes (Graph, Clustering,
// GraphGPU, LouvainGPU) as thin C++ wrappers over the C ABI of
// libnido_b200.so, with the reference's names and meanings:
//   Graph       graph.hpp:14-102      Vite reader, CSR accessors, print_stats, coloring
//   Clustering  clustering.hpp:7-41   composed community ids, dump_partition
//   GraphGPU    graph_gpu.hpp:14-248  device graph and step operators
//   LouvainGPU  louvain_gpu.hpp:6-24  the phase / iteration driver
// Failures print the library's message and exit, as the reference does on
// a file it cannot open (graph.cpp:437-441).
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

using GraphElem = int64_t;
using GraphWeight = double;

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
  ~Graph() { nido_csr_free(&g_); }
  Graph(const Graph&) = delete;
  Graph& operator=(const Graph&) = delete;

  GraphElem get_num_vertices() const { return g_.nv; }
  GraphElem get_num_edges() const { return g_.ne; }
  GraphElem get_num_adjacent_vertices(GraphElem i) const { return g_.off[i + 1] - g_.off[i]; }
  GraphElem* get_adjacent_vertices(GraphElem i) { return g_.adj + g_.off[i]; }
  GraphWeight* get_adjacent_weights(GraphElem i) { return g_.w + g_.off[i]; }
  GraphElem* get_index_ranges() { return g_.off; }
  GraphElem* get_edges() { return g_.adj; }
  GraphWeight* get_edge_weights() { return g_.w; }
  GraphElem get_max_order() const {
    GraphElem m = 0;
    for (GraphElem v = 0; v < g_.nv; ++v) m = std::max(m, g_.off[v + 1] - g_.off[v]);
    return m;
  }
  const nido_csr& csr() const { return g_; }

  // graph.cpp:280-320 (degree statistics)
  void print_stats() const { print_graph_stats(g_.off, g_.nv, g_.ne); }

  // graph.cpp:651-797: colour, relabel the CSR in place so that colour
  // classes are contiguous, return new_orders (new position -> old id);
  // release with delete[].
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
    nido_csr_free(&g_);
    g_ = out;
    num_colors_ = ncolors;
    return new_orders;
  }
  GraphElem num_colors() const { return num_colors_; }

 private:
  nido_csr g_{};
  GraphElem num_colors_ = 0;
};

class GraphGPU {
 public:
  GraphGPU(Graph* graph, int nbatches, nido_ctx ctx) : nv0_(graph->get_num_vertices()) {
    const nido_csr& c = graph->csr();
    nido_check(nido_graph_upload(ctx, c.nv, c.ne, c.off, c.adj, c.w, nbatches, &g_), "GraphGPU");
  }
  // Graph(file) + GraphGPU in one step: the Vite file streams to the device
  // (nido_graph_upload_vite) and only the offsets come back for the
  // statistics the reference prints while reading.
  GraphGPU(const std::string& binfile, int nbatches, nido_ctx ctx) {
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
  ~GraphGPU() { nido_graph_free(g_); }
  GraphGPU(const GraphGPU&) = delete;
  GraphGPU& operator=(const GraphGPU&) = delete;

  void set_community_ids(const GraphElem* c) { nido_check(nido_set_community_ids(g_, c), "set_community_ids"); }
  void singleton_partition() { nido_check(nido_singleton_partition(g_), "singleton_partition"); }
  GraphWeight compute_modularity() {
    double q = 0.;
    nido_check(nido_compute_modularity(g_, &q), "compute_modularity");
    return q;
  }
  void louvain_update(int batch, int tie = NIDO_TIE_SMALLEST_ID) {
    nido_check(nido_louvain_update(g_, batch, tie), "louvain_update");
  }
  void update_community_weights(int batch) {
    nido_check(nido_update_community_weights(g_, batch), "update_community_weights");
  }
  void update_community_ids(int batch) { nido_check(nido_update_community_ids(g_, batch), "update_community_ids"); }
  void restore_community() { nido_check(nido_restore_community(g_), "restore_community"); }
  bool aggregation() {
    int32_t done = 0;
    nido_check(nido_aggregation(g_, &done), "aggregation");
    return done != 0;
  }
  void dump_partition(const std::string& file, const GraphElem* new_orders) {
    nido_check(nido_dump_partition(g_, file.c_str(), new_orders), "dump_partition");
  }
  nido_graph handle() const { return g_; }
  GraphElem original_vertices() const { return nv0_; }

 private:
  nido_graph g_ = nullptr;
  GraphElem nv0_;
};

class LouvainGPU {
 public:
  LouvainGPU(GraphElem maxLoops, GraphWeight tol, int nbatches, int tie = NIDO_TIE_SMALLEST_ID)
      : maxLoops_(maxLoops), tol_(tol), nbatches_(nbatches), tie_(tie) {}
  // louvain_gpu.cpp:6-139, printing the reference's per-loop and summary lines
  nido_run_stats run(GraphGPU* graph, bool verbose = true) {
    nido_params p{};
    p.nbatches = nbatches_;
    p.tie_mode = tie_;
    p.tau = tol_;
    p.max_iter = maxLoops_;
    p.verbose = verbose ? 1 : 0;
    nido_run_stats st{};
    nido_check(nido_run(graph->handle(), &p, nullptr, &st), "LouvainGPU::run");
    if (verbose) {
      const double total = st.total_ms / 1e3;
      printf("Total time elapse: %g s\n", total);
      printf("Total Loops: %lld\n", (long long)st.total_loops);
      printf("Time per loop: %g s/loop\n", st.total_loops ? total / st.total_loops : 0.);
    }
    return st;
  }

 private:
  GraphElem maxLoops_;
  GraphWeight tol_;
  int nbatches_;
  int tie_;
};

#endif
