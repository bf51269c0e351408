// ref_harness.cu -- drives the UNMODIFIED reference (sg0/nido) objects step
// by step so that its outputs can be recorded as golden fixtures.
//
// TEST INFRASTRUCTURE ONLY.  Built by oracle/Makefile.ref into oracle/_ref/
// against objects compiled from the reference sources in place; it runs on a
// B200 and writes raw little-endian arrays into an output directory.  The
// reference's private members are reached with -Dprivate=public on this
// translation unit only.
//
//   ref_harness move    g.bin assign.i64 nbatches batch outdir
//       set_community_ids(assign) (graph_gpu.cpp:433-448), louvain_update(
//       batch) (graph_gpu.cpp:602-624); writes newcomm.i64 (all vertices),
//       a.f64 (commWeights), k.f64 (vertexWeights), scalars.txt (m, Q)
//   ref_harness coarsen g.bin assign.i64 outdir
//       set_community_ids(assign), aggregation() (graph_gpu.cpp:1382-1545);
//       writes newid.i64, coff.i64, cadj.i64, cw.f64, scalars.txt
//   ref_harness run     g.bin nbatches tau maxloops out_partition
//       LouvainGPU::run (louvain_gpu.cpp:6-139) with 17-digit printing, then
//       dump_partition (clustering.cpp:23-46)
#include <cstdio>
#include <cstdlib>
#include <iomanip>
#include <iostream>
#include <string>
#include <vector>

#include "cuda_wrapper.hpp"
#include "graph.hpp"
#include "graph_gpu.hpp"
#include "louvain_gpu.hpp"
#include "types.hpp"

static std::vector<GraphElem> read_i64(const std::string& p) {
  FILE* f = fopen(p.c_str(), "rb");
  if (!f) { fprintf(stderr, "cannot open %s\n", p.c_str()); exit(2); }
  fseek(f, 0, SEEK_END);
  long n = ftell(f) / 8;
  fseek(f, 0, SEEK_SET);
  std::vector<GraphElem> v(n);
  if ((long)fread(v.data(), 8, n, f) != n) exit(2);
  fclose(f);
  return v;
}

template <typename T>
static void write_arr(const std::string& p, const T* x, size_t n) {
  FILE* f = fopen(p.c_str(), "wb");
  if (!f) { fprintf(stderr, "cannot write %s\n", p.c_str()); exit(2); }
  fwrite(x, sizeof(T), n, f);
  fclose(f);
}

static void write_scalars(const std::string& dir, double m, double q, long long extra) {
  FILE* f = fopen((dir + "/scalars.txt").c_str(), "w");
  fprintf(f, "m %.17g %016llx\nQ %.17g %016llx\nextra %lld\n", m,
          *(unsigned long long*)&m, q, *(unsigned long long*)&q, extra);
  fclose(f);
}

int main(int argc, char** argv) {
  if (argc < 3) { fprintf(stderr, "usage: see header\n"); return 2; }
  std::string mode = argv[1];
  Graph* g = new Graph(std::string(argv[2]));
  const GraphElem nv = g->get_num_vertices();
  if (mode == "move" && argc == 7) {
    std::vector<GraphElem> assign = read_i64(argv[3]);
    int nb = atoi(argv[4]), batch = atoi(argv[5]);
    std::string out = argv[6];
    GraphGPU* gg = new GraphGPU(g, nb, 1, 1);
    gg->set_community_ids(assign.data());
    double q = gg->compute_modularity();
    gg->louvain_update(batch, 0);
    CudaDeviceSynchronize();
    std::vector<GraphElem> nc(nv);
    std::vector<double> a(nv), k(nv);
    cudaMemcpy(nc.data(), gg->newCommIds_[0], 8 * nv, cudaMemcpyDeviceToHost);
    cudaMemcpy(a.data(), gg->commWeights_[0], 8 * nv, cudaMemcpyDeviceToHost);
    cudaMemcpy(k.data(), gg->vertexWeights_[0], 8 * nv, cudaMemcpyDeviceToHost);
    write_arr(out + "/newcomm.i64", nc.data(), nv);
    write_arr(out + "/a.f64", a.data(), nv);
    write_arr(out + "/k.f64", k.data(), nv);
    write_arr(out + "/cuts.i64", gg->vertex_per_batch_[0], nb + 1);
    write_scalars(out, gg->mass_, q, 0);
    delete gg;
  } else if (mode == "coarsen" && argc == 5) {
    std::vector<GraphElem> assign = read_i64(argv[3]);
    std::string out = argv[4];
    GraphGPU* gg = new GraphGPU(g, 1, 1, 1);
    gg->set_community_ids(assign.data());
    double q = gg->compute_modularity();
    bool done = gg->aggregation();
    std::vector<GraphElem> newid(gg->commIdsHost_, gg->commIdsHost_ + nv);
    write_arr(out + "/newid.i64", newid.data(), nv);
    if (!done) {
      GraphElem cnv = gg->NV_;
      write_arr(out + "/coff.i64", gg->indicesHost_, cnv + 1);
      write_arr(out + "/cadj.i64", gg->edgesHost_, gg->indicesHost_[cnv]);
      write_arr(out + "/cw.f64", gg->edgeWeightsHost_, gg->indicesHost_[cnv]);
    }
    write_scalars(out, gg->mass_, q, done ? 1 : 0);
    delete gg;
  } else if (mode == "run" && argc == 7) {
    int nb = atoi(argv[3]);
    double tau = atof(argv[4]);
    long long iters = atoll(argv[5]);
    std::cout << std::setprecision(17);
    GraphGPU* gg = new GraphGPU(g, nb, 1, 1);
    LouvainGPU* lv = new LouvainGPU(iters, tau, nb);
    lv->run(gg);
    gg->dump_partition(argv[6], nullptr);
    delete lv;
    delete gg;
  } else {
    fprintf(stderr, "bad arguments for mode %s\n", mode.c_str());
    return 2;
  }
  delete g;
  cudaDeviceReset();
  return 0;
}
