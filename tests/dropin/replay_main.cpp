// replay_main.cpp -- a program written the way a user of sg0/nido writes
// one: the reference's header names (include/nido_compat), its classes and
// signatures, and the call sequence of the reference's own main
// (main.cpp:84-163): Graph(file), optional coloring(), GraphGPU(graph,
// nbatches, 1, 1), LouvainGPU(maxLoops, tau, nbatches), run, dump_partition,
// deletes.  Built against libnido_b200.so only.
//
//   replay_main -f g.bin [-b nbatches] [-t tau] [-i maxLoops] [-c] [-o out] [-s]
//
// -s drives the phase loop by hand through GraphGPU's step methods, in the
// order of louvain_gpu.cpp:28-124 (singleton_partition, compute_modularity,
// per batch louvain_update / update_community_weights / update_community_ids
// with host_id 0, restore_community when Q fell, aggregation), instead of
// LouvainGPU::run; the partition must be the same.
#include <unistd.h>

#include <cstdlib>
#include <iostream>
#include <string>

#include "cuda_wrapper.hpp"
#include "graph.hpp"
#include "graph_gpu.hpp"
#include "louvain_gpu.hpp"
#include "types.hpp"

static void run_by_steps(GraphGPU* g, const Int& maxLoops, const Float& tau, const int& nbatches) {
  bool done = false;
  Int phases = 0;
  while (!done && phases < MAX_PHASES) {
    g->singleton_partition();
    Float Q = g->compute_modularity();
    const Float Q_old = Q;
    Float dQ = 1e300;
    Int loops = 0;
    while (tau < dQ && loops < maxLoops) {
      for (int batch = 0; batch < nbatches; ++batch) {
        g->louvain_update(batch, 0);
        g->update_community_weights(batch, 0);
        g->update_community_ids(batch, 0);
      }
      const Float Qtmp = g->compute_modularity();
      dQ = Qtmp - Q;
      ++loops;
      if (dQ < 0)
        g->restore_community();
      else
        Q = Qtmp;
    }
    std::cout << "PHASE #" << phases << " loops " << loops << " Final Q: " << Q << std::endl;
    done = Q - Q_old > tau ? g->aggregation() : true;
    ++phases;
  }
}

int main(int argc, char** argv) {
  std::string inputFileName, outFileName;
  bool is_colored = false, output_communities = false, by_steps = false;
  int nbatches = DEFAULT_BATCHES;
  Int maxLoops = DEFAULT_ITERATIONS;
  Float tau = DEFAULT_THRESHOLD;
  int ret;
  optind = 1;
  while ((ret = getopt(argc, argv, "f:b:i:t:co:s")) != -1) {
    switch (ret) {
      case 'f': inputFileName.assign(optarg); break;
      case 'b': nbatches = atoi(optarg); break;
      case 'i': maxLoops = (Int)atoll(optarg); break;
      case 't': tau = (Float)atof(optarg); break;
      case 'c': is_colored = true; break;
      case 'o': output_communities = true; outFileName.assign(optarg); break;
      case 's': by_steps = true; break;
      default: return EXIT_FAILURE;
    }
  }
  if (inputFileName.empty()) {
    std::cerr << "Input graph arguments missing. Use -f." << std::endl;
    return EXIT_FAILURE;
  }
  Graph* graph = new Graph(inputFileName);
  std::cout << "#Batches: " << nbatches << std::endl;
  std::cout << "#Threshold: " << tau << std::endl;
  std::cout << "Max #iterations: " << maxLoops << std::endl;
  std::cout << "#NGPUs: " << NGPU << std::endl;
  GraphElem* new_orders = nullptr;
  if (is_colored) new_orders = graph->coloring();
  GraphGPU* graph_gpu = new GraphGPU(graph, nbatches, 1, 1);
  LouvainGPU* louvain = new LouvainGPU(maxLoops, tau, nbatches);
  if (by_steps)
    run_by_steps(graph_gpu, maxLoops, tau, nbatches);
  else
    louvain->run(graph_gpu);
  if (output_communities) graph_gpu->dump_partition(outFileName, new_orders);
  if (is_colored) delete[] new_orders;
  delete louvain;
  delete graph_gpu;
  delete graph;
  for (int i = 0; i < NGPU; ++i) {
    CudaSetDevice(i);
    CudaCall(cudaDeviceReset());
  }
  return 0;
}
