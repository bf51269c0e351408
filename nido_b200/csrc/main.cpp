// main.cpp -- drop-in command line of the reference (main.cpp:15-177):
//   nido_louvain -f graph.bin [-b nbatches] [-t threshold] [-i maxIter] [-c] [-o out]
// Same options, defaults (types.hpp:24-38) and stdout lines.  -r (random BA
// graph) is not provided; -p accepts only the default "1 1".  --tie=nido
// selects the reference's tie rule for parity runs; --color-batches sweeps
// every phase's colour classes as conflict-free batches instead of the -b
// cuts.
#include <getopt.h>
#include <omp.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <sstream>
#include <string>
#include <vector>

#include "nido_b200.h"
#include "nido_host.hpp"

int main(int argc, char** argv) {
  std::string inputFileName, outFileName;
  bool is_colored = false, bin_graph = false, output_communities = false, help_text = false;
  int nbatches = 2;
  long long maxLoops = 500;
  double tau = 1.0E-06;
  int tie = NIDO_TIE_SMALLEST_ID;
  bool color_batches = false;
  int kept = 1;  // the long options are taken out before getopt sees the rest
  for (int i = 1; i < argc; ++i) {
    if (strcmp(argv[i], "--tie=nido") == 0) tie = NIDO_TIE_NIDO;
    else if (strcmp(argv[i], "--color-batches") == 0) color_batches = true;
    else argv[kept++] = argv[i];
  }
  argc = kept;
  int ret;
  optind = 1;
  while ((ret = getopt(argc, argv, "f:p:r:cb:i:t:ho:")) != -1) {
    switch (ret) {
      case 'f': bin_graph = true; inputFileName.assign(optarg); break;
      case 'p':
        if (std::string(optarg) != "1 1") {
          fprintf(stderr, "-p: only the default partitioning \"1 1\" is supported\n");
          return EXIT_FAILURE;
        }
        break;
      case 'r':
        fprintf(stderr, "-r (random graph) is not supported; generate a Vite binary and use -f\n");
        return EXIT_FAILURE;
      case 'o': output_communities = true; outFileName.assign(optarg); break;
      case 't': tau = atof(optarg); break;
      case 'i': maxLoops = atoll(optarg); break;
      case 'b': nbatches = atoi(optarg); break;
      case 'c': is_colored = true; break;
      case 'h':
        printf("Sample usage [1] (use real-world file): ./nido_louvain [-f /path/to/binary/file.bin] (see README)\n");
        help_text = true;
        break;
      default: printf("Reached default -- please check the passed options.\n"); break;
    }
  }
  if (help_text) return EXIT_SUCCESS;
  if (!bin_graph) {
    fprintf(stderr, "Input graph arguments missing. Use -f or -r options.\n");
    return -1;
  }
  if (nbatches < 1) {
    fprintf(stderr, "-b must be at least 1\n");
    return EXIT_FAILURE;
  }
  nido_ctx ctx = nullptr;
  nido_check(nido_ctx_create(0, 0, &ctx), "nido_ctx_create");
  GraphElem* new_orders = nullptr;
  if (is_colored) {  // the relabel needs the CSR on the host
    Graph graph(inputFileName);
    printf("#Batches: %d\n#Threshold: %g\nMax #iterations: %lld\n#NGPUs: 1\n", nbatches, tau, maxLoops);
    printf("--------------------------------------\n");
    const double t0 = omp_get_wtime();
    new_orders = graph.coloring(ctx);
    printf("Coloring Time: %g s\n", omp_get_wtime() - t0);
    GraphGPU graph_gpu(&graph, nbatches, ctx);
    graph_gpu.set_tie_rule(tie);
    graph_gpu.set_color_batches(color_batches);
    LouvainGPU louvain(maxLoops, tau, nbatches);
    louvain.run(&graph_gpu);
    if (output_communities) graph_gpu.dump_partition(outFileName, new_orders);
  } else {  // the file streams to the device
    GraphGPU graph_gpu(inputFileName, nbatches, ctx);
    graph_gpu.set_tie_rule(tie);
    graph_gpu.set_color_batches(color_batches);
    printf("#Batches: %d\n#Threshold: %g\nMax #iterations: %lld\n#NGPUs: 1\n", nbatches, tau, maxLoops);
    printf("--------------------------------------\n");
    LouvainGPU louvain(maxLoops, tau, nbatches);
    louvain.run(&graph_gpu);
    if (output_communities) graph_gpu.dump_partition(outFileName, new_orders);
  }
  delete[] new_orders;
  nido_ctx_destroy(ctx);
  fflush(stdout);
  return 0;
}
