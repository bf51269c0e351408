// oracle_main.cpp -- command-line driver for the CPU oracle (test
// infrastructure: used to time the CPU restatement as a baseline).
//   nido_oracle_run -f graph.bin [-b B] [-t tau] [-i maxIter] [-o out] [-n]
// -n selects nido's tie rule; default is smallest community id.
#include <omp.h>
#include <stdio.h>
#include <stdlib.h>
#include <unistd.h>

#include <vector>

#include "nido_oracle.h"

int main(int argc, char** argv) {
  const char* in = nullptr;
  const char* out = nullptr;
  int nb = 2, tie = ORC_TIE_SMALLEST_ID;
  double tau = 1.0E-06;
  long long iters = 500;
  int c;
  while ((c = getopt(argc, argv, "f:b:t:i:o:n")) != -1) {
    switch (c) {
      case 'f': in = optarg; break;
      case 'b': nb = atoi(optarg); break;
      case 't': tau = atof(optarg); break;
      case 'i': iters = atoll(optarg); break;
      case 'o': out = optarg; break;
      case 'n': tie = ORC_TIE_NIDO; break;
      default: break;
    }
  }
  if (!in) { fprintf(stderr, "usage: %s -f graph.bin [-b B] [-t tau] [-i it] [-o out] [-n]\n", argv[0]); return 2; }
  int64_t nv, ne, *off, *adj;
  double* w;
  if (orc_read_vite(in, &nv, &ne, &off, &adj, &w) != 0) { fprintf(stderr, "cannot read %s\n", in); return 1; }
  std::vector<int64_t> cl(nv);
  orc_stats st;
  double t0 = omp_get_wtime();
  orc_louvain(nv, off, adj, w, nb, tau, iters, tie, 1, cl.data(), &st);
  double t1 = omp_get_wtime();
  printf("Total time elapse: %.6f s\nTotal Loops: %lld\nthreads: %d\n", t1 - t0,
         (long long)st.total_loops, omp_get_max_threads());
  if (out) {
    FILE* f = fopen(out, "w");
    for (int64_t i = 0; i < nv; ++i) fprintf(f, "%lld\n", (long long)cl[i]);
    fclose(f);
  }
  orc_free(off); orc_free(adj); orc_free(w);
  return 0;
}
