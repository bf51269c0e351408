// cuts.cuh -- the -b batch cut rule of partition_graph_edge_batch
// (graph_gpu.cpp:303-339), shared by the one-graph and many-graph drivers.
#ifndef NIDO_CUTS_CUH_
#define NIDO_CUTS_CUH_
#include <stdint.h>

namespace nido {

// Cuts of the nv vertices behind off (nv+1 offsets, any base) into nb
// edge-balanced batches, written to cuts[0..nb] as vertex indices relative to
// off; parts needs nb+2 entries.  The reference walks vertices linearly until
// a batch holds more than the average edge count; each cut here is the same
// first index, found by a binary search.
__device__ inline void batch_cuts(const int64_t* __restrict__ off, int64_t nv, int nb,
                                  int64_t* __restrict__ cuts, int64_t* __restrict__ parts) {
  const int64_t ave = (off[nv] - off[0]) / nb;
  int np = 0;
  parts[np++] = 0;
  int64_t start = 0;
  while (np <= nb + 1) {
    // first i in (start, nv] with off[i] - off[start] > ave
    const int64_t target = off[start] + ave;
    int64_t lo = start + 1, hi = nv + 1;
    while (lo < hi) {
      const int64_t mid = lo + (hi - lo) / 2;
      if (off[mid] > target) hi = mid; else lo = mid + 1;
    }
    if (lo <= nv) {
      parts[np++] = lo;
      start = lo;
      if (lo == nv) break;
    } else {
      parts[np++] = nv;
      break;
    }
  }
  if (np > nb + 1) {
    const int64_t nnv = (nv - parts[nb]) / nb;
    for (int i = 1; i < nb; ++i) parts[i] += nnv;
    parts[nb] = nv;
  } else {
    while (np < nb + 1) parts[np++] = nv;
  }
  for (int i = 0; i <= nb; ++i) cuts[i] = parts[i];
}

}  // namespace nido
#endif
