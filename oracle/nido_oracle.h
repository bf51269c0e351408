/*
 * nido_oracle.h -- CPU restatement of sg0/nido's Louvain algorithm.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker for the CUDA engine
 * in nido_b200/: only tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline leg may load it.  The product never links or calls it.
 *
 * Every function restates one piece of the reference (file:line cited beside
 * it) with the same operation order wherever the reference fixes one, so that
 * results are bit-identical on integer-weighted graphs and, for k_v, m and Q
 * given identical inputs, on any weights.  The one order the reference leaves
 * to a library (Thrust reduce_by_key for e_uc, graph_gpu.cpp:499-500) is
 * restated as a left fold in CSR edge order.
 *
 * Pinning: the restatement is checked against outputs of the reference's own
 * code (fixtures under tests/golden/, produced by oracle/ref_harness.cu linked
 * against the unmodified reference objects) and against hand-derived cases.
 *
 * Ids are int64 and weights FP64, as in the reference (types.hpp:14-22).
 */
#ifndef NIDO_ORACLE_H_
#define NIDO_ORACLE_H_
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* tie rules for the best-move argmax */
#define ORC_TIE_SMALLEST_ID 0 /* smallest community id among equal gains */
#define ORC_TIE_NIDO 1        /* nido's 8-lane strided scan + shuffle tree (graph_cuda.cu:1493-1526) */

/* Vite binary reader (graph.cpp:322-495 with GRAPH_FT_LOAD defined). Arrays are
 * malloc'ed; release with orc_free.  Returns 0, or -1 when the file cannot be
 * opened or is truncated. */
int orc_read_vite(const char* path, int64_t* nv, int64_t* ne, int64_t** off,
                  int64_t** adj, double** w);
int orc_write_vite(const char* path, int64_t nv, const int64_t* off,
                   const int64_t* adj, const double* w);
void orc_free(void* p);

/* -b batch cut points, edge balanced (graph_gpu.cpp:280-359, NGPU=1,
 * part_on_batch=1).  cuts has nbatches+1 entries. */
void orc_batch_cuts(int64_t nv, const int64_t* off, int nbatches, int64_t* cuts);

/* k_v = sum of incident weights, self-loops included, 32-lane strided order
 * (graph_cuda.cu:302-346). */
void orc_vertex_weights(int64_t nv, const int64_t* off, const double* w, double* k);
/* m = 0.5 * sum k_v in the reference's 4096x32 + 1x1024 order
 * (graph_cuda.cu:1786-1856). */
double orc_mass(int64_t nv, const double* k);
/* comm[v]=v, newcomm[v]=v, a[v]=k[v] (graph_cuda.cu:410-429) */
void orc_singleton(int64_t nv, const double* k, int64_t* comm, int64_t* newcomm, double* a);
/* a[c] = sum of k_v over comm[v]==c (graph_cuda.cu:370-390); a must be zeroed */
void orc_community_weights(int64_t nv, const int64_t* comm, const double* k, double* a);

/* Best move for every v in [v0,v1): newcomm[v] (graph_gpu.cpp:457-517,
 * graph_cuda.cu:49-98, 2289-2318, 1450-1540). */
void orc_move(int64_t nv, const int64_t* off, const int64_t* adj, const double* w,
              const int64_t* comm, const double* a, const double* k, double m,
              int64_t v0, int64_t v1, int tie, int64_t* newcomm);
/* Same, also reporting the winning gain-minus-self value per vertex (NaN when
 * the vertex had no candidate community). */
void orc_move_gain(int64_t nv, const int64_t* off, const int64_t* adj, const double* w,
                   const int64_t* comm, const double* a, const double* k, double m,
                   int64_t v0, int64_t v1, int tie, int64_t* newcomm, double* gain);
/* FP64 community-degree update then id swap over [v0,v1)
 * (graph_cuda.cu:1222-1251, 1182-1197). */
void orc_commit(int64_t v0, int64_t v1, int64_t* comm, int64_t* newcomm,
                const double* k, double* a);
/* Undo one iteration (graph_gpu.cpp:822-842). */
void orc_restore(int64_t nv, int64_t* comm, int64_t* newcomm, const double* k, double* a);

/* Q in the reference's reduction order (graph_cuda.cu:2078-2134, 1806-1835,
 * graph_gpu.cpp:862-905). */
double orc_modularity(int64_t nv, const int64_t* off, const int64_t* adj, const double* w,
                      const int64_t* comm, const double* a, double m);

/* Coarsening (graph_gpu.cpp:1151-1304, 1382-1400).  newid[v] = dense id of
 * v's community (ascending old id order).  Returns the coarse vertex count and
 * allocates the coarse CSR (release with orc_free). */
int64_t orc_coarsen(int64_t nv, const int64_t* off, const int64_t* adj, const double* w,
                    const int64_t* comm, int64_t* newid, int64_t** coff, int64_t** cadj,
                    double** cw, int64_t* cne);

/* Colour-class relabel of the CSR (graph.cpp:611-693): new vertex p is old
 * vertex new_orders[p], vertices ordered by (colour, old id).  Output arrays
 * are caller-allocated with the input sizes. */
void orc_color_relabel(int64_t nv, const int64_t* off, const int64_t* adj, const double* w,
                       const int64_t* colors, int64_t* new_orders, int64_t* noff,
                       int64_t* nadj, double* nw);
/* nido's greedy colouring run on one thread (graph.cpp:548-606): priorities
 * from std::mt19937_64(1) and uniform_int_distribution(0, 4*nv). */
void orc_color_nido_seq(int64_t nv, const int64_t* off, const int64_t* adj, int64_t* colors);

/* Whole Louvain run (louvain_gpu.cpp:28-124).  clustering has nv entries and
 * receives the community of every input vertex, as written by -o
 * (clustering.cpp:12-21).  q_phase / loops_phase receive up to 200 entries. */
typedef struct {
  int64_t phases;
  int64_t total_loops;
  double final_q;              /* Q printed as "Final Q" by the last phase */
  double q_phase[200];
  int64_t loops_phase[200];
  int64_t nv_phase[200];
  int64_t ne_phase[200];
} orc_stats;
int orc_louvain(int64_t nv, const int64_t* off, const int64_t* adj, const double* w,
                int nbatches, double tau, int64_t max_loops, int tie, int verbose,
                int64_t* clustering, orc_stats* st);
/* the same, stopping after max_phases phases (bounded timing samples) */
int orc_louvain_capped(int64_t nv, const int64_t* off, const int64_t* adj, const double* w,
                       int nbatches, double tau, int64_t max_loops, int tie, int verbose,
                       int max_phases, int64_t* clustering, orc_stats* st);

/* Plain FP64 modularity of a partition of the original graph (any community
 * ids), summed per vertex in CSR order: used to compare final partitions. */
double orc_partition_modularity(int64_t nv, const int64_t* off, const int64_t* adj,
                                const double* w, const int64_t* part);

/* Normalised mutual information of two labelings (arithmetic-mean normaliser). */
double orc_nmi(int64_t n, const int64_t* a, const int64_t* b);

/* Jones-Plassmann-Luby colouring as the engine runs it (hashed priorities,
 * rounds that see only earlier rounds' colours); returns the colour count. */
int64_t orc_color_jpl(int64_t nv, const int64_t* off, const int64_t* adj, uint64_t seed, int64_t* colors);
/* orc_louvain_capped plus color_batches: every phase's JPL colour classes
 * (seed 1) are its batches, in colour order, instead of the -b cuts. */
int orc_louvain_ex(int64_t nv0, const int64_t* off0, const int64_t* adj0, const double* w0, int nbatches,
                   double tau, int64_t max_loops, int tie, int verbose, int max_phases, int color_batches,
                   int64_t* clustering, orc_stats* st);

#ifdef __cplusplus
}
#endif
#endif
