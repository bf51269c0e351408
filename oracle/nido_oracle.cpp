// nido_oracle.cpp -- CPU restatement of sg0/nido's Louvain path.
//
// TEST INFRASTRUCTURE ONLY (the checker, never the product): loaded by tests/,
// __graft_entry__.smoke() and bench.py's CPU-baseline leg.  See nido_oracle.h
// for the contract.  Compiled with -ffp-contract=off; the one place where the
// reference's CUDA build fuses a multiply-add (ac += w*w at
// graph_cuda.cu:2119, contracted by nvcc's default -fmad=true) is written as
// an explicit fma().
#include "nido_oracle.h"

#include <math.h>
#include <omp.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <random>
#include <set>
#include <unordered_map>
#include <vector>

static const double kMaxFloat = 1.0E+308;  // cuda_wrapper.hpp:94 (MAX_FLOAT)

extern "C" void orc_free(void* p) { free(p); }

// ---------------------------------------------------------------------------
// Vite binary reader.  graph.cpp:322-495.  With GRAPH_FT_LOAD defined (the
// reference Makefile always defines it) the edge records are read starting
// right after the offsets, for indices[nv]-indices[0] records (graph.cpp:
// 397-435); offsets are then rebased to start at 0 (graph.cpp:470-472).
extern "C" int orc_read_vite(const char* path, int64_t* nv_out, int64_t* ne_out,
                             int64_t** off_out, int64_t** adj_out, double** w_out) {
  FILE* f = fopen(path, "rb");
  if (!f) return -1;
  int64_t hdr[2];
  if (fread(hdr, sizeof(int64_t), 2, f) != 2) { fclose(f); return -1; }
  int64_t nv = hdr[0];
  if (nv < 0) { fclose(f); return -1; }
  int64_t* off = (int64_t*)malloc(sizeof(int64_t) * (nv + 1));
  if ((int64_t)fread(off, sizeof(int64_t), nv + 1, f) != nv + 1) { free(off); fclose(f); return -1; }
  int64_t ne = off[nv] - off[0];
  if (ne < 0) { free(off); fclose(f); return -1; }
  struct Rec { int64_t tail; double w; };
  Rec* recs = (Rec*)malloc(sizeof(Rec) * (ne > 0 ? ne : 1));
  if ((int64_t)fread(recs, sizeof(Rec), ne, f) != ne) { free(off); free(recs); fclose(f); return -1; }
  fclose(f);
  int64_t* adj = (int64_t*)malloc(sizeof(int64_t) * (ne > 0 ? ne : 1));
  double* w = (double*)malloc(sizeof(double) * (ne > 0 ? ne : 1));
  for (int64_t i = 0; i < ne; ++i) { adj[i] = recs[i].tail; w[i] = recs[i].w; }
  free(recs);
  int64_t base = off[0];
  for (int64_t i = 0; i <= nv; ++i) off[i] -= base;
  *nv_out = nv; *ne_out = ne; *off_out = off; *adj_out = adj; *w_out = w;
  return 0;
}

extern "C" int orc_write_vite(const char* path, int64_t nv, const int64_t* off,
                              const int64_t* adj, const double* w) {
  FILE* f = fopen(path, "wb");
  if (!f) return -1;
  int64_t hdr[2] = {nv, off[nv] - off[0]};
  fwrite(hdr, sizeof(int64_t), 2, f);
  fwrite(off, sizeof(int64_t), nv + 1, f);
  for (int64_t e = off[0]; e < off[nv]; ++e) {
    fwrite(&adj[e], sizeof(int64_t), 1, f);
    fwrite(&w[e], sizeof(double), 1, f);
  }
  fclose(f);
  return 0;
}

// ---------------------------------------------------------------------------
// Batch cuts.  graph_gpu.cpp:303-339 (part_on_batch = 1, one device so
// V0 = 0, nv = NV, ne = NE).
extern "C" void orc_batch_cuts(int64_t nv, const int64_t* off, int nbatches, int64_t* cuts) {
  int64_t ne = off[nv] - off[0];
  int64_t ave_ne = ne / nbatches;
  std::vector<int64_t> parts;
  parts.push_back(0);
  int64_t start = 0;
  for (int64_t i = 1; i <= nv; ++i) {
    if (off[i] - off[start] > ave_ne) {
      parts.push_back(i);
      start = i;
    } else if (i == nv) {
      parts.push_back(nv);
    }
  }
  if ((int64_t)parts.size() > nbatches + 1) {
    int64_t remain = nv - parts[nbatches];
    int64_t nnv = remain / nbatches;
    for (int i = 1; i < nbatches; ++i) parts[i] += nnv;
    parts[nbatches] = nv;
  } else {
    while ((int64_t)parts.size() < nbatches + 1) parts.push_back(nv);
  }
  for (int i = 0; i <= nbatches; ++i) cuts[i] = parts[i];
}

// ---------------------------------------------------------------------------
// Reductions that restate a warp shuffle-down tree: lane 0 ends with the
// pairwise tree x[i] += x[i+off], off = n/2 .. 1 (graph_cuda.cu:339-340).
static double tree_sum(double* x, int n) {
  for (int o = n / 2; o > 0; o /= 2)
    for (int i = 0; i < o; ++i) x[i] = x[i] + x[i + o];
  return x[0];
}

// k_v: graph_cuda.cu:302-346, one 32-lane tile per vertex, lane l sums edges
// start+l, start+l+32, ... then the shuffle tree.
extern "C" void orc_vertex_weights(int64_t nv, const int64_t* off, const double* w, double* k) {
#pragma omp parallel for schedule(dynamic, 1024)
  for (int64_t v = 0; v < nv; ++v) {
    double lane[32];
    for (int l = 0; l < 32; ++l) {
      double s = 0.;
      for (int64_t e = off[v] + l; e < off[v + 1]; e += 32) s += w[e];
      lane[l] = s;
    }
    k[v] = tree_sum(lane, 32);
  }
}

// reduce_vector_kernel<32><<<1,1024>>> (graph_cuda.cu:1806-1835): thread t
// folds x[t], x[t+1024], ...; warp trees; then warp 0's tree over 32 partials.
static double reduce_vector_1024(const double* x, int64_t n) {
  double thr[1024];
  for (int t = 0; t < 1024; ++t) {
    double s = 0.;
    for (int64_t i = t; i < n; i += 1024) s += x[i];
    thr[t] = s;
  }
  double warp[32];
  for (int wv = 0; wv < 32; ++wv) warp[wv] = tree_sum(thr + 32 * wv, 32);
  return tree_sum(warp, 32);
}

// m: compute_mass_reduce_kernel<32><<<4096,32>>> + reduce_vector_kernel,
// then 0.5 * m (graph_cuda.cu:1786-1804, 1837-1856).
extern "C" double orc_mass(int64_t nv, const double* k) {
  std::vector<double> blk(4096);
  for (int b = 0; b < 4096; ++b) {
    double lane[32];
    for (int l = 0; l < 32; ++l) {
      double s = 0.;
      for (int64_t i = l + 32 * (int64_t)b; i < nv; i += 32 * 4096) s += k[i];
      lane[l] = s;
    }
    blk[b] = tree_sum(lane, 32);
  }
  return 0.5 * reduce_vector_1024(blk.data(), 4096);
}

extern "C" void orc_singleton(int64_t nv, const double* k, int64_t* comm, int64_t* newcomm, double* a) {
  for (int64_t v = 0; v < nv; ++v) { comm[v] = v; newcomm[v] = v; a[v] = k[v]; }
}

extern "C" void orc_community_weights(int64_t nv, const int64_t* comm, const double* k, double* a) {
  for (int64_t v = 0; v < nv; ++v) a[comm[v]] += k[v];
}

// ---------------------------------------------------------------------------
// Move step.  Per vertex v the reference builds the unique (v, c) keys with
// e_vc = sum of edge weights to community c, self-loops contributing weight 0
// but still producing the key (v, comm[v]) (graph_cuda.cu:2306-2316,
// graph_gpu.cpp:484-515).  louvain_update_kernel (graph_cuda.cu:1481-1537):
//   gain_c = (e_vc - ki*a_c/(2m)) / m        for c != own
//   self   = (e_own - ki*(a_own-ki)/(2m)) / m
//   newcomm = best if gain_best - self > 0 else own.
namespace {
struct MoveScratch {
  std::vector<double> acc;
  std::vector<int64_t> touched;
  std::vector<char> seen;
};

inline void move_one(int64_t v, const int64_t* off, const int64_t* adj, const double* w,
                     const int64_t* comm, const double* a, const double* k, double m, int tie,
                     MoveScratch& s, int64_t* newcomm, double* gain_out) {
  const int64_t own = comm[v];
  const double ki = k[v];
  s.touched.clear();
  for (int64_t j = off[v]; j < off[v + 1]; ++j) {
    const int64_t u = adj[j];
    const int64_t c = comm[u];
    const double wt = (u == v) ? 0. : w[j];
    if (!s.seen[c]) { s.seen[c] = 1; s.acc[c] = 0.; s.touched.push_back(c); }
    s.acc[c] += wt;
  }
  double self_e = s.seen[own] ? s.acc[own] : 0.;
  int64_t dest = own;
  double best = -kMaxFloat;
  if (tie == ORC_TIE_SMALLEST_ID) {
    // larger gain wins; equal gains go to the smaller community id
    int64_t bestc = INT64_MAX;
    for (int64_t c : s.touched) {
      if (c == own) continue;
      double g = s.acc[c];
      g -= ki * a[c] / (2. * m);
      g /= m;
      if (g > best || (g == best && c < bestc)) { best = g; bestc = c; }
    }
    if (bestc != INT64_MAX) dest = bestc;
  } else {
    // nido: unique keys sorted by community id; 8 lanes take entries
    // i = lane, lane+8, ... keeping the first strict maximum, then a
    // shuffle-down tree (offsets 4, 2, 1) keeps the lower lane on ties.
    std::sort(s.touched.begin(), s.touched.end());
    double lg[8];
    int64_t ld[8];
    for (int l = 0; l < 8; ++l) { lg[l] = -kMaxFloat; ld[l] = own; }
    for (size_t i = 0; i < s.touched.size(); ++i) {
      const int64_t c = s.touched[i];
      if (c == own) continue;
      double g = s.acc[c];
      g -= ki * a[c] / (2. * m);
      g /= m;
      const int l = (int)(i & 7);
      if (g > lg[l]) { lg[l] = g; ld[l] = c; }
    }
    for (int o = 4; o > 0; o /= 2) {
      double ng[8];
      int64_t nd[8];
      for (int l = 0; l < 8; ++l) { ng[l] = lg[l]; nd[l] = ld[l]; }
      for (int l = 0; l + o < 8; ++l)
        if (lg[l + o] > lg[l]) { ng[l] = lg[l + o]; nd[l] = ld[l + o]; }
      for (int l = 0; l < 8; ++l) { lg[l] = ng[l]; ld[l] = nd[l]; }
    }
    best = lg[0];
    dest = ld[0];
  }
  double self = self_e;
  self -= ki * (a[own] - ki) / (2. * m);
  self /= m;
  double g = best - self;
  newcomm[v] = (g > 0) ? dest : own;
  if (gain_out) gain_out[v] = (best == -kMaxFloat) ? NAN : g;
  for (int64_t c : s.touched) s.seen[c] = 0;
}
}  // namespace

extern "C" void orc_move_gain(int64_t nv, const int64_t* off, const int64_t* adj, const double* w,
                              const int64_t* comm, const double* a, const double* k, double m,
                              int64_t v0, int64_t v1, int tie, int64_t* newcomm, double* gain) {
#pragma omp parallel
  {
    MoveScratch s;
    s.acc.assign(nv, 0.);
    s.seen.assign(nv, 0);
#pragma omp for schedule(dynamic, 256)
    for (int64_t v = v0; v < v1; ++v) move_one(v, off, adj, w, comm, a, k, m, tie, s, newcomm, gain);
  }
}

// The move step over the vertices of a list (a colour class).
static void move_list(int64_t nv, const int64_t* off, const int64_t* adj, const double* w, const int64_t* comm,
                      const double* a, const double* k, double m, const std::vector<int64_t>& list, int tie,
                      int64_t* newcomm) {
#pragma omp parallel
  {
    MoveScratch s;
    s.acc.assign(nv, 0.);
    s.seen.assign(nv, 0);
#pragma omp for schedule(dynamic, 256)
    for (int64_t i = 0; i < (int64_t)list.size(); ++i)
      move_one(list[i], off, adj, w, comm, a, k, m, tie, s, newcomm, nullptr);
  }
}

static void commit_list(const std::vector<int64_t>& list, int64_t* comm, int64_t* newcomm, const double* k,
                        double* a) {
  for (int64_t v : list) {
    const int64_t src = comm[v], dst = newcomm[v];
    if (src != dst) { a[src] += -k[v]; a[dst] += k[v]; }
  }
  for (int64_t v : list) { int64_t t = comm[v]; comm[v] = newcomm[v]; newcomm[v] = t; }
}

// Jones-Plassmann-Luby colouring as the engine runs it (color.cu): in rounds,
// every uncoloured vertex whose (hashed priority, id) beats all its uncoloured
// neighbours takes the smallest colour no coloured neighbour has; a round
// sees only the colours of earlier rounds.  Deterministic for a seed.
static inline uint64_t jpl_prio(uint64_t seed, int64_t v) {
  uint64_t z = seed + 0x9E3779B97F4A7C15ull * (uint64_t)(v + 1);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

extern "C" int64_t orc_color_jpl(int64_t nv, const int64_t* off, const int64_t* adj, uint64_t seed,
                                 int64_t* colors) {
  std::vector<int64_t> cin(nv, -1), cout(nv, -1);
  int64_t left = nv;
  while (left > 0) {
#pragma omp parallel for schedule(dynamic, 1024)
    for (int64_t v = 0; v < nv; ++v) {
      if (cin[v] >= 0) continue;
      const uint64_t pv = jpl_prio(seed, v);
      bool beaten = false;
      for (int64_t j = off[v]; j < off[v + 1] && !beaten; ++j) {
        const int64_t u = adj[j];
        if (u == v || cin[u] >= 0) continue;
        const uint64_t pu = jpl_prio(seed, u);
        if (pu > pv || (pu == pv && u > v)) beaten = true;
      }
      if (beaten) continue;
      std::vector<char> used;
      for (int64_t j = off[v]; j < off[v + 1]; ++j) {
        const int64_t c = cin[adj[j]];
        if (c < 0) continue;
        if ((int64_t)used.size() <= c) used.resize(c + 1, 0);
        used[c] = 1;
      }
      int64_t c = 0;
      while (c < (int64_t)used.size() && used[c]) ++c;
      cout[v] = c;
    }
    left = 0;
    for (int64_t v = 0; v < nv; ++v) {
      cin[v] = cout[v];
      left += cin[v] < 0;
    }
  }
  int64_t nc = 0;
  for (int64_t v = 0; v < nv; ++v) {
    colors[v] = cin[v];
    nc = std::max(nc, cin[v] + 1);
  }
  return nc;
}

extern "C" void orc_move(int64_t nv, const int64_t* off, const int64_t* adj, const double* w,
                         const int64_t* comm, const double* a, const double* k, double m,
                         int64_t v0, int64_t v1, int tie, int64_t* newcomm) {
  orc_move_gain(nv, off, adj, w, comm, a, k, m, v0, v1, tie, newcomm, nullptr);
}

// update_community_weights_kernel + exchange_vector_kernel
// (graph_cuda.cu:1234-1250, 1191-1196).
extern "C" void orc_commit(int64_t v0, int64_t v1, int64_t* comm, int64_t* newcomm,
                           const double* k, double* a) {
  for (int64_t v = v0; v < v1; ++v) {
    const int64_t src = comm[v], dst = newcomm[v];
    if (src != dst) { a[src] += -k[v]; a[dst] += k[v]; }
  }
  for (int64_t v = v0; v < v1; ++v) { int64_t t = comm[v]; comm[v] = newcomm[v]; newcomm[v] = t; }
}

extern "C" void orc_restore(int64_t nv, int64_t* comm, int64_t* newcomm, const double* k, double* a) {
  orc_commit(0, nv, comm, newcomm, k, a);
}

// ---------------------------------------------------------------------------
// Modularity.  compute_modularity_reduce_kernel<128,16> (graph_cuda.cu:
// 2096-2134) with grid min(ceil(nv/8), 65535) (2184-2186): thread slot t folds
// the in-community weights of vertices t, t+S, ... (S = 128*grid) in edge
// order and ac = fma(a_v, a_v, ac); 16-lane shuffle trees; lane 0 writes
// self/(2m) - ac/(4m*m) to mod[t/16] (mod zeroed, 524280 entries,
// graph_gpu.cpp:872-875); reduce_vector_kernel sums mod (graph_cuda.cu:2249).
extern "C" double orc_modularity(int64_t nv, const int64_t* off, const int64_t* adj,
                                 const double* w, const int64_t* comm, const double* a, double m) {
  if (nv <= 0) return 0.;
  int64_t grid = (nv + 7) / 8;
  if (grid > 65535) grid = 65535;
  const int64_t S = 128 * grid;
  const int64_t nslots = std::min<int64_t>(S, nv);
  const int64_t ngroups = (nslots + 15) / 16;
  std::vector<double> mod(524280, 0.);
#pragma omp parallel for schedule(dynamic, 64)
  for (int64_t g = 0; g < ngroups; ++g) {
    double sw[16], ac[16];
    for (int l = 0; l < 16; ++l) {
      const int64_t t = 16 * g + l;
      double s = 0., q = 0.;
      for (int64_t v = t; v < nv; v += S) {
        const int64_t own = comm[v];
        for (int64_t j = off[v]; j < off[v + 1]; ++j)
          if (comm[adj[j]] == own) s += w[j];
        q = fma(a[v], a[v], q);
      }
      sw[l] = s;
      ac[l] = q;
    }
    double self = tree_sum(sw, 16);
    double acs = tree_sum(ac, 16);
    self /= (2. * m);
    self -= acs / (4. * m * m);
    mod[g] += self;
  }
  return reduce_vector_1024(mod.data(), 524280);
}

// ---------------------------------------------------------------------------
// Coarsening.  sort_vertex_by_community_ids (graph_gpu.cpp:1151-1222): new id
// = rank of the old community id among used ids, members listed in ascending
// vertex order; shuffle_edge_list (1088-1149) concatenates the members'
// adjacency; compress_edges (1224-1304) maps neighbours to new ids and merges
// duplicates keeping first-occurrence order, summing weights in edge order.
extern "C" int64_t orc_coarsen(int64_t nv, const int64_t* off, const int64_t* adj,
                               const double* w, const int64_t* comm, int64_t* newid,
                               int64_t** coff_out, int64_t** cadj_out, double** cw_out,
                               int64_t* cne_out) {
  std::vector<int64_t> order(nv);
  for (int64_t i = 0; i < nv; ++i) order[i] = i;
  std::stable_sort(order.begin(), order.end(),
                   [&](int64_t x, int64_t y) { return comm[x] < comm[y]; });
  std::vector<int64_t> group_end;
  int64_t target = nv > 0 ? comm[order[0]] : 0;
  for (int64_t i = 0; i < nv; ++i) {
    if (comm[order[i]] != target) { group_end.push_back(i); target = comm[order[i]]; }
  }
  group_end.push_back(nv);
  const int64_t cnv = (int64_t)group_end.size();
  for (int64_t g = 0, j = 0; g < cnv; ++g)
    for (; j < group_end[g]; ++j) newid[order[j]] = g;

  int64_t* coff = (int64_t*)malloc(sizeof(int64_t) * (cnv + 1));
  std::vector<int64_t> tadj;
  std::vector<double> tw;
  tadj.reserve(off[nv]);
  tw.reserve(off[nv]);
  coff[0] = 0;
  for (int64_t g = 0, j = 0; g < cnv; ++g) {
    std::unordered_map<int64_t, int64_t> pos;
    const int64_t base = (int64_t)tadj.size();
    for (; j < group_end[g]; ++j) {
      const int64_t v = order[j];
      for (int64_t e = off[v]; e < off[v + 1]; ++e) {
        const int64_t x = newid[adj[e]];
        auto it = pos.find(x);
        if (it != pos.end()) {
          tw[base + it->second] += w[e];
        } else {
          pos.emplace(x, (int64_t)tadj.size() - base);
          tadj.push_back(x);
          tw.push_back(w[e]);
        }
      }
    }
    coff[g + 1] = (int64_t)tadj.size();
  }
  const int64_t cne = (int64_t)tadj.size();
  int64_t* cadj = (int64_t*)malloc(sizeof(int64_t) * (cne > 0 ? cne : 1));
  double* cw = (double*)malloc(sizeof(double) * (cne > 0 ? cne : 1));
  if (cne) {
    memcpy(cadj, tadj.data(), sizeof(int64_t) * cne);
    memcpy(cw, tw.data(), sizeof(double) * cne);
  }
  *coff_out = coff; *cadj_out = cadj; *cw_out = cw; *cne_out = cne;
  return cnv;
}

// ---------------------------------------------------------------------------
// Colour relabel (graph.cpp:611-693).
extern "C" void orc_color_relabel(int64_t nv, const int64_t* off, const int64_t* adj,
                                  const double* w, const int64_t* colors, int64_t* new_orders,
                                  int64_t* noff, int64_t* nadj, double* nw) {
  std::vector<int64_t> idx(nv);
  for (int64_t i = 0; i < nv; ++i) idx[i] = i;
  std::sort(idx.begin(), idx.end(), [&](int64_t x, int64_t y) {
    return colors[x] != colors[y] ? colors[x] < colors[y] : x < y;
  });
  std::vector<int64_t> orders(nv);
  for (int64_t i = 0; i < nv; ++i) { new_orders[i] = idx[i]; orders[idx[i]] = i; }
  noff[0] = 0;
  for (int64_t i = 0; i < nv; ++i) noff[i + 1] = noff[i] + (off[idx[i] + 1] - off[idx[i]]);
  for (int64_t p = 0; p < nv; ++p) {
    const int64_t v = idx[p];
    for (int64_t j = 0; j < off[v + 1] - off[v]; ++j) {
      nadj[noff[p] + j] = orders[adj[off[v] + j]];
      nw[noff[p] + j] = w[off[v] + j];
    }
  }
}

// nido's colouring loop on one thread (graph.cpp:548-606).
extern "C" void orc_color_nido_seq(int64_t nv, const int64_t* off, const int64_t* adj,
                                   int64_t* colors) {
  std::vector<int64_t> prio(nv);
  std::mt19937_64 eng(1 << 0);
  std::uniform_int_distribution<int64_t> dist(0., nv * 4LL);
  for (int64_t i = 0; i < nv; ++i) prio[i] = dist(eng);
  for (int64_t i = 0; i < nv; ++i) colors[i] = -1;
  int64_t remain = nv;
  while (remain != 0) {
    int64_t num = 0;
    for (int64_t i = 0; i < nv; ++i) {
      if (colors[i] != -1) continue;
      const int64_t ir = prio[i];
      std::set<int64_t> cs;
      for (int64_t e = off[i]; e < off[i + 1]; ++e) {
        const int64_t j = adj[e];
        if (ir <= prio[j] && colors[j] != -1) cs.insert(colors[j]);
      }
      for (int64_t c = 0; c < nv; ++c)
        if (!cs.count(c)) { colors[i] = c; break; }
      ++num;
    }
    remain -= num;
  }
}

// ---------------------------------------------------------------------------
// Whole run: LouvainGPU::run (louvain_gpu.cpp:28-124) over GraphGPU's state,
// with aggregation (graph_gpu.cpp:1382-1545) and Clustering (clustering.cpp).
// max_phases below 200 stops early (used to time bounded samples).
extern "C" int orc_louvain_capped(int64_t nv0, const int64_t* off0, const int64_t* adj0,
                                  const double* w0, int nbatches, double tau, int64_t max_loops,
                                  int tie, int verbose, int max_phases, int64_t* clustering,
                                  orc_stats* st);

extern "C" int orc_louvain(int64_t nv0, const int64_t* off0, const int64_t* adj0,
                           const double* w0, int nbatches, double tau, int64_t max_loops,
                           int tie, int verbose, int64_t* clustering, orc_stats* st) {
  return orc_louvain_capped(nv0, off0, adj0, w0, nbatches, tau, max_loops, tie, verbose, 200,
                            clustering, st);
}

extern "C" int orc_louvain_ex(int64_t nv0, const int64_t* off0, const int64_t* adj0, const double* w0,
                              int nbatches, double tau, int64_t max_loops, int tie, int verbose, int max_phases,
                              int color_batches, int64_t* clustering, orc_stats* st);

extern "C" int orc_louvain_capped(int64_t nv0, const int64_t* off0, const int64_t* adj0,
                                  const double* w0, int nbatches, double tau, int64_t max_loops,
                                  int tie, int verbose, int max_phases, int64_t* clustering,
                                  orc_stats* st) {
  return orc_louvain_ex(nv0, off0, adj0, w0, nbatches, tau, max_loops, tie, verbose, max_phases, 0, clustering,
                        st);
}

// With color_batches, every phase colours its graph (orc_color_jpl, seed 1)
// and its colour classes, in colour order and ascending id within a class,
// are the batches instead of the -b cuts.
extern "C" int orc_louvain_ex(int64_t nv0, const int64_t* off0, const int64_t* adj0, const double* w0,
                              int nbatches, double tau, int64_t max_loops, int tie, int verbose, int max_phases,
                              int color_batches, int64_t* clustering, orc_stats* st) {
  if (nbatches < 1) return -1;
  memset(st, 0, sizeof(*st));
  std::vector<int64_t> off(off0, off0 + nv0 + 1), adj(adj0, adj0 + off0[nv0]);
  std::vector<double> w(w0, w0 + off0[nv0]);
  int64_t nv = nv0;
  for (int64_t i = 0; i < nv0; ++i) clustering[i] = i;
  std::vector<double> k(nv), a(nv);
  std::vector<int64_t> comm(nv), newcomm(nv), cuts(nbatches + 1);
  orc_vertex_weights(nv, off.data(), w.data(), k.data());
  double m = orc_mass(nv, k.data());
  orc_batch_cuts(nv, off.data(), nbatches, cuts.data());
  bool done = false;
  int64_t phases = 0;
  while (!done && phases < 200 && phases < max_phases) {
    if (verbose) printf("PHASE #%lld: \n", (long long)phases);
    orc_singleton(nv, k.data(), comm.data(), newcomm.data(), a.data());
    std::vector<std::vector<int64_t>> classes;
    if (color_batches) {
      std::vector<int64_t> col(nv);
      const int64_t nc = orc_color_jpl(nv, off.data(), adj.data(), 1, col.data());
      classes.assign((size_t)std::max<int64_t>(nc, 1), {});
      for (int64_t v = 0; v < nv; ++v) classes[col[v]].push_back(v);
    }
    double Q = orc_modularity(nv, off.data(), adj.data(), w.data(), comm.data(), a.data(), m);
    const double Q_old = Q;
    double dQ = kMaxFloat;
    int64_t loops = 0;
    while (tau < dQ && loops < max_loops) {
      if (color_batches) {
        for (const std::vector<int64_t>& cls : classes) {
          move_list(nv, off.data(), adj.data(), w.data(), comm.data(), a.data(), k.data(), m, cls, tie,
                    newcomm.data());
          commit_list(cls, comm.data(), newcomm.data(), k.data(), a.data());
        }
      } else {
      for (int b = 0; b < nbatches; ++b) {
        orc_move(nv, off.data(), adj.data(), w.data(), comm.data(), a.data(), k.data(), m,
                 cuts[b], cuts[b + 1], tie, newcomm.data());
        orc_commit(cuts[b], cuts[b + 1], comm.data(), newcomm.data(), k.data(), a.data());
      }
      }
      const double Qtmp = orc_modularity(nv, off.data(), adj.data(), w.data(), comm.data(), a.data(), m);
      dQ = Qtmp - Q;
      ++loops;
      if (dQ < 0) orc_restore(nv, comm.data(), newcomm.data(), k.data(), a.data());
      else Q = Qtmp;
      if (verbose) printf("%lld \t%.17g \t%.17g\n", (long long)loops, Qtmp, dQ);
    }
    st->q_phase[phases] = Q;
    st->loops_phase[phases] = loops;
    st->nv_phase[phases] = nv;
    st->ne_phase[phases] = off[nv];
    st->total_loops += loops;
    st->final_q = Q;
    if (verbose) printf("Final Q: %.17g\n", Q);
    if (Q - Q_old > tau && phases + 1 < max_phases) {
      std::vector<int64_t> newid(nv);
      int64_t *coff, *cadj, cne;
      double* cw;
      const int64_t cnv = orc_coarsen(nv, off.data(), adj.data(), w.data(), comm.data(),
                                      newid.data(), &coff, &cadj, &cw, &cne);
      for (int64_t i = 0; i < nv0; ++i) clustering[i] = newid[clustering[i]];
      if (cnv == nv || cnv == 1) {
        done = true;
      } else {
        nv = cnv;
        off.assign(coff, coff + cnv + 1);
        adj.assign(cadj, cadj + cne);
        w.assign(cw, cw + cne);
        k.assign(nv, 0.); a.assign(nv, 0.);
        comm.assign(nv, 0); newcomm.assign(nv, 0);
        orc_vertex_weights(nv, off.data(), w.data(), k.data());
        m = orc_mass(nv, k.data());
        orc_batch_cuts(nv, off.data(), nbatches, cuts.data());
      }
      free(coff); free(cadj); free(cw);
    } else {
      done = true;
    }
    ++phases;
  }
  st->phases = phases;
  return 0;
}

extern "C" double orc_partition_modularity(int64_t nv, const int64_t* off, const int64_t* adj,
                                           const double* w, const int64_t* part) {
  int64_t maxc = 0;
  for (int64_t v = 0; v < nv; ++v) maxc = std::max(maxc, part[v]);
  std::vector<double> k(nv, 0.), a(maxc + 1, 0.);
  double twom = 0., in = 0.;
  for (int64_t v = 0; v < nv; ++v) {
    for (int64_t j = off[v]; j < off[v + 1]; ++j) {
      k[v] += w[j];
      if (part[adj[j]] == part[v]) in += w[j];
    }
    twom += k[v];
    a[part[v]] += k[v];
  }
  double sq = 0.;
  for (double x : a) sq += x * x;
  return in / twom - sq / (twom * twom);
}

extern "C" double orc_nmi(int64_t n, const int64_t* x, const int64_t* y) {
  std::unordered_map<int64_t, double> cx, cy;
  for (int64_t i = 0; i < n; ++i) { cx[x[i]] += 1; cy[y[i]] += 1; }
  std::unordered_map<int64_t, std::unordered_map<int64_t, double>> joint;
  for (int64_t i = 0; i < n; ++i) joint[x[i]][y[i]] += 1;
  double hx = 0., hy = 0., mi = 0.;
  const double N = (double)n;
  for (auto& p : cx) hx -= p.second / N * log(p.second / N);
  for (auto& p : cy) hy -= p.second / N * log(p.second / N);
  for (auto& p : joint)
    for (auto& q : p.second) {
      const double pxy = q.second / N;
      mi += pxy * log(pxy / ((cx[p.first] / N) * (cy[q.first] / N)));
    }
  if (hx + hy == 0.) return 1.;
  return 2. * mi / (hx + hy);
}
