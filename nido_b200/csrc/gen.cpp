// gen.cpp -- seeded synthetic graph generators (planted partition, R-MAT,
// stochastic block model) producing the reference's CSR layout.
//
// Every random draw comes from a counter-based stream (seed, stream id, item
// index), so the output is identical for any thread count.  Edges are
// generated as undirected pairs and stored in both directions; each adjacency
// list is sorted by neighbour id.  Duplicate pairs are dropped for unit
// weights and merged by summing (in ascending weight order, so that both
// directions get the same sum) otherwise.
#include <math.h>
#include <omp.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "nido_b200.h"
#include "nido_internal.h"

namespace {

inline uint64_t mix64(uint64_t z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

struct Rng {
  uint64_t s;
  Rng(uint64_t seed, uint64_t stream, uint64_t item)
      : s(mix64(seed ^ mix64((stream << 56) ^ mix64(item)))) {}
  uint64_t next() { s += 0x9E3779B97F4A7C15ull; return mix64(s); }
  double uni() { return (double)(next() >> 11) * 0x1.0p-53; }                 // [0,1)
  int64_t below(int64_t n) { return (int64_t)(((unsigned __int128)next() * (uint64_t)n) >> 64); }
  double normal() {
    double u1 = 1.0 - uni(), u2 = uni();
    return sqrt(-2.0 * log(u1)) * cos(6.283185307179586 * u2);
  }
};

inline double draw_weight(int wmode, Rng& r) {
  switch (wmode) {
    case NIDO_W_UNIFORM: return 0.5 + r.uni();
    case NIDO_W_LOGNORMAL: return exp(0.5 * r.normal());
    case NIDO_W_INT8: return (double)(1 + r.below(8));
    default: return 1.0;
  }
}

struct Entry { int64_t nbr; double w; };

// Undirected pairs -> symmetric CSR.  Self-loops are dropped when requested,
// otherwise stored once.
int build_csr(int64_t nv, const std::vector<int64_t>& su, const std::vector<int64_t>& sv,
              const std::vector<double>& sw, bool drop_self, bool sum_dups, nido_csr* out) {
  const int64_t M = (int64_t)su.size();
  std::vector<int64_t> deg(nv + 1, 0);
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < M; ++i) {
    const int64_t u = su[i], v = sv[i];
    if (u == v) {
      if (!drop_self) __atomic_fetch_add(&deg[u + 1], 1, __ATOMIC_RELAXED);
    } else {
      __atomic_fetch_add(&deg[u + 1], 1, __ATOMIC_RELAXED);
      __atomic_fetch_add(&deg[v + 1], 1, __ATOMIC_RELAXED);
    }
  }
  for (int64_t i = 0; i < nv; ++i) deg[i + 1] += deg[i];
  const int64_t E0 = deg[nv];
  std::vector<Entry> ent(E0 > 0 ? E0 : 1);
  std::vector<int64_t> pos(deg.begin(), deg.end() - 1);
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < M; ++i) {
    const int64_t u = su[i], v = sv[i];
    const double w = sw[i];
    if (u == v) {
      if (drop_self) continue;
      int64_t p = __atomic_fetch_add(&pos[u], 1, __ATOMIC_RELAXED);
      ent[p] = {v, w};
    } else {
      int64_t p = __atomic_fetch_add(&pos[u], 1, __ATOMIC_RELAXED);
      ent[p] = {v, w};
      p = __atomic_fetch_add(&pos[v], 1, __ATOMIC_RELAXED);
      ent[p] = {u, w};
    }
  }
  std::vector<int64_t> ndeg(nv + 1, 0);
#pragma omp parallel for schedule(dynamic, 1024)
  for (int64_t v = 0; v < nv; ++v) {
    Entry* b = ent.data() + deg[v];
    Entry* e = ent.data() + deg[v + 1];
    std::sort(b, e, [](const Entry& x, const Entry& y) {
      return x.nbr != y.nbr ? x.nbr < y.nbr : x.w < y.w;
    });
    int64_t n = 0;
    for (Entry* p = b; p < e; ++p) {
      if (n > 0 && b[n - 1].nbr == p->nbr) {
        if (sum_dups) b[n - 1].w += p->w;
      } else {
        b[n++] = *p;
      }
    }
    ndeg[v + 1] = n;
  }
  for (int64_t i = 0; i < nv; ++i) ndeg[i + 1] += ndeg[i];
  const int64_t E = ndeg[nv];
  out->nv = nv;
  out->ne = E;
  out->off = (int64_t*)malloc(sizeof(int64_t) * (nv + 1));
  out->adj = (int64_t*)malloc(sizeof(int64_t) * (E > 0 ? E : 1));
  out->w = (double*)malloc(sizeof(double) * (E > 0 ? E : 1));
  if (!out->off || !out->adj || !out->w) {
    nido_csr_free(out);
    return nido_set_error(NIDO_E_NOMEM, "generator: host allocation failed");
  }
  memcpy(out->off, ndeg.data(), sizeof(int64_t) * (nv + 1));
#pragma omp parallel for schedule(dynamic, 1024)
  for (int64_t v = 0; v < nv; ++v) {
    const int64_t n = ndeg[v + 1] - ndeg[v];
    for (int64_t j = 0; j < n; ++j) {
      out->adj[ndeg[v] + j] = ent[deg[v] + j].nbr;
      out->w[ndeg[v] + j] = ent[deg[v] + j].w;
    }
  }
  return NIDO_OK;
}

}  // namespace

extern "C" int nido_gen_planted(int64_t nblocks, int64_t bs, double avg_degree, double p_intra,
                                int32_t wmode, uint64_t seed, nido_csr* out) {
  if (!out || nblocks < 1 || bs < 2 || avg_degree < 0 || p_intra < 0 || p_intra > 1)
    return nido_set_error(NIDO_E_INVALID, "nido_gen_planted: bad arguments");
  memset(out, 0, sizeof(*out));
  const int64_t nv = nblocks * bs;
  const int64_t M = llround((double)nv * avg_degree / 2.0);
  std::vector<int64_t> su(M), sv(M);
  std::vector<double> sw(M);
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < M; ++i) {
    Rng r(seed, 1, (uint64_t)i);
    int64_t u, v;
    if (nblocks == 1 || r.uni() < p_intra) {
      const int64_t b = r.below(nblocks);
      u = b * bs + r.below(bs);
      do { v = b * bs + r.below(bs); } while (v == u);
    } else {
      u = r.below(nv);
      do { v = r.below(nv); } while (v / bs == u / bs);
    }
    su[i] = u; sv[i] = v; sw[i] = draw_weight(wmode, r);
  }
  return build_csr(nv, su, sv, sw, true, wmode != NIDO_W_ONE, out);
}

extern "C" int nido_gen_rmat(int64_t nv, int64_t npairs, double a, double b, double c,
                             int32_t wmode, uint64_t seed, nido_csr* out) {
  if (!out || nv < 2 || npairs < 0 || a < 0 || b < 0 || c < 0 || a + b + c > 1)
    return nido_set_error(NIDO_E_INVALID, "nido_gen_rmat: bad arguments");
  memset(out, 0, sizeof(*out));
  int scale = 0;
  while (((int64_t)1 << scale) < nv) ++scale;
  std::vector<int64_t> su(npairs), sv(npairs);
  std::vector<double> sw(npairs);
  const double ab = a + b, abc = a + b + c;
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < npairs; ++i) {
    Rng r(seed, 2, (uint64_t)i);
    int64_t u = 0, v = 0;
    for (int tries = 0; tries < 64; ++tries) {
      u = 0; v = 0;
      for (int l = 0; l < scale; ++l) {
        const double x = r.uni();
        const int bu = x >= ab, bv = (x >= a && x < ab) || x >= abc;
        u = 2 * u + bu;
        v = 2 * v + bv;
      }
      if (u < nv && v < nv) break;
      u = v = 0;  // give up after 64 tries: the pair becomes a dropped self-loop
    }
    su[i] = u; sv[i] = v; sw[i] = draw_weight(wmode, r);
  }
  return build_csr(nv, su, sv, sw, true, wmode != NIDO_W_ONE, out);
}

extern "C" int nido_gen_sbm(int64_t nv, double alpha, int64_t cmin, int64_t cmax, double avg_degree,
                            double p_intra, int32_t wmode, int32_t permute, uint64_t seed,
                            nido_csr* out) {
  if (!out || nv < 2 || cmin < 1 || cmax < cmin || alpha <= 1.0 || p_intra < 0 || p_intra > 1)
    return nido_set_error(NIDO_E_INVALID, "nido_gen_sbm: bad arguments");
  memset(out, 0, sizeof(*out));
  // community sizes: continuous power law p(x) ~ x^-alpha on [cmin, cmax],
  // drawn by inverse CDF until they cover nv; the last one is truncated
  std::vector<int64_t> start{0};
  const double e = 1.0 - alpha;
  const double lo = pow((double)cmin, e), hi = pow((double)cmax + 1.0, e);
  for (int64_t j = 0; start.back() < nv; ++j) {
    Rng r(seed, 3, (uint64_t)j);
    int64_t s = (int64_t)floor(pow(lo + r.uni() * (hi - lo), 1.0 / e));
    s = std::min(std::max(s, cmin), cmax);
    start.push_back(std::min(nv, start.back() + s));
  }
  const int64_t nc = (int64_t)start.size() - 1;
  std::vector<int32_t> cpos(nv);
#pragma omp parallel for schedule(static)
  for (int64_t c = 0; c < nc; ++c)
    for (int64_t p = start[c]; p < start[c + 1]; ++p) cpos[p] = (int32_t)c;
  std::vector<int64_t> perm(nv);
  for (int64_t p = 0; p < nv; ++p) perm[p] = p;
  if (permute) {
    Rng r(seed, 4, 0);
    for (int64_t p = nv - 1; p > 0; --p) std::swap(perm[p], perm[r.below(p + 1)]);
  }
  const int64_t M = llround((double)nv * avg_degree / 2.0);
  std::vector<int64_t> su(M), sv(M);
  std::vector<double> sw(M);
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < M; ++i) {
    Rng r(seed, 5, (uint64_t)i);
    const int64_t p = r.below(nv);
    const int64_t c = cpos[p];
    const int64_t sz = start[c + 1] - start[c];
    int64_t q = p;
    if (r.uni() < p_intra && sz > 1) {
      do { q = start[c] + r.below(sz); } while (q == p);
    } else if (nc > 1) {
      for (int t = 0; t < 1000; ++t) { q = r.below(nv); if (cpos[q] != c) break; }
    }
    su[i] = perm[p]; sv[i] = perm[q]; sw[i] = draw_weight(wmode, r);
  }
  return build_csr(nv, su, sv, sw, true, wmode != NIDO_W_ONE, out);
}
