// host_io.cpp -- Vite binary graph files and library-wide error state.
//
// File layout (graph.cpp:341-395): int64 NV, int64 NE, int64 offsets[NV+1],
// then {int64 tail; double weight} records (types.hpp:49-55).  As in the
// reference's first-touch read path (graph.cpp:397-435, always compiled in by
// its Makefile) the records are read right after the offsets, for
// offsets[NV]-offsets[0] records; a header NE that disagrees is reported with
// the reference's message (graph.cpp:376-382) and the offsets win; offsets
// are rebased to start at 0 (graph.cpp:470-472).
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <vector>

#include "nido_b200.h"
#include "nido_internal.h"

static thread_local char g_err[512] = "";
static unsigned long long g_launches = 0;

extern "C" void nido_count_launch(void) { __atomic_fetch_add(&g_launches, 1ull, __ATOMIC_RELAXED); }
extern "C" void nido_count_launches(uint64_t n) { __atomic_fetch_add(&g_launches, (unsigned long long)n, __ATOMIC_RELAXED); }
extern "C" uint64_t nido_launch_count(void) { return __atomic_load_n(&g_launches, __ATOMIC_RELAXED); }

extern "C" int nido_set_error(int code, const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
  return code;
}

extern "C" const char* nido_last_error(void) { return g_err; }
extern "C" const char* nido_version(void) { return "nido_b200 0.1 (sm_100a)"; }

extern "C" void nido_csr_free(nido_csr* g) {
  if (!g) return;
  free(g->off);
  free(g->adj);
  free(g->w);
  g->off = nullptr;
  g->adj = nullptr;
  g->w = nullptr;
  g->nv = g->ne = 0;
}

extern "C" int nido_read_vite(const char* path, nido_csr* out) {
  if (!path || !out) return nido_set_error(NIDO_E_INVALID, "nido_read_vite: null argument");
  memset(out, 0, sizeof(*out));
  FILE* f = fopen(path, "rb");
  if (!f) return nido_set_error(NIDO_E_IO, " Error opening file! (%s)", path);
  int64_t hdr[2];
  if (fread(hdr, sizeof(int64_t), 2, f) != 2 || hdr[0] < 0) {
    fclose(f);
    return nido_set_error(NIDO_E_IO, "%s: truncated header", path);
  }
  const int64_t nv = hdr[0];
  int64_t* off = (int64_t*)malloc(sizeof(int64_t) * (nv + 1));
  if (!off) { fclose(f); return nido_set_error(NIDO_E_NOMEM, "read_vite: host allocation failed"); }
  if ((int64_t)fread(off, sizeof(int64_t), nv + 1, f) != nv + 1) {
    free(off); fclose(f);
    return nido_set_error(NIDO_E_IO, "%s: truncated offsets", path);
  }
  const int64_t ne = off[nv] - off[0];
  if (ne < 0) { free(off); fclose(f); return nido_set_error(NIDO_E_IO, "%s: decreasing offsets", path); }
  if (ne != hdr[1]) {
    printf("!!! The graph has been modified in edges\n");
    printf("Original edges: %lld\nNew edges: %lld\n", (long long)hdr[1], (long long)ne);
  }
  int64_t* adj = (int64_t*)malloc(sizeof(int64_t) * (ne > 0 ? ne : 1));
  double* w = (double*)malloc(sizeof(double) * (ne > 0 ? ne : 1));
  if (!adj || !w) {
    free(off); free(adj); free(w); fclose(f);
    return nido_set_error(NIDO_E_NOMEM, "read_vite: host allocation failed");
  }
  // records are read in 64 MiB chunks and split into the two arrays
  const int64_t chunk = (int64_t)1 << 22;
  std::vector<int64_t> buf(2 * (size_t)(ne < chunk ? (ne > 0 ? ne : 1) : chunk));
  for (int64_t done = 0; done < ne;) {
    const int64_t n = (ne - done) < chunk ? (ne - done) : chunk;
    if ((int64_t)fread(buf.data(), 16, n, f) != n) {
      free(off); free(adj); free(w); fclose(f);
      return nido_set_error(NIDO_E_IO, "%s: truncated edge records", path);
    }
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) {
      adj[done + i] = buf[2 * i];
      memcpy(&w[done + i], &buf[2 * i + 1], 8);
    }
    done += n;
  }
  fclose(f);
  const int64_t base = off[0];
  for (int64_t i = 0; i <= nv; ++i) off[i] -= base;
  out->nv = nv; out->ne = ne; out->off = off; out->adj = adj; out->w = w;
  return NIDO_OK;
}

extern "C" int nido_write_vite(const char* path, const nido_csr* g) {
  if (!path || !g || !g->off) return nido_set_error(NIDO_E_INVALID, "nido_write_vite: null argument");
  FILE* f = fopen(path, "wb");
  if (!f) return nido_set_error(NIDO_E_IO, "cannot open %s for writing", path);
  const int64_t base = g->off[0];
  const int64_t ne = g->off[g->nv] - base;
  int64_t hdr[2] = {g->nv, ne};
  bool ok = fwrite(hdr, 8, 2, f) == 2 && (int64_t)fwrite(g->off, 8, g->nv + 1, f) == g->nv + 1;
  const int64_t chunk = (int64_t)1 << 22;
  std::vector<int64_t> buf(2 * (size_t)(ne < chunk ? (ne > 0 ? ne : 1) : chunk));
  for (int64_t done = 0; ok && done < ne;) {
    const int64_t n = (ne - done) < chunk ? (ne - done) : chunk;
    for (int64_t i = 0; i < n; ++i) {
      buf[2 * i] = g->adj[base + done + i];
      memcpy(&buf[2 * i + 1], &g->w[base + done + i], 8);
    }
    ok = (int64_t)fwrite(buf.data(), 16, n, f) == n;
    done += n;
  }
  if (fclose(f) != 0) ok = false;
  return ok ? NIDO_OK : nido_set_error(NIDO_E_IO, "short write to %s", path);
}
