"""Seeded synthetic graph sets of the many-graph and serving workloads.

Many-graph batch: ngraphs independent graphs, vertex counts log-uniform in
[100, 1,000,000], each an SBM (power-law community sizes, exponent 2.5,
clipped 16..65,536, 70% intra-community edges) or an R-MAT ((0.57, 0.19,
0.19, 0.05), vertex count not a power of two handled by rejection) with
probability 1/2, average degree uniform in [8, 64], integer weights uniform in
{1..8} stored as FP64.  When the drawn total of directed edges exceeds the
cap, every vertex count is scaled by cap / total (clamped at >= 100), which
keeps the log-uniform shape and the degree law.

Serving stream: requests with vertex counts log-uniform in [1e3, 1e7], half
SBM (as above, average degree 32) and half R-MAT with edge factor 16, all
with weights uniform in [0.5, 1.5], Poisson arrivals at a given rate.
"""
from __future__ import annotations

import numpy as np

from . import capi


def single_graph(name: str) -> capi.Csr:
    """The one-graph workloads: 'rmat22' (R-MAT scale 22, edge factor 16,
    (0.57,0.19,0.19,0.05), weights 1.0, seed 2), 'rmat20' (the same at scale
    20), 'planted' (65,536 vertices in 256 blocks, average degree 32, 80%
    intra, U[0.5,1.5] weights, seed 1), 'sbm' (16,777,216 vertices, power-law
    communities 2.5 in 16..65,536, average degree 32, 70% intra, lognormal
    weights, seed 3)."""
    if name == "rmat22":
        return capi.gen_rmat(1 << 22, 16 << 22, wmode=capi.W_ONE, seed=2)
    if name == "rmat20":
        return capi.gen_rmat(1 << 20, 16 << 20, wmode=capi.W_ONE, seed=2)
    if name == "planted":
        return capi.gen_planted(256, 256, 32.0, 0.8, capi.W_UNIFORM, 1)
    if name == "sbm":
        return capi.gen_sbm(1 << 24, 2.5, 16, 65536, 32.0, 0.7, capi.W_LOGNORMAL, True, 3)
    raise ValueError(f"unknown workload {name}")


def many_graph_plan(ngraphs: int = 4096, seed: int = 4, max_edges: float = 1.5e9,
                    vmin: int = 100, vmax: int = 1_000_000):
    """(vertex counts, average degrees, kinds) with kind 0 = SBM, 1 = R-MAT."""
    rng = np.random.default_rng(seed)
    V = np.exp(rng.uniform(np.log(vmin), np.log(vmax), ngraphs))
    d = rng.uniform(8.0, 64.0, ngraphs)
    kind = rng.integers(0, 2, ngraphs)
    total = float((V * d).sum())
    if total > max_edges:
        V = V * (max_edges / total)
    V = np.maximum(np.rint(V), vmin).astype(np.int64)
    return V, d, kind


def make_one(nv: int, degree: float, kind: int, wmode: int, seed: int) -> capi.Csr:
    if kind == 0:
        return capi.gen_sbm(int(nv), 2.5, 16, 65536, float(degree), 0.7, wmode, True, seed)
    return capi.gen_rmat(int(nv), int(round(nv * degree / 2)), wmode=wmode, seed=seed)


def many_graphs_packed(ngraphs: int = 4096, seed: int = 4, max_edges: float = 1.5e9):
    """The many-graph batch packed as one CSR without holding every graph
    twice: returns (vbase, union Csr, plan)."""
    V, d, kind = many_graph_plan(ngraphs, seed, max_edges)
    # each generated pair gives at most two directed edges
    bound = int(sum(2 * int(round(v * x / 2)) + 2 for v, x in zip(V, d)))
    adj = np.empty(bound, np.int64)
    w = np.empty(bound, np.float64)
    off = np.empty(int(V.sum()) + 1, np.int64)
    vbase = np.zeros(ngraphs + 1, np.int64)
    np.cumsum(V, out=vbase[1:])
    e = 0
    for i in range(ngraphs):
        g = make_one(V[i], d[i], kind[i], capi.W_INT8, seed * 1_000_003 + i)
        assert g.nv == V[i]
        off[vbase[i]:vbase[i + 1]] = g.off[:-1] + e
        adj[e:e + g.ne] = g.adj + vbase[i]
        w[e:e + g.ne] = g.w
        e += g.ne
    off[-1] = e
    return vbase, capi.Csr(off, adj[:e], w[:e]), (V, d, kind)


def unpack(vbase: np.ndarray, u: capi.Csr, i: int) -> capi.Csr:
    """Graph i of a packed set as its own CSR."""
    v0, v1 = int(vbase[i]), int(vbase[i + 1])
    e0, e1 = int(u.off[v0]), int(u.off[v1])
    return capi.Csr(u.off[v0:v1 + 1] - e0, u.adj[e0:e1] - v0, u.w[e0:e1])


def serving_requests(n: int, rate: float, seed: int = 5, vmin: float = 1e3, vmax: float = 1e7):
    """Arrival times (s, Poisson at `rate` per second) and (nv, kind) of n
    requests; kind 0 = SBM with average degree 32, 1 = R-MAT edge factor 16."""
    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.exponential(1.0 / rate, n))
    V = np.rint(np.exp(rng.uniform(np.log(vmin), np.log(vmax), n))).astype(np.int64)
    kind = rng.integers(0, 2, n)
    return t, V, kind


def make_request(nv: int, kind: int, seed: int) -> capi.Csr:
    if kind == 0:
        return capi.gen_sbm(int(nv), 2.5, 16, 65536, 32.0, 0.7, capi.W_UNIFORM, True, seed)
    return capi.gen_rmat(int(nv), 16 * int(nv), wmode=capi.W_UNIFORM, seed=seed)
