"""Many graphs in one run (nido_batch_*): every graph's result must equal
the one-graph run of the same engine on that graph alone -- bit-exact
clusterings, final Q, phase and loop counts on integer weights; NMI >= 0.95
and |dQ| <= 1e-3 on lognormal weights."""
import numpy as np
import pytest

from conftest import load_golden

pytestmark = pytest.mark.gpu


def bits(x):
    return np.asarray(x, np.float64).view(np.uint64)


def same_q(a, b):
    return (np.isnan(a) and np.isnan(b)) or bits(a) == bits(b)


def tiny(capi, nv, edges, w=1.0):
    """Undirected CSR from an edge list (both directions stored)."""
    src = [u for u, v in edges] + [v for u, v in edges if u != v]
    dst = [v for u, v in edges] + [u for u, v in edges if u != v]
    order = np.lexsort((dst, src)) if src else np.zeros(0, np.int64)
    src = np.asarray(src, np.int64)[order]
    dst = np.asarray(dst, np.int64)[order]
    off = np.zeros(nv + 1, np.int64)
    np.add.at(off, src + 1, 1)
    return capi.Csr(np.cumsum(off), dst, np.full(len(dst), w, np.float64))


def mixed_graphs(capi):
    gs = [
        capi.gen_rmat(1 << 15, 16 << 15, wmode=capi.W_INT8, seed=41),   # hub tier
        capi.gen_planted(64, 64, 16.0, 0.8, capi.W_INT8, 42),
        tiny(capi, 0, []),                                               # empty graph
        capi.gen_sbm(20000, cmin=16, cmax=2048, avg_degree=20.0, wmode=capi.W_INT8, seed=43),
        tiny(capi, 1, []),                                               # one isolated vertex
        tiny(capi, 2, [(0, 1)], 3.0),
        capi.gen_rmat(1 << 8, 16 << 8, wmode=capi.W_ONE, seed=44),
    ]
    for name in ("sparse_isolated", "selfloop_int", "planted_int"):
        d = load_golden(name)
        gs.append(capi.Csr(d["off"], d["adj"], d["w"]))
    rng = np.random.default_rng(45)
    for i in range(16):
        s = int(rng.integers(5, 13))
        gs.append(capi.gen_rmat(1 << s, int(rng.integers(4, 24)) << s,
                                wmode=capi.W_INT8 if i % 2 else capi.W_ONE, seed=100 + i))
    return gs


@pytest.fixture(scope="module")
def mixed(nido_lib):
    return mixed_graphs(nido_lib)


def plain_runs(capi, ctx, graphs, nb, tie, **kw):
    res = []
    for G in graphs:
        if G.nv == 0:
            res.append(None)
            continue
        with capi.Graph(ctx, G, nb) as g:
            cl, st = g.run(tie=tie, **kw)
        res.append((cl, st.final_q, st.phases, st.total_loops))
    return res


@pytest.mark.parametrize("nb,tie", [(1, 0), (2, 0), (2, 1), (3, 1)])
def test_batch_equals_plain_integer(nido_lib, ctx, mixed, nb, tie):
    want = plain_runs(nido_lib, ctx, mixed, nb, tie)
    with nido_lib.Batch(ctx, mixed, nb) as b:
        parts, q, ph, lo, st = b.run(tie=tie)
    assert st.phases >= max(w[2] for w in want if w is not None)
    for i, w in enumerate(want):
        if w is None:
            assert len(parts[i]) == 0 and ph[i] == 0 and lo[i] == 0
            continue
        cl, fq, phases, loops = w
        assert np.array_equal(parts[i], cl), f"graph {i}"
        assert same_q(q[i], fq), f"graph {i}: {q[i]} vs {fq}"
        assert ph[i] == phases and lo[i] == loops, f"graph {i}"


def test_batch_rerun_and_limits(nido_lib, ctx, mixed):
    with nido_lib.Batch(ctx, mixed, 2) as b:
        first = b.run()
        again = b.run()
        for x, y in zip(first[0], again[0]):
            assert np.array_equal(x, y)
        assert np.array_equal(bits(first[1]), bits(again[1]))
        # loop cap and a large threshold end graphs early; still per-graph equal
        parts, q, ph, lo, _ = b.run(tau=1e-2, max_iter=2)
    want = plain_runs(nido_lib, ctx, mixed, 2, 0, tau=1e-2, max_iter=2)
    for i, w in enumerate(want):
        if w is None:
            continue
        assert np.array_equal(parts[i], w[0]) and same_q(q[i], w[1])
        assert ph[i] == w[2] and lo[i] == w[3]


def test_batch_lognormal_quality(nido_lib, ctx, orc):
    gs = [nido_lib.gen_sbm(int(n), cmin=16, cmax=1024, avg_degree=16.0, wmode=nido_lib.W_LOGNORMAL, seed=50 + i)
          for i, n in enumerate((3000, 12000, 800, 20000))]
    want = plain_runs(nido_lib, ctx, gs, 2, 0)
    with nido_lib.Batch(ctx, gs, 2) as b:
        parts, q, _, _, _ = b.run()
    for i, G in enumerate(gs):
        assert abs(q[i] - want[i][1]) <= 1e-3
        assert orc.nmi(parts[i], want[i][0]) >= 0.95
        assert abs(orc.partition_modularity(G.off, G.adj, G.w, parts[i]) - q[i]) <= 1e-5


def test_batch_rejects_crossing_edges(nido_lib, ctx):
    a = tiny(nido_lib, 3, [(0, 1), (1, 2)])
    vbase, u = nido_lib.pack_graphs([a, a])
    u.adj[0] = 4  # vertex 0 of graph 0 now points into graph 1
    with pytest.raises(nido_lib.NidoError):
        nido_lib.Batch(ctx, packed=(vbase, u))
    with pytest.raises(nido_lib.NidoError):
        nido_lib.Batch(ctx, packed=(np.array([0, 4, 3], np.int64), nido_lib.pack_graphs([a, a])[1]))


def test_stopped_graphs_leave_the_lists_by_compaction(nido_lib, ctx):
    """Many small planted graphs that converge in a few sweeps beside one
    R-MAT graph that iterates longer: once the stopped graphs hold a quarter of
    the listed vertices their vertices leave the tier lists (a stable
    compaction, timed in host_ms[2]), and every graph still equals its run
    alone."""
    graphs = [nido_lib.gen_planted(32, 64, 12.0, 0.9, nido_lib.W_INT8, 600 + i) for i in range(24)]
    graphs.append(nido_lib.gen_rmat(1 << 13, 12 << 13, wmode=nido_lib.W_INT8, seed=650))
    want = plain_runs(nido_lib, ctx, graphs, 2, 0)
    with nido_lib.Batch(ctx, graphs, 2) as b:
        parts, q, ph, lo, st = b.run()
    assert st.host_ms[2] > 0  # the lists were compacted at least once
    for i, (cl, fq, phases, loops) in enumerate(want):
        assert np.array_equal(parts[i], cl), f"graph {i}"
        assert same_q(q[i], fq) and ph[i] == phases and lo[i] == loops, f"graph {i}"
