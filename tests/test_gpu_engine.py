"""Parity of the CUDA engine (through the C ABI) with the reference fixtures
and the CPU oracle.

Bar: bit-exact move targets, community degrees, coarsened graphs and
partitions on integer-weighted graphs (every FP64 sum is exact there);
k_v, m and Q bit-exact on any weights given the same inputs; elsewhere
Q within 1e-12 relative per step, final Q within 1e-3 and NMI >= 0.95.
"""
import numpy as np
import pytest

from conftest import INTEGER_CASES, golden_cases, load_golden

pytestmark = pytest.mark.gpu
CASES = golden_cases()


def bits(x):
    return np.asarray(x, np.float64).view(np.uint64)


def csr_of(capi, d):
    return capi.Csr(d["off"], d["adj"], d["w"])


# ---------------------------------------------------------------- fixtures ----
@pytest.mark.parametrize("name", CASES)
def test_k_m_batches_vs_reference(nido_lib, ctx, name):
    d = load_golden(name)
    for nb, tag in ((1, "move_singleton_b1_0"), (3, "move_singleton_b3_1")):
        with nido_lib.Graph(ctx, csr_of(nido_lib, d), nb) as g:
            k, m = g.vertex_weights()
            assert np.array_equal(bits(k), bits(d["k"]))
            assert bits(m) == d[tag + "_mbits"][0]
            assert np.array_equal(g.batches(), d[tag + "_cuts"])


@pytest.mark.parametrize("name", CASES)
@pytest.mark.parametrize("assign", ["singleton", "random"])
def test_modularity_vs_reference(nido_lib, ctx, name, assign):
    d = load_golden(name)
    tag = f"move_{assign}_b1_0"
    with nido_lib.Graph(ctx, csr_of(nido_lib, d), 1) as g:
        g.set_community_ids(d[f"assign_{assign}"])
        _, _, a = g.state()
        q = g.compute_modularity()
        ref_q = d[tag + "_qbits"][0:1].view(np.float64)[0]
        if name in INTEGER_CASES:
            assert np.array_equal(a, d[tag + "_a"])
            assert bits(q) == d[tag + "_qbits"][0]
        else:
            assert np.allclose(a, d[tag + "_a"], rtol=1e-12, atol=0)
            assert abs(q - ref_q) <= 1e-12 * abs(ref_q)


@pytest.mark.parametrize("name", CASES)
@pytest.mark.parametrize("assign", ["singleton", "random"])
@pytest.mark.parametrize("nb,batch", [(1, 0), (3, 1)])
def test_move_vs_reference(nido_lib, ctx, name, assign, nb, batch):
    d = load_golden(name)
    tag = f"move_{assign}_b{nb}_{batch}"
    with nido_lib.Graph(ctx, csr_of(nido_lib, d), nb) as g:
        g.set_community_ids(d[f"assign_{assign}"])
        g.louvain_update(batch, nido_lib.NIDO_TIE_NIDO)
        _, newc, _ = g.state()
        cuts = d[tag + "_cuts"]
        v0, v1 = cuts[batch], cuts[batch + 1]
        ref = d[tag + "_newcomm"][v0:v1]
        if name in INTEGER_CASES:
            assert np.array_equal(newc[v0:v1], ref)
        else:
            assert np.mean(newc[v0:v1] == ref) >= 0.99


@pytest.mark.parametrize("name", CASES)
def test_coarsen_vs_reference(nido_lib, ctx, name):
    d = load_golden(name)
    with nido_lib.Graph(ctx, csr_of(nido_lib, d), 1) as g:
        g.set_community_ids(d["assign_random"])
        done = g.aggregation()
        assert done == bool(d["coarsen_random_done"][0])
        c = g.download()
        assert np.array_equal(c.off, d["coarsen_random_off"])
        assert np.array_equal(c.adj, d["coarsen_random_adj"])
        if name in INTEGER_CASES:
            assert np.array_equal(c.w, d["coarsen_random_w"])
        else:
            assert np.allclose(c.w, d["coarsen_random_w"], rtol=1e-12, atol=0)
        assert np.array_equal(g.clustering(), d["coarsen_random_newid"])


@pytest.mark.parametrize("name", CASES)
@pytest.mark.parametrize("nb", [1, 2])
def test_full_run_vs_reference(nido_lib, ctx, orc, name, nb):
    d = load_golden(name)
    with nido_lib.Graph(ctx, csr_of(nido_lib, d), nb) as g:
        cl, st = g.run(tie=nido_lib.NIDO_TIE_NIDO)
    ref_q = d[f"run_b{nb}_final_q"]
    q = np.array(st.q_phase[: st.phases])
    if name in INTEGER_CASES:
        assert np.array_equal(q, ref_q)
        assert np.array_equal(cl, d[f"run_b{nb}_partition"])
    else:
        assert abs(q[-1] - ref_q[-1]) <= 1e-3
        assert orc.nmi(cl, d[f"run_b{nb}_partition"]) >= 0.95


@pytest.mark.parametrize("name", CASES)
def test_default_tie_rule_quality(nido_lib, ctx, orc, name):
    """Smallest-id ties (the engine's default) reach the reference's quality."""
    d = load_golden(name)
    with nido_lib.Graph(ctx, csr_of(nido_lib, d), 2) as g:
        cl, st = g.run()
    ref = d["run_b2_partition"]
    q_ref = orc.partition_modularity(d["off"], d["adj"], d["w"], ref)
    q = orc.partition_modularity(d["off"], d["adj"], d["w"], cl)
    assert q >= q_ref - 1e-3


# ------------------------------------------------------------ vs oracle ----
def generated(capi):
    return {
        "planted_c1_int": capi.gen_planted(256, 256, 32.0, 0.8, capi.W_INT8, 1),
        "rmat_s14_int": capi.gen_rmat(1 << 14, 16 << 14, wmode=capi.W_INT8, seed=21),
        "rmat_s16_unit": capi.gen_rmat(1 << 16, 16 << 16, wmode=capi.W_ONE, seed=22),
        "sbm_int": capi.gen_sbm(50000, cmin=16, cmax=4096, avg_degree=24.0, wmode=capi.W_INT8, seed=23),
    }


@pytest.fixture(scope="module")
def graphs(nido_lib):
    return generated(nido_lib)


@pytest.mark.parametrize("gname", ["planted_c1_int", "rmat_s14_int", "rmat_s16_unit", "sbm_int"])
@pytest.mark.parametrize("tie", [0, 1])
def test_move_commit_vs_oracle(nido_lib, ctx, orc, graphs, gname, tie):
    G = graphs[gname]
    rng = np.random.default_rng(5)
    comm0 = rng.integers(0, max(2, G.nv // 16), G.nv).astype(np.int64)
    nb = 3
    with nido_lib.Graph(ctx, G, nb) as g:
        k, m = g.vertex_weights()
        cuts = g.batches()
        assert np.array_equal(cuts, orc.batch_cuts(G.off, nb))
        g.set_community_ids(comm0)
        comm, newc_o, a = comm0.copy(), comm0.copy(), orc.community_weights(comm0, k)
        for b in range(nb):
            g.louvain_update(b, tie)
            _, newc_g, _ = g.state()
            want, _ = orc.move(G.off, G.adj, G.w, comm, a, k, m, cuts[b], cuts[b + 1], tie=tie)
            v0, v1 = cuts[b], cuts[b + 1]
            assert np.array_equal(newc_g[v0:v1], want[v0:v1]), f"batch {b}"
            g.update_community_weights(b)
            g.update_community_ids(b)
            newc_o[v0:v1] = want[v0:v1]
            orc.commit(v0, v1, comm, newc_o, k, a)
            cg, ng, ag = g.state()
            assert np.array_equal(cg, comm) and np.array_equal(ag, a)
        q = g.compute_modularity()
        assert bits(q) == bits(orc.modularity(G.off, G.adj, G.w, comm, a, m))
        g.restore_community()
        orc.commit(0, G.nv, comm, newc_o, k, a)
        cg, _, ag = g.state()
        assert np.array_equal(cg, comm0) and np.array_equal(cg, comm) and np.array_equal(ag, a)


@pytest.mark.parametrize("gname", ["planted_c1_int", "rmat_s14_int", "sbm_int"])
def test_coarsen_vs_oracle(nido_lib, ctx, orc, graphs, gname):
    G = graphs[gname]
    rng = np.random.default_rng(6)
    comm = rng.integers(0, max(2, G.nv // 64), G.nv).astype(np.int64)
    newid, (off, adj, w) = orc.coarsen(G.off, G.adj, G.w, comm)
    with nido_lib.Graph(ctx, G, 1) as g:
        g.set_community_ids(comm)
        assert not g.aggregation()
        c = g.download()
        assert np.array_equal(c.off, off) and np.array_equal(c.adj, adj) and np.array_equal(c.w, w)
        assert np.array_equal(g.clustering(), newid)
        k, m = g.vertex_weights()
        assert np.array_equal(bits(k), bits(orc.vertex_weights(off, w)))


@pytest.mark.parametrize("gname", ["planted_c1_int", "rmat_s14_int", "sbm_int"])
@pytest.mark.parametrize("tie", [0, 1])
def test_full_run_vs_oracle(nido_lib, ctx, orc, graphs, gname, tie):
    G = graphs[gname]
    want, st_o = orc.louvain(G.off, G.adj, G.w, nbatches=2, tie=tie)
    with nido_lib.Graph(ctx, G, 2) as g:
        cl, st = g.run(tie=tie)
    assert st.phases == st_o.phases and st.total_loops == st_o.total_loops
    assert np.array_equal(np.array(st.q_phase[: st.phases]), np.array(st_o.q_phase[: st_o.phases]))
    assert np.array_equal(cl, want)


@pytest.mark.parametrize("scale", [1.0, float(1 << 27)])
def test_integer_weight_paths_vs_oracle(nido_lib, ctx, orc, graphs, scale):
    """Integer weights run the move tables in int32 while every vertex's sum
    of |w| stays below 2^31 and in FP64 above (weights scaled by 2^27 push
    the sums past it); both are exact, so both match the oracle bit for bit."""
    G0 = graphs["sbm_int"]
    G = nido_lib.Csr(G0.off, G0.adj, G0.w * scale)
    want, st_o = orc.louvain(G.off, G.adj, G.w, nbatches=2)
    with nido_lib.Graph(ctx, G, 2) as g:
        cl, st = g.run()
    assert st.phases == st_o.phases and st.total_loops == st_o.total_loops
    assert np.array_equal(np.array(st.q_phase[: st.phases]), np.array(st_o.q_phase[: st_o.phases]))
    assert np.array_equal(cl, want)


def test_lognormal_run_quality(nido_lib, ctx, orc):
    G = nido_lib.gen_sbm(40000, cmin=16, cmax=2048, avg_degree=20.0, wmode=nido_lib.W_LOGNORMAL, seed=31)
    want, st_o = orc.louvain(G.off, G.adj, G.w, nbatches=2)
    with nido_lib.Graph(ctx, G, 2) as g:
        cl, st = g.run()
    assert abs(st.final_q - st_o.final_q) <= 1e-3
    assert orc.nmi(cl, want) >= 0.95
    q = orc.partition_modularity(G.off, G.adj, G.w, cl)
    assert abs(q - st.final_q) <= 1e-5


def test_determinism_integer(nido_lib, ctx, graphs):
    G = graphs["rmat_s16_unit"]
    outs = []
    for _ in range(2):
        with nido_lib.Graph(ctx, G, 2) as g:
            outs.append(g.run()[0])
    assert np.array_equal(outs[0], outs[1])


# ---------------------------------------------------------- colouring ----
def test_coloring_proper_and_relabel(nido_lib, ctx, orc, graphs):
    G = graphs["rmat_s14_int"]
    colors, nc = ctx.color(G, seed=7)
    src = np.repeat(np.arange(G.nv), np.diff(G.off))
    mask = src != G.adj
    assert colors.min() >= 0 and nc == colors.max() + 1
    assert not np.any(colors[src[mask]] == colors[G.adj[mask]])
    colors2, _ = ctx.color(G, seed=7)
    assert np.array_equal(colors, colors2)
    out, no = ctx.color_relabel(G, colors)
    no_o, (off, adj, w) = orc.color_relabel(G.off, G.adj, G.w, colors)
    assert np.array_equal(no, no_o)
    assert np.array_equal(out.off, off) and np.array_equal(out.adj, adj) and np.array_equal(out.w, w)


# ------------------------------------------------------------- edge cases ----
def test_edge_cases(nido_lib, ctx, orc):
    capi = nido_lib
    # no edges: nothing moves, one phase
    G = capi.Csr(np.zeros(6, np.int64), np.zeros(0, np.int64), np.zeros(0))
    with capi.Graph(ctx, G, 2) as g:
        cl, st = g.run()
        assert np.array_equal(cl, np.arange(5))
    # more batches than vertices
    G = capi.gen_planted(2, 4, 3.0, 0.9, capi.W_INT8, 3)
    with capi.Graph(ctx, G, 16) as g:
        assert np.array_equal(g.batches(), orc.batch_cuts(G.off, 16))
        cl, _ = g.run()
    want, _ = orc.louvain(G.off, G.adj, G.w, nbatches=16)
    assert np.array_equal(cl, want)
    # invalid inputs are rejected with an error, not a fault
    bad = capi.Csr(G.off.copy(), G.adj.copy(), G.w.copy())
    bad.adj[0] = G.nv + 5
    with pytest.raises(capi.NidoError):
        capi.Graph(ctx, bad, 1)
    with capi.Graph(ctx, G, 1) as g:
        with pytest.raises(capi.NidoError):
            g.set_community_ids(np.full(G.nv, -1, np.int64))
        with pytest.raises(capi.NidoError):
            g.louvain_update(3)
    with pytest.raises(capi.NidoError):
        capi.Graph(ctx, G, 0)


def test_full_size_rmat_properties(nido_lib, ctx, orc):
    """Scale-18 R-MAT: size-independent checks of a whole run."""
    G = nido_lib.gen_rmat(1 << 18, 16 << 18, wmode=nido_lib.W_ONE, seed=2)
    with nido_lib.Graph(ctx, G, 2) as g:
        cl, st = g.run()
    assert st.phases >= 2
    q = orc.partition_modularity(G.off, G.adj, G.w, cl)
    assert abs(q - st.final_q) <= 1e-5
    # communities are dense ids 0..n-1
    u = np.unique(cl)
    assert u[0] == 0 and u[-1] == len(u) - 1


def test_freed_blocks_reused_and_trimmed(nido_lib):
    """A context keeps the blocks of a freed graph and its next upload of the
    same sizes reuses them (the cache does not grow); results are unchanged;
    nido_ctx_trim hands the cached bytes back to the driver."""
    G = nido_lib.gen_rmat(1 << 15, 16 << 15, wmode=nido_lib.W_INT8, seed=5)
    with nido_lib.Context(0) as c:
        with nido_lib.Graph(c, G, 2) as g:
            want, st0 = g.run()
            used = g.device_bytes()
        held = c.trim()
        assert held >= used * 0.9
        assert c.trim() == 0
        for _ in range(3):
            with nido_lib.Graph(c, G, 2) as g:
                got, st = g.run()
            assert np.array_equal(got, want) and st.final_q == st0.final_q
        assert c.trim() == held  # three uploads, one set of blocks


def test_vite_streamed_to_device(nido_lib, ctx, orc, tmp_path):
    """nido_graph_upload_vite gives the graph that nido_read_vite +
    nido_graph_upload give: same device CSR (offsets rebased), and on integer
    weights the same run bit for bit (FP64 weights leave the last bit of Q to
    the order of the community-weight atomics); a missing or truncated file
    is an error."""
    G = nido_lib.gen_sbm(20000, cmin=16, cmax=1024, avg_degree=24.0, wmode=nido_lib.W_LOGNORMAL, seed=9)
    p = str(tmp_path / "g.bin")
    nido_lib.write_vite(p, G)
    with nido_lib.Graph(ctx, nido_lib.read_vite(p), 2) as a, nido_lib.Graph.from_vite(ctx, p, 2) as b:
        da, db = a.download(), b.download()
        assert np.array_equal(da.off, db.off) and np.array_equal(da.adj, db.adj)
        assert np.array_equal(da.w.view(np.uint64), db.w.view(np.uint64))
        ca, sa = a.run()
        cb, sb = b.run()
        assert abs(sa.final_q - sb.final_q) <= 1e-12 and orc.nmi(ca, cb) >= 0.99
    # offsets starting above 0 are rebased; records span several stream chunks
    raw = open(p, "rb").read()
    nv, ne = np.frombuffer(raw[:16], np.int64)
    off = np.frombuffer(raw[16:16 + 8 * (nv + 1)], np.int64) + 1000
    p2 = str(tmp_path / "g2.bin")
    open(p2, "wb").write(raw[:16] + off.tobytes() + raw[16 + 8 * (nv + 1):])
    with nido_lib.Graph.from_vite(ctx, p2, 2) as c:
        dc = c.download()
        assert np.array_equal(dc.off, da.off) and np.array_equal(dc.adj, da.adj)
    big = nido_lib.gen_rmat(1 << 20, 16 << 20, wmode=nido_lib.W_INT8, seed=4)  # > 4M records: 8 chunks
    p3 = str(tmp_path / "g3.bin")
    nido_lib.write_vite(p3, big)
    with nido_lib.Graph.from_vite(ctx, p3, 2) as d, nido_lib.Graph(ctx, big, 2) as e:
        dd = d.download()
        assert np.array_equal(dd.off, big.off) and np.array_equal(dd.adj, big.adj)
        assert np.array_equal(dd.w, big.w)
        cd, sd = d.run()
        ce, se = e.run()
        assert np.array_equal(cd, ce) and sd.final_q == se.final_q and sd.total_loops == se.total_loops
    open(p2, "wb").write(raw[: len(raw) - 8])
    with pytest.raises(nido_lib.NidoError):
        nido_lib.Graph.from_vite(ctx, p2, 2)
    with pytest.raises(nido_lib.NidoError):
        nido_lib.Graph.from_vite(ctx, str(tmp_path / "missing.bin"), 2)
