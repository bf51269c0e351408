"""Graphs larger than the HBM budget: a context (or a server) whose budget
cannot hold a graph's edges keeps them in mapped page-locked host memory and
streams them over the host link as the kernels read them; the vertex state,
offsets and scratch stay in HBM.  The results are the in-HBM run's bit for
bit on integer weights, for a graph whose in-HBM footprint is several times
the budget; the server admits such a request instead of refusing it."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def big(nido_lib):
    return nido_lib.gen_rmat(1 << 20, 24 << 20, wmode=nido_lib.W_INT8, seed=51)


def test_overbudget_graph_streams_edges_and_matches(nido_lib, ctx, big):
    G = big
    full = nido_lib.graph_footprint(G.nv, G.ne, 2)
    streamed = nido_lib.graph_footprint_streamed(G.nv, G.ne, 2)
    budget = streamed + (64 << 20)
    assert full >= 3 * budget  # the graph is several times the budget
    with nido_lib.Graph(ctx, G, 2) as g:
        assert not g.host_edges()
        want, st_w = g.run()
        want_nido, st_wn = g.run(tie=nido_lib.NIDO_TIE_NIDO)
    with nido_lib.Context(0, budget) as small:
        with nido_lib.Graph(small, G, 2) as g:
            assert g.host_edges()
            assert g.device_bytes() <= budget
            got, st = g.run()
            got_nido, st_n = g.run(tie=nido_lib.NIDO_TIE_NIDO)
            c = g.download()  # the coarse CSR of the last phase comes back from host memory too
    assert np.array_equal(got, want)
    assert st.final_q == st_w.final_q and st.phases == st_w.phases and st.total_loops == st_w.total_loops
    assert np.array_equal(got_nido, want_nido) and st_n.final_q == st_wn.final_q
    assert c.off[-1] == len(c.adj) == len(c.w)


def test_overbudget_refused_when_vertex_state_does_not_fit(nido_lib, big):
    G = big
    streamed = nido_lib.graph_footprint_streamed(G.nv, G.ne, 2)
    with nido_lib.Context(0, streamed // 4) as tiny:
        with pytest.raises(nido_lib.NidoError) as e:
            nido_lib.Graph(tiny, G, 2)
        assert e.value.code == -3  # NIDO_E_NOMEM


def test_server_admits_overbudget_request(nido_lib, ctx, big):
    G = big
    small = nido_lib.gen_planted(32, 64, 12.0, 0.8, nido_lib.W_INT8, 52)
    with nido_lib.Graph(ctx, G, 2) as g:
        want, st_w = g.run()
    with nido_lib.Graph(ctx, small, 2) as g:
        want_s, _ = g.run()
    streamed = nido_lib.graph_footprint_streamed(G.nv, G.ne, 2)
    budget = streamed + nido_lib.graph_footprint(small.nv, small.ne, 2) + (64 << 20)
    assert nido_lib.graph_footprint(G.nv, G.ne, 2) > budget
    with nido_lib.Server(0, budget, workers=2) as srv:
        tb = srv.submit(G)
        ts = srv.submit(small)
        out, info = srv.wait(tb)
        out_s, info_s = srv.wait(ts)
    assert info.status == 0 and info.host_edges == 1 and info.hbm_bytes == streamed
    assert np.array_equal(out, want) and info.final_q == st_w.final_q
    assert info_s.host_edges == 0 and np.array_equal(out_s, want_s)
