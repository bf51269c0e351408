"""Degree-tier configuration and its autotuner: any valid configuration gives
the same results on integer weights (bit for bit), the tuner returns a valid
configuration, and invalid ones are rejected."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def rmat16(nido_lib):
    return nido_lib.gen_rmat(1 << 16, 16 << 16, wmode=nido_lib.W_INT8, seed=71)


def test_lowered_thresholds_same_result(nido_lib, ctx, rmat16):
    with nido_lib.Graph(ctx, rmat16, 2) as g:
        want, st0 = g.run()
        c = g.tier_config()
        assert (c.warp_max_degree, c.cta_s_max_degree, c.cta_m_max_degree, c.cta_l_max_degree,
                c.cta_x_max_degree) == (192, 768, 1536, 2048, 12288)
        for warp, ctas, ctam, ctal, ctax, wave in ((64, 256, 1024, 1024, 1024, 1 << 16), (32, 32, 32, 32, 32, 1 << 16),
                                                   (96, 384, 768, 1536, 4096, 8 << 20), (128, 512, 1024, 2048, 2048, 4 << 20),
                                                   (128, 512, 1024, 2048, 12288, 4 << 20),
                                                   (192, 768, 1536, 3072, 12288, 4 << 20)):
            for clusters in (0, 1):  # hubs in global tables / on thread-block clusters
                c = nido_lib.TierConfig(warp, ctas, ctam, ctal, ctax, clusters, wave)
                g.set_tier_config(c)
                got, st = g.run()
                assert np.array_equal(got, want)
                assert st.final_q == st0.final_q and st.total_loops == st0.total_loops


def test_invalid_configs_rejected(nido_lib, ctx, rmat16):
    with nido_lib.Graph(ctx, rmat16, 2) as g:
        for bad in ((193, 512, 1024, 2048, 8192, 1 << 20), (128, 100, 1024, 2048, 8192, 1 << 20),
                    (64, 512, 1537, 2048, 8192, 1 << 20), (64, 512, 1024, 4096, 8192, 1 << 20),
                    (64, 512, 1024, 2048, 1024, 1 << 20), (64, 512, 1024, 2048, 12289, 1 << 20),
                    (64, 512, 1024, 2048, 8192, 10)):
            w, s, m, l, x, wave = bad
            with pytest.raises(nido_lib.NidoError):
                g.set_tier_config(nido_lib.TierConfig(w, s, m, l, x, 0, wave))
        with pytest.raises(nido_lib.NidoError):  # hub_clusters is 0 or 1
            g.set_tier_config(nido_lib.TierConfig(64, 512, 1024, 2048, 8192, 2, 1 << 20))


@pytest.mark.parametrize("tie", [0, 1])
def test_tuned_run_same_result(nido_lib, ctx, rmat16, tie):
    with nido_lib.Graph(ctx, rmat16, 2) as g:
        want, _ = g.run(tie=tie)
    with nido_lib.Graph(ctx, rmat16, 2) as g:
        got, st = g.run(tie=tie, tune=True)
        c = g.tier_config()
        assert 32 <= c.warp_max_degree <= c.cta_s_max_degree <= c.cta_m_max_degree <= c.cta_l_max_degree <= 3072
        assert c.cta_l_max_degree <= c.cta_x_max_degree <= 12288
        assert st.host_ms[6] > 0
        assert np.array_equal(got, want)
        best, ms = g.tune(tie=tie)
        assert ms > 0


def test_tuned_batch_same_result(nido_lib, ctx):
    gs = [nido_lib.gen_rmat(1 << s, 12 << s, wmode=nido_lib.W_INT8, seed=80 + s) for s in (9, 12, 14, 15)]
    with nido_lib.Batch(ctx, gs, 2) as b:
        want = b.run()[0]
    with nido_lib.Batch(ctx, gs, 2) as b:
        got = b.run(tune=True)[0]
    for x, y in zip(want, got):
        assert np.array_equal(x, y)


@pytest.mark.parametrize("ctax", [1024, 4096])
def test_cluster_hub_tier_vs_oracle(nido_lib, ctx, orc, ctax):
    """With the CTA-XL tier capped low, vertices above the cap are hubs; on
    integer weights with the smallest-id rule they run on thread-block
    clusters (tables in distributed shared memory), and the run still matches
    the oracle bit for bit."""
    G = nido_lib.gen_rmat(1 << 15, 16 << 15, wmode=nido_lib.W_INT8, seed=91)
    want, st_o = orc.louvain(G.off, G.adj, G.w, nbatches=2)
    with nido_lib.Graph(ctx, G, 2) as g:
        g.set_tier_config(nido_lib.TierConfig(192, 768, 1024, 1024, ctax, 1, 4 << 20))
        assert g.tier_config().hub_clusters == 1
        cl, st = g.run()
    assert st.phases == st_o.phases and st.total_loops == st_o.total_loops
    assert np.array_equal(np.array(st.q_phase[: st.phases]), np.array(st_o.q_phase[: st_o.phases]))
    assert np.array_equal(cl, want)


@pytest.mark.parametrize("tie", [0, 1])
def test_staged_edges_same_result(nido_lib, ctx, rmat16, tie):
    """The CTA-S and CTA-M tiers with their edges staged in shared memory by
    bulk copies give the same partitions as the unstaged default."""
    with nido_lib.Graph(ctx, rmat16, 2) as g:
        want, st0 = g.run(tie=tie)
        c = g.tier_config()
        assert c.staged_edges == 0
        c.staged_edges = 1
        g.set_tier_config(c)
        assert g.tier_config().staged_edges == 1
        got, st = g.run(tie=tie)
    assert np.array_equal(got, want) and st.final_q == st0.final_q
