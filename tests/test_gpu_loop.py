"""The device-resident iteration loop (one CUDA graph with a conditional while
node per phase, loop.cu; per batched sweep loop, batch.cu) against the host-
driven loop of the reference's shape (one Q readback per iteration).

Both loops run the same kernels in the same order, so on integer weights
every partition, every phase's Q and every loop count are identical; with
FP64 weights the commit's atomics may add in another order, so runs are held
to the run-level tolerance (final Q within 1e-3, NMI >= 0.95).  The verbose
per-loop lines (the reference's `LOOP# Q dQ` table) are the same text."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def graphs(capi):
    return {
        "planted_int": capi.gen_planted(128, 128, 24.0, 0.8, capi.W_INT8, 3),
        "rmat_s14_int": capi.gen_rmat(1 << 14, 16 << 14, wmode=capi.W_INT8, seed=31),
        "rmat_s16_unit": capi.gen_rmat(1 << 16, 16 << 16, wmode=capi.W_ONE, seed=32),
        "sbm_int": capi.gen_sbm(40000, cmin=16, cmax=4096, avg_degree=24.0, wmode=capi.W_INT8, seed=33),
    }


@pytest.fixture(scope="module")
def gs(nido_lib):
    return graphs(nido_lib)


def bits(x):
    return np.asarray(x, np.float64).view(np.uint64)


@pytest.mark.parametrize("gname", ["planted_int", "rmat_s14_int", "rmat_s16_unit", "sbm_int"])
@pytest.mark.parametrize("nb,tie", [(1, 0), (2, 0), (2, 1), (3, 1)])
def test_device_loop_equals_host_loop(nido_lib, ctx, gs, gname, nb, tie):
    G = gs[gname]
    with nido_lib.Graph(ctx, G, nb) as g:
        cd, sd = g.run(tie=tie, device_loop=True)
        ch, sh = g.run(tie=tie, host_loop=True)
    assert np.array_equal(cd, ch)
    assert sd.phases == sh.phases and sd.total_loops == sh.total_loops
    n = sd.phases
    assert np.array_equal(bits(sd.q_phase[:n]), bits(sh.q_phase[:n]))
    assert list(sd.loops_phase[:n]) == list(sh.loops_phase[:n])
    assert bits(sd.final_q) == bits(sh.final_q)
    assert sd.move_ms > 0 and sd.q_ms > 0
    # the same algorithmic work is counted either way
    assert sd.move_bytes == sh.move_bytes and sd.edges_scanned == sh.edges_scanned


@pytest.mark.parametrize("max_iter,tau", [(0, 1e-6), (1, 1e-6), (2, 1e-6), (500, 1e-2), (3, -1.0)])
def test_device_loop_limits(nido_lib, ctx, gs, max_iter, tau):
    """Loop caps and thresholds end the loop where the host loop ends it (a
    negative tau keeps iterating until the cap, undo steps included)."""
    G = gs["rmat_s14_int"]
    with nido_lib.Graph(ctx, G, 2) as g:
        cd, sd = g.run(tau=tau, max_iter=max_iter, device_loop=True)
        ch, sh = g.run(tau=tau, max_iter=max_iter, host_loop=True)
    assert np.array_equal(cd, ch)
    assert sd.phases == sh.phases and sd.total_loops == sh.total_loops
    assert bits(sd.final_q) == bits(sh.final_q)
    assert all(sd.loops_phase[p] <= max(max_iter, 0) for p in range(sd.phases))


def test_device_loop_lognormal_within_tolerance(nido_lib, ctx, orc):
    G = nido_lib.gen_sbm(30000, cmin=16, cmax=2048, avg_degree=20.0, wmode=nido_lib.W_LOGNORMAL, seed=34)
    with nido_lib.Graph(ctx, G, 2) as g:
        cd, sd = g.run(device_loop=True)
        ch, sh = g.run(host_loop=True)
    assert abs(sd.final_q - sh.final_q) <= 1e-3
    assert orc.nmi(cd, ch) >= 0.95


def test_device_loop_prints_the_reference_lines(nido_lib, ctx, gs, capfd):
    G = gs["planted_int"]
    with nido_lib.Graph(ctx, G, 2) as g:
        capfd.readouterr()
        g.run(verbose=True, device_loop=True)
        dev = capfd.readouterr().out
        g.run(verbose=True, host_loop=True)
        host = capfd.readouterr().out
    assert dev == host
    assert "PHASE #0:" in dev and "LOOP# \tQ \t\tdQ" in dev and "Final Q:" in dev
    assert dev.count("\n1 \t") >= 1  # the first iteration's line of every phase


@pytest.mark.parametrize("nb,tie", [(1, 0), (2, 1)])
def test_batched_device_loop_equals_host_loop(nido_lib, ctx, gs, nb, tie):
    rng = np.random.default_rng(35)
    many = list(gs.values()) + [
        nido_lib.gen_rmat(1 << int(s), int(d) << int(s), wmode=nido_lib.W_INT8, seed=400 + i)
        for i, (s, d) in enumerate(zip(rng.integers(6, 12, 12), rng.integers(4, 20, 12)))]
    with nido_lib.Batch(ctx, many, nb) as b:
        pd, qd, phd, lod, sd = b.run(tie=tie, device_loop=True)
        ph_, qh, phh, loh, sh = b.run(tie=tie, host_loop=True)
    for x, y in zip(pd, ph_):
        assert np.array_equal(x, y)
    assert np.array_equal(bits(qd), bits(qh))
    assert np.array_equal(phd, phh) and np.array_equal(lod, loh)
    assert sd.total_loops == sh.total_loops and sd.move_bytes == sh.move_bytes
    # far fewer host round trips: the device loop launches its sweeps as graphs
    assert sd.move_ms > 0


def test_default_is_the_host_loop(nido_lib, ctx, gs):
    """With neither option the host drives the iterations (measured the faster
    on B200: the loop graphs cost more to build than the round trips they
    save); the loop graphs' build time shows which ran.  Results do not
    depend on it, for one graph and for graph sets."""
    small = gs["rmat_s14_int"]
    with nido_lib.Graph(ctx, small, 2) as g:
        cl, st = g.run()
        assert st.host_ms[7] == 0  # no loop graph was built
        cd, sd = g.run(device_loop=True)
        assert sd.host_ms[7] > 0 and np.array_equal(cl, cd) and st.final_q == sd.final_q
    with nido_lib.Batch(ctx, list(gs.values()), 2) as b:
        p0, q0, _, _, s0 = b.run()
        p1, q1, _, _, s1 = b.run(device_loop=True)
    assert s0.host_ms[7] == 0 and s1.host_ms[7] > 0
    assert all(np.array_equal(x, y) for x, y in zip(p0, p1)) and np.array_equal(bits(q0), bits(q1))
