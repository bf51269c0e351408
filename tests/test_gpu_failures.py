"""Bounded device waits end with an error status instead of hanging: a kernel
waits on an mbarrier nothing arrives at (the wait of the staged move tiers,
bounded by an attempt count and about a second of %globaltimer), gives up and
reports it through the C ABI; the context then runs a graph as before.  No
test here faults, traps or hangs a GPU."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_bounded_wait_gives_up_and_context_stays_usable(nido_lib, ctx, orc):
    gave_up, ms = ctx.check_bounded_wait()
    assert gave_up and 0 <= ms <= 5000
    G = nido_lib.gen_planted(32, 64, 12.0, 0.8, nido_lib.W_INT8, 61)
    with nido_lib.Graph(ctx, G, 2) as g:
        cl, st = g.run()
    want, st_o = orc.louvain(G.off, G.adj, G.w, nbatches=2)
    assert np.array_equal(cl, want) and st.final_q == st_o.final_q
