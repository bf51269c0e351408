"""nido_modularity_noalloc: modularity from caller-owned device arrays with no
memory allocation, for callers that cannot call cudaMalloc (a stream being
captured into a CUDA graph, an allocator callback, a process whose device
memory is all given to a fixed pool).

The entry point keeps its partial sums in a fixed array inside the library
that every call shares, so two calls in a row must each return the value the
allocating entry point (nido_compute_modularity) returns for its own inputs:
bit for bit on integer weights, within 1e-12 relative otherwise (the
tolerance of the engine's other modularity tests).  This file is collected
last; it runs alone or after the other tests.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _reference_q(capi, ctx, G, comm):
    """Q, community degrees and mass from the allocating entry points."""
    with capi.Graph(ctx, G, 1) as g:
        g.set_community_ids(comm)
        _, _, a = g.state()
        _, m = g.vertex_weights()
        return g.compute_modularity(), a, m


@pytest.mark.parametrize("wmode,exact", [(3, True), (2, False)])
def test_noalloc_matches_allocating_entry_point(nido_lib, ctx, orc, wmode, exact):
    import torch

    capi = nido_lib
    if wmode == 3:
        G = capi.gen_rmat(1 << 15, 12 << 15, wmode=capi.W_INT8, seed=41)
    else:
        G = capi.gen_sbm(60000, cmin=16, cmax=2048, avg_degree=16.0, wmode=capi.W_LOGNORMAL, seed=42)
    rng = np.random.default_rng(7)
    dev = torch.device("cuda", 0)
    d_off = torch.from_numpy(G.off).to(dev)
    d_adj = torch.from_numpy(G.adj).to(dev)
    d_w = torch.from_numpy(G.w).to(dev)
    d_q = torch.zeros(1, dtype=torch.float64, device=dev)
    for call in range(2):  # two calls in a row share the library's scratch array
        comm = rng.integers(0, max(2, G.nv // (8 + 24 * call)), G.nv).astype(np.int64)
        q_ref, a, m = _reference_q(capi, ctx, G, comm)
        d_comm = torch.from_numpy(comm).to(dev)
        d_a = torch.from_numpy(a).to(dev)
        torch.cuda.synchronize()
        st = capi.lib().nido_modularity_noalloc(
            None, G.nv, C.c_void_p(d_off.data_ptr()), C.c_void_p(d_adj.data_ptr()), C.c_void_p(d_w.data_ptr()),
            C.c_void_p(d_comm.data_ptr()), C.c_void_p(d_a.data_ptr()), m, C.c_void_p(d_q.data_ptr()))
        assert st == 0, capi.lib().nido_last_error()
        torch.cuda.synchronize()
        q = float(d_q.item())
        # and directly against the CPU oracle's modularity of the same inputs
        q_orc = orc.modularity(G.off, G.adj, G.w, comm, a, m)
        if exact:
            assert np.float64(q).view(np.uint64) == np.float64(q_ref).view(np.uint64), (call, q, q_ref)
            assert np.float64(q).view(np.uint64) == np.float64(q_orc).view(np.uint64), (call, q, q_orc)
        else:
            assert abs(q - q_ref) <= 1e-12 * abs(q_ref), (call, q, q_ref)
            assert abs(q - q_orc) <= 1e-12 * abs(q_orc), (call, q, q_orc)


def test_noalloc_graph_without_edges(nido_lib, ctx):
    """Four isolated vertices: Q = 0.  The argument checks (null arrays, too
    many vertices) are tested without a GPU in test_host.py, so no call here
    hands the kernels a pointer they may not read."""
    import torch

    lib = nido_lib.lib()
    dev = torch.device("cuda", 0)
    nv = 4
    off = torch.zeros(nv + 1, dtype=torch.int64, device=dev)
    adj = torch.zeros(1, dtype=torch.int64, device=dev)
    w = torch.zeros(1, dtype=torch.float64, device=dev)
    comm = torch.arange(nv, dtype=torch.int64, device=dev)
    a = torch.zeros(nv, dtype=torch.float64, device=dev)
    q = torch.full((1,), 7.0, dtype=torch.float64, device=dev)
    p = lambda t: C.c_void_p(t.data_ptr())  # noqa: E731
    torch.cuda.synchronize()
    assert lib.nido_modularity_noalloc(None, nv, p(off), p(adj), p(w), p(comm), p(a), 1.0, p(q)) == 0
    torch.cuda.synchronize()
    assert float(q.item()) == 0.0
