"""Colour-class batches (nido_params.color_batches, CLI --color-batches):
every phase colours its graph on the device (Jones-Plassmann-Luby, seed 1)
and sweeps the colour classes in colour order, one class per batch, so no two
neighbours move in the same batch.  The oracle runs the same colouring
(orc_color_jpl) and the same batches, so on integer weights every colouring,
partition, per-phase Q and loop count is bit-exact."""
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu
CLI = os.path.join(ROOT, "nido_b200", "bin", "nido_louvain")


def graphs(capi):
    return {
        "planted_int": capi.gen_planted(96, 96, 16.0, 0.8, capi.W_INT8, 7),
        "rmat_s13_int": capi.gen_rmat(1 << 13, 12 << 13, wmode=capi.W_INT8, seed=8),
        "sbm_int": capi.gen_sbm(20000, cmin=16, cmax=2048, avg_degree=16.0, wmode=capi.W_INT8, seed=9),
        "rmat_s15_unit": capi.gen_rmat(1 << 15, 16 << 15, wmode=capi.W_ONE, seed=10),
    }


@pytest.fixture(scope="module")
def gs(nido_lib):
    return graphs(nido_lib)


def bits(x):
    return np.asarray(x, np.float64).view(np.uint64)


@pytest.mark.parametrize("gname", ["planted_int", "rmat_s13_int", "sbm_int", "rmat_s15_unit"])
def test_device_colouring_equals_oracle(nido_lib, ctx, orc, gs, gname):
    G = gs[gname]
    colors, nc = ctx.color(G, seed=1)
    want, nc_o = orc.color_jpl(G.off, G.adj, seed=1)
    assert nc == nc_o and np.array_equal(colors, want)
    src = np.repeat(np.arange(G.nv), np.diff(G.off))
    assert np.all((src == G.adj) | (colors[src] != colors[G.adj]))  # proper: classes are conflict-free


@pytest.mark.parametrize("gname", ["planted_int", "rmat_s13_int", "sbm_int", "rmat_s15_unit"])
@pytest.mark.parametrize("tie", [0, 1])
@pytest.mark.parametrize("host_loop", [False, True])
def test_color_batch_runs_equal_oracle(nido_lib, ctx, orc, gs, gname, tie, host_loop):
    G = gs[gname]
    want, st_o = orc.louvain(G.off, G.adj, G.w, nbatches=2, tie=tie, color_batches=True)
    with nido_lib.Graph(ctx, G, 2) as g:
        cl, st = g.run(tie=tie, color_batches=True, host_loop=host_loop)
        with pytest.raises(nido_lib.NidoError):
            g.batches()  # colour classes are not vertex ranges
        # the next run without the option is the ordinary -b run again
        cl_b, st_b = g.run(tie=tie, host_loop=host_loop)
        assert len(g.batches()) == 3
    assert st.phases == st_o.phases and st.total_loops == st_o.total_loops
    assert np.array_equal(bits(st.q_phase[: st.phases]), bits(st_o.q_phase[: st_o.phases]))
    assert np.array_equal(cl, want)
    want_b, st_ob = orc.louvain(G.off, G.adj, G.w, nbatches=2, tie=tie)
    assert np.array_equal(cl_b, want_b) and bits(st_b.final_q) == bits(st_ob.final_q)


def test_color_batches_cli(nido_lib, orc, gs, tmp_path):
    G = gs["rmat_s13_int"]
    path = str(tmp_path / "g.bin")
    out = str(tmp_path / "p.txt")
    nido_lib.write_vite(path, G)
    r = subprocess.run([CLI, "-f", path, "--color-batches", "-o", out], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    with open(out, "rb") as f:
        got = np.array(f.read().split(), dtype=np.int64)
    want, _ = orc.louvain(G.off, G.adj, G.w, nbatches=2, color_batches=True)
    assert np.array_equal(got, want)


def test_color_batches_refused_for_graph_sets(nido_lib, ctx, gs):
    with nido_lib.Batch(ctx, [gs["planted_int"], gs["rmat_s13_int"]], 2) as b:
        p = nido_lib._Params(2, 0, 1e-6, 500, 0, 0, 0.0, 0, 0, 1)
        import ctypes as C
        import numpy as np_
        out = np_.empty(b.nv, np_.int64)
        st = nido_lib.lib().nido_batch_run(b.h, C.byref(p), out.ctypes.data_as(C.POINTER(C.c_int64)), None, None,
                                           None, None)
        assert st == -1  # NIDO_E_INVALID
