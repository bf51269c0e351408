"""Programs written against the reference's classes, built on this library.

* tests/dropin/replay_main: this repository's program with the reference's
  header names (include/nido_compat), classes, signatures and the call
  sequence of the reference's main (Graph(file), coloring(), GraphGPU(graph,
  nbatches, 1, 1), LouvainGPU(maxLoops, tau, nbatches), run, dump_partition);
  with -s it drives the phase loop through GraphGPU's step methods instead.
* oracle/_ref/ref_main_on_nido_b200: the reference's own main.cpp, unchanged,
  compiled against the same headers and linked with libnido_b200.so only
  (built by oracle/Makefile.ref where the reference sources are present).

Every -o file must equal the CPU oracle's partition bit for bit (integer
weights); with -c, the oracle runs on the same colouring's relabelled CSR and
its partition is mapped back through new_orders.
"""
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu

REPLAY = os.path.join(ROOT, "tests", "dropin", "_build", "replay_main")
REF_MAIN = os.path.join(ROOT, "oracle", "_ref", "ref_main_on_nido_b200")


def read_partition(path):
    with open(path, "rb") as f:
        return np.array(f.read().split(), dtype=np.int64)


@pytest.fixture(scope="module")
def graph_file(nido_lib, tmp_path_factory):
    G = nido_lib.gen_rmat(1 << 13, 10 << 13, wmode=nido_lib.W_INT8, seed=21)
    p = str(tmp_path_factory.mktemp("dropin") / "g.bin")
    nido_lib.write_vite(p, G)
    return G, p


def run(prog, *args):
    r = subprocess.run([prog, *args], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    return r.stdout


def oracle_partition(orc, ctx, G, nb, colored):
    if not colored:
        return orc.louvain(G.off, G.adj, G.w, nbatches=nb)[0]
    colors, _ = ctx.color(G)  # the device colouring the program's coloring() uses (seed 1)
    new_orders, (off, adj, w) = orc.color_relabel(G.off, G.adj, G.w, colors)
    cl = orc.louvain(off, adj, w, nbatches=nb)[0]
    out = np.empty_like(cl)
    out[new_orders] = cl
    return out


@pytest.mark.parametrize("nb", [1, 2, 3])
@pytest.mark.parametrize("steps", [False, True])
def test_replay_main_equals_oracle(graph_file, orc, ctx, tmp_path, nb, steps):
    assert os.path.exists(REPLAY), "tests/dropin/replay_main is not built (make -C tests/dropin)"
    G, path = graph_file
    out = str(tmp_path / "p.txt")
    args = ["-f", path, "-b", str(nb), "-o", out] + (["-s"] if steps else [])
    text = run(REPLAY, *args)
    assert f"#Batches: {nb}" in text and f"Number of vertices: {G.nv}" in text
    assert np.array_equal(read_partition(out), oracle_partition(orc, ctx, G, nb, False))


def test_replay_main_colored(graph_file, orc, ctx, tmp_path):
    G, path = graph_file
    out = str(tmp_path / "pc.txt")
    run(REPLAY, "-f", path, "-c", "-o", out)
    assert np.array_equal(read_partition(out), oracle_partition(orc, ctx, G, 2, True))


@pytest.mark.skipif(not os.path.exists(REF_MAIN), reason="reference sources absent when the tree was built")
@pytest.mark.parametrize("extra,nb,colored", [([], 2, False), (["-b", "3"], 3, False), (["-c"], 2, True)])
def test_reference_main_on_this_library(graph_file, orc, ctx, tmp_path, extra, nb, colored):
    G, path = graph_file
    out = str(tmp_path / "pr.txt")
    text = run(REF_MAIN, "-f", path, "-o", out, *extra)
    for line in (f"#Batches: {nb}", "#Threshold: 1e-06", "Max #iterations: 500", "#NGPUs: 1",
                 "PHASE #0:", "Final Q:", "Total time elapse:"):
        assert line in text
    assert np.array_equal(read_partition(out), oracle_partition(orc, ctx, G, nb, colored))
