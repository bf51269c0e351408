"""The drop-in command line on a GPU: `nido_louvain -f graph.bin -o out` reads
the Vite file (streamed to the device), prints the reference's lines and
writes one "%lld\\n" community id per vertex -- on integer weights exactly the
oracle's partition; `-c` takes the colouring path through the host CSR."""
import os
import re
import subprocess

import numpy as np
import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu

CLI = os.path.join(ROOT, "nido_b200", "bin", "nido_louvain")


def run_cli(*args):
    r = subprocess.run([CLI, *args], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    return r.stdout


def read_partition(path):
    with open(path) as f:
        return np.array([int(x) for x in f.read().split()], np.int64)


@pytest.fixture(scope="module")
def graph_file(nido_lib, tmp_path_factory):
    G = nido_lib.gen_planted(64, 96, 12.0, 0.8, nido_lib.W_INT8, 5)
    p = str(tmp_path_factory.mktemp("cli") / "g.bin")
    nido_lib.write_vite(p, G)
    return G, p


@pytest.mark.parametrize("nb", [1, 2])
def test_cli_partition_equals_oracle(graph_file, orc, tmp_path, nb):
    G, path = graph_file
    out = str(tmp_path / "part.txt")
    text = run_cli("-f", path, "-b", str(nb), "-o", out)
    for line in (f"#Batches: {nb}", "#Threshold: 1e-06", "Max #iterations: 500", f"Number of vertices: {G.nv}",
                 f"Number of edges: {G.ne}", "PHASE #0:", "Total time elapse:"):
        assert line in text
    want, st = orc.louvain(G.off, G.adj, G.w, nbatches=nb)
    got = read_partition(out)
    assert np.array_equal(got, want)
    finals = [float(x) for x in re.findall(r"Final Q: (\S+)", text)]
    assert abs(finals[-1] - st.final_q) <= 1e-5  # printed with %g


def test_cli_header_mismatch_warns(graph_file, tmp_path):
    G, path = graph_file
    raw = bytearray(open(path, "rb").read())
    raw[8:16] = np.int64(G.ne + 7).tobytes()  # header edge count disagrees with the offsets
    p2 = str(tmp_path / "g2.bin")
    open(p2, "wb").write(bytes(raw))
    text = run_cli("-f", p2, "-o", str(tmp_path / "p.txt"))
    assert "!!! The graph has been modified in edges" in text
    assert f"New edges: {G.ne}" in text


def test_cli_colored_path(graph_file, orc, tmp_path):
    G, path = graph_file
    out = str(tmp_path / "part_c.txt")
    text = run_cli("-f", path, "-c", "-o", out)
    assert "Coloring Time:" in text
    part = read_partition(out)
    assert len(part) == G.nv and part.min() == 0
    u = np.unique(part)
    assert u[-1] == len(u) - 1  # dense ids
    finals = [float(x) for x in re.findall(r"Final Q: (\S+)", text)]
    q = orc.partition_modularity(G.off, G.adj, G.w, part)
    assert abs(q - finals[-1]) <= 1e-5
