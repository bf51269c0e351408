"""Whole runs at the benchmark configurations' full size, against runs of the
unmodified reference recorded on a B200 (tests/golden/configs/*.json, made by
`tests/golden/make_ref_fixtures.py --configs c1,c2`) and against the CPU
oracle.

  c1  planted partition, 65,536 vertices, weights U[0.5,1.5], -b 1: the
      e_vc sums are not exact in FP64, so the bar is the run-level one:
      final Q within 1e-3 of the reference's and NMI >= 0.95 against the
      reference's partition.
  c2  R-MAT scale 22, unit weights, -b 2: every sum is exact, so under the
      reference's tie rule every phase's final Q, every phase's loop count
      and the partition file (sha256) equal the reference's bit for bit;
      under the default smallest-id rule the final Q equals the CPU oracle's
      whole run bit for bit.
  c3  SBM 16,777,216 vertices, lognormal weights, -b 32: when the reference
      program has been built (oracle/_ref/run_1_100), it runs here on the
      same file: final Q within 1e-3 and NMI >= 0.95.
"""
import hashlib
import json
import os
import re
import shutil
import subprocess
import tempfile

import numpy as np
import pytest

from conftest import GOLDEN, ROOT

pytestmark = pytest.mark.gpu
CONFIGS = os.path.join(GOLDEN, "configs")
REFBIN = os.path.join(ROOT, "oracle", "_ref", "run_1_100")


def load_config(name):
    path = os.path.join(CONFIGS, name + ".json")
    if not os.path.exists(path):
        pytest.fail(f"{path} is missing: record it with tests/golden/make_ref_fixtures.py --configs {name}")
    with open(path) as f:
        return json.load(f)


@pytest.fixture(scope="module")
def c2_graph(nido_lib):
    from nido_b200 import workloads
    return workloads.single_graph("rmat22")


def test_c1_vs_reference(nido_lib, ctx, orc):
    from nido_b200 import workloads
    rec = load_config("c1")
    g = workloads.single_graph("planted")
    assert (g.nv, g.ne) == (rec["nv"], rec["ne"])
    ref_part = np.load(os.path.join(CONFIGS, "c1_partition.npz"))["partition"]
    ref_q = float(rec["phases"][-1]["final_q"])
    with nido_lib.Graph(ctx, g, rec["nbatches"]) as dg:
        for tie in (nido_lib.NIDO_TIE_NIDO, nido_lib.NIDO_TIE_SMALLEST_ID):
            cl, st = dg.run(tau=rec["tau"], max_iter=rec["max_iter"], tie=tie)
            assert abs(st.final_q - ref_q) <= 1e-3, (st.final_q, ref_q)
            assert orc.nmi(cl, ref_part) >= 0.95
            # the returned partition's own modularity is the reported Q
            assert abs(orc.partition_modularity(g.off, g.adj, g.w, cl) - st.final_q) <= 1e-9


def test_c2_vs_reference_bit_exact(nido_lib, ctx, c2_graph, tmp_path):
    rec = load_config("c2")
    g = c2_graph
    assert (g.nv, g.ne) == (rec["nv"], rec["ne"])
    with nido_lib.Graph(ctx, g, rec["nbatches"]) as dg:
        _, st = dg.run(tau=rec["tau"], max_iter=rec["max_iter"], tie=nido_lib.NIDO_TIE_NIDO)
        ph = rec["phases"]
        assert st.phases == len(ph)
        for p, rp in enumerate(ph):
            assert st.q_phase[p] == float(rp["final_q"]), (p, st.q_phase[p], rp["final_q"])
            assert st.loops_phase[p] == len(rp["loop_q"]), (p, st.loops_phase[p], len(rp["loop_q"]))
        out = str(tmp_path / "c2_part.txt")
        dg.dump_partition(out)
        with open(out, "rb") as f:
            assert hashlib.sha256(f.read()).hexdigest() == rec["partition_sha256"]


def test_c2_default_rule_vs_oracle(nido_lib, ctx, orc, c2_graph):
    g = c2_graph
    with nido_lib.Graph(ctx, g, 2) as dg:
        cl, st = dg.run(tau=1e-6, max_iter=500)
    want, st_o = orc.louvain(g.off, g.adj, g.w, nbatches=2, tau=1e-6)
    assert st.final_q == st_o.final_q
    assert st.phases == st_o.phases and st.total_loops == st_o.total_loops
    assert np.array_equal(cl, want)


def _ref_final_qs(out):
    return [float(x) for x in re.findall(r"Final Q: (\S+)", out)]


@pytest.mark.skipif(not os.path.exists(REFBIN), reason="reference program not built (oracle/Makefile.ref)")
def test_c3_vs_reference_program(nido_lib, ctx, orc):
    from nido_b200 import workloads
    g = workloads.single_graph("sbm")
    tmp = tempfile.mkdtemp()
    try:
        need = 16 * g.ne + 8 * g.nv + 64
        if shutil.disk_usage(tmp).free < 3 * need:
            pytest.skip("not enough scratch disk for the C3 Vite file")
        path = os.path.join(tmp, "c3.bin")
        part = os.path.join(tmp, "c3_part.txt")
        nido_lib.write_vite(path, g)
        r = subprocess.run([REFBIN, "-f", path, "-b", "32", "-o", part], capture_output=True, text=True,
                           timeout=900)
        assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
        ref_q = _ref_final_qs(r.stdout)[-1]
        with open(part, "rb") as f:
            ref_part = np.array(f.read().split(), dtype=np.int64)
    finally:
        shutil.rmtree(tmp, ignore_errors=True)
    with nido_lib.Graph(ctx, g, 32) as dg:
        cl, st = dg.run(tau=1e-6, max_iter=500)
    assert len(ref_part) == g.nv
    assert abs(st.final_q - ref_q) <= 1e-3, (st.final_q, ref_q)
    assert orc.nmi(cl, ref_part) >= 0.95
