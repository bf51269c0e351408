"""Host-side pieces that need no GPU: the C ABI's exported symbols, Vite
files, the generators, graph packing for batched runs, the command line's
option handling, and the replica plumbing of bench.py over gloo."""
import ctypes as C
import os
import re
import socket
import subprocess

import numpy as np
import pytest

from conftest import ROOT, load_golden

HEADER = os.path.join(ROOT, "include", "nido_b200.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(nido_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol(nido_lib):
    names = declared_functions()
    assert len(names) >= 40
    L = C.CDLL(nido_lib.LIB_PATH)
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing
    assert nido_lib.lib().nido_version().decode()


def test_no_device_is_an_error_not_a_fallback(nido_lib):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(nido_lib.NidoError) as e:
        nido_lib.Context(0)
    assert e.value.code == -7  # NIDO_E_NODEVICE


def test_noalloc_argument_checks_without_a_device(nido_lib):
    """nido_modularity_noalloc checks its arguments before any CUDA call, so
    the refusals are tested here, where no GPU exists and no pointer can be
    dereferenced: a negative size, each missing array once there are
    vertices, and more vertices than the fixed scratch array covers."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present: argument refusals are tested only where no kernel can run")
    lib = nido_lib.lib()
    fake = [C.c_void_p(0x1000 * (i + 1)) for i in range(6)]  # never dereferenced: no device here
    assert lib.nido_modularity_noalloc(None, -1, *fake[:5], 1.0, fake[5]) == -1
    for missing in range(6):
        args = list(fake)
        args[missing] = None
        assert lib.nido_modularity_noalloc(None, 4, *args[:5], 1.0, args[5]) == -1, missing
    st = lib.nido_modularity_noalloc(None, (1 << 31) + 5, *fake[:5], 1.0, fake[5])
    assert st == -5 and b"exceed" in lib.nido_last_error()


def test_vite_round_trip_and_errors(nido_lib, tmp_path):
    d = load_golden("selfloop_int")
    g = nido_lib.Csr(d["off"], d["adj"], d["w"])
    p = str(tmp_path / "g.bin")
    nido_lib.write_vite(p, g)
    h = nido_lib.read_vite(p)
    assert np.array_equal(h.off, g.off) and np.array_equal(h.adj, g.adj) and np.array_equal(h.w, g.w)
    # header (nv, ne) then (nv+1) offsets, ne (tail, weight) records
    raw = open(p, "rb").read()
    assert len(raw) == 16 + 8 * (g.nv + 1) + 16 * g.ne
    open(p, "wb").write(raw[: len(raw) - 8])
    with pytest.raises(nido_lib.NidoError):
        nido_lib.read_vite(p)
    with pytest.raises(nido_lib.NidoError):
        nido_lib.read_vite(str(tmp_path / "missing.bin"))


@pytest.mark.parametrize("kind", ["planted", "rmat", "sbm"])
def test_generators_symmetric_and_seeded(nido_lib, kind):
    c = nido_lib
    make = {
        "planted": lambda s: c.gen_planted(16, 32, 8.0, 0.8, c.W_INT8, s),
        "rmat": lambda s: c.gen_rmat(1 << 10, 8 << 10, wmode=c.W_ONE, seed=s),
        "sbm": lambda s: c.gen_sbm(3000, cmin=16, cmax=256, avg_degree=10.0, wmode=c.W_LOGNORMAL, seed=s),
    }[kind]
    g, g2, g3 = make(7), make(7), make(8)
    assert np.array_equal(g.adj, g2.adj) and np.array_equal(g.w, g2.w)
    assert not (g.ne == g3.ne and np.array_equal(g.adj, g3.adj))
    src = np.repeat(np.arange(g.nv), np.diff(g.off))
    fwd = dict(zip(zip(src.tolist(), g.adj.tolist()), g.w.tolist()))
    assert all(fwd.get((v, u)) == w for (u, v), w in fwd.items())  # symmetric with equal weights
    assert (g.adj != src).all() or kind != "rmat"  # R-MAT drops self-loops
    for v in range(g.nv):  # sorted, no duplicates
        row = g.adj[g.off[v]:g.off[v + 1]]
        assert (np.diff(row) > 0).all()


def test_pack_graphs_layout(nido_lib):
    c = nido_lib
    a = c.gen_planted(4, 8, 4.0, 0.8, c.W_INT8, 1)
    b = c.Csr(np.zeros(1, np.int64), np.zeros(0, np.int64), np.zeros(0))
    d = c.gen_rmat(64, 256, wmode=c.W_ONE, seed=3)
    vbase, u = c.pack_graphs([a, b, d])
    assert vbase.tolist() == [0, a.nv, a.nv, a.nv + d.nv]
    assert u.nv == a.nv + d.nv and u.ne == a.ne + d.ne
    assert np.array_equal(u.off[: a.nv + 1], a.off)
    assert np.array_equal(u.off[a.nv:] - a.ne, d.off)
    assert np.array_equal(u.adj[a.ne:] - a.nv, d.adj)
    src = np.repeat(np.arange(u.nv), np.diff(u.off))
    g_of = np.searchsorted(vbase, src, side="right") - 1
    assert (u.adj >= vbase[g_of]).all() and (u.adj < vbase[g_of + 1]).all()


CLI = os.path.join(ROOT, "nido_b200", "bin", "nido_louvain")


@pytest.mark.skipif(not os.path.exists(CLI), reason="command-line program not built")
def test_cli_options():
    r = subprocess.run([CLI, "-h"], capture_output=True, text=True)
    assert r.returncode == 0 and "-f" in r.stdout
    r = subprocess.run([CLI, "-r", "100"], capture_output=True, text=True)
    assert r.returncode != 0 and "not supported" in r.stderr
    r = subprocess.run([CLI], capture_output=True, text=True)
    assert r.returncode != 0 and "missing" in r.stderr
    r = subprocess.run([CLI, "-f", "/nonexistent.bin"], capture_output=True, text=True)
    assert r.returncode != 0


def test_package_cli_options():
    """python -m nido_b200: one of --file / --workload / --many is required, and
    the batched many-graph run is offered."""
    import sys
    r = subprocess.run([sys.executable, "-m", "nido_b200", "--help"], capture_output=True, text=True, cwd=ROOT)
    assert r.returncode == 0 and "--many" in r.stdout and "--many-edges" in r.stdout
    r = subprocess.run([sys.executable, "-m", "nido_b200"], capture_output=True, text=True, cwd=ROOT)
    assert r.returncode != 0 and "one of the arguments" in r.stderr


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _replica_worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world),
                      RANK=str(rank), LOCAL_RANK=str(rank))
    import sys
    sys.path.insert(0, ROOT)
    import bench
    w, r, _ = bench.dist_setup(None)
    bench.barrier(w)
    mx = bench.reduce_max(10.0 + r, w)
    import torch.distributed as dist
    dist.destroy_process_group()
    q.put((r, w, mx))


def test_bench_replica_plumbing_gloo():
    """bench.py --gpus 2 runs independent replicas: ranks meet only at the
    barrier and the max-over-ranks of the timed region."""
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_replica_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    for p in ps:
        p.join(120)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=10) for _ in range(2))
    assert got == [(0, 2, 11.0), (1, 2, 11.0)]


def test_many_graph_plan_rule():
    """4,096 graphs, log-uniform sizes scaled so the drawn directed edges total
    1.5e9 (clamped at 100 vertices), 50/50 SBM / R-MAT, degrees in [8, 64]."""
    from nido_b200 import workloads as W
    V, d, kind = W.many_graph_plan()
    assert len(V) == 4096 and V.min() >= 100
    assert (d >= 8).all() and (d <= 64).all()
    assert 0.45 < kind.mean() < 0.55
    assert abs((V * d).sum() / 1.5e9 - 1) < 0.02  # clamping adds a little
    V2, _, _ = W.many_graph_plan(max_edges=1e15)  # no scaling: the drawn law itself
    lv = np.log10(V2)
    assert 2.0 <= lv.min() and lv.max() <= 6.0 and abs(lv.mean() - 4.0) < 0.1
    assert np.array_equal(W.many_graph_plan()[0], V)  # seeded


def test_serving_requests_law():
    from nido_b200 import workloads as W
    t, V, kind = W.serving_requests(4000, rate=10.0)
    gaps = np.diff(np.concatenate([[0.0], t]))
    assert abs(gaps.mean() - 0.1) < 0.01 and abs(gaps.std() - 0.1) < 0.01  # exponential
    lv = np.log10(V)
    assert 3.0 <= lv.min() and lv.max() <= 7.0 and abs(lv.mean() - 5.0) < 0.1


def test_many_graphs_packed_small(nido_lib):
    from nido_b200 import workloads as W
    vbase, u, (V, d, kind) = W.many_graphs_packed(24, max_edges=2e5)
    assert vbase[-1] == u.nv and len(vbase) == 25 and np.array_equal(np.diff(vbase), V)
    src = np.repeat(np.arange(u.nv), np.diff(u.off))
    g_of = np.searchsorted(vbase, src, side="right") - 1
    assert (u.adj >= vbase[g_of]).all() and (u.adj < vbase[g_of + 1]).all()
    assert (u.w >= 1).all() and (u.w == np.round(u.w)).all()  # integer weights (duplicates summed)
    g5 = W.unpack(vbase, u, 5)
    assert g5.nv == V[5] and g5.off[0] == 0 and (g5.adj < V[5]).all()


_CTYPES = {"int64_t": "c_long", "int32_t": "c_int", "double": "c_double", "uint64_t": "c_ulong"}


def header_structs():
    """Field (name, C type, array length) lists of the header's typedef structs."""
    text = re.sub(r"/\*.*?\*/", "", open(HEADER).read(), flags=re.S)
    out = {}
    for body, name in re.findall(r"typedef struct \{(.*?)\}\s*(nido_\w+);", text, flags=re.S):
        fields = []
        for decl in body.split(";"):
            m = re.match(r"\s*(const\s+)?(\w+)\s*(\*?)\s*(\w+)\s*(\[(\d+)\])?\s*$", decl)
            if m:
                ctype = "pointer" if m.group(3) else m.group(2)
                fields.append((m.group(4), ctype, int(m.group(6)) if m.group(6) else 0))
        out[name] = fields
    return out


@pytest.mark.parametrize("cname,pyname", [("nido_csr", "_Csr"), ("nido_params", "_Params"),
                                          ("nido_run_stats", "RunStats"), ("nido_tier_config", "TierConfig"),
                                          ("nido_request_info", "RequestInfo")])
def test_ctypes_structs_match_header(nido_lib, cname, pyname):
    """The Python mirrors of the C ABI's structs have the header's fields in
    the header's order with the same widths, so no field is read at the
    wrong offset."""
    want = header_structs()[cname]
    cls = getattr(nido_lib, pyname)
    got = cls._fields_
    assert [f[0] for f in got] == [f[0] for f in want], cname
    for (name, ctype), (_, htype, n) in zip(got, want):
        if htype == "pointer":
            assert C.sizeof(ctype) == 8, name
            continue
        base = ctype._type_ if n else ctype
        if n:
            assert ctype._length_ == n, name
        assert C.sizeof(base) == C.sizeof(getattr(C, _CTYPES[htype])), name


def test_result_buffer_validation():
    """run(out=...) takes a contiguous int64 array of the right length (a
    page-locked one downloads at full link speed) and refuses anything else."""
    import numpy as np

    from nido_b200 import capi
    good = np.empty(10, np.int64)
    assert capi._out_array(good, 10) is good
    assert capi._out_array(None, 3).shape == (3,)
    for bad in (np.empty(10, np.int32), np.empty(9, np.int64), np.empty((2, 5), np.int64), np.empty(20, np.int64)[::2]):
        with pytest.raises(ValueError):
            capi._out_array(bad, 10)
