"""ctypes binding of the CPU oracle (oracle/_build/libnido_oracle.so).

TEST INFRASTRUCTURE ONLY: the checker for the CUDA engine.  Only tests/,
__graft_entry__.smoke() and bench.py's CPU-baseline leg may import this
module; the product (nido_b200/) never does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_build", "libnido_oracle.so")
RUN_PATH = os.path.join(_HERE, "_build", "nido_oracle_run")
TIE_SMALLEST_ID = 0
TIE_NIDO = 1

_i64p = C.POINTER(C.c_int64)
_f64p = C.POINTER(C.c_double)
_lib = None


class Stats(C.Structure):
    _fields_ = [("phases", C.c_int64), ("total_loops", C.c_int64), ("final_q", C.c_double),
                ("q_phase", C.c_double * 200), ("loops_phase", C.c_int64 * 200),
                ("nv_phase", C.c_int64 * 200), ("ne_phase", C.c_int64 * 200)]


def build():
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        L.orc_batch_cuts.argtypes = [C.c_int64, _i64p, C.c_int, _i64p]
        L.orc_vertex_weights.argtypes = [C.c_int64, _i64p, _f64p, _f64p]
        L.orc_mass.argtypes = [C.c_int64, _f64p]
        L.orc_mass.restype = C.c_double
        L.orc_singleton.argtypes = [C.c_int64, _f64p, _i64p, _i64p, _f64p]
        L.orc_community_weights.argtypes = [C.c_int64, _i64p, _f64p, _f64p]
        L.orc_move_gain.argtypes = [C.c_int64, _i64p, _i64p, _f64p, _i64p, _f64p, _f64p, C.c_double,
                                    C.c_int64, C.c_int64, C.c_int, _i64p, _f64p]
        L.orc_commit.argtypes = [C.c_int64, C.c_int64, _i64p, _i64p, _f64p, _f64p]
        L.orc_restore.argtypes = [C.c_int64, _i64p, _i64p, _f64p, _f64p]
        L.orc_modularity.argtypes = [C.c_int64, _i64p, _i64p, _f64p, _i64p, _f64p, C.c_double]
        L.orc_modularity.restype = C.c_double
        L.orc_coarsen.argtypes = [C.c_int64, _i64p, _i64p, _f64p, _i64p, _i64p, C.POINTER(_i64p),
                                  C.POINTER(_i64p), C.POINTER(_f64p), _i64p]
        L.orc_coarsen.restype = C.c_int64
        L.orc_color_relabel.argtypes = [C.c_int64, _i64p, _i64p, _f64p, _i64p, _i64p, _i64p, _i64p, _f64p]
        L.orc_color_nido_seq.argtypes = [C.c_int64, _i64p, _i64p, _i64p]
        L.orc_louvain.argtypes = [C.c_int64, _i64p, _i64p, _f64p, C.c_int, C.c_double, C.c_int64, C.c_int,
                                  C.c_int, _i64p, C.POINTER(Stats)]
        L.orc_louvain_capped.argtypes = [C.c_int64, _i64p, _i64p, _f64p, C.c_int, C.c_double, C.c_int64,
                                         C.c_int, C.c_int, C.c_int, _i64p, C.POINTER(Stats)]
        L.orc_color_jpl.argtypes = [C.c_int64, _i64p, _i64p, C.c_uint64, _i64p]
        L.orc_color_jpl.restype = C.c_int64
        L.orc_louvain_ex.argtypes = [C.c_int64, _i64p, _i64p, _f64p, C.c_int, C.c_double, C.c_int64, C.c_int,
                                     C.c_int, C.c_int, C.c_int, _i64p, C.c_void_p]
        L.orc_partition_modularity.argtypes = [C.c_int64, _i64p, _i64p, _f64p, _i64p]
        L.orc_partition_modularity.restype = C.c_double
        L.orc_nmi.argtypes = [C.c_int64, _i64p, _i64p]
        L.orc_nmi.restype = C.c_double
        L.orc_free.argtypes = [C.c_void_p]
        L.orc_read_vite.argtypes = [C.c_char_p, _i64p, _i64p, C.POINTER(_i64p), C.POINTER(_i64p),
                                    C.POINTER(_f64p)]
        _lib = L
    return _lib


def _i(a):
    return np.ascontiguousarray(a, dtype=np.int64)


def _f(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _p(a):
    return a.ctypes.data_as(_i64p)


def _pf(a):
    return a.ctypes.data_as(_f64p)


def read_vite(path):
    nv, ne = C.c_int64(), C.c_int64()
    off, adj, w = _i64p(), _i64p(), _f64p()
    if lib().orc_read_vite(path.encode(), C.byref(nv), C.byref(ne), C.byref(off), C.byref(adj), C.byref(w)):
        raise IOError(path)
    o = np.ctypeslib.as_array(off, shape=(nv.value + 1,)).copy()
    a = np.ctypeslib.as_array(adj, shape=(max(ne.value, 1),))[:ne.value].copy()
    ww = np.ctypeslib.as_array(w, shape=(max(ne.value, 1),))[:ne.value].copy()
    for p in (off, adj, w):
        lib().orc_free(C.cast(p, C.c_void_p))
    return o, a, ww


def batch_cuts(off, nbatches):
    off = _i(off)
    cuts = np.empty(nbatches + 1, np.int64)
    lib().orc_batch_cuts(len(off) - 1, _p(off), nbatches, _p(cuts))
    return cuts


def vertex_weights(off, w):
    off, w = _i(off), _f(w)
    k = np.empty(len(off) - 1, np.float64)
    lib().orc_vertex_weights(len(off) - 1, _p(off), _pf(w), _pf(k))
    return k


def mass(k):
    k = _f(k)
    return lib().orc_mass(len(k), _pf(k))


def community_weights(comm, k):
    comm, k = _i(comm), _f(k)
    a = np.zeros(len(k), np.float64)
    lib().orc_community_weights(len(k), _p(comm), _pf(k), _pf(a))
    return a


def move(off, adj, w, comm, a, k, m, v0, v1, tie=TIE_SMALLEST_ID):
    """newcomm for [v0, v1) (others keep comm) and the gain-minus-self values."""
    off, adj, w, comm, a, k = _i(off), _i(adj), _f(w), _i(comm), _f(a), _f(k)
    newc = comm.copy()
    gain = np.full(len(comm), np.nan)
    lib().orc_move_gain(len(comm), _p(off), _p(adj), _pf(w), _p(comm), _pf(a), _pf(k), m, v0, v1, tie,
                        _p(newc), _pf(gain))
    return newc, gain


def commit(v0, v1, comm, newc, k, a):
    """In-place community-degree update and id swap (arrays must be int64/float64)."""
    lib().orc_commit(v0, v1, _p(comm), _p(newc), _pf(k), _pf(a))


def modularity(off, adj, w, comm, a, m):
    off, adj, w, comm, a = _i(off), _i(adj), _f(w), _i(comm), _f(a)
    return lib().orc_modularity(len(comm), _p(off), _p(adj), _pf(w), _p(comm), _pf(a), m)


def coarsen(off, adj, w, comm):
    off, adj, w, comm = _i(off), _i(adj), _f(w), _i(comm)
    nv = len(comm)
    newid = np.empty(nv, np.int64)
    coff, cadj, cw = _i64p(), _i64p(), _f64p()
    cne = C.c_int64()
    cnv = lib().orc_coarsen(nv, _p(off), _p(adj), _pf(w), _p(comm), _p(newid), C.byref(coff), C.byref(cadj),
                            C.byref(cw), C.byref(cne))
    o = np.ctypeslib.as_array(coff, shape=(cnv + 1,)).copy()
    a = np.ctypeslib.as_array(cadj, shape=(max(cne.value, 1),))[:cne.value].copy()
    ww = np.ctypeslib.as_array(cw, shape=(max(cne.value, 1),))[:cne.value].copy()
    for p in (coff, cadj, cw):
        lib().orc_free(C.cast(p, C.c_void_p))
    return newid, (o, a, ww)


def color_relabel(off, adj, w, colors):
    off, adj, w, colors = _i(off), _i(adj), _f(w), _i(colors)
    nv, ne = len(off) - 1, len(adj)
    no = np.empty(nv, np.int64)
    noff = np.empty(nv + 1, np.int64)
    nadj = np.empty(max(ne, 1), np.int64)
    nw = np.empty(max(ne, 1), np.float64)
    lib().orc_color_relabel(nv, _p(off), _p(adj), _pf(w), _p(colors), _p(no), _p(noff), _p(nadj), _pf(nw))
    return no, (noff, nadj[:ne], nw[:ne])


def color_nido_seq(off, adj):
    off, adj = _i(off), _i(adj)
    c = np.empty(len(off) - 1, np.int64)
    lib().orc_color_nido_seq(len(off) - 1, _p(off), _p(adj), _p(c))
    return c


def louvain(off, adj, w, nbatches=2, tau=1e-6, max_loops=500, tie=TIE_SMALLEST_ID, verbose=False,
            max_phases=200, color_batches=False):
    off, adj, w = _i(off), _i(adj), _f(w)
    cl = np.empty(len(off) - 1, np.int64)
    st = Stats()
    rc = lib().orc_louvain_ex(len(off) - 1, _p(off), _p(adj), _pf(w), nbatches, tau, max_loops, tie,
                              int(verbose), max_phases, int(color_batches), _p(cl),
                              C.cast(C.byref(st), C.c_void_p))
    if rc:
        raise ValueError("orc_louvain failed")
    return cl, st


def color_jpl(off, adj, seed=1):
    """The engine's Jones-Plassmann-Luby colouring: (colours, colour count)."""
    off, adj = _i(off), _i(adj)
    c = np.empty(len(off) - 1, np.int64)
    nc = lib().orc_color_jpl(len(off) - 1, _p(off), _p(adj), seed, _p(c))
    return c, nc


def partition_modularity(off, adj, w, part):
    off, adj, w, part = _i(off), _i(adj), _f(w), _i(part)
    return lib().orc_partition_modularity(len(off) - 1, _p(off), _p(adj), _pf(w), _p(part))


def nmi(x, y):
    x, y = _i(x), _i(y)
    return lib().orc_nmi(len(x), _p(x), _p(y))
