"""ctypes binding of libnido_b200.so (declarations in include/nido_b200.h).

The library is the product; this module only marshals numpy arrays across the
C ABI.  It refuses to run without the compiled library: there is no Python or
CPU fallback for any device operation.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "lib", "libnido_b200.so")

NIDO_OK = 0
NIDO_TIE_SMALLEST_ID = 0
NIDO_TIE_NIDO = 1
W_ONE, W_UNIFORM, W_LOGNORMAL, W_INT8 = 0, 1, 2, 3

_i64p = C.POINTER(C.c_int64)
_f64p = C.POINTER(C.c_double)


class NidoError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"nido error {code}: {msg}")
        self.code = code


class _Csr(C.Structure):
    _fields_ = [("nv", C.c_int64), ("ne", C.c_int64), ("off", _i64p), ("adj", _i64p), ("w", _f64p)]


class _Params(C.Structure):
    _fields_ = [("nbatches", C.c_int32), ("tie_mode", C.c_int32), ("tau", C.c_double),
                ("max_iter", C.c_int64), ("verbose", C.c_int32), ("tune", C.c_int32),
                ("tau_phase", C.c_double), ("tau_phase_set", C.c_int32), ("host_loop", C.c_int32),
                ("color_batches", C.c_int32), ("reserved", C.c_int32)]


class RunStats(C.Structure):
    _fields_ = [("phases", C.c_int64), ("total_loops", C.c_int64), ("final_q", C.c_double),
                ("total_ms", C.c_double), ("move_ms", C.c_double), ("move_bytes", C.c_double),
                ("edges_scanned", C.c_double), ("move_launches", C.c_int64),
                ("kernel_launches", C.c_int64), ("host_ms", C.c_double * 8), ("q_phase", C.c_double * 200),
                ("loops_phase", C.c_int64 * 200), ("nv_phase", C.c_int64 * 200),
                ("ne_phase", C.c_int64 * 200), ("q_ms", C.c_double), ("agg_ms", C.c_double)]


_lib = None


class TierConfig(C.Structure):
    _fields_ = [("warp_max_degree", C.c_int32), ("cta_s_max_degree", C.c_int32),
                ("cta_m_max_degree", C.c_int32), ("cta_l_max_degree", C.c_int32),
                ("cta_x_max_degree", C.c_int32), ("hub_clusters", C.c_int32), ("hub_wave_slots", C.c_int64),
                ("staged_edges", C.c_int32), ("reserved", C.c_int32)]

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_}


class RequestInfo(C.Structure):
    _fields_ = [("status", C.c_int32), ("worker", C.c_int32), ("final_q", C.c_double),
                ("phases", C.c_int64), ("total_loops", C.c_int64), ("queue_ms", C.c_double),
                ("run_ms", C.c_double), ("latency_ms", C.c_double), ("device_ms", C.c_double),
                ("hbm_bytes", C.c_int64), ("host_edges", C.c_int32), ("pad", C.c_int32)]


def lib() -> C.CDLL:
    """Load the compiled library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with `make -C nido_b200/csrc` "
                              "(or __graft_entry__.build())")
        L = C.CDLL(LIB_PATH)
        vp = C.c_void_p
        sig = {
            "nido_last_error": (C.c_char_p, []),
            "nido_version": (C.c_char_p, []),
            "nido_launch_count": (C.c_uint64, []),
            "nido_ctx_create": (C.c_int, [C.c_int, C.c_size_t, C.POINTER(vp)]),
            "nido_ctx_destroy": (C.c_int, [vp]),
            "nido_ctx_sync": (C.c_int, [vp]),
            "nido_ctx_stream": (C.c_int, [vp, C.POINTER(vp)]),
            "nido_ctx_trim": (C.c_int, [vp, C.POINTER(C.c_size_t)]),
            "nido_graph_upload_vite": (C.c_int, [vp, C.c_char_p, C.c_int32, C.POINTER(vp)]),
            "nido_graph_upload": (C.c_int, [vp, C.c_int64, C.c_int64, _i64p, _i64p, _f64p, C.c_int32,
                                            C.POINTER(vp)]),
            "nido_graph_free": (C.c_int, [vp]),
            "nido_graph_size": (C.c_int, [vp, _i64p, _i64p]),
            "nido_graph_download": (C.c_int, [vp, _i64p, _i64p, _f64p]),
            "nido_graph_batches": (C.c_int, [vp, _i64p]),
            "nido_graph_vertex_weights": (C.c_int, [vp, _f64p, _f64p]),
            "nido_graph_reset": (C.c_int, [vp]),
            "nido_check_bounded_wait": (C.c_int, [vp, C.POINTER(C.c_int32), C.POINTER(C.c_int32)]),
            "nido_host_register": (C.c_int, [vp, C.c_size_t]),
            "nido_host_unregister": (C.c_int, [vp]),
            "nido_singleton_partition": (C.c_int, [vp]),
            "nido_set_community_ids": (C.c_int, [vp, _i64p]),
            "nido_compute_community_weights": (C.c_int, [vp]),
            "nido_compute_modularity": (C.c_int, [vp, _f64p]),
            "nido_louvain_update": (C.c_int, [vp, C.c_int32, C.c_int32]),
            "nido_update_community_weights": (C.c_int, [vp, C.c_int32]),
            "nido_update_community_ids": (C.c_int, [vp, C.c_int32]),
            "nido_restore_community": (C.c_int, [vp]),
            "nido_aggregation": (C.c_int, [vp, C.POINTER(C.c_int32)]),
            "nido_get_state": (C.c_int, [vp, _i64p, _i64p, _f64p]),
            "nido_get_clustering": (C.c_int, [vp, _i64p]),
            "nido_dump_partition": (C.c_int, [vp, C.c_char_p, _i64p]),
            "nido_run": (C.c_int, [vp, C.POINTER(_Params), _i64p, C.POINTER(RunStats)]),
            "nido_modularity_noalloc": (C.c_int, [vp, C.c_int64, vp, vp, vp, vp, vp, C.c_double, vp]),
            "nido_batch_upload": (C.c_int, [vp, C.c_int32, _i64p, C.c_int64, C.c_int64, _i64p, _i64p, _f64p,
                                            C.c_int32, C.POINTER(vp)]),
            "nido_batch_run": (C.c_int, [vp, C.POINTER(_Params), _i64p, _f64p, _i64p, _i64p,
                                         C.POINTER(RunStats)]),
            "nido_batch_size": (C.c_int, [vp, C.POINTER(C.c_int32), _i64p, _i64p]),
            "nido_batch_free": (C.c_int, [vp]),
            "nido_graph_footprint": (C.c_int64, [C.c_int64, C.c_int64, C.c_int32]),
            "nido_graph_footprint_streamed": (C.c_int64, [C.c_int64, C.c_int64, C.c_int32]),
            "nido_graph_host_edges": (C.c_int, [vp, C.POINTER(C.c_int32)]),
            "nido_get_tier_config": (C.c_int, [vp, C.POINTER(TierConfig)]),
            "nido_set_tier_config": (C.c_int, [vp, C.POINTER(TierConfig)]),
            "nido_tune": (C.c_int, [vp, C.c_int32, C.c_int32, C.POINTER(TierConfig), _f64p]),
            "nido_graph_device_bytes": (C.c_int, [vp, _i64p]),
            "nido_server_create": (C.c_int, [C.c_int, C.c_size_t, C.c_int32, C.POINTER(vp)]),
            "nido_server_submit": (C.c_int, [vp, C.POINTER(_Csr), C.POINTER(_Params), _i64p, _i64p]),
            "nido_server_poll": (C.c_int, [vp, C.c_int64, C.POINTER(C.c_int32)]),
            "nido_server_wait": (C.c_int, [vp, C.c_int64, C.c_double, C.POINTER(RequestInfo)]),
            "nido_server_budget": (C.c_int, [vp, _i64p, _i64p, C.POINTER(C.c_int32), C.POINTER(C.c_int32)]),
            "nido_server_destroy": (C.c_int, [vp]),
            "nido_color": (C.c_int, [vp, C.POINTER(_Csr), C.c_uint64, _i64p, _i64p]),
            "nido_color_relabel": (C.c_int, [vp, C.POINTER(_Csr), _i64p, C.POINTER(_Csr), _i64p]),
            "nido_read_vite": (C.c_int, [C.c_char_p, C.POINTER(_Csr)]),
            "nido_write_vite": (C.c_int, [C.c_char_p, C.POINTER(_Csr)]),
            "nido_csr_free": (None, [C.POINTER(_Csr)]),
            "nido_gen_planted": (C.c_int, [C.c_int64, C.c_int64, C.c_double, C.c_double, C.c_int32,
                                           C.c_uint64, C.POINTER(_Csr)]),
            "nido_gen_rmat": (C.c_int, [C.c_int64, C.c_int64, C.c_double, C.c_double, C.c_double,
                                        C.c_int32, C.c_uint64, C.POINTER(_Csr)]),
            "nido_gen_sbm": (C.c_int, [C.c_int64, C.c_double, C.c_int64, C.c_int64, C.c_double,
                                       C.c_double, C.c_int32, C.c_int32, C.c_uint64, C.POINTER(_Csr)]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def _check(st: int):
    if st != NIDO_OK:
        raise NidoError(st, lib().nido_last_error().decode())


def _p64(a: np.ndarray):
    return a.ctypes.data_as(_i64p)


def _pf(a: np.ndarray):
    return a.ctypes.data_as(_f64p)


@dataclass
class Csr:
    """Host CSR in the reference's layout: int64 offsets and ids, FP64 weights."""
    off: np.ndarray
    adj: np.ndarray
    w: np.ndarray

    @property
    def nv(self) -> int:
        return len(self.off) - 1

    @property
    def ne(self) -> int:
        return int(self.off[-1])

    def _struct(self) -> _Csr:
        self.off = np.ascontiguousarray(self.off, dtype=np.int64)
        self.adj = np.ascontiguousarray(self.adj, dtype=np.int64)
        self.w = np.ascontiguousarray(self.w, dtype=np.float64)
        return _Csr(self.nv, self.ne, _p64(self.off), _p64(self.adj), _pf(self.w))

    def degrees(self) -> np.ndarray:
        return np.diff(self.off)


def _take(s: _Csr) -> Csr:
    nv, ne = s.nv, s.ne
    off = np.ctypeslib.as_array(s.off, shape=(nv + 1,)).copy()
    adj = np.ctypeslib.as_array(s.adj, shape=(max(ne, 1),))[:ne].copy()
    w = np.ctypeslib.as_array(s.w, shape=(max(ne, 1),))[:ne].copy()
    lib().nido_csr_free(C.byref(s))
    return Csr(off, adj, w)


def gen_planted(nblocks=256, block_size=256, avg_degree=32.0, p_intra=0.8, wmode=W_UNIFORM, seed=1) -> Csr:
    s = _Csr()
    _check(lib().nido_gen_planted(nblocks, block_size, avg_degree, p_intra, wmode, seed, C.byref(s)))
    return _take(s)


def gen_rmat(nv, npairs, a=0.57, b=0.19, c=0.19, wmode=W_ONE, seed=2) -> Csr:
    s = _Csr()
    _check(lib().nido_gen_rmat(nv, npairs, a, b, c, wmode, seed, C.byref(s)))
    return _take(s)


def gen_sbm(nv, alpha=2.5, cmin=16, cmax=65536, avg_degree=32.0, p_intra=0.7, wmode=W_LOGNORMAL,
            permute=True, seed=3) -> Csr:
    s = _Csr()
    _check(lib().nido_gen_sbm(nv, alpha, cmin, cmax, avg_degree, p_intra, wmode, int(permute), seed,
                              C.byref(s)))
    return _take(s)


def host_register(a: np.ndarray):
    """Page-lock a numpy array's memory (cudaHostRegister)."""
    _check(lib().nido_host_register(a.ctypes.data, a.nbytes))


def host_unregister(a: np.ndarray):
    _check(lib().nido_host_unregister(a.ctypes.data))


def read_vite(path: str) -> Csr:
    s = _Csr()
    _check(lib().nido_read_vite(path.encode(), C.byref(s)))
    return _take(s)


def write_vite(path: str, g: Csr):
    s = g._struct()
    _check(lib().nido_write_vite(path.encode(), C.byref(s)))


class Context:
    """One CUDA device and stream (nido_ctx)."""

    def __init__(self, device: int = 0, hbm_budget: int = 0):
        h = C.c_void_p()
        _check(lib().nido_ctx_create(device, hbm_budget, C.byref(h)))
        self.h = h

    def sync(self):
        _check(lib().nido_ctx_sync(self.h))

    def stream(self) -> int:
        s = C.c_void_p()
        _check(lib().nido_ctx_stream(self.h, C.byref(s)))
        return s.value or 0

    def check_bounded_wait(self):
        """nido_check_bounded_wait: (gave_up, waited_ms) of a device wait on a
        barrier nothing arrives at."""
        gave_up, ms = C.c_int32(), C.c_int32()
        _check(lib().nido_check_bounded_wait(self.h, C.byref(gave_up), C.byref(ms)))
        return bool(gave_up.value), int(ms.value)

    def trim(self) -> int:
        """Return the device blocks cached from freed graphs to the driver;
        the number of bytes released."""
        n = C.c_size_t()
        _check(lib().nido_ctx_trim(self.h, C.byref(n)))
        return n.value

    def close(self):
        if self.h:
            lib().nido_ctx_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def color(self, g: Csr, seed: int = 1):
        colors = np.empty(g.nv, dtype=np.int64)
        nc = C.c_int64()
        s = g._struct()
        _check(lib().nido_color(self.h, C.byref(s), seed, _p64(colors), C.byref(nc)))
        return colors, nc.value

    def color_relabel(self, g: Csr, colors: np.ndarray):
        colors = np.ascontiguousarray(colors, dtype=np.int64)
        out = Csr(np.empty(g.nv + 1, np.int64), np.empty(max(g.ne, 1), np.int64),
                  np.empty(max(g.ne, 1), np.float64))
        so = _Csr(g.nv, g.ne, _p64(out.off), _p64(out.adj), _pf(out.w))
        new_orders = np.empty(g.nv, dtype=np.int64)
        s = g._struct()
        _check(lib().nido_color_relabel(self.h, C.byref(s), _p64(colors), C.byref(so), _p64(new_orders)))
        out.adj = out.adj[:g.ne]
        out.w = out.w[:g.ne]
        return out, new_orders


class Graph:
    """A graph resident on the device (nido_graph), with GraphGPU's operators."""

    def __init__(self, ctx: Context, g: Csr, nbatches: int = 2):
        self.ctx = ctx
        self.nv0 = g.nv
        self.nbatches = nbatches
        s = g._struct()
        h = C.c_void_p()
        _check(lib().nido_graph_upload(ctx.h, s.nv, s.ne, s.off, s.adj, s.w, nbatches, C.byref(h)))
        self.h = h

    @classmethod
    def from_vite(cls, ctx: Context, path: str, nbatches: int = 2) -> "Graph":
        """Stream a Vite binary file straight to the device
        (nido_graph_upload_vite)."""
        self = cls.__new__(cls)
        self.ctx = ctx
        self.nbatches = nbatches
        h = C.c_void_p()
        _check(lib().nido_graph_upload_vite(ctx.h, os.fsencode(path), nbatches, C.byref(h)))
        self.h = h
        self.nv0 = self.size()[0]
        return self

    def close(self):
        if self.h:
            lib().nido_graph_free(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def size(self):
        nv, ne = C.c_int64(), C.c_int64()
        _check(lib().nido_graph_size(self.h, C.byref(nv), C.byref(ne)))
        return nv.value, ne.value

    def download(self) -> Csr:
        nv, ne = self.size()
        off = np.empty(nv + 1, np.int64)
        adj = np.empty(max(ne, 1), np.int64)
        w = np.empty(max(ne, 1), np.float64)
        _check(lib().nido_graph_download(self.h, _p64(off), _p64(adj), _pf(w)))
        return Csr(off, adj[:ne], w[:ne])

    def batches(self) -> np.ndarray:
        cuts = np.empty(self.nbatches + 1, np.int64)
        _check(lib().nido_graph_batches(self.h, _p64(cuts)))
        return cuts

    def vertex_weights(self):
        nv, _ = self.size()
        k = np.empty(nv, np.float64)
        m = C.c_double()
        _check(lib().nido_graph_vertex_weights(self.h, _pf(k), C.byref(m)))
        return k, m.value

    def reset(self):
        _check(lib().nido_graph_reset(self.h))

    def singleton_partition(self):
        _check(lib().nido_singleton_partition(self.h))

    def set_community_ids(self, comm: np.ndarray):
        comm = np.ascontiguousarray(comm, dtype=np.int64)
        _check(lib().nido_set_community_ids(self.h, _p64(comm)))

    def compute_community_weights(self):
        _check(lib().nido_compute_community_weights(self.h))

    def compute_modularity(self) -> float:
        q = C.c_double()
        _check(lib().nido_compute_modularity(self.h, C.byref(q)))
        return q.value

    def louvain_update(self, batch: int, tie: int = NIDO_TIE_SMALLEST_ID):
        _check(lib().nido_louvain_update(self.h, batch, tie))

    def update_community_weights(self, batch: int):
        _check(lib().nido_update_community_weights(self.h, batch))

    def update_community_ids(self, batch: int):
        _check(lib().nido_update_community_ids(self.h, batch))

    def restore_community(self):
        _check(lib().nido_restore_community(self.h))

    def aggregation(self) -> bool:
        d = C.c_int32()
        _check(lib().nido_aggregation(self.h, C.byref(d)))
        return bool(d.value)

    def state(self):
        nv, _ = self.size()
        comm = np.empty(nv, np.int64)
        newc = np.empty(nv, np.int64)
        a = np.empty(nv, np.float64)
        _check(lib().nido_get_state(self.h, _p64(comm), _p64(newc), _pf(a)))
        return comm, newc, a

    def clustering(self) -> np.ndarray:
        c = np.empty(self.nv0, np.int64)
        _check(lib().nido_get_clustering(self.h, _p64(c)))
        return c

    def dump_partition(self, path: str, new_orders: np.ndarray | None = None):
        p = None if new_orders is None else _p64(np.ascontiguousarray(new_orders, dtype=np.int64))
        _check(lib().nido_dump_partition(self.h, path.encode(), p))

    def tier_config(self) -> TierConfig:
        c = TierConfig()
        _check(lib().nido_get_tier_config(self.h, C.byref(c)))
        return c

    def set_tier_config(self, c: TierConfig):
        _check(lib().nido_set_tier_config(self.h, C.byref(c)))

    def tune(self, tie: int = NIDO_TIE_SMALLEST_ID, sweeps: int = 2):
        c = TierConfig()
        ms = C.c_double()
        _check(lib().nido_tune(self.h, tie, sweeps, C.byref(c), C.byref(ms)))
        return c, ms.value

    def host_edges(self) -> bool:
        """True when the graph's edges are in mapped host memory (over budget)."""
        x = C.c_int32()
        _check(lib().nido_graph_host_edges(self.h, C.byref(x)))
        return bool(x.value)

    def device_bytes(self) -> int:
        b = C.c_int64()
        _check(lib().nido_graph_device_bytes(self.h, C.byref(b)))
        return b.value

    def run(self, tau: float = 1e-6, max_iter: int = 500, tie: int = NIDO_TIE_SMALLEST_ID,
            verbose: bool = False, tune: bool = False, host_loop: bool = False, tau_phase: float | None = None,
            color_batches: bool = False, device_loop: bool = False, out: np.ndarray | None = None):
        """LouvainGPU::run; returns (clustering of the input vertices, RunStats).
        host_loop / device_loop: who drives each phase's iterations (the host,
        one readback per iteration, the default; or the device-resident loop
        graph, one readback per phase).  color_batches: every
        phase's colour classes are its batches (conflict-free) instead of the
        -b cuts.  out: an int64 array of nv entries to write the clustering
        into (page-locked with host_register, the download runs at full link
        speed); a new array by default."""
        p = _Params(self.nbatches, tie, tau, max_iter, int(verbose), int(tune),
                    0.0 if tau_phase is None else tau_phase, int(tau_phase is not None),
                    _loop_mode(host_loop, device_loop), int(color_batches))
        out = _out_array(out, self.nv0)
        st = RunStats()
        _check(lib().nido_run(self.h, C.byref(p), _p64(out), C.byref(st)))
        return out, st


def _out_array(out, n: int) -> np.ndarray:
    if out is None:
        return np.empty(n, np.int64)
    if out.dtype != np.int64 or out.ndim != 1 or out.shape[0] != n or not out.flags.c_contiguous:
        raise ValueError(f"out must be a contiguous int64 array of {n} entries")
    return out


def _loop_mode(host_loop: bool, device_loop: bool) -> int:
    """nido_params.host_loop: 1 host, 2 device, 0 the library's default (host)."""
    if host_loop and device_loop:
        raise ValueError("host_loop and device_loop are exclusive")
    return 1 if host_loop else (2 if device_loop else 0)


def pack_graphs(graphs: list[Csr]):
    """Disjoint union of graphs as one CSR: returns (vbase, Csr) where graph i
    owns vertices [vbase[i], vbase[i+1]) and its neighbour ids are shifted by
    vbase[i]."""
    nvs = np.array([g.nv for g in graphs], np.int64)
    nes = np.array([g.ne for g in graphs], np.int64)
    vbase = np.zeros(len(graphs) + 1, np.int64)
    np.cumsum(nvs, out=vbase[1:])
    ebase = np.zeros(len(graphs) + 1, np.int64)
    np.cumsum(nes, out=ebase[1:])
    off = np.empty(vbase[-1] + 1, np.int64)
    adj = np.empty(ebase[-1], np.int64)
    w = np.empty(ebase[-1], np.float64)
    for i, g in enumerate(graphs):
        off[vbase[i]:vbase[i + 1]] = g.off[:-1] + ebase[i]
        adj[ebase[i]:ebase[i + 1]] = g.adj + vbase[i]
        w[ebase[i]:ebase[i + 1]] = g.w
    off[-1] = ebase[-1]
    return vbase, Csr(off, adj, w)


class Batch:
    """Many independent graphs resident on the device as one packed CSR
    (nido_batch), run together by nido_batch_run."""

    def __init__(self, ctx: Context, graphs: list[Csr] | None = None, nbatches: int = 2,
                 packed: tuple[np.ndarray, Csr] | None = None):
        self.ctx = ctx
        vbase, u = packed if packed is not None else pack_graphs(graphs)
        self.vbase = np.ascontiguousarray(vbase, dtype=np.int64)
        self.ngraphs = len(self.vbase) - 1
        self.nv = u.nv
        self.nbatches = nbatches
        s = u._struct()
        h = C.c_void_p()
        _check(lib().nido_batch_upload(ctx.h, self.ngraphs, _p64(self.vbase), s.nv, s.ne, s.off, s.adj, s.w,
                                       nbatches, C.byref(h)))
        self.h = h

    def close(self):
        if self.h:
            lib().nido_batch_free(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def run(self, tau: float = 1e-6, max_iter: int = 500, tie: int = NIDO_TIE_SMALLEST_ID,
            tune: bool = False, host_loop: bool = False, device_loop: bool = False, out: np.ndarray | None = None):
        """Returns (per-graph clusterings, final Q per graph, phases per graph,
        loops per graph, RunStats).  out: as Graph.run, nv entries (the
        clusterings are views into it)."""
        p = _Params(self.nbatches, tie, tau, max_iter, 0, int(tune), 0.0, 0, _loop_mode(host_loop, device_loop))
        out = _out_array(out, self.nv)
        q = np.empty(self.ngraphs, np.float64)
        ph = np.empty(self.ngraphs, np.int64)
        lo = np.empty(self.ngraphs, np.int64)
        st = RunStats()
        _check(lib().nido_batch_run(self.h, C.byref(p), _p64(out), _pf(q), _p64(ph), _p64(lo), C.byref(st)))
        parts = [out[self.vbase[i]:self.vbase[i + 1]] for i in range(self.ngraphs)]
        return parts, q, ph, lo, st


def graph_footprint(nv: int, ne: int, nbatches: int = 2) -> int:
    return int(lib().nido_graph_footprint(nv, ne, nbatches))


def graph_footprint_streamed(nv: int, ne: int, nbatches: int = 2) -> int:
    return int(lib().nido_graph_footprint_streamed(nv, ne, nbatches))


class Server:
    """Request loop on one GPU (nido_server_*): submit() queues a run and
    returns a ticket, wait() returns (clustering, RequestInfo)."""

    def __init__(self, device: int = 0, hbm_budget: int = 0, workers: int = 4):
        h = C.c_void_p()
        _check(lib().nido_server_create(device, hbm_budget, workers, C.byref(h)))
        self.h = h
        self._keep = {}

    def submit(self, g: Csr, nbatches: int = 2, tau: float = 1e-6, max_iter: int = 500,
               tie: int = NIDO_TIE_SMALLEST_ID) -> int:
        s = g._struct()
        p = _Params(nbatches, tie, tau, max_iter, 0, 0)
        out = np.empty(g.nv, np.int64)
        t = C.c_int64()
        _check(lib().nido_server_submit(self.h, C.byref(s), C.byref(p), _p64(out), C.byref(t)))
        self._keep[t.value] = (g, out)  # the engine reads and writes these until wait()
        return t.value

    def poll(self, ticket: int) -> int:
        st = C.c_int32()
        _check(lib().nido_server_poll(self.h, ticket, C.byref(st)))
        return st.value

    def wait(self, ticket: int, timeout: float = -1.0):
        info = RequestInfo()
        rc = lib().nido_server_wait(self.h, ticket, timeout, C.byref(info))
        if rc != 0:
            st = C.c_int32()
            if lib().nido_server_poll(self.h, ticket, C.byref(st)) == 0:
                # still live (timed out, or another thread waits on it): the
                # engine may still use its buffers
                _check(rc)
        kept = self._keep.pop(ticket, None)
        _check(rc)
        out = kept[1]
        return out, info

    def budget(self):
        b, r = C.c_int64(), C.c_int64()
        run, q = C.c_int32(), C.c_int32()
        _check(lib().nido_server_budget(self.h, C.byref(b), C.byref(r), C.byref(run), C.byref(q)))
        return b.value, r.value, run.value, q.value

    def close(self):
        if self.h:
            lib().nido_server_destroy(self.h)
            self.h = None
            self._keep.clear()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()
