"""ctypes binding of ``libzogcu.so`` (the C ABI declared in ``include/zogcu.h``).

The library is loaded from this package directory (built in-tree by
``python -m zog_b200.build``).  There is no fallback: if the library is missing
or no sm_100 device is present, calls raise ``ZogCudaError``.
"""
from __future__ import annotations

import ctypes as C
import os
import threading

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libzogcu.so")

ZOGCU_OK = 0
STATUS_NAMES = {
    0: "ok", 1: "invalid argument", 2: "node not found", 3: "out of memory", 4: "CUDA error",
    5: "no usable device", 6: "device wait timed out", 7: "I/O error", 8: "too large", 9: "internal error",
}
PREC_FP64 = 0
PREC_MIXED = 1
LOSS_LOG_MSE = 0
LOSS_KL = 1

#: every entry point declared in include/zogcu.h
EXPORTS = (
    "zogcu_status_string", "zogcu_last_error", "zogcu_abi_version",
    "zogcu_graph_create_from_edges", "zogcu_graph_create_from_device_edges",
    "zogcu_graph_create_from_arraygraph", "zogcu_graph_generate_rmat", "zogcu_rmat_raw_device",
    "zogcu_read_edgelist", "zogcu_graph_destroy", "zogcu_graph_info", "zogcu_graph_export_csr",
    "zogcu_free", "zogcu_pagerank", "zogcu_pagerank_ex", "zogcu_betweenness_unweighted",
    "zogcu_betweenness_unweighted_ex", "zogcu_bfs_sigma", "zogcu_pagerank_noalloc",
    "zogcu_katz", "zogcu_alpha_centrality", "zogcu_eigenvector",
    "zogcu_graph_generate_ba", "zogcu_graph_generate_ws",
    "zogcu_gnn_num_params", "zogcu_gnn_create", "zogcu_gnn_destroy", "zogcu_gnn_get_params",
    "zogcu_gnn_set_params", "zogcu_gnn_loss_grad", "zogcu_gnn_train_step", "zogcu_gnn_predict",
    "zogcu_gnn_save", "zogcu_gnn_load",
    "zogcu_batch_create", "zogcu_batch_destroy", "zogcu_batch_info", "zogcu_batch_pagerank",
    "zogcu_ppr", "zogcu_betweenness_weighted", "zogcu_graph_export_weights",
    "zogcu_graph_create_from_arraygraph_weighted", "zogcu_release_cached_memory",
)


class ZogCudaError(RuntimeError):
    """A libzogcu call returned a non-zero status."""

    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS_NAMES.get(status, 'status %d' % status)}: {message}")
        self.status = status


class Stats(C.Structure):
    _fields_ = [
        ("iterations", C.c_uint64), ("residual", C.c_double), ("elapsed_ms", C.c_double),
        ("bytes_moved", C.c_double), ("sources", C.c_uint64), ("max_depth", C.c_uint32),
        ("sigma_overflow", C.c_uint32), ("launches", C.c_uint64), ("polish_iterations", C.c_uint64),
        ("kernel_config", C.c_uint32), ("reserved", C.c_uint32),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class PrOpts(C.Structure):
    _fields_ = [
        ("struct_size", C.c_uint32), ("precision", C.c_int32), ("x0", C.c_void_p),
        ("teleport", C.c_void_p), ("device_pointers", C.c_int32), ("reserved", C.c_int32),
        ("stream", C.c_void_p),
    ]


class BatchOpts(C.Structure):
    _fields_ = [
        ("struct_size", C.c_uint32), ("config", C.c_int32), ("device_pointers", C.c_int32),
        ("reserved", C.c_int32), ("stream", C.c_void_p),
    ]


class BcOpts(C.Structure):
    _fields_ = [
        ("struct_size", C.c_uint32), ("batch", C.c_uint32), ("sources", C.c_void_p),
        ("num_sources", C.c_uint64), ("device_pointers", C.c_int32), ("reserved", C.c_int32),
        ("stream", C.c_void_p),
    ]


_lib = None
_lock = threading.Lock()


def load(path: str | None = None):
    """Load libzogcu.so (raises if it has not been built)."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        p = path or LIB_PATH
        if not os.path.exists(p):
            raise ZogCudaError(5, f"{p} is missing; build it with `python -m zog_b200.build`")
        L = C.CDLL(p)
        vp, u32, u64, dbl, i32 = C.c_void_p, C.c_uint32, C.c_uint64, C.c_double, C.c_int
        pp = C.POINTER(C.c_void_p)
        L.zogcu_status_string.restype = C.c_char_p
        L.zogcu_status_string.argtypes = [i32]
        L.zogcu_last_error.restype = C.c_char_p
        L.zogcu_last_error.argtypes = []
        L.zogcu_abi_version.restype = i32
        L.zogcu_graph_create_from_edges.argtypes = [u32, vp, vp, vp, u64, pp]
        L.zogcu_graph_create_from_device_edges.argtypes = [u32, vp, vp, u64, vp, pp]
        L.zogcu_graph_create_from_arraygraph.argtypes = [u32, vp, vp, u64, vp, vp, vp, pp]
        L.zogcu_graph_generate_rmat.argtypes = [i32, i32, u64, dbl, dbl, dbl, i32, pp]
        L.zogcu_rmat_raw_device.argtypes = [i32, u64, dbl, dbl, dbl, u64, u64, vp, vp]
        L.zogcu_read_edgelist.argtypes = [C.c_char_p, i32, i32, pp, C.POINTER(u32),
                                          C.POINTER(C.c_void_p), C.POINTER(u64)]
        L.zogcu_graph_destroy.argtypes = [vp]
        L.zogcu_graph_info.argtypes = [vp, C.POINTER(u32), C.POINTER(u64), C.POINTER(u64)]
        L.zogcu_graph_export_csr.argtypes = [vp, vp, vp, vp, vp, vp]
        L.zogcu_free.argtypes = [vp]
        L.zogcu_free.restype = None
        L.zogcu_pagerank.argtypes = [vp, dbl, u64, dbl, vp, C.POINTER(Stats)]
        L.zogcu_pagerank_ex.argtypes = [vp, dbl, u64, dbl, C.POINTER(PrOpts), vp, C.POINTER(Stats)]
        L.zogcu_betweenness_unweighted.argtypes = [vp, vp, C.POINTER(Stats)]
        L.zogcu_betweenness_unweighted_ex.argtypes = [vp, C.POINTER(BcOpts), vp, C.POINTER(Stats)]
        L.zogcu_bfs_sigma.argtypes = [vp, vp, u64, vp, vp, C.POINTER(u32)]
        L.zogcu_pagerank_noalloc.argtypes = [vp, vp, vp, u32, u64, dbl, u64, dbl, vp, C.POINTER(Stats), vp]
        L.zogcu_katz.argtypes = [vp, dbl, dbl, u64, dbl, vp, C.POINTER(Stats)]
        L.zogcu_graph_generate_ba.argtypes = [u32, u32, u64, i32, pp]
        L.zogcu_graph_generate_ws.argtypes = [u32, u32, dbl, u64, i32, pp]
        L.zogcu_alpha_centrality.argtypes = [vp, dbl, dbl, u64, dbl, vp, C.POINTER(Stats)]
        L.zogcu_eigenvector.argtypes = [vp, u64, dbl, vp, C.POINTER(Stats)]
        fp = C.POINTER(C.c_float)
        L.zogcu_gnn_num_params.argtypes = []
        L.zogcu_gnn_create.argtypes = [u64, pp]
        L.zogcu_gnn_destroy.argtypes = [vp]
        L.zogcu_gnn_get_params.argtypes = [vp, vp]
        L.zogcu_gnn_set_params.argtypes = [vp, vp]
        L.zogcu_gnn_loss_grad.argtypes = [vp, vp, vp, i32, fp, vp]
        L.zogcu_gnn_train_step.argtypes = [vp, vp, vp, i32, C.c_float, fp]
        L.zogcu_gnn_predict.argtypes = [vp, vp, vp, i32, vp, vp]
        L.zogcu_gnn_save.argtypes = [vp, C.c_char_p]
        L.zogcu_gnn_load.argtypes = [C.c_char_p, pp]
        L.zogcu_betweenness_weighted.argtypes = [vp, C.POINTER(BcOpts), vp, C.POINTER(Stats)]
        L.zogcu_graph_export_weights.argtypes = [vp, vp]
        L.zogcu_graph_create_from_arraygraph_weighted.argtypes = [u32, vp, vp, u64, vp, vp, vp, vp, pp]
        L.zogcu_ppr.argtypes = [vp, vp, u32, dbl, u64, dbl, C.POINTER(PrOpts), vp, vp, C.POINTER(Stats)]
        L.zogcu_batch_create.argtypes = [vp, u32, pp]
        L.zogcu_batch_destroy.argtypes = [vp]
        L.zogcu_batch_info.argtypes = [vp, C.POINTER(u32), C.POINTER(u64), C.POINTER(u64), vp]
        L.zogcu_batch_pagerank.argtypes = [vp, dbl, u64, dbl, C.POINTER(BatchOpts), vp, vp, C.POINTER(Stats)]
        L.zogcu_release_cached_memory.argtypes = []
        for name in EXPORTS:  # every other entry point returns a zogcu_status
            if name not in ("zogcu_status_string", "zogcu_last_error", "zogcu_free"):
                getattr(L, name).restype = C.c_int
        _lib = L
        return L


def check(status: int):
    if status != ZOGCU_OK:
        L = load()
        msg = L.zogcu_last_error().decode(errors="replace")
        raise ZogCudaError(status, msg)


def _ptr(a: np.ndarray | None):
    return None if a is None else a.ctypes.data


class Graph:
    """Owning wrapper of a ``zogcu_graph*`` (a device-resident CSR)."""

    def __init__(self, handle):
        self._h = C.c_void_p(handle) if not isinstance(handle, C.c_void_p) else handle
        self._released = False

    @property
    def handle(self):
        if self._released or not self._h:
            raise ZogCudaError(1, "graph resource already destroyed")
        return self._h

    # -- constructors ------------------------------------------------------
    @classmethod
    def from_edges(cls, node_count: int, frm, to, weight=None) -> "Graph":
        L = load()
        frm = np.ascontiguousarray(frm, dtype=np.uint32)
        to = np.ascontiguousarray(to, dtype=np.uint32)
        if frm.shape != to.shape:
            raise ValueError("from / to length mismatch")
        w = None if weight is None else np.ascontiguousarray(weight, dtype=np.float64)
        h = C.c_void_p()
        check(L.zogcu_graph_create_from_edges(int(node_count), _ptr(frm), _ptr(to), _ptr(w), frm.size,
                                              C.byref(h)))
        return cls(h)

    @classmethod
    def from_device_edges(cls, node_count: int, d_from_ptr: int, d_to_ptr: int, num_edges: int,
                          stream: int | None = None) -> "Graph":
        L = load()
        h = C.c_void_p()
        check(L.zogcu_graph_create_from_device_edges(int(node_count), d_from_ptr, d_to_ptr, int(num_edges),
                                                     stream, C.byref(h)))
        return cls(h)

    @classmethod
    def from_arraygraph(cls, first_edge, node_deleted, to, next_edge, edge_deleted, data=None) -> "Graph":
        L = load()
        fe = np.ascontiguousarray(first_edge, dtype=np.uint32)
        nd = None if node_deleted is None else np.ascontiguousarray(node_deleted, dtype=np.uint8)
        to_ = np.ascontiguousarray(to, dtype=np.uint32)
        ne = np.ascontiguousarray(next_edge, dtype=np.uint32)
        ed = None if edge_deleted is None else np.ascontiguousarray(edge_deleted, dtype=np.uint8)
        h = C.c_void_p()
        if data is None:
            check(L.zogcu_graph_create_from_arraygraph(fe.size, _ptr(fe), _ptr(nd), to_.size, _ptr(to_), _ptr(ne),
                                                       _ptr(ed), C.byref(h)))
        else:
            dt = np.ascontiguousarray(data, dtype=np.float64)
            check(L.zogcu_graph_create_from_arraygraph_weighted(fe.size, _ptr(fe), _ptr(nd), to_.size, _ptr(to_),
                                                                _ptr(ne), _ptr(ed), _ptr(dt), C.byref(h)))
        return cls(h)

    @classmethod
    def rmat(cls, scale: int, edge_factor: int, seed: int, a=0.57, b=0.19, c=0.19, directed=True) -> "Graph":
        L = load()
        h = C.c_void_p()
        check(L.zogcu_graph_generate_rmat(scale, edge_factor, seed, a, b, c, 1 if directed else 0, C.byref(h)))
        return cls(h)

    @classmethod
    def barabasi_albert(cls, n: int, m: int, seed: int, directed=True) -> "Graph":
        h = C.c_void_p()
        check(load().zogcu_graph_generate_ba(n, m, seed, 1 if directed else 0, C.byref(h)))
        return cls(h)

    @classmethod
    def watts_strogatz(cls, n: int, k: int, beta: float, seed: int, directed=False) -> "Graph":
        h = C.c_void_p()
        check(load().zogcu_graph_generate_ws(n, k, beta, seed, 1 if directed else 0, C.byref(h)))
        return cls(h)

    @classmethod
    def read_edgelist(cls, path: str, directed=True, integer_labels=False):
        L = load()
        h = C.c_void_p()
        nid = C.c_uint32(0)
        lab = C.c_void_p()
        ln = C.c_uint64(0)
        check(L.zogcu_read_edgelist(os.fsencode(path), 1 if directed else 0, 1 if integer_labels else 0,
                                    C.byref(h), C.byref(nid), C.byref(lab), C.byref(ln)))
        labels = None
        if lab.value:
            raw = C.string_at(lab.value, ln.value)
            L.zogcu_free(lab)
            labels = raw.decode().split("\n") if raw else []
        elif not integer_labels:
            labels = []
        return cls(h), int(nid.value), labels

    # -- lifetime ------------------------------------------------------------
    def destroy(self):
        if not self._released and self._h:
            check(load().zogcu_graph_destroy(self._h))
        self._released = True

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass

    # -- queries ---------------------------------------------------------------
    def info(self):
        V = C.c_uint32(0); E = C.c_uint64(0); n = C.c_uint64(0)
        check(load().zogcu_graph_info(self.handle, C.byref(V), C.byref(E), C.byref(n)))
        return int(V.value), int(E.value), int(n.value)

    def export_csr(self):
        V, E, _ = self.info()
        in_off = np.zeros(V + 1, np.uint64); out_off = np.zeros(V + 1, np.uint64)
        in_col = np.zeros(max(E, 1), np.uint32); out_col = np.zeros(max(E, 1), np.uint32)
        deg = np.zeros(max(V, 1), np.uint32)
        check(load().zogcu_graph_export_csr(self.handle, _ptr(in_off), _ptr(in_col), _ptr(out_off),
                                            _ptr(out_col), _ptr(deg)))
        return in_off, in_col[:E], out_off, out_col[:E], deg[:V]

    # -- algorithms ----------------------------------------------------------
    def pagerank(self, damping=0.85, max_iterations=100, tolerance=1e-4, *, precision=PREC_FP64, x0=None,
                 teleport=None, out=None, stats=False):
        V, _, _ = self.info()
        res = np.zeros(max(V, 1), np.float64) if out is None else out
        st = Stats()
        x0a = None if x0 is None else np.ascontiguousarray(x0, dtype=np.float64)
        tpa = None if teleport is None else np.ascontiguousarray(teleport, dtype=np.float64)
        for a in (x0a, tpa):
            if a is not None and a.size != V:
                raise ValueError("x0 / teleport must have node-capacity length")
        if precision == PREC_FP64 and x0a is None and tpa is None:
            check(load().zogcu_pagerank(self.handle, float(damping), int(max_iterations), float(tolerance),
                                        _ptr(res), C.byref(st)))
        else:
            o = PrOpts(C.sizeof(PrOpts), int(precision), _ptr(x0a), _ptr(tpa), 0, 0, None)
            check(load().zogcu_pagerank_ex(self.handle, float(damping), int(max_iterations), float(tolerance),
                                           C.byref(o), _ptr(res), C.byref(st)))
        r = res[:V]
        return (r, st.as_dict()) if stats else r

    def betweenness_unweighted(self, sources=None, stats=False):
        V, _, _ = self.info()
        res = np.zeros(max(V, 1), np.float64)
        st = Stats()
        if sources is None:
            check(load().zogcu_betweenness_unweighted(self.handle, _ptr(res), C.byref(st)))
        else:
            src = np.ascontiguousarray(sources, dtype=np.uint32)
            o = BcOpts(C.sizeof(BcOpts), 0, _ptr(src), src.size, 0, 0, None)
            check(load().zogcu_betweenness_unweighted_ex(self.handle, C.byref(o), _ptr(res), C.byref(st)))
        r = res[:V]
        return (r, st.as_dict()) if stats else r

    def betweenness_weighted(self, sources=None, stats=False):
        """Weighted (Dijkstra) betweenness over the arc weights."""
        V, _, _ = self.info()
        res = np.zeros(max(V, 1), np.float64)
        st = Stats()
        src = None if sources is None else np.ascontiguousarray(sources, dtype=np.uint32)
        o = BcOpts(C.sizeof(BcOpts), 0, _ptr(src), 0 if src is None else src.size, 0, 0, None)
        check(load().zogcu_betweenness_weighted(self.handle, C.byref(o), _ptr(res), C.byref(st)))
        r = res[:V]
        return (r, st.as_dict()) if stats else r

    def betweenness_weighted_device(self, out_ptr: int, sources=None, stream=None) -> dict:
        """Weighted betweenness into a device buffer (length V, f64)."""
        st = Stats()
        src = None if sources is None else np.ascontiguousarray(sources, dtype=np.uint32)
        o = BcOpts(C.sizeof(BcOpts), 0, _ptr(src), 0 if src is None else src.size, 1, 0, stream)
        check(load().zogcu_betweenness_weighted(self.handle, C.byref(o), out_ptr, C.byref(st)))
        return st.as_dict()

    def export_weights(self):
        """Arc weights in successor (out-CSR) order."""
        _, E, _ = self.info()
        w = np.zeros(max(E, 1), np.float64)
        check(load().zogcu_graph_export_weights(self.handle, _ptr(w)))
        return w[:E]

    def pagerank_device(self, out_ptr: int, damping=0.85, max_iterations=100, tolerance=1e-4, *,
                        precision=PREC_FP64, x0_ptr=None, teleport_ptr=None, stream=None) -> dict:
        """PageRank into a device buffer (length V, f64) on a caller stream."""
        st = Stats()
        o = PrOpts(C.sizeof(PrOpts), int(precision), x0_ptr, teleport_ptr, 1, 0, stream)
        check(load().zogcu_pagerank_ex(self.handle, float(damping), int(max_iterations), float(tolerance),
                                       C.byref(o), out_ptr, C.byref(st)))
        return st.as_dict()

    def betweenness_device(self, out_ptr: int, sources=None, stream=None) -> dict:
        """Betweenness (summed over `sources`, default all) into a device buffer."""
        st = Stats()
        src = None if sources is None else np.ascontiguousarray(sources, dtype=np.uint32)
        o = BcOpts(C.sizeof(BcOpts), 0, _ptr(src), 0 if src is None else src.size, 1, 0, stream)
        check(load().zogcu_betweenness_unweighted_ex(self.handle, C.byref(o), out_ptr, C.byref(st)))
        return st.as_dict()

    def katz(self, alpha=0.1, beta=1.0, max_iterations=100, tolerance=1e-4, stats=False):
        V, _, _ = self.info()
        res = np.zeros(max(V, 1), np.float64)
        st = Stats()
        check(load().zogcu_katz(self.handle, float(alpha), float(beta), int(max_iterations), float(tolerance),
                                _ptr(res), C.byref(st)))
        return (res[:V], st.as_dict()) if stats else res[:V]

    def alpha_centrality(self, alpha=0.5, initial=1.0, max_iterations=100, tolerance=1e-4, stats=False):
        V, _, _ = self.info()
        res = np.zeros(max(V, 1), np.float64)
        st = Stats()
        check(load().zogcu_alpha_centrality(self.handle, float(alpha), float(initial), int(max_iterations),
                                            float(tolerance), _ptr(res), C.byref(st)))
        return (res[:V], st.as_dict()) if stats else res[:V]

    def eigenvector(self, max_iterations=100, tolerance=1e-4, stats=False):
        V, _, _ = self.info()
        res = np.zeros(max(V, 1), np.float64)
        st = Stats()
        check(load().zogcu_eigenvector(self.handle, int(max_iterations), float(tolerance), _ptr(res), C.byref(st)))
        return (res[:V], st.as_dict()) if stats else res[:V]

    def ppr(self, seeds, damping=0.85, max_iterations=100, tolerance=1e-4, stats=False):
        """Personalised PageRank of every seed: (num_seeds, V) array and the
        per-seed iteration counts."""
        V, _, _ = self.info()
        sd = np.ascontiguousarray(seeds, dtype=np.uint32)
        res = np.zeros((max(sd.size, 1), max(V, 1)), np.float64)
        its = np.zeros(max(sd.size, 1), np.uint64)
        st = Stats()
        check(load().zogcu_ppr(self.handle, _ptr(sd), sd.size, float(damping), int(max_iterations),
                               float(tolerance), None, _ptr(res), _ptr(its), C.byref(st)))
        r = (res[:sd.size, :V], its[:sd.size])
        return (*r, st.as_dict()) if stats else r

    def ppr_device(self, seeds, out_ptr: int, damping=0.85, max_iterations=100, tolerance=1e-4, stream=None):
        """Personalised PageRank into a device buffer (num_seeds * V, f64, seed-major)."""
        sd = np.ascontiguousarray(seeds, dtype=np.uint32)
        its = np.zeros(max(sd.size, 1), np.uint64)
        st = Stats()
        o = PrOpts(C.sizeof(PrOpts), PREC_FP64, None, None, 1, 0, stream)
        check(load().zogcu_ppr(self.handle, _ptr(sd), sd.size, float(damping), int(max_iterations),
                               float(tolerance), C.byref(o), out_ptr, _ptr(its), C.byref(st)))
        d = st.as_dict()
        d["per_seed_iterations"] = its[:sd.size]
        return d

    def bfs_sigma(self, sources):
        V, _, _ = self.info()
        src = np.ascontiguousarray(sources, dtype=np.uint32)
        dist = np.zeros((src.size, V), np.uint32)
        sigma = np.zeros((src.size, V), np.uint64)
        ovf = C.c_uint32(0)
        check(load().zogcu_bfs_sigma(self.handle, _ptr(src), src.size, _ptr(dist), _ptr(sigma), C.byref(ovf)))
        return dist, sigma, bool(ovf.value)


def release_cached_memory():
    """Returns the device memory the library's pool keeps in reserve to the driver."""
    check(load().zogcu_release_cached_memory())


def rmat_raw_device(scale, seed, i0, m, a=0.57, b=0.19, c=0.19):
    """Raw R-MAT endpoints computed by the CUDA generator (returns host arrays)."""
    import torch  # device buffers only

    s = torch.empty(m, dtype=torch.int32, device="cuda")
    d = torch.empty(m, dtype=torch.int32, device="cuda")
    check(load().zogcu_rmat_raw_device(scale, seed, a, b, c, i0, m, s.data_ptr(), d.data_ptr()))
    return s.cpu().numpy().view(np.uint32), d.cpu().numpy().view(np.uint32)


class WarmStart:
    """Owning wrapper of a ``zogcu_gnn*``: the learned PageRank start vector.

    The network predicts y = log(n * pagerank) from degree features; its
    softmax is handed to ``Graph.pagerank(x0=...)``, which still iterates to
    the caller's tolerance.
    """

    def __init__(self, handle):
        self._h = handle if isinstance(handle, C.c_void_p) else C.c_void_p(handle)

    @classmethod
    def create(cls, seed: int = 0) -> "WarmStart":
        h = C.c_void_p()
        check(load().zogcu_gnn_create(int(seed), C.byref(h)))
        return cls(h)

    @classmethod
    def load_file(cls, path: str) -> "WarmStart":
        h = C.c_void_p()
        check(load().zogcu_gnn_load(os.fsencode(path), C.byref(h)))
        return cls(h)

    @staticmethod
    def num_params() -> int:
        return int(load().zogcu_gnn_num_params())

    def destroy(self):
        if self._h:
            check(load().zogcu_gnn_destroy(self._h))
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass

    def save(self, path: str):
        check(load().zogcu_gnn_save(self._h, os.fsencode(path)))

    def get_params(self) -> np.ndarray:
        p = np.zeros(self.num_params(), np.float32)
        check(load().zogcu_gnn_get_params(self._h, _ptr(p)))
        return p

    def set_params(self, p):
        p = np.ascontiguousarray(p, dtype=np.float32)
        if p.size != self.num_params():
            raise ValueError("parameter vector has the wrong length")
        check(load().zogcu_gnn_set_params(self._h, _ptr(p)))

    def loss_grad(self, g: Graph, target_pr, loss_kind: int = LOSS_KL):
        V, _, _ = g.info()
        t = np.ascontiguousarray(target_pr, dtype=np.float64)
        if t.size != V:
            raise ValueError("target must have node-capacity length")
        loss = C.c_float(0)
        grad = np.zeros(self.num_params(), np.float32)
        check(load().zogcu_gnn_loss_grad(self._h, g.handle, _ptr(t), int(loss_kind), C.byref(loss), _ptr(grad)))
        return float(loss.value), grad

    def train_step(self, g: Graph, d_target_ptr: int, lr: float, loss_kind: int = LOSS_KL) -> float:
        loss = C.c_float(0)
        check(load().zogcu_gnn_train_step(self._h, g.handle, d_target_ptr, int(loss_kind), float(lr),
                                          C.byref(loss)))
        return float(loss.value)

    def predict(self, g: Graph, raw=False):
        """Start vector x0 (host, length V); with raw=True also the output y."""
        V, _, _ = g.info()
        x0 = np.zeros(max(V, 1), np.float64)
        y = np.zeros(max(V, 1), np.float32) if raw else None
        check(load().zogcu_gnn_predict(self._h, g.handle, _ptr(x0), 0, None, _ptr(y)))
        return (x0[:V], y[:V]) if raw else x0[:V]

    def predict_device(self, g: Graph, x0_ptr: int, stream=None):
        """Start vector into a device buffer (length V, f64) on a caller stream."""
        check(load().zogcu_gnn_predict(self._h, g.handle, x0_ptr, 1, stream, None))


class Batch:
    """Owning wrapper of a ``zogcu_batch*``: copies of several graphs solved
    together in one persistent launch."""

    def __init__(self, graphs):
        arr = (C.c_void_p * max(len(graphs), 1))(*[g.handle.value for g in graphs])
        self._h = C.c_void_p()
        check(load().zogcu_batch_create(arr, len(graphs), C.byref(self._h)))

    def destroy(self):
        if self._h:
            check(load().zogcu_batch_destroy(self._h))
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass

    def info(self):
        n = C.c_uint32(0); V = C.c_uint64(0); E = C.c_uint64(0)
        check(load().zogcu_batch_info(self._h, C.byref(n), C.byref(V), C.byref(E), None))
        offs = np.zeros(n.value + 1, np.uint64)
        check(load().zogcu_batch_info(self._h, None, None, None, _ptr(offs)))
        return int(n.value), int(V.value), int(E.value), offs

    def pagerank(self, damping=0.85, max_iterations=100, tolerance=1e-4, config=-1, stats=False):
        """Scores of every graph (a list of arrays) and their iteration counts."""
        n, V, _, offs = self.info()
        out = np.zeros(max(V, 1), np.float64)
        its = np.zeros(max(n, 1), np.uint64)
        st = Stats()
        o = BatchOpts(C.sizeof(BatchOpts), int(config), 0, 0, None)
        check(load().zogcu_batch_pagerank(self._h, float(damping), int(max_iterations), float(tolerance),
                                          C.byref(o), _ptr(out), _ptr(its), C.byref(st)))
        res = [out[int(offs[i]):int(offs[i + 1])] for i in range(n)]
        return (res, its[:n], st.as_dict()) if stats else (res, its[:n])

    def pagerank_device(self, out_ptr: int, damping=0.85, max_iterations=100, tolerance=1e-4, config=-1,
                        stream=None):
        """Scores into a device buffer (total node slots, f64); returns stats."""
        n, _, _, _ = self.info()
        its = np.zeros(max(n, 1), np.uint64)
        st = Stats()
        o = BatchOpts(C.sizeof(BatchOpts), int(config), 1, 0, stream)
        check(load().zogcu_batch_pagerank(self._h, float(damping), int(max_iterations), float(tolerance),
                                          C.byref(o), out_ptr, _ptr(its), C.byref(st)))
        d = st.as_dict()
        d["per_graph_iterations"] = its[:n]
        return d
