"""ctypes front end of the CPU oracle (``liboracle_zog.so``).

TEST INFRASTRUCTURE ONLY: imported by ``tests/``, ``__graft_entry__.smoke()``
and the CPU-baseline leg of ``bench.py`` as the checker.  The library under test
(``zog_b200``) never imports this module.

The C++ behind it restates the reference's Zig code loop for loop
(``priv/zog/src/centrality.zig:858-965`` PageRank, ``:687-798`` unweighted
Brandes, ``priv/zog/src/models/array_graph.zig`` storage); see the header of
``zog_oracle.cpp`` for the full line map.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle_zog.so")
_lib = None

_u32p = np.ctypeslib.ndpointer(dtype=np.uint32, flags="C_CONTIGUOUS")
_u64p = np.ctypeslib.ndpointer(dtype=np.uint64, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_u8p = np.ctypeslib.ndpointer(dtype=np.uint8, flags="C_CONTIGUOUS")


def build(force: bool = False) -> str:
    """Compile the oracle with its Makefile (g++ -O3, no FP contraction)."""
    src = os.path.join(_HERE, "zog_oracle.cpp")
    if force or not os.path.exists(_LIB_PATH) or os.path.getmtime(_LIB_PATH) < os.path.getmtime(src):
        subprocess.check_call(["make", "-s", "-C", _HERE, "liboracle_zog.so"])
    return _LIB_PATH


def lib():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(_LIB_PATH):
        build()
    L = C.CDLL(_LIB_PATH)
    vp = C.c_void_p
    L.og_new.restype = vp
    L.og_new.argtypes = [C.c_uint32]
    L.og_free.argtypes = [vp]
    L.og_add_edge.argtypes = [vp, C.c_uint32, C.c_uint32, C.c_double]
    L.og_add_edges.argtypes = [vp, _u32p, _u32p, C.c_void_p, C.c_uint64]
    L.og_remove_edge.argtypes = [vp, C.c_uint32, C.c_uint32]
    L.og_remove_node.argtypes = [vp, C.c_uint32]
    for f in ("og_node_capacity", "og_edge_capacity", "og_live_nodes", "og_live_edges"):
        getattr(L, f).restype = C.c_uint64
        getattr(L, f).argtypes = [vp]
    L.og_export.argtypes = [vp, _u32p, _u8p, _u32p, _u32p, _u8p, _f64p]
    L.og_successor_csr.argtypes = [vp, _u64p, _u32p]
    L.og_pagerank.argtypes = [vp, C.c_double, C.c_uint64, C.c_double, _f64p,
                              C.POINTER(C.c_uint64), C.POINTER(C.c_double)]
    L.og_betweenness_unweighted.argtypes = [vp, _f64p, C.POINTER(C.c_uint32)]
    L.og_katz.argtypes = [vp, C.c_double, C.c_double, C.c_uint64, C.c_double, _f64p,
                          C.POINTER(C.c_uint64), C.POINTER(C.c_double)]
    L.og_alpha_centrality.argtypes = [vp, C.c_double, C.c_double, C.c_uint64, C.c_double, _f64p,
                                      C.POINTER(C.c_uint64), C.POINTER(C.c_double)]
    L.og_eigenvector.argtypes = [vp, C.c_uint64, C.c_double, _f64p, C.POINTER(C.c_uint64),
                                 C.POINTER(C.c_int)]
    L.og_betweenness_sources.argtypes = [vp, _u32p, C.c_uint64, _f64p, C.POINTER(C.c_uint32)]
    L.og_bfs.argtypes = [vp, C.c_uint32, _u32p, _u64p, C.POINTER(C.c_uint32)]
    L.og_pagerank_csr.restype = C.c_uint64
    L.og_pagerank_csr.argtypes = [C.c_uint32, _u64p, _u32p, _u32p, C.c_void_p, C.c_double,
                                  C.c_uint64, C.c_double, _f64p, C.POINTER(C.c_double),
                                  C.POINTER(C.c_double)]
    L.og_pagerank_ext.restype = C.c_uint64
    L.og_pagerank_ext.argtypes = [C.c_uint32, _u64p, _u32p, _u32p, C.c_void_p, C.c_void_p,
                                  C.c_double, C.c_uint64, C.c_double, _f64p,
                                  C.POINTER(C.c_double)]
    L.og_pagerank_csr_mt.argtypes = [C.c_uint32, _u64p, _u32p, _u32p, C.c_void_p, C.c_void_p, C.c_double,
                                     C.c_uint64, C.c_double, _f64p, C.POINTER(C.c_double),
                                     C.POINTER(C.c_double), C.c_int]
    L.og_pagerank_csr_mt.restype = C.c_uint64
    L.og_bfs_csr_many.argtypes = [C.c_uint32, _u64p, _u32p, _u32p, C.c_uint64, _u32p, _u64p, _u8p, C.c_int]
    L.og_betweenness_csr_sources_mt.argtypes = [C.c_uint32, _u64p, _u32p, _u32p, C.c_uint64, _f64p,
                                                C.POINTER(C.c_uint32), C.c_int]
    L.og_betweenness_csr_sources.argtypes = [C.c_uint32, _u64p, _u32p, _u32p, C.c_uint64, _f64p,
                                             C.POINTER(C.c_uint32), C.POINTER(C.c_double)]
    L.og_rmat.restype = vp
    L.og_rmat.argtypes = [C.c_int, C.c_int, C.c_uint64, C.c_double, C.c_double, C.c_double, C.c_int]
    L.og_edges_count.restype = C.c_uint64
    L.og_betweenness_weighted.argtypes = [vp, C.c_void_p, C.c_uint64, _f64p, C.POINTER(C.c_uint32)]
    L.og_ba.argtypes = [C.c_uint32, C.c_uint32, C.c_uint64, C.c_int]
    L.og_ba.restype = vp
    L.og_ws.argtypes = [C.c_uint32, C.c_uint32, C.c_double, C.c_uint64, C.c_int]
    L.og_ws.restype = vp
    L.og_edges_count.argtypes = [vp]
    L.og_edges_nodes.restype = C.c_uint32
    L.og_edges_nodes.argtypes = [vp]
    L.og_edges_copy.argtypes = [vp, _u32p, _u32p]
    L.og_edges_free.argtypes = [vp]
    L.og_rmat_raw.argtypes = [C.c_int, C.c_uint64, C.c_double, C.c_double, C.c_double,
                              C.c_uint64, C.c_uint64, _u32p, _u32p]
    L.og_in_csr.argtypes = [C.c_uint32, _u32p, _u32p, C.c_uint64, _u64p, _u32p, _u32p]
    L.og_read_edgelist.restype = vp
    L.og_read_edgelist.argtypes = [C.c_char_p, C.c_int, C.c_int, C.POINTER(C.c_uint32),
                                   C.POINTER(C.c_char_p), C.POINTER(C.c_uint64)]
    L.og_free_buf.argtypes = [C.c_char_p]
    _lib = L
    return L


class ArrayGraph:
    """The reference's ArrayGraph(void, f64) (array_graph.zig:13-38), built by
    the NIF's buildGraph loop (.Elixir.Zog.ResourceGraph.zig:26-35)."""

    def __init__(self, node_count: int, frm=None, to=None, weight=None, handle=None):
        L = lib()
        self._h = handle if handle is not None else L.og_new(int(node_count))
        if frm is not None and len(frm):
            frm = np.ascontiguousarray(frm, dtype=np.uint32)
            to = np.ascontiguousarray(to, dtype=np.uint32)
            w = None
            if weight is not None:
                w = np.ascontiguousarray(weight, dtype=np.float64)
            rc = L.og_add_edges(self._h, frm, to, w.ctypes.data if w is not None else None, len(frm))
            if rc != 0:
                raise ValueError("NodeNotFound")

    def close(self):
        if self._h:
            lib().og_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def node_capacity(self) -> int:
        return int(lib().og_node_capacity(self._h))

    @property
    def edge_capacity(self) -> int:
        return int(lib().og_edge_capacity(self._h))

    def add_edge(self, f, t, w=1.0):
        if lib().og_add_edge(self._h, f, t, w) != 0:
            raise ValueError("NodeNotFound")

    def remove_edge(self, f, t):
        if lib().og_remove_edge(self._h, f, t) != 0:
            raise ValueError("NodeNotFound")

    def remove_node(self, i):
        if lib().og_remove_node(self._h, i) != 0:
            raise ValueError("NodeNotFound")

    def export(self):
        """Raw slices: first_edge, node_deleted, to, next_edge, edge_deleted, data."""
        V, E = self.node_capacity, self.edge_capacity
        fe = np.zeros(V, np.uint32); nd = np.zeros(V, np.uint8)
        to = np.zeros(max(E, 1), np.uint32); ne = np.zeros(max(E, 1), np.uint32)
        ed = np.zeros(max(E, 1), np.uint8); da = np.zeros(max(E, 1), np.float64)
        if V == 0:
            fe = np.zeros(1, np.uint32); nd = np.zeros(1, np.uint8)
        lib().og_export(self._h, fe, nd, to, ne, ed, da)
        return fe[:V], nd[:V], to[:E], ne[:E], ed[:E], da[:E]

    def successor_csr(self):
        V, E = self.node_capacity, self.edge_capacity
        off = np.zeros(V + 1, np.uint64)
        col = np.zeros(max(E, 1), np.uint32)
        lib().og_successor_csr(self._h, off, col)
        return off, col[: int(off[-1])]

    def pagerank(self, damping=0.85, max_iterations=100, tolerance=1e-4):
        out = np.zeros(max(self.node_capacity, 1), np.float64)
        it = C.c_uint64(0); l1 = C.c_double(0)
        lib().og_pagerank(self._h, damping, max_iterations, tolerance, out, C.byref(it), C.byref(l1))
        return out[: self.node_capacity], int(it.value), float(l1.value)

    def katz(self, alpha=0.1, beta=1.0, max_iterations=100, tolerance=1e-4):
        """centrality.zig:1190-1251."""
        out = np.zeros(max(self.node_capacity, 1), np.float64)
        it = C.c_uint64(0); l1 = C.c_double(0)
        lib().og_katz(self._h, alpha, beta, max_iterations, tolerance, out, C.byref(it), C.byref(l1))
        return out[: self.node_capacity], int(it.value), float(l1.value)

    def alpha_centrality(self, alpha=0.5, initial=1.0, max_iterations=100, tolerance=1e-4):
        """centrality.zig:1262-1321."""
        out = np.zeros(max(self.node_capacity, 1), np.float64)
        it = C.c_uint64(0); l1 = C.c_double(0)
        lib().og_alpha_centrality(self._h, alpha, initial, max_iterations, tolerance, out, C.byref(it),
                                  C.byref(l1))
        return out[: self.node_capacity], int(it.value), float(l1.value)

    def eigenvector(self, max_iterations=100, tolerance=1e-4):
        """centrality.zig:1050-1180; returns (scores, iterations, how)."""
        out = np.zeros(max(self.node_capacity, 1), np.float64)
        it = C.c_uint64(0); how = C.c_int(0)
        lib().og_eigenvector(self._h, max_iterations, tolerance, out, C.byref(it), C.byref(how))
        return out[: self.node_capacity], int(it.value), int(how.value)

    def betweenness_unweighted(self):
        out = np.zeros(max(self.node_capacity, 1), np.float64)
        ovf = C.c_uint32(0)
        lib().og_betweenness_unweighted(self._h, out, C.byref(ovf))
        return out[: self.node_capacity], bool(ovf.value)

    def betweenness_sources(self, sources):
        src = np.ascontiguousarray(sources, dtype=np.uint32)
        out = np.zeros(max(self.node_capacity, 1), np.float64)
        ovf = C.c_uint32(0)
        lib().og_betweenness_sources(self._h, src, len(src), out, C.byref(ovf))
        return out[: self.node_capacity], bool(ovf.value)

    def betweenness_weighted(self, sources=None):
        """nif_betweenness_f64 restated (centrality.zig:528-682): every live
        source ascending, or `sources`."""
        out = np.zeros(max(self.node_capacity, 1), np.float64)
        ovf = C.c_uint32(0)
        if sources is None:
            lib().og_betweenness_weighted(self._h, None, 0, out, C.byref(ovf))
        else:
            src = np.ascontiguousarray(sources, dtype=np.uint32)
            lib().og_betweenness_weighted(self._h, src.ctypes.data, len(src), out, C.byref(ovf))
        return out[: self.node_capacity], bool(ovf.value)

    def bfs(self, s):
        V = self.node_capacity
        dist = np.zeros(V, np.uint32); sigma = np.zeros(V, np.uint64)
        ovf = C.c_uint32(0)
        lib().og_bfs(self._h, s, dist, sigma, C.byref(ovf))
        return dist, sigma, bool(ovf.value)


def rmat(scale: int, edge_factor: int, seed: int, a=0.57, b=0.19, c=0.19, directed=True):
    """Seeded R-MAT edge list (self-loops and duplicates removed, sorted), as
    (V, from, to) in insertion order."""
    L = lib()
    h = L.og_rmat(scale, edge_factor, seed, a, b, c, 1 if directed else 0)
    try:
        m = int(L.og_edges_count(h))
        V = int(L.og_edges_nodes(h))
        frm = np.zeros(max(m, 1), np.uint32); to = np.zeros(max(m, 1), np.uint32)
        L.og_edges_copy(h, frm, to)
    finally:
        L.og_edges_free(h)
    return V, frm[:m], to[:m]


def _edges(h):
    L = lib()
    try:
        m = int(L.og_edges_count(h))
        V = int(L.og_edges_nodes(h))
        frm = np.zeros(max(m, 1), np.uint32); to = np.zeros(max(m, 1), np.uint32)
        L.og_edges_copy(h, frm, to)
    finally:
        L.og_edges_free(h)
    return V, frm[:m], to[:m]


def barabasi_albert(n: int, m: int, seed: int, directed=True):
    """Seeded Barabasi-Albert edge list (V, from, to) in insertion order."""
    return _edges(lib().og_ba(n, m, seed, 1 if directed else 0))


def watts_strogatz(n: int, k: int, beta: float, seed: int, directed=False):
    """Seeded Watts-Strogatz edge list (V, from, to) in insertion order."""
    return _edges(lib().og_ws(n, k, beta, seed, 1 if directed else 0))


def rmat_raw(scale, seed, i0, m, a=0.57, b=0.19, c=0.19):
    src = np.zeros(m, np.uint32); dst = np.zeros(m, np.uint32)
    lib().og_rmat_raw(scale, seed, a, b, c, i0, m, src, dst)
    return src, dst


def read_edgelist(path: str, directed=True, integer_labels=False):
    """nif_read_edgelist restated; returns (ArrayGraph, next_id, labels)."""
    L = lib()
    nid = C.c_uint32(0); buf = C.c_char_p(); blen = C.c_uint64(0)
    h = L.og_read_edgelist(path.encode(), 1 if directed else 0, 1 if integer_labels else 0,
                           C.byref(nid), C.byref(buf), C.byref(blen))
    if not h:
        raise FileNotFoundError(path)
    raw = C.string_at(buf, blen.value) if blen.value else b""
    L.og_free_buf(buf)
    labels = raw.decode().split("\n") if raw else []
    return ArrayGraph(0, handle=h), int(nid.value), labels


def in_csr_from_edges(V, frm, to):
    """in_neighbors as a CSR with sources ascending per row (centrality.zig:893-899
    order) plus out-degrees, from an insertion-order edge list."""
    if len(frm) > 1_000_000:
        frm = np.ascontiguousarray(frm, np.uint32); to = np.ascontiguousarray(to, np.uint32)
        off = np.zeros(V + 1, np.uint64); col = np.zeros(max(len(frm), 1), np.uint32)
        deg = np.zeros(max(V, 1), np.uint32)
        lib().og_in_csr(V, frm, to, len(frm), off, col, deg)
        return off, col[: len(frm)], deg[:V]
    frm = np.asarray(frm, np.uint64); to = np.asarray(to, np.uint64)
    key = to * np.uint64(1 << 32) + frm
    order = np.argsort(key, kind="stable")
    col = frm[order].astype(np.uint32)
    counts = np.bincount(to.astype(np.int64), minlength=V)
    off = np.zeros(V + 1, np.uint64)
    off[1:] = np.cumsum(counts)
    outdeg = np.bincount(frm.astype(np.int64), minlength=V).astype(np.uint32)
    return off, col, outdeg


def pagerank_csr(V, in_off, in_col, outdeg, damping=0.85, max_iterations=100, tolerance=1e-4,
                 live=None):
    out = np.zeros(max(V, 1), np.float64)
    l1 = C.c_double(0); secs = C.c_double(0)
    lv = None
    if live is not None:
        lv = np.ascontiguousarray(live, dtype=np.uint8)
    it = lib().og_pagerank_csr(V, np.ascontiguousarray(in_off, np.uint64),
                               np.ascontiguousarray(in_col, np.uint32),
                               np.ascontiguousarray(outdeg, np.uint32),
                               lv.ctypes.data if lv is not None else None,
                               damping, max_iterations, tolerance, out, C.byref(l1), C.byref(secs))
    return out[:V], int(it), float(l1.value), float(secs.value)


def pagerank_ext(V, in_off, in_col, outdeg, x0=None, p=None, damping=0.85, max_iterations=100,
                 tolerance=1e-4):
    out = np.zeros(max(V, 1), np.float64)
    l1 = C.c_double(0)
    x0a = None if x0 is None else np.ascontiguousarray(x0, np.float64)
    pa = None if p is None else np.ascontiguousarray(p, np.float64)
    it = lib().og_pagerank_ext(V, np.ascontiguousarray(in_off, np.uint64),
                               np.ascontiguousarray(in_col, np.uint32),
                               np.ascontiguousarray(outdeg, np.uint32),
                               x0a.ctypes.data if x0a is not None else None,
                               pa.ctypes.data if pa is not None else None,
                               damping, max_iterations, tolerance, out, C.byref(l1))
    return out[:V], int(it), float(l1.value)


def betweenness_csr_sources(V, off, col, sources):
    out = np.zeros(max(V, 1), np.float64)
    ovf = C.c_uint32(0); secs = C.c_double(0)
    src = np.ascontiguousarray(sources, np.uint32)
    lib().og_betweenness_csr_sources(V, np.ascontiguousarray(off, np.uint64),
                                     np.ascontiguousarray(col, np.uint32), src, len(src), out,
                                     C.byref(ovf), C.byref(secs))
    return out[:V], bool(ovf.value), float(secs.value)


def pagerank_csr_mt(V, in_off, in_col, outdeg, damping=0.85, max_iterations=100, tolerance=1e-4,
                    x0=None, p=None, threads=0):
    """The reference PageRank loop with its row sums spread over host threads;
    iterates are bit for bit those of pagerank_csr (see og_pagerank_csr_mt).
    Returns (scores, iterations, last L1 step, loop seconds)."""
    out = np.zeros(max(V, 1), np.float64)
    l1 = C.c_double(0); secs = C.c_double(0)
    x0a = None if x0 is None else np.ascontiguousarray(x0, np.float64)
    pa = None if p is None else np.ascontiguousarray(p, np.float64)
    it = lib().og_pagerank_csr_mt(V, np.ascontiguousarray(in_off, np.uint64),
                                  np.ascontiguousarray(in_col, np.uint32),
                                  np.ascontiguousarray(outdeg, np.uint32),
                                  x0a.ctypes.data if x0a is not None else None,
                                  pa.ctypes.data if pa is not None else None,
                                  damping, max_iterations, tolerance, out, C.byref(l1), C.byref(secs),
                                  int(threads))
    return out[:V], int(it), float(l1.value), float(secs.value)


def bfs_csr_many(V, off, col, sources, threads=0):
    """Per-source BFS distances (0xFFFFFFFF = unreached) and wrapping u64 path
    counts over a successor CSR, sources spread over host threads.  Returns
    (dist [S, V] u32, sigma [S, V] u64, overflow [S] bool)."""
    src = np.ascontiguousarray(sources, np.uint32)
    S = len(src)
    dist = np.empty((S, max(V, 1)), np.uint32)
    sigma = np.empty((S, max(V, 1)), np.uint64)
    ovf = np.zeros(max(S, 1), np.uint8)
    lib().og_bfs_csr_many(V, np.ascontiguousarray(off, np.uint64), np.ascontiguousarray(col, np.uint32),
                          src, S, dist, sigma, ovf, int(threads))
    return dist[:, :V], sigma[:, :V], ovf[:S].astype(bool)


def betweenness_csr_sources_mt(V, off, col, sources, threads=0):
    """betweenness_csr_sources with the sources split over host threads; agrees
    with it to rounding (the sum over sources is taken in another order)."""
    out = np.zeros(max(V, 1), np.float64)
    ovf = C.c_uint32(0)
    src = np.ascontiguousarray(sources, np.uint32)
    lib().og_betweenness_csr_sources_mt(V, np.ascontiguousarray(off, np.uint64),
                                        np.ascontiguousarray(col, np.uint32), src, len(src), out,
                                        C.byref(ovf), int(threads))
    return out[:V], bool(ovf.value)
