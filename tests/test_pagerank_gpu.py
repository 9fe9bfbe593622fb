"""PageRank parity: the CUDA path (through the C ABI) against the CPU oracle.

Tolerance (FP64 form): relative L1 <= 1e-9 against the oracle, and the same
iteration count.  Rows summed by one thread use the reference's summation
order, so most graphs come out bit-identical; longer rows are reassociated.
"""
import json
import os

import numpy as np
import pytest

from conftest import GOLDEN, rel_l1

pytestmark = pytest.mark.gpu
TOL = 1e-9
N_CONFIGS = 11  # kernel configurations of pr_iter_kernel / pr_iter_kernel_pipe


def golden(name):
    return dict(np.load(os.path.join(GOLDEN, name + ".npz")))


def golden_names():
    with open(os.path.join(GOLDEN, "manifest.json")) as f:
        return sorted(json.load(f))


@pytest.mark.parametrize("name", golden_names())
def test_golden_pagerank(native, name):
    g = golden(name)
    V = int(g["V"])
    if "ag_first_edge" in g:
        G = native.Graph.from_arraygraph(g["ag_first_edge"], g["ag_node_deleted"], g["ag_to"], g["ag_next_edge"],
                                         g["ag_edge_deleted"])
    else:
        G = native.Graph.from_edges(V, g["from"], g["to"])
    try:
        for key, (d, it, tol) in {"pr_default": (0.85, 100, 1e-4), "pr_tight": (0.85, 200, 1e-9),
                                  "pr_d99": (0.99, 100, 1e-4)}.items():
            x, st = G.pagerank(d, it, tol, stats=True)
            assert x.shape == g[key].shape
            assert rel_l1(x, g[key]) <= TOL, key
            if V > 1:
                assert st["iterations"] == int(g[key + "_iters"]), key
    finally:
        G.destroy()


def test_rmat_scale14_config(native, oracle):
    """Directed R-MAT scale 14, ef 8 (131,072 raw edges), d 0.85, tol 1e-9, 200 iterations."""
    V, f, t = oracle.rmat(14, 8, 1014, directed=True)
    G = native.Graph.from_edges(V, f, t)
    try:
        x, st = G.pagerank(0.85, 200, 1e-9, stats=True)
        ref, it, l1 = oracle.ArrayGraph(V, f, t).pagerank(0.85, 200, 1e-9)
        assert rel_l1(x, ref) <= TOL
        assert st["iterations"] == it
        # the L1 step is a sum of differences of nearly equal values, so it only
        # agrees to a few digits once the row sums are reassociated
        assert abs(st["residual"] - l1) <= 1e-3 * l1 and st["residual"] < 1e-9
    finally:
        G.destroy()


def test_device_generator_matches_oracle_generator(native, oracle):
    """The CUDA R-MAT generator and the oracle's produce the same graph."""
    for scale, directed in ((12, True), (11, False)):
        V, f, t = oracle.rmat(scale, 8, 77 + scale, directed=directed)
        G = native.Graph.rmat(scale, 8, 77 + scale, directed=directed)
        try:
            in_off, in_col, out_off, out_col, deg = G.export_csr()
            off_r, col_r, deg_r = oracle.in_csr_from_edges(V, f, t)
            assert np.array_equal(in_off, off_r) and np.array_equal(in_col, col_r)
            assert np.array_equal(deg, deg_r)
        finally:
            G.destroy()
    s, d = native.rmat_raw_device(10, 1010, 0, 4096)
    g = golden("rmat10_dir")
    assert np.array_equal(s, g["raw_src"]) and np.array_equal(d, g["raw_dst"])


def test_in_csr_order_matches_reference(native, oracle):
    """in-CSR rows hold sources ascending (centrality.zig:893-899) and the
    out-CSR rows successors in reverse insertion order (array_graph.zig:94-104)."""
    g = golden("multi_selfloop")
    V = int(g["V"])
    G = native.Graph.from_edges(V, g["from"], g["to"])
    try:
        in_off, in_col, out_off, out_col, deg = G.export_csr()
        off_r, col_r, deg_r = oracle.in_csr_from_edges(V, g["from"], g["to"])
        assert np.array_equal(in_off, off_r) and np.array_equal(in_col, col_r) and np.array_equal(deg, deg_r)
        so, sc = oracle.ArrayGraph(V, g["from"], g["to"]).successor_csr()
        assert np.array_equal(out_off, so) and np.array_equal(out_col, sc)
    finally:
        G.destroy()


@pytest.mark.parametrize("sources_sorted", [True, False])
def test_large_host_arc_lists_build_the_reference_csr(native, oracle, sources_sorted):
    """Host arc lists of at least 2^22 arcs have their destinations sorted on
    the device while the sources are still being copied; when the sources
    are non-decreasing the in-CSR is then a gather of them, otherwise the
    plain two-sort build runs.  Both against the oracle's CSRs, with
    self-loops and duplicate arcs, from pageable arrays large enough for the
    pipelined bounce copies (33.5 MB each)."""
    rng = np.random.default_rng(2023)
    V, E = 1 << 16, (1 << 23) + 7
    f = rng.integers(0, V, E, dtype=np.uint32)
    t = rng.integers(0, V, E, dtype=np.uint32)
    t[:1000] = f[:1000]  # self-loops
    f[1000:3000] = f[1000]  # a hub with duplicate arcs
    t[1000:3000] = t[1000:1100].repeat(20)
    if sources_sorted:
        order = np.argsort(f, kind="stable")
        f, t = np.ascontiguousarray(f[order]), np.ascontiguousarray(t[order])
    G = native.Graph.from_edges(V, f, t)
    try:
        in_off, in_col, out_off, out_col, deg = G.export_csr()
        off_r, col_r, deg_r = oracle.in_csr_from_edges(V, f, t)
        assert np.array_equal(in_off, off_r) and np.array_equal(in_col, col_r) and np.array_equal(deg, deg_r)
        A = oracle.ArrayGraph(V, f, t)
        try:
            so, sc = A.successor_csr()
        finally:
            A.close()
        assert np.array_equal(out_off, so) and np.array_equal(out_col, sc)
    finally:
        G.destroy()


@pytest.mark.parametrize("runs", ["1", "0"])
def test_sorted_sources_sent_as_runs_build_the_reference_csr(native, oracle, monkeypatch, runs):
    """Sorted host sources cross PCIe as per-chunk run offsets when those take
    at most half the chunk's bytes, and as they are otherwise.  Here the first
    chunks hold 100 heavy sources whose runs cross chunk boundaries (coded),
    the last ones sources spread over every node with gaps between them (sent
    as they are); with the coding switched off (ZOGCU_UPLOAD_RUNS=0) every
    chunk is sent as it is.  Both CSRs against the oracle's."""
    monkeypatch.setenv("ZOGCU_UPLOAD_RUNS", runs)
    rng = np.random.default_rng(404)
    V = 1 << 21
    f = np.concatenate([rng.integers(0, V, 1 << 21), rng.integers(1000, 1100, (1 << 21) + 11)]).astype(np.uint32)
    f.sort()
    t = rng.integers(0, V, f.size, dtype=np.uint32)
    G = native.Graph.from_edges(V, f, t)
    try:
        in_off, in_col, out_off, out_col, deg = G.export_csr()
        off_r, col_r, deg_r = oracle.in_csr_from_edges(V, f, t)
        assert np.array_equal(in_off, off_r) and np.array_equal(in_col, col_r) and np.array_equal(deg, deg_r)
        A = oracle.ArrayGraph(V, f, t)
        try:
            so, sc = A.successor_csr()
        finally:
            A.close()
        assert np.array_equal(out_off, so) and np.array_equal(out_col, sc)
    finally:
        G.destroy()


@pytest.mark.parametrize("bad", ["from", "to"])
def test_large_host_arc_list_with_missing_node_is_rejected(native, bad):
    """An endpoint >= node_count in a chunk-uploaded arc list is reported as
    node not found (addEdge's hasNode check, array_graph.zig:88-89); the
    chunks' destination counts skip such keys before validation runs."""
    rng = np.random.default_rng(7)
    V, E = 1 << 12, (1 << 22) + 3
    f = np.sort(rng.integers(0, V, E, dtype=np.uint32))
    t = rng.integers(0, V, E, dtype=np.uint32)
    (f if bad == "from" else t)[E // 2] = V + 5
    with pytest.raises(native.ZogCudaError) as ei:
        native.Graph.from_edges(V, f, t)
    assert ei.value.status == 2


@pytest.mark.parametrize("max_iter", [0, 1, 2, 7, 60])
def test_iteration_prefix_exact(native, oracle, max_iter):
    """Stopping after k iterations returns the k-th iterate (the swap happens
    before the tolerance test, centrality.zig:953-957).  60 iterations run as
    a CUDA-graph while loop that must stop exactly at max_iter."""
    V, f, t = oracle.rmat(13, 8, 4242, directed=True)
    G = native.Graph.from_edges(V, f, t)
    try:
        x, st = G.pagerank(0.85, max_iter, 0.0, stats=True)
        ref, it, _ = oracle.ArrayGraph(V, f, t).pagerank(0.85, max_iter, 0.0)
        assert st["iterations"] == it == max_iter
        assert rel_l1(x, ref) <= 1e-13
    finally:
        G.destroy()


def test_heavy_rows_use_long_row_chunks(native, oracle):
    """A hub with in-degree far above one block (2048 arcs) and many medium rows."""
    rng = np.random.default_rng(5)
    V = 20000
    hub_src = rng.integers(0, V, 50000).astype(np.uint32)
    f = np.concatenate([hub_src, rng.integers(0, V, 60000).astype(np.uint32), np.arange(1, 400, dtype=np.uint32)])
    t = np.concatenate([np.zeros(50000, np.uint32), rng.integers(0, 300, 60000).astype(np.uint32),
                        np.full(399, 7, np.uint32)])
    G = native.Graph.from_edges(V, f, t)
    try:
        x, st = G.pagerank(0.85, 200, 1e-10, stats=True)
        ref, it, _ = oracle.ArrayGraph(V, f, t).pagerank(0.85, 200, 1e-10)
        assert rel_l1(x, ref) <= TOL and st["iterations"] == it
        x2 = G.pagerank(0.85, 200, 1e-10)
        assert np.array_equal(x, x2)  # deterministic reduction order
    finally:
        G.destroy()


@pytest.mark.parametrize("cfg", range(N_CONFIGS))
def test_every_kernel_configuration_matches_oracle(native, oracle, cfg):
    """Each kernel configuration (hub sizes, item sizes, pipelined gathers),
    forced with ZOGCU_PR_CONFIG, on a graph with row blocks, single heavy rows
    and chunked long rows, in FP64 and in the precision form."""
    rng = np.random.default_rng(11 + cfg)
    V = 30000
    f = np.concatenate([rng.integers(0, V, 40000), rng.integers(0, V, 150000), rng.integers(0, V, 9000)])
    t = np.concatenate([np.zeros(40000, np.int64), rng.integers(0, V, 150000), rng.integers(1, 40, 9000)])
    f = f.astype(np.uint32); t = t.astype(np.uint32)
    ref, it, _ = oracle.ArrayGraph(V, f, t).pagerank(0.85, 200, 1e-10)
    G = native.Graph.from_edges(V, f, t)
    try:
        os.environ["ZOGCU_PR_CONFIG"] = str(cfg)  # read by the graph's first solve
        try:
            x, st = G.pagerank(0.85, 200, 1e-10, stats=True)
        finally:
            del os.environ["ZOGCU_PR_CONFIG"]
        assert st["kernel_config"] == cfg
        assert rel_l1(x, ref) <= TOL and st["iterations"] == it
        assert np.array_equal(x, G.pagerank(0.85, 200, 1e-10))
        xm = G.pagerank(0.85, 200, 1e-10, precision=native.PREC_MIXED)
        assert rel_l1(xm, ref) <= 12e-10
    finally:
        G.destroy()


def test_warm_start_and_personalised(native, oracle):
    """Extensions against the generalised oracle: a start vector x0 and a
    personalisation (teleport) vector p."""
    V, f, t = oracle.rmat(12, 8, 99, directed=True)
    off, col, deg = oracle.in_csr_from_edges(V, f, t)
    rng = np.random.default_rng(1)
    x0 = rng.random(V); x0 /= x0.sum()
    p = np.zeros(V); p[rng.integers(0, V)] = 1.0
    G = native.Graph.from_edges(V, f, t)
    try:
        x = G.pagerank(0.85, 200, 1e-10, x0=x0)
        ref, it, _ = oracle.pagerank_ext(V, off, col, deg, x0=x0, max_iterations=200, tolerance=1e-10)
        assert rel_l1(x, ref) <= TOL
        x = G.pagerank(0.85, 200, 1e-10, teleport=p)
        ref, it, _ = oracle.pagerank_ext(V, off, col, deg, p=p, max_iterations=200, tolerance=1e-10)
        assert rel_l1(x, ref) <= TOL
    finally:
        G.destroy()


@pytest.mark.slow
def test_large_graph_properties(native, oracle):
    """Directed R-MAT scale 20 (ef 16): the oracle's first iterations agree, the
    converged vector sums to 1 and its own next step is below tolerance."""
    G = native.Graph.rmat(20, 16, 1020, directed=True)
    try:
        V, E, n = G.info()
        in_off, in_col, _, _, deg = G.export_csr()
        for k in (1, 3):
            x = G.pagerank(0.85, k, 0.0)
            ref, it, _, _ = oracle.pagerank_csr(V, in_off, in_col, deg, 0.85, k, 0.0)
            # the oracle sums ~5e5 dangling terms sequentially (as the reference
            # does); its own rounding, not the GPU's, dominates this difference
            assert rel_l1(x, ref) <= 1e-11
        x, st = G.pagerank(0.85, 200, 1e-9, stats=True)
        assert abs(x.sum() - 1.0) < 1e-9
        y, it, l1, _ = oracle.pagerank_csr(V, in_off, in_col, deg, 0.85, 1, 0.0)  # from uniform
        assert st["residual"] < 1e-9 and st["iterations"] < 200
    finally:
        G.destroy()


@pytest.mark.parametrize("scale", [13, 16])
def test_mixed_precision_bound(native, oracle, scale):
    """Precision form: FP32 contributions, FP64 sums / residual / dangling,
    then an FP64 polish to the same L1 step.  Both results satisfy
    ||x - x*||_1 <= d/(1-d) * tol (Sigma x = 1), so they differ from the FP64
    oracle's by at most 2 * d/(1-d) * tol < 12 * tol."""
    V, f, t = oracle.rmat(scale, 16, 500 + scale, directed=True)
    G = native.Graph.from_edges(V, f, t)
    try:
        tol = 1e-10
        x, st = G.pagerank(0.85, 200, tol, precision=native.PREC_MIXED, stats=True)
        ref, it, _ = oracle.ArrayGraph(V, f, t).pagerank(0.85, 200, tol)
        assert rel_l1(x, ref) <= 12 * tol
        assert st["residual"] < tol and st["polish_iterations"] >= 1
        assert st["iterations"] > st["polish_iterations"]
        x64 = G.pagerank(0.85, 200, tol)
        assert rel_l1(x64, ref) <= TOL
    finally:
        G.destroy()


@pytest.mark.slow
def test_in_solve_tuning_matches_each_configuration(native):
    """Directed R-MAT scale 19 (ef 16, > 2^22 arcs): the first solve on a graph
    times each kernel configuration on its own early iterations and finishes
    with the fastest.  Its result agrees with a solve forced to any one
    configuration, and later solves reuse the choice and repeat bit for bit."""
    G = native.Graph.rmat(19, 16, 1919, directed=True)
    try:
        V, E, _ = G.info()
        assert E >= 1 << 22
        x, st = G.pagerank(0.85, 200, 1e-10, stats=True)
        x2, st2 = G.pagerank(0.85, 200, 1e-10, stats=True)
        assert st2["kernel_config"] == st["kernel_config"]
        assert np.array_equal(x2, G.pagerank(0.85, 200, 1e-10))
        in_off, in_col, out_off, out_col, deg = G.export_csr()
    finally:
        G.destroy()
    src = np.repeat(np.arange(V, dtype=np.uint32), np.diff(out_off).astype(np.int64))
    for cfg in range(N_CONFIGS):
        os.environ["ZOGCU_PR_CONFIG"] = str(cfg)
        try:
            H = native.Graph.from_edges(V, src, out_col)
            y, sty = H.pagerank(0.85, 200, 1e-10, stats=True)
            H.destroy()
        finally:
            del os.environ["ZOGCU_PR_CONFIG"]
        assert sty["kernel_config"] == cfg
        assert rel_l1(x, y) <= 1e-12
        assert abs(sty["iterations"] - st["iterations"]) <= 1


def test_graphs_reuse_pool_memory_and_release_it(native, oracle):
    """Graph arrays come from the device's stream-ordered pool: destroying a
    graph and building it again gives the same scores, and
    zogcu_release_cached_memory hands the pool's reserve back to the driver."""
    import torch

    V, f, t = oracle.rmat(14, 8, 3141, directed=True)
    ref, it, _ = oracle.ArrayGraph(V, f, t).pagerank(0.85, 200, 1e-10)
    first = None
    for _ in range(3):
        G = native.Graph.from_edges(V, f, t)
        try:
            x = G.pagerank(0.85, 200, 1e-10)
        finally:
            G.destroy()
        assert rel_l1(x, ref) <= TOL
        if first is None:
            first = x
        assert np.array_equal(x, first)
    free_before, _ = torch.cuda.mem_get_info()
    native.release_cached_memory()
    free_after, _ = torch.cuda.mem_get_info()
    assert free_after >= free_before
    G = native.Graph.from_edges(V, f, t)
    try:
        assert np.array_equal(G.pagerank(0.85, 200, 1e-10), first)
    finally:
        G.destroy()


@pytest.mark.parametrize("order", ["sorted", "shuffled"])
def test_csr_build_sorted_and_unsorted_sources(native, oracle, order):
    """The CSR build places the out-CSR with one scatter when the sources come
    non-decreasing, and sorts otherwise.  Both give the reference's successor
    order (reverse insertion, array_graph.zig:94-104), in-neighbour order and
    weights; multi-arcs and self-loops included."""
    rng = np.random.default_rng(8 if order == "sorted" else 9)
    V = 5000
    f = rng.integers(0, V, 60000).astype(np.uint32)
    t = rng.integers(0, V, 60000).astype(np.uint32)
    t[:500] = f[:500]                                    # self-loops
    f = np.concatenate([f, f[:3000]]); t = np.concatenate([t, t[:3000]])  # multi-arcs
    if order == "sorted":
        p = np.argsort(f, kind="stable"); f, t = f[p], t[p]
    w = rng.uniform(1.0, 100.0, f.size)
    G = native.Graph.from_edges(V, f, t, weight=w)
    try:
        in_off, in_col, out_off, out_col, deg = G.export_csr()
        off_r, col_r, deg_r = oracle.in_csr_from_edges(V, f, t)
        assert np.array_equal(in_off, off_r) and np.array_equal(in_col, col_r) and np.array_equal(deg, deg_r)
        so, sc = oracle.ArrayGraph(V, f, t).successor_csr()
        assert np.array_equal(out_off, so) and np.array_equal(out_col, sc)
        # weights in successor order: each source's arcs, last inserted first
        wexp = np.concatenate([w[np.flatnonzero(f == v)][::-1] for v in range(V)])
        assert np.array_equal(G.export_weights(), wexp)
        x = G.pagerank(0.85, 100, 1e-10)
        ref, it, _ = oracle.ArrayGraph(V, f, t).pagerank(0.85, 100, 1e-10)
        assert rel_l1(x, ref) <= TOL
    finally:
        G.destroy()
