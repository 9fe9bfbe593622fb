"""Propagation-blocked FP32 phase of the precision form (ZOGCU_PR_BLOCKED=1
forces it on graphs below its default of 2^23 nodes and 2^24 arcs).

The blocked iteration computes the same update as the gather kernels from
the same FP32 contributions; only the row sums differ: each message is
rounded to a multiple of 2^-56 and the sums are exact integers, so they do
not depend on the order of the additions.  Bars:
  * precision form against the FP64 oracle: rel L1 <= 2 * d/(1-d) * tol
    (< 12 * tol), as for the gather form (tests/test_pagerank_gpu.py);
  * FP32 iterates against the gather kernels' FP32 iterates: rel L1 <= 1e-6
    (both carry FP32 contributions);
  * repeated solves are bit-identical.
The graphs span several row partitions (24,576 rows or about 2^20 arcs
each) and source blocks, include dangling nodes, duplicate arcs, self-loops,
deleted nodes and a row of more than 2^20 arcs.
"""
import os

import numpy as np
import pytest

from conftest import rel_l1

pytestmark = pytest.mark.gpu


class Blocked:
    def __init__(self, value):
        self.value = value

    def __enter__(self):
        self.old = os.environ.get("ZOGCU_PR_BLOCKED")
        os.environ["ZOGCU_PR_BLOCKED"] = self.value

    def __exit__(self, *exc):
        if self.old is None:
            del os.environ["ZOGCU_PR_BLOCKED"]
        else:
            os.environ["ZOGCU_PR_BLOCKED"] = self.old


def hub_graph(seed=5):
    """30,000 nodes: 1.1M arcs into node 7 (one row above 2^20 arcs), random
    arcs with duplicates and self-loops, nodes 29,000+ dangling."""
    rng = np.random.default_rng(seed)
    V = 30000
    f = np.concatenate([rng.integers(0, 29000, 1_100_000), rng.integers(0, 29000, 300_000),
                        np.arange(100, 200), np.arange(100, 200)])
    t = np.concatenate([np.full(1_100_000, 7), rng.integers(0, V, 300_000), np.arange(100, 200),
                        np.arange(150, 250)])
    return V, f.astype(np.uint32), t.astype(np.uint32)


@pytest.mark.parametrize("which", ["rmat16", "rmat17", "hub"])
def test_blocked_precision_form_bound(native, oracle, which):
    if which == "hub":
        V, f, t = hub_graph()
    else:
        s = int(which[4:])
        V, f, t = oracle.rmat(s, 16, 700 + s, directed=True)
    tol = 1e-10
    ref, it, _ = oracle.ArrayGraph(V, f, t).pagerank(0.85, 200, tol)
    G = native.Graph.from_edges(V, f, t)
    try:
        with Blocked("1"):
            x, st = G.pagerank(0.85, 200, tol, precision=native.PREC_MIXED, stats=True)
            x2 = G.pagerank(0.85, 200, tol, precision=native.PREC_MIXED)
        assert st["reserved"] == 1, "the blocked FP32 phase did not run"
        assert rel_l1(x, ref) <= 12 * tol
        assert st["residual"] < tol and st["polish_iterations"] >= 1
        assert st["iterations"] > st["polish_iterations"]
        assert np.array_equal(x, x2)
        assert np.all(x >= 0) and abs(x.sum() - 1.0) < 1e-9
    finally:
        G.destroy()


@pytest.mark.parametrize("k", [1, 4])
def test_blocked_fp32_iterates_match_gather_kernels(native, oracle, k):
    """k FP32 iterations only (max_iterations = k leaves the polish none):
    blocked against the gather kernels and against the oracle's FP64
    iterates."""
    V, f, t = oracle.rmat(16, 16, 716, directed=True)
    in_ref, _, _ = oracle.ArrayGraph(V, f, t).pagerank(0.85, k, 0.0)
    G = native.Graph.from_edges(V, f, t)
    try:
        with Blocked("1"):
            xb, sb = G.pagerank(0.85, k, 0.0, precision=native.PREC_MIXED, stats=True)
        with Blocked("0"):
            xg, sg = G.pagerank(0.85, k, 0.0, precision=native.PREC_MIXED, stats=True)
        assert sb["reserved"] == 1 and sg["reserved"] == 0
        assert sb["iterations"] == sg["iterations"] == k
        assert rel_l1(xb, xg) <= 1e-6
        assert rel_l1(xb, in_ref) <= 1e-6
    finally:
        G.destroy()


def test_blocked_with_start_and_teleport(native, oracle):
    """Warm start and personalised teleport in the precision form, against the
    generalised oracle."""
    V, f, t = oracle.rmat(16, 8, 816, directed=True)
    rng = np.random.default_rng(3)
    off, col, deg = oracle.in_csr_from_edges(V, f, t)
    x0 = rng.random(V)
    x0 /= x0.sum()
    p = np.zeros(V)
    p[rng.choice(V, 3, replace=False)] = 1.0 / 3
    tol = 1e-10
    G = native.Graph.from_edges(V, f, t)
    try:
        with Blocked("1"):
            x, st = G.pagerank(0.85, 200, tol, precision=native.PREC_MIXED, x0=x0, teleport=p, stats=True)
        assert st["reserved"] == 1
        ref, _, _ = oracle.pagerank_ext(V, off, col, deg, x0=x0, p=p, max_iterations=200, tolerance=tol)
        assert rel_l1(x, ref) <= 12 * tol
    finally:
        G.destroy()


def test_blocked_with_deleted_nodes(native, oracle):
    """An ArrayGraph with deleted nodes (tombstones): their slots score 0."""
    V, f, t = oracle.rmat(16, 8, 916, directed=True)
    ag = oracle.ArrayGraph(V, f, t)
    rng = np.random.default_rng(4)
    for node in rng.choice(V, 300, replace=False):
        ag.remove_node(int(node))
    tol = 1e-10
    ref, _, _ = ag.pagerank(0.85, 200, tol)
    fe, nd, to, ne, ed, _ = ag.export()
    G = native.Graph.from_arraygraph(fe, nd, to, ne, ed)
    try:
        with Blocked("1"):
            x, st = G.pagerank(0.85, 200, tol, precision=native.PREC_MIXED, stats=True)
        assert st["reserved"] == 1
        assert rel_l1(x, ref) <= 12 * tol
        assert np.all(x[nd == 1] == 0.0)
    finally:
        G.destroy()
