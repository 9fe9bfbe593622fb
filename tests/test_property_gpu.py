"""Property-based parity on random small graphs, after the reference's own
(test/zog_parity_test.exs:71-135: StreamData, random undirected graphs of 1-15
nodes and at most 30 edges, 100 runs, copy-in, ResourceGraph and pure Elixir
compared to 1e-3).

Here each random graph -- directed or undirected, with self-loops, repeated
edges and isolated nodes -- goes through the ResourceGraph mirror (the C ABI on
the GPU) and through the copy-in/out Centrality API, and is compared with the
CPU oracle's ArrayGraph: PageRank (d 0.85, tol 1e-9, at most 200 iterations)
to relative L1 1e-9, betweenness to 1e-9 with the oracle's exact zeros, the
undirected halving included (resource_graph.ex:2633-2637).  Both APIs must
agree with each other bit for bit, since they run the same kernels."""
import numpy as np
import pytest
from hypothesis import HealthCheck, given, settings
from hypothesis import strategies as st

import zog_b200 as zog
from conftest import rel_l1

RG = zog.ResourceGraph
pytestmark = pytest.mark.gpu
TOL = 1e-9


@st.composite
def small_graphs(draw):
    n = draw(st.integers(1, 15))
    directed = draw(st.booleans())
    node = st.integers(0, n - 1)
    edges = draw(st.lists(st.tuples(node, node), max_size=30))
    return n, directed, edges


def _close(x, ref):
    x, ref = np.asarray(x, np.float64), np.asarray(ref, np.float64)
    if np.abs(ref).sum() == 0.0:
        return bool(np.all(x == 0.0))
    return rel_l1(x, ref) <= TOL


@settings(max_examples=100, deadline=None, suppress_health_check=[HealthCheck.too_slow])
@given(small_graphs())
def test_random_graphs_match_oracle(native, oracle, g):
    n, directed, edges = g
    b = zog.directed() if directed else zog.undirected()
    for i in range(n):
        b.add_node(i)  # labels 0..n-1 get ids 0..n-1
    for a, c in edges:
        b.add_edge(a, c, 1.0)
    f, t, _ = b.to_edge_arrays()

    res = RG.new(b)
    try:
        pr = RG.pagerank(res, 0.85, 200, TOL, raw=True)
        bc = RG.betweenness_unweighted(res, raw=True)
    finally:
        RG.destroy(res)
    C = zog.Centrality
    cpr = C.pagerank(b, 0.85, 200, TOL)
    cbc = C.betweenness_unweighted(b)
    assert [cpr[i] for i in range(n)] == pr
    assert [cbc[i] for i in range(n)] == bc

    A = oracle.ArrayGraph(n, np.asarray(f, np.uint32), np.asarray(t, np.uint32))
    try:
        ref_pr, _, _ = A.pagerank(0.85, 200, TOL)
        ref_bc, _ = A.betweenness_unweighted()
    finally:
        A.close()
    if not directed:
        ref_bc = ref_bc * 0.5
    assert _close(pr, ref_pr), (g, pr, ref_pr)
    assert _close(bc, ref_bc), (g, bc, ref_bc)
    assert np.array_equal(np.asarray(bc) == 0.0, ref_bc == 0.0), g
