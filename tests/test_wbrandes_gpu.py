"""Weighted (Dijkstra) Brandes on the GPU against the oracle's restatement of
centrality.zig:528-682: relative L1 <= 1e-9 with exact zeros, on real-valued
and integer weights (many tied shortest paths), directed and undirected
graphs, multi-arcs, deleted nodes, source subsets; unit weights reproduce the
unweighted kernels; bad weights are rejected."""
import numpy as np
import pytest

from conftest import rel_l1

pytestmark = pytest.mark.gpu
TOL = 1e-9


def compare(native, oracle, V, f, t, w, sources=None, name=""):
    G = native.Graph.from_edges(V, f, t, w)
    try:
        bc = G.betweenness_weighted(sources=sources)
        ref, _ = oracle.ArrayGraph(V, f, t, w).betweenness_weighted(sources)
        assert rel_l1(bc, ref) <= TOL, (name, rel_l1(bc, ref))
        assert np.all(bc[ref == 0.0] == 0.0), name
        return bc
    finally:
        G.destroy()


def test_known_answers(native, oracle):
    bc = compare(native, oracle, 3, np.array([0, 1], np.uint32), np.array([1, 2], np.uint32), np.array([1.0, 1.0]))
    np.testing.assert_array_equal(bc, [0.0, 1.0, 0.0])
    bc = compare(native, oracle, 3, np.array([0, 1, 0], np.uint32), np.array([1, 2, 2], np.uint32),
                 np.array([1.0, 1.0, 10.0]))
    assert bc[1] > 0.0


@pytest.mark.parametrize("directed,kind,scale", [(True, "real", 10), (False, "real", 10), (True, "int", 10),
                                                 (False, "int", 9), (True, "real", 12)])
def test_weighted_matches_oracle(native, oracle, directed, kind, scale):
    rng = np.random.default_rng(scale + (0 if directed else 100))
    V, f, t = oracle.rmat(scale, 8, 300 + scale, directed=directed)
    m = f.size if directed else f.size // 2
    w = rng.uniform(0.5, 20.0, m) if kind == "real" else rng.integers(1, 4, m).astype(np.float64)
    if not directed:
        w = np.repeat(w, 2)
    src = None if scale <= 10 else np.arange(0, V, 7, dtype=np.uint32)
    compare(native, oracle, V, f, t, w, src, f"{directed}-{kind}-{scale}")


def test_multi_arcs_self_loops_and_unit_weights(native, oracle):
    rng = np.random.default_rng(5)
    V = 300
    f = rng.integers(0, V, 2500).astype(np.uint32)
    t = rng.integers(0, V, 2500).astype(np.uint32)
    f[:40] = t[:40]                       # self-loops
    f[40:80], t[40:80] = f[80:120], t[80:120]  # duplicated arcs
    w = rng.integers(1, 3, f.size).astype(np.float64)
    compare(native, oracle, V, f, t, w, name="multi")
    # no weights: every weight 1.0, the unweighted kernels' result
    G = native.Graph.from_edges(V, f, t)
    try:
        np.testing.assert_array_equal(G.export_weights(), np.ones(f.size))
        bw = G.betweenness_weighted()
        bu = G.betweenness_unweighted()
        assert rel_l1(bw, bu) <= TOL
    finally:
        G.destroy()


def test_arraygraph_with_deleted_nodes(native, oracle):
    rng = np.random.default_rng(8)
    V = 200
    f = rng.integers(0, V, 1200).astype(np.uint32)
    t = rng.integers(0, V, 1200).astype(np.uint32)
    w = rng.uniform(1.0, 5.0, f.size)
    ag = oracle.ArrayGraph(V, f, t, w)
    for node in (3, 50, 199):
        ag.remove_node(node)
    fe, nd, to, ne, ed, data = ag.export()
    G = native.Graph.from_arraygraph(fe, nd, to, ne, ed, data)
    try:
        bc = G.betweenness_weighted()
        ref, _ = ag.betweenness_weighted()
        assert rel_l1(bc, ref) <= TOL
        assert bc[3] == 0.0 and bc[50] == 0.0
    finally:
        G.destroy()


def test_bad_weights_are_rejected(native):
    for bad in (0.0, -1.0, np.inf, np.nan):
        G = native.Graph.from_edges(3, np.array([0, 1], np.uint32), np.array([1, 2], np.uint32),
                                    np.array([1.0, bad]))
        try:
            with pytest.raises(native.ZogCudaError):
                G.betweenness_weighted()
        finally:
            G.destroy()


def test_zero_length_arc_reported_from_a_lane(native, monkeypatch):
    """An arc of effective length zero on a shortest path (fl(d + w) == d)
    makes the reference's sigma depend on its heap's tie order, so it is an
    error.  The check runs inside the batches, which lanes with their own host
    threads drive: with 160 sources (five batches over four lanes) and the
    error in a worker thread's batch, the status and the message must still
    reach the caller, and the call must end."""
    monkeypatch.setenv("ZOGCU_BC_STREAMS", "4")
    n = 160
    # nodes 0-31 (the first batch, lane 0 on the calling thread) are isolated;
    # a chain 32 -> 33 -> ... -> 159 with the arc 40 -> 41 of weight 1e20, so
    # only sources 32-40 (the second batch, lane 1 on a worker thread) see
    # fl(d(41) + 1) == d(41) on the shortest path to 42
    f = np.arange(32, n - 1).astype(np.uint32)
    t = (f + 1).astype(np.uint32)
    w = np.ones(f.size)
    w[40 - 32] = 1e20
    G = native.Graph.from_edges(n, f, t, w)
    try:
        with pytest.raises(native.ZogCudaError) as ei:
            G.betweenness_weighted()
        assert ei.value.status == 1
        assert "effective length zero" in str(ei.value)
    finally:
        G.destroy()
