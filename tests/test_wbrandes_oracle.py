"""The oracle's weighted (Dijkstra) Brandes -- the restatement of
centrality.zig:528-682 -- pinned on the CPU: the reference's own known answers
(test/centrality_test.exs:54-78), agreement with the unweighted path at unit
weights, and networkx's weighted betweenness on simple graphs."""
import networkx as nx
import numpy as np
import pytest


def test_known_answers_from_the_reference_tests(oracle):
    # "weighted bridge node has highest score" (centrality_test.exs:55-65): A->B->C
    bc, _ = oracle.ArrayGraph(3, [0, 1], [1, 2], [1.0, 1.0]).betweenness_weighted()
    assert bc[1] > bc[0] and bc[1] > bc[2]
    np.testing.assert_array_equal(bc, [0.0, 1.0, 0.0])
    # "weights affect shortest paths" (:67-77): A->B->C (2) beats A->C (10)
    bc, _ = oracle.ArrayGraph(3, [0, 1, 0], [1, 2, 2], [1.0, 1.0, 10.0]).betweenness_weighted()
    assert bc[1] > 0.0
    # with a cheaper direct arc B lies on no shortest path
    bc, _ = oracle.ArrayGraph(3, [0, 1, 0], [1, 2, 2], [1.0, 1.0, 1.5]).betweenness_weighted()
    assert bc[1] == 0.0


def test_unit_weights_equal_unweighted(oracle):
    for directed in (True, False):
        V, f, t = oracle.rmat(9, 8, 21, directed=directed)
        g = oracle.ArrayGraph(V, f, t)
        bu, _ = g.betweenness_unweighted()
        bw, _ = g.betweenness_weighted()
        assert np.abs(bu - bw).sum() <= 1e-12 * np.abs(bu).sum()


@pytest.mark.parametrize("directed,seed", [(True, 1), (False, 2), (True, 3)])
def test_weighted_matches_networkx(oracle, directed, seed):
    rng = np.random.default_rng(seed)
    V, f, t = oracle.rmat(8, 6, 40 + seed, directed=directed)
    if directed:
        w = rng.uniform(1.0, 10.0, f.size)
    else:  # both arcs of an edge share its weight
        w = np.repeat(rng.uniform(1.0, 10.0, f.size // 2), 2)
    bc, _ = oracle.ArrayGraph(V, f, t, w).betweenness_weighted()
    G = nx.DiGraph() if directed else nx.Graph()
    G.add_nodes_from(range(V))
    for a, b, x in zip(f.tolist(), t.tolist(), w.tolist()):
        G.add_edge(a, b, weight=x)
    ref = nx.betweenness_centrality(G, weight="weight", normalized=False)
    ref = np.array([ref[i] for i in range(V)])
    if not directed:
        ref = ref * 2.0  # networkx halves undirected scores; the Zig core does not
    assert np.abs(bc - ref).sum() <= 1e-9 * np.abs(ref).sum()


def test_integer_weights_count_tied_paths(oracle):
    # a 2 x 3 grid with unit weights plus a diagonal arc of weight 2 that ties
    # with the two-step paths: several equal shortest paths per pair
    frm = [0, 1, 3, 4, 0, 1, 2, 0]
    to = [1, 2, 4, 5, 3, 4, 5, 4]
    w = [1.0, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0, 2.0]
    bc, _ = oracle.ArrayGraph(6, frm, to, w).betweenness_weighted()
    G = nx.MultiDiGraph()
    G.add_nodes_from(range(6))
    for a, b, x in zip(frm, to, w):
        G.add_edge(a, b, weight=x)
    ref = nx.betweenness_centrality(nx.DiGraph(G), weight="weight", normalized=False)
    np.testing.assert_allclose(bc, [ref[i] for i in range(6)], rtol=1e-12, atol=1e-12)
