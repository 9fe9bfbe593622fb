"""Host-side logic of the ResourceGraph mirror (CPU only): SoA id assignment
and arc order, result shaping, undirected halving.  The native graph is
replaced by a stub that returns fixed scores, so no GPU is needed."""
import numpy as np
import pytest

import zog_b200 as zog
from zog_b200 import resource_graph as RG


def test_soa_ids_and_arc_order():
    """soa.ex:85-128: ids by first appearance; undirected edges store the
    forward then the reverse arc; to_edge_arrays in insertion order."""
    b = zog.undirected().add_edge("A", "B", 1).add_edge("B", "C", 2.5).add_node("D")
    assert b.label_to_id == {"A": 0, "B": 1, "C": 2, "D": 3}
    f, t, w = b.to_edge_arrays()
    assert f.tolist() == [0, 1, 1, 2] and t.tolist() == [1, 0, 2, 1]
    assert w.tolist() == [1.0, 1.0, 2.5, 2.5]
    assert b.node_count() == 4 and b.edge_count() == 4
    assert b.nodes == ["D", "C", "B", "A"]
    assert b.all_labels() == ["A", "B", "C", "D"]


def test_soa_weight_coercion():
    """soa.ex:282-285: nil / non-numbers give 1.0, integers become floats."""
    b = zog.directed().add_edge(1, 2, None).add_edge(2, 3, "x").add_edge(3, 1, 4)
    assert b.to_edge_arrays()[2].tolist() == [1.0, 1.0, 4.0]


def test_soa_bulk_matches_single_adds():
    a = zog.undirected()
    for i in range(5):
        a.ensure_node(i)
    a.add_id_edges([0, 1, 3], [1, 2, 4])
    b = zog.undirected()
    for i in range(5):
        b.ensure_node(i)
    for s, d in ((0, 1), (1, 2), (3, 4)):
        b.add_edge(s, d)
    for x, y in zip(a.to_edge_arrays(), b.to_edge_arrays()):
        assert np.array_equal(x, y)


class StubGraph:
    def __init__(self, scores):
        self.scores = np.asarray(scores, np.float64)

    def pagerank(self, *a, **k):
        return self.scores.copy()

    def betweenness_unweighted(self, sources=None):
        return self.scores.copy()

    def destroy(self):
        self.destroyed = True


def test_map_scores_labels_and_raw():
    """resource_graph.ex:2609-2619 and 1672-1685: labels via reversed nodes; raw list."""
    b = zog.directed().add_edge("x", "y").add_edge("y", "z")
    g = RG.ResourceGraph(StubGraph([0.1, 0.2, 0.7]), b)
    assert RG.pagerank(g) == {"x": 0.1, "y": 0.2, "z": 0.7}
    assert RG.pagerank(g, raw=True) == [0.1, 0.2, 0.7]


def test_integer_labels_shape():
    b = zog.SoA.with_integer_ids("directed", 3)
    g = RG.ResourceGraph(StubGraph([0.5, 0.25, 0.25]), b)
    assert RG.pagerank(g) == {0: 0.5, 1: 0.25, 2: 0.25}


def test_undirected_betweenness_is_halved_before_shaping():
    """resource_graph.ex:1591-1601 + 2633-2637."""
    b = zog.undirected().add_edge("A", "B").add_edge("B", "C")
    g = RG.ResourceGraph(StubGraph([0.0, 2.0, 0.0]), b)
    assert RG.betweenness_unweighted(g) == {"A": 0.0, "B": 1.0, "C": 0.0}
    assert RG.betweenness_unweighted(g, raw=True) == [0.0, 1.0, 0.0]
    assert RG.betweenness_centrality is RG.betweenness_unweighted
    d = zog.directed().add_edge("A", "B").add_edge("B", "C")
    gd = RG.ResourceGraph(StubGraph([0.0, 1.0, 0.0]), d)
    assert RG.betweenness_unweighted(gd) == {"A": 0.0, "B": 1.0, "C": 0.0}


def test_destroy_returns_ok():
    s = StubGraph([1.0])
    assert RG.destroy(RG.ResourceGraph(s, zog.directed().add_node("A"))) == "ok"
    assert s.destroyed


def test_hash_graph_backend_is_refused():
    with pytest.raises(NotImplementedError):
        RG.new(zog.directed().add_edge("A", "B"), backend="hash_graph")


def test_unknown_option_rejected():
    b = zog.directed().add_edge("x", "y")
    g = RG.ResourceGraph(StubGraph([0.5, 0.5]), b)
    with pytest.raises(TypeError):
        RG.pagerank(g, bogus=1)
