"""The ResourceGraph mirror end to end on the GPU, written after the
reference's own tests (test/resource_graph_test.exs, test/centrality_test.exs,
test/hash_graph_parity_test.exs)."""
import os

import numpy as np
import pytest

import zog_b200 as zog
from conftest import GOLDEN, rel_l1

RG = zog.ResourceGraph
pytestmark = pytest.mark.gpu


def test_new_destroy_empty_single(native):
    """resource_graph_test.exs:11-38."""
    b = zog.undirected().add_edge("A", "B", 1.0).add_edge("B", "C", 1.0)
    g = RG.new(b)
    assert g.builder is b
    assert RG.destroy(g) == "ok"
    g = RG.new(zog.undirected())
    assert RG.pagerank(g) == {} and RG.betweenness_unweighted(g) == {}
    RG.destroy(g)
    g = RG.new(zog.undirected().add_node("A"))
    assert RG.pagerank(g) == {"A": 1.0} and RG.betweenness_unweighted(g) == {"A": 0.0}
    RG.destroy(g)


def test_betweenness_path_graph(native):
    """resource_graph_test.exs:40-55."""
    g = RG.new(zog.undirected().add_edge("A", "B", 1.0).add_edge("B", "C", 1.0))
    s = RG.betweenness_unweighted(g)
    assert s["B"] > s["A"] and s["B"] > s["C"] and s["B"] == 1.0
    RG.destroy(g)


def test_betweenness_directed_bridge_exact_zeros(native):
    """centrality_test.exs:11-24."""
    g = RG.new(zog.directed().add_edge("A", "B", 1.0).add_edge("B", "C", 1.0))
    s = RG.betweenness_centrality(g)
    assert s == {"A": 0.0, "B": 1.0, "C": 0.0}
    RG.destroy(g)


def test_star(native):
    """resource_graph_test.exs:85-101 and centrality_test.exs:26-39."""
    b = zog.undirected()
    for leaf in ("A", "B", "C"):
        b.add_edge("center", leaf, 1.0)
    g = RG.new(b)
    pr = RG.pagerank(g)
    assert all(pr["center"] > pr[x] for x in "ABC")
    bc = RG.betweenness_unweighted(g)
    assert bc["center"] == 3.0 and all(bc[x] == 0.0 for x in "ABC")
    RG.destroy(g)


def test_triangle_known_values(native):
    g = RG.new(zog.undirected().add_edge("A", "B").add_edge("B", "C").add_edge("C", "A"))
    pr = RG.pagerank(g)
    assert all(abs(v - 1 / 3) < 1e-15 for v in pr.values())
    assert RG.betweenness_unweighted(g) == {"A": 0.0, "B": 0.0, "C": 0.0}
    RG.destroy(g)


def test_raw_lists(native):
    """resource_graph_test.exs:501-541."""
    g = RG.new(zog.undirected().add_edge("A", "B").add_edge("B", "C").add_edge("C", "A").add_edge("B", "D"))
    pr = RG.pagerank(g, raw=True)
    assert isinstance(pr, list) and len(pr) == 4 and all(isinstance(x, float) for x in pr)
    assert isinstance(RG.betweenness_unweighted(g, raw=True), list)
    RG.destroy(g)


def test_integer_labels_edgelist(native, tmp_path):
    """resource_graph_test.exs:544-570."""
    p = tmp_path / "edge_list_int.txt"
    p.write_text("0 1 1.5\n1 2 2.0\n2 0 1.0\n")
    g = RG.read_edgelist(str(p), integer_labels=True)
    assert g.builder.integer_labels and g.builder.next_id == 3
    pr = RG.pagerank(g)
    assert set(pr) == {0, 1, 2}
    raw = RG.pagerank(g, raw=True)
    assert isinstance(raw, list) and len(raw) == 3
    RG.destroy(g)


def test_read_edgelist_fixture_matches_oracle(native, oracle, tmp_path):
    """io_test.exs:11-23 (wiki_vote_sample.txt, 86 nodes): labels, PageRank and
    betweenness equal the oracle's restatement of the NIF reader."""
    raw = np.load(os.path.join(GOLDEN, "wiki_vote_sample_text.npz"))["text"].tobytes()
    p = tmp_path / "wiki_vote_sample.txt"
    p.write_bytes(raw)
    g = RG.read_edgelist(str(p), directed=True)
    assert g.builder.node_count() == 86
    ag, nid, labels = oracle.read_edgelist(str(p), directed=True)
    assert g.builder.all_labels() == labels
    pr = RG.pagerank(g, raw=True, tolerance=1e-9, max_iterations=200)
    x, _, _ = ag.pagerank(0.85, 200, 1e-9)
    assert rel_l1(pr, x) <= 1e-9
    bc = RG.betweenness_unweighted(g, raw=True)
    ref, _ = ag.betweenness_unweighted()
    assert rel_l1(bc, ref) <= 1e-9
    RG.destroy(g)


def test_read_edgelist_undirected_and_placeholders(native, oracle, tmp_path):
    p = tmp_path / "e.txt"
    p.write_text("# c\nsource target\n0 5\n5 0 2.0\n2,2\n3\t4\n\n7 x\n")
    g = RG.read_edgelist(str(p), directed=False, integer_labels=True)
    ag, nid, _ = oracle.read_edgelist(str(p), directed=False, integer_labels=True)
    assert g.builder.next_id == nid == 6
    _, _, out_off, out_col, _ = g.resource.export_csr()
    so, sc = ag.successor_csr()
    assert np.array_equal(out_off, so) and np.array_equal(out_col, sc)
    RG.destroy(g)


def test_several_algorithms_one_resource(native):
    """resource_graph_test.exs:458-479: one resource, many calls."""
    b = zog.directed()
    rng = np.random.default_rng(3)
    for s, d in rng.integers(0, 50, (300, 2)):
        b.add_edge(int(s), int(d))
    g = RG.new(b)
    a1 = RG.pagerank(g, raw=True)
    b1 = RG.betweenness_unweighted(g, raw=True)
    a2 = RG.pagerank(g, raw=True)
    b2 = RG.betweenness_unweighted(g, raw=True)
    assert a1 == a2 and b1 == b2
    RG.destroy(g)
    with pytest.raises(zog._native.ZogCudaError):
        g.resource.pagerank()


def test_node_not_found_error(native):
    with pytest.raises(zog._native.ZogCudaError) as ei:
        zog._native.Graph.from_edges(3, [0, 5], [1, 2])
    assert ei.value.status == 2


# ---- copy-in/copy-out API (lib/zog/centrality.ex), test/centrality_test.exs --

def test_centrality_betweenness_known_answers(native):
    """centrality_test.exs:11-51."""
    C = zog.Centrality
    s = C.betweenness_unweighted(zog.directed().add_edge("A", "B", 1.0).add_edge("B", "C", 1.0))
    assert s["B"] > s["A"] and s["B"] > s["C"] and s["A"] == 0.0 and s["C"] == 0.0
    b = zog.undirected()
    for leaf in "abc":
        b.add_edge("center", leaf, 1.0)
    s = C.betweenness_unweighted(b)
    assert s["center"] > 0.0 and all(s[x] == 0.0 for x in "abc")
    assert C.betweenness_unweighted(zog.directed()) == {}
    assert C.betweenness_unweighted(zog.directed().add_node("A")) == {"A": 0.0}


def test_centrality_pagerank_known_answers(native, oracle):
    """centrality_test.exs:137-163, and equality with the resource API."""
    C = zog.Centrality
    s = C.pagerank(zog.directed().add_edge("A", "B", 1.0).add_edge("C", "B", 1.0))
    assert s["B"] > s["A"] and s["B"] > s["C"]
    chain = zog.directed().add_edge("A", "B", 1.0).add_edge("B", "C", 1.0)
    for d in (0.85, 0.99):
        assert C.pagerank(chain, damping=d)["A"] > 0.0
    g = RG.new(chain)
    assert RG.pagerank(g, damping=0.99) == C.pagerank(chain, damping=0.99)
    RG.destroy(g)
