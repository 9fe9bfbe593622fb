"""Katz, alpha and eigenvector centrality (centrality.zig:1050-1321) on the
GPU against the CPU oracle.  Tolerance: relative L1 <= 1e-9 and the same
iteration count / exit; the eigenvector L2 norm is reassociated."""
import json
import os

import numpy as np
import pytest

import zog_b200 as zog
from conftest import GOLDEN, rel_l1

pytestmark = pytest.mark.gpu
TOL = 1e-9


def golden(name):
    return dict(np.load(os.path.join(GOLDEN, name + ".npz")))


def golden_names():
    with open(os.path.join(GOLDEN, "manifest.json")) as f:
        return sorted(n for n in json.load(f) if n != "tombstones")


def graphs(native, oracle):
    for name in golden_names():
        g = golden(name)
        V = int(g["V"])
        yield name, native.Graph.from_edges(V, g["from"], g["to"]), oracle.ArrayGraph(V, g["from"], g["to"])
    V, f, t = oracle.rmat(13, 8, 13, directed=True)
    yield "rmat13", native.Graph.from_edges(V, f, t), oracle.ArrayGraph(V, f, t)
    V, f, t = oracle.rmat(12, 8, 12, directed=False)
    yield "rmat12u", native.Graph.from_edges(V, f, t), oracle.ArrayGraph(V, f, t)


def test_katz_and_alpha_match_oracle(native, oracle):
    for name, G, ag in graphs(native, oracle):
        try:
            for a, b in ((0.1, 1.0), (0.01, 2.0)):
                x, st = G.katz(a, b, 100, 1e-10, stats=True)
                ref, it, _ = ag.katz(a, b, 100, 1e-10)
                assert rel_l1(x, ref) <= TOL, name
                assert st["iterations"] == it, name
            x, st = G.alpha_centrality(0.05, 1.0, 100, 1e-12, stats=True)
            ref, it, _ = ag.alpha_centrality(0.05, 1.0, 100, 1e-12)
            assert rel_l1(x, ref) <= TOL, name
            assert st["iterations"] == it, name
        finally:
            G.destroy()


def test_eigenvector_matches_oracle(native, oracle):
    for name, G, ag in graphs(native, oracle):
        try:
            x, st = G.eigenvector(100, 1e-6, stats=True)
            ref, it, how = ag.eigenvector(100, 1e-6)
            assert rel_l1(x, ref) <= 1e-8, (name, rel_l1(x, ref))
            assert st["iterations"] == it, name
        finally:
            G.destroy()


def test_eigenvector_degenerate_and_cycle(native):
    """A DAG converges to the zero vector -> uniform 1/sqrt(n); a directed
    3-cycle never settles and returns the last vector after max_iterations."""
    R = zog.ResourceGraph
    g = R.new(zog.directed().add_edge("A", "B").add_edge("B", "C"))
    e = R.eigenvector(g)
    assert all(abs(v - 1 / 3 ** 0.5) < 1e-15 for v in e.values())
    R.destroy(g)
    g = R.new(zog.directed().add_edge("A", "B").add_edge("B", "C").add_edge("C", "A"))
    e = R.eigenvector(g, raw=True)
    assert all(abs(v - 1 / 3 ** 0.5) < 0.01 for v in e)  # centrality_test.exs cycle case
    R.destroy(g)


def test_resource_and_copy_in_out_api(native):
    b = zog.undirected().add_edge("A", "B").add_edge("B", "C").add_edge("C", "A").add_edge("B", "D")
    g = zog.ResourceGraph.new(b)
    for fn in ("katz", "alpha_centrality", "eigenvector"):
        r = getattr(zog.ResourceGraph, fn)(g, raw=True)
        assert isinstance(r, list) and len(r) == 4  # resource_graph_test.exs:501-541
        assert getattr(zog.Centrality, fn)(b) == getattr(zog.ResourceGraph, fn)(g)
    zog.ResourceGraph.destroy(g)
