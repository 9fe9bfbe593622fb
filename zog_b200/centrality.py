"""Host-side mirror of ``Zog.Centrality`` (``lib/zog/centrality.ex``), the
copy-in/copy-out API: every call builds the device graph from the builder's
edge arrays, runs the GPU kernel and frees the graph again -- the resource
pattern of ``Zog.ResourceGraph`` without keeping the resource.

=====================================  =========================================
this module                            reference
=====================================  =========================================
``pagerank(builder, ...)``             ``pagerank/2``                centrality.ex:237-247
``betweenness_unweighted(builder)``    ``betweenness_unweighted/1``  centrality.ex:191-197
``eigenvector(builder, ...)``          ``eigenvector/2``             centrality.ex:253-275
``katz(builder, ...)``                 ``katz/2``                    centrality.ex:281-293
``alpha_centrality(builder, ...)``     ``alpha_centrality/2``        centrality.ex:300-313
=====================================  =========================================

Scores map labels in insertion order to values (``map_scores``,
centrality.ex:319-324); betweenness of undirected builders is halved first
(centrality.ex:326-330).
"""
from __future__ import annotations

from . import _native
from .soa import SoA


def _map_scores(builder: SoA, scores):
    """centrality.ex:319-324: all_labels zipped with the scores."""
    return {lbl: float(s) for lbl, s in zip(builder.all_labels(), scores)}


def _graph(builder: SoA) -> _native.Graph:
    frm, to, w = builder.to_edge_arrays()
    return _native.Graph.from_edges(builder.node_count(), frm, to, w)


def pagerank(builder: SoA, damping: float = 0.85, max_iterations: int = 100, tolerance: float = 0.0001):
    """centrality.ex:237-247 (defaults 0.85 / 100 / 1e-4)."""
    g = _graph(builder)
    try:
        scores = g.pagerank(damping, max_iterations, tolerance)
    finally:
        g.destroy()
    return _map_scores(builder, scores)


def betweenness_unweighted(builder: SoA):
    """centrality.ex:191-197: unnormalised; halved for undirected builders."""
    g = _graph(builder)
    try:
        scores = g.betweenness_unweighted()
    finally:
        g.destroy()
    if builder.kind == "undirected":
        scores = scores * 0.5
    return _map_scores(builder, scores)


def betweenness_f64(builder: SoA):
    """centrality.ex:203-209: weighted (Dijkstra) betweenness over the
    builder's f64 weights, unnormalised; halved for undirected builders."""
    g = _graph(builder)
    try:
        scores = g.betweenness_weighted()
    finally:
        g.destroy()
    if builder.kind == "undirected":
        scores = scores * 0.5
    return _map_scores(builder, scores)


def eigenvector(builder: SoA, max_iterations: int = 100, tolerance: float = 0.0001):
    """centrality.ex:253-275, including the zero-vector fallback to a uniform
    1/sqrt(n) when every score is 0.0 and there is more than one node."""
    g = _graph(builder)
    try:
        scores = g.eigenvector(max_iterations, tolerance)
    finally:
        g.destroy()
    mapped = _map_scores(builder, scores)
    n = builder.node_count()
    if n > 1 and all(v == 0.0 for v in mapped.values()):
        u = 1.0 / (n ** 0.5)
        mapped = {k: u for k in mapped}
    return mapped


def katz(builder: SoA, alpha: float = 0.1, beta: float = 1.0, max_iterations: int = 100,
         tolerance: float = 0.0001):
    """centrality.ex:281-293."""
    g = _graph(builder)
    try:
        scores = g.katz(alpha, beta, max_iterations, tolerance)
    finally:
        g.destroy()
    return _map_scores(builder, scores)


def alpha_centrality(builder: SoA, alpha: float = 0.5, initial: float = 1.0, max_iterations: int = 100,
                     tolerance: float = 0.0001):
    """centrality.ex:300-313."""
    g = _graph(builder)
    try:
        scores = g.alpha_centrality(alpha, initial, max_iterations, tolerance)
    finally:
        g.destroy()
    return _map_scores(builder, scores)
