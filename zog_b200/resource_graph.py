"""Host-side mirror of ``Zog.ResourceGraph`` for the two GPU hot paths.

Same functions, option names, defaults and result shapes as the reference
(``lib/zog/resource_graph.ex``), with the ``:soa`` backend's algorithms running
in ``libzogcu`` on the GPU:

=====================================  =========================================
this module                            reference
=====================================  =========================================
``new(builder, backend="soa")``        ``new/2``            resource_graph.ex:1394-1403
``read_edgelist(path, ...)``           ``read_edgelist/2``  resource_graph.ex:1475-1485
``destroy(g)``                         ``destroy/1``        resource_graph.ex:1578-1581
``pagerank(g, ...)``                   ``pagerank/2``       resource_graph.ex:1672-1685
``betweenness_unweighted(g, ...)``     ``betweenness_unweighted/2`` resource_graph.ex:1591-1601
``betweenness_f64(g, ...)``            ``betweenness_f64/2`` resource_graph.ex:1611-1621
``betweenness_centrality``             alias of ``betweenness_unweighted``
=====================================  =========================================

Result shaping follows ``map_scores`` (resource_graph.ex:2609-2619): ``raw=True``
returns the flat list indexed by internal id; otherwise integer-labelled graphs
give ``{id: score}`` and labelled graphs ``{label: score}``.  Betweenness scores
of undirected builders are halved first (``maybe_scale_undirected``,
resource_graph.ex:2633-2637).

Only ``backend="soa"`` is accelerated.  ``:hash_graph`` is the reference's
mutable-graph backend and has no GPU path here: asking for it raises.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from . import _native
from .soa import SoA


@dataclass
class ResourceGraph:
    """``%{resource: ref, builder: SoA}`` of the reference."""

    resource: _native.Graph
    builder: SoA


def _check_backend(backend: str):
    if backend not in ("soa", ":soa"):
        raise NotImplementedError(f"backend {backend!r} has no GPU implementation; use backend='soa'")


def new(builder: SoA, backend: str = "soa") -> ResourceGraph:
    """resource_graph.ex:1394-1403: builds the native resource from the
    builder's insertion-order edge arrays (the NIF ``new`` -> buildGraph)."""
    _check_backend(backend)
    frm, to, w = builder.to_edge_arrays()
    g = _native.Graph.from_edges(builder.node_count(), frm, to, w)
    return ResourceGraph(g, builder)


def read_edgelist(path, directed: bool = True, backend: str = "soa", integer_labels: bool = False) -> ResourceGraph:
    """resource_graph.ex:1475-1485 + build_from_labels (:1531-1572)."""
    _check_backend(backend)
    import os

    g, next_id, labels = _native.Graph.read_edgelist(os.path.abspath(os.path.expanduser(str(path))),
                                                     directed=directed, integer_labels=integer_labels)
    kind = "directed" if directed else "undirected"
    if integer_labels:
        b = SoA.with_integer_ids(kind, next_id)
    else:
        b = SoA(kind)
        for lbl in labels:
            b.ensure_node(lbl)
    return ResourceGraph(g, b)


def destroy(g: ResourceGraph) -> str:
    """resource_graph.ex:1578-1581: frees the device graph; returns ``"ok"``."""
    g.resource.destroy()
    return "ok"


def _map_scores(builder: SoA, scores: np.ndarray):
    """resource_graph.ex:2609-2619."""
    vals = [float(x) for x in scores]
    if builder.integer_labels:
        return {i: s for i, s in enumerate(vals)}
    # nodes_rev zipped with the reversed scores, truncated to the shorter list
    return {lbl: s for lbl, s in zip(builder.nodes, reversed(vals))}


def _maybe_scale_undirected(builder: SoA, scores: np.ndarray) -> np.ndarray:
    """resource_graph.ex:2633-2637."""
    return scores * 0.5 if builder.kind == "undirected" else scores


def pagerank(g: ResourceGraph, damping: float = 0.85, max_iterations: int = 100, tolerance: float = 0.0001,
             raw: bool = False, **ext):
    """resource_graph.ex:1672-1685 (defaults 0.85 / 100 / 1e-4).

    Extensions (keyword-only, default off = the reference's behaviour):
    ``precision`` ("fp64" | "mixed"), ``x0`` (warm-start vector) and
    ``teleport`` (personalisation vector)."""
    prec = ext.pop("precision", "fp64")
    if ext.keys() - {"x0", "teleport"}:
        raise TypeError(f"unknown options {sorted(ext.keys() - {'x0', 'teleport'})}")
    p = {"fp64": _native.PREC_FP64, "mixed": _native.PREC_MIXED}[prec]
    scores = g.resource.pagerank(damping, max_iterations, tolerance, precision=p, x0=ext.get("x0"),
                                 teleport=ext.get("teleport"))
    if raw:
        return [float(x) for x in scores]
    return _map_scores(g.builder, scores)


def betweenness_unweighted(g: ResourceGraph, raw: bool = False, sources=None):
    """resource_graph.ex:1591-1601.  ``sources`` (extension) restricts the
    outer Brandes loop to a subset of source ids."""
    scores = g.resource.betweenness_unweighted(sources=sources)
    scores = _maybe_scale_undirected(g.builder, scores)
    if raw:
        return [float(x) for x in scores]
    return _map_scores(g.builder, scores)


def betweenness_f64(g: ResourceGraph, raw: bool = False, sources=None):
    """resource_graph.ex:1611-1621: weighted (Dijkstra) betweenness over the
    edges' f64 weights; halved for undirected builders like the unweighted
    form.  ``sources`` (extension) restricts the outer loop."""
    scores = g.resource.betweenness_weighted(sources=sources)
    scores = _maybe_scale_undirected(g.builder, scores)
    if raw:
        return [float(x) for x in scores]
    return _map_scores(g.builder, scores)


def eigenvector(g: ResourceGraph, max_iterations: int = 100, tolerance: float = 0.0001, raw: bool = False):
    """resource_graph.ex:1697-1709 (defaults 100 / 1e-4)."""
    scores = g.resource.eigenvector(max_iterations, tolerance)
    return [float(x) for x in scores] if raw else _map_scores(g.builder, scores)


def katz(g: ResourceGraph, alpha: float = 0.1, beta: float = 1.0, max_iterations: int = 100,
         tolerance: float = 0.0001, raw: bool = False):
    """resource_graph.ex:1723-1737 (defaults 0.1 / 1.0 / 100 / 1e-4)."""
    scores = g.resource.katz(alpha, beta, max_iterations, tolerance)
    return [float(x) for x in scores] if raw else _map_scores(g.builder, scores)


def alpha_centrality(g: ResourceGraph, alpha: float = 0.5, initial: float = 1.0, max_iterations: int = 100,
                     tolerance: float = 0.0001, raw: bool = False):
    """resource_graph.ex:1751-1765 (defaults 0.5 / 1.0 / 100 / 1e-4)."""
    scores = g.resource.alpha_centrality(alpha, initial, max_iterations, tolerance)
    return [float(x) for x in scores] if raw else _map_scores(g.builder, scores)


#: The name used for this path in the project's goal statement; the reference
#: only exports ``betweenness_unweighted/2``.
betweenness_centrality = betweenness_unweighted
