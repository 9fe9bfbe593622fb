"""zog_b200 -- B200-native (sm_100a) PageRank and Brandes betweenness behind
Zog's ``ResourceGraph`` API.

    import zog_b200 as zog
    b = zog.directed().add_edge("A", "B").add_edge("B", "C")
    g = zog.ResourceGraph.new(b)
    zog.ResourceGraph.pagerank(g, tolerance=1e-9, max_iterations=200)
    zog.ResourceGraph.betweenness_unweighted(g)
    zog.ResourceGraph.destroy(g)

The compute runs in ``libzogcu.so`` (CUDA, built by ``python -m
zog_b200.build``); this package is the host-side mirror of the reference's
Elixir API and holds no CPU implementation of either algorithm.
"""
import os as _os

# The betweenness call runs its source batches as up to eight independent
# branches of one CUDA graph, and the driver's default of 8 hardware work
# queues per context lets branches share a queue.  At scale 16, 4 of 8
# processes with 8 queues ran at 136-181 GTEPS instead of about 230; with 32
# queues, 4 of 24 did (with 4, 6 or 8 lanes alike), so queue sharing is at
# most part of the cause.  The count is read when the process creates its
# CUDA context, so it is set here, before any, unless the operator chose one.
_os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")

from . import _native
from . import centrality as Centrality
from . import resource_graph as ResourceGraph
from .soa import SoA, directed, undirected

__all__ = ["Centrality", "ResourceGraph", "SoA", "directed", "undirected", "_native"]
