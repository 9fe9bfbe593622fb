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
# branches of one CUDA graph.  With the driver's default of 8 hardware work
# queues per context, branches can share a queue and run one after another:
# at scale 16, 2 of 4 processes measured 171-181 GTEPS instead of 235; with 32
# queues, 1 of 10 (179 against 224-236).  The count is read when the process
# creates its CUDA context, so it is set here, before any, unless the operator
# chose one.
_os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")

from . import _native
from . import centrality as Centrality
from . import resource_graph as ResourceGraph
from .soa import SoA, directed, undirected

__all__ = ["Centrality", "ResourceGraph", "SoA", "directed", "undirected", "_native"]
