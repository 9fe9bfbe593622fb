"""Brandes parity: the CUDA path (through the C ABI) against the CPU oracle.

Bars: BFS distances and path counts sigma bit-exact (integers); betweenness
relative L1 <= 1e-9 (FP64, the dependency sum is reassociated) with exact
zeros where the oracle has exact zeros.
"""
import json
import os

import numpy as np
import pytest

from conftest import GOLDEN, rel_l1

pytestmark = pytest.mark.gpu
TOL = 1e-9


def golden(name):
    return dict(np.load(os.path.join(GOLDEN, name + ".npz")))


def golden_names():
    with open(os.path.join(GOLDEN, "manifest.json")) as f:
        return sorted(json.load(f))


def make(native, g):
    if "ag_first_edge" in g:
        return native.Graph.from_arraygraph(g["ag_first_edge"], g["ag_node_deleted"], g["ag_to"],
                                            g["ag_next_edge"], g["ag_edge_deleted"])
    return native.Graph.from_edges(int(g["V"]), g["from"], g["to"])


@pytest.mark.parametrize("name", golden_names())
def test_golden_betweenness(native, name):
    g = golden(name)
    G = make(native, g)
    try:
        bc = G.betweenness_unweighted()
        assert bc.shape == g["bc"].shape
        assert rel_l1(bc, g["bc"]) <= TOL
        assert np.array_equal(bc == 0.0, g["bc"] == 0.0)
        srcs = g["bfs_sources"]
        if srcs.size and int(g["V"]) and not ("ag_node_deleted" in g and g["ag_node_deleted"][srcs].any()):
            dist, sigma, _ = G.bfs_sigma(srcs)
            for i, s in enumerate(srcs.tolist()):
                assert np.array_equal(dist[i], g[f"bfs_{s}_dist"])
                assert np.array_equal(sigma[i], g[f"bfs_{s}_sigma"])
    finally:
        G.destroy()


def test_scale14_all_sources(native, oracle):
    """Directed R-MAT scale 14 (the small benchmark graph): every source."""
    V, f, t = oracle.rmat(14, 8, 1014, directed=True)
    G = native.Graph.from_edges(V, f, t)
    try:
        bc, st = G.betweenness_unweighted(stats=True)
        ref, ovf = oracle.ArrayGraph(V, f, t).betweenness_unweighted()
        assert rel_l1(bc, ref) <= TOL
        assert np.array_equal(bc == 0.0, ref == 0.0)
        assert st["sources"] == V and bool(st["sigma_overflow"]) == ovf
    finally:
        G.destroy()


def test_scale16_undirected_sigma_bit_exact(native, oracle):
    """Undirected R-MAT scale 16 (the scale benchmark graph): dist and sigma of
    sampled sources bit-exact; betweenness over those sources."""
    V, f, t = oracle.rmat(16, 16, 1016, directed=False)
    G = native.Graph.from_edges(V, f, t)
    try:
        ag = oracle.ArrayGraph(V, f, t)
        rng = np.random.default_rng(16)
        srcs = np.unique(rng.integers(0, V, 70)).astype(np.uint32)
        dist, sigma, _ = G.bfs_sigma(srcs)
        for i, s in enumerate(srcs[:24].tolist()):
            d_ref, s_ref, _ = ag.bfs(s)
            assert np.array_equal(dist[i], d_ref)
            assert np.array_equal(sigma[i], s_ref)
        bc = G.betweenness_unweighted(sources=srcs)
        ref, _ = ag.betweenness_sources(srcs)
        assert rel_l1(bc, ref) <= TOL
    finally:
        G.destroy()


def test_batches_and_partial_batch(native, oracle):
    """130 sources = two full batches of 64 plus a partial one; duplicates and
    unreachable parts included."""
    V, f, t = oracle.rmat(12, 4, 5, directed=True)
    G = native.Graph.from_edges(V, f, t)
    try:
        srcs = np.arange(0, 130, dtype=np.uint32) * 7 % V
        bc = G.betweenness_unweighted(sources=srcs)
        ref, _ = oracle.ArrayGraph(V, f, t).betweenness_sources(srcs)
        assert rel_l1(bc, ref) <= TOL
    finally:
        G.destroy()


def test_long_path_deep_bfs(native, oracle):
    """A path of 3,000 nodes: BFS depth far beyond typical R-MAT levels."""
    V = 3000
    f = np.arange(V - 1, dtype=np.uint32)
    t = f + 1
    frm = np.concatenate([f, t]); to = np.concatenate([t, f])  # undirected arcs
    G = native.Graph.from_edges(V, frm, to)
    try:
        srcs = np.array([0, 1500, 2999], np.uint32)
        bc, st = G.betweenness_unweighted(sources=srcs, stats=True)
        ref, _ = oracle.ArrayGraph(V, frm, to).betweenness_sources(srcs)
        assert rel_l1(bc, ref) <= TOL and st["max_depth"] == 2999
    finally:
        G.destroy()


def test_sigma_overflow_wraps_like_usize(native, oracle):
    """A chain of 70 diamonds gives 2^70 shortest paths: sigma wraps modulo 2^64
    exactly like the reference's usize additions, and the overflow is flagged."""
    k = 70
    frm, to = [], []
    for i in range(k):
        a, b, c, d = 3 * i, 3 * i + 1, 3 * i + 2, 3 * i + 3
        frm += [a, a, b, c]; to += [b, c, d, d]
    V = 3 * k + 1
    G = native.Graph.from_edges(V, frm, to)
    try:
        dist, sigma, ovf = G.bfs_sigma(np.array([0], np.uint32))
        d_ref, s_ref, ovf_ref = oracle.ArrayGraph(V, frm, to).bfs(0)
        assert ovf and ovf_ref
        assert np.array_equal(dist[0], d_ref) and np.array_equal(sigma[0], s_ref)
    finally:
        G.destroy()


@pytest.mark.parametrize("directed", [True, False])
def test_hubs_split_over_several_ctas(native, oracle, directed):
    """Hubs far above the 1,024-arc work item: one with 5,000 in- and 3,000
    out-arcs, one with 2,500 duplicated in-arcs, on a random background.  The
    forward (in-arcs) and backward (out-arcs) steps split each hub over
    several CTAs and add the chunk partials in chunk order.  dist and sigma
    stay bit-exact; betweenness within the FP64 bar."""
    rng = np.random.default_rng(21 if directed else 22)
    V = 9000
    bg_f = rng.integers(0, V, 30000); bg_t = rng.integers(0, V, 30000)
    hub_in = rng.integers(0, V, 5000); hub_out = rng.integers(0, V, 3000)
    dup = np.repeat(rng.integers(0, V, 500), 5)
    f = np.concatenate([bg_f, hub_in, np.zeros(3000, np.int64), dup]).astype(np.uint32)
    t = np.concatenate([bg_t, np.zeros(5000, np.int64), hub_out, np.full(2500, 7)]).astype(np.uint32)
    if not directed:  # store both arcs of every edge, as undirected SoA graphs do
        f, t = np.concatenate([f, t]), np.concatenate([t, f])
    G = native.Graph.from_edges(V, f, t)
    try:
        srcs = np.concatenate([np.array([0, 7], np.uint32), (np.arange(126, dtype=np.uint32) * 71 + 3) % V])
        bc = G.betweenness_unweighted(sources=srcs)
        A = oracle.ArrayGraph(V, f, t)
        ref, _ = A.betweenness_sources(srcs)
        assert rel_l1(bc, ref) <= TOL
        assert np.array_equal(bc == 0.0, ref == 0.0)
        dist, sigma, _ = G.bfs_sigma(srcs[:3])
        for i, s in enumerate(srcs[:3]):
            d_ref, s_ref, _ = A.bfs(int(s))
            assert np.array_equal(dist[i], d_ref) and np.array_equal(sigma[i], s_ref)
        assert np.array_equal(bc, G.betweenness_unweighted(sources=srcs))  # deterministic
    finally:
        G.destroy()


def test_one_graph_serves_every_source_count(native, oracle):
    """A graph resource keeps its lanes' workspaces and instantiated CUDA
    graphs between calls, and the batches come from device-side cursors, so
    one graph serves any source count.  Successive calls on one resource:
    1 source, one batch, a partial third batch, more batches than one graph
    launch holds (8 lanes x 8 slots = 4,096 sources; 8,192 sources take two
    launches), a repeat of an earlier count, and every source.  Each against
    the oracle over the same sources; repeats bit-identical."""
    V, f, t = oracle.rmat(13, 8, 1313, directed=False)
    G = native.Graph.from_edges(V, f, t)
    try:
        _, _, out_off, out_col, _ = G.export_csr()
        rng = np.random.default_rng(13)
        perm = rng.permutation(V).astype(np.uint32)
        seen = {}
        for n in (1, 64, 130, 4100, 64, V):
            srcs = np.sort(perm[:n]) if n < V else None
            bc, st = G.betweenness_unweighted(sources=srcs, stats=True)
            ref, _ = oracle.betweenness_csr_sources_mt(V, out_off, out_col,
                                                       np.arange(V, dtype=np.uint32) if srcs is None else srcs)
            assert rel_l1(bc, ref) <= TOL, n
            assert np.array_equal(bc == 0.0, ref == 0.0), n
            assert st["sources"] == n
            if n in seen:
                assert np.array_equal(bc, seen[n]), n
            seen[n] = bc
        assert st["reserved"] == 2  # every source: 128 batches, two launches of the cached graph
    finally:
        G.destroy()
