"""Batched PageRank (many graphs in one persistent launch) against the same
graphs solved one by one through zogcu_pagerank and against the CPU oracle:
every graph's scores within relative L1 1e-12 of the single solve (same
iteration count), and within 1e-9 of the oracle, for every kernel
configuration the autotuner chooses from."""
import numpy as np
import pytest

from conftest import rel_l1

pytestmark = pytest.mark.gpu

N_CONFIGS = 6


def uneven_graphs(native, oracle, count=24, seed=7):
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        scale = int(rng.integers(3, 12))
        ef = int(rng.integers(1, 17))
        V, f, t = oracle.rmat(scale, ef, 100 + i, directed=True)
        out.append((V, f, t))
    # special shapes: one node, no arcs, all dangling, a self-loop cycle, a star
    out.append((1, np.zeros(0, np.uint32), np.zeros(0, np.uint32)))
    out.append((5, np.zeros(0, np.uint32), np.zeros(0, np.uint32)))
    out.append((3, np.array([0, 1, 2, 2], np.uint32), np.array([1, 2, 0, 2], np.uint32)))
    k = 300
    out.append((k + 1, np.arange(1, k + 1, dtype=np.uint32), np.zeros(k, np.uint32)))  # in-star: long row
    return out


def test_batch_matches_single_solves_and_oracle(native, oracle):
    specs = uneven_graphs(native, oracle)
    graphs = [native.Graph.from_edges(V, f, t) for V, f, t in specs]
    try:
        single = [g.pagerank(0.85, 200, 1e-10, stats=True) for g in graphs]
        B = native.Batch(graphs)
        try:
            n, V, E, offs = B.info()
            assert n == len(graphs) and V == sum(s[0] for s in specs)
            for cfg in list(range(N_CONFIGS)) + [-1]:
                res, its = B.pagerank(0.85, 200, 1e-10, config=cfg)
                for i, (x, (ref, st)) in enumerate(zip(res, single)):
                    assert rel_l1(x, ref) <= 1e-12, (cfg, i)
                    assert its[i] == st["iterations"], (cfg, i, its[i], st["iterations"])
            for i in (0, 5, 11, len(specs) - 1, len(specs) - 2, len(specs) - 4):
                Vg, f, t = specs[i]
                ref, it, _ = oracle.ArrayGraph(Vg, f, t).pagerank(0.85, 200, 1e-10)
                assert rel_l1(res[i], ref) <= 1e-9, i
                assert its[i] == it, i
        finally:
            B.destroy()
    finally:
        for g in graphs:
            g.destroy()


def test_batch_respects_max_iterations_and_trivial_graphs(native, oracle):
    specs = uneven_graphs(native, oracle, count=6, seed=3)
    graphs = [native.Graph.from_edges(V, f, t) for V, f, t in specs]
    B = native.Batch(graphs)
    try:
        res, its = B.pagerank(0.85, 3, 0.0)
        for g, x, k in zip(graphs, res, its):
            ref, st = g.pagerank(0.85, 3, 0.0, stats=True)
            assert k == st["iterations"]
            assert rel_l1(x, ref) <= 1e-12
        res, its = B.pagerank(0.85, 0, 1e-9)  # no iterations: the uniform start
        for (V, _, _), x in zip(specs, res):
            assert np.allclose(x, 1.0 / V) or V <= 1
    finally:
        B.destroy()
        for g in graphs:
            g.destroy()


def test_empty_batch(native):
    B = native.Batch([])
    try:
        res, its = B.pagerank()
        assert res == [] and its.size == 0
    finally:
        B.destroy()
