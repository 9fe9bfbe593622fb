"""Personalised PageRank for many seeds (one CSR SpMM) against the CPU
oracle's generalised iteration (og_pagerank_ext with a one-hot teleport):
every seed within relative L1 1e-9 and with the same iteration count, also
across passes (more than 256 seeds) and for seeds that stop early."""
import numpy as np
import pytest

from conftest import rel_l1

pytestmark = pytest.mark.gpu
TOL = 1e-9


def check_seeds(native, oracle, G, seeds, max_it=200, tol=1e-10, sample=None):
    V, _, _ = G.info()
    res, its = G.ppr(seeds, 0.85, max_it, tol)
    assert res.shape == (len(seeds), V)
    in_off, in_col, _, _, deg = G.export_csr()
    idx = range(len(seeds)) if sample is None else sample
    for i in idx:
        p = np.zeros(V)
        p[seeds[i]] = 1.0
        ref, it, _ = oracle.pagerank_ext(V, in_off, in_col, deg, None, p, 0.85, max_it, tol)
        assert rel_l1(res[i], ref) <= TOL, (i, rel_l1(res[i], ref))
        assert its[i] == it, (i, its[i], it)
    return res, its


def test_ppr_matches_oracle_small_graphs(native, oracle):
    V, f, t = oracle.rmat(10, 8, 77, directed=True)
    G = native.Graph.from_edges(V, f, t)
    try:
        seeds = np.random.default_rng(1).choice(V, 40, replace=False).astype(np.uint32)
        check_seeds(native, oracle, G, seeds)
    finally:
        G.destroy()
    G = native.Graph.barabasi_albert(3000, 3, 12, directed=True)
    try:
        seeds = np.random.default_rng(2).choice(3000, 100, replace=False).astype(np.uint32)
        check_seeds(native, oracle, G, seeds, sample=range(0, 100, 7))
    finally:
        G.destroy()


def test_ppr_many_passes_hub_rows_and_repeated_seeds(native, oracle):
    # an in-star with a 5000-arc row (chunked hub row) plus an R-MAT part
    V, f, t = oracle.rmat(12, 4, 5, directed=True)
    hub_src = np.arange(1, 5001, dtype=np.uint32) % V
    f2 = np.concatenate([f, hub_src]).astype(np.uint32)
    t2 = np.concatenate([t, np.zeros(5000, np.uint32)]).astype(np.uint32)
    G = native.Graph.from_edges(V, f2, t2)
    try:
        rng = np.random.default_rng(3)
        seeds = rng.integers(0, V, 300).astype(np.uint32)  # two passes, repeats allowed
        seeds[5] = 0  # the hub itself
        res, its = check_seeds(native, oracle, G, seeds, sample=[0, 5, 100, 255, 256, 299])
        dup = np.nonzero(seeds == seeds[7])[0]
        for j in dup:
            np.testing.assert_array_equal(res[j], res[7])
    finally:
        G.destroy()


@pytest.mark.parametrize("width", [32, 64, 128, 256])
def test_ppr_every_pass_width(native, oracle, monkeypatch, width):
    """Each kernel width (ZOGCU_PPR_PASS) over 100 seeds, with a hub row long
    enough to be cut into chunks: several passes at the narrow widths and a
    partial last pass, every sampled seed against the oracle."""
    monkeypatch.setenv("ZOGCU_PPR_PASS", str(width))
    V, f, t = oracle.rmat(11, 6, 11, directed=True)
    hub_src = np.arange(1, 6001, dtype=np.uint32) % V
    f2 = np.concatenate([f, hub_src]).astype(np.uint32)
    t2 = np.concatenate([t, np.full(6000, 9, np.uint32)]).astype(np.uint32)
    G = native.Graph.from_edges(V, f2, t2)
    try:
        seeds = np.random.default_rng(width).choice(V, 100, replace=False).astype(np.uint32)
        seeds[3] = 9  # the hub
        check_seeds(native, oracle, G, seeds, sample=[0, 3, 31, 32, 63, 64, 99])
    finally:
        G.destroy()


def test_ppr_iteration_cap_and_errors(native, oracle):
    V, f, t = oracle.rmat(9, 8, 9, directed=True)
    G = native.Graph.from_edges(V, f, t)
    try:
        seeds = np.array([1, 2, 3], np.uint32)
        res, its = check_seeds(native, oracle, G, seeds, max_it=4, tol=0.0)
        assert np.all(its == 4)
        res, its = G.ppr(seeds, 0.85, 0, 1e-9)
        assert np.allclose(res, 1.0 / V) and np.all(its == 0)
        with pytest.raises(native.ZogCudaError):
            G.ppr(np.array([V], np.uint32))
    finally:
        G.destroy()
