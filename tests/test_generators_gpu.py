"""The library's seeded Barabasi-Albert and Watts-Strogatz generators against
the oracle's independent restatement of the same definitions (same seed ->
the same arc multiset), plus the models' structural properties."""
import numpy as np
import pytest

from oracle import gnn_oracle as GO

pytestmark = pytest.mark.gpu


def same_graph(G, V, f, t):
    in_off, in_col, _, _, deg = G.export_csr()
    ref = GO.Csr.from_edges(V, f, t)
    assert G.info()[0] == V
    np.testing.assert_array_equal(in_off.astype(np.int64), ref.in_off)
    np.testing.assert_array_equal(in_col.astype(np.int64), ref.in_col)
    np.testing.assert_array_equal(deg, ref.out_deg)


@pytest.mark.parametrize("n,m,seed,directed", [(50, 1, 3, True), (2000, 3, 5, True), (3000, 8, 7, False),
                                               (20000, 16, 11, True)])
def test_barabasi_albert_matches_oracle(native, oracle, n, m, seed, directed):
    G = native.Graph.barabasi_albert(n, m, seed, directed=directed)
    try:
        V, f, t = oracle.barabasi_albert(n, m, seed, directed=directed)
        same_graph(G, V, f, t)
        arcs = (m * (m - 1) // 2 + (n - m) * m) * (1 if directed else 2)
        assert f.size == arcs
        # every new node links to m distinct older nodes
        if directed:
            fo, to = f[m * (m - 1) // 2:], t[m * (m - 1) // 2:]
            assert np.all(fo > to)
            pairs = np.unique(fo.astype(np.int64) << 32 | to)
            assert pairs.size == fo.size
        # heavy-tailed in-degree: the largest hub is far above the mean
        indeg = np.bincount(t, minlength=V)
        assert indeg.max() > 5 * indeg.mean()
    finally:
        G.destroy()


@pytest.mark.parametrize("n,k,beta,seed,directed", [(100, 4, 0.0, 1, False), (1200, 10, 0.1, 6, False),
                                                    (5000, 10, 0.3, 9, True), (12, 10, 0.9, 2, False)])
def test_watts_strogatz_matches_oracle(native, oracle, n, k, beta, seed, directed):
    G = native.Graph.watts_strogatz(n, k, beta, seed, directed=directed)
    try:
        V, f, t = oracle.watts_strogatz(n, k, beta, seed, directed=directed)
        same_graph(G, V, f, t)
        # rewiring keeps the edge count n*k/2 and creates no self-loops
        assert f.size == n * k // 2 * (1 if directed else 2)
        assert not np.any(f == t)
        if beta == 0.0:
            assert np.all(np.bincount(f, minlength=n) == k)
    finally:
        G.destroy()


def test_generator_arguments_are_checked(native):
    with pytest.raises(native.ZogCudaError):
        native.Graph.barabasi_albert(4, 4, 1)
    with pytest.raises(native.ZogCudaError):
        native.Graph.watts_strogatz(100, 3, 0.1, 1)
    with pytest.raises(native.ZogCudaError):
        native.Graph.watts_strogatz(100, 4, 1.5, 1)
