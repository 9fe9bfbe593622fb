"""Parity against the oracle at the measured workloads' full sizes.

The oracle's multi-threaded PageRank (og_pagerank_csr_mt) spreads the row
sums of the reference loop (centrality.zig:924-958) over the host's threads
and keeps the two global sums in ascending node order, so its iterates are
bit for bit those of the single-threaded restatement (tests/test_oracle.py
checks that); it makes a full solve at scale 24 take seconds instead of the
single thread's ~50 s.  The graphs come from the oracle's own generator and
CSR builder, independently of the library's.

* PageRank, directed R-MAT scale 24 (edge factor 16, seed 1024; 16.8 M nodes,
  263 M arcs), FP64, d 0.85, tol 1e-9, at most 200 iterations: relative L1
  <= 1e-9 against the oracle and the same iteration count; the precision form
  within 2*d/(1-d)*tol of the oracle.
* PageRank, directed Barabasi-Albert n = 4,194,304, m = 8 (seed 4096): the
  same bars.
* Brandes, undirected R-MAT scale 16 (edge factor 16, seed 1016): for 2,048
  seeded sources, dist and sigma bit-exact against the oracle's BFS (sources
  spread over host threads), and the betweenness summed over those sources
  within relative L1 1e-9 of the oracle's, with the same exact zeros.
"""
import numpy as np
import pytest

from conftest import rel_l1

pytestmark = [pytest.mark.gpu, pytest.mark.slow]
D, TOL, MAX_IT = 0.85, 1e-9, 200


@pytest.fixture(scope="module")
def rmat24(oracle):
    """Directed R-MAT scale 24 from the oracle's generator, with its in-CSR."""
    V, f, t = oracle.rmat(24, 16, 1024, directed=True)
    return V, f, t, oracle.in_csr_from_edges(V, f, t)


def _pagerank_vs_oracle(native, oracle, V, f, t, csr=None):
    in_off, in_col, deg = csr if csr is not None else oracle.in_csr_from_edges(V, f, t)
    ref, it, l1, _ = oracle.pagerank_csr_mt(V, in_off, in_col, deg, D, MAX_IT, TOL)
    del in_off, in_col, deg
    G = native.Graph.from_edges(V, f, t)
    try:
        x, st = G.pagerank(D, MAX_IT, TOL, stats=True)
        assert st["iterations"] == it, (st["iterations"], it)
        assert rel_l1(x, ref) <= TOL, rel_l1(x, ref)
        assert l1 < TOL and st["residual"] < TOL
        xm, sm = G.pagerank(D, MAX_IT, TOL, precision=native.PREC_MIXED, stats=True)
        assert rel_l1(xm, ref) <= 2 * D / (1 - D) * TOL, rel_l1(xm, ref)
        return it, sm
    finally:
        G.destroy()


def test_pagerank_rmat24_matches_oracle(native, oracle, rmat24):
    import torch

    V, f, t, csr = rmat24
    assert V == 1 << 24 and len(f) > 2.6e8
    it, sm = _pagerank_vs_oracle(native, oracle, V, f, t, csr)
    assert it == 28
    assert sm["reserved"] == 1, "the blocked FP32 phase did not run at full size"
    torch.cuda.empty_cache()


def test_pagerank_rmat24_tight_fp64_matches_oracle(native, oracle, rmat24):
    """The tightly converged FP64 vector (tol 1e-14) that the errors of the
    precision form and the learned start are reported against: the GPU's and
    the oracle's agree to 1e-12 (each lies within ~1e-14 of the fixed point)."""
    import torch

    tight = 1e-14
    V, f, t, (in_off, in_col, deg) = rmat24
    ref, it, l1, _ = oracle.pagerank_csr_mt(V, in_off, in_col, deg, D, MAX_IT, tight)
    assert l1 < tight and it < MAX_IT
    G = native.Graph.from_edges(V, f, t)
    try:
        x, st = G.pagerank(D, MAX_IT, tight, stats=True)
        assert st["residual"] < tight
        assert rel_l1(x, ref) <= 1e-12, rel_l1(x, ref)
    finally:
        G.destroy()
        torch.cuda.empty_cache()


def test_pagerank_ba4m_matches_oracle(native, oracle):
    import torch

    V, f, t = oracle.barabasi_albert(1 << 22, 8, 4096, directed=True)
    _pagerank_vs_oracle(native, oracle, V, f, t)
    torch.cuda.empty_cache()


def test_brandes_rmat16_2048_sources_bit_exact(native, oracle):
    V, f, t = oracle.rmat(16, 16, 1016, directed=False)
    G = native.Graph.from_edges(V, f, t)
    try:
        _, _, out_off, out_col, _ = G.export_csr()
        A = oracle.ArrayGraph(V, f, t)
        so, sc = A.successor_csr()
        A.close()
        # the successor CSR the oracle walks (reverse insertion order per node)
        assert np.array_equal(so, out_off) and np.array_equal(sc, out_col)
        srcs = np.sort(np.random.default_rng(2048).choice(V, 2048, replace=False)).astype(np.uint32)
        for chunk in np.array_split(srcs, 8):
            d_gpu, s_gpu, ovf_gpu = G.bfs_sigma(chunk)
            d_ref, s_ref, ovf_ref = oracle.bfs_csr_many(V, so, sc, chunk)
            assert np.array_equal(d_gpu, d_ref)
            assert np.array_equal(s_gpu, s_ref)
            assert ovf_gpu == bool(ovf_ref.any())
        bc = G.betweenness_unweighted(sources=srcs)
        ref, _ = oracle.betweenness_csr_sources_mt(V, so, sc, srcs)
        assert rel_l1(bc, ref) <= 1e-9, rel_l1(bc, ref)
        assert np.array_equal(bc == 0, ref == 0)
    finally:
        G.destroy()
