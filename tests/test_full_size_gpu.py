"""Properties at the measured workloads' full sizes, where the oracle would run
for minutes.  Each holds at any size, so it checks the very graphs and kernels
that the bench times:

* PageRank, directed R-MAT scale 24 (edge factor 16, seed 1024; 16.8 M nodes,
  263 M arcs), FP64, d 0.85, tol 1e-9: the vector sums to 1, no entry is below
  the teleport term (1-d)/n, and one more step of the reference's update
  (centrality.zig:924-946), computed independently in torch FP64 from the
  exported in-CSR, moves it by at most d times the solver's last residual.
  The update is an L1 contraction with factor d (column-stochastic once the
  dangling mass is spread uniformly), so |T(x_k) - x_k| <= d |x_k - x_{k-1}|.
* The precision form on the same graph (propagation-blocked FP32 phase, then
  FP64 polish): within 2*d/(1-d)*tol of the FP64 vector, and the same
  one-step bound.
* Personalised PageRank, directed R-MAT scale 22 (edge factor 16, seed 1022),
  64 seeds in one call: every row sums to 1 and, for sampled seeds, one more
  step with the one-hot teleport moves it by at most d * tol.
* Brandes, undirected R-MAT scale 16 (edge factor 16, seed 1016): for a
  single source s the dependencies sum to sum_t (dist(s,t) - 1) over reached
  t != s (every shortest s-t path has dist-1 interior nodes), with dist from
  the oracle's BFS; the all-source scores equal the sum of the scores of four
  disjoint source batches.
"""
import numpy as np
import pytest

from conftest import rel_l1

pytestmark = [pytest.mark.gpu, pytest.mark.slow]
D = 0.85


class TorchStep:
    """x -> (1-d)/n + d*(sum_{deg 0} x/n + sum_{u->v} x_u/deg_u) in torch FP64,
    or (1-d)*p_v in place of (1-d)/n when a teleport vector p is given (the
    personalised form, dangling mass still spread uniformly)."""

    def __init__(self, in_off, in_col, deg):
        import torch

        dev = torch.device("cuda")
        self.V = int(deg.size)
        counts = torch.from_numpy(np.diff(in_off.astype(np.int64))).to(dev)
        self.dst = torch.repeat_interleave(torch.arange(self.V, device=dev), counts)
        self.col = torch.from_numpy(in_col.view(np.int32)).to(dev).long()
        degt = torch.from_numpy(deg.astype(np.float64)).to(dev)
        self.dangling = degt == 0
        self.deg = degt.clamp(min=1.0)

    def __call__(self, x, p=None):
        import torch

        contrib = torch.where(self.dangling, torch.zeros_like(x), x / self.deg)
        sink = x[self.dangling].sum() / self.V
        y = torch.zeros_like(x).index_add_(0, self.dst, contrib[self.col])
        tele = (1.0 - D) / self.V if p is None else (1.0 - D) * p
        return tele + D * (sink + y)


def l1(a, b):
    return float((a - b).abs().sum())


def test_pagerank_scale24_contraction_and_precision_form(native):
    import torch

    tol = 1e-9
    G = native.Graph.rmat(24, 16, 1024, directed=True)
    try:
        V, E, n = G.info()
        assert V == 1 << 24 and n == V and E > 2.6e8
        in_off, in_col, _, _, deg = G.export_csr()
        step = TorchStep(in_off, in_col, deg)
        del in_col

        x, st = G.pagerank(D, 200, tol, stats=True)
        assert st["residual"] < tol and st["iterations"] < 200
        assert abs(x.sum() - 1.0) < 1e-9
        assert x.min() >= (1.0 - D) / V * (1.0 - 1e-9)
        xt = torch.from_numpy(x).cuda()
        assert l1(step(xt), xt) <= D * st["residual"] + 1e-12

        xm, sm = G.pagerank(D, 200, tol, precision=native.PREC_MIXED, stats=True)
        assert sm["reserved"] == 1, "the blocked FP32 phase did not run at full size"
        assert sm["residual"] < tol and sm["polish_iterations"] >= 1
        assert rel_l1(xm, x) <= 2 * D / (1 - D) * tol
        xmt = torch.from_numpy(xm).cuda()
        assert l1(step(xmt), xmt) <= D * sm["residual"] + 1e-12
    finally:
        G.destroy()
        torch.cuda.empty_cache()


def test_ppr_scale22_rows_and_contraction(native):
    import torch

    tol = 1e-9
    G = native.Graph.rmat(22, 16, 1022, directed=True)
    try:
        V, _, _ = G.info()
        seeds = np.random.default_rng(1022).choice(V, 64, replace=False).astype(np.uint32)
        out = torch.empty(seeds.size * V, dtype=torch.float64, device="cuda")
        st = G.ppr_device(seeds, out.data_ptr(), D, 200, tol)
        torch.cuda.synchronize()
        its = st["per_seed_iterations"]
        assert np.all(its < 200) and np.all(its >= 1)
        X = out.view(seeds.size, V)
        assert float((X.sum(dim=1) - 1.0).abs().max()) < 1e-9
        assert float(X.min()) >= 0.0
        in_off, in_col, _, _, deg = G.export_csr()
        step = TorchStep(in_off, in_col, deg)
        for i in (0, 17, 42, 63):
            p = torch.zeros(V, dtype=torch.float64, device="cuda")
            p[int(seeds[i])] = 1.0
            x = X[i].contiguous()
            assert l1(step(x, p), x) <= D * tol + 1e-12, f"seed {i}"
    finally:
        G.destroy()
        torch.cuda.empty_cache()


def test_brandes_scale16_path_length_identity_and_batch_sum(native, oracle):
    V, f, t = oracle.rmat(16, 16, 1016, directed=False)
    G = native.Graph.from_edges(V, f, t)
    A = oracle.ArrayGraph(V, f, t)
    try:
        srcs = np.random.default_rng(16).choice(V, 24, replace=False).astype(np.uint32)
        for s in srcs:
            dist, _, _ = A.bfs(int(s))
            reached = (dist != 0xFFFFFFFF) & (np.arange(V) != s)
            expect = float((dist[reached].astype(np.int64) - 1).sum())
            got = G.betweenness_unweighted(sources=[s]).sum()
            assert abs(got - expect) <= 1e-12 * max(expect, 1.0), f"source {s}"
        full = G.betweenness_unweighted()
        parts = np.zeros(V)
        order = np.random.default_rng(7).permutation(V).astype(np.uint32)
        for chunk in np.array_split(order, 4):
            parts += G.betweenness_unweighted(sources=np.sort(chunk))
        assert rel_l1(parts, full) <= 1e-12
        assert np.array_equal(parts == 0, full == 0)
    finally:
        A.close()
        G.destroy()
