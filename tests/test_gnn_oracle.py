"""The warm-start network's CPU oracle (hand-derived backward pass) against
torch autograd on the CPU: the oracle the GPU kernels are checked against is
itself pinned by an independent differentiation."""
import numpy as np
import pytest
import torch

from oracle import gnn_oracle as G


def torch_loss(p, g: G.Csr, pr, kind="kl"):
    """The model written with torch ops; autograd gives the reference gradient."""
    p = torch.tensor(G.bf16_round(p).astype(np.float64), requires_grad=True)
    offs, head = G.layer_offsets()
    rows = torch.from_numpy(g.rows)
    cols = torch.from_numpy(g.in_col)
    inv = torch.from_numpy(g.inv32)

    def agg(M):
        return torch.zeros_like(M).index_add(0, rows, M[cols])

    def b16(x):  # BF16 rounding in the forward pass, identity in the backward pass
        return x + (x.float().to(torch.bfloat16).double() - x).detach()

    F = torch.from_numpy(g.features())
    X = b16(F)
    for l in range(G.LAYERS):
        d, r, o = G.layer_in(l), G.layer_msg(l), offs[l]
        if l == 0:
            M = (F.float() * inv.float()[:, None]).double()
        else:
            U = p[o:o + d * r].reshape(d, r)
            o += d * r
            M = b16(inv[:, None] * (X @ U))
        Ws = p[o:o + d * G.HID].reshape(d, G.HID)
        Wn = p[o + d * G.HID:o + d * G.HID + r * G.HID].reshape(r, G.HID)
        b = p[o + d * G.HID + r * G.HID:o + d * G.HID + r * G.HID + G.HID]
        X = b16(torch.relu(X @ Ws + b16(agg(M)) @ Wn + b))
    y = X @ p[head:head + G.HID] + p[head + G.HID]
    live = torch.from_numpy(g.live)
    if kind == "mse":
        t = torch.from_numpy(G.target(pr, g))
        r = torch.where(live, y - t, torch.zeros_like(y))
        loss = (r * r).sum() / max(g.n, 1)
    else:
        logx = torch.log_softmax(y[live], dim=0)
        q = torch.from_numpy(np.asarray(pr, np.float64))[live]
        pos = q > 0
        loss = (q[pos] * (torch.log(q[pos]) - logx[pos])).sum()
    loss.backward()
    return float(loss.detach()), p.grad.numpy(), y.detach().numpy()


def random_graph(rng, V, E):
    frm = rng.integers(0, V, E)
    to = rng.integers(0, V, E)
    return frm, to


@pytest.mark.parametrize("seed,kind", [(1, "mse"), (2, "mse"), (3, "kl"), (4, "kl")])
def test_oracle_gradient_matches_autograd(seed, kind):
    rng = np.random.default_rng(seed)
    V = 300
    frm, to = random_graph(rng, V, 1500)
    g = G.Csr.from_edges(V, frm, to)
    pr = rng.random(V) + 0.1
    pr /= pr.sum()
    p = G.glorot_init(seed)
    p[G.layer_offsets()[1] - 1] = 0.05  # a non-zero bias somewhere
    loss, grad = G.loss_grad(p, g, pr, kind)
    tl, tg, ty = torch_loss(p, g, pr, kind)
    y, _ = G.forward(p, g)
    np.testing.assert_allclose(y, ty, rtol=1e-12, atol=1e-12)
    assert abs(loss - tl) <= 1e-12 * max(1.0, abs(tl))
    np.testing.assert_allclose(grad, tg, rtol=1e-9, atol=1e-12)


def test_oracle_handles_deleted_slots_and_isolated_nodes():
    rng = np.random.default_rng(7)
    V = 120
    frm, to = random_graph(rng, V, 400)
    keep = (frm % 10 != 3) & (to % 10 != 3)
    g0 = G.Csr.from_edges(V, frm[keep], to[keep])
    deg = g0.out_deg.copy()
    deg[np.arange(V) % 10 == 3] = G.DELETED
    g = G.Csr(g0.in_off, g0.in_col, deg)
    pr = np.where(g.live, 1.0 / g.n, 0.0)
    p = G.glorot_init(11)
    for kind in ("mse", "kl"):
        loss, grad = G.loss_grad(p, g, pr, kind)
        tl, tg, _ = torch_loss(p, g, pr, kind)
        assert abs(loss - tl) <= 1e-12 * max(1.0, abs(tl))
        np.testing.assert_allclose(grad, tg, rtol=1e-9, atol=1e-12)
    y, _ = G.forward(p, g)
    x0 = G.start_vector(y, g)
    assert abs(x0.sum() - 1.0) < 1e-12 and np.all(x0[~g.live] == 0)


def test_bf16_round_ties_to_even():
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -8, -2.5, 3.14159265], np.float32)
    r = G.bf16_round(x)
    np.testing.assert_array_equal(r[:4], np.array([1.0, 1.0, 1.0 + 2 ** -6, -2.5], np.float32))
    assert r[4] == np.float32(torch.tensor(3.14159265).to(torch.bfloat16).float().item())
