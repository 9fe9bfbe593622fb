"""CPU oracle of the learned PageRank warm start (test infrastructure only:
the tests import it to check the CUDA forward and backward kernels; nothing in
the library calls it).

The reference has no learned start -- PageRank always starts from 1/n
(priv/zog/src/centrality.zig:912-918) -- so this is the oracle of the
library's own extension, written directly from the model's definition with a
hand-derived backward pass (float64 throughout).  The CPU tests pin it against
torch autograd; the GPU tests compare the CUDA kernels with it.

Model (hidden 64; parameters in one flat FP32 vector, BF16-rounded for the
forward pass; b() = round to BF16, nearest-even):
    features  F(v) = [log(1+indeg), log(1+outdeg), outdeg == 0, 1/n]  (FP32)
    agg(X)(v) = sum_{u in in(v)} X(u) / outdeg(u)
    layer l   A_l = agg(H_{l-1}),  H_0 = F
              H_l = b(relu(b(H_{l-1}) Ws_l + b(A_l) Wn_l + b_l)),  l = 1..3
    head      y = H_3 w_o + b_o      (a prediction of log(n * pr))
    loss      "mse": mean over live nodes of (y - log(n pr))^2
              "kl":  KL(pr || softmax(y)) = sum_v pr(v) log(pr(v) / x0(v))
    start     x0 = softmax(y) over live nodes
Flat layout: per layer [Ws (din x 64) | Wn (din x 64) | b (64)], then
[w_o (64) | b_o].  The roundings b() pass gradients straight through.
"""
from __future__ import annotations

import numpy as np

HID = 64
NFEAT = 4
LAYERS = 3
DELETED = 0xFFFFFFFF


def layer_in(l):
    return NFEAT if l == 0 else HID


def layer_offsets():
    offs, o = [], 0
    for l in range(LAYERS):
        offs.append(o)
        o += 2 * layer_in(l) * HID + HID
    return offs, o


def num_params():
    _, head = layer_offsets()
    return head + HID + 1


def bf16_round(p):
    """Round float32 values to the nearest BF16 (ties to even), as float32."""
    b = np.ascontiguousarray(p, np.float32).view(np.uint32).astype(np.uint64)
    r = ((b + 0x7FFF + ((b >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32)


def unpack(p):
    p = np.asarray(p, np.float64)
    offs, head = layer_offsets()
    layers = []
    for l in range(LAYERS):
        d, o = layer_in(l), offs[l]
        Ws = p[o:o + d * HID].reshape(d, HID)
        Wn = p[o + d * HID:o + 2 * d * HID].reshape(d, HID)
        b = p[o + 2 * d * HID:o + 2 * d * HID + HID]
        layers.append((Ws, Wn, b))
    return layers, p[head:head + HID], p[head + HID]


class Csr:
    """In-CSR (rows = destinations, sources ascending) plus out-degrees."""

    def __init__(self, in_off, in_col, out_deg):
        self.in_off = np.asarray(in_off, np.int64)
        self.in_col = np.asarray(in_col, np.int64)
        self.out_deg = np.asarray(out_deg, np.uint32)
        self.V = self.out_deg.size
        self.live = self.out_deg != DELETED
        self.n = int(self.live.sum())
        od = self.out_deg.astype(np.float64)
        self.inv = np.where(self.live & (self.out_deg > 0), 1.0 / np.where(od > 0, od, 1.0), 0.0)
        self.rows = np.repeat(np.arange(self.V), np.diff(self.in_off))

    @classmethod
    def from_edges(cls, V, frm, to):
        frm = np.asarray(frm, np.int64)
        to = np.asarray(to, np.int64)
        order = np.lexsort((frm, to))  # rows by destination, sources ascending
        in_col = frm[order]
        in_off = np.zeros(V + 1, np.int64)
        np.add.at(in_off, to + 1, 1)
        in_off = np.cumsum(in_off)
        out_deg = np.bincount(frm, minlength=V).astype(np.uint32)
        return cls(in_off, in_col, out_deg)

    def agg(self, X):
        A = np.zeros_like(X)
        np.add.at(A, self.rows, X[self.in_col] * self.inv[self.in_col, None])
        return A

    def agg_t(self, G):
        """Transpose of agg: out(u) = inv(u) * sum over arcs u->v of G(v)."""
        out = np.zeros_like(G)
        np.add.at(out, self.in_col, G[self.rows])
        return out * self.inv[:, None]

    def features(self):
        """FP32 features (as float64 values)."""
        indeg = np.diff(self.in_off).astype(np.float32)
        od = np.where(self.live, self.out_deg, 0).astype(np.float32)
        F = np.stack([np.log1p(indeg), np.log1p(od), (self.live & (self.out_deg == 0)).astype(np.float32),
                      np.full(self.V, np.float32(1.0) / np.float32(max(self.n, 1)), np.float32)], axis=1)
        return (F * self.live[:, None]).astype(np.float64)


def b16(x):
    """BF16 rounding of float64 values (through float32)."""
    return bf16_round(np.asarray(x, np.float32)).astype(np.float64)


def forward(p, g: Csr):
    """Network output y (float64) and the activations the backward pass needs
    (per layer: the rounded dense operands Xb, Ab and the output H)."""
    layers, wo, bo = unpack(bf16_round(p))
    X = g.features()
    cache = []
    for Ws, Wn, b in layers:
        A = g.agg(X)
        Xb, Ab = b16(X), b16(A)
        H = b16(np.maximum(Xb @ Ws + Ab @ Wn + b, 0.0))
        cache.append((Xb, Ab, H))
        X = H
    y = X @ wo + bo
    return y, cache


def target(pr, g: Csr):
    return np.where(g.live, np.log(np.maximum(np.asarray(pr, np.float64) * g.n, 1e-30)), 0.0)


def loss_grad(p, g: Csr, pr, kind: str = "kl"):
    """Loss and its gradient with respect to the (BF16-rounded) parameters."""
    layers, wo, bo = unpack(bf16_round(p))
    y, cache = forward(p, g)
    pr = np.asarray(pr, np.float64)
    if kind == "mse":
        r = np.where(g.live, y - target(pr, g), 0.0)
        n = max(g.n, 1)
        loss = float((r * r).sum() / n)
        dy = 2.0 * r / n
    elif kind == "kl":
        x0 = start_vector(y, g)
        m = y[g.live].max()
        lse = np.log(np.exp(y[g.live] - m).sum()) + m
        pos = g.live & (pr > 0)
        loss = float((pr[pos] * (np.log(pr[pos]) - y[pos] + lse)).sum())
        dy = np.where(g.live, x0 - pr, 0.0)
    else:
        raise ValueError(kind)
    offs, head = layer_offsets()
    grad = np.zeros(num_params())
    H3 = cache[-1][2]
    grad[head:head + HID] = H3.T @ dy
    grad[head + HID] = dy.sum()
    dH = np.outer(dy, wo)
    for l in range(LAYERS - 1, -1, -1):
        X, A, H = cache[l]
        Ws, Wn, _ = layers[l]
        d, o = layer_in(l), offs[l]
        dP = dH * (H > 0)
        grad[o:o + d * HID] = (X.T @ dP).ravel()
        grad[o + d * HID:o + 2 * d * HID] = (A.T @ dP).ravel()
        grad[o + 2 * d * HID:o + 2 * d * HID + HID] = dP.sum(axis=0)
        if l > 0:
            dH = dP @ Ws.T + g.agg_t(dP @ Wn.T)
    return loss, grad


def start_vector(y, g: Csr):
    """x0 = softmax(y) over live nodes (0 on deleted slots)."""
    y = np.asarray(y, np.float64)
    m = y[g.live].max() if g.n else 0.0
    e = np.where(g.live, np.exp(y - m), 0.0)
    s = e.sum()
    return e / s if s > 0 else e


def glorot_init(seed):
    """Initial weights of zogcu_gnn_create(seed): Glorot-uniform from a
    SplitMix64 stream (24-bit uniforms), biases zero."""
    mask = (1 << 64) - 1
    state = [seed & mask]

    def nxt():
        state[0] = (state[0] + 0x9E3779B97F4A7C15) & mask
        z = state[0]
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & mask
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & mask
        return z ^ (z >> 31)

    p = np.zeros(num_params(), np.float32)
    offs, head = layer_offsets()
    for l in range(LAYERS):
        d = layer_in(l)
        a = np.float32(np.sqrt(np.float32(6.0) / np.float32(d + HID)))
        for i in range(2 * d * HID):
            u = np.float32((nxt() >> 40) * (1.0 / 16777216.0)) * np.float32(2.0) - np.float32(1.0)
            p[offs[l] + i] = a * u
    a = np.float32(np.sqrt(np.float32(6.0) / np.float32(HID + 1)))
    for i in range(HID):
        u = np.float32((nxt() >> 40) * (1.0 / 16777216.0)) * np.float32(2.0) - np.float32(1.0)
        p[head + i] = a * u
    return p
