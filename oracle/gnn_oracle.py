"""CPU oracle of the learned PageRank warm start (test infrastructure only:
the tests import it to check the CUDA forward and backward kernels; nothing in
the library calls it).

The reference has no learned start -- PageRank always starts from 1/n
(priv/zog/src/centrality.zig:912-918) -- so this is the oracle of the
library's own extension, written directly from the model's definition with a
hand-derived backward pass (float64 throughout).  The CPU tests pin it against
torch autograd; the GPU tests compare the CUDA kernels with it.

Model (hidden 64, messages 8 wide; parameters in one flat FP32 vector,
BF16-rounded for the forward pass; b() = round to BF16, nearest-even):
    features  F(v) = [log(1+indeg), log(1+outdeg), outdeg == 0, 1/n]  (FP32)
    inv(u)    = 1/outdeg(u) (0 for dangling and deleted nodes)
    layer 0   M_0(u) = F(u) inv(u)                         (FP32, 4 wide)
              A_0(v) = sum_{u in in(v)} M_0(u)
              H_0 = b(relu(b(F) Ws_0 + b(A_0) Wn_0 + b_0))
    layer l   M_l(u) = b(inv(u) (H_{l-1}(u) U_l))         (8 wide, l = 1, 2)
              A_l(v) = sum_{u in in(v)} M_l(u)
              H_l = b(relu(H_{l-1} Ws_l + b(A_l) Wn_l + b_l))
    head      y = H_2 w_o + b_o      (a prediction of log(n * pr))
    loss      "mse": mean over live nodes of (y - log(n pr))^2
              "kl":  KL(pr || softmax(y)) = sum_v pr(v) log(pr(v) / x0(v))
    start     x0 = softmax(y) over live nodes
Each layer's aggregate is the PageRank propagation of a message; the message
of layers 1 and 2 is a learned 8-wide projection U_l of the hidden state, so
the aggregate H -> agg(H) Wn of a full-width layer is replaced by the
rank-8 form agg(H U) Wn, and every arc carries 16 bytes instead of 128.
Flat layout: layer 0 [Ws (4 x 64) | Wn (4 x 64) | b (64)]; layers 1, 2
[U (64 x 8) | Ws (64 x 64) | Wn (8 x 64) | b (64)]; then [w_o (64) | b_o].
The roundings b() pass gradients straight through.
"""
from __future__ import annotations

import numpy as np

HID = 64
NFEAT = 4
MSG = 8
LAYERS = 3
DELETED = 0xFFFFFFFF


def layer_in(l):
    return NFEAT if l == 0 else HID


def layer_msg(l):
    """Width of layer l's message (and aggregate)."""
    return NFEAT if l == 0 else MSG


def layer_size(l):
    d, r = layer_in(l), layer_msg(l)
    return (0 if l == 0 else d * r) + d * HID + r * HID + HID


def layer_offsets():
    offs, o = [], 0
    for l in range(LAYERS):
        offs.append(o)
        o += layer_size(l)
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
    """Per layer (U or None, Ws, Wn, b), then w_o and b_o."""
    p = np.asarray(p, np.float64)
    offs, head = layer_offsets()
    layers = []
    for l in range(LAYERS):
        d, r, o = layer_in(l), layer_msg(l), offs[l]
        U = None
        if l > 0:
            U = p[o:o + d * r].reshape(d, r)
            o += d * r
        Ws = p[o:o + d * HID].reshape(d, HID)
        Wn = p[o + d * HID:o + d * HID + r * HID].reshape(r, HID)
        b = p[o + d * HID + r * HID:o + d * HID + r * HID + HID]
        layers.append((U, Ws, Wn, b))
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
        self.inv32 = self.inv.astype(np.float32).astype(np.float64)  # the kernels' FP32 1/outdeg
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

    def agg(self, M):
        """A(v) = sum over in-arcs u->v of M(u)."""
        A = np.zeros_like(M)
        np.add.at(A, self.rows, M[self.in_col])
        return A

    def agg_t(self, G):
        """Transpose of agg: out(u) = sum over arcs u->v of G(v)."""
        out = np.zeros_like(G)
        np.add.at(out, self.in_col, G[self.rows])
        return out

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
    (per layer: the dense operands X, b(A) and the output H)."""
    layers, wo, bo = unpack(bf16_round(p))
    F = g.features()
    X = b16(F)
    cache = []
    for l, (U, Ws, Wn, b) in enumerate(layers):
        if l == 0:
            M = (F.astype(np.float32) * g.inv32.astype(np.float32)[:, None]).astype(np.float64)
        else:
            M = b16(g.inv32[:, None] * (X @ U))
        Ab = b16(g.agg(M))
        H = b16(np.maximum(X @ Ws + Ab @ Wn + b, 0.0))
        cache.append((X, Ab, H))
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
    H_last = cache[-1][2]
    grad[head:head + HID] = H_last.T @ dy
    grad[head + HID] = dy.sum()
    dH = np.outer(dy, wo)
    for l in range(LAYERS - 1, -1, -1):
        X, Ab, H = cache[l]
        U, Ws, Wn, _ = layers[l]
        d, r, o = layer_in(l), layer_msg(l), offs[l]
        if l > 0:
            o_u, o = o, o + d * r
        dP = dH * (H > 0)
        grad[o:o + d * HID] = (X.T @ dP).ravel()
        grad[o + d * HID:o + d * HID + r * HID] = (Ab.T @ dP).ravel()
        grad[o + d * HID + r * HID:o + d * HID + r * HID + HID] = dP.sum(axis=0)
        if l > 0:
            dQ = g.inv32[:, None] * g.agg_t(dP @ Wn.T)  # through M = b(inv * (X U))
            grad[o_u:o_u + d * r] = (X.T @ dQ).ravel()
            dH = dP @ Ws.T + dQ @ U.T
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
    SplitMix64 stream (24-bit uniforms) in flat-layout order, each matrix with
    its own fan (din + dout), biases zero."""
    mask = (1 << 64) - 1
    state = [seed & mask]

    def nxt():
        state[0] = (state[0] + 0x9E3779B97F4A7C15) & mask
        z = state[0]
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & mask
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & mask
        return z ^ (z >> 31)

    def fill(p, o, rows, cols):
        a = np.float32(np.sqrt(np.float32(6.0) / np.float32(rows + cols)))
        for i in range(rows * cols):
            u = np.float32((nxt() >> 40) * (1.0 / 16777216.0)) * np.float32(2.0) - np.float32(1.0)
            p[o + i] = a * u
        return o + rows * cols

    p = np.zeros(num_params(), np.float32)
    offs, head = layer_offsets()
    for l in range(LAYERS):
        d, r, o = layer_in(l), layer_msg(l), offs[l]
        if l > 0:
            o = fill(p, o, d, r)
        o = fill(p, o, d, HID)
        fill(p, o, r, HID)
    fill(p, head, HID, 1)
    return p
