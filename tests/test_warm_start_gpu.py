"""The learned PageRank warm start on the GPU: forward pass, loss and gradient
of the CUDA kernels against the CPU oracle (oracle/gnn_oracle.py, itself
pinned against torch autograd), the start vector, the weight file, training
on the GPU, and what the trained network gains over the uniform start."""
import os

import numpy as np
import pytest

from oracle import gnn_oracle as GO

pytestmark = pytest.mark.gpu

# The kernels and the oracle round the same values to BF16, but their FP32 and
# FP64 sums can land on different sides of a rounding boundary, which moves an
# element of a hidden state by one BF16 unit (2^-8 relative).
Y_TOL = 1e-2        # max |y - y_ref| / (1 + max |y_ref|)
Y_MEAN_TOL = 1e-3   # mean |y - y_ref| / (1 + max |y_ref|)
GRAD_TOL = 2e-2     # relative L2 error per parameter block


def csr_of(G):
    in_off, in_col, _, _, deg = G.export_csr()
    return GO.Csr(in_off.astype(np.int64), in_col.astype(np.int64), deg)


def sample_graphs(native, oracle):
    V, f, t = oracle.rmat(10, 8, 31, directed=True)
    yield "rmat10", native.Graph.from_edges(V, f, t)
    yield "ba", native.Graph.barabasi_albert(1500, 3, 5, directed=True)
    yield "ws", native.Graph.watts_strogatz(1200, 10, 0.1, 6, directed=False)
    # isolated nodes and a self-loop
    yield "small", native.Graph.from_edges(7, np.array([0, 1, 2, 2, 5], np.uint32),
                                           np.array([1, 2, 0, 2, 0], np.uint32))


def param_blocks():
    """Boundaries of every weight matrix, bias and the head in the flat vector."""
    offs, head = GO.layer_offsets()
    b = []
    for l in range(GO.LAYERS):
        d, r, o = GO.layer_in(l), GO.layer_msg(l), offs[l]
        b.append(o)
        if l > 0:
            o += d * r
            b.append(o)
        b += [o + d * GO.HID, o + d * GO.HID + r * GO.HID]
    return sorted(set(b + [head, head + GO.HID, GO.num_params()]))


def perturbed_params(seed):
    p = GO.glorot_init(seed)
    rng = np.random.default_rng(seed)
    return (p + rng.normal(0, 0.05, p.size)).astype(np.float32)


def test_initial_weights_match_oracle(native):
    net = native.WarmStart.create(17)
    try:
        np.testing.assert_array_equal(net.get_params(), GO.glorot_init(17))
        assert net.num_params() == GO.num_params()
    finally:
        net.destroy()


def test_forward_and_start_vector_match_oracle(native, oracle):
    net = native.WarmStart.create(3)
    try:
        net.set_params(perturbed_params(3))
        p = net.get_params()
        for name, G in sample_graphs(native, oracle):
            try:
                g = csr_of(G)
                x0, y = net.predict(G, raw=True)
                y_ref, _ = GO.forward(p, g)
                scale = 1 + np.abs(y_ref).max()
                assert np.abs(y - y_ref).max() <= Y_TOL * scale, (name, np.abs(y - y_ref).max())
                assert np.abs(y - y_ref).mean() <= Y_MEAN_TOL * scale, (name, np.abs(y - y_ref).mean())
                # the softmax of the kernel's own y, in FP64
                ref = GO.start_vector(y.astype(np.float64), g)
                np.testing.assert_allclose(x0, ref, rtol=1e-12, atol=1e-300, err_msg=name)
                assert abs(x0.sum() - 1.0) < 1e-12
            finally:
                G.destroy()
    finally:
        net.destroy()


def test_loss_and_gradient_match_oracle(native, oracle):
    net = native.WarmStart.create(5)
    try:
        net.set_params(perturbed_params(5))
        p = net.get_params()
        for name, G in sample_graphs(native, oracle):
            try:
                g = csr_of(G)
                pr = G.pagerank(0.85, 200, 1e-12)
                for kind, code in (("mse", native.LOSS_LOG_MSE), ("kl", native.LOSS_KL)):
                    loss, grad = net.loss_grad(G, pr, code)
                    loss_ref, grad_ref = GO.loss_grad(p, g, pr, kind)
                    assert abs(loss - loss_ref) <= 1e-2 * abs(loss_ref) + 1e-6, (name, kind, loss, loss_ref)
                    bounds = param_blocks()
                    scale = np.linalg.norm(grad_ref)
                    for a, b in zip(bounds[:-1], bounds[1:]):
                        err = np.linalg.norm(grad[a:b] - grad_ref[a:b])
                        assert err <= GRAD_TOL * np.linalg.norm(grad_ref[a:b]) + 1e-6 * scale, (name, kind, a, b, err)
            finally:
                G.destroy()
    finally:
        net.destroy()


def test_weight_file_round_trip(native, tmp_path):
    net = native.WarmStart.create(9)
    try:
        net.set_params(perturbed_params(9))
        path = str(tmp_path / "w.zogn")
        net.save(path)
        net2 = native.WarmStart.load_file(path)
        try:
            np.testing.assert_array_equal(net2.get_params(), GO.bf16_round(net.get_params()))
        finally:
            net2.destroy()
        with open(path, "r+b") as f:
            f.seek(4)
            f.write(b"\x07\x00\x00\x00")  # unknown version
        with pytest.raises(native.ZogCudaError):
            native.WarmStart.load_file(path)
    finally:
        net.destroy()


def test_training_on_gpu_gains_over_uniform_start(native):
    """Train on small seeded graphs with the CUDA kernels, then solve held-out
    graphs from both starts: the same answer (the power iteration decides it), and on
    the skewed R-MAT graph a start much closer to it and fewer iterations; the
    learned start never costs more than one extra iteration."""
    import torch

    from zog_b200 import warm_start as W

    torch.cuda.init()
    net = native.WarmStart.create(1)
    try:
        hist = W.train(net, W.training_specs(48, seed=5, min_log2n=10, max_log2n=13), epochs=25, lr=3e-3,
                       log=lambda *_: None)
        assert hist[-1] < 0.5 * hist[0], hist
        held = [native.Graph.rmat(14, 8, 1014, directed=True), native.Graph.barabasi_albert(8192, 4, 99),
                native.Graph.watts_strogatz(8192, 10, 0.1, 98)]
        for i, G in enumerate(held):
            try:
                r = W.compare_starts(net, G, tol=1e-9, repeats=1)
                assert r["rel_l1_between"] <= 1e-7, r
                assert r["learned"]["iterations"] <= r["uniform"]["iterations"] + 1, r
                if i == 0:
                    assert r["start_l1_learned"] < 0.5 * r["start_l1_uniform"], r
                    assert r["learned"]["iterations"] <= r["uniform"]["iterations"] - 2, r
            finally:
                G.destroy()
    finally:
        net.destroy()


@pytest.mark.skipif(not os.path.exists(os.path.join(os.path.dirname(__file__), "..", "zog_b200", "data",
                                                    "warm_start.zogn")), reason="no trained weights shipped")
def test_shipped_weights_gain_over_uniform_start(native):
    from zog_b200 import warm_start as W

    net = W.load_default()
    try:
        for i, G in enumerate((native.Graph.rmat(16, 16, 1016, directed=True),
                               native.Graph.barabasi_albert(1 << 16, 8, 4242, directed=True))):
            try:
                r = W.compare_starts(net, G, tol=1e-9, repeats=1)
                assert r["rel_l1_between"] <= 1e-7, r
                assert r["start_l1_learned"] < r["start_l1_uniform"], r
                if i == 0:  # R-MAT: a start ~20x closer, several iterations fewer
                    assert r["start_l1_learned"] < 0.2 * r["start_l1_uniform"], r
                    assert r["learned"]["iterations"] <= r["uniform"]["iterations"] - 3, r
                else:
                    assert r["learned"]["iterations"] <= r["uniform"]["iterations"], r
            finally:
                G.destroy()
    finally:
        net.destroy()


def test_tcgen05_inference_matches_mma_sync(native, oracle, monkeypatch):
    """The tensor-memory inference kernels against the mma.sync ones and the
    oracle: the one-tile kernels (ZOGCU_GNN_TC=1) and the four-slot ones
    (ZOGCU_GNN_TC=2) compute the same products in another accumulation order
    than mma.sync, so outputs agree to the BF16 tolerances above; the two
    tcgen05 forms run the same products and agree bit for bit."""
    net = native.WarmStart.create(13)
    try:
        net.set_params(perturbed_params(13))
        p = net.get_params()
        graphs = list(sample_graphs(native, oracle))
        V, f, t = oracle.rmat(14, 8, 1014, directed=True)  # several 128-node tiles, a ragged last one
        graphs.append(("rmat14", native.Graph.from_edges(V, f, t)))
        for name, G in graphs:
            try:
                monkeypatch.setenv("ZOGCU_GNN_TC", "0")
                x_s, y_s = net.predict(G, raw=True)
                monkeypatch.setenv("ZOGCU_GNN_TC", "1")
                x_t, y_t = net.predict(G, raw=True)
                x_t2, y_t2 = net.predict(G, raw=True)
                assert np.array_equal(y_t, y_t2), name  # deterministic
                scale = 1 + np.abs(y_s).max()
                assert np.abs(y_t - y_s).max() <= Y_TOL * scale, (name, np.abs(y_t - y_s).max())
                assert np.abs(y_t - y_s).mean() <= Y_MEAN_TOL * scale, name
                y_ref, _ = GO.forward(p, csr_of(G))
                assert np.abs(y_t - y_ref).max() <= Y_TOL * (1 + np.abs(y_ref).max()), name
                assert abs(x_t.sum() - 1.0) < 1e-12
                monkeypatch.setenv("ZOGCU_GNN_TC", "2")
                x_q, y_q = net.predict(G, raw=True)
                assert np.array_equal(y_q, y_t), (name, np.abs(y_q - y_t).max())
                assert np.array_equal(x_q, x_t), name
            finally:
                G.destroy()
    finally:
        monkeypatch.delenv("ZOGCU_GNN_TC", raising=False)
        net.destroy()


def test_async_and_register_staged_aggregation(native, oracle, monkeypatch):
    """The aggregate with its gathers copied straight to shared memory
    (cp.async, the default) and the register-staged one (ZOGCU_GNN_AGG_ASYNC=0)
    against the oracle and each other, on graphs with hub rows that span many
    128-arc chunks: their partial sums meet through atomics in either order,
    and a last-bit difference can flip a BF16 rounding of the aggregate, so
    the two agree to the BF16 tolerances above, not bit for bit."""
    net = native.WarmStart.create(21)
    try:
        net.set_params(perturbed_params(21))
        p = net.get_params()
        graphs = list(sample_graphs(native, oracle))
        V, f, t = oracle.rmat(14, 8, 1014, directed=True)
        graphs.append(("rmat14", native.Graph.from_edges(V, f, t)))
        for name, G in graphs:
            try:
                y_ref, _ = GO.forward(p, csr_of(G))
                ys = {}
                for mode in ("1", "0"):
                    monkeypatch.setenv("ZOGCU_GNN_AGG_ASYNC", mode)
                    x, y = net.predict(G, raw=True)
                    assert np.abs(y - y_ref).max() <= Y_TOL * (1 + np.abs(y_ref).max()), (name, mode)
                    assert abs(x.sum() - 1.0) < 1e-12
                    ys[mode] = y
                scale = 1 + np.abs(ys["0"]).max()
                assert np.abs(ys["1"] - ys["0"]).max() <= Y_TOL * scale, name
                assert np.abs(ys["1"] - ys["0"]).mean() <= Y_MEAN_TOL * scale, name
            finally:
                G.destroy()
    finally:
        monkeypatch.delenv("ZOGCU_GNN_AGG_ASYNC", raising=False)
        net.destroy()
