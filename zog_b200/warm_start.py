"""Training and use of the learned PageRank warm start (``zogcu_gnn_*``).

The reference always starts PageRank from the uniform vector
(priv/zog/src/centrality.zig:912-918).  Here a 3-layer message-passing network
(hidden 64, BF16 weights, FP32 accumulation; kernels in csrc/gnn.cu) predicts
log(n * pagerank) from degree features, its softmax becomes the start vector,
and power iteration still runs to the caller's tolerance -- the plain method
decides the result; the network only sets where it starts.

Training data are seeded synthetic graphs (R-MAT scales 12-18, Barabasi-Albert
m = 2-16, Watts-Strogatz k = 10, p = 0.1; n = 4k-262k), plus a smaller set of
larger R-MAT (scales 19-22) and Barabasi-Albert (n = 2^19-2^22) graphs so that
the network has seen the sizes it is used on; targets are FP64 PageRank
vectors the plain GPU method computes to L1 1e-9.  Every step of training
(forward, backward, Adam) runs in the library's own CUDA kernels.

    python -m zog_b200.warm_start --graphs 2000 --large 256 --epochs 24 --out zog_b200/data/warm_start.zogn
"""
from __future__ import annotations

import argparse
import math
import os
import time

import numpy as np

from . import _native

HERE = os.path.dirname(os.path.abspath(__file__))
DEFAULT_WEIGHTS = os.path.join(HERE, "data", "warm_start.zogn")


def load_default() -> _native.WarmStart:
    """The network trained by this module's main(), shipped with the package."""
    return _native.WarmStart.load_file(DEFAULT_WEIGHTS)


# ---- seeded training / evaluation graphs --------------------------------------

def training_specs(count: int, seed: int = 2024, min_log2n: float = 12.0, max_log2n: float = 18.0):
    """`count` graph descriptions, cycling R-MAT / BA / WS, sizes log-uniform."""
    rng = np.random.default_rng(seed)
    specs = []
    for i in range(count):
        kind = ("rmat", "ba", "ws")[i % 3]
        gseed = int(rng.integers(1, 2 ** 62))
        if kind == "rmat":
            scale = int(rng.integers(int(min_log2n), int(max_log2n) + 1))
            specs.append(("rmat", dict(scale=scale, edge_factor=int(rng.integers(4, 17)), seed=gseed)))
        else:
            n = int(round(2 ** rng.uniform(min_log2n, max_log2n)))
            if kind == "ba":
                specs.append(("ba", dict(n=n, m=int(rng.integers(2, 17)), seed=gseed)))
            else:
                specs.append(("ws", dict(n=n, k=10, beta=0.1, seed=gseed)))
    return specs


def large_specs(count: int, seed: int = 4048):
    """`count` larger graph descriptions, alternating R-MAT scales 19-22 and
    Barabasi-Albert n = 2^19-2^22 (log-uniform), for size generalisation."""
    rng = np.random.default_rng(seed)
    specs = []
    for i in range(count):
        gseed = int(rng.integers(1, 2 ** 62))
        if i % 2 == 0:
            specs.append(("rmat", dict(scale=int(rng.integers(19, 23)), edge_factor=int(rng.integers(4, 17)),
                                       seed=gseed)))
        else:
            specs.append(("ba", dict(n=int(round(2 ** rng.uniform(19, 22))), m=int(rng.integers(2, 17)),
                                     seed=gseed)))
    return specs


def make_graph(kind: str, p: dict) -> _native.Graph:
    if kind == "rmat":
        return _native.Graph.rmat(p["scale"], p["edge_factor"], p["seed"], directed=True)
    if kind == "ba":
        return _native.Graph.barabasi_albert(p["n"], p["m"], p["seed"], directed=True)
    if kind == "ws":
        return _native.Graph.watts_strogatz(p["n"], p["k"], p["beta"], p["seed"], directed=False)
    raise ValueError(kind)


def solve(g: _native.Graph, damping=0.85, tol=1e-9, max_iterations=200):
    """FP64 PageRank from the uniform start into a device tensor (torch, f64)."""
    import torch

    V, _, _ = g.info()
    out = torch.empty(max(V, 1), dtype=torch.float64, device="cuda")
    st = g.pagerank_device(out.data_ptr(), damping, max_iterations, tol,
                           stream=torch.cuda.current_stream().cuda_stream)
    torch.cuda.current_stream().synchronize()
    return out, st


# ---- training ------------------------------------------------------------------

def train(net: _native.WarmStart, specs, epochs: int = 8, lr: float = 3e-3, lr_min: float = 1e-4,
          seed: int = 0, loss_kind: int = _native.LOSS_KL, log=print):
    """Adam over the graphs of `specs` (all held on the device), cosine decay
    of the learning rate; returns the mean loss of every epoch.  The default
    loss, KL(pr || softmax(y)), weights each node's error by its rank mass --
    the quantity the L1 residual of the power iteration measures."""
    t0 = time.time()
    data = []
    for kind, p in specs:
        g = make_graph(kind, p)
        pr, _ = solve(g)
        data.append((g, pr))
    log(f"built {len(data)} graphs with targets in {time.time() - t0:.1f} s")
    rng = np.random.default_rng(seed)
    steps = epochs * len(data)
    history = []
    k = 0
    for ep in range(epochs):
        losses = []
        for i in rng.permutation(len(data)):
            g, pr = data[i]
            a = lr_min + 0.5 * (lr - lr_min) * (1 + math.cos(math.pi * k / max(steps, 1)))
            losses.append(net.train_step(g, pr.data_ptr(), a, loss_kind))
            k += 1
        history.append(float(np.mean(losses)))
        log(f"epoch {ep}: mean loss {history[-1]:.4f} ({time.time() - t0:.1f} s)")
    for g, _ in data:
        g.destroy()
    return history


# ---- evaluation ----------------------------------------------------------------

def compare_starts(net: _native.WarmStart, g: _native.Graph, damping=0.85, tol=1e-9, max_iterations=200,
                   repeats: int = 3):
    """Iterations and device time to `tol` from the uniform and the learned
    start (the learned time includes the network's inference), plus the
    relative L1 distance of both results to each other."""
    import torch

    V, _, _ = g.info()
    stream = torch.cuda.current_stream()
    sp = stream.cuda_stream
    xu = torch.empty(max(V, 1), dtype=torch.float64, device="cuda")
    xl = torch.empty_like(xu)
    x0 = torch.empty_like(xu)
    res = {}
    for name in ("uniform", "learned"):
        times = []
        for _ in range(repeats + 1):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            if name == "uniform":
                st = g.pagerank_device(xu.data_ptr(), damping, max_iterations, tol, stream=sp)
            else:
                net.predict_device(g, x0.data_ptr(), stream=sp)
                st = g.pagerank_device(xl.data_ptr(), damping, max_iterations, tol, x0_ptr=x0.data_ptr(),
                                       stream=sp)
            e1.record(stream)
            e1.synchronize()
            times.append(e0.elapsed_time(e1))
        res[name] = dict(iterations=int(st["iterations"]), ms=float(np.median(times[1:])))
    times = []
    for _ in range(repeats + 1):  # the network's inference alone
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        net.predict_device(g, x0.data_ptr(), stream=sp)
        e1.record(stream)
        e1.synchronize()
        times.append(e0.elapsed_time(e1))
    res["inference_ms"] = float(np.median(times[1:]))
    den = float(xu[:V].abs().sum())
    res["rel_l1_between"] = float((xu[:V] - xl[:V]).abs().sum()) / den if den else 0.0
    # quality of the start itself: L1 distance to the converged vector
    res["start_l1_uniform"] = float((xu[:V] - 1.0 / max(V, 1)).abs().sum())
    res["start_l1_learned"] = float((xu[:V] - x0[:V]).abs().sum())
    return res


def time_inference(scale: int, reps: int) -> list:
    """CUDA-event time of each of `reps` inference calls (start vector into a
    device buffer) of the shipped network on a seeded directed R-MAT graph."""
    import torch

    g = _native.Graph.rmat(scale, 16, 1000 + scale, directed=True)
    net = load_default()
    try:
        V, _, _ = g.info()
        x0 = torch.empty(max(V, 1), dtype=torch.float64, device="cuda")
        stream = torch.cuda.current_stream()
        times = []
        for _ in range(reps):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            net.predict_device(g, x0.data_ptr(), stream=stream.cuda_stream)
            e1.record(stream)
            torch.cuda.synchronize()
            times.append(e0.elapsed_time(e1))
            print(f"rmat {scale}: inference {times[-1]:.3f} ms", flush=True)
        return times
    finally:
        net.destroy()
        g.destroy()


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--graphs", type=int, default=2000)
    ap.add_argument("--large", type=int, default=256, help="extra graphs of 2^19-2^22 nodes")
    ap.add_argument("--epochs", type=int, default=24)
    ap.add_argument("--lr", type=float, default=3e-3)
    ap.add_argument("--seed", type=int, default=2024)
    ap.add_argument("--init-seed", type=int, default=1)
    ap.add_argument("--loss", choices=("kl", "mse"), default="kl")
    ap.add_argument("--out", default=DEFAULT_WEIGHTS)
    ap.add_argument("--eval-rmat", type=int, default=20, help="held-out R-MAT scale to report (0 = none)")
    ap.add_argument("--time-rmat", type=int, default=0,
                    help="no training: time the shipped network's inference on a seeded directed R-MAT graph "
                         "of this scale (edge factor 16, seed 1000 + scale)")
    ap.add_argument("--reps", type=int, default=4, help="inference calls timed with --time-rmat")
    args = ap.parse_args(argv)
    if args.time_rmat:
        time_inference(args.time_rmat, args.reps)
        return
    net = _native.WarmStart.create(args.init_seed)
    kind = _native.LOSS_KL if args.loss == "kl" else _native.LOSS_LOG_MSE
    specs = training_specs(args.graphs, args.seed) + large_specs(args.large, args.seed + 1)
    train(net, specs, args.epochs, args.lr, loss_kind=kind)
    os.makedirs(os.path.dirname(os.path.abspath(args.out)), exist_ok=True)
    net.save(args.out)
    print(f"saved {args.out}")
    if args.eval_rmat:
        g = _native.Graph.rmat(args.eval_rmat, 16, 1000 + args.eval_rmat, directed=True)
        print({"rmat": args.eval_rmat, **compare_starts(net, g)})
        g.destroy()
        g = _native.Graph.barabasi_albert(1 << args.eval_rmat, 8, 77, directed=True)
        print({"ba": 1 << args.eval_rmat, **compare_starts(net, g)})
        g.destroy()


if __name__ == "__main__":
    main()
