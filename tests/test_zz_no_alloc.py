"""zogcu_pagerank_noalloc: PageRank for callers that cannot allocate device
memory (for example a NIF whose process shares the GPU with a runtime that owns
the device memory pool).  The caller owns the in-CSR, degree and output
buffers; the library's scratch is a fixed device array that the first call on
a device sets up.

The tests call the entry point through the C ABI: twice in a row against the
regular entry point (zogcu_pagerank), and against the CPU oracle on a graph
with dangling nodes, at the 262,144-node limit, with a cap of 0 iterations
(the uniform start vector) and with a cap of UINT64_MAX (the call must still
stop once the chain has converged).  The tolerance is the one the other
PageRank tests use.  This file sorts last so that a run stopping at its first
failure has already run every other test.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
TOL = 1e-9  # relative L1, as in tests/test_pagerank_gpu.py
MAX_NODES = 1 << 18


def rel_l1(a, b):
    return float(np.abs(a - b).sum() / np.abs(b).sum())


def _device_csr(V, f, t):
    """In-CSR (sources ascending per row) and out-degrees on the device."""
    import torch
    from oracle import oracle as O

    in_off, in_col, deg = O.in_csr_from_edges(V, np.asarray(f, np.uint32), np.asarray(t, np.uint32))
    d_off = torch.from_numpy(in_off.astype(np.uint32).view(np.int32)).cuda()
    col = in_col if in_col.size else np.zeros(1, np.uint32)
    d_col = torch.from_numpy(col.view(np.int32)).cuda()
    d_deg = torch.from_numpy(np.ascontiguousarray(deg, np.uint32).view(np.int32)).cuda()
    return (in_off, in_col, deg), (d_off, d_col, d_deg)


def _noalloc(L, dev, V, E, max_iter, tol=1e-9, damping=0.85):
    import torch
    from zog_b200 import _native

    d_off, d_col, d_deg = dev
    out = torch.full((V,), -1.0, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    s = _native.Stats()
    rc = L.zogcu_pagerank_noalloc(d_off.data_ptr(), d_col.data_ptr(), d_deg.data_ptr(), V, E, damping,
                                  C.c_uint64(max_iter), tol, out.data_ptr(), C.byref(s),
                                  torch.cuda.current_stream().cuda_stream)
    assert rc == 0, L.zogcu_last_error().decode()
    return out.cpu().numpy(), s


@pytest.fixture(scope="module")
def lib():
    import torch

    assert torch.cuda.is_available(), "GPU test run without a visible CUDA device"
    from zog_b200 import _native, build

    build.build()
    return _native.load()


def test_noalloc_matches_regular_entry_point_twice(lib):
    from oracle import oracle as O
    from zog_b200 import _native

    V, f, t = O.rmat(14, 8, 1014, directed=True)  # the small R-MAT configuration
    G = _native.Graph.from_edges(V, f, t)
    try:
        ref, st = G.pagerank(0.85, 200, 1e-9, stats=True)
    finally:
        G.destroy()
    host, dev = _device_csr(V, f, t)
    for call in range(2):
        x, s = _noalloc(lib, dev, V, host[1].size, 200)
        assert rel_l1(x, ref) <= TOL, (call, rel_l1(x, ref))
        assert s.iterations == st["iterations"], call


def test_noalloc_against_oracle_with_dangling_nodes(lib):
    from oracle import oracle as O

    # sinks (4, 6, 7), a self-loop, a duplicate arc and an isolated node (7)
    f = [0, 0, 1, 2, 2, 3, 3, 5, 5, 0]
    t = [1, 2, 2, 0, 3, 4, 3, 6, 6, 1]
    V = 8
    ref, it, _ = O.ArrayGraph(V, f, t).pagerank(0.85, 200, 1e-9)
    host, dev = _device_csr(V, f, t)
    x, s = _noalloc(lib, dev, V, len(f), 200)
    assert rel_l1(x, ref) <= TOL
    assert s.iterations == it


def test_noalloc_at_its_node_limit(lib):
    from oracle import oracle as O

    V, f, t = O.rmat(18, 8, 1018, directed=True)
    assert V == MAX_NODES
    host, dev = _device_csr(V, f, t)
    ref, it, _, _ = O.pagerank_csr_mt(V, host[0], host[1], host[2], 0.85, 200, 1e-9)
    x, s = _noalloc(lib, dev, V, host[1].size, 200)
    assert rel_l1(x, ref) <= TOL, rel_l1(x, ref)
    assert s.iterations == it


def test_noalloc_zero_and_unbounded_caps(lib):
    from oracle import oracle as O

    V, f, t = O.rmat(12, 8, 1012, directed=True)
    host, dev = _device_csr(V, f, t)
    x0, s0 = _noalloc(lib, dev, V, host[1].size, 0)
    assert s0.iterations == 0
    assert np.array_equal(x0, np.full(V, 1.0 / V))  # the uniform start (centrality.zig:912-918)
    ref, it, _, _ = O.pagerank_csr_mt(V, host[0], host[1], host[2], 0.85, 200, 1e-9)
    x, s = _noalloc(lib, dev, V, host[1].size, 2**64 - 1)
    assert s.iterations == it
    assert rel_l1(x, ref) <= TOL
    # the initial kernel, the iteration launches of the chunks run, the copy-out
    assert s.launches <= 2 + ((it + 31) // 32) * 32


def test_noalloc_rejects_graphs_above_its_limit(lib):
    rc = lib.zogcu_pagerank_noalloc(None, None, None, MAX_NODES + 1, 0, 0.85, 10, 1e-4, None, None, None)
    assert rc == 8  # ZOGCU_ERR_TOO_LARGE
    assert b"262144" in lib.zogcu_last_error()
