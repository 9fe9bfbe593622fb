"""zogcu_pagerank_noalloc: PageRank for callers that cannot allocate device
memory (for example a NIF whose process shares the GPU with a runtime that owns
the device memory pool).  The caller owns the in-CSR, degree and output
buffers; the library's scratch is a fixed device array reserved at load time.

The test calls the entry point through the C ABI twice in a row and checks
both results against the regular entry point (zogcu_pagerank) with the same
tolerance the other PageRank tests use.  This file sorts last so that a run
stopping at its first failure has already run every other test.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
TOL = 1e-9  # relative L1, as in tests/test_pagerank_gpu.py


def rel_l1(a, b):
    return float(np.abs(a - b).sum() / np.abs(b).sum())


def test_noalloc_matches_regular_entry_point_twice():
    import torch

    assert torch.cuda.is_available(), "GPU test run without a visible CUDA device"
    from oracle import oracle as O
    from zog_b200 import _native, build

    build.build()
    L = _native.load()
    V, f, t = O.rmat(14, 8, 1014, directed=True)  # the small R-MAT configuration
    G = _native.Graph.from_edges(V, f, t)
    try:
        ref, st = G.pagerank(0.85, 200, 1e-9, stats=True)
        in_off, in_col, _, _, deg = G.export_csr()
    finally:
        G.destroy()
    d_off = torch.from_numpy(in_off.astype(np.uint32).view(np.int32)).cuda()
    d_col = torch.from_numpy(in_col.view(np.int32)).cuda()
    d_deg = torch.from_numpy(deg.view(np.int32)).cuda()
    out = torch.empty(V, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    stream = torch.cuda.current_stream().cuda_stream
    for call in range(2):
        out.fill_(-1.0)
        torch.cuda.synchronize()
        s = _native.Stats()
        rc = L.zogcu_pagerank_noalloc(d_off.data_ptr(), d_col.data_ptr(), d_deg.data_ptr(), V, in_col.size,
                                      0.85, 200, 1e-9, out.data_ptr(), C.byref(s), stream)
        assert rc == 0, L.zogcu_last_error().decode()
        x = out.cpu().numpy()
        assert rel_l1(x, ref) <= TOL, (call, rel_l1(x, ref))
        assert s.iterations == st["iterations"], call


def test_noalloc_rejects_graphs_above_its_limit():
    from zog_b200 import _native

    L = _native.load()
    rc = L.zogcu_pagerank_noalloc(None, None, None, (1 << 18) + 1, 0, 0.85, 10, 1e-4, None, None, None)
    assert rc == 8  # ZOGCU_ERR_TOO_LARGE
    assert b"262144" in L.zogcu_last_error()
