"""C ABI checks that need no GPU: the library builds for sm_100a, loads, and
exports every entry point declared in include/zogcu.h."""
import ctypes as C
import os
import re

import pytest

from conftest import ROOT


def header_functions():
    with open(os.path.join(ROOT, "include", "zogcu.h")) as f:
        text = f.read()
    return sorted(set(re.findall(r"ZOGCU_API\s+[\w\s\*]+?\b(zogcu_\w+)\s*\(", text)))


@pytest.fixture(scope="module")
def lib():
    from zog_b200 import build

    path = build.build()
    return C.CDLL(path)


def test_header_declares_entry_points():
    names = header_functions()
    for must in ("zogcu_graph_create_from_edges", "zogcu_pagerank", "zogcu_betweenness_unweighted",
                 "zogcu_graph_destroy", "zogcu_status_string", "zogcu_read_edgelist"):
        assert must in names


def test_every_declared_symbol_is_exported(lib):
    for name in header_functions():
        assert hasattr(lib, name), name


def test_python_binding_lists_every_export():
    from zog_b200 import _native

    assert sorted(_native.EXPORTS) == header_functions()


def test_status_strings(lib):
    lib.zogcu_status_string.restype = C.c_char_p
    assert lib.zogcu_status_string(0) == b"ok"
    assert lib.zogcu_status_string(2) == b"node not found"
    assert lib.zogcu_status_string(999) == b"unknown status"
    lib.zogcu_abi_version.restype = C.c_int
    assert lib.zogcu_abi_version() == 1


def test_invalid_arguments_fail_without_device(lib):
    """Argument errors are reported as status codes before any device work."""
    lib.zogcu_graph_create_from_edges.restype = C.c_int
    assert lib.zogcu_graph_create_from_edges(3, None, None, None, 0, None) == 1
    out = C.c_void_p()
    frm = (C.c_uint32 * 2)(0, 1)
    # one of the edge arrays missing
    assert lib.zogcu_graph_create_from_edges(3, frm, None, None, 2, C.byref(out)) == 1
    assert not out.value
    lib.zogcu_last_error.restype = C.c_char_p
    assert b"null" in lib.zogcu_last_error()
    assert lib.zogcu_pagerank(None, C.c_double(0.85), C.c_uint64(10), C.c_double(1e-4), None, None) == 1
    lib.zogcu_read_edgelist.restype = C.c_int
    assert lib.zogcu_read_edgelist(b"/nonexistent/file.txt", 1, 0, C.byref(out), None, None, None) == 1
    assert lib.zogcu_graph_destroy(None) == 0


def test_no_device_is_loud():
    """Without a GPU the product path raises; there is no CPU fallback."""
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is visible")
    from zog_b200 import _native

    with pytest.raises(_native.ZogCudaError) as ei:
        _native.Graph.from_edges(3, [0, 1], [1, 2])
    assert ei.value.status == 5
