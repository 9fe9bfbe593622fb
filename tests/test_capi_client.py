"""The C ABI from a plain C caller (tests/capi_client.c), compiled against
include/zogcu.h and linked to the library the way the NIF shim would be.

Without a GPU: the argument and status checks.  With one: PageRank and
Brandes of two graphs through the C program's host buffers, against the
oracle (rel L1 <= 1e-9, the same iteration count; the betweenness zeros
exact)."""
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT, rel_l1

TOL = 1e-9


@pytest.fixture(scope="module")
def client(tmp_path_factory):
    from zog_b200 import build

    so = build.build()
    libdir = os.path.dirname(os.path.abspath(so))
    exe = str(tmp_path_factory.mktemp("capi") / "capi_client")
    subprocess.run(["gcc", "-std=c99", "-O1", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "capi_client.c"), "-L", libdir, "-lzogcu",
                    f"-Wl,-rpath,{libdir}", "-o", exe], check=True)
    return exe


def test_c_caller_argument_checks(client):
    r = subprocess.run([client, "check"], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    assert r.stdout.strip() == "check ok"


def _run(client, tmp_path, V, f, t, damping=0.85, max_iter=200, tol=1e-9):
    path = tmp_path / "edges.txt"
    with open(path, "w") as fh:
        fh.write(f"{V}\n")
        fh.writelines(f"{a} {b}\n" for a, b in zip(f, t))
    r = subprocess.run([client, "run", str(path), repr(damping), str(max_iter), repr(tol)],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    pr = np.zeros(V)
    bc = np.zeros(V)
    it = None
    for line in r.stdout.splitlines():
        k, *rest = line.split()
        if k == "iterations":
            it = int(rest[0])
        elif k == "pr":
            pr[int(rest[0])] = float(rest[1])
        elif k == "bc":
            bc[int(rest[0])] = float(rest[1])
    return pr, bc, it


@pytest.mark.gpu
@pytest.mark.parametrize("graph", ["dangling", "rmat10"])
def test_c_caller_matches_oracle(client, oracle, tmp_path, graph):
    if graph == "dangling":
        # sinks (4, 6, 7), a self-loop, a duplicate arc and an isolated node (7)
        V, f, t = 8, [0, 0, 1, 2, 2, 3, 3, 5, 5, 0], [1, 2, 2, 0, 3, 4, 3, 6, 6, 1]
    else:
        V, f, t = oracle.rmat(10, 8, 1010, directed=True)
        f, t = list(map(int, f)), list(map(int, t))
    pr, bc, it = _run(client, tmp_path, V, f, t)
    A = oracle.ArrayGraph(V, f, t)
    try:
        ref_pr, ref_it, _ = A.pagerank(0.85, 200, 1e-9)
        ref_bc, _ = A.betweenness_unweighted()
    finally:
        A.close()
    assert it == ref_it
    assert rel_l1(pr, ref_pr) <= TOL
    assert rel_l1(bc, ref_bc) <= TOL
    assert np.array_equal(bc == 0, ref_bc == 0)
