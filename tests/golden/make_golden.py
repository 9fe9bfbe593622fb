"""Generates the golden fixtures under tests/golden/ with the CPU oracle.

    python tests/golden/make_golden.py --reference-root DIR   (or ZOG_REFERENCE_ROOT=DIR)

Each fixture is an .npz holding a graph in NIF insertion order (node count,
from, to, directed flag) and the oracle's outputs on it:
  pr_default   pagerank with the reference defaults (0.85, 100, 1e-4)
  pr_tight     pagerank with the benchmark options (0.85, 200, 1e-9)
  pr_d99       pagerank with damping 0.99 (centrality_test.exs:151-163)
  bc           unweighted betweenness, unscaled (the NIF's output)
  bfs_*        dist / sigma of two sources
The graphs are the reference's own test graphs (file:line in GRAPHS below),
its edge-list fixture test/fixtures/wiki_vote_sample.txt parsed by the oracle's
restatement of nif_read_edgelist (read only when the reference tree is
present), a multi-edge / self-loop graph, a tombstoned ArrayGraph and two small
R-MAT graphs.  The oracle is deterministic, so re-running reproduces the files
bit for bit; tests/test_oracle.py checks that.
"""
from __future__ import annotations

import argparse
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402


def labelled(kind, edges, extra_nodes=()):
    """SoA semantics (lib/zog/soa.ex:85-128): ids by first appearance, an
    undirected edge stores the forward then the reverse arc."""
    ids = {}

    def nid(x):
        if x not in ids:
            ids[x] = len(ids)
        return ids[x]

    frm, to = [], []
    for a, b in edges:
        s, d = nid(a), nid(b)
        frm.append(s); to.append(d)
        if kind == "undirected":
            frm.append(d); to.append(s)
    for x in extra_nodes:
        nid(x)
    return len(ids), np.array(frm, np.uint32), np.array(to, np.uint32), list(ids)


GRAPHS = {
    # centrality_test.exs:11-24 (directed A->B->C)
    "ref_directed_path": ("directed", [("A", "B"), ("B", "C")]),
    # resource_graph_test.exs:40-55 (undirected path)
    "ref_undirected_path": ("undirected", [("A", "B"), ("B", "C")]),
    # centrality_test.exs:26-39, resource_graph_test.exs:85-101 (star)
    "ref_star_undirected": ("undirected", [("center", "A"), ("center", "B"), ("center", "C")]),
    # resource_graph_test.exs:57-83, 103-129 (triangle)
    "ref_triangle_undirected": ("undirected", [("A", "B"), ("B", "C"), ("C", "A")]),
    # centrality_test.exs:137-149; centrality.zig:1456-1476 (0->1, 2->1)
    "ref_in_degree": ("directed", [("A", "B"), ("C", "B")]),
    # centrality_test.exs:151-163 (A->B->C, damping variants)
    "ref_damping_chain": ("directed", [("A", "B"), ("B", "C")]),
    # resource_graph_test.exs:501-541 (raw: true, 4 nodes)
    "ref_raw_4": ("undirected", [("A", "B"), ("B", "C"), ("C", "A"), ("B", "D")]),
    # hash_graph_parity_test.exs:9-28 (undirected path A-B-C-D)
    "ref_path4_undirected": ("undirected", [("A", "B"), ("B", "C"), ("C", "D")]),
}


def outputs(ag: O.ArrayGraph, V: int):
    out = {}
    for key, (d, it, tol) in {"pr_default": (0.85, 100, 1e-4), "pr_tight": (0.85, 200, 1e-9),
                              "pr_d99": (0.99, 100, 1e-4)}.items():
        x, iters, l1 = ag.pagerank(d, it, tol)
        out[key] = x
        out[key + "_iters"] = np.array(iters, np.uint64)
        out[key + "_l1"] = np.array(l1)
    bc, ovf = ag.betweenness_unweighted()
    out["bc"] = bc
    out["bc_overflow"] = np.array(int(ovf))
    srcs = sorted({0, V // 2}) if V else []
    for s in srcs:
        dist, sigma, _ = ag.bfs(s)
        out[f"bfs_{s}_dist"] = dist
        out[f"bfs_{s}_sigma"] = sigma
    out["bfs_sources"] = np.array(srcs, np.uint32)
    return out


def save(name, V, frm, to, directed, extra=None, labels=None, ag=None):
    if ag is None:
        ag = O.ArrayGraph(V, frm, to)
    d = {"V": np.array(V, np.uint32), "from": np.asarray(frm, np.uint32), "to": np.asarray(to, np.uint32),
         "directed": np.array(int(directed))}
    d.update(outputs(ag, ag.node_capacity))
    if extra:
        d.update(extra)
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **d)
    meta = {"V": int(V), "E": int(len(frm)), "directed": bool(directed),
            "pr_tight_iters": int(d["pr_tight_iters"]), "pr_default_iters": int(d["pr_default_iters"])}
    if labels is not None:
        meta["labels"] = [str(x) for x in labels]
    return meta


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference-root", default=os.environ.get("ZOG_REFERENCE_ROOT"),
                    help="root of the reference checkout (or set ZOG_REFERENCE_ROOT)")
    args = ap.parse_args()
    if not args.reference_root:
        ap.error("give --reference-root or set ZOG_REFERENCE_ROOT")
    O.build()
    manifest = {}
    for name, (kind, edges) in GRAPHS.items():
        V, frm, to, labels = labelled(kind, edges)
        manifest[name] = save(name, V, frm, to, kind == "directed", labels=labels)
    # single node (centrality_test.exs:47-51) and empty graph (:41-45)
    manifest["ref_single_node"] = save("ref_single_node", 1, [], [], True, labels=["A"])
    manifest["ref_empty"] = save("ref_empty", 0, [], [], True, labels=[])
    # resource_graph_test.exs:544-570: "0 1 1.5\n1 2 2.0\n2 0 1.0\n", integer labels
    manifest["ref_int_edgelist"] = save("ref_int_edgelist", 3, [0, 1, 2], [1, 2, 0], True)

    # multi-edges and self-loops (kept by the SoA builder, soa.ex:111-128)
    rng = np.random.default_rng(20261203)
    V = 40
    frm = rng.integers(0, V, 400).astype(np.uint32)
    to = rng.integers(0, V, 400).astype(np.uint32)
    frm[:15] = to[:15]  # self-loops
    frm[15:40] = frm[40:65]; to[15:40] = to[40:65]  # duplicates
    manifest["multi_selfloop"] = save("multi_selfloop", V, frm, to, True)

    # tombstones: removeNode / removeEdge on an ArrayGraph (array_graph.zig:110-152)
    V = 30
    frm = rng.integers(0, V, 150).astype(np.uint32)
    to = rng.integers(0, V, 150).astype(np.uint32)
    ag = O.ArrayGraph(V, frm, to)
    ag.remove_node(3); ag.remove_node(17)
    ag.remove_edge(int(frm[10]), int(to[10]))
    fe, nd, t_, ne, ed, _ = ag.export()
    manifest["tombstones"] = save("tombstones", V, frm, to, True, ag=ag,
                                  extra={"ag_first_edge": fe, "ag_node_deleted": nd, "ag_to": t_,
                                         "ag_next_edge": ne, "ag_edge_deleted": ed})

    # small R-MAT graphs (same generator definition as the CUDA library)
    for scale, directed, seed in ((10, True, 1010), (10, False, 1010)):
        Vr, f, t = O.rmat(scale, 8, seed, directed=directed)
        nm = f"rmat{scale}_{'dir' if directed else 'undir'}"
        raw_s, raw_d = O.rmat_raw(scale, seed, 0, 4096)
        manifest[nm] = save(nm, Vr, f, t, directed, extra={"raw_src": raw_s, "raw_dst": raw_d,
                                                           "seed": np.array(seed), "scale": np.array(scale)})

    # the reference's edge-list fixture, read as io_test.exs:11-23 does (directed)
    fx = os.path.join(args.reference_root, "test", "fixtures", "wiki_vote_sample.txt")
    if os.path.exists(fx):
        ag, next_id, labels = O.read_edgelist(fx, directed=True, integer_labels=False)
        off, col = ag.successor_csr()
        # insertion order of the directed reader = file order; recover it from the
        # head-insertion lists by reversing each node's successor run
        frm, to = [], []
        fe, nd, t_, ne, ed, _ = ag.export()
        E = len(t_)
        src_of = np.zeros(E, np.uint32)
        for v in range(next_id):
            e = fe[v]
            while e != 0xFFFFFFFF:
                src_of[e] = v
                e = ne[e]
        frm = src_of
        to = t_
        manifest["wiki_vote_sample"] = save("wiki_vote_sample", next_id, frm, to, True, labels=labels)
        with open(fx, "rb") as fh:
            raw = fh.read()
        np.savez_compressed(os.path.join(HERE, "wiki_vote_sample_text.npz"),
                            text=np.frombuffer(raw, np.uint8))
    with open(os.path.join(HERE, "manifest.json"), "w") as f:
        json.dump(manifest, f, indent=1, sort_keys=True)
    print(f"wrote {len(manifest)} fixtures to {HERE}")


if __name__ == "__main__":
    main()
