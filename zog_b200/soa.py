"""Label-keyed graph builder, the host-side counterpart of ``Zog.SoA``
(``lib/zog/soa.ex``).

It keeps the reference's id assignment (first-seen label gets the next id,
``soa.ex:85-103``), its edge list in insertion order, and stores both arcs of an
undirected edge -- the forward arc first, then the reverse (``soa.ex:111-128``).
``to_edge_arrays`` returns what ``Zog.SoA.to_edge_arrays/1`` hands to the NIF
(``soa.ex:268-279``).
"""
from __future__ import annotations

from typing import Any, Hashable

import numpy as np


class SoA:
    """Mutable builder; every mutator returns ``self`` so calls chain like the
    reference's pipelines (``Zog.directed() |> Zog.add_edge(...)``)."""

    def __init__(self, kind: str = "directed"):
        if kind not in ("directed", "undirected"):
            raise ValueError("kind must be 'directed' or 'undirected'")
        self.kind = kind
        self.label_to_id: dict[Hashable, int] = {}
        self.id_to_label: dict[int, Hashable] = {}
        self._labels: list[Hashable] = []  # insertion order (the reference keeps it reversed)
        self._from: list[int] = []
        self._to: list[int] = []
        self._w: list[float] = []
        self._bulk: list[tuple[np.ndarray, np.ndarray, np.ndarray]] = []
        self.next_id = 0
        self.integer_labels = False

    # -- nodes -------------------------------------------------------------
    def ensure_node(self, label: Hashable) -> int:
        """soa.ex:85-103: existing id, or the next id for a new label."""
        i = self.label_to_id.get(label)
        if i is not None:
            return i
        i = self.next_id
        self.label_to_id[label] = i
        self.id_to_label[i] = label
        self._labels.append(label)
        self.next_id = i + 1
        return i

    def add_node(self, label: Hashable) -> "SoA":
        self.ensure_node(label)
        return self

    # -- edges -------------------------------------------------------------
    def add_edge(self, frm: Hashable, to: Hashable, weight: Any = 1.0) -> "SoA":
        """soa.ex:111-128: undirected edges store the forward and the reverse arc."""
        s = self.ensure_node(frm)
        d = self.ensure_node(to)
        w = _to_float(weight)
        self._from.append(s); self._to.append(d); self._w.append(w)
        if self.kind == "undirected":
            self._from.append(d); self._to.append(s); self._w.append(w)
        return self

    def add_unweighted_edge(self, frm, to) -> "SoA":
        return self.add_edge(frm, to, 1.0)

    def add_id_edges(self, frm, to, weight=None) -> "SoA":
        """Bulk append of edges between existing integer ids (array inputs, for
        large synthetic graphs).  Undirected edges interleave forward and reverse
        arcs exactly like repeated add_edge calls."""
        frm = np.ascontiguousarray(frm, dtype=np.uint32)
        to = np.ascontiguousarray(to, dtype=np.uint32)
        w = np.ones(frm.size) if weight is None else np.ascontiguousarray(weight, dtype=np.float64)
        if frm.size and int(max(frm.max(), to.max())) >= self.next_id:
            raise ValueError("edge endpoint is not a node of the builder")
        if self.kind == "undirected":
            f2 = np.empty(2 * frm.size, np.uint32); t2 = np.empty(2 * frm.size, np.uint32)
            f2[0::2] = frm; f2[1::2] = to; t2[0::2] = to; t2[1::2] = frm
            frm, to, w = f2, t2, np.repeat(w, 2)
        self._flush()
        self._bulk.append((frm, to, w))
        return self

    def _flush(self):
        if self._from:
            self._bulk.append((np.asarray(self._from, np.uint32), np.asarray(self._to, np.uint32),
                               np.asarray(self._w, np.float64)))
            self._from, self._to, self._w = [], [], []

    # -- queries -------------------------------------------------------------
    def node_count(self) -> int:
        return self.next_id

    def edge_count(self) -> int:
        return len(self._from) + sum(b[0].size for b in self._bulk)

    def all_labels(self) -> list:
        if self.integer_labels:
            return list(range(self.next_id))
        return list(self._labels)

    @property
    def nodes(self) -> list:
        """Labels newest first, the reference's ``nodes`` field layout."""
        return list(reversed(self._labels))

    def label_of(self, i: int):
        return i if self.integer_labels else self.id_to_label.get(i)

    def id_of(self, label):
        return label if self.integer_labels else self.label_to_id.get(label)

    def to_edge_arrays(self):
        """soa.ex:268-279: (from, to, weight) in insertion order."""
        self._flush()
        if not self._bulk:
            return np.zeros(0, np.uint32), np.zeros(0, np.uint32), np.zeros(0, np.float64)
        if len(self._bulk) > 1:
            f = np.concatenate([b[0] for b in self._bulk]); t = np.concatenate([b[1] for b in self._bulk])
            w = np.concatenate([b[2] for b in self._bulk])
            self._bulk = [(f, t, w)]
        return self._bulk[0]

    @classmethod
    def with_integer_ids(cls, kind: str, node_count: int) -> "SoA":
        """An integer-labelled builder (what ``build_from_labels`` makes for
        ``integer_labels: true`` readers, resource_graph.ex:1531-1548)."""
        b = cls(kind)
        b.next_id = int(node_count)
        b.integer_labels = True
        return b


def _to_float(w) -> float:
    """soa.ex:282-285: nil and non-numbers become 1.0, integers become floats."""
    if w is None or isinstance(w, bool):
        return 1.0
    if isinstance(w, (int, float, np.integer, np.floating)):
        return float(w)
    return 1.0


def directed() -> SoA:
    return SoA("directed")


def undirected() -> SoA:
    return SoA("undirected")
