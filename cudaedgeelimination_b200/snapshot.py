"""GraphSnapshot mirror (include/cuda_edge_elimination/graph.hpp:13-37) on numpy arrays.

The layout is the reference's: integer coordinates, a stable edge list whose positions are the
edge ids, and an active-only CSR with rows ascending by neighbour.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field

import numpy as np

from . import _native

EUC_2D = 0
CEIL_2D = 1


def _ptr(array: np.ndarray, ctype):
    return array.ctypes.data_as(ctypes.POINTER(ctype))


@dataclass
class GraphSnapshot:
    n: int
    dist_type: int
    x: np.ndarray  # int64 [n]
    y: np.ndarray  # int64 [n]
    edge_u: np.ndarray  # int32 [m]
    edge_v: np.ndarray  # int32 [m]
    edge_w: np.ndarray  # int64 [m]
    active: np.ndarray  # uint8 [m]
    row_offsets: np.ndarray = field(default=None)  # int32 [n+1]
    neighbors: np.ndarray = field(default=None)
    csr_edge_ids: np.ndarray = field(default=None)
    csr_weights: np.ndarray = field(default=None)

    def __post_init__(self):
        self.x = np.ascontiguousarray(self.x, dtype=np.int64)
        self.y = np.ascontiguousarray(self.y, dtype=np.int64)
        self.edge_u = np.ascontiguousarray(self.edge_u, dtype=np.int32)
        self.edge_v = np.ascontiguousarray(self.edge_v, dtype=np.int32)
        self.edge_w = np.ascontiguousarray(self.edge_w, dtype=np.int64)
        self.active = np.ascontiguousarray(self.active, dtype=np.uint8)
        if self.row_offsets is None:
            self.rebuild_csr()

    @property
    def m(self) -> int:
        return int(self.edge_u.shape[0])

    def copy(self) -> "GraphSnapshot":
        return GraphSnapshot(self.n, self.dist_type, self.x.copy(), self.y.copy(), self.edge_u.copy(),
                             self.edge_v.copy(), self.edge_w.copy(), self.active.copy())

    def rebuild_csr(self) -> None:
        """GraphSnapshot::RebuildCsr (src/common/graph.cpp:230-282): slots are filled in edge-id
        order (u-row then v-row per edge); when the edge list is not canonically sorted by (u,v)
        each row is sorted by (neighbour, edge id, weight)."""
        act = np.flatnonzero(self.active).astype(np.int64)
        u, v, w = self.edge_u[act], self.edge_v[act], self.edge_w[act]
        k = act.shape[0]
        frm = np.empty(2 * k, np.int32)
        to = np.empty(2 * k, np.int32)
        ids = np.empty(2 * k, np.int32)
        ws = np.empty(2 * k, np.int64)
        frm[0::2], frm[1::2] = u, v
        to[0::2], to[1::2] = v, u
        ids[0::2] = ids[1::2] = act
        ws[0::2] = ws[1::2] = w
        eu, ev = self.edge_u, self.edge_v
        canonical = bool(np.all(eu < ev)) and (
            self.m < 2 or bool(np.all((eu[:-1] < eu[1:]) | ((eu[:-1] == eu[1:]) & (ev[:-1] <= ev[1:])))))
        if canonical:
            order = np.argsort(frm, kind="stable")
        else:
            order = np.lexsort((ws, ids, to, frm))
        self.neighbors = np.ascontiguousarray(to[order])
        self.csr_edge_ids = np.ascontiguousarray(ids[order])
        self.csr_weights = np.ascontiguousarray(ws[order])
        counts = np.bincount(frm, minlength=self.n) if k else np.zeros(self.n, np.int64)
        self.row_offsets = np.zeros(self.n + 1, np.int32)
        self.row_offsets[1:] = np.cumsum(counts)

    def degree(self) -> np.ndarray:
        return np.diff(self.row_offsets)

    def has_active_edge(self, u: int, v: int) -> bool:
        row = self.neighbors[self.row_offsets[u]:self.row_offsets[u + 1]]
        i = np.searchsorted(row, v)
        return bool(i < row.shape[0] and row[i] == v)

    def distance(self, u: int, v: int) -> int:
        import math
        s = int(self.x[u] - self.x[v]) ** 2 + int(self.y[u] - self.y[v]) ** 2
        r = math.isqrt(s)
        if self.dist_type == EUC_2D:
            return r + (1 if s - r * r > r else 0)
        return r + (1 if r * r != s else 0)

    def check_layout(self) -> None:
        """Raw pointers are handed to native code: every array must be C-contiguous with the
        documented dtype."""
        for name, dtype in (("x", np.int64), ("y", np.int64), ("edge_u", np.int32), ("edge_v", np.int32),
                            ("edge_w", np.int64), ("active", np.uint8), ("row_offsets", np.int32),
                            ("neighbors", np.int32), ("csr_edge_ids", np.int32)):
            a = getattr(self, name)
            if a.dtype != dtype or not a.flags.c_contiguous:
                raise ValueError(f"snapshot array {name} must be C-contiguous {np.dtype(dtype).name}")

    def view(self) -> _native.GraphView:
        """cee_graph_view over this snapshot's arrays (valid while the snapshot lives)."""
        self.check_layout()
        g = _native.GraphView()
        g.n = self.n
        g.dist_type = self.dist_type
        g.x = _ptr(self.x, ctypes.c_int64)
        g.y = _ptr(self.y, ctypes.c_int64)
        g.m = self.m
        g.edge_u = _ptr(self.edge_u, ctypes.c_int32)
        g.edge_v = _ptr(self.edge_v, ctypes.c_int32)
        g.edge_w = _ptr(self.edge_w, ctypes.c_int64)
        g.active = _ptr(self.active, ctypes.c_uint8)
        g.adjacency = int(self.row_offsets[-1])
        g.row_offsets = _ptr(self.row_offsets, ctypes.c_int32)
        g.neighbors = _ptr(self.neighbors, ctypes.c_int32)
        g.csr_edge_ids = _ptr(self.csr_edge_ids, ctypes.c_int32)
        return g

    @staticmethod
    def from_edges(x, y, edges, dist_type: int = EUC_2D, weights=None) -> "GraphSnapshot":
        """Builds a snapshot from (u, v) pairs with weight = exact distance unless given."""
        x = np.asarray(x, np.int64)
        y = np.asarray(y, np.int64)
        edges = np.asarray(edges, np.int64).reshape(-1, 2)
        g = GraphSnapshot(int(x.shape[0]), dist_type, x, y, edges[:, 0].astype(np.int32),
                          edges[:, 1].astype(np.int32), np.zeros(edges.shape[0], np.int64),
                          np.ones(edges.shape[0], np.uint8))
        if weights is None:
            g.edge_w = np.array([g.distance(int(a), int(b)) for a, b in edges], np.int64)
        else:
            g.edge_w = np.ascontiguousarray(weights, dtype=np.int64)
        g.rebuild_csr()
        return g
