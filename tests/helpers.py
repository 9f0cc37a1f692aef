"""Snapshot constructors shared by the tests (seeded; no reference data)."""
import numpy as np

from cudaedgeelimination_b200 import GraphSnapshot


def random_graph(n, m_target, seed, coord=10_000, dist_type=0, shuffle=False, active_frac=1.0):
    """Random sparse graph with distinct integer points; edges canonical unless shuffled."""
    rng = np.random.default_rng(seed)
    pts = set()
    xs, ys = [], []
    while len(xs) < n:
        p = (int(rng.integers(0, coord)), int(rng.integers(0, coord)))
        if p not in pts:
            pts.add(p)
            xs.append(p[0])
            ys.append(p[1])
    edges = set()
    while len(edges) < m_target:
        a, b = (int(v) for v in rng.integers(0, n, 2))
        if a != b:
            edges.add((min(a, b), max(a, b)))
    edges = sorted(edges)
    if shuffle:
        order = rng.permutation(len(edges))
        edges = [edges[i] for i in order]
    g = GraphSnapshot.from_edges(xs, ys, edges, dist_type)
    if active_frac < 1.0:
        g.active = (rng.random(g.m) < active_frac).astype(np.uint8)
        g.rebuild_csr()
    return g


def knn_graph(n, k, seed, coord=10_000, dist_type=0):
    rng = np.random.default_rng(seed)
    pts = np.unique(rng.integers(0, coord, (n * 2, 2)), axis=0)
    pts = pts[rng.permutation(pts.shape[0])[:n]]
    d2 = ((pts[:, None, :] - pts[None, :, :]) ** 2).sum(-1).astype(np.int64)
    np.fill_diagonal(d2, np.iinfo(np.int64).max)
    edges = set()
    for i in range(n):
        order = np.lexsort((np.arange(n), d2[i]))[:k]
        for j in order:
            edges.add((min(i, int(j)), max(i, int(j))))
    return GraphSnapshot.from_edges(pts[:, 0], pts[:, 1], sorted(edges), dist_type)


def complete_graph(xs, ys, dist_type=0):
    n = len(xs)
    return GraphSnapshot.from_edges(xs, ys, [(i, j) for i in range(n) for j in range(i + 1, n)], dist_type)


def commit(port, g, witness):
    """Applies the reference's commit gate to a witness array; returns the next snapshot."""
    ids = np.flatnonzero(witness >= 0).astype(np.int32)
    committed, _, active = port.jv_commit(g, ids, witness[ids])
    nxt = g.copy()
    nxt.active = active
    nxt.rebuild_csr()
    return nxt, len(committed)
