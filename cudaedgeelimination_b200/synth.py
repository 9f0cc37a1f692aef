"""Seeded synthetic workloads (libcee_synth.so, csrc/synth.cpp). The reference's own inputs
(TSPLIB pcb3038 / rl5915 / d15112 with ElimTSP edge sets) do not ship with it; these seeded
instances of the same shapes stand in for them.

  jv_small()        300 nodes in [0,10^4)^2, union of 10-NN, EUC_2D          (CPU-runnable JV case)
  jv_clustered()    3,000 nodes: 30 Gaussian clusters (sigma 300) + 600 uniform in [0,10^5)^2,
                    8-NN plus 2 nearest per quadrant, EUC_2D                  (multi-epoch JV)
  kopt_instance()   15,000 nodes uniform in [0,10^6)^2, 10-NN, CEIL_2D, with 200,000 leaf rows
                    of k in {3,4,5} in thirds                                 (k-opt cost matrix)
  batch_instance(i) instance i of the 4,096-instance mix (n log-uniform in [100,5000])
  ServeWorkload()   the serving stream: 10,000 jobs, 70% JV epochs on instances of the batching
                    mix with n log-uniform in [200,20000], 30% k-opt leaf batches of 1k-50k rows
                    (k = 3/4/5 in thirds) on CEIL_2D instances of the same n range
"""
from __future__ import annotations

import ctypes
import pathlib

import numpy as np

from .api import KOPT_TASK_DTYPE
from .snapshot import CEIL_2D, EUC_2D, GraphSnapshot

_LIB_PATH = pathlib.Path(__file__).resolve().parent / "libcee_synth.so"
_lib = None

SEED_BASE = 0x5EED0000


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not _LIB_PATH.exists():
            raise ImportError(f"{_LIB_PATH} is missing: build it with `python -m cudaedgeelimination_b200.build`")
        L = ctypes.CDLL(str(_LIB_PATH))
        vp = ctypes.c_void_p
        L.cees_uniform_knn.restype = vp
        L.cees_uniform_knn.argtypes = [ctypes.c_int32, ctypes.c_int64, ctypes.c_int32, ctypes.c_int32, ctypes.c_uint64]
        L.cees_clustered_knn.restype = vp
        L.cees_clustered_knn.argtypes = [ctypes.c_int32, ctypes.c_int64, ctypes.c_int32, ctypes.c_double,
                                         ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
                                         ctypes.c_uint64]
        L.cees_batch_instance.restype = vp
        L.cees_batch_instance.argtypes = [ctypes.c_uint64, ctypes.c_uint64, ctypes.c_double, ctypes.c_double]
        L.cees_free.argtypes = [vp]
        L.cees_n.restype = ctypes.c_int32
        L.cees_n.argtypes = [vp]
        L.cees_m.restype = ctypes.c_int64
        L.cees_m.argtypes = [vp]
        L.cees_dist_type.restype = ctypes.c_int32
        L.cees_dist_type.argtypes = [vp]
        L.cees_copy.argtypes = [vp, vp, vp, vp, vp, vp]
        L.cees_kopt_rows.restype = ctypes.c_int32
        L.cees_kopt_rows.argtypes = [vp, ctypes.c_int64, vp, ctypes.c_uint64, vp]
        _lib = L
    return _lib


class _Handle:
    def __init__(self, handle):
        if not handle:
            raise RuntimeError("synthetic generator failed")
        self.handle = handle

    def snapshot(self) -> GraphSnapshot:
        L = lib()
        n, m = L.cees_n(self.handle), L.cees_m(self.handle)
        x = np.empty(n, np.int64)
        y = np.empty(n, np.int64)
        eu = np.empty(m, np.int32)
        ev = np.empty(m, np.int32)
        w = np.empty(m, np.int64)
        L.cees_copy(self.handle, x.ctypes.data, y.ctypes.data, eu.ctypes.data, ev.ctypes.data, w.ctypes.data)
        return GraphSnapshot(n, L.cees_dist_type(self.handle), x, y, eu, ev, w, np.ones(m, np.uint8))

    def kopt_rows(self, ks: np.ndarray, seed: int) -> np.ndarray:
        ks = np.ascontiguousarray(ks, np.uint8)
        out = np.zeros(ks.shape[0], KOPT_TASK_DTYPE)
        rc = lib().cees_kopt_rows(self.handle, ks.shape[0], ks.ctypes.data, seed, out.ctypes.data)
        if rc != 0:
            raise RuntimeError(f"k-opt row generation failed ({rc})")
        return out

    def __del__(self):
        if getattr(self, "handle", None):
            lib().cees_free(self.handle)
            self.handle = None


def uniform_knn(n: int, coord_range: int, k: int, dist_type: int, seed: int) -> GraphSnapshot:
    return _Handle(lib().cees_uniform_knn(n, coord_range, k, dist_type, seed)).snapshot()


def jv_small(seed: int = SEED_BASE + 0) -> GraphSnapshot:
    return uniform_knn(300, 10_000, 10, EUC_2D, seed)


def jv_clustered(seed: int = SEED_BASE + 1) -> GraphSnapshot:
    return _Handle(lib().cees_clustered_knn(3000, 100_000, 30, 300.0, 600, 8, 2, EUC_2D, seed)).snapshot()


def kopt_instance(rows: int = 200_000, n: int = 15_000, seed: int = SEED_BASE + 2):
    """The instance and its rows grouped by k: returns (snapshot, {k: tasks})."""
    h = _Handle(lib().cees_uniform_knn(n, 1_000_000, 10, CEIL_2D, seed))
    third = -(-rows // 3)
    counts = {3: third, 4: third, 5: rows - 2 * third}
    ks = np.concatenate([np.full(c, k, np.uint8) for k, c in counts.items()])
    tasks = h.kopt_rows(ks, seed + 1)
    out, start = {}, 0
    for k, c in counts.items():
        out[k] = tasks[start:start + c]
        start += c
    return h.snapshot(), out


def batch_instance(index: int, seed: int = SEED_BASE + 3, n_lo: float = 100.0, n_hi: float = 5000.0) -> GraphSnapshot:
    return _Handle(lib().cees_batch_instance(seed, index, n_lo, n_hi)).snapshot()


class BatchUnion:
    """The 4,096-instance batching mix as one disjoint-union snapshot: global node and edge ids,
    per-instance offsets node_begin / edge_begin, and the union CSR."""

    def __init__(self, count: int = 4096, seed: int = SEED_BASE + 3, n_lo: float = 100.0, n_hi: float = 5000.0):
        L = lib()
        L.cees_batch_build.restype = ctypes.c_void_p
        L.cees_batch_build.argtypes = [ctypes.c_uint64, ctypes.c_int32, ctypes.c_double, ctypes.c_double]
        L.cees_batch_free.argtypes = [ctypes.c_void_p]
        L.cees_batch_sizes.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
        L.cees_batch_copy.argtypes = [ctypes.c_void_p] * 11
        handle = L.cees_batch_build(seed, count, n_lo, n_hi)
        if not handle:
            raise RuntimeError("batch generation failed")
        try:
            nodes, edges = ctypes.c_int64(0), ctypes.c_int64(0)
            L.cees_batch_sizes(handle, ctypes.byref(nodes), ctypes.byref(edges))
            n, m = nodes.value, edges.value
            if n >= 2**31 or 2 * m >= 2**31:
                raise ValueError("batch exceeds the int32 id range")
            self.count = count
            self.node_begin = np.empty(count + 1, np.int64)
            self.edge_begin = np.empty(count + 1, np.int64)
            x, y = np.empty(n, np.int64), np.empty(n, np.int64)
            eu, ev, w = np.empty(m, np.int32), np.empty(m, np.int32), np.empty(m, np.int64)
            ro, nb, ids = np.empty(n + 1, np.int32), np.empty(2 * m, np.int32), np.empty(2 * m, np.int32)
            L.cees_batch_copy(handle, *(a.ctypes.data for a in (self.node_begin, self.edge_begin, x, y, eu, ev, w,
                                                                  ro, nb, ids)))
        finally:
            L.cees_batch_free(handle)
        g = GraphSnapshot.__new__(GraphSnapshot)
        g.n, g.dist_type, g.x, g.y = int(n), EUC_2D, x, y
        g.edge_u, g.edge_v, g.edge_w, g.active = eu, ev, w, np.ones(m, np.uint8)
        g.row_offsets, g.neighbors, g.csr_edge_ids = ro, nb, ids
        g.csr_weights = np.ascontiguousarray(w[ids])
        self.graph = g

    def instance(self, i: int) -> GraphSnapshot:
        """Instance i as a standalone snapshot (local ids)."""
        n0, n1 = int(self.node_begin[i]), int(self.node_begin[i + 1])
        e0, e1 = int(self.edge_begin[i]), int(self.edge_begin[i + 1])
        g = self.graph
        return GraphSnapshot(n1 - n0, g.dist_type, g.x[n0:n1], g.y[n0:n1], g.edge_u[e0:e1] - n0,
                             g.edge_v[e0:e1] - n0, g.edge_w[e0:e1], g.active[e0:e1])


class ServeWorkload:
    """The serving stream. Snapshots come from fixed pools that stay resident on the device
    (`jv_pool` instances of the batching mix with n log-uniform in [n_lo, n_hi]; `kopt_pool`
    uniform CEIL_2D 10-NN instances of the same n range, each with a pool of leaf rows per k);
    job j is a JV epoch on a pool snapshot (probability 0.7) or a k-opt batch of
    rows ~ floor(exp(U[ln rows_lo, ln rows_hi])) split over k = 3/4/5 in thirds, taken as
    contiguous slices of a k-opt snapshot's row pools. `gaps` are unit-rate exponential
    inter-arrival times (scale by 1/lambda for a Poisson stream of rate lambda)."""

    def __init__(self, jobs: int = 10_000, jv_pool: int = 192, kopt_pool: int = 8, seed: int = SEED_BASE + 4,
                 n_lo: float = 200.0, n_hi: float = 20_000.0, rows_lo: float = 1_000.0, rows_hi: float = 50_000.0):
        rng = np.random.default_rng(seed)
        self.seed = seed
        self.jv = [batch_instance(i, seed, n_lo, n_hi) for i in range(jv_pool)]
        self.per_k = int(rows_hi) // 3 + 1
        self.kopt = []
        for i in range(kopt_pool):
            n = int(np.floor(np.exp(rng.uniform(np.log(n_lo), np.log(n_hi)))))
            h = _Handle(lib().cees_uniform_knn(n, 1_000_000, 10, CEIL_2D, seed + 1000 + i))
            rows = h.kopt_rows(np.repeat(np.array([3, 4, 5], np.uint8), self.per_k), seed + 2000 + i)
            self.kopt.append((h.snapshot(), {k: rows[j * self.per_k:(j + 1) * self.per_k] for j, k in enumerate((3, 4, 5))}))
        is_jv = rng.random(jobs) < 0.7
        self.jobs = []
        for j in range(jobs):
            if is_jv[j]:
                self.jobs.append(("jv", int(rng.integers(jv_pool)), None))
                continue
            rows = int(np.floor(np.exp(rng.uniform(np.log(rows_lo), np.log(rows_hi)))))
            third = -(-rows // 3)
            counts = (third, third, rows - 2 * third)
            offsets = tuple(int(rng.integers(0, self.per_k - c + 1)) for c in counts)
            self.jobs.append(("kopt", int(rng.integers(kopt_pool)), tuple(zip(counts, offsets))))
        self.gaps = rng.exponential(1.0, jobs)

    def kopt_tasks(self, job):
        """The three task slices (k = 3, 4, 5) of a k-opt job."""
        _, s, parts = job
        pools = self.kopt[s][1]
        return [pools[k][off:off + c] for k, (c, off) in zip((3, 4, 5), parts)]

    def output_bytes(self, job) -> int:
        if job[0] == "jv":
            return 4 * self.jv[job[1]].m
        return sum(8 * c * t for (c, _), t in zip(job[2], (4, 25, 208)))
