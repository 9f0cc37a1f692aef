"""Test infrastructure: ctypes access to the CPU checkers.

  Port       -- oracle/_build/libcee_oracle.so, the plain-C restatement (cee_oracle.c)
  Reference  -- oracle/_ref/libcudaee_ref.so, the reference's own CPU sources compiled by
                oracle/Makefile (CUDA seam = the reference's stubs), or, with dropin=True,
                oracle/_ref/libcudaee_dropin.so (CUDA seam = this project's shim over libcee.so),
                or, with variant="refcuda", oracle/_ref/libcudaee_refcuda.so (CUDA seam = the
                reference's own CUDA units built for sm_100a: the comparison arm)

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use this package, and only
as the checker or as the timed CPU baseline.
"""
from __future__ import annotations

import ctypes
import pathlib
import subprocess

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
PORT_LIB = HERE / "_build" / "libcee_oracle.so"
REF_LIB = HERE / "_ref" / "libcudaee_ref.so"
DROPIN_LIB = HERE / "_ref" / "libcudaee_dropin.so"
REFCUDA_LIB = HERE / "_ref" / "libcudaee_refcuda.so"
LIBS = {"ref": REF_LIB, "dropin": DROPIN_LIB, "refcuda": REFCUDA_LIB}

i32p = ctypes.POINTER(ctypes.c_int32)
i64p = ctypes.POINTER(ctypes.c_int64)
u8p = ctypes.POINTER(ctypes.c_uint8)
u64p = ctypes.POINTER(ctypes.c_uint64)
vp = ctypes.c_void_p


def _p(a: np.ndarray, t):
    return a.ctypes.data_as(ctypes.POINTER(t))


class CeoGraph(ctypes.Structure):
    _fields_ = [("n", ctypes.c_int32), ("dist_type", ctypes.c_int32), ("x", i64p), ("y", i64p),
                ("m", ctypes.c_int64), ("edge_u", i32p), ("edge_v", i32p), ("edge_w", i64p), ("active", u8p),
                ("row_offsets", i32p), ("neighbors", i32p), ("csr_edge_ids", i32p), ("csr_weights", i64p)]


def build_port() -> None:
    """Builds the C restatement if it is missing (gcc is part of the image)."""
    if not PORT_LIB.exists():
        subprocess.run(["make", "-C", str(HERE), "port"], check=True, capture_output=True)


class Port:
    """The plain-C oracle over a snapshot-like object (n, dist_type, x, y, edge_u/v/w, active,
    row_offsets, neighbors, csr_edge_ids, csr_weights)."""

    def __init__(self):
        build_port()
        L = ctypes.CDLL(str(PORT_LIB))
        G = ctypes.POINTER(CeoGraph)
        L.ceo_isqrt.restype = ctypes.c_uint64
        L.ceo_isqrt.argtypes = [ctypes.c_uint64]
        L.ceo_distance.restype = ctypes.c_int64
        L.ceo_distance.argtypes = [ctypes.c_int64] * 4 + [ctypes.c_int32]
        L.ceo_distance_pairs.restype = None
        L.ceo_distance_pairs.argtypes = [i64p, i64p, ctypes.c_int32, ctypes.c_int64, i32p, i32p, i64p]
        L.ceo_rebuild_csr.argtypes = [ctypes.c_int32, ctypes.c_int64, i32p, i32p, i64p, u8p, i32p, i32p, i32p, i64p]
        L.ceo_jv_screen.restype = ctypes.c_int64
        L.ceo_jv_screen.argtypes = [G, i32p, i64p]
        L.ceo_jv_screen_range.restype = ctypes.c_int64
        L.ceo_jv_screen_range.argtypes = [G, ctypes.c_int64, ctypes.c_int64, i32p, i64p]
        L.ceo_jv_verify.argtypes = [G, ctypes.c_int32, ctypes.c_int32]
        L.ceo_content_hash.restype = ctypes.c_uint64
        L.ceo_content_hash.argtypes = [G]
        L.ceo_jv_commit.restype = ctypes.c_int64
        L.ceo_jv_commit.argtypes = [G, i32p, i32p, ctypes.c_int64, i32p, i32p, u8p]
        L.ceo_jv_eliminate.restype = ctypes.c_int32
        L.ceo_jv_eliminate.argtypes = [ctypes.c_int32, ctypes.c_int32, i64p, i64p, ctypes.c_int64, i32p, i32p, i64p,
                                       u8p, ctypes.c_uint32, i64p, i64p, u64p]
        L.ceo_kopt_templates.restype = ctypes.c_int32
        L.ceo_kopt_templates.argtypes = [ctypes.c_uint32, u8p, u64p]
        L.ceo_kopt_costs.argtypes = [ctypes.c_int32, i64p, i64p, ctypes.c_uint32, vp, ctypes.c_int64, u8p,
                                     ctypes.c_int32, i64p]
        L.ceo_cd_tasks.restype = ctypes.c_int64
        L.ceo_cd_tasks.argtypes = [G, ctypes.c_int32, ctypes.c_int32, ctypes.c_uint32, ctypes.c_uint32, i32p, i32p, u8p]
        L.ceo_cd_screen.argtypes = [G, ctypes.c_int32, ctypes.c_int32, i32p, i32p, u8p, ctypes.c_int64,
                                    ctypes.c_int32, u8p]
        L.ceo_ht_targets.restype = ctypes.c_int64
        L.ceo_ht_targets.argtypes = [G, ctypes.c_int32, i32p]
        L.ceo_ht_reply_count.restype = ctypes.c_int64
        L.ceo_ht_reply_count.argtypes = [G, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32]
        L.ceo_ht_replies.restype = ctypes.c_int64
        L.ceo_ht_replies.argtypes = [G, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, i32p, ctypes.c_int64]
        L.ceo_ht_end_replies.restype = ctypes.c_int64
        L.ceo_ht_end_replies.argtypes = [G, ctypes.c_int32, ctypes.c_int32, i32p, ctypes.c_int64]
        L.ceo_cd_finalize.restype = ctypes.c_int64
        L.ceo_cd_finalize.argtypes = [G, ctypes.c_int32, ctypes.c_int32, i32p, i32p, u8p, ctypes.c_int64,
                                      ctypes.c_uint32, i32p, i32p, u64p]
        L.ceo_batch_expect.argtypes = [G, i64p, i64p, ctypes.c_int64, ctypes.c_int64] + [ctypes.c_uint32] * 3 + \
            [ctypes.c_int32, ctypes.c_uint32, ctypes.c_uint32] + [vp] * 9
        self.L = L

    def graph(self, g) -> CeoGraph:
        for name in ("x", "y", "edge_u", "edge_v", "edge_w", "active", "row_offsets", "neighbors", "csr_edge_ids",
                     "csr_weights"):
            if not getattr(g, name).flags.c_contiguous:
                raise ValueError(f"oracle input {name} must be C-contiguous")
        s = CeoGraph()
        s.n, s.dist_type = g.n, g.dist_type
        s.x, s.y = _p(g.x, ctypes.c_int64), _p(g.y, ctypes.c_int64)
        s.m = g.edge_u.shape[0]
        s.edge_u, s.edge_v = _p(g.edge_u, ctypes.c_int32), _p(g.edge_v, ctypes.c_int32)
        s.edge_w, s.active = _p(g.edge_w, ctypes.c_int64), _p(g.active, ctypes.c_uint8)
        s.row_offsets, s.neighbors = _p(g.row_offsets, ctypes.c_int32), _p(g.neighbors, ctypes.c_int32)
        s.csr_edge_ids, s.csr_weights = _p(g.csr_edge_ids, ctypes.c_int32), _p(g.csr_weights, ctypes.c_int64)
        s._keep = g
        return s

    def isqrt(self, v: int) -> int:
        return int(self.L.ceo_isqrt(v))

    def distance(self, x1, y1, x2, y2, t) -> int:
        return int(self.L.ceo_distance(x1, y1, x2, y2, t))

    def distance_pairs(self, x, y, t, pair_i, pair_j) -> np.ndarray:
        x = np.ascontiguousarray(x, np.int64)
        y = np.ascontiguousarray(y, np.int64)
        pi = np.ascontiguousarray(pair_i, np.int32)
        pj = np.ascontiguousarray(pair_j, np.int32)
        out = np.empty(pi.shape[0], np.int64)
        self.L.ceo_distance_pairs(_p(x, ctypes.c_int64), _p(y, ctypes.c_int64), int(t), int(pi.shape[0]),
                                  _p(pi, ctypes.c_int32), _p(pj, ctypes.c_int32), _p(out, ctypes.c_int64))
        return out

    def csr(self, n, edge_u, edge_v, edge_w, active):
        m = edge_u.shape[0]
        slots = int(2 * np.count_nonzero(active))
        ro = np.empty(n + 1, np.int32)
        nb = np.empty(slots, np.int32)
        ids = np.empty(slots, np.int32)
        ws = np.empty(slots, np.int64)
        self.L.ceo_rebuild_csr(n, m, _p(edge_u, ctypes.c_int32), _p(edge_v, ctypes.c_int32),
                               _p(edge_w, ctypes.c_int64), _p(active, ctypes.c_uint8), _p(ro, ctypes.c_int32),
                               _p(nb, ctypes.c_int32), _p(ids, ctypes.c_int32), _p(ws, ctypes.c_int64))
        return ro, nb, ids, ws

    def jv_screen(self, g, with_evals: bool = False, first: int = 0, last: int | None = None):
        m = g.edge_u.shape[0]
        last = m if last is None else last
        witness = np.full(m, -1, np.int32)
        evals = np.zeros(m, np.int64) if with_evals else None
        self.L.ceo_jv_screen_range(self.graph(g), first, last, _p(witness, ctypes.c_int32),
                                   _p(evals, ctypes.c_int64) if with_evals else None)
        return (witness, evals) if with_evals else witness

    def jv_verify(self, g, edge_id: int, witness: int) -> bool:
        return bool(self.L.ceo_jv_verify(self.graph(g), edge_id, witness))

    def content_hash(self, g) -> int:
        return int(self.L.ceo_content_hash(self.graph(g)))

    def jv_commit(self, g, cand_edges: np.ndarray, cand_witness: np.ndarray):
        cand_edges = np.ascontiguousarray(cand_edges, np.int32)
        cand_witness = np.ascontiguousarray(cand_witness, np.int32)
        out_e = np.empty(cand_edges.shape[0], np.int32)
        out_w = np.empty(cand_edges.shape[0], np.int32)
        active = np.empty_like(g.active)
        k = self.L.ceo_jv_commit(self.graph(g), _p(cand_edges, ctypes.c_int32), _p(cand_witness, ctypes.c_int32),
                                 cand_edges.shape[0], _p(out_e, ctypes.c_int32), _p(out_w, ctypes.c_int32),
                                 _p(active, ctypes.c_uint8))
        return out_e[:k], out_w[:k], active

    def jv_eliminate(self, g, max_rounds: int = 100):
        """Returns (final active, per-epoch edges_before, per-epoch committed, final hash)."""
        active = g.active.copy()
        before = np.zeros(max_rounds, np.int64)
        committed = np.zeros(max_rounds, np.int64)
        h = ctypes.c_uint64(0)
        epochs = self.L.ceo_jv_eliminate(g.n, g.dist_type, _p(g.x, ctypes.c_int64), _p(g.y, ctypes.c_int64),
                                         g.edge_u.shape[0], _p(g.edge_u, ctypes.c_int32), _p(g.edge_v, ctypes.c_int32),
                                         _p(g.edge_w, ctypes.c_int64), _p(active, ctypes.c_uint8), max_rounds,
                                         _p(before, ctypes.c_int64), _p(committed, ctypes.c_int64), ctypes.byref(h))
        return active, before[:epochs], committed[:epochs], int(h.value)

    def kopt_templates(self, k: int):
        mates = np.full((208, 14), 0xFF, np.uint8)
        h = ctypes.c_uint64(0)
        count = self.L.ceo_kopt_templates(k, _p(mates, ctypes.c_uint8), ctypes.byref(h))
        return mates[:count].copy(), int(h.value)

    def kopt_costs(self, g, k: int, tasks: np.ndarray, mates: np.ndarray | None = None) -> np.ndarray:
        if mates is None:
            mates, _ = self.kopt_templates(k)
        mates = np.ascontiguousarray(mates, np.uint8)
        tasks = np.ascontiguousarray(tasks)
        costs = np.empty((tasks.shape[0], mates.shape[0]), np.int64)
        self.L.ceo_kopt_costs(g.dist_type, _p(g.x, ctypes.c_int64), _p(g.y, ctypes.c_int64), k,
                              tasks.ctypes.data, tasks.shape[0], _p(mates, ctypes.c_uint8), mates.shape[0],
                              _p(costs, ctypes.c_int64))
        return costs

    def cd_tasks(self, g, u: int, v: int, max_neighborhood: int = 25, max_degree: int = 50):
        cap = max(1, g.n * (g.n - 1) // 2) if max_neighborhood == 0 else max_neighborhood * (max_neighborhood - 1) // 2 + 1
        c = np.empty(cap, np.int32)
        d = np.empty(cap, np.int32)
        a = np.empty(cap, np.uint8)
        count = self.L.ceo_cd_tasks(self.graph(g), u, v, max_neighborhood, max_degree, _p(c, ctypes.c_int32),
                                    _p(d, ctypes.c_int32), _p(a, ctypes.c_uint8))
        return c[:count].copy(), d[:count].copy(), a[:count].copy()

    def cd_screen(self, g, u: int, v: int, c, d, active, mode: int) -> np.ndarray:
        c = np.ascontiguousarray(c, np.int32)
        d = np.ascontiguousarray(d, np.int32)
        active = np.ascontiguousarray(active, np.uint8)
        flags = np.empty(c.shape[0], np.uint8)
        self.L.ceo_cd_screen(self.graph(g), u, v, _p(c, ctypes.c_int32), _p(d, ctypes.c_int32),
                             _p(active, ctypes.c_uint8), c.shape[0], mode, _p(flags, ctypes.c_uint8))
        return flags

    def ht_targets(self, g, order: int = 1) -> np.ndarray:
        out = np.empty(max(1, g.edge_u.shape[0]), np.int32)
        count = self.L.ceo_ht_targets(self.graph(g), order, _p(out, ctypes.c_int32))
        return out[:count].copy()

    def cd_finalize(self, g, u: int, v: int, c, d, flags, max_cd: int = 5) -> np.ndarray:
        """FinalizeCdCandidates: the flagged (c, d) ranked by (reply product, c, d), first max_cd
        kept; rows (c, d, product)."""
        c = np.ascontiguousarray(c, np.int32)
        d = np.ascontiguousarray(d, np.int32)
        flags = np.ascontiguousarray(flags, np.uint8)
        cap = max(1, int(flags.sum()))
        oc, od = np.empty(cap, np.int32), np.empty(cap, np.int32)
        op = np.empty(cap, np.uint64)
        count = self.L.ceo_cd_finalize(self.graph(g), u, v, _p(c, ctypes.c_int32), _p(d, ctypes.c_int32),
                                       _p(flags, ctypes.c_uint8), c.shape[0], max_cd, _p(oc, ctypes.c_int32),
                                       _p(od, ctypes.c_int32), _p(op, ctypes.c_uint64))
        out = np.empty((count, 3), np.int64)
        out[:, 0], out[:, 1] = oc[:count], od[:count]
        out[:, 2] = np.minimum(op[:count], np.uint64(np.iinfo(np.int64).max)).astype(np.int64)
        return out

    def batch_expect(self, batch, opt, threads: int | None = None):
        """The batched step of every instance of `batch` (node_begin, edge_begin, graph = the
        disjoint union), as the reference's CPU code computes it, in the batched screen's output
        layout: a dict of witness [m], target_ids [I, T], target_count [I], nbhd [I, T, NB],
        flags [I, T, words] and, when opt.max_cd_candidates > 0, cand_c / cand_d / cand_product
        [I, T, K] and cand_count [I, T]. Instance ranges run on `threads` host threads."""
        import concurrent.futures
        import os
        g = batch.graph
        node_begin = np.ascontiguousarray(batch.node_begin, np.int64)
        edge_begin = np.ascontiguousarray(batch.edge_begin, np.int64)
        I, T, NB, K = int(node_begin.shape[0] - 1), opt.targets, opt.max_neighborhood, opt.max_cd_candidates
        W = opt.flag_words
        out = {"witness": np.empty(g.edge_u.shape[0], np.int32), "target_ids": np.empty((I, T), np.int32),
               "target_count": np.empty(I, np.int32), "nbhd": np.empty((I, T, NB), np.int32),
               "flags": np.empty((I, T, W), np.uint32)}
        if K > 0:
            out.update(cand_c=np.empty((I, T, K), np.int32), cand_d=np.empty((I, T, K), np.int32),
                       cand_product=np.empty((I, T, K), np.int64), cand_count=np.empty((I, T), np.int32))
        view = self.graph(g)

        def ptr(name):
            return ctypes.c_void_p(out[name].ctypes.data) if name in out else None

        def run(first, last):
            rc = self.L.ceo_batch_expect(view, _p(node_begin, ctypes.c_int64), _p(edge_begin, ctypes.c_int64), first,
                                         last, T, NB, opt.max_candidate_degree, opt.cd_mode, W, K, ptr("witness"),
                                         ptr("target_ids"), ptr("target_count"), ptr("nbhd"), ptr("flags"),
                                         ptr("cand_c"), ptr("cand_d"), ptr("cand_product"), ptr("cand_count"))
            if rc != 0:
                raise MemoryError("ceo_batch_expect ran out of memory")

        threads = threads or os.cpu_count() or 1
        step = max(1, min(64, -(-I // (4 * threads))))
        with concurrent.futures.ThreadPoolExecutor(max_workers=threads) as pool:
            list(pool.map(lambda f: run(f, min(I, f + step)), range(0, I, step)))
        return out

    def kopt_costs_parallel(self, g, k: int, tasks: np.ndarray, threads: int | None = None,
                            mates: np.ndarray | None = None) -> np.ndarray:
        """kopt_costs over row blocks on `threads` host threads (the same matrix)."""
        import concurrent.futures
        import os
        if mates is None:
            mates, _ = self.kopt_templates(k)
        mates = np.ascontiguousarray(mates, np.uint8)
        tasks = np.ascontiguousarray(tasks)
        rows = tasks.shape[0]
        costs = np.empty((rows, mates.shape[0]), np.int64)
        threads = threads or os.cpu_count() or 1
        step = max(1, -(-rows // (4 * threads)))

        def run(first):
            last = min(rows, first + step)
            self.L.ceo_kopt_costs(g.dist_type, _p(g.x, ctypes.c_int64), _p(g.y, ctypes.c_int64), k,
                                  tasks.ctypes.data + first * tasks.itemsize, last - first, _p(mates, ctypes.c_uint8),
                                  mates.shape[0], _p(costs[first:last], ctypes.c_int64))

        with concurrent.futures.ThreadPoolExecutor(max_workers=threads) as pool:
            list(pool.map(run, range(0, rows, step)))
        return costs

    def ht_reply_count(self, g, u: int, v: int, center: int) -> int:
        return int(self.L.ceo_ht_reply_count(self.graph(g), min(u, v), max(u, v), center))

    def ht_replies(self, g, u: int, v: int, centers) -> tuple[np.ndarray, np.ndarray]:
        """The Hamilton replies of each center for target (u, v), concatenated in center order:
        (offsets [len + 1] uint64, replies [total, 3] int32 rows (center, first, second))."""
        view = self.graph(g)
        lists = []
        for c in centers:
            k = int(self.L.ceo_ht_replies(view, min(u, v), max(u, v), int(c), None, 0))
            out = np.empty((max(k, 1), 3), np.int32)
            self.L.ceo_ht_replies(view, min(u, v), max(u, v), int(c), _p(out, ctypes.c_int32), k)
            lists.append(out[:k])
        return _concat(lists, 3)

    def ht_end_replies(self, g, tasks) -> tuple[np.ndarray, np.ndarray]:
        """The end replies of each (endpoint, internal neighbour) task: (offsets, replies [total, 2]
        int32 rows (lower, higher)); a task whose internal neighbour is not adjacent raises."""
        view = self.graph(g)
        lists = []
        for e, w in np.asarray(tasks, np.int64).reshape(-1, 2):
            k = int(self.L.ceo_ht_end_replies(view, int(e), int(w), None, 0))
            if k < 0:
                raise ValueError(f"internal neighbour {w} is not adjacent to {e}")
            out = np.empty((max(k, 1), 2), np.int32)
            self.L.ceo_ht_end_replies(view, int(e), int(w), _p(out, ctypes.c_int32), k)
            lists.append(out[:k])
        return _concat(lists, 2)


def _concat(lists, width: int) -> tuple[np.ndarray, np.ndarray]:
    offsets = np.zeros(len(lists) + 1, np.uint64)
    offsets[1:] = np.cumsum([len(x) for x in lists], dtype=np.uint64)
    rows = np.concatenate(lists) if lists else np.empty((0, width), np.int32)
    return offsets, rows.reshape(-1, width).astype(np.int32)


def reference_available(dropin: bool = False, variant: str | None = None) -> bool:
    return LIBS[variant or ("dropin" if dropin else "ref")].exists()


class Reference:
    """The reference library itself (compiled from its sources by oracle/Makefile)."""

    def __init__(self, dropin: bool = False, variant: str | None = None):
        path = LIBS[variant or ("dropin" if dropin else "ref")]
        if not path.exists():
            raise FileNotFoundError(f"{path} is not built (oracle/Makefile needs the reference sources)")
        L = ctypes.CDLL(str(path))
        L.ref_last_error.restype = ctypes.c_char_p
        L.ref_isqrt.restype = ctypes.c_uint64
        L.ref_isqrt.argtypes = [ctypes.c_uint64]
        L.ref_exact_distance.argtypes = [ctypes.c_int64] * 4 + [ctypes.c_int, i64p]
        L.ref_graph_new.argtypes = [ctypes.c_int32, ctypes.c_int, i64p, i64p, ctypes.c_int64, i32p, i32p, i64p, u8p,
                                    ctypes.POINTER(vp)]
        L.ref_graph_free.argtypes = [vp]
        L.ref_graph_set_active.argtypes = [vp, u8p]
        L.ref_graph_sizes.argtypes = [vp, i64p, i64p]
        L.ref_graph_csr.argtypes = [vp, i32p, i32p, i32p, i64p]
        L.ref_graph_active.argtypes = [vp, u8p]
        L.ref_graph_hash.restype = ctypes.c_uint64
        L.ref_graph_hash.argtypes = [vp]
        L.ref_jv_cpu.argtypes = [vp, i32p]
        L.ref_jv_cuda.argtypes = [vp, i32p, i32p, u64p]
        L.ref_cuda_available.argtypes = [ctypes.c_char_p, ctypes.c_int]
        L.ref_jv_verify.argtypes = [vp, ctypes.c_int32, ctypes.c_int32]
        L.ref_run_jv.argtypes = [vp, ctypes.c_int, ctypes.c_uint32, i64p, ctypes.c_int32, i32p, ctypes.c_int64, i64p,
                                 u64p, u64p]
        L.ref_write_proof_cpu.argtypes = [vp, ctypes.c_uint32, ctypes.c_char_p]
        L.ref_replay_proof_file.argtypes = [vp, ctypes.c_char_p]
        L.ref_write_active_edges.argtypes = [vp, ctypes.c_char_p]
        L.ref_kopt_table.argtypes = [ctypes.c_uint32, u8p, u64p]
        L.ref_kopt_costs.argtypes = [vp, ctypes.c_uint32, vp, ctypes.c_int64, ctypes.c_int, i64p, i64p]
        L.ref_cd_candidates.argtypes = [vp, ctypes.c_int32, ctypes.c_int32, ctypes.c_uint32, ctypes.c_uint32,
                                        ctypes.c_uint32, ctypes.c_int, ctypes.c_int, i64p, ctypes.c_int32]
        L.ref_ht_targets.argtypes = [vp, ctypes.c_int, i32p, ctypes.c_int32]
        L.ref_cd_tasks.argtypes = [vp, ctypes.c_int32, ctypes.c_int32, ctypes.c_uint32, ctypes.c_uint32, i32p, i32p,
                                   u8p, ctypes.c_int64]
        L.ref_cd_screen_cpu.argtypes = [vp, ctypes.c_int32, ctypes.c_int32, i32p, i32p, u8p, ctypes.c_int64,
                                        ctypes.c_int, u8p]
        L.ref_set_omp_threads.argtypes = [ctypes.c_int]
        L.ref_graph_new_many.argtypes = [ctypes.c_int32, ctypes.c_int] + [vp] * 9
        L.ref_batch_step.argtypes = [vp, ctypes.c_int32, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32,
                                     ctypes.c_int, ctypes.c_int32, i64p, i64p]
        L.ref_batch_parts_1core.argtypes = [vp, ctypes.c_int32, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32,
                                            ctypes.c_int, ctypes.POINTER(ctypes.c_double),
                                            ctypes.POINTER(ctypes.c_double), i64p, i64p]
        dp = ctypes.POINTER(ctypes.c_double)
        L.ref_seam_jv_timed.argtypes = [vp, ctypes.c_int32, dp, i32p]
        L.ref_seam_kopt_timed.argtypes = [vp, ctypes.c_uint32, vp, ctypes.c_int64, ctypes.c_int32, dp, i64p]
        L.ref_seam_cd_timed.argtypes = [vp, ctypes.c_int32, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32,
                                        ctypes.c_int, dp, i64p, i64p]
        L.ref_ht_hamilton_replies.argtypes = [vp, ctypes.c_int32, ctypes.c_int32, i32p, ctypes.c_int64, ctypes.c_int,
                                              ctypes.c_int, u64p, i32p, ctypes.c_int64, i64p, i32p]
        L.ref_ht_end_replies.argtypes = [vp, i32p, ctypes.c_int64, ctypes.c_int, ctypes.c_int, u64p, i32p,
                                         ctypes.c_int64, i64p, i32p]
        L.ref_seam_ht_replies_timed.argtypes = [vp, ctypes.c_int32, ctypes.c_int32, i32p, ctypes.c_int64,
                                                ctypes.c_int32, dp, i64p]
        self.L = L

    def error(self) -> str:
        return self.L.ref_last_error().decode()

    def _check(self, rc: int) -> int:
        if rc < 0:
            raise RuntimeError(self.error())
        return rc

    def graph(self, g) -> "RefGraph":
        return RefGraph(self, g)

    def isqrt(self, v: int) -> int:
        return int(self.L.ref_isqrt(v))

    def distance(self, x1, y1, x2, y2, t) -> int:
        out = ctypes.c_int64(0)
        self._check(self.L.ref_exact_distance(x1, y1, x2, y2, t, ctypes.byref(out)))
        return int(out.value)

    def kopt_table(self, k: int):
        mates = np.full((208, 14), 0xFF, np.uint8)
        h = ctypes.c_uint64(0)
        count = self._check(self.L.ref_kopt_table(k, _p(mates, ctypes.c_uint8), ctypes.byref(h)))
        return mates[:count].copy(), int(h.value)

    def set_omp_threads(self, threads: int) -> None:
        """OpenMP threads of this host thread's next parallel regions (EvaluateKOptTemplateCosts(kCpu)
        caps them at 8 itself)."""
        self.L.ref_set_omp_threads(int(threads))

    def batch_graphs(self, batch) -> "RefBatch":
        """GraphSnapshots of every instance of a disjoint union (node_begin, edge_begin, graph)."""
        return RefBatch(self, batch)


class RefBatch:
    """The reference's GraphSnapshots of every instance of a batch, built once."""

    def __init__(self, ref: Reference, batch):
        g = batch.graph
        arrays = [np.ascontiguousarray(batch.node_begin, np.int64), np.ascontiguousarray(batch.edge_begin, np.int64),
                  g.x, g.y, g.edge_u, g.edge_v, g.edge_w, g.active]
        self.ref = ref
        self.count = int(batch.node_begin.shape[0] - 1)
        self.handles = (vp * self.count)()
        ref._check(ref.L.ref_graph_new_many(self.count, g.dist_type, *(a.ctypes.data for a in arrays), self.handles))

    def step(self, instances, threads: int, targets: int = 64, nb: int = 25, max_deg: int = 50, mode: int = 0):
        """One ref_batch_step over the given instance indices: FindJvCandidatesCpu, then
        SelectHtTargetEdgeIds and BuildCdScreenTasks + ScreenCdTasksCpu for the first `targets`
        targets, per instance, on `threads` host threads. Returns (edges, c,d tasks) screened."""
        chosen = (vp * len(instances))(*[self.handles[i] for i in instances])
        edges, tasks = ctypes.c_int64(0), ctypes.c_int64(0)
        self.ref._check(self.ref.L.ref_batch_step(chosen, len(instances), targets, nb, max_deg, mode, threads,
                                                  ctypes.byref(edges), ctypes.byref(tasks)))
        return int(edges.value), int(tasks.value)

    def parts_1core(self, instances, targets: int = 64, nb: int = 25, max_deg: int = 50, mode: int = 0):
        """ref_batch_parts_1core: (JV seconds, c,d seconds, edges screened, c,d tasks screened) of the
        batched step's CPU work on one thread, the two parts timed apart."""
        chosen = (vp * len(instances))(*[self.handles[i] for i in instances])
        jv, cd = ctypes.c_double(0), ctypes.c_double(0)
        edges, tasks = ctypes.c_int64(0), ctypes.c_int64(0)
        self.ref._check(self.ref.L.ref_batch_parts_1core(chosen, len(instances), targets, nb, max_deg, mode,
                                                         ctypes.byref(jv), ctypes.byref(cd), ctypes.byref(edges),
                                                         ctypes.byref(tasks)))
        return jv.value, cd.value, int(edges.value), int(tasks.value)

    def seam_cd_timed(self, instances, targets: int = 64, nb: int = 25, max_deg: int = 50, mode: int = 0):
        """ref_seam_cd_timed over the given instances: (seconds, c,d tasks screened, flags set)."""
        chosen = (vp * len(instances))(*[self.handles[i] for i in instances])
        sec, tasks, flags = ctypes.c_double(0), ctypes.c_int64(0), ctypes.c_int64(0)
        self.ref._check(self.ref.L.ref_seam_cd_timed(chosen, len(instances), targets, nb, max_deg, mode,
                                                     ctypes.byref(sec), ctypes.byref(tasks), ctypes.byref(flags)))
        return float(sec.value), int(tasks.value), int(flags.value)

    def __del__(self):
        if getattr(self, "handles", None) is not None:
            for h in self.handles:
                if h:
                    self.ref.L.ref_graph_free(h)
            self.handles = None


class RefGraph:
    """A GraphSnapshot owned by the reference library."""

    def __init__(self, ref: Reference, g):
        for name in ("x", "y", "edge_u", "edge_v", "edge_w", "active"):
            if not getattr(g, name).flags.c_contiguous:
                raise ValueError(f"reference input {name} must be C-contiguous")
        self.ref = ref
        self.m = int(g.edge_u.shape[0])
        handle = vp()
        ref._check(ref.L.ref_graph_new(g.n, g.dist_type, _p(g.x, ctypes.c_int64), _p(g.y, ctypes.c_int64), self.m,
                                       _p(g.edge_u, ctypes.c_int32), _p(g.edge_v, ctypes.c_int32),
                                       _p(g.edge_w, ctypes.c_int64), _p(g.active, ctypes.c_uint8), ctypes.byref(handle)))
        self.handle = handle
        self.n = g.n

    def __del__(self):
        if getattr(self, "handle", None):
            self.ref.L.ref_graph_free(self.handle)
            self.handle = None

    def set_active(self, active: np.ndarray) -> None:
        active = np.ascontiguousarray(active, np.uint8)
        self.ref._check(self.ref.L.ref_graph_set_active(self.handle, _p(active, ctypes.c_uint8)))

    def csr(self):
        m, adj = ctypes.c_int64(0), ctypes.c_int64(0)
        self.ref.L.ref_graph_sizes(self.handle, ctypes.byref(m), ctypes.byref(adj))
        ro = np.empty(self.n + 1, np.int32)
        nb = np.empty(adj.value, np.int32)
        ids = np.empty(adj.value, np.int32)
        ws = np.empty(adj.value, np.int64)
        self.ref.L.ref_graph_csr(self.handle, _p(ro, ctypes.c_int32), _p(nb, ctypes.c_int32), _p(ids, ctypes.c_int32),
                                 _p(ws, ctypes.c_int64))
        return ro, nb, ids, ws

    def active(self) -> np.ndarray:
        out = np.empty(self.m, np.uint8)
        self.ref.L.ref_graph_active(self.handle, _p(out, ctypes.c_uint8))
        return out

    def content_hash(self) -> int:
        return int(self.ref.L.ref_graph_hash(self.handle))

    def write_proof_cpu(self, path, max_rounds: int = 100) -> int:
        """RunJvElimination(kCpu) in place and WriteProof of the run; returns the epoch count."""
        return self.ref._check(self.ref.L.ref_write_proof_cpu(self.handle, max_rounds, str(path).encode()))

    def write_active_edges(self, path) -> None:
        """GraphSnapshot::WriteActiveEdges of the snapshot as it stands."""
        self.ref._check(self.ref.L.ref_write_active_edges(self.handle, str(path).encode()))

    def replay_proof_file(self, path) -> int:
        """ReadProof + ReplayProof on a copy of this snapshot; the records replayed (raises when rejected)."""
        return self.ref._check(self.ref.L.ref_replay_proof_file(self.handle, str(path).encode()))

    def jv_cpu(self) -> np.ndarray:
        w = np.empty(self.m, np.int32)
        self.ref._check(self.ref.L.ref_jv_cpu(self.handle, _p(w, ctypes.c_int32)))
        return w

    def jv_cuda(self):
        w = np.empty(self.m, np.int32)
        usage = np.zeros(3, np.int32)
        resident = ctypes.c_uint64(0)
        self.ref._check(self.ref.L.ref_jv_cuda(self.handle, _p(w, ctypes.c_int32), _p(usage, ctypes.c_int32),
                                               ctypes.byref(resident)))
        return w, usage, int(resident.value)

    def jv_verify(self, edge_id: int, witness: int) -> bool:
        return bool(self.ref.L.ref_jv_verify(self.handle, edge_id, witness))

    def seam_jv_timed(self, reps: int):
        """ref_seam_jv_timed: (ms of each of `reps` FindJvCandidatesCuda calls, last witnesses)."""
        ms = np.zeros(reps, np.float64)
        w = np.empty(self.m, np.int32)
        self.ref._check(self.ref.L.ref_seam_jv_timed(self.handle, reps, _p(ms, ctypes.c_double), _p(w, ctypes.c_int32)))
        return ms, w

    def seam_kopt_timed(self, k: int, tasks: np.ndarray, reps: int):
        """ref_seam_kopt_timed: (ms of each of `reps` EvaluateKOptTemplateCostsCuda calls, last matrix)."""
        tasks = np.ascontiguousarray(tasks)
        T = {3: 4, 4: 25, 5: 208}[k]
        ms = np.zeros(reps, np.float64)
        costs = np.empty((tasks.shape[0], T), np.int64)
        self.ref._check(self.ref.L.ref_seam_kopt_timed(self.handle, k, tasks.ctypes.data, tasks.shape[0], reps,
                                                       _p(ms, ctypes.c_double), _p(costs, ctypes.c_int64)))
        return ms, costs

    def run_jv(self, backend: int, max_rounds: int = 100):
        """RunJvElimination in place; backend 1 = CPU, 2 = CUDA. Returns (epoch stats [e,3],
        proof records [r,3] = (epoch, edge_id, witness), initial hash, final hash)."""
        stats = np.zeros((max_rounds, 3), np.int64)
        cap = max(1, self.m)
        records = np.zeros((cap, 3), np.int32)
        count = ctypes.c_int64(0)
        h0, h1 = ctypes.c_uint64(0), ctypes.c_uint64(0)
        epochs = self.ref._check(self.ref.L.ref_run_jv(self.handle, backend, max_rounds, _p(stats, ctypes.c_int64),
                                                       max_rounds, _p(records, ctypes.c_int32), cap,
                                                       ctypes.byref(count), ctypes.byref(h0), ctypes.byref(h1)))
        return stats[:epochs].copy(), records[:count.value].copy(), int(h0.value), int(h1.value)

    def kopt_costs(self, k: int, tasks: np.ndarray, backend: int = 1):
        tasks = np.ascontiguousarray(tasks)
        T = {3: 4, 4: 25, 5: 208}[k]
        costs = np.empty((tasks.shape[0], T), np.int64)
        meta = np.zeros(5, np.int64)
        self.ref._check(self.ref.L.ref_kopt_costs(self.handle, k, tasks.ctypes.data, tasks.shape[0], backend,
                                                  _p(costs, ctypes.c_int64), _p(meta, ctypes.c_int64)))
        return costs, meta

    def cd_tasks(self, u: int, v: int, max_neighborhood: int = 25, max_degree: int = 50):
        cap = max(1, self.n * (self.n - 1) // 2)
        c = np.empty(cap, np.int32)
        d = np.empty(cap, np.int32)
        a = np.empty(cap, np.uint8)
        count = self.ref._check(self.ref.L.ref_cd_tasks(self.handle, u, v, max_neighborhood, max_degree,
                                                        _p(c, ctypes.c_int32), _p(d, ctypes.c_int32),
                                                        _p(a, ctypes.c_uint8), cap))
        return c[:count].copy(), d[:count].copy(), a[:count].copy()

    def cd_screen(self, u, v, c, d, active, mode: int) -> np.ndarray:
        c = np.ascontiguousarray(c, np.int32)
        d = np.ascontiguousarray(d, np.int32)
        active = np.ascontiguousarray(active, np.uint8)
        flags = np.empty(c.shape[0], np.uint8)
        self.ref._check(self.ref.L.ref_cd_screen_cpu(self.handle, u, v, _p(c, ctypes.c_int32), _p(d, ctypes.c_int32),
                                                     _p(active, ctypes.c_uint8), c.shape[0], mode,
                                                     _p(flags, ctypes.c_uint8)))
        return flags

    def cd_candidates(self, u, v, max_neighborhood=25, max_cd=5, max_degree=50, mode=0, backend=1):
        cap = 1 << 16
        out = np.empty((cap, 3), np.int64)
        count = self.ref._check(self.ref.L.ref_cd_candidates(self.handle, u, v, max_neighborhood, max_cd, max_degree,
                                                             mode, backend, _p(out, ctypes.c_int64), cap))
        return out[:count].copy()

    def ht_hamilton_replies(self, u: int, v: int, centers, backend: int = 1, dedup: bool = True):
        """EvaluateHtHamiltonReplies (backend 1 = kCpu, 2 = kCuda): (offsets, replies [total, 3],
        used: 2 = the CUDA seam's lists, checked by the reference against its CPU lists; 1 = CPU;
        0 = CPU fallback)."""
        centers = np.ascontiguousarray(centers, np.int32)
        offsets = np.zeros(centers.shape[0] + 1, np.uint64)
        total, used = ctypes.c_int64(0), ctypes.c_int32(0)
        cap = 1 << 20
        out = np.empty((cap, 3), np.int32)
        self.ref._check(self.ref.L.ref_ht_hamilton_replies(
            self.handle, u, v, _p(centers, ctypes.c_int32), centers.shape[0], backend, int(dedup),
            _p(offsets, ctypes.c_uint64), _p(out, ctypes.c_int32), cap, ctypes.byref(total), ctypes.byref(used)))
        assert total.value <= cap
        return offsets, out[:total.value].copy(), used.value

    def ht_end_replies(self, tasks, backend: int = 1, dedup: bool = True):
        """EvaluateHtEndReplies, as ht_hamilton_replies; tasks [k, 2] (endpoint, internal neighbour)."""
        tasks = np.ascontiguousarray(np.asarray(tasks, np.int32).reshape(-1, 2))
        offsets = np.zeros(tasks.shape[0] + 1, np.uint64)
        total, used = ctypes.c_int64(0), ctypes.c_int32(0)
        cap = 1 << 20
        out = np.empty((cap, 2), np.int32)
        self.ref._check(self.ref.L.ref_ht_end_replies(
            self.handle, _p(tasks, ctypes.c_int32), tasks.shape[0], backend, int(dedup), _p(offsets, ctypes.c_uint64),
            _p(out, ctypes.c_int32), cap, ctypes.byref(total), ctypes.byref(used)))
        assert total.value <= cap
        return offsets, out[:total.value].copy(), used.value

    def seam_ht_replies_timed(self, u: int, v: int, centers, reps: int):
        """ref_seam_ht_replies_timed: (ms of each detail::EvaluateHtHamiltonRepliesCuda call, reply total)."""
        centers = np.ascontiguousarray(centers, np.int32)
        ms = np.zeros(reps, np.float64)
        total = ctypes.c_int64(0)
        self.ref._check(self.ref.L.ref_seam_ht_replies_timed(self.handle, u, v, _p(centers, ctypes.c_int32),
                                                             centers.shape[0], reps, _p(ms, ctypes.c_double),
                                                             ctypes.byref(total)))
        return ms, total.value

    def ht_targets(self, order: int = 1) -> np.ndarray:
        out = np.empty(max(1, self.m), np.int32)
        count = self.ref._check(self.ref.L.ref_ht_targets(self.handle, order, _p(out, ctypes.c_int32), out.shape[0]))
        return out[:count].copy()
