"""Python mirror of the reference's CUDA-backend seam, calling the B200 kernels via the C ABI.

Names, argument meaning and error behaviour follow the reference's C++ entry points:
  CudaBackendAvailable / FindJvCandidatesCuda / ClearJvCudaCache
      include/cuda_edge_elimination/elimination.hpp:333-338
  KOptCostCudaAvailable / EvaluateKOptTemplateCostsCuda / ClearKOptCostCudaCache /
  BuildKOptReconnectTable
      include/cuda_edge_elimination/local_search.hpp:49, 235-242
  HtCdCudaAvailable / ScreenHtCdCandidatesCuda
      include/cuda_edge_elimination/hamilton_tutte.hpp:527-531
Caches live in one context per (host thread, device), as the reference keeps thread-local
per-device caches (src/cuda/jv_cuda.cu:138-139). Errors raise NativeError (a RuntimeError).
"""
from __future__ import annotations

import ctypes
import json
import math
import os
import pathlib
import threading
from dataclasses import dataclass

import numpy as np

from . import _native
from .snapshot import GraphSnapshot

KOPT_TASK_DTYPE = np.dtype([("port_nodes", np.int32, (10,)), ("deleted_cost", np.int64)])
CD_TASK_DTYPE = np.dtype([("c", np.int32), ("d", np.int32), ("active", np.uint8), ("pad", np.uint8, (3,))])
# cee_jv_proof_record / cee_jv_epoch_metrics (include/cee.h)
JV_PROOF_RECORD_DTYPE = np.dtype([("epoch", np.uint32), ("edge_id", np.int32), ("u", np.int32), ("v", np.int32),
                                  ("witness", np.int32), ("reserved", np.int32), ("snapshot_hash", np.uint64)])
JV_EPOCH_METRICS_DTYPE = np.dtype([("epoch", np.uint32), ("reserved", np.uint32), ("edges_before", np.int64),
                                   ("proposed", np.int64), ("verified", np.int64), ("rejected", np.int64),
                                   ("committed", np.int64), ("propose_ms", np.float64), ("verify_ms", np.float64)])


def content_hash(graph: GraphSnapshot) -> int:
    """GraphSnapshot::ContentHash of the snapshot (host FNV-1a, cee_content_hash)."""
    view = graph.view()
    out = ctypes.c_uint64(0)
    _native.check(None, _native.lib().cee_content_hash(ctypes.byref(view), ctypes.byref(out)))
    return int(out.value)


def jv_proof(graph: GraphSnapshot, epochs: int, edge_epoch: np.ndarray, witness: np.ndarray):
    """Proof records of an elimination that started from `graph` (cee_jv_proof): returns
    (records as JV_PROOF_RECORD_DTYPE, hashes[epochs + 1]: before every epoch, then the final hash)."""
    edge_epoch = np.ascontiguousarray(edge_epoch, np.int32)
    witness = np.ascontiguousarray(witness, np.int32)
    view = graph.view()
    count = ctypes.c_int64(0)
    hashes = np.zeros(epochs + 1, np.uint64)
    cap = int((edge_epoch >= 0).sum())
    records = np.zeros(cap, JV_PROOF_RECORD_DTYPE)
    _native.check(None, _native.lib().cee_jv_proof(
        ctypes.byref(view), epochs, edge_epoch.ctypes.data_as(_native.c_i32p), witness.ctypes.data_as(_native.c_i32p),
        records.ctypes.data_as(ctypes.c_void_p), cap, ctypes.byref(count), hashes.ctypes.data_as(_native.c_u64p)))
    return records[:count.value], hashes


def write_active_edges(path, graph: GraphSnapshot, active: np.ndarray | None = None) -> None:
    """The Concorde .edg file of the snapshot's active edges (cee_write_active_edges); `active` overrides
    the snapshot's flags (e.g. the final flags of jv_eliminate)."""
    view = graph.view()
    flags = None
    if active is not None:
        active = np.ascontiguousarray(active, np.uint8)
        assert active.shape == (graph.m,)
        flags = active.ctypes.data_as(_native.c_u8p)
    _native.check(None, _native.lib().cee_write_active_edges(str(path).encode(), ctypes.byref(view), flags))


def write_jv_proof(path, backend: str, records: np.ndarray, hashes: np.ndarray, metrics: np.ndarray) -> None:
    """CUDAEE_PROOF_V1 file (cee_jv_write_proof): initial hash hashes[0], final hash hashes[-1]."""
    records = np.ascontiguousarray(records, JV_PROOF_RECORD_DTYPE)
    metrics = np.ascontiguousarray(metrics, JV_EPOCH_METRICS_DTYPE)
    _native.check(None, _native.lib().cee_jv_write_proof(
        str(path).encode(), backend.encode(), int(hashes[0]), int(hashes[-1]), records.ctypes.data_as(ctypes.c_void_p),
        int(records.shape[0]), metrics.ctypes.data_as(ctypes.c_void_p), int(metrics.shape[0])))
assert KOPT_TASK_DTYPE.itemsize == 48 and CD_TASK_DTYPE.itemsize == 12

INVALID_KOPT_COST = np.iinfo(np.int64).max
KOPT_TEMPLATE_COUNTS = {3: 4, 4: 25, 5: 208}


# ---- batched screen ----------------------------------------------------------------------

@dataclass
class BatchOptions:
    """Per-instance work of the batched screen: HT targets per instance and the c,d screen's
    HtShallowOptions (neighbourhood, degree cap, mode); the reference defaults are 64/25/50/0."""
    targets: int = 64
    max_neighborhood: int = 25
    max_candidate_degree: int = 50
    cd_mode: int = 0
    max_cd_candidates: int = 0  # 0: flags only; else FinalizeCdCandidates' ranked list (reference default 5)

    def native(self) -> _native.BatchOptions:
        return _native.BatchOptions(self.targets, self.max_neighborhood, self.max_candidate_degree, self.cd_mode,
                                    self.max_cd_candidates)

    @property
    def flag_words(self) -> int:
        return (self.max_neighborhood * (self.max_neighborhood - 1) // 2 + 31) // 32


@dataclass
class BatchResult:
    witness: np.ndarray       # [m] JV witness (global node id) or -1
    target_ids: np.ndarray    # [I, T] global edge ids, -1 padding
    target_count: np.ndarray  # [I]
    nbhd: np.ndarray          # [I, T, NB] global node ids, -1 padding
    flags: np.ndarray         # [I, T, flag_words] uint32 bit sets over the pair order i < j

    def pair_flags(self, i: int, t: int) -> np.ndarray:
        """The flags of target t of instance i as 0/1 bytes in task order."""
        size = int((self.nbhd[i, t] >= 0).sum())
        pairs = size * (size - 1) // 2
        bits = np.unpackbits(self.flags[i, t].view(np.uint8), bitorder="little")
        return bits[:pairs].astype(np.uint8)


def batch_view(batch, graph: GraphSnapshot):
    """cee_batch_view over a batch (node_begin / edge_begin arrays) and its union snapshot."""
    view = _native.BatchView()
    view.instances = int(batch.node_begin.shape[0] - 1)
    view.node_begin = batch.node_begin.ctypes.data_as(_native.c_i64p)
    view.edge_begin = batch.edge_begin.ctypes.data_as(_native.c_i64p)
    view.graph = graph.view()
    return view


def _batch_outputs(m: int, instances: int, opt: BatchOptions) -> BatchResult:
    T, NB = opt.targets, opt.max_neighborhood
    return BatchResult(np.empty(m, np.int32), np.empty((instances, T), np.int32), np.empty(instances, np.int32),
                       np.empty((instances, T, NB), np.int32), np.empty((instances, T, opt.flag_words), np.uint32))


def _ptrs(r: BatchResult):
    return [ctypes.c_void_p(a.ctypes.data) for a in (r.witness, r.target_ids, r.target_count, r.nbhd, r.flags)]


class BatchMixin:
    def batch_prepare(self, batch, opt: BatchOptions, graph: GraphSnapshot | None = None) -> _native.BatchStats:
        graph = batch.graph if graph is None else graph
        self._batch = (batch, graph, opt)
        view = batch_view(batch, graph)
        stats = _native.BatchStats()
        _native.check(self.handle, _native.lib().cee_batch_prepare(self.handle, ctypes.byref(view),
                                                                   ctypes.byref(opt.native()), ctypes.byref(stats)))
        return stats

    def batch_launch(self) -> None:
        _native.check(self.handle, _native.lib().cee_batch_launch(self.handle))

    def batch_launch_plain(self) -> None:
        _native.check(self.handle, _native.lib().cee_batch_launch_plain(self.handle))

    def batch_fetch(self) -> BatchResult:
        batch, graph, opt = self._batch
        out = _batch_outputs(graph.m, int(batch.node_begin.shape[0] - 1), opt)
        _native.check(self.handle, _native.lib().cee_batch_fetch(self.handle, *_ptrs(out)))
        return out

    def batch_screen(self, batch, opt: BatchOptions, graph: GraphSnapshot | None = None, out: BatchResult | None = None):
        graph = batch.graph if graph is None else graph
        self._batch = (batch, graph, opt)
        if out is None:
            out = _batch_outputs(graph.m, int(batch.node_begin.shape[0] - 1), opt)
        view = batch_view(batch, graph)
        stats = _native.BatchStats()
        _native.check(self.handle, _native.lib().cee_batch_screen(self.handle, ctypes.byref(view),
                                                                  ctypes.byref(opt.native()), *_ptrs(out),
                                                                  ctypes.byref(stats)))
        return out, stats

    def batch_fetch_candidates(self):
        """The finalised c,d candidates of the last launch: (c, d, product) arrays [I, T, K] and the
        count per (instance, target) [I, T]."""
        batch, graph, opt = self._batch
        I, T, K = int(batch.node_begin.shape[0] - 1), opt.targets, opt.max_cd_candidates
        c = np.empty((I, T, K), np.int32)
        d = np.empty((I, T, K), np.int32)
        product = np.empty((I, T, K), np.int64)
        count = np.empty((I, T), np.int32)
        _native.check(self.handle, _native.lib().cee_batch_fetch_candidates(
            self.handle, c.ctypes.data, d.ctypes.data, product.ctypes.data, count.ctypes.data))
        return c, d, product, count

    def batch_tuning(self) -> _native.BatchTuning:
        t = _native.BatchTuning()
        _native.check(self.handle, _native.lib().cee_batch_get_tuning(self.handle, ctypes.byref(t)))
        return t

    def set_batch_tuning(self, jv_tile: int, blocks_per_sm: int, chunks: int) -> None:
        t = _native.BatchTuning(jv_tile, blocks_per_sm, chunks)
        _native.check(self.handle, _native.lib().cee_batch_set_tuning(self.handle, ctypes.byref(t)))

    def batch_autotune(self, reps: int = 3, cache: "TuningCache | None" = None) -> _native.BatchTuning:
        """cee_batch_autotune on the prepared batch. With a cache, a shape stored for this device's SM
        count and the batch's size bucket is applied instead of timing, and a timed one is stored."""
        key = None
        if cache is not None and getattr(self, "_batch", None) is not None:
            batch, graph, _ = self._batch
            sizes = np.diff(np.asarray(batch.node_begin, np.int64))
            key = cache.key(self.sm_count, "batch", largest_instance=int(sizes.max(initial=0)),
                            instances=int(sizes.shape[0]), edges=int(graph.m))
            hit = cache.get(key)
            if hit is not None:
                self.set_batch_tuning(hit["jv_tile"], hit["blocks_per_sm"], hit["chunks"])
                return _native.BatchTuning(hit["jv_tile"], hit["blocks_per_sm"], hit["chunks"])
        t = _native.BatchTuning()
        _native.check(self.handle, _native.lib().cee_batch_autotune(self.handle, reps, ctypes.byref(t)))
        if key is not None:
            cache.put(key, {"jv_tile": t.jv_tile, "blocks_per_sm": t.blocks_per_sm, "chunks": t.chunks})
        return t



# ---- serving loop ------------------------------------------------------------------------

@dataclass
class ServeConfig:
    """cee_serve_config: the device arena (HBM budget), jobs in flight, kernel shape, idle exit."""
    hbm_budget_bytes: int = 4 << 30
    slots: int = 64
    blocks_per_sm: int = 0
    idle_ms: int = 20

    def native(self) -> _native.ServeConfig:
        return _native.ServeConfig(self.hbm_budget_bytes, self.slots, self.blocks_per_sm, self.idle_ms)


class ServeMixin:
    """Request loop: snapshots stay in device memory, jobs are admitted while an HBM budget and
    a slot are free, one persistent kernel runs all admitted jobs item by item. Submission calls
    return None when the loop is full (CEE_BUSY): poll, then retry."""

    def serve_start(self, config: ServeConfig | None = None) -> None:
        config = ServeConfig() if config is None else config
        # a running loop is released first (its in-flight downloads land before that returns): only
        # then may the buffers of its jobs go
        rc = _native.lib().cee_serve_start(self.handle, ctypes.byref(config.native()))
        self._serve_jobs = {}
        # k-opt task arrays by job: page-locked rows are read in place while the job runs
        self._serve_rows = {}
        _native.check(self.handle, rc)

    def serve_add_snapshot(self, graph: GraphSnapshot) -> int | None:
        sid = ctypes.c_int32(-1)
        view = graph.view()
        rc = _native.lib().cee_serve_add_snapshot(self.handle, ctypes.byref(view), ctypes.byref(sid))
        if rc == _native.CEE_BUSY:
            return None
        _native.check(self.handle, rc)
        return sid.value

    def serve_release_snapshot(self, sid: int) -> None:
        _native.check(self.handle, _native.lib().cee_serve_release_snapshot(self.handle, sid))

    def serve_submit_jv(self, sid: int, m: int, tag: int = 0, out: np.ndarray | None = None) -> int | None:
        """Screens every edge of snapshot `sid` (m edges); the witness array is returned by serve_poll."""
        out = np.empty(m, np.int32) if out is None else out
        assert out.dtype == np.int32 and out.flags.c_contiguous and out.shape[0] >= m
        job = ctypes.c_int32(-1)
        rc = _native.lib().cee_serve_submit_jv(self.handle, sid, ctypes.c_void_p(out.ctypes.data), tag,
                                               ctypes.byref(job))
        if rc == _native.CEE_BUSY:
            return None
        _native.check(self.handle, rc)
        self._serve_jobs[job.value] = out
        return job.value

    def serve_submit_kopt(self, sid: int, ks, task_lists, tag: int = 0, outs=None) -> int | None:
        """k-opt leaf costs of up to three segments on snapshot `sid`'s coordinates (the library's
        proper templates); the list of cost matrices is returned by serve_poll."""
        tasks = [np.ascontiguousarray(t, dtype=KOPT_TASK_DTYPE) for t in task_lists]
        n = len(ks)
        if outs is None:
            outs = [np.empty((t.shape[0], KOPT_TEMPLATE_COUNTS.get(k, 0)), np.int64) for k, t in zip(ks, tasks)]
        karr = (ctypes.c_uint32 * n)(*ks)
        tptr = (ctypes.c_void_p * n)(*[t.ctypes.data for t in tasks])
        rows = np.array([t.shape[0] for t in tasks], np.int64)
        optr = (ctypes.c_void_p * n)(*[o.ctypes.data for o in outs])
        job = ctypes.c_int32(-1)
        rc = _native.lib().cee_serve_submit_kopt(self.handle, sid, n, karr, tptr, rows.ctypes.data_as(_native.c_i64p),
                                                 optr, tag, ctypes.byref(job))
        if rc == _native.CEE_BUSY:
            return None
        _native.check(self.handle, rc)
        self._serve_jobs[job.value] = outs
        self._serve_rows[job.value] = tasks
        return job.value

    def serve_submit_kopt_improving(self, sid: int, ks, task_lists, tag: int = 0, outs=None) -> int | None:
        """The same k-opt job returning kopt_improving_multi's outputs instead of the cost matrices:
        serve_poll gives (masks, firsts), one array of each per segment. `outs` = (masks, firsts) to
        write into (caller buffers, e.g. page-locked)."""
        tasks = [np.ascontiguousarray(t, dtype=KOPT_TASK_DTYPE) for t in task_lists]
        n = len(ks)
        if outs is None:
            masks = [np.empty((t.shape[0], (KOPT_TEMPLATE_COUNTS.get(k, 0) + 31) // 32), np.uint32)
                     for k, t in zip(ks, tasks)]
            firsts = [np.empty(t.shape[0], np.int32) for t in tasks]
        else:
            masks, firsts = outs
        karr = (ctypes.c_uint32 * n)(*ks)
        tptr = (ctypes.c_void_p * n)(*[t.ctypes.data for t in tasks])
        rows = np.array([t.shape[0] for t in tasks], np.int64)
        mptr = (ctypes.c_void_p * n)(*[m.ctypes.data for m in masks])
        fptr = (ctypes.c_void_p * n)(*[f.ctypes.data for f in firsts])
        job = ctypes.c_int32(-1)
        rc = _native.lib().cee_serve_submit_kopt_improving(self.handle, sid, n, karr, tptr,
                                                           rows.ctypes.data_as(_native.c_i64p), mptr, fptr, None,
                                                           tag, ctypes.byref(job))
        if rc == _native.CEE_BUSY:
            return None
        _native.check(self.handle, rc)
        self._serve_jobs[job.value] = (masks, firsts)
        self._serve_rows[job.value] = tasks
        return job.value

    def serve_poll(self, capacity: int = 256, with_status: bool = False):
        """Completed jobs as (job, tag, outputs) tuples; a job that failed raises NativeError, unless
        with_status, which returns (job, tag, outputs, status) tuples instead."""
        events = getattr(self, "_serve_events", None)
        if events is None or len(events) < capacity:
            events = self._serve_events = (_native.ServeEvent * capacity)()
        count = ctypes.c_int32(0)
        _native.check(self.handle, _native.lib().cee_serve_poll(self.handle, events, capacity, ctypes.byref(count)))
        done = [(events[i].job, events[i].tag, self._serve_jobs.pop(events[i].job), events[i].status)
                for i in range(count.value)]
        for d in done:
            self._serve_rows.pop(d[0], None)
        if with_status:
            return done
        for _, _, _, status in done:
            _native.check(self.handle, status)
        return [d[:3] for d in done]

    def serve_pending(self) -> tuple[int, int]:
        jobs = ctypes.c_int32(0)
        used = ctypes.c_uint64(0)
        _native.check(self.handle, _native.lib().cee_serve_pending(self.handle, ctypes.byref(jobs), ctypes.byref(used)))
        return jobs.value, used.value

    def serve_stats(self) -> dict:
        """Totals since serve_start: jobs posted, k-opt row bytes uploaded, result bytes downloaded, and
        result bytes the kernel wrote in place into page-locked buffers."""
        st = _native.ServeStats()
        _native.check(self.handle, _native.lib().cee_serve_get_stats(self.handle, ctypes.byref(st)))
        return {name: int(getattr(st, name)) for name, _ in st._fields_}

    def serve_stop(self) -> None:
        # the loop's queued downloads into dropped jobs' buffers complete inside cee_serve_stop:
        # the buffers are released after it
        rc = _native.lib().cee_serve_stop(self.handle)
        self._serve_jobs = {}
        self._serve_rows = {}
        _native.check(self.handle, rc)


class TuningCache:
    """Launch shapes chosen by the autotuners, kept in a JSON file across runs and keyed by the
    device's SM count and a size bucket of the workload (each size rounded to a power of two), so
    that a later run on a similar workload applies the stored shape without timing. The file is
    $CEE_TUNING_CACHE, else ~/.cache/cudaedgeelimination_b200/tuning.json, unless a path is given."""

    VERSION = 1

    def __init__(self, path: str | os.PathLike | None = None):
        default = pathlib.Path.home() / ".cache" / "cudaedgeelimination_b200" / "tuning.json"
        self.path = pathlib.Path(path or os.environ.get("CEE_TUNING_CACHE") or default)
        self._entries = {}
        try:
            data = json.loads(self.path.read_text())
            if data.get("version") == self.VERSION:
                self._entries = dict(data.get("entries", {}))
        except (OSError, ValueError):
            pass

    @staticmethod
    def bucket(value: int) -> int:
        return 0 if value <= 0 else 1 << math.ceil(math.log2(value))

    def key(self, sm_count: int, kind: str, **sizes: int) -> str:
        return f"sm{sm_count}/{kind}/" + ",".join(f"{k}={self.bucket(v)}" for k, v in sorted(sizes.items()))

    def get(self, key: str):
        return self._entries.get(key)

    def put(self, key: str, value: dict) -> None:
        self._entries[key] = value
        self.path.parent.mkdir(parents=True, exist_ok=True)
        tmp = self.path.with_suffix(f".{os.getpid()}.tmp")
        tmp.write_text(json.dumps({"version": self.VERSION, "entries": self._entries}, indent=1, sort_keys=True))
        os.replace(tmp, self.path)


class Context(BatchMixin, ServeMixin):
    """One cee_ctx: a device, a stream and the resident caches."""

    def __init__(self, device: int = -1):
        L = _native.lib()
        handle = ctypes.c_void_p()
        _native.check(None, L.cee_create(device, ctypes.byref(handle)))
        self.handle = handle
        self.device = L.cee_ctx_device(handle)

    def close(self) -> None:
        if self.handle:
            _native.lib().cee_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def stream(self) -> int:
        return _native.lib().cee_ctx_stream(self.handle) or 0

    @property
    def sm_count(self) -> int:
        return int(_native.lib().cee_ctx_sm_count(self.handle))

    def synchronize(self) -> None:
        _native.check(self.handle, _native.lib().cee_ctx_synchronize(self.handle))

    def resident_bytes(self) -> int:
        return int(_native.lib().cee_ctx_resident_bytes(self.handle))

    def set_option(self, option: int, value: int) -> None:
        """Launch-shape option (cee_ctx_set_option); results never depend on it."""
        _native.check(self.handle, _native.lib().cee_ctx_set_option(self.handle, option, value))

    def clear(self, what: int = 0xF) -> None:
        _native.check(self.handle, _native.lib().cee_ctx_clear(self.handle, what))

    # ---- JV -------------------------------------------------------------------------
    def jv_screen(self, graph: GraphSnapshot, out: np.ndarray | None = None,
                  static_unchanged: bool = False) -> tuple[np.ndarray, _native.JvStats]:
        """cee_jv_screen; with static_unchanged, cee_jv_screen_ex's CEE_JV_STATIC_UNCHANGED hint (the
        caller vouches that coordinates, endpoints and weights equal this context's previous JV call's)."""
        witness = np.empty(graph.m, np.int32) if out is None else out
        assert witness.dtype == np.int32 and witness.flags.c_contiguous and witness.shape[0] >= graph.m
        stats = _native.JvStats()
        view = graph.view()
        flags = _native.CEE_JV_STATIC_UNCHANGED if static_unchanged else 0
        _native.check(self.handle, _native.lib().cee_jv_screen_ex(
            self.handle, ctypes.byref(view), witness.ctypes.data_as(_native.c_i32p), ctypes.byref(stats), flags))
        return witness, stats

    def ht_replies(self, graph: GraphSnapshot, u: int, v: int, centers) -> tuple[np.ndarray, np.ndarray]:
        """cee_ht_replies + cee_ht_replies_fetch: the Hamilton replies of each center for target
        (u, v) (detail::EvaluateHtHamiltonRepliesCuda): (offsets [len + 1] uint64, replies [total, 3]
        int32 rows (center, first, second)). The stats of the call are kept in `last_reply_stats`."""
        centers = np.ascontiguousarray(centers, np.int32)
        offsets = np.zeros(centers.shape[0] + 1, np.uint64)
        stats = _native.HtReplyStats()
        view = graph.view()
        lib = _native.lib()
        _native.check(self.handle, lib.cee_ht_replies(self.handle, ctypes.byref(view), min(u, v), max(u, v),
                                                       centers.ctypes.data_as(_native.c_i32p), centers.shape[0],
                                                       offsets.ctypes.data_as(_native.c_u64p), ctypes.byref(stats)))
        replies = np.empty((int(offsets[-1]), 3), np.int32)
        _native.check(self.handle, lib.cee_ht_replies_fetch(self.handle, replies.ctypes.data_as(ctypes.c_void_p)))
        self.last_reply_stats = stats
        return offsets, replies

    def ht_end_replies(self, graph: GraphSnapshot, tasks) -> tuple[np.ndarray, np.ndarray]:
        """cee_ht_end_replies + cee_ht_replies_fetch: for each (endpoint, internal neighbour) task the
        endpoint's other edges (detail::EvaluateHtEndRepliesCuda): (offsets, replies [total, 2] int32
        rows (lower, higher))."""
        tasks = np.ascontiguousarray(np.asarray(tasks, np.int32).reshape(-1, 2))
        offsets = np.zeros(tasks.shape[0] + 1, np.uint64)
        stats = _native.HtReplyStats()
        view = graph.view()
        lib = _native.lib()
        _native.check(self.handle, lib.cee_ht_end_replies(self.handle, ctypes.byref(view),
                                                           tasks.ctypes.data_as(_native.c_i32p), tasks.shape[0],
                                                           offsets.ctypes.data_as(_native.c_u64p), ctypes.byref(stats)))
        replies = np.empty((int(offsets[-1]), 2), np.int32)
        _native.check(self.handle, lib.cee_ht_replies_fetch(self.handle, replies.ctypes.data_as(ctypes.c_void_p)))
        self.last_reply_stats = stats
        return offsets, replies

    def jv_prepare(self, graph: GraphSnapshot) -> _native.JvStats:
        stats = _native.JvStats()
        view = graph.view()
        _native.check(self.handle, _native.lib().cee_jv_prepare(self.handle, ctypes.byref(view), ctypes.byref(stats)))
        return stats

    def jv_launch(self) -> None:
        _native.check(self.handle, _native.lib().cee_jv_launch(self.handle))

    def jv_fetch(self, m: int) -> np.ndarray:
        witness = np.empty(m, np.int32)
        _native.check(self.handle, _native.lib().cee_jv_fetch(self.handle, witness.ctypes.data_as(_native.c_i32p)))
        return witness

    def jv_eliminate(self, graph: GraphSnapshot, max_rounds: int = 100):
        """JV elimination to a fixed point on the device (cee_jv_eliminate). Returns (final active,
        witness per eliminated edge or -1, epoch per eliminated edge or -1, active edges before each
        epoch, edges committed per epoch, stats)."""
        m = graph.m
        active = np.empty(m, np.uint8)
        witness = np.empty(m, np.int32)
        epoch = np.empty(m, np.int32)
        before = np.zeros(max_rounds, np.int64)
        committed = np.zeros(max_rounds, np.int64)
        stats = _native.JvElimStats()
        view = graph.view()
        _native.check(self.handle, _native.lib().cee_jv_eliminate(
            self.handle, ctypes.byref(view), max_rounds, active.ctypes.data_as(_native.c_u8p),
            witness.ctypes.data_as(_native.c_i32p), epoch.ctypes.data_as(_native.c_i32p),
            before.ctypes.data_as(_native.c_i64p), committed.ctypes.data_as(_native.c_i64p), ctypes.byref(stats)))
        e = stats.epochs
        return active, witness, epoch, before[:e], committed[:e], stats

    def jv_eliminate_metrics(self, epochs: int):
        """(candidates proposed, screen + commit-gate ms) per epoch of the last jv_eliminate."""
        proposed = np.zeros(epochs, np.int64)
        ms = np.zeros(epochs, np.float64)
        _native.check(self.handle, _native.lib().cee_jv_eliminate_metrics(
            self.handle, proposed.ctypes.data_as(_native.c_i64p), ms.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
            epochs))
        return proposed, ms

    def jv_eliminate_with_proof(self, graph: GraphSnapshot, path, max_rounds: int = 100):
        """jv_eliminate, then the run's CUDAEE_PROOF_V1 file at `path` (records with the snapshot hash of
        every epoch, one metrics line per epoch; the device path has no CPU re-verification, so
        verified = proposed and rejected = 0). Returns jv_eliminate's tuple plus the proof records."""
        active, witness, epoch, before, committed, stats = self.jv_eliminate(graph, max_rounds)
        records, hashes = jv_proof(graph, stats.epochs, epoch, witness)
        proposed, ms = self.jv_eliminate_metrics(stats.epochs)
        metrics = np.zeros(stats.epochs, JV_EPOCH_METRICS_DTYPE)
        metrics["epoch"] = np.arange(stats.epochs)
        metrics["edges_before"], metrics["proposed"], metrics["verified"] = before, proposed, proposed
        metrics["committed"], metrics["propose_ms"] = committed, ms
        write_jv_proof(path, "cuda", records, hashes, metrics)
        return active, witness, epoch, before, committed, stats, records

    # ---- k-opt ----------------------------------------------------------------------
    def kopt_costs(self, graph: GraphSnapshot, table: "KOptReconnectTable", tasks: np.ndarray):
        tasks = np.ascontiguousarray(tasks, dtype=KOPT_TASK_DTYPE)
        rows = int(tasks.shape[0])
        T = len(table.templates)
        costs = np.empty((rows, T), np.int64)
        mates = np.ascontiguousarray(table.templates, dtype=np.uint8)
        stats = _native.KoptStats()
        _native.check(self.handle, _native.lib().cee_kopt_costs(
            self.handle, graph.n, graph.dist_type, graph.x.ctypes.data_as(_native.c_i64p),
            graph.y.ctypes.data_as(_native.c_i64p), table.k, mates.ctypes.data_as(_native.c_u8p), T,
            table.generator_hash, tasks.ctypes.data_as(ctypes.c_void_p), rows,
            costs.ctypes.data_as(_native.c_i64p), ctypes.byref(stats)))
        return costs, stats

    def _multi_args(self, ks, task_lists):
        n = len(ks)
        tasks = [np.ascontiguousarray(t, dtype=KOPT_TASK_DTYPE) for t in task_lists]
        karr = (ctypes.c_uint32 * n)(*ks)
        tptr = (ctypes.c_void_p * n)(*[t.ctypes.data for t in tasks])
        rows = np.array([t.shape[0] for t in tasks], np.int64)
        return tasks, karr, tptr, rows

    def kopt_costs_multi(self, graph: GraphSnapshot, ks, task_lists, outs=None):
        tasks, karr, tptr, rows = self._multi_args(ks, task_lists)
        if outs is None:
            outs = [np.empty((int(r), KOPT_TEMPLATE_COUNTS[k]), np.int64) for k, r in zip(ks, rows)]
        optr = (ctypes.c_void_p * len(ks))(*[o.ctypes.data for o in outs])
        stats = _native.KoptStats()
        _native.check(self.handle, _native.lib().cee_kopt_costs_multi(
            self.handle, graph.n, graph.dist_type, graph.x.ctypes.data_as(_native.c_i64p),
            graph.y.ctypes.data_as(_native.c_i64p), len(ks), karr, tptr, rows.ctypes.data_as(_native.c_i64p),
            optr, ctypes.byref(stats)))
        return outs, stats

    def kopt_improving_multi(self, graph: GraphSnapshot, ks, task_lists, with_costs: bool = False):
        """Fused leaf consume (cee_kopt_improving_multi): per segment the improving-template bit
        masks [rows, ceil(T/32)] uint32, the first improving template per row (-1: none) and, with
        with_costs, the full cost matrix."""
        tasks, karr, tptr, rows = self._multi_args(ks, task_lists)
        words = [(KOPT_TEMPLATE_COUNTS[k] + 31) // 32 for k in ks]
        masks = [np.empty((int(r), w), np.uint32) for r, w in zip(rows, words)]
        firsts = [np.empty(int(r), np.int32) for r in rows]
        costs = [np.empty((int(r), KOPT_TEMPLATE_COUNTS[k]), np.int64) for k, r in zip(ks, rows)] if with_costs else None
        n = len(ks)
        mptr = (ctypes.c_void_p * n)(*[a.ctypes.data for a in masks])
        fptr = (ctypes.c_void_p * n)(*[a.ctypes.data for a in firsts])
        cptr = (ctypes.c_void_p * n)(*[a.ctypes.data for a in costs]) if with_costs else None
        stats = _native.KoptStats()
        _native.check(self.handle, _native.lib().cee_kopt_improving_multi(
            self.handle, graph.n, graph.dist_type, graph.x.ctypes.data_as(_native.c_i64p),
            graph.y.ctypes.data_as(_native.c_i64p), n, karr, tptr, rows.ctypes.data_as(_native.c_i64p),
            mptr, fptr, cptr, ctypes.byref(stats)))
        return masks, firsts, costs, stats

    def kopt_prepare_multi(self, graph: GraphSnapshot, ks, task_lists) -> _native.KoptStats:
        tasks, karr, tptr, rows = self._multi_args(ks, task_lists)
        self._kopt_rows = {}
        for k, r in zip(ks, rows):
            self._kopt_rows[int(k)] = self._kopt_rows.get(int(k), 0) + int(r)
        stats = _native.KoptStats()
        _native.check(self.handle, _native.lib().cee_kopt_prepare_multi(
            self.handle, graph.n, graph.dist_type, graph.x.ctypes.data_as(_native.c_i64p),
            graph.y.ctypes.data_as(_native.c_i64p), len(ks), karr, tptr, rows.ctypes.data_as(_native.c_i64p),
            ctypes.byref(stats)))
        return stats

    def kopt_launch(self) -> None:
        _native.check(self.handle, _native.lib().cee_kopt_launch(self.handle))

    def kopt_tuning(self) -> _native.KoptTuning:
        t = _native.KoptTuning()
        _native.check(self.handle, _native.lib().cee_kopt_get_tuning(self.handle, ctypes.byref(t)))
        return t

    def set_kopt_tuning(self, kernel: int, rows_per_tile=(0, 0, 0)) -> None:
        t = _native.KoptTuning(kernel, (ctypes.c_int32 * 3)(*rows_per_tile), 0.0)
        _native.check(self.handle, _native.lib().cee_kopt_set_tuning(self.handle, ctypes.byref(t)))

    def kopt_autotune(self, reps: int = 3, cache: "TuningCache | None" = None) -> _native.KoptTuning:
        """cee_kopt_autotune on the prepared k-opt launch (see kopt_prepare_multi). With a cache, a shape
        stored for this device's SM count and the launch's rows per k is applied instead of timing,
        and a timed one is stored."""
        key = None
        if cache is not None and getattr(self, "_kopt_rows", None) is not None:
            key = cache.key(self.sm_count, "kopt", **{f"k{k}_rows": r for k, r in self._kopt_rows.items()})
            hit = cache.get(key)
            if hit is not None:
                self.set_kopt_tuning(hit["kernel"], hit["rows_per_tile"])
                return self.kopt_tuning()
        t = _native.KoptTuning()
        _native.check(self.handle, _native.lib().cee_kopt_autotune(self.handle, reps, ctypes.byref(t)))
        if key is not None:
            cache.put(key, {"kernel": t.kernel, "rows_per_tile": list(t.rows_per_tile), "ms": t.ms})
        return t

    def kopt_fetch(self, outs) -> None:
        optr = (ctypes.c_void_p * len(outs))(*[o.ctypes.data for o in outs])
        _native.check(self.handle, _native.lib().cee_kopt_fetch(self.handle, optr))

    # ---- c,d ------------------------------------------------------------------------
    def cd_screen(self, graph: GraphSnapshot, target, tasks: np.ndarray, mode: int) -> np.ndarray:
        tasks = np.ascontiguousarray(tasks, dtype=CD_TASK_DTYPE)
        flags = np.empty(tasks.shape[0], np.uint8)
        view = graph.view()
        _native.check(self.handle, _native.lib().cee_cd_screen(
            self.handle, ctypes.byref(view), int(target[0]), int(target[1]),
            tasks.ctypes.data_as(ctypes.c_void_p), int(tasks.shape[0]), int(mode),
            flags.ctypes.data_as(_native.c_u8p)))
        return flags


    def sqrt_estimate_error(self) -> float:
        """Largest relative error of the device's FP32 square-root estimate over every float in
        [1, 2^44) (the small span class is exact while it stays below 2^-21.6)."""
        out = ctypes.c_double(0.0)
        _native.check(self.handle, _native.lib().cee_sqrt_estimate_error(self.handle, ctypes.byref(out)))
        return out.value

    def exact_distances(self, x, y, dist_type: int, pair_i, pair_j):
        """Exact TSPLIB distances of point pairs, evaluated on the device by the routine the screens
        use for this point set's span class; returns (distances int32, span class)."""
        x = np.ascontiguousarray(x, dtype=np.int64)
        y = np.ascontiguousarray(y, dtype=np.int64)
        pi = np.ascontiguousarray(pair_i, dtype=np.int32)
        pj = np.ascontiguousarray(pair_j, dtype=np.int32)
        out = np.empty(pi.shape[0], np.int32)
        span = ctypes.c_int32(-1)
        _native.check(self.handle, _native.lib().cee_exact_distances(
            self.handle, int(x.shape[0]), x.ctypes.data_as(ctypes.c_void_p), y.ctypes.data_as(ctypes.c_void_p),
            int(dist_type), int(pi.shape[0]), pi.ctypes.data_as(ctypes.c_void_p), pj.ctypes.data_as(ctypes.c_void_p),
            out.ctypes.data_as(ctypes.c_void_p), ctypes.byref(span)))
        return out, int(span.value)


# ---- the reference seam, one context per (thread, device) ------------------------------

_tls = threading.local()


def _context(device: int = -1) -> Context:
    contexts = getattr(_tls, "contexts", None)
    if contexts is None:
        contexts = _tls.contexts = {}
    if device < 0:
        device = getattr(_tls, "preferred", -1)
    if device < 0 or device not in contexts:
        ctx = Context(device)
        contexts[ctx.device] = ctx
        _tls.preferred = ctx.device
        return ctx
    return contexts[device]


def device_count() -> int:
    count = ctypes.c_int(0)
    _native.lib().cee_device_count(ctypes.byref(count))
    return int(count.value)


def CudaBackendAvailable() -> tuple[bool, str]:
    if device_count() == 0:
        return False, "no visible CUDA device"
    return True, ""


KOptCostCudaAvailable = CudaBackendAvailable
HtCdCudaAvailable = CudaBackendAvailable


@dataclass
class Candidate:
    edge_id: int
    witness: int
    method: int = 1  # EliminationMethod::kJv


@dataclass
class JvCudaCacheUsage:
    static_hit: bool
    workspace_hit: bool
    resident_bytes: int
    h2d_ms: float
    kernel_ms: float
    d2h_ms: float


def FindJvCandidatesCuda(graph: GraphSnapshot) -> tuple[list[Candidate], int, JvCudaCacheUsage]:
    """Candidates in ascending edge id, the selected device and the cache usage."""
    ctx = _context()
    witness, stats = ctx.jv_screen(graph)
    ids = np.flatnonzero(witness >= 0)
    usage = JvCudaCacheUsage(bool(stats.static_hit), bool(stats.workspace_hit), int(stats.resident_bytes),
                             stats.h2d_ms, stats.kernel_ms, stats.d2h_ms)
    return [Candidate(int(e), int(witness[e])) for e in ids], ctx.device, usage


def ClearJvCudaCache() -> None:
    for ctx in getattr(_tls, "contexts", {}).values():
        ctx.clear(1)


@dataclass
class KOptReconnectTable:
    k: int
    templates: np.ndarray  # uint8 [T, 14]
    generator_hash: int


def BuildKOptReconnectTable(k: int) -> KOptReconnectTable:
    mates = np.full((208, 14), 0xFF, np.uint8)
    h = ctypes.c_uint64(0)
    count = _native.lib().cee_kopt_templates(k, mates.ctypes.data_as(_native.c_u8p), ctypes.byref(h))
    if count <= 0:
        raise ValueError("k must lie in [3,5]")
    return KOptReconnectTable(k, mates[:count].copy(), int(h.value))


def EvaluateKOptTemplateCostsCuda(graph: GraphSnapshot, table: KOptReconnectTable, tasks: np.ndarray):
    """Row-major int64 cost matrix [rows, T] (INVALID_KOPT_COST for invalid cells)."""
    costs, stats = _context().kopt_costs(graph, table, tasks)
    return costs, stats


def ClearKOptCostCudaCache() -> None:
    for ctx in getattr(_tls, "contexts", {}).values():
        ctx.clear(2)


def ScreenHtCdCandidatesCuda(graph: GraphSnapshot, target, tasks: np.ndarray, mode: int) -> np.ndarray:
    return _context().cd_screen(graph, target, tasks, mode)


def HtHamiltonReplyCudaAvailable() -> tuple[bool, str]:
    return HtCdCudaAvailable()


def EvaluateHtHamiltonRepliesCuda(graph: GraphSnapshot, target, centers) -> tuple[np.ndarray, np.ndarray]:
    """HtHamiltonReplyDeviceBatch: (offsets [len + 1] uint64, replies [total, 3] int32 rows
    (center, first, second)) for target (u, v) and each center."""
    return _context().ht_replies(graph, int(target[0]), int(target[1]), centers)


def HtEndReplyCudaAvailable() -> tuple[bool, str]:
    return HtCdCudaAvailable()


def EvaluateHtEndRepliesCuda(graph: GraphSnapshot, tasks) -> tuple[np.ndarray, np.ndarray]:
    """HtEndReplyDeviceBatch: (offsets, replies [total, 2] int32 rows (lower, higher)) for each
    (endpoint, internal neighbour) task."""
    return _context().ht_end_replies(graph, tasks)


def ClearHtReplyCudaCache() -> None:
    for ctx in getattr(_tls, "contexts", {}).values():
        ctx.clear(64)
