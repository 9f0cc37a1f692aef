"""ctypes binding of libcee.so (include/cee.h). Loading fails loudly when the library is absent:
there is no CPU fallback for any entry point."""
from __future__ import annotations

import ctypes
import pathlib

PKG = pathlib.Path(__file__).resolve().parent
LIB_PATH = PKG / "libcee.so"
CEE_JV_STATIC_UNCHANGED = 1  # include/cee.h

c_i32p = ctypes.POINTER(ctypes.c_int32)
c_i64p = ctypes.POINTER(ctypes.c_int64)
c_u8p = ctypes.POINTER(ctypes.c_uint8)
c_u64p = ctypes.POINTER(ctypes.c_uint64)

CEE_OK = 0
CEE_BUSY = 1
CEE_ERR_INVALID = -1
CEE_ERR_RANGE = -2
CEE_ERR_CUDA = -3
CEE_ERR_NOMEM = -4
CEE_ERR_NODEVICE = -5
CEE_ERR_TIMEOUT = -6
CEE_ERR_STATE = -7

OPT_JV_KERNEL = 1
OPT_JV_WAVES = 2
OPT_KOPT_ROWS_K3 = 3
OPT_KOPT_ROWS_K4 = 4
OPT_KOPT_ROWS_K5 = 5
OPT_KOPT_KERNEL = 6


class GraphView(ctypes.Structure):
    _fields_ = [
        ("n", ctypes.c_int32), ("dist_type", ctypes.c_int32),
        ("x", c_i64p), ("y", c_i64p),
        ("m", ctypes.c_int64),
        ("edge_u", c_i32p), ("edge_v", c_i32p), ("edge_w", c_i64p), ("active", c_u8p),
        ("adjacency", ctypes.c_int64),
        ("row_offsets", c_i32p), ("neighbors", c_i32p), ("csr_edge_ids", c_i32p),
    ]


class DeviceGraph(ctypes.Structure):
    """cee_device_graph: a snapshot in device memory (all pointers are device addresses)."""
    _fields_ = [
        ("n", ctypes.c_int32), ("dist_type", ctypes.c_int32), ("m", ctypes.c_int64), ("adjacency", ctypes.c_int64),
        ("xy", ctypes.c_void_p), ("edge_uv", ctypes.c_void_p), ("edge_w", ctypes.c_void_p), ("active", ctypes.c_void_p),
        ("row_offsets", ctypes.c_void_p), ("neighbors", ctypes.c_void_p), ("csr_edge_ids", ctypes.c_void_p),
    ]


class JvStats(ctypes.Structure):
    _fields_ = [
        ("static_hit", ctypes.c_int32), ("workspace_hit", ctypes.c_int32),
        ("resident_bytes", ctypes.c_uint64),
        ("h2d_ms", ctypes.c_double), ("kernel_ms", ctypes.c_double), ("d2h_ms", ctypes.c_double),
        ("h2d_bytes", ctypes.c_int64), ("d2h_bytes", ctypes.c_int64), ("edges_screened", ctypes.c_int64),
    ]


class KoptStats(ctypes.Structure):
    _fields_ = [
        ("snapshot_hit", ctypes.c_int32), ("template_hit", ctypes.c_int32), ("workspace_hit", ctypes.c_int32),
        ("resident_bytes", ctypes.c_uint64),
        ("h2d_ms", ctypes.c_double), ("kernel_ms", ctypes.c_double), ("d2h_ms", ctypes.c_double),
        ("h2d_bytes", ctypes.c_int64), ("d2h_bytes", ctypes.c_int64),
    ]


class BatchView(ctypes.Structure):
    _fields_ = [("instances", ctypes.c_int32), ("node_begin", c_i64p), ("edge_begin", c_i64p), ("graph", GraphView)]


class BatchOptions(ctypes.Structure):
    _fields_ = [("targets", ctypes.c_int32), ("max_neighborhood", ctypes.c_int32),
                ("max_candidate_degree", ctypes.c_int32), ("cd_mode", ctypes.c_int32),
                ("max_cd_candidates", ctypes.c_int32)]


class BatchTuning(ctypes.Structure):
    _fields_ = [("jv_tile", ctypes.c_int32), ("blocks_per_sm", ctypes.c_int32), ("chunks", ctypes.c_int32)]


class KoptTuning(ctypes.Structure):
    _fields_ = [("kernel", ctypes.c_int32), ("rows_per_tile", ctypes.c_int32 * 3), ("ms", ctypes.c_float)]


class BatchStats(ctypes.Structure):
    _fields_ = [("nodes", ctypes.c_int64), ("edges", ctypes.c_int64), ("adjacency", ctypes.c_int64),
                ("targets", ctypes.c_int64), ("pairs", ctypes.c_int64), ("flag_words", ctypes.c_int64),
                ("resident_bytes", ctypes.c_uint64), ("h2d_bytes", ctypes.c_int64), ("d2h_bytes", ctypes.c_int64),
                ("h2d_ms", ctypes.c_double), ("kernel_ms", ctypes.c_double), ("d2h_ms", ctypes.c_double),
                ("total_ms", ctypes.c_double)]


class JvElimStats(ctypes.Structure):
    _fields_ = [("epochs", ctypes.c_int32), ("committed", ctypes.c_int64), ("total_ms", ctypes.c_double),
                ("resident_bytes", ctypes.c_uint64)]


class ServeConfig(ctypes.Structure):
    _fields_ = [("hbm_budget_bytes", ctypes.c_uint64), ("slots", ctypes.c_int32), ("blocks_per_sm", ctypes.c_int32),
                ("idle_ms", ctypes.c_int32)]


class ServeEvent(ctypes.Structure):
    _fields_ = [("job", ctypes.c_int32), ("status", ctypes.c_int32), ("tag", ctypes.c_uint64)]


class HtReplyStats(ctypes.Structure):
    _fields_ = [("graph_hit", ctypes.c_int32), ("workspace_hit", ctypes.c_int32), ("resident_bytes", ctypes.c_uint64)]


class ServeStats(ctypes.Structure):
    _fields_ = [("jobs", ctypes.c_uint64), ("rows_bytes", ctypes.c_uint64), ("download_bytes", ctypes.c_uint64),
                ("direct_bytes", ctypes.c_uint64)]


class NativeError(RuntimeError):
    """A non-zero status from libcee; `code` is the CEE_ERR_* value."""

    def __init__(self, code: int, message: str):
        super().__init__(f"libcee error {code}: {message}")
        self.code = code


_lib = None


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise ImportError(f"{LIB_PATH} is missing: build it with `python -m cudaedgeelimination_b200.build`")
        L = ctypes.CDLL(str(LIB_PATH))
        vp = ctypes.c_void_p
        sig = {
            "cee_abi_version": (ctypes.c_int, []),
            "cee_device_count": (ctypes.c_int, [ctypes.POINTER(ctypes.c_int)]),
            "cee_select_device": (ctypes.c_int, [ctypes.POINTER(ctypes.c_int)]),
            "cee_create": (ctypes.c_int, [ctypes.c_int, ctypes.POINTER(vp)]),
            "cee_destroy": (None, [vp]),
            "cee_last_error": (ctypes.c_char_p, [vp]),
            "cee_ctx_device": (ctypes.c_int, [vp]),
            "cee_ctx_stream": (vp, [vp]),
            "cee_ctx_sm_count": (ctypes.c_int, [vp]),
            "cee_kopt_set_tuning": (ctypes.c_int, [vp, ctypes.POINTER(KoptTuning)]),
            "cee_kopt_get_tuning": (ctypes.c_int, [vp, ctypes.POINTER(KoptTuning)]),
            "cee_kopt_autotune": (ctypes.c_int, [vp, ctypes.c_int32, ctypes.POINTER(KoptTuning)]),
            "cee_ctx_synchronize": (ctypes.c_int, [vp]),
            "cee_ctx_resident_bytes": (ctypes.c_uint64, [vp]),
            "cee_ctx_clear": (ctypes.c_int, [vp, ctypes.c_uint]),
            "cee_ctx_set_option": (ctypes.c_int, [vp, ctypes.c_int32, ctypes.c_int64]),
            "cee_jv_screen": (ctypes.c_int, [vp, ctypes.POINTER(GraphView), c_i32p, ctypes.POINTER(JvStats)]),
            "cee_jv_screen_ex": (ctypes.c_int, [vp, ctypes.POINTER(GraphView), c_i32p, ctypes.POINTER(JvStats),
                                                ctypes.c_uint32]),
            "cee_jv_prepare": (ctypes.c_int, [vp, ctypes.POINTER(GraphView), ctypes.POINTER(JvStats)]),
            "cee_jv_launch": (ctypes.c_int, [vp]),
            "cee_jv_fetch": (ctypes.c_int, [vp, c_i32p]),
            "cee_jv_screen_noalloc": (ctypes.c_int, [ctypes.POINTER(DeviceGraph), vp, vp]),
            "cee_jv_eliminate": (ctypes.c_int, [vp, ctypes.POINTER(GraphView), ctypes.c_uint32, c_u8p, c_i32p, c_i32p,
                                                c_i64p, c_i64p, ctypes.POINTER(JvElimStats)]),
            "cee_jv_eliminate_metrics": (ctypes.c_int, [vp, c_i64p, ctypes.POINTER(ctypes.c_double), ctypes.c_int32]),
            "cee_content_hash": (ctypes.c_int, [ctypes.POINTER(GraphView), c_u64p]),
            "cee_jv_proof": (ctypes.c_int, [ctypes.POINTER(GraphView), ctypes.c_uint32, c_i32p, c_i32p, vp,
                                            ctypes.c_int64, c_i64p, c_u64p]),
            "cee_write_active_edges": (ctypes.c_int, [ctypes.c_char_p, ctypes.POINTER(GraphView), c_u8p]),
            "cee_jv_write_proof": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_uint64, ctypes.c_uint64,
                                                  vp, ctypes.c_int64, vp, ctypes.c_int32]),
            "cee_kopt_templates": (ctypes.c_int, [ctypes.c_uint32, c_u8p, c_u64p]),
            "cee_kopt_costs": (ctypes.c_int, [vp, ctypes.c_int32, ctypes.c_int32, c_i64p, c_i64p, ctypes.c_uint32,
                                              c_u8p, ctypes.c_int32, ctypes.c_uint64, vp, ctypes.c_int64, c_i64p,
                                              ctypes.POINTER(KoptStats)]),
            "cee_kopt_costs_multi": (ctypes.c_int, [vp, ctypes.c_int32, ctypes.c_int32, c_i64p, c_i64p,
                                                    ctypes.c_int32, ctypes.POINTER(ctypes.c_uint32),
                                                    ctypes.POINTER(vp), c_i64p, ctypes.POINTER(vp),
                                                    ctypes.POINTER(KoptStats)]),
            "cee_kopt_improving_multi": (ctypes.c_int, [vp, ctypes.c_int32, ctypes.c_int32, c_i64p, c_i64p,
                                                        ctypes.c_int32, ctypes.POINTER(ctypes.c_uint32),
                                                        ctypes.POINTER(vp), c_i64p, ctypes.POINTER(vp), ctypes.POINTER(vp),
                                                        ctypes.POINTER(vp), ctypes.POINTER(KoptStats)]),
            "cee_kopt_prepare_multi": (ctypes.c_int, [vp, ctypes.c_int32, ctypes.c_int32, c_i64p, c_i64p,
                                                      ctypes.c_int32, ctypes.POINTER(ctypes.c_uint32),
                                                      ctypes.POINTER(vp), c_i64p, ctypes.POINTER(KoptStats)]),
            "cee_kopt_launch": (ctypes.c_int, [vp]),
            "cee_kopt_fetch": (ctypes.c_int, [vp, ctypes.POINTER(vp)]),
            "cee_cd_screen": (ctypes.c_int, [vp, ctypes.POINTER(GraphView), ctypes.c_int32, ctypes.c_int32, vp,
                                             ctypes.c_int64, ctypes.c_int32, c_u8p]),
            "cee_exact_distances": (ctypes.c_int, [vp, ctypes.c_int32, vp, vp, ctypes.c_int32, ctypes.c_int64, vp,
                                                   vp, vp, ctypes.POINTER(ctypes.c_int32)]),
            "cee_sqrt_estimate_error": (ctypes.c_int, [vp, ctypes.POINTER(ctypes.c_double)]),
            "cee_batch_prepare": (ctypes.c_int, [vp, ctypes.POINTER(BatchView), ctypes.POINTER(BatchOptions),
                                                 ctypes.POINTER(BatchStats)]),
            "cee_batch_launch": (ctypes.c_int, [vp]),
            "cee_batch_launch_plain": (ctypes.c_int, [vp]),
            "cee_batch_fetch": (ctypes.c_int, [vp, vp, vp, vp, vp, vp]),
            "cee_batch_screen": (ctypes.c_int, [vp, ctypes.POINTER(BatchView), ctypes.POINTER(BatchOptions),
                                                vp, vp, vp, vp, vp, ctypes.POINTER(BatchStats)]),
            "cee_batch_fetch_candidates": (ctypes.c_int, [vp, vp, vp, vp, vp]),
            "cee_batch_set_tuning": (ctypes.c_int, [vp, ctypes.POINTER(BatchTuning)]),
            "cee_batch_get_tuning": (ctypes.c_int, [vp, ctypes.POINTER(BatchTuning)]),
            "cee_batch_autotune": (ctypes.c_int, [vp, ctypes.c_int32, ctypes.POINTER(BatchTuning)]),
            "cee_serve_start": (ctypes.c_int, [vp, ctypes.POINTER(ServeConfig)]),
            "cee_serve_add_snapshot": (ctypes.c_int, [vp, ctypes.POINTER(GraphView), c_i32p]),
            "cee_serve_release_snapshot": (ctypes.c_int, [vp, ctypes.c_int32]),
            "cee_serve_submit_jv": (ctypes.c_int, [vp, ctypes.c_int32, vp, ctypes.c_uint64, c_i32p]),
            "cee_serve_submit_kopt": (ctypes.c_int, [vp, ctypes.c_int32, ctypes.c_int32, ctypes.POINTER(ctypes.c_uint32),
                                                     ctypes.POINTER(vp), c_i64p, ctypes.POINTER(vp), ctypes.c_uint64,
                                                     c_i32p]),
            "cee_serve_submit_kopt_improving": (ctypes.c_int, [vp, ctypes.c_int32, ctypes.c_int32,
                                                               ctypes.POINTER(ctypes.c_uint32), ctypes.POINTER(vp),
                                                               c_i64p, ctypes.POINTER(vp), ctypes.POINTER(vp),
                                                               ctypes.POINTER(vp), ctypes.c_uint64, c_i32p]),
            "cee_serve_poll": (ctypes.c_int, [vp, ctypes.POINTER(ServeEvent), ctypes.c_int32, c_i32p]),
            "cee_serve_pending": (ctypes.c_int, [vp, c_i32p, c_u64p]),
            "cee_ht_replies": (ctypes.c_int, [vp, ctypes.POINTER(GraphView), ctypes.c_int32, ctypes.c_int32, c_i32p,
                                              ctypes.c_int64, c_u64p, ctypes.POINTER(HtReplyStats)]),
            "cee_ht_end_replies": (ctypes.c_int, [vp, ctypes.POINTER(GraphView), c_i32p, ctypes.c_int64, c_u64p,
                                                  ctypes.POINTER(HtReplyStats)]),
            "cee_ht_replies_fetch": (ctypes.c_int, [vp, vp]),
            "cee_serve_get_stats": (ctypes.c_int, [vp, ctypes.POINTER(ServeStats)]),
            "cee_serve_stop": (ctypes.c_int, [vp]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(ctx, status: int) -> None:
    if status != CEE_OK:
        message = lib().cee_last_error(ctx)
        raise NativeError(status, message.decode() if message else "")
