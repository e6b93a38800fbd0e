"""ctypes binding of libbingo.so (include/bingo.h, include/bingo_gen.h).

The shared library is built in-tree (``make -C bingo_b200``). Importing this
module raises if it is missing: there is no fallback implementation.
"""
from __future__ import annotations

import ctypes
import os
from ctypes import POINTER, c_char_p, c_double, c_int, c_int32, c_uint8, c_uint32, c_uint64, c_void_p

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libbingo.so")


class BingoConfig(ctypes.Structure):
    _fields_ = [
        ("device", c_int32),
        ("node2vec", c_uint32),
        ("synchronous", c_uint32),
        ("weight_mode", c_uint32),
        ("arena_factor", c_double),
        ("arena_bytes", c_uint64),
    ]


class BingoWalkJob(ctypes.Structure):
    _fields_ = [
        ("app", c_int32),
        ("length", c_uint32),
        ("starts", c_void_p),
        ("n_starts", c_uint64),
        ("first", c_uint32),
        ("job_id", c_uint32),
        ("seed", c_uint64),
        ("flags", c_uint32),
        ("reserved0", c_uint32),
        ("p", c_double),
        ("q", c_double),
        ("stop_prob", c_double),
        ("out", c_void_p),
    ]


class BingoOp(ctypes.Structure):
    _fields_ = [
        ("kind", c_int32),
        ("n_jobs", c_uint32),
        ("jobs", POINTER(BingoWalkJob)),
        ("a", c_void_p),
        ("b", c_void_p),
        ("c", c_void_p),
        ("k", c_uint64),
        ("out_slots", c_void_p),
    ]


class BingoServeConfig(ctypes.Structure):
    _fields_ = [
        ("output_budget_bytes", c_uint64),
        ("max_jobs", c_uint32),
        ("max_update_batch", c_uint32),
        ("idle_timeout_us", c_uint32),
        ("reserved0", c_uint32),
    ]


class BingoServeStatus(ctypes.Structure):
    _fields_ = [
        ("done", c_int32),
        ("status", c_int32),
        ("kind", c_int32),
        ("reserved0", c_int32),
        ("version", c_uint64),
        ("latency_ns", c_uint64),
        ("ready_ns", c_uint64),
    ]


TUNING_FIELDS = ("walk_chunk", "walk_blocks_per_sm", "walk_split", "walk_order", "update_chunk",
                 "apply_blocks_per_sm")


class BingoTuning(ctypes.Structure):
    _fields_ = [(f, c_uint32) for f in TUNING_FIELDS] + [("reserved", c_uint32 * 2)]


class BingoTuneRequest(ctypes.Structure):
    _fields_ = [("jobs", c_void_p), ("n_jobs", c_uint32), ("repeats", c_uint32), ("ins_src", c_void_p),
                ("ins_dst", c_void_p), ("ins_w", c_void_p), ("n_ins", c_uint64), ("del_u", c_void_p),
                ("del_slot", c_void_p), ("n_del", c_uint64)]


class BingoTuneReport(ctypes.Structure):
    _fields_ = [("best", BingoTuning), ("walk_ms_start", ctypes.c_double), ("walk_ms_best", ctypes.c_double),
                ("update_ms_start", ctypes.c_double), ("update_ms_best", ctypes.c_double),
                ("candidates", c_uint32), ("reserved0", c_uint32)]


class BingoServeMetrics(ctypes.Structure):
    _fields_ = [(f, c_uint64) for f in ("submitted", "completed", "walk_kernel_launches", "scheduler_passes",
                                         "admit_ns", "complete_ns", "update_ns", "drain_wait_ns", "max_inflight",
                                         "queue_ns", "device_ns", "copy_ns", "drain_inflight_ns")]


class BingoStats(ctypes.Structure):
    _fields_ = [
        ("n", c_uint32),
        ("weight_mode", c_uint32),
        ("slots", c_uint64),
        ("live_edges", c_uint64),
        ("arena_bytes", c_uint64),
        ("arena_used", c_uint64),
        ("scratch_bytes", c_uint64),
        ("walk_steps", c_uint64),
        ("kernel_launches", c_uint64),
        ("walk_trials", c_uint64),
        ("walk_probes", c_uint64),
    ]


class BingoCheckReport(ctypes.Structure):
    _fields_ = [(f, c_uint64) for f in ("vertices", "live_edges", "weight_sum", "members", "alias_slots",
                                         "bad_vertices")] + [("kinds", c_uint32), ("first_bad", c_uint32)]


CHECK_KINDS = {1: "extent", 2: "count", 4: "member", 8: "alias", 16: "hash", 32: "range"}


# Every symbol include/bingo.h and include/bingo_gen.h declare, with its
# ctypes signature (restype, argtypes).
SIGNATURES = {
    "bingo_config_init": (None, [POINTER(BingoConfig)]),
    "bingo_create": (c_int, [POINTER(BingoConfig), POINTER(c_void_p)]),
    "bingo_destroy": (c_int, [c_void_p]),
    "bingo_last_error": (c_char_p, [c_void_p]),
    "bingo_load_edges": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_uint64, c_uint32]),
    "bingo_insert_batch": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_uint64, c_void_p]),
    "bingo_delete_batch": (c_int, [c_void_p, c_void_p, c_void_p, c_uint64]),
    "bingo_delete_pairs": (c_int, [c_void_p, c_void_p, c_void_p, c_uint64]),
    "bingo_load_edges_f32": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_uint64, c_uint32]),
    "bingo_insert_batch_f32": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_uint64, c_void_p]),
    "bingo_weights_to_fixed16": (c_uint64, [c_void_p, c_uint64, c_void_p]),
    "bingo_walk": (c_int, [c_void_p, POINTER(BingoWalkJob), c_uint32, c_uint32]),
    "bingo_walk_noalloc": (c_int, [c_void_p, POINTER(BingoWalkJob), c_uint32]),
    "bingo_run": (c_int, [c_void_p, POINTER(BingoOp), c_uint32, c_uint32]),
    "bingo_sync": (c_int, [c_void_p]),
    "bingo_serve_start": (c_int, [c_void_p, POINTER(BingoServeConfig)]),
    "bingo_serve_submit_walk": (c_int, [c_void_p, POINTER(BingoWalkJob), POINTER(c_uint64)]),
    "bingo_serve_submit_update": (c_int, [c_void_p, c_int32, c_void_p, c_void_p, c_void_p, c_uint64, c_void_p,
                                          POINTER(c_uint64)]),
    "bingo_serve_poll": (c_int, [c_void_p, c_uint64, POINTER(BingoServeStatus)]),
    "bingo_serve_wait": (c_int, [c_void_p, c_uint64, c_uint64, POINTER(BingoServeStatus)]),
    "bingo_serve_stop": (c_int, [c_void_p]),
    "bingo_serve_get_metrics": (c_int, [c_void_p, POINTER(BingoServeMetrics)]),
    "bingo_save": (c_int, [c_void_p, ctypes.c_char_p]),
    "bingo_restore": (c_int, [c_void_p, ctypes.c_char_p]),
    "bingo_check": (c_int, [c_void_p, POINTER(BingoCheckReport)]),
    "bingo_get_tuning": (c_int, [c_void_p, POINTER(BingoTuning)]),
    "bingo_set_tuning": (c_int, [c_void_p, POINTER(BingoTuning)]),
    "bingo_autotune": (c_int, [c_void_p, POINTER(BingoTuneRequest), POINTER(BingoTuneReport)]),
    "bingo_set_stream": (c_int, [c_void_p, c_void_p]),
    "bingo_get_stats": (c_int, [c_void_p, POINTER(BingoStats)]),
    "bingo_dump_sizes": (c_int, [c_void_p, POINTER(c_uint64)]),
    "bingo_dump_state": (c_int, [c_void_p] + [c_void_p] * 13),
    "bingo_philox": (c_int, [c_void_p, c_void_p, c_uint64, c_uint64, c_void_p]),
    "bingo_probe_gather": (c_int, [c_void_p, c_uint64, c_void_p]),
    "bingo_gen_rmat": (c_uint64, [c_uint32, c_uint32, c_double, c_double, c_double, c_uint64, c_void_p, c_void_p]),
    "bingo_gen_weights": (None, [c_uint64, c_int, c_double, c_double, c_double, c_uint64, c_void_p]),
    "bingo_updgen_create": (c_void_p, [c_uint32, c_void_p, c_void_p, c_uint64, c_uint64]),
    "bingo_updgen_destroy": (None, [c_void_p]),
    "bingo_updgen_inserts": (c_uint64, [c_void_p, c_uint64, c_int, c_double, c_double, c_double, c_void_p,
                                        c_void_p, c_void_p]),
    "bingo_updgen_deletes": (c_uint64, [c_void_p, c_uint64, c_void_p, c_void_p]),
    "bingo_updgen_live": (c_uint64, [c_void_p]),
    "bingo_edge_list_read": (c_int, [ctypes.c_char_p, c_void_p, c_void_p, c_uint64, POINTER(c_uint64),
                                     POINTER(c_uint32)]),
    "bingo_driver_weights": (c_int, [c_int, c_void_p, c_void_p, c_uint64, c_uint32, c_void_p]),
}

_lib = None


def lib() -> ctypes.CDLL:
    """Load libbingo.so once; raise if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with `make -C bingo_b200` "
                              "(the engine has no non-CUDA fallback)")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


STATUS = {
    0: "BINGO_OK",
    1: "BINGO_ERR_INVALID_ARGUMENT",
    2: "BINGO_ERR_OUT_OF_RANGE",
    3: "BINGO_ERR_ZERO_WEIGHT",
    4: "BINGO_ERR_INVALID_SLOT",
    5: "BINGO_ERR_CAPACITY",
    6: "BINGO_ERR_CUDA",
    7: "BINGO_ERR_NOT_LOADED",
    8: "BINGO_ERR_TIMEOUT",
    9: "BINGO_ERR_NO_DEVICE",
    10: "BINGO_ERR_UNSUPPORTED",
    11: "BINGO_ERR_BUSY",
    12: "BINGO_ERR_CORRUPT",
}


class BingoError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS.get(status, status)}: {message}")
        self.status = status
        self.name = STATUS.get(status, str(status))
