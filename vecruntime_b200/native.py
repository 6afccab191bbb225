"""ctypes binding of libvrgpu (include/vrgpu.h).

The structs below mirror vrgpu.h field by field; ``lib()`` loads the in-tree
library (vecruntime_b200/lib/libvrgpu.so) and raises when it is missing:
there is no CPU fallback behind this package.
"""
from __future__ import annotations

import ctypes as C
import os
import threading

# ---- status codes / lanes / kinds (vrgpu.h) -------------------------------
VR_OK = 0
VR_ERR_INVALID = 1
VR_ERR_OOM = 2
VR_ERR_OVERFLOW = 3
VR_ERR_DECIMAL_PRECISION = 4
VR_ERR_TIMEOUT = 5
VR_ERR_CUDA = 6
VR_ERR_UNSUPPORTED = 7
VR_ERR_STATE = 8
VR_ERR_ADMISSION = 9
VR_ERR_DECIMAL_OVERFLOW = 10

VR_INT32, VR_INT64, VR_FLOAT64, VR_BOOL, VR_DECIMAL128, VR_DICT32, VR_UTF8 = 1, 2, 3, 4, 5, 6, 7

VR_FN_COUNT_STAR = 1
VR_FN_COUNT = 2
VR_FN_SUM_LONG = 3
VR_FN_SUM_DOUBLE = 4
VR_FN_AVG_DOUBLE = 5
VR_FN_MIN = 6
VR_FN_MAX = 7
VR_FN_SUM_DECIMAL = 8
VR_FN_AVG_DECIMAL = 9
VR_FN_COUNT_MERGE = 10
VR_FN_AVG_DOUBLE_MERGE = 11
VR_FN_SUM_DECIMAL_MERGE = 12
VR_FN_AVG_DECIMAL_MERGE = 13

VR_FN_CHECKED = 1
VR_FN_NULL_ON_OVERFLOW = 2
VR_FN_FINAL = 4
VR_FN_STRICT = 8

VR_SPEC_FORCE_GLOBAL = 1
VR_SPEC_FORCE_SHARED = 2
VR_SPEC_FORCE_DIRECT = 4
VR_SPEC_NO_WARP_AGG = 8
VR_SPEC_WARP_AGG = 16
VR_SPEC_NO_TMA = 32
VR_SPEC_TRACE = 64
VR_SPEC_NO_JIT = 128

VR_COL_BATCH_DICTIONARY = 1

VR_HOST, VR_DEVICE = 0, 1
VR_BATCHED_PERSISTENT, VR_BATCHED_PLAIN = 0, 1


class VrError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"{msg} (status {status})")
        self.status = status


class ColumnType(C.Structure):
    _fields_ = [("lane", C.c_int32), ("precision", C.c_int32), ("scale", C.c_int32),
                ("nullable", C.c_int32), ("dict_size", C.c_int32), ("flags", C.c_int32)]


class Term(C.Structure):
    _fields_ = [("column", C.c_int32), ("sign", C.c_int32), ("addend", C.c_int64)]


class AggFn(C.Structure):
    _fields_ = [("kind", C.c_int32), ("input", C.c_int32), ("input2", C.c_int32), ("flags", C.c_int32),
                ("precision", C.c_int32), ("scale", C.c_int32), ("num_terms", C.c_int32),
                ("product_precision", C.c_int32), ("terms", Term * 3), ("result_precision", C.c_int32),
                ("result_scale", C.c_int32)]


class AggSpec(C.Structure):
    _fields_ = [("num_columns", C.c_int32), ("columns", C.POINTER(ColumnType)),
                ("num_keys", C.c_int32), ("key_columns", C.POINTER(C.c_int32)),
                ("num_fns", C.c_int32), ("fns", C.POINTER(AggFn)),
                ("est_groups", C.c_int64), ("max_batch_rows", C.c_int64),
                ("device", C.c_int32), ("flags", C.c_int32)]


VR_PQ_PLAIN, VR_PQ_RLE_DICTIONARY = 0, 1


class PqPage(C.Structure):
    _fields_ = [("data", C.c_void_p), ("length", C.c_int64), ("num_values", C.c_int32),
                ("max_def_level", C.c_int32), ("v2", C.c_int32), ("levels_length", C.c_int32),
                ("encoding", C.c_int32), ("value_bytes", C.c_int32)]


class Dictionary(C.Structure):
    _fields_ = [("size", C.c_int32), ("reserved", C.c_int32), ("offsets", C.c_void_p), ("data", C.c_void_p),
                ("validity", C.c_void_p), ("hashes", C.c_void_p)]


class Column(C.Structure):
    _fields_ = [("data", C.c_void_p), ("validity", C.c_void_p), ("offsets", C.c_void_p),
                ("dictionary", C.POINTER(Dictionary))]


class Batch(C.Structure):
    _fields_ = [("num_rows", C.c_int64), ("columns", C.POINTER(Column)), ("selection", C.c_void_p),
                ("location", C.c_int32), ("reserved", C.c_int32)]


class OutColumn(C.Structure):
    _fields_ = [("data", C.c_void_p), ("validity", C.c_void_p)]


class AggStats(C.Structure):
    _fields_ = [("tier", C.c_int32), ("warp_agg", C.c_int32), ("table_capacity", C.c_int64),
                ("slot_bytes", C.c_int64), ("groups", C.c_int64), ("rows", C.c_int64),
                ("batches", C.c_int64), ("rehashes", C.c_int64), ("deferred_rows", C.c_int64),
                ("threads", C.c_int32), ("blocks", C.c_int32), ("smem_bytes", C.c_int32),
                ("tile_rows", C.c_int32), ("last_kernel_ms", C.c_double), ("total_kernel_ms", C.c_double),
                ("total_h2d_ms", C.c_double), ("total_d2h_ms", C.c_double), ("kernel_launches", C.c_int64),
                ("jit", C.c_int32), ("reserved", C.c_int32)]


class TuneChoice(C.Structure):
    _fields_ = [("tier", C.c_int32), ("warp_agg", C.c_int32), ("threads", C.c_int32),
                ("blocks_per_sm", C.c_int32), ("tile_rows", C.c_int32), ("smem_slots", C.c_int32),
                ("table_capacity", C.c_int64)]


class PlanInfo(C.Structure):
    _fields_ = [("key_words", C.c_int32), ("acc_words", C.c_int32), ("slot_words", C.c_int32),
                ("num_ops", C.c_int32), ("num_outputs", C.c_int32), ("staged_columns", C.c_int32),
                ("sentinel_layout", C.c_int32), ("direct_ok", C.c_int32), ("direct_slots", C.c_int64),
                ("reason", C.c_char * 160)]


class BatchedPlan(C.Structure):
    _fields_ = [("num_instances", C.c_int32), ("instances", C.POINTER(C.c_void_p)),
                ("batches", C.POINTER(Batch)), ("mode", C.c_int32), ("use_graph", C.c_int32),
                ("shape", C.POINTER(TuneChoice))]


class BatchedInfo(C.Structure):
    _fields_ = [("threads", C.c_int32), ("tile_rows", C.c_int32), ("stages", C.c_int32), ("blocks", C.c_int32),
                ("smem_bytes", C.c_int32), ("smem_slots_max", C.c_int32), ("whole_tables", C.c_int32),
                ("caches", C.c_int32), ("hbm_only", C.c_int32), ("jit", C.c_int32), ("total_tiles", C.c_int64),
                ("total_rows", C.c_int64), ("table_bytes", C.c_int64)]


class SrvConfig(C.Structure):
    _fields_ = [("device", C.c_int32), ("slots", C.c_int32), ("hbm_cap_bytes", C.c_int64),
                ("staging_bytes_per_slot", C.c_int64), ("flags", C.c_int32), ("reserved", C.c_int32)]


class SrvStats(C.Structure):
    _fields_ = [("submitted", C.c_int64), ("completed", C.c_int64), ("admitted_immediately", C.c_int64),
                ("queued", C.c_int64), ("rejected", C.c_int64), ("rows", C.c_int64),
                ("p50_ms", C.c_double), ("p99_ms", C.c_double), ("max_ms", C.c_double),
                ("mean_ms", C.c_double), ("hbm_in_use", C.c_int64), ("hbm_peak", C.c_int64),
                ("p99_wait_ms", C.c_double), ("p99_service_ms", C.c_double), ("max_in_flight", C.c_int64)]


LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "lib", "libvrgpu.so")

# (name, restype, argtypes) of every entry point in vrgpu.h
_P = C.c_void_p
PROTOTYPES = [
    ("vr_agg_create", C.c_int, [C.POINTER(AggSpec), C.POINTER(_P)]),
    ("vr_agg_create_tuned", C.c_int, [C.POINTER(AggSpec), C.POINTER(TuneChoice), C.POINTER(_P)]),
    ("vr_agg_update", C.c_int, [_P, C.POINTER(Batch)]),
    ("vr_agg_sync", C.c_int, [_P]),
    ("vr_agg_num_groups", C.c_int, [_P, C.POINTER(C.c_int64)]),
    ("vr_agg_output_schema", C.c_int, [_P, C.POINTER(C.c_int32), C.POINTER(ColumnType), C.c_int32]),
    ("vr_agg_emit", C.c_int, [_P, C.c_int64, C.c_int64, C.POINTER(OutColumn), C.c_int32]),
    ("vr_agg_reset", C.c_int, [_P]),
    ("vr_agg_error_value", C.c_int, [_P, C.POINTER(C.c_int64), C.POINTER(C.c_int64), C.POINTER(C.c_int32),
                                     C.POINTER(C.c_int32)]),
    ("vr_agg_key_dictionary", C.c_int, [_P, C.c_int32, C.POINTER(C.c_int32), _P, _P, C.c_int64,
                                        C.POINTER(C.c_int64)]),
    ("vr_agg_destroy", None, [_P]),
    ("vr_agg_get_stats", C.c_int, [_P, C.POINTER(AggStats)]),
    ("vr_agg_last_error", C.c_int, [_P, C.c_char_p, C.c_size_t]),
    ("vr_status_string", C.c_char_p, [C.c_int]),
    ("vr_thread_last_error", C.c_char_p, []),
    ("vr_agg_stream", _P, [_P]),
    ("vr_host_alloc", C.c_int, [C.c_size_t, C.POINTER(_P)]),
    ("vr_host_free", C.c_int, [_P]),
    ("vr_host_register", C.c_int, [_P, C.c_size_t]),
    ("vr_host_unregister", C.c_int, [_P]),
    ("vr_hash_rows", C.c_int, [C.c_int32, C.POINTER(ColumnType), C.POINTER(Column), C.c_int64, _P, C.c_int32, _P]),
    ("vr_hash_dictionary", C.c_int, [C.POINTER(Dictionary), _P, _P]),
    ("vr_hash_rows_noalloc", C.c_int, [C.c_int32, C.POINTER(ColumnType), C.POINTER(Column), C.c_int64, _P, C.c_int32,
                                       _P]),
    ("vr_batched_create", C.c_int, [C.POINTER(BatchedPlan), C.POINTER(_P)]),
    ("vr_batched_run", C.c_int, [_P, _P]),
    ("vr_batched_get_info", C.c_int, [_P, C.POINTER(BatchedInfo)]),
    ("vr_batched_tune", C.c_int, [_P, C.c_int32, C.POINTER(C.c_double)]),
    ("vr_batched_destroy", None, [_P]),
    ("vr_tune_lookup", C.c_int, [C.POINTER(AggSpec), C.c_int64, C.POINTER(TuneChoice)]),
    ("vr_tune_record", C.c_int, [C.POINTER(AggSpec), C.c_int64, C.POINTER(TuneChoice), C.c_double]),
    ("vr_tune_load", C.c_int, [C.c_char_p]),
    ("vr_tune_save", C.c_int, [C.c_char_p]),
    ("vr_tune_search", C.c_int, [C.POINTER(AggSpec), C.POINTER(Batch), C.c_int32, C.POINTER(TuneChoice),
                                 C.POINTER(C.c_double)]),
    ("vr_jit_compile", C.c_int, [C.POINTER(AggSpec), C.c_int32, C.POINTER(C.c_int64), C.c_char_p, C.c_size_t]),
    ("vr_jit_compile_shape", C.c_int, [C.POINTER(AggSpec), C.c_int32, C.c_int32, C.c_int32, C.POINTER(C.c_int64),
                                       C.c_char_p, C.c_size_t]),
    ("vr_agg_plan", C.c_int, [C.POINTER(AggSpec), C.POINTER(PlanInfo), C.POINTER(ColumnType), C.c_int32]),
    ("vr_srv_create", C.c_int, [C.POINTER(SrvConfig), C.POINTER(_P)]),
    ("vr_srv_open_query", C.c_int, [_P, C.POINTER(AggSpec), C.POINTER(C.c_int32)]),
    ("vr_srv_submit", C.c_int, [_P, C.c_int32, C.POINTER(Batch), C.POINTER(C.c_uint64)]),
    ("vr_srv_wait", C.c_int, [_P, C.c_uint64, C.POINTER(C.c_double)]),
    ("vr_srv_query_handle", C.c_int, [_P, C.c_int32, C.POINTER(_P)]),
    ("vr_srv_close_query", C.c_int, [_P, C.c_int32]),
    ("vr_srv_get_stats", C.c_int, [_P, C.POINTER(SrvStats)]),
    ("vr_srv_drain", C.c_int, [_P]),
    ("vr_srv_destroy", None, [_P]),
    ("vr_pq_create", C.c_int, [C.c_int32, C.c_int64, C.c_int64, C.POINTER(_P)]),
    ("vr_pq_decode", C.c_int, [_P, C.c_int32, C.POINTER(PqPage), _P, _P, _P]),
    ("vr_pq_sync", C.c_int, [_P, C.POINTER(C.c_int64)]),
    ("vr_pq_destroy", None, [_P]),
    ("vr_pq_plain_dictionary", C.c_int, [_P, C.c_int64, C.c_int32, _P, _P, C.POINTER(C.c_int64)]),
]

_lib = None
_lock = threading.Lock()


def lib() -> C.CDLL:
    """The loaded libvrgpu; raises ImportError when it was never built."""
    global _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                raise ImportError(f"libvrgpu.so not built at {LIB_PATH}: run `make -C vecruntime_b200/csrc`")
            L = C.CDLL(LIB_PATH)
            for name, res, args in PROTOTYPES:
                fn = getattr(L, name)
                fn.restype = res
                fn.argtypes = args
            _lib = L
    return _lib


def status_string(status: int) -> str:
    return lib().vr_status_string(status).decode()


def check(status: int, what: str, handle=None) -> None:
    if status == VR_OK:
        return
    msg = ""
    if handle:
        buf = C.create_string_buffer(512)
        lib().vr_agg_last_error(handle, buf, 512)
        msg = buf.value.decode(errors="replace")
    if not msg:
        msg = (lib().vr_thread_last_error() or b"").decode(errors="replace")
    raise VrError(status, f"{what}: {status_string(status)}: {msg}")
