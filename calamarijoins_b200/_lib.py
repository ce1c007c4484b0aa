"""ctypes binding of libcj_b200.so (declarations in include/cj_b200.h).

The shared library is built in-tree by calamarijoins_b200/build.py. Loading
fails loudly when it is missing: there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os

_PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_PKG, "libcj_b200.so")

PAGE_SIZE = 8192

# status codes (cj_status)
CJ_OK = 0
STATUS_NAMES = {
    0: "CJ_OK", 1: "CJ_ERR_INVALID_ARGUMENT", 2: "CJ_ERR_INVALID_PLAN", 3: "CJ_ERR_MALFORMED_PAGE",
    4: "CJ_ERR_OUT_OF_MEMORY", 5: "CJ_ERR_CUDA", 6: "CJ_ERR_UNSUPPORTED", 7: "CJ_ERR_LIMIT",
    8: "CJ_ERR_NO_DEVICE", 9: "CJ_ERR_REJECTED", 10: "CJ_ERR_TIMEOUT", 11: "CJ_ERR_CANCELLED",
    12: "CJ_ERR_INTERNAL",
}

CJ_NODE_HASH_JOIN = 0
CJ_NODE_SCAN = 1
CJ_EXEC_RESULT_ON_DEVICE = 1

CJ_OPT_NESTED_LOOP_MAX_BUILD = 0
CJ_OPT_SLOTS_PER_PARTITION = 1
CJ_OPT_PROFILE_KERNELS = 2
CJ_OPT_BLOCK_THREADS = 3
CJ_OPT_VARCHAR_TILE_ROWS = 4
CJ_OPT_CTAS_PER_SM = 5
CJ_OPT_DENSE_KEYS = 6
CJ_OPT_BUFFER_CACHE_BYTES = 7
CJ_OPT_FAIL_ALLOC_AT = 8
CJ_TUNE_QUICK = 1


class ColumnDesc(C.Structure):
    _fields_ = [("type", C.c_int32), ("reserved", C.c_uint32), ("num_pages", C.c_uint64),
                ("pages", C.POINTER(C.c_void_p))]


class TableDesc(C.Structure):
    _fields_ = [("num_rows", C.c_uint64), ("num_columns", C.c_uint64),
                ("columns", C.POINTER(ColumnDesc))]


class Attr(C.Structure):
    _fields_ = [("index", C.c_uint64), ("type", C.c_int32), ("reserved", C.c_uint32)]


class PlanNodeDesc(C.Structure):
    _fields_ = [("node_type", C.c_int32), ("build_left", C.c_int32), ("base_table_id", C.c_uint64),
                ("left", C.c_uint64), ("right", C.c_uint64), ("left_attr", C.c_uint64),
                ("right_attr", C.c_uint64), ("num_output_attrs", C.c_uint64),
                ("output_attrs", C.POINTER(Attr))]


class PlanDesc(C.Structure):
    _fields_ = [("num_nodes", C.c_uint64), ("nodes", C.POINTER(PlanNodeDesc)),
                ("num_inputs", C.c_uint64), ("inputs", C.POINTER(TableDesc)),
                ("resident_inputs", C.POINTER(C.c_void_p)), ("root", C.c_uint64)]


class PredNodeC(C.Structure):
    _fields_ = [("kind", C.c_int32), ("op", C.c_int32), ("column", C.c_uint64), ("left", C.c_uint64),
                ("right", C.c_uint64), ("literal_type", C.c_int32), ("reserved", C.c_uint32), ("i64", C.c_int64),
                ("f64", C.c_double), ("str", C.c_char_p), ("str_len", C.c_uint64)]


class PredicateC(C.Structure):
    _fields_ = [("num_nodes", C.c_uint64), ("nodes", C.POINTER(PredNodeC)), ("root", C.c_uint64)]


class TimingStatsC(C.Structure):
    _fields_ = [(n, C.c_int64) for n in (
        "hashtable_build_ms", "hash_join_probe_ms", "nested_loop_join_ms", "materialize_ms",
        "setup_ms", "total_execution_ms", "intermediate_ms")]


class ExecStatsC(C.Structure):
    _fields_ = ([(n, C.c_double) for n in (
        "upload_us", "decode_us", "build_us", "probe_us", "nested_loop_us", "intermediate_us",
        "materialize_us", "download_us", "total_us")]
        + [(n, C.c_uint64) for n in (
            "h2d_bytes", "d2h_bytes", "num_joins", "num_hash_joins", "num_nested_loop_joins",
            "probe_rows", "matches", "probe_reruns", "output_rows", "output_pages",
            "kernel_launches", "num_direct_joins", "num_open_joins", "host_syncs")])


class CacheMetaC(C.Structure):
    _fields_ = [("num_rows", C.c_uint64), ("num_columns", C.c_uint64), ("types", C.c_int32 * 16),
                ("num_pages", C.c_uint64 * 16)]


class BatchStatsC(C.Structure):
    _fields_ = ([(n, C.c_uint64) for n in (
        "num_plans", "num_levels", "num_joins", "num_hash_joins", "num_nested_loop_joins", "probe_rows",
        "matches", "probe_reruns", "kernel_launches", "syncs", "h2d_bytes", "d2h_bytes")]
        + [("total_us", C.c_double)])


class ServerConfigC(C.Structure):
    _fields_ = [("device", C.c_int32), ("slots", C.c_uint32), ("memory_budget", C.c_uint64),
                ("exec_flags", C.c_uint32), ("max_batch", C.c_uint32), ("age_limit_us", C.c_uint64),
                ("host_cache_bytes", C.c_uint64), ("device_reserve_bytes", C.c_uint64)]


class ServerStatsC(C.Structure):
    _fields_ = ([(n, C.c_uint64) for n in (
        "submitted", "completed", "failed", "rejected", "cancelled", "queued", "running", "admitted_bytes",
        "peak_admitted_bytes", "memory_budget")]
        + [(n, C.c_double) for n in ("p50_us", "p99_us", "mean_us", "max_us", "wall_s", "plans_per_s")]
        + [("batches", C.c_uint64), ("skipped_ahead", C.c_uint64), ("mean_batch", C.c_double),
           ("batch_fallbacks", C.c_uint64), ("pinned_allocs", C.c_uint64), ("pinned_alloc_bytes", C.c_uint64),
           ("pool_high_bytes", C.c_uint64)])


# every function of include/cj_b200.h: name -> (restype, argtypes)
_P = C.c_void_p
_SIGS = {
    "cj_context_create": (C.c_int, [C.c_int, C.POINTER(_P)]),
    "cj_context_destroy": (None, [_P]),
    "cj_context_set_option": (C.c_int, [_P, C.c_int32, C.c_int64]),
    "cj_context_get_option": (C.c_int, [_P, C.c_int32, C.POINTER(C.c_int64)]),
    "cj_profile_reset": (C.c_int, [_P]),
    "cj_profile_count": (C.c_int, [_P, C.POINTER(C.c_uint64)]),
    "cj_profile_entry": (C.c_int, [_P, C.c_uint64, C.POINTER(C.c_char_p), C.POINTER(C.c_uint64),
                                   C.POINTER(C.c_double)]),
    "cj_context_stream": (C.c_int, [_P, C.POINTER(_P)]),
    "cj_context_memory": (C.c_int, [_P, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]),
    "cj_table_upload": (C.c_int, [_P, C.POINTER(TableDesc), C.POINTER(_P)]),
    "cj_table_from_device": (C.c_int, [_P, C.c_uint64, C.c_uint64, C.POINTER(C.c_int32),
                                       C.POINTER(C.c_uint64), C.POINTER(_P), C.POINTER(_P)]),
    "cj_table_column_pages": (C.c_int, [_P, C.c_uint64, C.POINTER(_P), C.POINTER(C.c_uint64)]),
    "cj_table_free": (None, [_P]),
    "cj_table_copy_column": (C.c_int, [_P, C.c_uint64, _P, C.c_uint64]),
    "cj_table_filter": (C.c_int, [_P, _P, C.POINTER(PredicateC), C.c_uint64, C.POINTER(C.c_uint64), C.POINTER(_P),
                                  C.POINTER(C.c_uint64)]),
    "cj_cache_read_meta": (C.c_int, [C.c_char_p, C.POINTER(CacheMetaC)]),
    "cj_table_write_cache": (C.c_int, [C.POINTER(TableDesc), C.c_char_p]),
    "cj_table_load_cache": (C.c_int, [_P, C.c_char_p, C.POINTER(_P)]),
    "cj_catalog_create": (C.c_int, [_P, C.POINTER(_P)]),
    "cj_catalog_destroy": (None, [_P]),
    "cj_catalog_add": (C.c_int, [_P, C.c_char_p, _P]),
    "cj_catalog_load": (C.c_int, [_P, C.c_char_p, C.c_char_p]),
    "cj_catalog_get": (C.c_int, [_P, C.c_char_p, C.POINTER(_P)]),
    "cj_catalog_size": (C.c_int, [_P, C.POINTER(C.c_uint64)]),
    "cj_catalog_name": (C.c_int, [_P, C.c_uint64, C.POINTER(C.c_char_p)]),
    "cj_execute": (C.c_int, [_P, C.POINTER(PlanDesc), C.c_uint32, C.POINTER(_P),
                             C.POINTER(TimingStatsC), C.POINTER(ExecStatsC)]),
    "cj_execute_batch": (C.c_int, [_P, C.POINTER(PlanDesc), C.c_uint64, C.c_uint32, C.POINTER(_P),
                                   C.POINTER(C.c_int32), C.POINTER(BatchStatsC)]),
    "cj_hash_join_noalloc": (C.c_int, [_P, _P, C.c_uint32, _P, _P, C.c_uint32, _P, _P, C.c_uint64, _P,
                                       C.POINTER(C.c_uint64), _P]),
    "cj_result_num_rows": (C.c_int, [_P, C.POINTER(C.c_uint64)]),
    "cj_result_num_columns": (C.c_int, [_P, C.POINTER(C.c_uint64)]),
    "cj_result_column": (C.c_int, [_P, C.c_uint64, C.POINTER(C.c_int32), C.POINTER(C.c_uint64),
                                   C.POINTER(_P)]),
    "cj_result_column_device": (C.c_int, [_P, C.c_uint64, C.POINTER(_P)]),
    "cj_result_copy_column": (C.c_int, [_P, C.c_uint64, _P, C.c_uint64]),
    "cj_result_free": (None, [_P]),
    "cj_autotune": (C.c_int, [_P, C.c_char_p, C.c_uint32]),
    "cj_tuning_load": (C.c_int, [_P, C.c_char_p]),
    "cj_tuning_check_file": (C.c_int, [C.c_char_p]),
    "cj_tuning_entry": (C.c_int, [_P, C.c_uint32, C.POINTER(C.c_int32), C.POINTER(C.c_int32),
                                  C.POINTER(C.c_int32)]),
    "cj_batch_prepare": (C.c_int, [_P, _P, C.c_uint64, C.c_uint32, C.POINTER(_P)]),
    "cj_batch_run": (C.c_int, [_P, C.POINTER(_P), C.POINTER(BatchStatsC)]),
    "cj_prepared_free": (None, [_P]),
    "cj_server_create": (C.c_int, [C.POINTER(ServerConfigC), C.POINTER(_P)]),
    "cj_server_submit": (C.c_int, [_P, C.POINTER(PlanDesc), C.POINTER(C.c_uint64)]),
    "cj_server_wait": (C.c_int, [_P, C.c_uint64, C.c_int64, C.POINTER(_P), C.POINTER(ExecStatsC)]),
    "cj_server_cancel": (C.c_int, [_P, C.c_uint64]),
    "cj_server_get_stats": (C.c_int, [_P, C.POINTER(ServerStatsC), C.c_int]),
    "cj_server_estimate": (C.c_int, [C.POINTER(PlanDesc), C.POINTER(C.c_uint64)]),
    "cj_server_destroy": (None, [_P]),
    "cj_host_alloc": (C.c_int, [C.c_uint64, C.POINTER(_P)]),
    "cj_host_free": (None, [_P]),
    "cj_encode_num_pages": (C.c_int, [C.c_int32, _P, C.POINTER(C.c_uint64), C.POINTER(C.c_uint8),
                                      C.c_uint64, C.POINTER(C.c_uint64)]),
    "cj_encode_column": (C.c_int, [C.c_int32, _P, C.POINTER(C.c_uint64), C.POINTER(C.c_uint8),
                                   C.c_uint64, _P, C.c_uint64, C.POINTER(C.c_uint64)]),
    "cj_last_error": (C.c_char_p, []),
    "cj_version": (C.c_char_p, []),
}

_lib = None


class CJError(RuntimeError):
    """A failed library call: `status` is the cj_status code."""

    def __init__(self, status: int, message: str):
        self.status = status
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")


def lib() -> C.CDLL:
    """The loaded library; raises if it was not built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with `python -m calamarijoins_b200.build`")
        h = C.CDLL(LIB_PATH)
        for name, (res, args) in _SIGS.items():
            f = getattr(h, name)
            f.restype = res
            f.argtypes = args
        _lib = h
    return _lib


def check(status: int) -> None:
    if status != CJ_OK:
        raise CJError(status, lib().cj_last_error().decode(errors="replace"))
