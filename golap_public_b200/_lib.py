"""ctypes binding of libgx.so (the C-ABI declared in include/gx.h).

The library is built in-tree by golap_public_b200.build.build().  There is no
fallback: if libgx.so cannot be loaded, every entry point raises.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

_PKG = Path(__file__).resolve().parent
LIB_PATH = _PKG / "libgx.so"

P = C.c_void_p
u8p = C.POINTER(C.c_uint8)

GX_OK, GX_ERR_CUDA, GX_ERR_CORRUPT, GX_ERR_CAPACITY, GX_ERR_TIMEOUT, GX_ERR_NOMEM, GX_ERR_INVALID = range(7)
GX_CODEC_NONE, GX_CODEC_LZ4, GX_CODEC_CASCADED = 0, 1, 2
GX_LZ4_LITERAL = 0xFFFFFFF0  # lz4_min_match admitting no match: every block one literal run
GX_STEP_FILTER, GX_STEP_PROBE, GX_STEP_CARRY, GX_STEP_VALUE, GX_STEP_GROUP = 1, 2, 4, 8, 16
GX_AGG_SUM, GX_AGG_SUM_PRODUCT, GX_AGG_COUNT, GX_AGG_BUILD, GX_AGG_SUM_DIFF = 0, 1, 2, 3, 4
GX_HT_LINEAR, GX_HT_BUCKET, GX_HT_DENSE = 0, 1, 2
GX_BATCH_AUTO, GX_BATCH_QUEUE, GX_BATCH_SHARED = 0, 1, 2
GX_FORM_AUTO, GX_FORM_WARP, GX_FORM_PIPE, GX_FORM_SHARED, GX_FORM_QUEUE = range(5)
GX_MAX_STEPS = 8


class GxError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"{_STATUS.get(status, status)}: {msg}")
        self.status = status


_STATUS = {0: "GX_OK", 1: "GX_ERR_CUDA", 2: "GX_ERR_CORRUPT", 3: "GX_ERR_CAPACITY", 4: "GX_ERR_TIMEOUT",
           5: "GX_ERR_NOMEM", 6: "GX_ERR_INVALID"}


class EncodeOpts(C.Structure):
    _fields_ = [("codec", C.c_uint32), ("rows_per_chunk", C.c_uint32), ("rows_per_block", C.c_uint32),
                ("lz4_segments", C.c_uint32), ("lz4_min_match", C.c_uint32), ("lz4_search_depth", C.c_uint32),
                ("casc_rle", C.c_uint32), ("casc_delta", C.c_uint32), ("casc_bitpack", C.c_uint32),
                ("threads", C.c_uint32)]


class ColumnInfo(C.Structure):
    _fields_ = [("n_rows", C.c_uint64), ("comp_bytes", C.c_uint64), ("uncomp_bytes", C.c_uint64),
                ("meta_bytes", C.c_uint64), ("codec", C.c_uint32), ("rows_per_chunk", C.c_uint32),
                ("rows_per_block", C.c_uint32), ("n_chunks", C.c_uint32), ("blocks_per_chunk", C.c_uint32),
                ("n_blocks", C.c_uint32), ("lz4_segments", C.c_uint32), ("on_device", C.c_uint32)]


class BlockInfo(C.Structure):
    _fields_ = [("offset", C.c_uint64), ("size", C.c_uint64), ("payload", C.c_uint64), ("tuples", C.c_uint64)]


class Pred(C.Structure):
    _fields_ = [("col_dev", P), ("lo", C.c_int32), ("hi", C.c_int32)]


class ScanStep(C.Structure):
    _fields_ = [("col", P), ("flags", C.c_uint32), ("lo", C.c_int32), ("hi", C.c_int32), ("ht", P),
                ("digit_base", C.c_int32), ("digit_card", C.c_uint32)]


class ScanPrune(C.Structure):
    _fields_ = [("col", P), ("lo", C.c_int32), ("hi", C.c_int32)]


class ScanPlan(C.Structure):
    _fields_ = [("n_steps", C.c_uint32), ("steps", ScanStep * GX_MAX_STEPS), ("agg", C.c_uint32),
                ("keep_chunks_dev", P), ("groupby", P), ("result_dev", P), ("n_prune", C.c_uint32),
                ("prune", ScanPrune * GX_MAX_STEPS), ("keep_out_dev", P), ("build_ht", P)]


class Query(C.Structure):
    _fields_ = [("plan", ScanPlan), ("row_lo", C.c_uint64), ("row_hi", C.c_uint64)]


class ServerOpts(C.Structure):
    _fields_ = [("max_inflight", C.c_uint32), ("max_batch", C.c_uint32), ("hbm_budget", C.c_uint64),
                ("batch_threads", C.c_uint32), ("batch_mode", C.c_uint32)]


class ServerStats(C.Structure):
    _fields_ = [(n, C.c_uint64) for n in ("submitted", "completed", "rejected", "batches", "queries_in_batches",
                                           "hbm_in_use", "hbm_peak", "queued")]


# name -> (restype, argtypes)
_SIGS = {
    "gx_status_str": (C.c_char_p, [C.c_int32]),
    "gx_last_error": (C.c_size_t, [C.c_char_p, C.c_size_t]),
    "gx_version": (C.c_char_p, []),
    "gx_device_count": (C.c_int32, [C.POINTER(C.c_int)]),
    "gx_encode_opts_default": (C.c_int32, [C.POINTER(EncodeOpts)]),
    "gx_column_encode": (C.c_int32, [P, C.c_uint64, C.POINTER(EncodeOpts), C.POINTER(P)]),
    "gx_column_encode_device": (C.c_int32, [P, C.c_uint64, C.POINTER(EncodeOpts), C.POINTER(P), P]),
    "gx_column_free": (C.c_int32, [P]),
    "gx_column_info_get": (C.c_int32, [P, C.POINTER(ColumnInfo)]),
    "gx_column_chunk_minmax": (C.c_int32, [P, P, P]),
    "gx_column_block_minmax": (C.c_int32, [P, P, P]),
    "gx_column_blocks": (C.c_int32, [P, P]),
    "gx_column_payload": (C.c_int32, [P, C.POINTER(u8p), C.POINTER(C.c_uint64)]),
    "gx_column_seg_index": (C.c_int32, [P, C.POINTER(C.POINTER(C.c_uint32)), C.POINTER(C.c_uint64)]),
    "gx_column_to_device": (C.c_int32, [P, C.c_int, P]),
    "gx_column_release_device": (C.c_int32, [P]),
    "gx_decompress_chunk": (C.c_int32, [P, C.c_uint64, P, P]),
    "gx_decompress_chunks": (C.c_int32, [P, C.c_uint64, C.c_uint64, P, P]),
    "gx_lz4_decompress_raw": (C.c_int32, [P, P, P, P, C.c_uint64, P, P]),
    "gx_check_minmax": (C.c_int32, [P, C.c_int32, C.c_int32, P, P]),
    "gx_combine_and": (C.c_int32, [P, P, P, C.c_uint64, P]),
    "gx_prune_minmax": (C.c_int32, [P, P, P, C.c_uint32, P, P]),
    "gx_hashtable_create": (C.c_int32, [C.c_uint64, C.POINTER(P)]),
    "gx_hashtable_create2": (C.c_int32, [C.c_uint64, C.c_uint32, C.POINTER(P)]),
    "gx_hashtable_free": (C.c_int32, [P]),
    "gx_hashtable_build": (C.c_int32, [P, P, P, C.c_uint64, P, C.c_uint32, P]),
    "gx_hashtable_count": (C.c_int32, [P, C.POINTER(C.c_uint64), P]),
    "gx_hashtable_probe": (C.c_int32, [P, P, C.c_uint64, P, P, P]),
    "gx_hashtable_view": (C.c_int32, [P, C.POINTER(P), C.POINTER(C.c_uint32)]),
    "gx_hashtable_view2": (C.c_int32, [P, C.POINTER(P), C.POINTER(C.c_uint32), C.POINTER(P)]),
    "gx_hashtable_clear": (C.c_int32, [P, P]),
    "gx_hashtable_keys": (C.c_int32, [P, P, C.c_uint64, P, P]),
    "gx_check_minmax_points": (C.c_int32, [P, P, P, C.c_uint64, P, P]),
    "gx_column_build_hist": (C.c_int32, [P, C.c_uint32, P]),
    "gx_check_hist": (C.c_int32, [P, C.c_int32, C.c_int32, P, P]),
    "gx_column_build_bloom": (C.c_int32, [P, C.c_uint64, C.c_double, P]),
    "gx_check_bloom": (C.c_int32, [P, C.c_int32, P, P]),
    "gx_column_meta_read": (C.c_int32, [P, P, P, C.POINTER(C.c_uint32), C.POINTER(C.c_uint64),
                                        C.POINTER(C.c_uint32), P]),
    "gx_minmax_reduce": (C.c_int32, [P, C.c_uint64, P, P]),
    "gx_groupby_view": (C.c_int32, [P, C.POINTER(P), C.POINTER(P), C.POINTER(C.c_uint32)]),
    "gx_groupby_create": (C.c_int32, [C.c_uint64, C.POINTER(P)]),
    "gx_groupby_free": (C.c_int32, [P]),
    "gx_groupby_reset": (C.c_int32, [P, P]),
    "gx_groupby_add": (C.c_int32, [P, P, P, C.c_uint64, P]),
    "gx_groupby_read": (C.c_int32, [P, P, P, C.c_uint64, C.POINTER(C.c_uint64), P]),
    "gx_scan": (C.c_int32, [C.POINTER(ScanPlan), P]),
    "gx_scan_static": (C.c_int32, [C.POINTER(ScanPlan), P]),
    "gx_scan_streamed": (C.c_int32, [C.POINTER(ScanPlan), C.c_uint32, P]),
    "gx_scan_set_form": (C.c_int32, [C.c_uint32]),
    "gx_scan_sync": (C.c_int32, [C.POINTER(ScanPlan), P, C.POINTER(C.c_uint64)]),
    "gx_scan_check": (C.c_int32, [P]),
    "gx_batch_create": (C.c_int32, [C.POINTER(Query), C.c_uint32, C.POINTER(P)]),
    "gx_batch_create2": (C.c_int32, [C.POINTER(Query), C.c_uint32, C.c_uint32, C.POINTER(P)]),
    "gx_batch_mode": (C.c_int32, [P, C.POINTER(C.c_uint32)]),
    "gx_batch_set_launch": (C.c_int32, [P, C.c_uint32, C.c_uint32]),
    "gx_batch_launch_get": (C.c_int32, [P, C.POINTER(C.c_uint32)]),
    "gx_batch_free": (C.c_int32, [P]),
    "gx_batch_run": (C.c_int32, [P, P]),
    "gx_batch_graph": (C.c_int32, [P, P]),
    "gx_batch_rows": (C.c_int32, [P, C.POINTER(C.c_uint64), P]),
    "gx_batch_assign": (C.c_int32, [P, C.POINTER(Query), C.c_uint32, P]),
    "gx_server_opts_default": (C.c_int32, [C.POINTER(ServerOpts)]),
    "gx_server_create": (C.c_int32, [C.POINTER(ServerOpts), C.POINTER(P)]),
    "gx_server_submit": (C.c_int32, [P, C.POINTER(Query), C.c_uint64, C.POINTER(C.c_uint64)]),
    "gx_server_wait": (C.c_int32, [P, C.c_uint64, C.c_double, C.POINTER(C.c_double)]),
    "gx_server_stats_get": (C.c_int32, [P, C.POINTER(ServerStats)]),
    "gx_server_free": (C.c_int32, [P]),
}

_lib = None


def lib():
    """Load libgx.so (raises if it is missing: there is no non-CUDA path)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise ImportError(f"{LIB_PATH} is not built; run golap_public_b200.build.build()")
        L = C.CDLL(str(LIB_PATH))
        for name, (res, args) in _SIGS.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def exported_symbols():
    return list(_SIGS)


def last_error() -> str:
    buf = C.create_string_buffer(1024)
    lib().gx_last_error(buf, 1024)
    return buf.value.decode(errors="replace")


def check(status: int) -> None:
    if status != GX_OK:
        raise GxError(status, last_error())
