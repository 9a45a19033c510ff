"""ctypes declarations of include/wadjet_gpu.h (the C ABI of libwadjetgpu.so)."""
from __future__ import annotations

import ctypes as C
import os

_PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_PKG, "libwadjetgpu.so")

# status codes
WG_OK, WG_E_NOMEM, WG_E_INVALID, WG_E_TIMEOUT, WG_E_CUDA, WG_E_UNSUPPORTED, WG_E_STATE, WG_E_CANCELLED = range(8)

# parquet.TypeID values (internal/storage/parquet/schema.go:13-34)
TYPE_BOOL, TYPE_INT32, TYPE_INT64, TYPE_FLOAT32, TYPE_FLOAT64 = 0, 1, 2, 3, 4
TYPE_STRING, TYPE_BYTES, TYPE_TIMESTAMP, TYPE_IPV4, TYPE_IPV6, TYPE_CIDR = 5, 6, 7, 8, 9, 10
TYPE_MAC, TYPE_PORT, TYPE_PROTOCOL, TYPE_DURATION, TYPE_UUID, TYPE_DATE, TYPE_DECIMAL = 11, 12, 13, 14, 15, 16, 17

# kernel.CompareOp
OP_EQ, OP_NE, OP_LT, OP_LE, OP_GT, OP_GE = range(6)
CONST_INT, CONST_FLOAT = 0, 1
# exec.AggFunc
AGG_SUM, AGG_COUNT, AGG_MIN, AGG_MAX, AGG_AVG = range(5)
JOIN_INNER, JOIN_LEFT, JOIN_SEMI, JOIN_ANTI = 0, 1, 5, 6
# parquet.Encoding of a page's values section
ENC_PLAIN, ENC_PLAIN_DICTIONARY, ENC_RLE_DICTIONARY = 0, 2, 8
# expression opcodes
EXPR_COL, EXPR_CONST_I, EXPR_CONST_F, EXPR_ADD, EXPR_SUB, EXPR_MUL, EXPR_DIV, EXPR_SHR, EXPR_AND = range(9)
EXPR_MAX_OPS = 12


class wg_int128(C.Structure):
    _fields_ = [("hi", C.c_int64), ("lo", C.c_uint64)]


class wg_column(C.Structure):
    _fields_ = [("type_id", C.c_int32), ("scale", C.c_int32), ("data", C.c_void_p),
                ("valid_words", C.c_void_p), ("len", C.c_int64)]


class wg_bytes(C.Structure):
    _fields_ = [("offsets", C.c_void_p), ("bytes", C.c_void_p)]


class wg_batch_desc(C.Structure):
    _fields_ = [("ncols", C.c_int32), ("_pad", C.c_int32), ("cols", C.POINTER(wg_column)),
                ("len", C.c_int64), ("sel", C.c_void_p), ("sel_len", C.c_int64)]


class wg_agg_spec(C.Structure):
    _fields_ = [("func", C.c_int32), ("input_col", C.c_int32), ("out_type", C.c_int32), ("_pad", C.c_int32)]


class wg_predicate(C.Structure):
    _fields_ = [("col", C.c_int32), ("op", C.c_int32), ("const_kind", C.c_int32), ("_pad", C.c_int32),
                ("const_i64", C.c_int64), ("const_f64", C.c_double)]


class wg_expr_op(C.Structure):
    _fields_ = [("opcode", C.c_int32), ("arg", C.c_int32), ("imm_i64", C.c_int64), ("imm_f64", C.c_double)]


class wg_expr(C.Structure):
    _fields_ = [("result_type", C.c_int32), ("n_ops", C.c_int32), ("ops", wg_expr_op * EXPR_MAX_OPS)]


class wg_group_export(C.Structure):
    _fields_ = [("keys", C.c_void_p), ("key_valid", C.c_void_p), ("count", C.c_void_p), ("i64", C.c_void_p),
                ("f64", C.c_void_p), ("dec", C.c_void_p), ("has", C.c_void_p)]


class wg_pipeline_desc(C.Structure):
    _fields_ = [("input", C.POINTER(wg_batch_desc)), ("n_filters", C.c_int32), ("n_exprs", C.c_int32),
                ("filters", C.POINTER(wg_predicate)), ("join", C.c_void_p), ("exprs", C.POINTER(wg_expr)),
                ("agg", C.c_void_p)]


class wg_batched_query(C.Structure):
    _fields_ = [("input", C.POINTER(wg_batch_desc)), ("n_filters", C.c_int32), ("n_aggs", C.c_int32),
                ("filters", C.POINTER(wg_predicate)), ("key_cols", C.POINTER(C.c_int32)), ("n_keys", C.c_int32),
                ("n_exprs", C.c_int32), ("aggs", C.POINTER(wg_agg_spec)), ("ndv_hint", C.c_int64),
                ("join", C.c_void_p), ("exprs", C.POINTER(wg_expr))]


class wg_tune_params(C.Structure):
    _fields_ = [("tile_rows", C.c_int32), ("block", C.c_int32), ("ctas_per_sm", C.c_int32),
                ("smem_max_groups", C.c_int32), ("max_load", C.c_double)]


class wg_page(C.Structure):
    _fields_ = [("encoding", C.c_int32), ("_pad", C.c_int32), ("num_values", C.c_int64),
                ("def_levels", C.c_void_p), ("def_len", C.c_int64), ("data", C.c_void_p), ("data_len", C.c_int64)]


class wg_column_chunk(C.Structure):
    _fields_ = [("type_id", C.c_int32), ("scale", C.c_int32), ("n_pages", C.c_int32), ("_pad", C.c_int32),
                ("pages", C.POINTER(wg_page)), ("dict", C.c_void_p), ("dict_len", C.c_int64)]


class wg_state_layout(C.Structure):
    _fields_ = [("key_words", C.c_int32), ("slot_words", C.c_int32), ("n_keys", C.c_int32), ("n_aggs", C.c_int32),
                ("key_type", C.c_int32 * 4), ("key_i32", C.c_int32 * 4), ("key_word", C.c_int32 * 4),
                ("key_shift", C.c_int32 * 4), ("null_word", C.c_int32), ("null_shift", C.c_int32),
                ("agg_kind", C.c_int32 * 8), ("agg_off", C.c_int32 * 8),
                ("agg_null_off", C.c_int32 * 8), ("agg_in_cls", C.c_int32 * 8), ("agg_in_scale", C.c_int32 * 8),
                ("agg_out_type", C.c_int32 * 8), ("agg_nullable", C.c_int32 * 8)]


class wg_serve_request(C.Structure):
    _fields_ = [("plan", C.POINTER(wg_pipeline_desc)), ("key_cols", C.POINTER(C.c_int32)),
                ("aggs", C.POINTER(wg_agg_spec)), ("n_keys", C.c_int32), ("n_aggs", C.c_int32),
                ("ndv_hint", C.c_int64), ("est_bytes", C.c_int64)]


class wg_serve_stats(C.Structure):
    _fields_ = [("submitted", C.c_int64), ("completed", C.c_int64), ("failed", C.c_int64),
                ("in_flight", C.c_int64), ("queued", C.c_int64), ("cancelled", C.c_int64),
                ("p50_s", C.c_double), ("p99_s", C.c_double),
                ("mean_s", C.c_double), ("max_s", C.c_double), ("qps", C.c_double),
                ("mean_queue_s", C.c_double), ("mean_service_s", C.c_double)]


P = C.c_void_p
PP = C.POINTER(C.c_void_p)
I32, I64, F64 = C.c_int32, C.c_int64, C.c_double
PI64 = C.POINTER(C.c_int64)

# name -> (restype, argtypes); every symbol include/wadjet_gpu.h declares
SIGNATURES = {
    "wg_last_error": (C.c_char_p, []),
    "wg_version": (C.c_char_p, []),
    "wg_ctx_create": (I32, [I32, I64, I64, PP]),
    "wg_ctx_create_child": (I32, [P, PP]),
    "wg_ctx_destroy": (I32, [P]),
    "wg_ctx_synchronize": (I32, [P]),
    "wg_ledger_stats": (I32, [P, PI64, PI64, PI64]),
    "wg_ledger_reserve": (I32, [P, I64]),
    "wg_ledger_release": (I32, [P, I64]),
    "wg_ctx_stream": (P, [P]),
    "wg_ctx_launch_count": (I64, [P]),
    "wg_filter_create": (I32, [P, I32, I32, I32, I64, F64, PP]),
    "wg_filter_execute": (I32, [P, C.POINTER(wg_batch_desc), P, PI64]),
    "wg_filter_execute_device": (I32, [P, C.POINTER(wg_batch_desc), P, PI64]),
    "wg_filter_destroy": (I32, [P]),
    "wg_filter_execute_device_noalloc": (I32, [P, C.POINTER(wg_column), P, I64, I32, I32, I64, F64, P, PI64]),
    "wg_join_create": (I32, [P, I32, I32, I32, I32, C.POINTER(C.c_int32), I64, PP]),
    "wg_join_build_append": (I32, [P, C.POINTER(wg_batch_desc)]),
    "wg_join_build_append_device": (I32, [P, C.POINTER(wg_batch_desc)]),
    "wg_join_build_finish": (I32, [P]),
    "wg_join_build_stats": (I32, [P, PI64, PI64]),
    "wg_join_probe": (I32, [P, C.POINTER(wg_batch_desc), P, P, I64, PI64, PI64]),
    "wg_join_gather": (I32, [P, I32, P, I64, P, P]),
    "wg_join_bloom_filter": (I32, [P, C.POINTER(wg_batch_desc), P, PI64]),
    "wg_join_reset": (I32, [P]),
    "wg_join_destroy": (I32, [P]),
    "wg_agg_create": (I32, [P, I32, C.POINTER(C.c_int32), I32, C.POINTER(wg_agg_spec), I64, PP]),
    "wg_agg_consume": (I32, [P, C.POINTER(wg_batch_desc)]),
    "wg_agg_consume_device": (I32, [P, C.POINTER(wg_batch_desc)]),
    "wg_agg_clone": (I32, [P, PP]),
    "wg_agg_merge": (I32, [P, P]),
    "wg_agg_finalize": (I32, [P, PI64]),
    "wg_agg_emit": (I32, [P, I64, I64, C.POINTER(wg_column), PI64]),
    "wg_agg_export": (I32, [P, C.POINTER(wg_group_export)]),
    "wg_agg_key_strings": (I32, [P, PI64, I64, P, P, I64, PI64]),
    "wg_agg_reset": (I32, [P]),
    "wg_agg_kernel_shape": (I32, [P]),
    "wg_batch_upload": (I32, [P, C.POINTER(wg_batch_desc), PP]),
    "wg_batch_device_desc": (I32, [P, C.POINTER(wg_batch_desc), C.POINTER(wg_column), I32]),
    "wg_batch_destroy": (I32, [P]),
    "wg_batch_decode": (I32, [P, C.POINTER(wg_column_chunk), I32, PP]),
    "wg_agg_state_layout": (I32, [P, C.POINTER(wg_state_layout)]),
    "wg_agg_partition_state": (I32, [P, I32, P, I64, PI64]),
    "wg_agg_merge_state": (I32, [P, C.POINTER(wg_state_layout), P, I64]),
    "wg_agg_destroy": (I32, [P]),
    "wg_pipeline_run": (I32, [P, C.POINTER(wg_pipeline_desc)]),
    "wg_pipeline_run_device": (I32, [P, C.POINTER(wg_pipeline_desc)]),
    "wg_batched_create": (I32, [P, I32, C.POINTER(wg_batched_query), C.POINTER(wg_tune_params), PP]),
    "wg_batched_run": (I32, [P, PI64]),
    "wg_batched_export": (I32, [P, I32, C.POINTER(wg_group_export)]),
    "wg_batched_destroy": (I32, [P]),
    "wg_server_create": (I32, [P, I32, PP]),
    "wg_server_submit": (I32, [P, C.POINTER(wg_serve_request), PI64]),
    "wg_server_wait": (I32, [P, I64, F64, PI64, C.POINTER(C.c_double)]),
    "wg_server_export": (I32, [P, I64, C.POINTER(wg_group_export)]),
    "wg_server_release": (I32, [P, I64]),
    "wg_server_cancel": (I32, [P, I64]),
    "wg_server_stats": (I32, [P, C.POINTER(wg_serve_stats)]),
    "wg_server_reset_stats": (I32, [P]),
    "wg_server_destroy": (I32, [P]),
    "wg_synth_starjoin_fact": (I32, [P, C.c_uint64, I64, I64, P, P, P, P]),
    "wg_synth_starjoin_dim": (I32, [P, C.c_uint64, I64, P, P]),
    "wg_synth_groupby": (I32, [P, C.c_uint64, I64, I64, I64, P, P, P, P]),
    "wg_synth_highcard": (I32, [P, C.c_uint64, I64, I64, P, P, P, P]),
    "wg_synth_batched_params": (I32, [C.c_uint64, I32, PI64, PI64, C.POINTER(C.c_int32)]),
    "wg_synth_batched": (I32, [P, C.c_uint64, I32, I64, I64, P, P, P, P]),
}

_lib = None


def load() -> C.CDLL:
    """Load libwadjetgpu.so from the package directory (built by wadjet_b200.build).

    There is no fallback: without the library the GPU operators do not exist.
    """
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m wadjet_b200.build`")
    lib = C.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib
