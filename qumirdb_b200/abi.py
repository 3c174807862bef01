"""ctypes mirror of include/qdb_gpu.h (structs, enums, entry points).

The layouts match the C header field for field; `qdb_column` / `qdb_rowset`
are the engine's TColumn / TRowSet (qdb/io/io.h:17-39).
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

# qdb_type
BOOL, I8, I16, I32, I64, U8, U16, U32, U64, F32, F64, DATE32, DECIMAL64, DECIMAL128, CHAR1 = range(1, 16)
STRING = 16   # Arrow layout: offsets (int32 / int64) into the bytes; hash-program keys
# qdb_expr_op
(COLUMN, CONST, NULL, ADD, SUB, MUL, DIV, NEG, CAST, EQ, NE, LT, LE, GT, GE, AND, OR, NOT, BETWEEN, IN_LIST,
 CASE, IS_NULL, IS_NOT_NULL, MOD) = range(1, 25)
# qdb_agg_func
COUNT_STAR, COUNT, SUM, MIN, MAX = range(1, 6)
# agg_dispatch ops
AGG_INIT, AGG_UPDATE, AGG_INIT_ROWS, AGG_SWITCH_TO_ROWS_AT, AGG_EXPECT_ROW_GROUPS = 0, 1, 3, 4, 5
# jr_dispatch ops
JR_INIT, JR_APPEND, JR_BUILD, JR_PROBE = 0, 1, 2, 3
JR_APPEND_NULL_KEYS, JR_EMIT_BY_MARK = 5, 6
# qdb_join_type (EJoinType order)
JOIN_INNER, JOIN_LEFT, JOIN_RIGHT, JOIN_FULL = 0, 1, 2, 3
JOIN_LEFT_SEMI, JOIN_RIGHT_SEMI, JOIN_LEFT_ANTI, JOIN_RIGHT_ANTI = 4, 5, 6, 7
OUT_DEVICE = 1

HASH_TABLE_SIZE = 304
ROW_ARENA_SIZE = 56
ROW_TABLE_SIZE = 48
ROW_SCRATCH_SIZE = 64
PAIR_BUFFER_SIZE = 24

WIDTH = {BOOL: 1, I8: 1, I16: 2, I32: 4, I64: 8, U8: 1, U16: 2, U32: 4, U64: 8, F32: 4, F64: 8, DATE32: 4,
         DECIMAL64: 8, DECIMAL128: 16, CHAR1: 1}


class Column(C.Structure):
    _fields_ = [("Data", C.c_void_p), ("DataBitOffset", C.c_int32), ("Mask", C.c_void_p),
                ("MaskBitOffset", C.c_int32), ("Offsets", C.c_void_p), ("OffsetWidth", C.c_uint8)]


class RowSet(C.Structure):
    pass


RowSet._fields_ = [("Columns", C.POINTER(Column)), ("ColumnCount", C.c_int64), ("RowCount", C.c_int64),
                   ("Selection", C.c_void_p), ("Hash", C.c_void_p),
                   ("Destroy", C.CFUNCTYPE(None, C.POINTER(RowSet))), ("Private", C.c_void_p),
                   ("RefCount", C.c_int64)]


class ColumnType(C.Structure):
    _fields_ = [("type", C.c_int32), ("precision", C.c_int32), ("scale", C.c_int32), ("nullable", C.c_int32)]


class Expr(C.Structure):
    _fields_ = [("op", C.c_int32), ("type", C.c_int32), ("scale", C.c_int32), ("column", C.c_int32),
                ("args", C.c_int32 * 3), ("list_len", C.c_int32), ("imm_lo", C.c_int64), ("imm_hi", C.c_int64),
                ("list", C.POINTER(C.c_int64))]


class AggItem(C.Structure):
    _fields_ = [("func", C.c_int32), ("arg", C.c_int32)]


class AggregateSpec(C.Structure):
    _fields_ = [("n_columns", C.c_int32), ("columns", C.POINTER(ColumnType)),
                ("n_nodes", C.c_int32), ("nodes", C.POINTER(Expr)), ("filter", C.c_int32),
                ("n_keys", C.c_int32), ("keys", C.POINTER(C.c_int32)),
                ("n_aggs", C.c_int32), ("aggs", C.POINTER(AggItem)),
                ("n_outputs", C.c_int32), ("outputs", C.POINTER(C.c_int32)),
                ("n_output_nodes", C.c_int32), ("output_nodes", C.POINTER(Expr)),
                ("flags", C.c_uint32), ("expected_groups", C.c_int64)]


class RowJoinSpec(C.Structure):
    _fields_ = [("join_type", C.c_int32), ("build_is_left", C.c_int32),
                ("n_build_columns", C.c_int32), ("build_columns", C.POINTER(ColumnType)),
                ("n_probe_columns", C.c_int32), ("probe_columns", C.POINTER(ColumnType)),
                ("n_keys", C.c_int32), ("build_keys", C.POINTER(C.c_int32)), ("probe_keys", C.POINTER(C.c_int32)),
                ("n_payload", C.c_int32), ("build_payload", C.POINTER(C.c_int32)),
                ("n_out", C.c_int32), ("out_side", C.POINTER(C.c_int32)), ("out_column", C.POINTER(C.c_int32)),
                ("n_build_nodes", C.c_int32), ("build_nodes", C.POINTER(Expr)), ("build_filter", C.c_int32),
                ("flags", C.c_uint32)]


class SortKey(C.Structure):
    _fields_ = [("column", C.c_int32), ("desc", C.c_int32), ("nulls_first", C.c_int32), ("pad", C.c_int32)]


class SortSpec(C.Structure):
    _fields_ = [("n_columns", C.c_int32), ("columns", C.POINTER(ColumnType)),
                ("n_keys", C.c_int32), ("keys", C.POINTER(SortKey)),
                ("n_out", C.c_int32), ("out_columns", C.POINTER(C.c_int32)), ("flags", C.c_uint32)]


class RfBuildState(C.Structure):
    """qdb_rf_build_state (RuntimeFilterBuild)."""
    _fields_ = [("MaxKeys", C.c_int64), ("Mode", C.c_int64), ("Want", C.c_int64), ("Keys", C.c_void_p),
                ("KeyCount", C.c_int64), ("SetCtrl", C.c_void_p), ("SetSlots", C.c_void_p),
                ("SetCapacity", C.c_int64), ("SortOrder", C.c_void_p), ("SortKeys", C.c_void_p),
                ("Bloom", C.c_void_p), ("BloomWords", C.c_int64)]


class RfPartial(C.Structure):
    """qdb_rf_partial (RuntimeFilterPartial)."""
    _fields_ = [("Keys", C.c_void_p), ("KeyCount", C.c_int64), ("Bloom", C.c_void_p), ("BloomWords", C.c_int64)]


class RfPublishState(C.Structure):
    """qdb_rf_publish_state (RuntimeFilterPublish)."""
    _fields_ = [("MaxKeys", C.c_int64), ("Keys", C.c_void_p), ("SetCtrl", C.c_void_p), ("SetSlots", C.c_void_p),
                ("SetCapacity", C.c_int64), ("Table", C.c_void_p), ("Bloom", C.c_void_p),
                ("BloomWords", C.c_int64), ("BloomSeeded", C.c_int64), ("Kind", C.c_int64),
                ("ExactKeys", C.c_int64), ("TableSize", C.c_int64), ("BloomSetBits", C.c_int64)]


class RfData(C.Structure):
    """qdb_rf_data (RuntimeFilterData)."""
    _fields_ = [("Kind", C.c_int64), ("Words", C.c_void_p), ("WordCount", C.c_int64)]


class CacheStats(C.Structure):
    """qdb_gpu_cache_stats."""
    _fields_ = [("hits", C.c_int64), ("misses", C.c_int64), ("evictions", C.c_int64), ("resident_bytes", C.c_int64),
                ("pinned_bytes", C.c_int64), ("h2d_bytes", C.c_int64), ("entries", C.c_int64)]


class KernelTime(C.Structure):
    _fields_ = [("name", C.c_char * 48), ("ms", C.c_double), ("units", C.c_int64)]


P = C.c_void_p
CI32, CI64, CU64, SZ, BOOLC = C.c_int32, C.c_int64, C.c_uint64, C.c_size_t, C.c_bool
PRS = C.POINTER(RowSet)

SIGNATURES = {
    "qdb_gpu_compile_aggregate": (P, [C.POINTER(AggregateSpec), C.c_char_p, SZ]),
    "qdb_gpu_compile_filter": (P, [CI32, C.POINTER(ColumnType), CI32, C.POINTER(Expr), CI32, C.c_char_p, SZ]),
    "qdb_gpu_compile_project": (P, [CI32, C.POINTER(ColumnType), CI32, C.POINTER(Expr), CI32, C.POINTER(CI32),
                                    C.c_char_p, SZ]),
    "qdb_gpu_compile_hash": (P, [CI32, C.POINTER(ColumnType), CI32, C.POINTER(CI32), C.c_char_p, SZ]),
    "qdb_gpu_compile_row_join": (P, [C.POINTER(RowJoinSpec), C.c_char_p, SZ]),
    "qdb_gpu_compile_join_aggregate": (P, [C.POINTER(RowJoinSpec), C.POINTER(AggregateSpec), C.c_char_p, SZ]),
    "qdb_gpu_compile_sort": (P, [C.POINTER(SortSpec), C.c_char_p, SZ]),
    "qdb_gpu_program_destroy": (None, [P]),
    "qdb_gpu_agg_dispatch": (CI64, [P, P, PRS, CI64, CI64]),
    "qdb_gpu_agg_finish_rowset": (CI64, [P, P, PRS]),
    "qdb_gpu_filter": (None, [P, PRS, P]),
    "qdb_gpu_project": (None, [P, PRS, C.POINTER(P), P, P]),
    "qdb_gpu_hash": (BOOLC, [P, PRS, P]),
    "qdb_gpu_jr_dispatch": (BOOLC, [P, P, P, P, P, PRS, CI64]),
    "qdb_gpu_jr_materialize": (CI64, [P, P, PRS, CI64, CI64, PRS]),
    "qdb_gpu_agg_release": (None, [P]),
    "qdb_gpu_agg_dispatch_batch": (CI64, [P, C.POINTER(P), C.POINTER(PRS), CI64]),
    "qdb_gpu_agg_finish_batch": (CI64, [P, C.POINTER(P), CI64, PRS]),
    "qdb_gpu_autotune_info": (CI64, [C.c_char_p, CI64]),
    "qdb_gpu_autotune_reset": (None, []),
    "qdb_gpu_release_rowsets": (None, [PRS, CI64]),
    "qdb_gpu_jr_release": (None, [P, P, P, P]),
    "qdb_gpu_join_aggregate_probe": (CI64, [P, P, P, P, PRS]),
    "qdb_gpu_sort_run": (CI64, [P, PRS, P, P, P, CI64, P, P, BOOLC, CI64, CI64, PRS]),
    "qdb_gpu_top_k_select": (CI64, [P, PRS, P, CI64, CI64]),
    "qdb_gpu_top_sort_update": (CI64, [P, PRS, PRS, P, P, P, CI64, BOOLC, P, P, CI64, PRS]),
    "qdb_gpu_agg_run_noalloc": (CI64, [P, PRS, C.POINTER(Column), CI64]),
    "qdb_gpu_rf_build": (CI64, [C.POINTER(RfBuildState), P, P, CI64]),
    "qdb_gpu_rf_publish": (CI64, [C.POINTER(RfPublishState), C.POINTER(RfPartial), CI64]),
    "qdb_gpu_rf_probe": (CI64, [C.POINTER(RfData), P, P, P, CI64, CI64, P, P]),
    "qdb_gpu_rf_merge": (CI64, [P, P, CI64]),
    "qdb_gpu_rf_probe_rowset": (CI64, [P, C.POINTER(RfData), PRS, P]),
    "qdb_gpu_shuffle": (CI64, [P, PRS, P, CI64, CI64, PRS]),
    "qdb_gpu_jr_build_batch": (BOOLC, [P, C.POINTER(P), C.POINTER(P), CI64]),
    "qdb_gpu_jr_append_batch": (BOOLC, [P, C.POINTER(P), C.POINTER(PRS), CI64]),
    "qdb_gpu_join_aggregate_probe_batch": (CI64, [P, C.POINTER(P), C.POINTER(P), C.POINTER(P), C.POINTER(PRS), CI64]),
    "qdb_gpu_cache_create": (P, [SZ, SZ]),
    "qdb_gpu_cache_destroy": (None, [P]),
    "qdb_gpu_cache_get": (CI64, [P, CU64, CI64, PRS, C.POINTER(ColumnType), C.POINTER(CI32), CI32, PRS]),
    "qdb_gpu_cache_invalidate": (CI64, [P, CU64]),
    "qdb_gpu_cache_get_stats": (None, [P, C.POINTER(CacheStats)]),
    "qdb_gpu_init": (C.c_int, [C.c_int]),
    "qdb_gpu_last_error": (C.c_char_p, []),
    "qdb_gpu_set_stream": (None, [P]),
    "qdb_gpu_get_stream": (P, []),
    "qdb_gpu_synchronize": (C.c_int, []),
    "qdb_gpu_alloc": (P, [SZ]),
    "qdb_gpu_free": (None, [P]),
    "qdb_gpu_host_alloc": (P, [SZ]),
    "qdb_gpu_host_free": (None, [P]),
    "qdb_gpu_memcpy": (C.c_int, [P, P, SZ]),
    "qdb_gpu_memset": (C.c_int, [P, C.c_int, SZ]),
    "qdb_gpu_profile_enable": (None, [C.c_int]),
    "qdb_gpu_profile_read": (CI64, [C.POINTER(KernelTime), CI64]),
    "qdb_gpu_launch_count": (CI64, [C.c_int]),
    "qdb_gen_lineitem": (None, [CU64, CI64, P, P, P, P, P, P, P]),
    "qdb_gen_join": (None, [CU64, CI64, CI64, CI64, P, P, P, P, P]),
    "qdb_gen_zipf": (None, [CU64, CI64, CI64, C.c_double, P, P, P]),
    "qdb_gen_sort": (None, [CU64, CI64, P, P, P]),
}


def header_symbols(header: Path) -> list[str]:
    """Names of the functions include/qdb_gpu.h declares."""
    import re
    text = header.read_text()
    return sorted(set(re.findall(r"\b(qdb_(?:gpu|gen)_[a-z0-9_]+)\s*\(", text)))


def bind(lib: C.CDLL) -> C.CDLL:
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib
