"""ctypes wrapper of the CPU oracle (oracle/oracle.cpp).

TEST INFRASTRUCTURE ONLY: used by tests/, __graft_entry__.smoke() and
bench.py's cpu_baseline / reference arm as the checker and the timed CPU
baseline; the product never imports it.
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

from qumirdb_b200 import abi

HERE = Path(__file__).resolve().parent
LIB = HERE / "_build" / "liboracle.so"

_lib = None


class OracleTable(C.Structure):
    _fields_ = [("rows", C.c_int64), ("cols", C.c_int32), ("types", C.POINTER(C.c_int32)),
                ("scales", C.POINTER(C.c_int32)), ("cells", C.POINTER(C.c_int64)), ("valid", C.POINTER(C.c_uint8))]


def build() -> Path:
    srcs = [HERE / "oracle.cpp", HERE / "oracle.h", HERE / "Makefile", HERE.parent / "include" / "qdb_gpu.h",
            HERE.parent / "qumirdb_b200" / "csrc" / "datagen.cpp"]
    if not LIB.exists() or LIB.stat().st_mtime < max(s.stat().st_mtime for s in srcs):
        subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return LIB


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(str(LIB))
        P = C.c_void_p
        sig = {
            "oracle_table_free": (None, [C.POINTER(OracleTable)]),
            "oracle_aggregate": (C.c_int, [C.POINTER(abi.AggregateSpec), C.POINTER(abi.RowSet), C.c_int32, C.c_int32,
                                           C.POINTER(OracleTable), C.c_char_p, C.c_size_t]),
            "oracle_filter": (C.c_int, [C.c_int32, P, C.c_int32, P, C.c_int32, C.POINTER(abi.RowSet), P, C.c_char_p,
                                        C.c_size_t]),
            "oracle_project": (C.c_int, [C.c_int32, P, C.c_int32, P, C.c_int32, P, C.POINTER(abi.RowSet),
                                         C.POINTER(P), C.POINTER(P), C.c_char_p, C.c_size_t]),
            "oracle_hash": (C.c_int, [C.c_int32, P, C.c_int32, P, C.POINTER(abi.RowSet), P, C.c_char_p, C.c_size_t]),
            "oracle_row_join": (C.c_int64, [C.POINTER(abi.RowJoinSpec), C.POINTER(abi.RowSet), C.c_int32,
                                            C.POINTER(abi.RowSet), P, C.c_int64, C.c_char_p, C.c_size_t]),
            "oracle_row_join_typed": (C.c_int64, [C.POINTER(abi.RowJoinSpec), C.POINTER(abi.RowSet), C.c_int32,
                                                  C.POINTER(abi.RowSet), C.c_int32, P, C.c_int64, C.c_char_p,
                                                  C.c_size_t]),
            "oracle_rf_build": (C.c_int64, [C.POINTER(abi.RfBuildState), P, P, C.c_int64]),
            "oracle_rf_publish": (C.c_int64, [C.POINTER(abi.RfPublishState), C.POINTER(abi.RfPartial), C.c_int64]),
            "oracle_rf_probe": (C.c_int64, [C.POINTER(abi.RfData), P, P, P, C.c_int64]),
            "oracle_rf_merge": (None, [P, P, C.c_int64]),
            "oracle_mt19937_64": (None, [C.c_uint64, C.c_int64, P]),
            "oracle_string_hash": (C.c_uint64, [P, C.c_int64]),
            "oracle_string_secret": (C.c_void_p, []),
            "oracle_route": (C.c_int64, [P, P, C.c_int64, P, C.c_int64, C.c_int64, P]),
            "oracle_join_aggregate": (C.c_int, [C.POINTER(abi.RowJoinSpec), C.POINTER(abi.AggregateSpec),
                                                C.POINTER(abi.RowSet), C.c_int32, C.POINTER(abi.RowSet), C.c_int32,
                                                C.c_int32, C.POINTER(OracleTable), C.c_char_p, C.c_size_t]),
            "oracle_sort": (C.c_int, [C.POINTER(abi.SortSpec), C.POINTER(abi.RowSet), P, C.c_int64, P, P,
                                      C.c_char_p, C.c_size_t]),
            "oracle_top_k": (C.c_int64, [C.POINTER(abi.SortSpec), C.POINTER(abi.RowSet), P, C.c_int64, C.c_int64,
                                         P, P]),
            "oracle_top_sort_update": (C.c_int64, [C.POINTER(abi.SortSpec), C.POINTER(abi.RowSet),
                                                   C.POINTER(abi.RowSet), P, C.c_int64, C.c_bool, P, P, C.c_int64,
                                                   C.c_char_p, C.c_size_t]),
            "oracle_bench_aggregate": (C.c_double, [C.POINTER(abi.AggregateSpec), C.POINTER(abi.RowSet), C.c_int32,
                                                    C.POINTER(C.c_int64)]),
            "oracle_bench_join_sum": (C.c_double, [P, P, P, C.c_int64, C.c_int32, P, P, C.c_int64, C.c_int32,
                                                   C.POINTER(C.c_int64), C.POINTER(C.c_int64)]),
            "oracle_bench_sort": (C.c_double, [P, P, C.c_int64, C.c_int32, P]),
            # The seeded workload generators (same code as the device library's).
            "qdb_gen_lineitem": (None, [C.c_uint64, C.c_int64, P, P, P, P, P, P, P]),
            "qdb_gen_join": (None, [C.c_uint64, C.c_int64, C.c_int64, C.c_int64, P, P, P, P, P]),
            "qdb_gen_zipf": (None, [C.c_uint64, C.c_int64, C.c_int64, C.c_double, P, P, P]),
            "qdb_gen_sort": (None, [C.c_uint64, C.c_int64, P, P, P]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(L, name)
            fn.restype, fn.argtypes = res, args
        _lib = L
    return _lib


def _table_rows(t: OracleTable) -> list[list]:
    rows = []
    for r in range(t.rows):
        row = []
        for c in range(t.cols):
            k = r * t.cols + c
            if not t.valid[k]:
                row.append(None)
                continue
            lo, hi = t.cells[2 * k], t.cells[2 * k + 1]
            ty = t.types[c]
            if ty in (abi.F64, abi.F32):
                row.append(float(np.array([lo], dtype=np.int64).view(np.float64)[0]))
            else:
                row.append((hi << 64) | (lo & ((1 << 64) - 1)))
        rows.append(row)
    return rows


def _rowsets(rowsets) -> C.Array:
    arr = (abi.RowSet * max(1, len(rowsets)))()
    for k, r in enumerate(rowsets):
        arr[k] = r.rs
    return arr


def aggregate(spec, rowsets, lanes: int = 1) -> list[list]:
    t = OracleTable()
    err = C.create_string_buffer(512)
    arr = _rowsets(rowsets)
    if lib().oracle_aggregate(C.byref(spec.struct), arr, len(rowsets), lanes, C.byref(t), err, 512) != 0:
        raise RuntimeError(err.value.decode())
    try:
        return _table_rows(t)
    finally:
        lib().oracle_table_free(C.byref(t))


def join_aggregate(jspec, aspec, build_rowsets, probe_rowsets) -> list[list]:
    t = OracleTable()
    err = C.create_string_buffer(512)
    b = _rowsets(build_rowsets)
    p = _rowsets(probe_rowsets)
    if lib().oracle_join_aggregate(C.byref(jspec.struct), C.byref(aspec.struct), b, len(build_rowsets), p,
                                   len(probe_rowsets), 1, C.byref(t), err, 512) != 0:
        raise RuntimeError(err.value.decode())
    try:
        return _table_rows(t)
    finally:
        lib().oracle_table_free(C.byref(t))


def row_join(jspec, build_rowsets, probe_rowset) -> np.ndarray:
    err = C.create_string_buffer(512)
    b = _rowsets(build_rowsets)
    n = lib().oracle_row_join(C.byref(jspec.struct), b, len(build_rowsets), probe_rowset.ptr, None, 0, err, 512)
    if n < 0:
        raise RuntimeError(err.value.decode())
    pairs = np.zeros(max(1, 2 * n), dtype=np.int64)
    lib().oracle_row_join(C.byref(jspec.struct), b, len(build_rowsets), probe_rowset.ptr, pairs.ctypes.data, n, err,
                          512)
    return pairs[: 2 * n].reshape(n, 2)


def row_join_typed(jspec, build_rowsets, probe_rowsets) -> np.ndarray:
    """Pairs of any served join type, in the engine's order: (probe batch << 32
    | probe row, or -1; build row over the concatenated build batches, or -1)."""
    err = C.create_string_buffer(512)
    b = _rowsets(build_rowsets)
    p = _rowsets(probe_rowsets)
    args = (C.byref(jspec.struct), b, len(build_rowsets), p, len(probe_rowsets))
    n = lib().oracle_row_join_typed(*args, None, 0, err, 512)
    if n < 0:
        raise RuntimeError(err.value.decode())
    pairs = np.zeros(max(1, 2 * n), dtype=np.int64)
    lib().oracle_row_join_typed(*args, pairs.ctypes.data, n, err, 512)
    return pairs[: 2 * n].reshape(n, 2)


def filter_rows(columns, eb, predicate, rowset) -> np.ndarray:
    from qumirdb_b200 import coltypes
    ct = coltypes(columns)
    nodes = eb.array()
    sel = np.zeros(max(1, rowset.rs.RowCount), dtype=np.uint8)
    err = C.create_string_buffer(512)
    if lib().oracle_filter(len(columns), C.cast(ct, C.c_void_p), len(eb.nodes), C.cast(nodes, C.c_void_p),
                           predicate, rowset.ptr, sel.ctypes.data, err, 512) != 0:
        raise RuntimeError(err.value.decode())
    return sel[: rowset.rs.RowCount]


def hash_rows(columns, keys, rowset) -> np.ndarray:
    from qumirdb_b200 import coltypes, i32s
    ct = coltypes(columns)
    k = i32s(keys)
    out = np.zeros(max(1, rowset.rs.RowCount), dtype=np.uint64)
    err = C.create_string_buffer(512)
    if lib().oracle_hash(len(columns), C.cast(ct, C.c_void_p), len(keys), C.cast(k, C.c_void_p), rowset.ptr,
                         out.ctypes.data, err, 512) != 0:
        raise RuntimeError(err.value.decode())
    return out[: rowset.rs.RowCount]


def sort(spec, store_rowsets, row_ids: np.ndarray, descs=None, nulls_firsts=None) -> np.ndarray:
    ids = np.ascontiguousarray(row_ids, dtype=np.int64).copy()
    store = _rowsets(store_rowsets)
    err = C.create_string_buffer(512)
    d = None if descs is None else np.asarray(descs, dtype=np.bool_)
    nf = None if nulls_firsts is None else np.asarray(nulls_firsts, dtype=np.bool_)
    if lib().oracle_sort(C.byref(spec.struct), store, ids.ctypes.data, len(ids),
                         None if d is None else d.ctypes.data, None if nf is None else nf.ctypes.data, err, 512) != 0:
        raise RuntimeError(err.value.decode())
    return ids


def top_k(spec, store_rowsets, row_ids: np.ndarray, limit: int, descs=None, nulls_firsts=None) -> np.ndarray:
    ids = np.ascontiguousarray(row_ids, dtype=np.int64).copy()
    store = _rowsets(store_rowsets)
    d = None if descs is None else np.asarray(descs, dtype=np.bool_)
    nf = None if nulls_firsts is None else np.asarray(nulls_firsts, dtype=np.bool_)
    k = lib().oracle_top_k(C.byref(spec.struct), store, ids.ctypes.data, len(ids), limit,
                           None if d is None else d.ctypes.data, None if nf is None else nf.ctypes.data)
    return ids[:k]


def _table_arrays(t: OracleTable) -> tuple[list[np.ndarray], list[np.ndarray]]:
    """Columns of an oracle table as numpy arrays: int64 for integers (object
    for 128-bit decimals), float64 for doubles, and a validity array each."""
    n, m = t.rows, t.cols
    if n == 0:
        return [np.zeros(0, np.int64) for _ in range(m)], [np.zeros(0, bool) for _ in range(m)]
    cells = np.ctypeslib.as_array(t.cells, shape=(n * m * 2,)).reshape(n, m, 2).copy()
    valid = np.ctypeslib.as_array(t.valid, shape=(n * m,)).reshape(n, m).astype(bool)
    values = []
    for c in range(m):
        ty = t.types[c]
        lo = cells[:, c, 0]
        if ty in (abi.F64, abi.F32):
            values.append(lo.view(np.float64))
        elif ty == abi.DECIMAL128:
            hi = cells[:, c, 1]
            values.append(np.array([(int(h) << 64) | (int(x) & ((1 << 64) - 1)) for x, h in zip(lo, hi)], dtype=object))
        else:
            values.append(lo)
    return values, [valid[:, c].copy() for c in range(m)]


def aggregate_arrays(spec, rowsets, lanes: int = 1) -> tuple[list[np.ndarray], list[np.ndarray]]:
    """oracle_aggregate with the result as numpy columns (for large tables)."""
    t = OracleTable()
    err = C.create_string_buffer(512)
    arr = _rowsets(rowsets)
    if lib().oracle_aggregate(C.byref(spec.struct), arr, len(rowsets), lanes, C.byref(t), err, 512) != 0:
        raise RuntimeError(err.value.decode())
    try:
        return _table_arrays(t)
    finally:
        lib().oracle_table_free(C.byref(t))


def sorted_row_indices(k1: np.ndarray, k2: np.ndarray, threads: int) -> np.ndarray:
    """Row indices in the stable order ORDER BY k1 DESC, k2 ASC (ties in
    input order) by the threaded LSD + k-way merge plan."""
    n = len(k1)
    out = np.empty(n, np.int64)
    lib().oracle_bench_sort(k1.ctypes.data, k2.ctypes.data, n, threads, out.ctypes.data)
    return out


class HostStorage:
    """The runtime filter's storage protocol over host arrays, with the
    oracle's rf_build / rf_publish / rf_probe / rf_merge: the same host logic
    (qumirdb_b200.rfilter) then drives the CPU restatement."""

    def alloc(self, nbytes: int) -> np.ndarray:
        return np.zeros(max(8, nbytes), dtype=np.uint8)

    @staticmethod
    def ptr(buf) -> int:
        return buf.ctypes.data

    def zero(self, buf, nbytes: int) -> None:
        buf[:nbytes] = 0

    def copy(self, dst, src, nbytes: int) -> None:
        dst[:nbytes] = src[:nbytes]

    def read_u64(self, buf, n: int) -> np.ndarray:
        return buf[: 8 * n].view(np.uint64).copy()

    def upload(self, arr: np.ndarray) -> np.ndarray:
        buf = self.alloc(arr.nbytes)
        buf[: arr.nbytes] = np.ascontiguousarray(arr).view(np.uint8)
        return buf

    def read_u8(self, buf, n: int) -> np.ndarray:
        return buf[:n].copy()

    def build(self, state, hashes, sel, n) -> int:
        return lib().oracle_rf_build(C.byref(state), hashes, sel, n)

    def publish(self, state, partials, n) -> int:
        return lib().oracle_rf_publish(C.byref(state), partials, n)

    def probe(self, data, hashes, sel, out, n) -> int:
        return lib().oracle_rf_probe(C.byref(data), hashes, sel, out, n)

    def merge(self, target, source, n) -> None:
        lib().oracle_rf_merge(target, source, n)

    def error(self) -> str:
        return "oracle"


def mt19937_64(seed: int, n: int) -> np.ndarray:
    """std::mt19937_64(seed)'s first n outputs."""
    out = np.zeros(max(1, n), dtype=np.uint64)
    lib().oracle_mt19937_64(seed, n, out.ctypes.data)
    return out[:n]


def route(hashes: np.ndarray, selection, routes, n_outputs: int) -> np.ndarray | None:
    """The shuffle's output per row (-1: unselected); None when a row's
    partition is routed nowhere."""
    h = np.ascontiguousarray(hashes, dtype=np.uint64)
    n = len(h)
    dest = np.zeros(max(1, n), dtype=np.int64)
    sel = None if selection is None else np.ascontiguousarray(selection, dtype=np.uint8)
    r = None if not routes else np.ascontiguousarray(routes, dtype=np.int64)
    rc = lib().oracle_route(h.ctypes.data, None if sel is None else sel.ctypes.data, n,
                            None if r is None else r.ctypes.data, 0 if r is None else len(r), n_outputs,
                            dest.ctypes.data)
    return None if rc < 0 else dest[:n]


def string_hash(b: bytes) -> int:
    """qdb_string_hash_bytes of one string (the oracle's restatement)."""
    buf = C.create_string_buffer(b, len(b)) if b else None
    return int(lib().oracle_string_hash(buf, len(b)))


def string_secret() -> bytes:
    """The engine's 136-byte XXH3 secret for strings above 16 bytes."""
    return C.string_at(lib().oracle_string_secret(), 136)
