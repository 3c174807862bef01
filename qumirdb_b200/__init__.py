"""qumirdb_b200 — B200 (sm_100a) execution hot path of QumirDB behind its C ABI.

Python host side: loads libqdb_gpu.so (built in-tree by qumirdb_b200/build.py),
builds expression/operator descriptors, and drives the reference-shaped entry
points the way the engine's processors do (TAggregateProcessor,
qdb/exec/aggregate_exec.cpp:70-136; TRowJoinProcessor,
qdb/exec/row_join_exec.cpp:93-220; TSortProcessor,
qdb/exec/sort_exec.cpp:393-490).  There is no CPU execution path here: a
missing library or a device error raises.
"""
from __future__ import annotations

import ctypes as C
import threading
from pathlib import Path

import numpy as np

from . import abi
from .abi import *  # noqa: F401,F403

_HERE = Path(__file__).resolve().parent
LIB_PATH = _HERE / "libqdb_gpu.so"
HEADER = _HERE.parent / "include" / "qdb_gpu.h"

_lib = None
_lock = threading.Lock()
_initialised: set[int] = set()


class QdbError(RuntimeError):
    pass


def lib() -> C.CDLL:
    """The device library; raises if it has not been built."""
    global _lib
    with _lock:
        if _lib is None:
            if not LIB_PATH.exists():
                raise QdbError(f"{LIB_PATH} is missing: run qumirdb_b200/build.py (or __graft_entry__.build())")
            _lib = abi.bind(C.CDLL(str(LIB_PATH)))
        return _lib


def last_error() -> str:
    return lib().qdb_gpu_last_error().decode()


def init(device: int = 0) -> None:
    """Binds the calling thread to `device` (creates the CUDA context)."""
    if lib().qdb_gpu_init(device) != 0:
        raise QdbError(f"qdb_gpu_init({device}) failed: {last_error()}")
    _initialised.add(threading.get_ident())


def _ensure_init() -> None:
    if threading.get_ident() not in _initialised:
        init(0)


# ---------------------------------------------------------------------------
# Expressions.
# ---------------------------------------------------------------------------
class ExprBuilder:
    """Flat expression node array (operands before their users)."""

    def __init__(self) -> None:
        self.nodes: list[tuple] = []
        self._lists: list = []

    def _add(self, op, type_, scale=0, column=0, args=(0, 0, 0), imm_lo=0, imm_hi=0, lst=None) -> int:
        self.nodes.append((op, type_, scale, column, tuple(args) + (0,) * (3 - len(args)), imm_lo, imm_hi, lst))
        return len(self.nodes) - 1

    def col(self, c: int, type_: int, scale: int = 0) -> int:
        return self._add(abi.COLUMN, type_, scale, column=c)

    def const(self, v, type_: int, scale: int = 0) -> int:
        if type_ in (abi.F64, abi.F32):
            bits = int(np.array([float(v)], dtype=np.float64).view(np.int64)[0])
            return self._add(abi.CONST, type_, scale, imm_lo=bits)
        v = int(v)
        lo = v & ((1 << 64) - 1)
        hi = (v >> 64) & ((1 << 64) - 1)
        to_s = lambda u: u - (1 << 64) if u >= (1 << 63) else u  # noqa: E731
        return self._add(abi.CONST, type_, scale, imm_lo=to_s(lo), imm_hi=to_s(hi))

    def null(self, type_: int = abi.I64) -> int:
        return self._add(abi.NULL, type_)

    def op(self, op: int, type_: int, *args: int, scale: int = 0) -> int:
        return self._add(op, type_, scale, args=args)

    def in_list(self, a: int, values, type_: int = abi.BOOL) -> int:
        arr = (C.c_int64 * len(values))(*[int(x) for x in values])
        self._lists.append(arr)
        idx = self._add(abi.IN_LIST, type_, 0, args=(a,), lst=arr)
        return idx

    def array(self):
        arr = (abi.Expr * max(1, len(self.nodes)))()
        for k, (op, t, s, c, args, lo, hi, lst) in enumerate(self.nodes):
            e = arr[k]
            e.op, e.type, e.scale, e.column = op, t, s, c
            e.args[0], e.args[1], e.args[2] = args
            e.imm_lo, e.imm_hi = lo, hi
            if lst is not None:
                e.list_len = len(lst)
                e.list = C.cast(lst, C.POINTER(C.c_int64))
        return arr


def coltypes(types) -> C.Array:
    """[(type, scale, nullable)] -> qdb_column_type array."""
    arr = (abi.ColumnType * max(1, len(types)))()
    for k, t in enumerate(types):
        t = (tuple(t) + (0, 0))[:3]
        arr[k].type, arr[k].scale, arr[k].nullable = t[0], t[1], t[2]
        arr[k].precision = 38 if t[0] == abi.DECIMAL128 else (18 if t[0] == abi.DECIMAL64 else 0)
    return arr


def i32s(vals) -> C.Array:
    return (C.c_int32 * max(1, len(vals)))(*vals)


# ---------------------------------------------------------------------------
# Row sets.
# ---------------------------------------------------------------------------
def _bitmap(valid: np.ndarray) -> np.ndarray:
    return np.packbits(valid.astype(np.uint8), bitorder="little")


class StringColumn:
    """A QDB_TYPE_STRING column in Arrow's layout: row r is
    data[offsets[r]:offsets[r + 1]], offsets int32 (utf8) or int64
    (large_utf8)."""

    def __init__(self, offsets, data):
        self.offsets = np.ascontiguousarray(offsets)
        if self.offsets.dtype not in (np.int32, np.int64):
            raise ValueError("string offsets must be int32 or int64")
        self.data = np.ascontiguousarray(data, dtype=np.uint8)

    @classmethod
    def of(cls, values, large: bool = False) -> "StringColumn":
        bs = [v if isinstance(v, bytes) else str(v).encode() for v in values]
        off = np.zeros(len(bs) + 1, np.int64 if large else np.int32)
        np.cumsum([len(b) for b in bs], out=off[1:])
        return cls(off, np.frombuffer(b"".join(bs), np.uint8).copy())

    def __len__(self) -> int:
        return len(self.offsets) - 1


def _host_column(col: "abi.Column", a) -> None:
    if isinstance(a, StringColumn):
        col.Data = a.data.ctypes.data if a.data.size else None
        col.Offsets = a.offsets.ctypes.data
        col.OffsetWidth = a.offsets.itemsize
    else:
        col.Data = a.ctypes.data if a.size else None


class HostRowSet:
    """A TRowSet over host numpy columns (kept alive by this object);
    string columns are StringColumn."""

    def __init__(self, columns, masks=None, selection=None, rows=None):
        self.arrays = [c if isinstance(c, StringColumn) else np.ascontiguousarray(c) for c in columns]
        n = rows if rows is not None else (len(self.arrays[0]) if self.arrays else 0)
        self.masks = [None if m is None else _bitmap(np.asarray(m, dtype=bool)) for m in (masks or [None] * len(columns))]
        self.selection = None if selection is None else np.ascontiguousarray(selection, dtype=np.uint8)
        self.cols = (abi.Column * max(1, len(self.arrays)))()
        for k, a in enumerate(self.arrays):
            _host_column(self.cols[k], a)
            if self.masks[k] is not None:
                self.cols[k].Mask = self.masks[k].ctypes.data
        self.rs = abi.RowSet()
        self.rs.Columns = self.cols
        self.rs.ColumnCount = len(self.arrays)
        self.rs.RowCount = n
        self.rs.Selection = None if self.selection is None else self.selection.ctypes.data
        self.rs.RefCount = 1

    @property
    def ptr(self):
        return C.byref(self.rs)


class DeviceBuffer:
    def __init__(self, nbytes: int):
        _ensure_init()
        self.nbytes = nbytes
        self.ptr = lib().qdb_gpu_alloc(max(16, nbytes))
        if not self.ptr:
            raise QdbError(f"device allocation failed: {last_error()}")

    def upload(self, host: np.ndarray, stream_sync: bool = True) -> "DeviceBuffer":
        host = np.ascontiguousarray(host)
        if lib().qdb_gpu_memcpy(self.ptr, host.ctypes.data, host.nbytes) != 0:
            raise QdbError(last_error())
        if stream_sync:
            synchronize()
        return self

    def download(self, dtype, count: int) -> np.ndarray:
        out = np.empty(count, dtype=dtype)
        if count and lib().qdb_gpu_memcpy(out.ctypes.data, self.ptr, out.nbytes) != 0:
            raise QdbError(last_error())
        synchronize()
        return out

    def free(self) -> None:
        if self.ptr:
            lib().qdb_gpu_free(self.ptr)
            self.ptr = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


def synchronize() -> None:
    if lib().qdb_gpu_synchronize() != 0:
        raise QdbError(last_error())


class DeviceRowSet:
    """A TRowSet whose columns live in HBM (the resident column cache)."""

    def __init__(self, columns, masks=None, selection=None, rows=None):
        host = HostRowSet(columns, masks, selection, rows)
        self.rows = host.rs.RowCount
        self.widths = [0 if isinstance(a, StringColumn) else a.dtype.itemsize for a in host.arrays]
        self.bufs = []
        self.cols = (abi.Column * max(1, len(host.arrays)))()
        for k, a in enumerate(host.arrays):
            if isinstance(a, StringColumn):
                ob = DeviceBuffer(a.offsets.nbytes).upload(a.offsets, stream_sync=False)
                db = DeviceBuffer(a.data.nbytes).upload(a.data, stream_sync=False)
                self.bufs += [ob, db]
                self.cols[k].Data = db.ptr
                self.cols[k].Offsets = ob.ptr
                self.cols[k].OffsetWidth = a.offsets.itemsize
            else:
                b = DeviceBuffer(a.nbytes).upload(a, stream_sync=False)
                self.bufs.append(b)
                self.cols[k].Data = b.ptr
            if host.masks[k] is not None:
                mb = DeviceBuffer(host.masks[k].nbytes).upload(host.masks[k], stream_sync=False)
                self.bufs.append(mb)
                self.cols[k].Mask = mb.ptr
        self.rs = abi.RowSet()
        self.rs.Columns = self.cols
        self.rs.ColumnCount = len(host.arrays)
        self.rs.RowCount = self.rows
        if host.selection is not None:
            sb = DeviceBuffer(host.selection.nbytes).upload(host.selection, stream_sync=False)
            self.bufs.append(sb)
            self.rs.Selection = sb.ptr
        self.rs.RefCount = 1
        synchronize()

    @property
    def ptr(self):
        return C.byref(self.rs)


class SliceRowSet:
    """Rows [lo, hi) of a DeviceRowSet as a row set of its own, without a
    copy: the column pointers move by lo values, validity by lo bits."""

    def __init__(self, base: "DeviceRowSet", lo: int, hi: int):
        self.base = base
        src = base.rs
        n = src.ColumnCount
        self.cols = (abi.Column * max(1, n))()
        for k in range(n):
            c = src.Columns[k]
            d = self.cols[k]
            d.Data = (c.Data or 0) + lo * base.widths[k]
            if c.Mask:
                d.Mask = c.Mask
                d.MaskBitOffset = c.MaskBitOffset + lo
        self.rs = abi.RowSet()
        self.rs.Columns = self.cols
        self.rs.ColumnCount = n
        self.rs.RowCount = hi - lo
        if src.Selection:
            self.rs.Selection = src.Selection + lo
        self.rs.RefCount = 1

    @property
    def ptr(self):
        return C.byref(self.rs)


def _fetch(ptr, nbytes: int, on_device: bool) -> np.ndarray:
    if nbytes <= 0:
        return np.zeros(0, np.uint8)
    if on_device:
        out = np.empty(nbytes, np.uint8)
        if lib().qdb_gpu_memcpy(out.ctypes.data, ptr, nbytes) != 0:
            raise QdbError(last_error())
        synchronize()
        return out
    return np.ctypeslib.as_array(C.cast(ptr, C.POINTER(C.c_uint8)), shape=(nbytes,)).copy()


def read_rowset(rs: abi.RowSet, types, on_device: bool = False) -> tuple[list[np.ndarray], list[np.ndarray]]:
    """Output row set -> (values, validity) numpy columns by qdb type; with
    on_device the row set's buffers are in device memory (QDB_OUT_DEVICE)."""
    n = rs.RowCount
    values, valid = [], []
    for k, t in enumerate(types):
        col = rs.Columns[k]
        w = abi.WIDTH[t]
        raw = _fetch(col.Data, n * w, on_device)
        if t == abi.DECIMAL128:
            words = raw.view(np.uint64).reshape(n, 2)
            vals = np.array([int(lo) | (int(hi) << 64) for lo, hi in words], dtype=object)
            vals = np.array([v - (1 << 128) if v >= (1 << 127) else v for v in vals], dtype=object)
        else:
            dt = {abi.I8: np.int8, abi.I16: np.int16, abi.I32: np.int32, abi.I64: np.int64, abi.U8: np.uint8,
                  abi.U16: np.uint16, abi.U32: np.uint32, abi.U64: np.uint64, abi.F32: np.float32,
                  abi.F64: np.float64, abi.DATE32: np.int32, abi.DECIMAL64: np.int64, abi.CHAR1: np.uint8,
                  abi.BOOL: np.uint8}[t]
            vals = raw.view(dt)
        values.append(vals)
        if col.Mask and n:
            off = col.MaskBitOffset
            bits = _fetch(col.Mask, (off + n + 7) // 8, on_device)
            valid.append(np.unpackbits(bits, bitorder="little")[off:off + n].astype(bool))
        else:
            valid.append(np.ones(n, dtype=bool))
    return values, valid


def release(rs: abi.RowSet) -> None:
    if rs.Destroy:
        rs.Destroy(C.byref(rs))


# ---------------------------------------------------------------------------
# Programs and processors.
# ---------------------------------------------------------------------------
class Program:
    def __init__(self, handle, keep=()):
        if not handle:
            raise QdbError(f"compile failed: {last_error()}")
        self.handle = handle
        self._keep = keep

    def __del__(self):
        try:
            if self.handle:
                lib().qdb_gpu_program_destroy(self.handle)
        except Exception:
            pass


def compile_aggregate(spec) -> Program:
    err = C.create_string_buffer(512)
    h = lib().qdb_gpu_compile_aggregate(C.byref(spec.struct), err, 512)
    if not h:
        raise QdbError(err.value.decode())
    return Program(h, keep=(spec,))


def compile_join_aggregate(jspec, aspec) -> Program:
    err = C.create_string_buffer(512)
    h = lib().qdb_gpu_compile_join_aggregate(C.byref(jspec.struct), C.byref(aspec.struct), err, 512)
    if not h:
        raise QdbError(err.value.decode())
    return Program(h, keep=(jspec, aspec))


def compile_row_join(jspec) -> Program:
    err = C.create_string_buffer(512)
    h = lib().qdb_gpu_compile_row_join(C.byref(jspec.struct), err, 512)
    if not h:
        raise QdbError(err.value.decode())
    return Program(h, keep=(jspec,))


class Aggregate:
    """The engine's TAggregateProcessor over the device table."""

    def __init__(self, prog: Program, initial_capacity: int = 8):
        _ensure_init()
        self.prog = prog
        self.ht = (C.c_uint8 * abi.HASH_TABLE_SIZE)()
        if lib().qdb_gpu_agg_dispatch(prog.handle, self.ht, None, initial_capacity, abi.AGG_INIT) == 0:
            raise QdbError(f"aggregate initialization failed: {last_error()}")

    @property
    def groups(self) -> int:
        return C.cast(self.ht, C.POINTER(C.c_int64))[9]

    def expect_groups(self, n: int) -> None:
        """The planner's group estimate (agg_dispatch ExpectRowGroups): the
        table is sized for it up front."""
        if lib().qdb_gpu_agg_dispatch(self.prog.handle, self.ht, None, n, abi.AGG_EXPECT_ROW_GROUPS) == 0:
            raise QdbError(f"aggregate ExpectRowGroups failed: {last_error()}")

    def add(self, rowset) -> int:
        r = lib().qdb_gpu_agg_dispatch(self.prog.handle, self.ht, rowset.ptr, 0, abi.AGG_UPDATE)
        if r < 0:
            raise QdbError(f"aggregate update failed: {last_error()}")
        return r

    def finish(self) -> abi.RowSet:
        out = abi.RowSet()
        n = lib().qdb_gpu_agg_finish_rowset(self.prog.handle, self.ht, C.byref(out))
        if n < 0:
            raise QdbError(f"aggregate finish failed: {last_error()}")
        return out

    def release(self) -> None:
        """Frees the device table of an aggregate that was not finished."""
        if self.ht is not None:
            lib().qdb_gpu_agg_release(self.ht)

    def __del__(self):
        try:
            self.release()
        except Exception:
            pass


class AggregateBatch:
    """Many independent aggregates of one program (the partitions of a
    partitioned GROUP BY, or small aggregations of many queries of one
    template), each updated like an Aggregate but all in one persistent
    launch (qdb_gpu_agg_dispatch_batch) and finished by one batched finalize
    (qdb_gpu_agg_finish_batch)."""

    def __init__(self, prog: Program, n: int):
        _ensure_init()
        self.prog = prog
        self.n = n
        # The n HashTable buffers side by side in one array.
        self._buf = (C.c_uint8 * (abi.HASH_TABLE_SIZE * max(n, 1)))()
        base = C.addressof(self._buf)
        self._ptrs = (C.c_void_p * max(n, 1))(*range(base, base + abi.HASH_TABLE_SIZE * n, abi.HASH_TABLE_SIZE))

    @property
    def groups(self) -> list[int]:
        words = np.frombuffer(self._buf, dtype=np.int64).reshape(max(self.n, 1), abi.HASH_TABLE_SIZE // 8)
        return words[: self.n, 9].tolist()

    def add(self, rowsets) -> None:
        """Updates aggregate i with rowsets[i] (row-set objects, or a
        RowSetPointers built once for a batch that repeats)."""
        if len(rowsets) != self.n:
            raise ValueError(f"{self.n} aggregates, {len(rowsets)} row sets")
        ptrs = rowsets.arr if isinstance(rowsets, RowSetPointers) else RowSetPointers(rowsets).arr
        if lib().qdb_gpu_agg_dispatch_batch(self.prog.handle, self._ptrs, ptrs, self.n) < 0:
            raise QdbError(f"batched aggregate update failed: {last_error()}")

    def finish(self) -> "RowSets":
        outs = (abi.RowSet * max(self.n, 1))()
        if lib().qdb_gpu_agg_finish_batch(self.prog.handle, self._ptrs, self.n, outs) < 0:
            raise QdbError(f"batched aggregate finish failed: {last_error()}")
        self._finished = True   # the states are destroyed and zeroed
        return RowSets(outs, self.n)

    def release(self) -> None:
        if getattr(self, "_finished", False):
            return
        for i in range(self.n):
            lib().qdb_gpu_agg_release(self._ptrs[i])

    def __del__(self):
        try:
            self.release()
        except Exception:
            pass


class RowSetPointers:
    """A C array of TRowSet pointers over row-set objects (kept alive)."""

    def __init__(self, rowsets):
        self.objs = list(rowsets)
        self.arr = (abi.PRS * max(1, len(self.objs)))(*[C.pointer(r.rs) for r in self.objs])

    def __len__(self) -> int:
        return len(self.objs)


class RowSets:
    """Output row sets of a batched finish: indexable like a list, released
    together by release() (one foreign call)."""

    def __init__(self, arr, n: int):
        self.arr = arr
        self.n = n

    def __len__(self) -> int:
        return self.n

    def __getitem__(self, i: int) -> abi.RowSet:
        if not -self.n <= i < self.n:
            raise IndexError(i)
        return self.arr[i % self.n]

    def __iter__(self):
        return (self.arr[i] for i in range(self.n))

    def release(self) -> None:
        lib().qdb_gpu_release_rowsets(self.arr, self.n)


def autotune_info() -> dict:
    import json
    n = lib().qdb_gpu_autotune_info(None, 0)
    buf = C.create_string_buffer(int(n) + 1)
    lib().qdb_gpu_autotune_info(buf, n + 1)
    return json.loads(buf.value.decode())


def autotune_reset() -> None:
    lib().qdb_gpu_autotune_reset()


class RowJoin:
    """The engine's TRowJoinProcessor state: arena, table, scratch, pairs,
    and for a LEFT_ANTI join the second arena of NULL-key build rows
    (qdb/exec/row_join_exec.cpp:80-220)."""

    def __init__(self, prog: Program, keeps_null_keys: bool = False):
        _ensure_init()
        self.prog = prog
        self.arena = (C.c_uint8 * abi.ROW_ARENA_SIZE)()
        self.table = (C.c_uint8 * abi.ROW_TABLE_SIZE)()
        self.scratch = (C.c_uint8 * abi.ROW_SCRATCH_SIZE)()
        self.pairs = (C.c_uint8 * abi.PAIR_BUFFER_SIZE)()
        self.null_arena = (C.c_uint8 * abi.ROW_ARENA_SIZE)() if keeps_null_keys else None
        self._op(None, abi.JR_INIT)
        if self.null_arena is not None:
            self._op(None, abi.JR_INIT, self.null_arena)

    def _op(self, batch, op, arena=None) -> None:
        ok = lib().qdb_gpu_jr_dispatch(self.prog.handle, self.arena if arena is None else arena, self.table,
                                       self.scratch, self.pairs, None if batch is None else batch.ptr, op)
        if not ok:
            raise QdbError(f"jr_dispatch({op}) failed: {last_error()}")

    def append(self, batch) -> None:
        self._op(batch, abi.JR_APPEND)
        if self.null_arena is not None:
            self._op(batch, abi.JR_APPEND_NULL_KEYS, self.null_arena)

    def emit_by_mark(self) -> int:
        """A SEMI/ANTI join's output pairs once the probe side has ended
        (TRowJoinProcessor::Finish): the arena's rows by mark, then the
        NULL-key arena's rows.  Returns the pair count."""
        C.cast(self.pairs, C.POINTER(C.c_int64))[0] = 0
        self._op(None, abi.JR_EMIT_BY_MARK)
        if self.null_arena is not None:
            self._op(None, abi.JR_EMIT_BY_MARK, self.null_arena)
        return self.pair_count

    def build(self) -> None:
        self._op(None, abi.JR_BUILD)

    def probe(self, batch) -> int:
        self._op(batch, abi.JR_PROBE)
        return self.pair_count

    @property
    def pair_count(self) -> int:
        return C.cast(self.pairs, C.POINTER(C.c_int64))[0]

    @property
    def arena_rows(self) -> int:
        return C.cast(self.arena, C.POINTER(C.c_int64))[5]

    def materialize(self, stream, start: int, limit: int) -> tuple[int, abi.RowSet]:
        out = abi.RowSet()
        n = lib().qdb_gpu_jr_materialize(self.prog.handle, self.pairs, None if stream is None else stream.ptr,
                                         start, limit, C.byref(out))
        if n < 0:
            raise QdbError(f"jr_materialize failed: {last_error()}")
        return n, out

    def probe_aggregate(self, agg: Aggregate, batch) -> int:
        n = lib().qdb_gpu_join_aggregate_probe(self.prog.handle, self.arena, self.table, agg.ht, batch.ptr)
        if n < 0:
            raise QdbError(f"join aggregate probe failed: {last_error()}")
        return n

    def release(self) -> None:
        """Frees the arena(s), table and pair buffer on the device."""
        lib().qdb_gpu_jr_release(self.arena, self.table, self.scratch, self.pairs)
        if self.null_arena is not None:
            lib().qdb_gpu_jr_release(self.null_arena, None, None, None)

    def __del__(self):
        try:
            self.release()
        except Exception:
            pass


def compile_hash(columns, key_columns) -> Program:
    """The join / shuffle key hash program (TKernelCompiler::CompileJoinHash):
    rh_hash of the key columns, as qdb_gpu_hash writes it."""
    ct = coltypes(columns)
    kc = i32s(key_columns)
    err = C.create_string_buffer(512)
    h = lib().qdb_gpu_compile_hash(len(columns), ct, len(key_columns), kc, err, 512)
    if not h:
        raise QdbError(err.value.decode())
    return Program(h, keep=(ct, kc))


def hash_rows(prog: Program, batch, out_ptr) -> None:
    """qdb_gpu_hash: one uint64 per selected row of `batch` into out_ptr
    (host or device memory)."""
    if not lib().qdb_gpu_hash(prog.handle, batch.ptr, out_ptr):
        raise QdbError(f"hash failed: {last_error()}")


def shuffle(hash_prog: Program, batch, n_outputs: int, routes=None) -> RowSets:
    """qdb_gpu_shuffle: the batch's selected rows split by key hash into
    n_outputs device-resident row sets (input order kept in each)."""
    outs = (abi.RowSet * max(1, n_outputs))()
    r = None if not routes else (C.c_int64 * len(routes))(*routes)
    n = lib().qdb_gpu_shuffle(hash_prog.handle, batch.ptr, r, 0 if r is None else len(routes), n_outputs, outs)
    if n < 0:
        raise QdbError(f"shuffle failed: {last_error()}")
    return RowSets(outs, n_outputs)


class CachedRowSet:
    """A device row set handed out by the column cache; its columns stay
    pinned in the cache until release()."""

    def __init__(self, rs: abi.RowSet, keep):
        self.rs = rs
        self._keep = keep

    @property
    def ptr(self):
        return C.byref(self.rs)

    def release(self) -> None:
        release(self.rs)

    def __del__(self):
        try:
            self.release()
        except Exception:
            pass


class ColumnCache:
    """Device column cache between scan sources and the kernels: batches of
    host columns staged into HBM and kept resident across queries under a
    byte budget (qdb_gpu_cache_*)."""

    def __init__(self, budget_bytes: int, staging_bytes: int = 0):
        _ensure_init()
        self.handle = lib().qdb_gpu_cache_create(budget_bytes, staging_bytes)
        if not self.handle:
            raise QdbError(f"column cache creation failed: {last_error()}")

    def get(self, source_id: int, batch_index: int, host, types, columns=None) -> CachedRowSet:
        ct = coltypes(types)
        cols = list(range(len(types))) if columns is None else list(columns)
        ci = i32s(cols)
        out = abi.RowSet()
        if lib().qdb_gpu_cache_get(self.handle, source_id, batch_index, host.ptr, ct, ci, len(cols), C.byref(out)) < 0:
            raise QdbError(f"column cache get failed: {last_error()}")
        return CachedRowSet(out, (ct, ci))

    def invalidate(self, source_id: int) -> int:
        return lib().qdb_gpu_cache_invalidate(self.handle, source_id)

    def stats(self) -> dict:
        st = abi.CacheStats()
        lib().qdb_gpu_cache_get_stats(self.handle, C.byref(st))
        return {f: getattr(st, f) for f, _ in abi.CacheStats._fields_}

    def close(self) -> None:
        if self.handle:
            lib().qdb_gpu_cache_destroy(self.handle)
            self.handle = None


class RowJoinBatch:
    """Many fused join-aggregates of one program (the partitions of a
    partitioned join, or the joins of many queries of one template): each
    join appends its own build rows, then every table is built in one batched
    call and every probe folded in one persistent launch."""

    def __init__(self, prog: Program, n: int):
        self.prog = prog
        self.n = n
        self.joins = [RowJoin(prog) for _ in range(n)]
        self.aggs = [Aggregate(prog) for _ in range(n)]

    def _ptrs(self, bufs):
        return (C.c_void_p * max(1, self.n))(*[C.cast(b, C.c_void_p) for b in bufs])

    def append(self, i: int, batch) -> None:
        self.joins[i].append(batch)

    def append_all(self, batches) -> None:
        """Every join's build batch at once (one device wait for all)."""
        rs = RowSetPointers(batches)
        if not lib().qdb_gpu_jr_append_batch(self.prog.handle, self._ptrs([j.arena for j in self.joins]), rs.arr,
                                             self.n):
            raise QdbError(f"batched join append failed: {last_error()}")

    def build(self) -> None:
        if not lib().qdb_gpu_jr_build_batch(self.prog.handle, self._ptrs([j.arena for j in self.joins]),
                                            self._ptrs([j.table for j in self.joins]), self.n):
            raise QdbError(f"batched join build failed: {last_error()}")

    def probe_aggregate(self, batches) -> int:
        rs = RowSetPointers(batches)
        m = lib().qdb_gpu_join_aggregate_probe_batch(self.prog.handle, self._ptrs([j.arena for j in self.joins]),
                                                      self._ptrs([j.table for j in self.joins]),
                                                      self._ptrs([a.ht for a in self.aggs]), rs.arr, self.n)
        if m < 0:
            raise QdbError(f"batched join probe failed: {last_error()}")
        return m

    def finish(self) -> "RowSets":
        """Every join's aggregate finished in one batched finalize (slices of
        shared output buffers; release each, or all with release())."""
        outs = (abi.RowSet * max(1, self.n))()
        if lib().qdb_gpu_agg_finish_batch(self.prog.handle, self._ptrs([a.ht for a in self.aggs]), self.n, outs) < 0:
            raise QdbError(f"batched join finish failed: {last_error()}")
        return RowSets(outs, self.n)

    def release(self) -> None:
        for j in self.joins:
            j.release()


def compile_sort(spec) -> Program:
    err = C.create_string_buffer(512)
    h = lib().qdb_gpu_compile_sort(C.byref(spec.struct), err, 512)
    if not h:
        raise QdbError(err.value.decode())
    return Program(h, keep=(spec,))


def rowset_array(rowsets) -> C.Array:
    """A contiguous TRowSet array (a sort store) over row-set objects."""
    arr = (abi.RowSet * max(1, len(rowsets)))()
    for k, r in enumerate(rowsets):
        arr[k] = r.rs
    return arr


class Sort:
    """TSortProcessor's kernel calls (qdb/exec/sort_exec.cpp:393-490) over a
    store of batches: qdb_sort_run and qdb_top_k_select.  Row ids are packed
    (batch << 32) | row, in a host int64 array or a DeviceBuffer."""

    def __init__(self, prog: Program, store):
        _ensure_init()
        self.prog = prog
        self.store_objs = list(store)
        self.store = rowset_array(self.store_objs)

    @staticmethod
    def _ids(row_ids):
        if isinstance(row_ids, DeviceBuffer):
            return row_ids.ptr, row_ids.nbytes // 8
        return row_ids.ctypes.data, len(row_ids)

    def sort(self, row_ids, descs=None, nulls_firsts=None, n=None) -> None:
        ptr, m = self._ids(row_ids)
        n = m if n is None else n
        d = None if descs is None else (C.c_bool * len(descs))(*descs)
        nf = None if nulls_firsts is None else (C.c_bool * len(nulls_firsts))(*nulls_firsts)
        out = abi.RowSet()
        r = lib().qdb_gpu_sort_run(self.prog.handle, self.store, ptr, None, None, n, d, nf, True, 0, 0,
                                   C.byref(out))
        if r < 0:
            raise QdbError(f"sort failed: {last_error()}")

    def materialize(self, row_ids, start: int, limit: int, n=None) -> tuple[int, abi.RowSet]:
        ptr, m = self._ids(row_ids)
        n = m if n is None else n
        out = abi.RowSet()
        r = lib().qdb_gpu_sort_run(self.prog.handle, self.store, ptr, None, None, n, None, None, False, start,
                                   limit, C.byref(out))
        if r < 0:
            raise QdbError(f"sort materialize failed: {last_error()}")
        return r, out

    def top_k(self, row_ids, limit: int, n=None) -> int:
        ptr, m = self._ids(row_ids)
        n = m if n is None else n
        k = lib().qdb_gpu_top_k_select(self.prog.handle, self.store, ptr, n, limit)
        if k < 0:
            raise QdbError(f"top-k failed: {last_error()}")
        return k


class TopSort:
    """TTopSortProcessor (qdb/exec/sort_exec.cpp:627-760) over the device:
    Add(batch) keeps the first `limit` rows of the order seen so far
    (qdb_gpu_top_sort_update), choosing top-K selection of the batch first
    when the engine's heap rule takes it (K <= 1024 and K <= rows / 4,
    sort_exec.cpp:56-65); state() is the kept rows, in order."""

    def __init__(self, prog: Program, limit: int):
        _ensure_init()
        self.prog = prog
        self.limit = limit
        self.state = abi.RowSet()
        self.calls = []

    def add(self, batch, selection=None) -> int:
        n = batch.rs.RowCount
        rows = np.arange(n, dtype=np.int64) if selection is None else np.flatnonzero(selection).astype(np.int64)
        if len(rows) == 0 or self.limit <= 0:
            return int(self.state.RowCount)
        ids = np.ascontiguousarray(rows)            # (0 << 32) | row
        sort_input = True
        m = len(ids)
        if self.limit <= 1024 and self.limit <= m // 4:
            one = rowset_array([batch])
            k = lib().qdb_gpu_top_k_select(self.prog.handle, one, ids.ctypes.data, m, self.limit)
            if k <= 0:
                raise QdbError(f"top-k failed: {last_error()}")
            m, sort_input = k, False
        cap = min(self.limit, int(self.state.RowCount) + m)
        ids = np.concatenate([ids, np.zeros(max(0, cap - len(ids)), np.int64)])
        src = np.zeros(max(cap, 1), np.uint8)
        idx = np.zeros(max(cap, 1), np.uint32)
        nxt = abi.RowSet()
        r = lib().qdb_gpu_top_sort_update(self.prog.handle, C.byref(self.state), batch.ptr, ids.ctypes.data, None,
                                          None, m, sort_input, src.ctypes.data, idx.ctypes.data, self.limit,
                                          C.byref(nxt))
        if r < 0:
            raise QdbError(f"top-sort update failed: {last_error()}")
        self.calls.append((src[:r].copy(), idx[:r].copy()))
        if r > 0:
            release(self.state)
            self.state = nxt
        return int(self.state.RowCount)

    def release(self) -> None:
        release(self.state)
        self.state = abi.RowSet()


def profile(on: bool) -> None:
    lib().qdb_gpu_profile_enable(1 if on else 0)


def profile_read(cap: int = 4096) -> list[tuple[str, float, int]]:
    buf = (abi.KernelTime * cap)()
    n = lib().qdb_gpu_profile_read(buf, cap)
    return [(buf[i].name.decode(), buf[i].ms, buf[i].units) for i in range(n)]


def launch_count(reset: bool = False) -> int:
    return lib().qdb_gpu_launch_count(1 if reset else 0)
