"""The aggregate entry point that allocates no device memory.

Some callers of this library cannot allocate device memory while a query
runs: an engine that hands the GPU a fixed memory budget up front and must
not go past it mid-query, or a process whose device allocator belongs to
another runtime.  qdb_gpu_agg_run_noalloc serves them: its table and scratch
come from a fixed device array inside the library, and inputs and outputs
from the caller.  These tests call it through the C ABI twice in a row and
compare each result with the regular agg_dispatch / agg_finish_rowset path
on the same inputs and with the oracle, including a keyless aggregate,
one-byte string keys written with their offsets, and the group limit of the
fixed table from both sides.  This file runs last, after every other test.
"""
import ctypes as C

import numpy as np
import pytest

import qumirdb_b200 as q
from oracle import oracle as O
from qumirdb_b200 import abi, queries

from .helpers import assert_same_groups, gpu_rows, lineitem, zipf_data

pytestmark = pytest.mark.gpu


def regular(spec, rowset):
    prog = q.compile_aggregate(spec)
    agg = q.Aggregate(prog)
    agg.add(rowset)
    out = agg.finish()
    try:
        return gpu_rows(out, _types(spec))
    finally:
        q.release(out)


def _types(spec):
    return spec.out_types


def run_noalloc(prog, drs, types, capacity, with_offsets=False):
    """Calls the entry point with caller-owned device outputs; returns the
    rows and, per one-byte string column given offsets, those offsets."""
    bufs = []
    offs = {}
    cols = (abi.Column * len(types))()
    words = (capacity + 31) // 32
    for k, t in enumerate(types):
        d = q.DeviceBuffer(capacity * abi.WIDTH[t])
        m = q.DeviceBuffer(words * 4)
        bufs += [d, m]
        cols[k].Data = d.ptr
        cols[k].Mask = m.ptr
        if with_offsets and t == abi.CHAR1:
            o = q.DeviceBuffer((capacity + 1) * 4)
            offs[k] = o
            cols[k].Offsets = o.ptr
            cols[k].OffsetWidth = 4
    n = q.lib().qdb_gpu_agg_run_noalloc(prog.handle, drs.ptr, cols, capacity)
    if n < 0:
        raise q.QdbError(q.last_error())
    host = []
    for k, t in enumerate(types):
        raw = bufs[2 * k].download(np.uint8, n * abi.WIDTH[t])
        bits = np.unpackbits(bufs[2 * k + 1].download(np.uint8, words * 4), bitorder="little").astype(bool)
        # Words past the last one holding a group stay clear (the mask is
        # cleared first; bits after the count inside that word are unspecified).
        assert not bits[(n + 31) // 32 * 32:].any()
        host.append((raw, bits[:n]))
    rows = []
    for r in range(n):
        row = []
        for k, t in enumerate(types):
            raw, bits = host[k]
            w = abi.WIDTH[t]
            cell = raw[r * w:(r + 1) * w]
            if not bits[r]:
                row.append(None)
            elif t == abi.F64:
                row.append(float(cell.view(np.float64)[0]))
            elif t == abi.DECIMAL128:
                lo, hi = (int(x) for x in cell.view(np.uint64))
                v = lo | (hi << 64)
                row.append(v - (1 << 128) if v >= (1 << 127) else v)
            elif t == abi.CHAR1:
                row.append(int(cell[0]))
            else:
                row.append(int(cell.view({4: np.int32, 8: np.int64}[w])[0]))
        rows.append(row)
    offsets = {k: o.download(np.int32, n + 1) for k, o in offs.items()}
    for b in bufs + list(offs.values()):
        b.free()
    return rows, offsets


def test_noalloc_lineitem_matches_regular_path_and_oracle_twice_in_a_row():
    cols = lineitem(200_000, seed=21)
    spec = queries.lineitem_agg(int(cols[6].max()) - 90)
    spec.out_types = queries.LINEITEM_OUT_TYPES
    prog = q.compile_aggregate(spec)
    drs = q.DeviceRowSet(cols)
    want = regular(spec, drs)
    oracle = O.aggregate(spec, [q.HostRowSet(cols)])
    assert_same_groups(want, oracle, queries.LINEITEM_OUT_TYPES, nkeys=2)
    for _ in range(2):
        got, offsets = run_noalloc(prog, drs, queries.LINEITEM_OUT_TYPES, capacity=64, with_offsets=True)
        assert_same_groups(got, want, queries.LINEITEM_OUT_TYPES, nkeys=2)
        assert_same_groups(got, oracle, queries.LINEITEM_OUT_TYPES, nkeys=2)
        # One-byte string keys: offsets 0, 1, ..., n over the written codes.
        assert sorted(offsets) == [0, 1]
        for o in offsets.values():
            np.testing.assert_array_equal(o, np.arange(len(got) + 1, dtype=np.int32))


def test_noalloc_many_groups_twice_in_a_row():
    cols = zipf_data(300_000, 40_000, seed=22)
    spec = queries.zipf_agg()
    spec.out_types = queries.ZIPF_OUT_TYPES
    prog = q.compile_aggregate(spec)
    drs = q.DeviceRowSet(cols)
    want = regular(spec, drs)
    oracle = O.aggregate(spec, [q.HostRowSet(cols)])
    for _ in range(2):
        got, _ = run_noalloc(prog, drs, queries.ZIPF_OUT_TYPES, capacity=len(want))
        assert_same_groups(got, want, queries.ZIPF_OUT_TYPES, nkeys=1)
        assert_same_groups(got, oracle, queries.ZIPF_OUT_TYPES, nkeys=1)


def test_noalloc_keyless_aggregate_twice_in_a_row():
    """No GROUP BY: one group exists before any row, also when the filter
    passes none (COUNT 0, SUM NULL)."""
    cols = zipf_data(100_000, 5_000, seed=24)
    types = [abi.I64, abi.I64, abi.I64, abi.F64]
    for cut in (0, -10**7):
        e = q.ExprBuilder()
        a, x = e.col(1, abi.I64), e.col(2, abi.F64)
        pred = e.op(abi.LT, abi.BOOL, a, e.const(cut, abi.I64))
        spec = queries.AggSpec(queries.ZIPF_COLUMNS, e, pred, [],
                               [(abi.COUNT_STAR, -1), (abi.SUM, a), (abi.MIN, a), (abi.SUM, x)])
        spec.out_types = types
        prog = q.compile_aggregate(spec)
        drs = q.DeviceRowSet(cols)
        want = regular(spec, drs)
        oracle = O.aggregate(spec, [q.HostRowSet(cols)])
        assert len(oracle) == 1
        if cut < -10**6:
            assert oracle == [[0, None, None, None]]
        for _ in range(2):
            got, _ = run_noalloc(prog, drs, types, capacity=4)
            assert_same_groups(got, want, types, nkeys=0)
            assert_same_groups(got, oracle, types, nkeys=0)


def _distinct_keys(groups, rows, seed):
    rng = np.random.default_rng(seed)
    key = np.concatenate([np.arange(groups, dtype=np.int64) * 7919 - 12345,
                          rng.integers(0, groups, rows - groups) * 7919 - 12345])
    rng.shuffle(key)
    a = rng.integers(-10**6, 10**6, rows).astype(np.int64)
    x = rng.random(rows)
    return [key, a, x]


def test_noalloc_group_limit_from_both_sides():
    """The fixed table of the zipf aggregate (five state words) holds 2^17
    groups: exactly that many succeed, one more is refused with the limit in
    the message, and a call after the refusal is correct again."""
    limit = 1 << 17
    spec = queries.zipf_agg()
    spec.out_types = queries.ZIPF_OUT_TYPES
    prog = q.compile_aggregate(spec)
    ok = _distinct_keys(limit, limit + 50_000, seed=25)
    drs = q.DeviceRowSet(ok)
    got, _ = run_noalloc(prog, drs, queries.ZIPF_OUT_TYPES, capacity=limit)
    assert len(got) == limit
    assert_same_groups(got, O.aggregate(spec, [q.HostRowSet(ok)], lanes=8), queries.ZIPF_OUT_TYPES, nkeys=1)
    over = _distinct_keys(limit + 1, limit + 50_000, seed=26)
    with pytest.raises(q.QdbError, match=str(limit)):
        run_noalloc(prog, q.DeviceRowSet(over), queries.ZIPF_OUT_TYPES, capacity=limit + 1)
    again, _ = run_noalloc(prog, drs, queries.ZIPF_OUT_TYPES, capacity=limit)
    assert_same_groups(again, got, queries.ZIPF_OUT_TYPES, nkeys=1)


def test_noalloc_rejects_what_does_not_fit():
    cols = zipf_data(50_000, 20_000, seed=23)
    prog = q.compile_aggregate(queries.zipf_agg())
    drs = q.DeviceRowSet(cols)
    with pytest.raises(q.QdbError, match="output capacity"):
        run_noalloc(prog, drs, queries.ZIPF_OUT_TYPES, capacity=10)
    host = q.HostRowSet(cols)
    empty = (abi.Column * 6)()
    assert q.lib().qdb_gpu_agg_run_noalloc(prog.handle, host.ptr, empty, 10) == -1
    assert "device memory" in q.last_error()
    # A mask that is not 4-byte aligned is refused before anything is written.
    bufs = [q.DeviceBuffer(64 * 8) for _ in range(6)]
    mask = q.DeviceBuffer(64)
    cols_out = (abi.Column * 6)()
    for k, b in enumerate(bufs):
        cols_out[k].Data = b.ptr
    cols_out[0].Mask = mask.ptr + 1
    assert q.lib().qdb_gpu_agg_run_noalloc(prog.handle, drs.ptr, cols_out, 64) == -1
    assert "aligned" in q.last_error()
