"""The aggregate entry point that allocates no device memory.

It serves callers that cannot allocate device memory while a query runs (a
fixed memory budget handed over up front, work recorded into a CUDA graph,
an allocator owned by another runtime): table and scratch come from a fixed
device array inside the library, inputs and outputs from the caller.  These
tests call it through the C ABI twice in a row and compare each result with
the regular agg_dispatch / agg_finish_rowset path on the same inputs.
"""
import ctypes as C

import numpy as np
import pytest

import qumirdb_b200 as q
from qumirdb_b200 import abi, queries

from .helpers import assert_same_groups, gpu_rows, lineitem, zipf_data

pytestmark = pytest.mark.gpu


def regular(spec, rowset):
    prog = q.compile_aggregate(spec)
    agg = q.Aggregate(prog)
    agg.add(rowset)
    out = agg.finish()
    try:
        return out.RowCount, out
    finally:
        pass


def run_noalloc(prog, drs, types, capacity):
    bufs = []
    cols = (abi.Column * len(types))()
    for k, t in enumerate(types):
        d = q.DeviceBuffer(capacity * abi.WIDTH[t])
        m = q.DeviceBuffer(((capacity + 31) // 32) * 4)
        bufs += [d, m]
        cols[k].Data = d.ptr
        cols[k].Mask = m.ptr
    n = q.lib().qdb_gpu_agg_run_noalloc(prog.handle, drs.ptr, cols, capacity)
    if n < 0:
        raise q.QdbError(q.last_error())
    rows = []
    host = []
    for k, t in enumerate(types):
        raw = bufs[2 * k].download(np.uint8, n * abi.WIDTH[t])
        bits = np.unpackbits(bufs[2 * k + 1].download(np.uint8, ((capacity + 31) // 32) * 4),
                             bitorder="little")[:n].astype(bool)
        host.append((raw, bits))
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
    for b in bufs:
        b.free()
    return rows


def test_noalloc_matches_the_regular_path_twice_in_a_row():
    cols = lineitem(200_000, seed=21)
    spec = queries.lineitem_agg(int(cols[6].max()) - 90)
    prog = q.compile_aggregate(spec)
    drs = q.DeviceRowSet(cols)
    _, out = regular(spec, drs)
    want = gpu_rows(out, queries.LINEITEM_OUT_TYPES)
    q.release(out)
    for _ in range(2):
        got = run_noalloc(prog, drs, queries.LINEITEM_OUT_TYPES, capacity=64)
        assert_same_groups(got, want, queries.LINEITEM_OUT_TYPES, nkeys=2)


def test_noalloc_many_groups_twice_in_a_row():
    cols = zipf_data(300_000, 40_000, seed=22)
    spec = queries.zipf_agg()
    prog = q.compile_aggregate(spec)
    drs = q.DeviceRowSet(cols)
    _, out = regular(spec, drs)
    want = gpu_rows(out, queries.ZIPF_OUT_TYPES)
    q.release(out)
    for _ in range(2):
        got = run_noalloc(prog, drs, queries.ZIPF_OUT_TYPES, capacity=len(want))
        assert_same_groups(got, want, queries.ZIPF_OUT_TYPES, nkeys=1)


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
