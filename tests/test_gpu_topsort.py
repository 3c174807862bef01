"""ORDER BY ... LIMIT K through TTopSortProcessor's kernel, qdb_top_sort_update
(TTopSortDispatch, qdb/kernel/compiler.h:570-583), against the oracle's
restatement of the same processor (qdb/exec/sort_exec.cpp:627-760): batch by
batch, the picks (state or batch row) and the kept rows must be identical,
for K above 1024 and K above rows/4 (the input is sorted on the device) and
for K that the heap rule takes (top-K selection first, then the merge)."""
import ctypes as C

import numpy as np
import pytest

import qumirdb_b200 as q
from oracle import oracle as O
from qumirdb_b200 import abi, queries

pytestmark = pytest.mark.gpu

TYPES = [abi.I64, abi.I32, abi.I64]


def batches(nb, rows, seed, nullable):
    rng = np.random.default_rng(seed)
    out = []
    for b in range(nb):
        k1 = rng.integers(-500, 500, rows).astype(np.int64)        # many ties
        k2 = rng.integers(0, 50, rows).astype(np.int32)
        rid = np.arange(b * rows, (b + 1) * rows, dtype=np.int64)
        masks = [rng.random(rows) > 0.1, None, None] if nullable else None
        out.append(([k1, k2, rid], masks))
    return out


def oracle_run(spec, data, limit):
    """TTopSortProcessor::Add over host row sets with the oracle; returns the
    kept rows (columns, validity) and the picks of every call."""
    state_cols = [np.zeros(0, np.int64), np.zeros(0, np.int32), np.zeros(0, np.int64)]
    state_valid = [np.zeros(0, bool)] * 3
    picks = []
    err = C.create_string_buffer(512)
    for cols, masks in data:
        batch = q.HostRowSet(cols, masks=masks)
        n = len(cols[0])
        ids = np.arange(n, dtype=np.int64)
        sort_input = True
        if limit <= 1024 and limit <= n // 4:
            ids = O.top_k(spec, [batch], ids, limit)
            sort_input = False
        m = len(ids)
        cap = min(limit, len(state_cols[0]) + m)
        src = np.zeros(max(cap, 1), np.uint8)
        idx = np.zeros(max(cap, 1), np.uint32)
        state = q.HostRowSet(state_cols, masks=[v if not v.all() else None for v in state_valid],
                             rows=len(state_cols[0]))
        ids = np.ascontiguousarray(ids)
        r = O.lib().oracle_top_sort_update(C.byref(spec.struct), state.ptr, batch.ptr, ids.ctypes.data, m,
                                           sort_input, src.ctypes.data, idx.ctypes.data, limit, err, 512)
        assert r >= 0, err.value
        src, idx = src[:r], idx[:r]
        picks.append((src.copy(), idx.copy()))
        bvalid = [np.ones(n, bool) if masks is None or masks[c] is None else masks[c] for c in range(3)]
        state_cols = [np.where(src == 0, state_cols[c][np.minimum(idx, max(len(state_cols[c]) - 1, 0))]
                               if len(state_cols[c]) else 0, cols[c][idx]).astype(cols[c].dtype) for c in range(3)]
        state_valid = [np.where(src == 0, state_valid[c][np.minimum(idx, max(len(state_valid[c]) - 1, 0))]
                                if len(state_valid[c]) else False, bvalid[c][idx]) for c in range(3)]
    return state_cols, state_valid, picks


@pytest.mark.parametrize("limit,rows,nullable", [(5000, 40_000, False), (3000, 8_000, False),
                                                 (700, 40_000, False), (5000, 40_000, True)])
@pytest.mark.parametrize("flags", [0, abi.OUT_DEVICE])
def test_top_sort_update_matches_oracle(limit, rows, nullable, flags):
    cols = [(abi.I64, 0, 1 if nullable else 0), (abi.I32,), (abi.I64,)]
    spec = queries.SortSpec(cols, [(0, 0, 0), (1, 1, 0)], flags=flags)       # k1 ASC, k2 DESC
    data = batches(6, rows, seed=limit + rows, nullable=nullable)
    want_cols, want_valid, want_picks = oracle_run(spec, data, limit)
    ts = q.TopSort(q.compile_sort(spec), limit)
    for cols_, masks in data:
        rs = q.DeviceRowSet(cols_, masks=masks) if flags else q.HostRowSet(cols_, masks=masks)
        ts.add(rs)
    assert len(ts.calls) == len(want_picks)
    for (gs, gi), (ws, wi) in zip(ts.calls, want_picks):
        np.testing.assert_array_equal(gs, ws)
        np.testing.assert_array_equal(gi, wi)
    vals, valid = q.read_rowset(ts.state, TYPES, on_device=bool(flags))
    assert ts.state.RowCount == min(limit, 6 * rows)
    for c in range(3):
        np.testing.assert_array_equal(valid[c], want_valid[c])
        np.testing.assert_array_equal(np.asarray(vals[c])[valid[c]], want_cols[c][want_valid[c]])
    ts.release()


def test_top_sort_rejects_a_partial_schema():
    spec = queries.SortSpec([(abi.I64,), (abi.I32,), (abi.I64,)], [(0, 0, 0)], out_columns=[0, 2])
    ts = q.TopSort(q.compile_sort(spec), 2000)
    cols, masks = batches(1, 10_000, 3, False)[0]
    with pytest.raises(q.QdbError, match="every input column"):
        ts.add(q.HostRowSet(cols))
