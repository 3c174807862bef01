"""The partial -> shuffle -> final aggregate plan (qumirdb_b200.cascade) on
the CPU: the oracle runs the partial aggregate per lane, the oracle's routing
splits the partial states by key hash, and the oracle runs the combine spec
per partition; the union must equal one aggregate over all rows (group
sets; f64 within 1e-12)."""
import numpy as np
import pytest

import qumirdb_b200 as q
from oracle import oracle as O
from qumirdb_b200 import abi, cascade, queries

from .helpers import assert_same_groups


def rows_to_rowset(rows, types):
    """Oracle result rows -> a host row set of the partial row schema."""
    n = len(rows)
    cols, masks = [], []
    for k, (t, _, _) in enumerate(types):
        vals = [r[k] for r in rows]
        valid = np.array([v is not None for v in vals], dtype=bool)
        if t == abi.DECIMAL128:
            words = []
            for v in vals:
                v = 0 if v is None else int(v) & (2**128 - 1)
                words += [v & (2**64 - 1), v >> 64]
            arr = np.array(words, dtype=np.uint64).view(np.int64)
        elif t == abi.F64:
            arr = np.array([0.0 if v is None else v for v in vals], dtype=np.float64)
        elif t == abi.CHAR1:
            arr = np.array([0 if v is None else v for v in vals], dtype=np.uint8)
        else:
            arr = np.array([0 if v is None else v for v in vals], dtype=np.int64)
        cols.append(arr)
        masks.append(valid)
    return q.HostRowSet(cols, masks, rows=n)


def oracle_cascade(spec, lanes, partitions):
    types = cascade.partial_row_types(spec)
    fspec = cascade.combine_spec(spec)
    nk = spec.struct.n_keys
    parts = [[] for _ in range(max(1, partitions))]
    for lane in lanes:
        rows = O.aggregate(spec_raw(spec), lane)
        if not rows:
            continue
        rs = rows_to_rowset(rows, types)
        if nk == 0:
            parts[0].append(rs)
            continue
        h = O.hash_rows(types, list(range(nk)), rs).astype(np.uint64)
        dest = O.route(h, None, None, partitions)
        for p in range(partitions):
            pick = [rows[i] for i in np.nonzero(dest == p)[0]]
            if pick:
                parts[p].append(rows_to_rowset(pick, types))
    out = []
    for p in parts:
        if p or nk == 0:
            out += O.aggregate(fspec, p)
    return out


def spec_raw(spec):
    return cascade.partial_spec(spec)


def zipf_lanes(seed, lanes, rows):
    out = []
    for i in range(lanes):
        c = [np.empty(rows, np.int64), np.empty(rows, np.int64), np.empty(rows, np.float64)]
        q.lib().qdb_gen_zipf(seed + i, rows, 3000, 1.1, *[x.ctypes.data for x in c])
        out.append(c)
    return out


@pytest.mark.parametrize("partitions", [1, 5])
def test_grouped_cascade_equals_one_aggregate(partitions):
    spec = queries.zipf_agg()
    data = zipf_lanes(7, 3, 20_000)
    lanes = [[q.HostRowSet(c)] for c in data]
    got = oracle_cascade(spec, lanes, partitions)
    want = O.aggregate(spec, [q.HostRowSet(c) for c in data])
    assert_same_groups(got, want, queries.ZIPF_OUT_TYPES, nkeys=1)


def test_lineitem_cascade_with_avg_outputs():
    n = 30_000
    lanes, allrs = [], []
    for i in range(3):
        cols = [np.empty(n, np.int64), np.empty(n, np.int64), np.empty(n, np.int64), np.empty(n, np.int64),
                np.empty(n, np.uint8), np.empty(n, np.uint8), np.empty(n, np.int32)]
        q.lib().qdb_gen_lineitem(20 + i, n, *[c.ctypes.data for c in cols])
        lanes.append([q.HostRowSet(cols)])
        allrs.append(q.HostRowSet(cols))
    spec = queries.lineitem_agg(int(lanes[0][0].arrays[6].max()) - 90)
    got = oracle_cascade(spec, lanes, 3)
    want = O.aggregate(spec, allrs)
    assert_same_groups(got, want, queries.LINEITEM_OUT_TYPES, nkeys=2)


def test_keyless_cascade_keeps_the_global_identity():
    """An empty global input: COUNT 0 and SUM NULL after the combine."""
    e = q.ExprBuilder()
    a = e.col(1, abi.I64)
    f = e.op(abi.LT, abi.BOOL, a, e.const(-10**9, abi.I64))     # no row passes
    spec = queries.AggSpec(queries.ZIPF_COLUMNS, e, f, [], [(abi.COUNT_STAR, -1), (abi.SUM, a), (abi.MAX, a)])
    lanes = [[q.HostRowSet(c)] for c in zipf_lanes(3, 2, 1000)]
    assert oracle_cascade(spec, lanes, 1) == [[0, None, None]] == O.aggregate(spec, [r[0] for r in lanes])
