"""Partial -> device shuffle -> final aggregation (PartialFinalAggregate)
against one oracle aggregate over the same rows: grouped Zipf lanes with
table flushes, lineitem with CHAR1 keys, decimal sums and AVG outputs, and
the keyless global identity."""
import numpy as np
import pytest

import qumirdb_b200 as q
from oracle import oracle as O
from qumirdb_b200 import abi, cascade, queries

from .helpers import assert_same_groups, gpu_rows
from .test_cascade import zipf_lanes

pytestmark = pytest.mark.gpu


def run(spec, lanes, partitions, types, max_groups=1 << 22):
    pf = cascade.PartialFinalAggregate(spec, partitions, max_groups)
    rows = []
    for out in pf.run(lanes):
        rows += gpu_rows(out, types)
        q.release(out)
    return rows


@pytest.mark.parametrize("partitions,max_groups", [(1, 1 << 22), (16, 1 << 22), (16, 20_000)])
def test_grouped_zipf_cascade(partitions, max_groups):
    data = zipf_lanes(40, 6, 400_000)
    lanes = [[q.DeviceRowSet([c[:200_000] for c in d]), q.DeviceRowSet([c[200_000:] for c in d])] for d in data]
    spec = queries.zipf_agg()
    got = run(spec, lanes, partitions, queries.ZIPF_OUT_TYPES, max_groups)
    want = O.aggregate(spec, [q.HostRowSet(d) for d in data])
    assert_same_groups(got, want, queries.ZIPF_OUT_TYPES, nkeys=1)


def test_lineitem_cascade():
    n = 500_000
    lanes, allrs = [], []
    for i in range(4):
        cols = [np.empty(n, np.int64), np.empty(n, np.int64), np.empty(n, np.int64), np.empty(n, np.int64),
                np.empty(n, np.uint8), np.empty(n, np.uint8), np.empty(n, np.int32)]
        q.lib().qdb_gen_lineitem(30 + i, n, *[c.ctypes.data for c in cols])
        lanes.append([q.DeviceRowSet(cols)])
        allrs.append(q.HostRowSet(cols))
    spec = queries.lineitem_agg(int(allrs[0].arrays[6].max()) - 90)
    got = run(spec, lanes, 4, queries.LINEITEM_OUT_TYPES)
    want = O.aggregate(spec, allrs)
    assert_same_groups(got, want, queries.LINEITEM_OUT_TYPES, nkeys=2)


def test_keyless_cascade_global_identity():
    e = q.ExprBuilder()
    a = e.col(1, abi.I64)
    f = e.op(abi.LT, abi.BOOL, a, e.const(-10**9, abi.I64))
    spec = queries.AggSpec(queries.ZIPF_COLUMNS, e, f, [], [(abi.COUNT_STAR, -1), (abi.SUM, a), (abi.MAX, a)])
    lanes = [[q.DeviceRowSet(c)] for c in zipf_lanes(3, 3, 5000)]
    assert run(spec, lanes, 1, [abi.I64, abi.I64, abi.I64]) == [[0, None, None]]
    spec2 = queries.AggSpec(queries.ZIPF_COLUMNS, e, None, [], [(abi.COUNT_STAR, -1), (abi.SUM, a), (abi.MAX, a)])
    data = zipf_lanes(3, 3, 5000)
    got = run(spec2, [[q.DeviceRowSet(c)] for c in data], 1, [abi.I64, abi.I64, abi.I64])
    assert got == O.aggregate(spec2, [q.HostRowSet(c) for c in data])
