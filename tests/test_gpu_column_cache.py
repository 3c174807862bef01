"""Device column cache: scan batches staged into HBM once and served from
there to the kernels across queries; least recently used columns evicted to
stay within the budget, columns in use never; results equal the uncached
path and the oracle."""
import numpy as np
import pytest

import qumirdb_b200 as q
from oracle import oracle as O
from qumirdb_b200 import abi, queries

from .helpers import assert_same_groups, gpu_rows

pytestmark = pytest.mark.gpu

BATCH = 1 << 18   # the Parquet source's batch rows


def lineitem_batches(n_batches, seed=0):
    out = []
    for b in range(n_batches):
        cols = [np.empty(BATCH, np.int64), np.empty(BATCH, np.int64), np.empty(BATCH, np.int64),
                np.empty(BATCH, np.int64), np.empty(BATCH, np.uint8), np.empty(BATCH, np.uint8),
                np.empty(BATCH, np.int32)]
        q.lib().qdb_gen_lineitem(seed + b, BATCH, *[c.ctypes.data for c in cols])
        out.append(q.HostRowSet(cols))
    return out


def run_query(spec, rowsets):
    agg = q.Aggregate(q.compile_aggregate(spec))
    for rs in rowsets:
        agg.add(rs)
    out = agg.finish()
    rows = gpu_rows(out, queries.LINEITEM_OUT_TYPES)
    q.release(out)
    return rows


def test_cached_queries_match_and_hit():
    host = lineitem_batches(6)
    spec = queries.lineitem_agg(int(host[0].arrays[6].max()) - 90)
    want = O.aggregate(spec, host)
    per_batch = sum(a.nbytes for a in host[0].arrays)
    cache = q.ColumnCache(budget_bytes=8 * per_batch)
    types = queries.LINEITEM_COLUMNS
    for query in range(3):
        views = [cache.get(7, b, rs, types) for b, rs in enumerate(host)]
        assert_same_groups(run_query(spec, views), want, queries.LINEITEM_OUT_TYPES, nkeys=2)
        for v in views:
            v.release()
        st = cache.stats()
        assert st["misses"] == 6 * 7 and st["hits"] == query * 6 * 7
        assert st["h2d_bytes"] == 6 * per_batch and st["pinned_bytes"] == 0
    cache.close()


def test_budget_eviction_and_pinning():
    host = lineitem_batches(4, seed=10)
    types = queries.LINEITEM_COLUMNS
    per_batch = sum(a.nbytes for a in host[0].arrays)
    cache = q.ColumnCache(budget_bytes=int(2.5 * per_batch), staging_bytes=1 << 20)
    a = cache.get(1, 0, host[0], types)
    b = cache.get(1, 1, host[1], types)
    # a third batch does not fit while both are in use
    with pytest.raises(q.QdbError):
        cache.get(1, 2, host[2], types)
    a.release()
    c = cache.get(1, 2, host[2], types)   # evicts batch 0, the least recently used
    st = cache.stats()
    assert st["evictions"] >= 1 and st["resident_bytes"] <= 2.5 * per_batch
    assert st["pinned_bytes"] == 2 * per_batch
    vals, _ = q.read_rowset(c.rs, [abi.I64, abi.DECIMAL64], on_device=True)
    assert (vals[0] == host[2].arrays[0]).all() and (vals[1] == host[2].arrays[1]).all()
    b.release()
    c.release()
    entries = cache.stats()["entries"]
    assert cache.invalidate(1) == entries and cache.stats()["resident_bytes"] == 0
    cache.close()


def test_masks_selection_and_column_subsets():
    rng = np.random.default_rng(2)
    n = 100_000
    k = rng.integers(0, 50, n).astype(np.int64)
    v = rng.integers(-10, 10, n).astype(np.int64)
    valid = rng.random(n) > 0.1
    sel = (rng.random(n) > 0.3).astype(np.uint8)
    host = q.HostRowSet([k, v], masks=[None, valid], selection=sel)
    cache = q.ColumnCache(budget_bytes=1 << 24)
    types = [(abi.I64,), (abi.I64, 0, 1)]
    e = q.ExprBuilder()
    spec = queries.AggSpec(types, e, None, [e.col(0, abi.I64)], [(abi.COUNT, e.col(1, abi.I64)),
                                                                (abi.SUM, 1)])
    want = O.aggregate(spec, [host])
    for _ in range(2):
        view = cache.get(3, 0, host, types)
        agg = q.Aggregate(q.compile_aggregate(spec))
        agg.add(view)
        out = agg.finish()
        got = gpu_rows(out, [abi.I64, abi.I64, abi.I64])
        q.release(out)
        view.release()
        assert_same_groups(got, want, [abi.I64, abi.I64, abi.I64], nkeys=1)
    sub = cache.get(3, 0, host, types, columns=[1])
    vals, vv = q.read_rowset(sub.rs, [abi.I64], on_device=True)
    assert (vv[0] == valid).all() and (vals[0][valid] == v[valid]).all()
    sub.release()
    assert cache.stats()["hits"] == 3 and cache.stats()["misses"] == 2
    cache.close()
