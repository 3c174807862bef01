"""Parity at the benchmark sizes: the device path against the oracle on the
same seeded inputs the benchmark measures.

* GROUP BY key over 200M Zipf(1.1) rows of 20M ranks (three 64M-row
  launches into one growing table): group sets equal, integers exact, f64
  sums within 1e-12 relative.
* The same query as 4096 independent partitions of log-uniform 1K-1M rows
  (585M rows) in one batched launch: each partition against its own oracle
  run.
* ORDER BY k1 DESC, k2 ASC over 300M row ids in 4M-row batches: the whole
  permutation equal to the oracle's stable order.
* ORDER BY k1 LIMIT 1000 over the same 300M rows: equal to the oracle's
  heap top-K.
"""
import concurrent.futures as cf
import os

import numpy as np
import pytest

import qumirdb_b200 as q
from oracle import oracle as O
from qumirdb_b200 import abi, queries

pytestmark = pytest.mark.gpu

THREADS = os.cpu_count() or 1


def gen_zipf(seed, n, distinct):
    cols = [np.empty(n, np.int64), np.empty(n, np.int64), np.empty(n, np.float64)]
    O.lib().qdb_gen_zipf(seed, n, distinct, 1.1, *[c.ctypes.data for c in cols])
    return cols


def by_key(values, valid):
    order = np.argsort(values[0], kind="stable")
    return [np.asarray(v)[order] for v in values], [np.asarray(m)[order] for m in valid]


def assert_same_arrays(got, want, types):
    (gv, gm), (wv, wm) = by_key(*got), by_key(*want)
    assert len(gv[0]) == len(wv[0]), f"group count {len(gv[0])} != {len(wv[0])}"
    for c, t in enumerate(types):
        np.testing.assert_array_equal(gm[c], wm[c], err_msg=f"column {c} validity")
        x, y = gv[c][gm[c]], wv[c][wm[c]]
        if t in (abi.F64, abi.F32):
            np.testing.assert_allclose(x, y, rtol=1e-12, atol=0, err_msg=f"column {c}")
        else:
            np.testing.assert_array_equal(x, y, err_msg=f"column {c}")


def test_zipf_group_by_200m_rows_matches_oracle():
    n, distinct = 200_000_000, 20_000_000
    cols = gen_zipf(2, n, distinct)
    spec = queries.zipf_agg(expected_groups=distinct)
    drs = q.DeviceRowSet(cols)
    agg = q.Aggregate(q.compile_aggregate(spec))
    agg.add(drs)
    out = agg.finish()
    got = q.read_rowset(out, queries.ZIPF_OUT_TYPES)
    q.release(out)
    del drs
    want = O.aggregate_arrays(spec, [q.HostRowSet(cols)], lanes=THREADS)
    assert len(want[0][0]) > 9_000_000
    assert_same_arrays(got, want, queries.ZIPF_OUT_TYPES)


def test_zipf_4096_partitions_batched_match_oracle_per_partition():
    rng = np.random.default_rng(5)
    sizes = np.exp(rng.uniform(np.log(1e3), np.log(1e6), 4096)).astype(np.int64)
    n = int(sizes.sum())
    cols = gen_zipf(6, n, 20_000_000)
    spec = queries.zipf_agg()
    prog = q.compile_aggregate(spec)
    drs = q.DeviceRowSet(cols)
    bounds = np.concatenate([[0], np.cumsum(sizes)])
    parts = q.RowSetPointers([q.SliceRowSet(drs, int(lo), int(hi)) for lo, hi in zip(bounds[:-1], bounds[1:])])
    batch = q.AggregateBatch(prog, len(parts))
    batch.add(parts)
    groups = batch.groups
    outs = batch.finish()

    def oracle_part(i):
        lo, hi = int(bounds[i]), int(bounds[i + 1])
        return O.aggregate_arrays(spec, [q.HostRowSet([c[lo:hi] for c in cols])])

    checked = 0
    with cf.ThreadPoolExecutor(THREADS) as ex:
        for start in range(0, len(sizes), 256):
            idx = range(start, min(start + 256, len(sizes)))
            wants = list(ex.map(oracle_part, idx))
            for i, want in zip(idx, wants):
                got = q.read_rowset(outs[i], queries.ZIPF_OUT_TYPES)
                assert groups[i] == len(got[0][0])
                assert_same_arrays(got, want, queries.ZIPF_OUT_TYPES)
                checked += 1
    outs.release()
    assert checked == 4096


def sort_store(n, batch):
    k1 = np.empty(n, np.int64)
    k2 = np.empty(n, np.int32)
    rowid = np.arange(n, dtype=np.int64)
    O.lib().qdb_gen_sort(3, n, k1.ctypes.data, k2.ctypes.data, None)
    sizes = [min(batch, n - b) for b in range(0, n, batch)]
    store, at = [], 0
    for m in sizes:
        store.append(q.DeviceRowSet([k1[at:at + m], k2[at:at + m], rowid[at:at + m]]))
        at += m
    ids = np.concatenate([(np.int64(b) << 32) | np.arange(m, dtype=np.int64) for b, m in enumerate(sizes)])
    return k1, k2, rowid, store, ids


def test_sort_300m_rows_permutation_matches_oracle():
    n, batch = 300_000_000, 1 << 22
    k1, k2, rowid, store, ids = sort_store(n, batch)
    del rowid
    sorter = q.Sort(q.compile_sort(queries.sort_k1_desc_k2(flags=abi.OUT_DEVICE)), store)
    dev = q.DeviceBuffer(ids.nbytes).upload(ids)
    del ids
    sorter.sort(dev)
    got = dev.download(np.int64, n)
    dev.free()
    # Packed (batch << 32 | row) -> position in the input.
    got = (got >> 32) * batch + (got & 0xFFFFFFFF)
    want = O.sorted_row_indices(k1, k2, THREADS)
    np.testing.assert_array_equal(got, want)


def test_top_1000_of_300m_rows_matches_oracle():
    n, batch = 300_000_000, 1 << 22
    k1, k2, rowid, store, ids = sort_store(n, batch)
    spec = queries.top_k1(flags=abi.OUT_DEVICE)
    topper = q.Sort(q.compile_sort(spec), store)
    dev = q.DeviceBuffer(ids.nbytes).upload(ids)
    k = topper.top_k(dev, 1000)
    assert k == 1000
    got = dev.download(np.int64, k)
    dev.free()
    hstore = []
    for b in range(len(store)):
        lo, hi = b * batch, min(n, (b + 1) * batch)
        hstore.append(q.HostRowSet([k1[lo:hi], k2[lo:hi], rowid[lo:hi]]))
    want = O.top_k(spec, hstore, ids, 1000)
    np.testing.assert_array_equal(got, want)
