"""Batched aggregation (qdb_gpu_agg_dispatch_batch / qdb_gpu_agg_finish_batch):
every aggregate of a batch gives exactly the groups it gives alone through
agg_dispatch / agg_finish_rowset (integers bit-exact, f64 sums within 1e-12
relative), whatever the mix of sizes, key skew, table growth and output
placement; the autotuner stores its choice and the graph replays."""
import numpy as np
import pytest

import qumirdb_b200 as q
from oracle import oracle as O
from qumirdb_b200 import abi, queries

from .helpers import assert_same_groups, gpu_rows, lineitem, shape_case, zipf_data

pytestmark = pytest.mark.gpu


def table(rs, types, on_device=False):
    vals, valid = q.read_rowset(rs, types, on_device)
    order = np.lexsort([vals[0]])
    return [np.asarray(v)[order] for v in vals], [np.asarray(m)[order] for m in valid]


def assert_tables_equal(a, b, types):
    (va, ma), (vb, mb) = a, b
    assert len(va[0]) == len(vb[0]), f"group count {len(va[0])} != {len(vb[0])}"
    for c, t in enumerate(types):
        assert np.array_equal(ma[c], mb[c]), f"column {c} validity"
        x, y = va[c][ma[c]], vb[c][mb[c]]
        if t in (abi.F64, abi.F32):
            np.testing.assert_allclose(x, y, rtol=1e-12, atol=0)
        else:
            assert np.array_equal(x, y), f"column {c}"


def partitions(seed, sizes, distinct, uniform=()):
    """Zipf key partitions; those listed in `uniform` get distinct keys over
    the full 64-bit range (every row its own group) and a few rows of key -1."""
    rng = np.random.default_rng(seed)
    out = []
    for i, n in enumerate(sizes):
        cols = zipf_data(n, distinct, seed=100 + i) if n else [np.zeros(0, np.int64), np.zeros(0, np.int64),
                                                               np.zeros(0, np.float64)]
        if i in uniform and n:
            cols[0] = rng.integers(-2**62, 2**62, n, dtype=np.int64)
            cols[0][:: max(1, n // 5)] = -1
        out.append(cols)
    return out


@pytest.mark.parametrize("flags", [0, abi.OUT_DEVICE])
def test_batch_matches_each_aggregate_alone(flags):
    rng = np.random.default_rng(7)
    sizes = [0, 1, 7, 1000] + [int(x) for x in np.exp(rng.uniform(np.log(500), np.log(120_000), 36))]
    parts = partitions(1, sizes, 40_000, uniform={5, 17, 30})
    prog = q.compile_aggregate(queries.zipf_agg(expected_groups=40_000, flags=flags))
    types = queries.ZIPF_OUT_TYPES
    # Two updates per aggregate: the second finds every state initialised.
    halves = [[c[: len(p[0]) // 2] for c in p] for p in parts], [[c[len(p[0]) // 2:] for c in p] for p in parts]
    batch = q.AggregateBatch(prog, len(parts))
    for h in halves:
        batch.add([q.DeviceRowSet(cols) for cols in h])
    groups = batch.groups
    outs = batch.finish()
    for i, cols in enumerate(parts):
        agg = q.Aggregate(prog)
        for h in halves:
            agg.add(q.DeviceRowSet(h[i]))
        assert agg.groups == groups[i]
        alone = agg.finish()
        assert outs[i].RowCount == alone.RowCount == groups[i]
        dev = flags == abi.OUT_DEVICE
        assert_tables_equal(table(outs[i], types, dev), table(alone, types, dev), types)
        q.release(alone)
    # Two aggregates against the oracle as well.
    for i in (3, 20):
        want = O.aggregate(queries.zipf_agg(), [q.HostRowSet(parts[i])])
        if flags != abi.OUT_DEVICE:
            assert_same_groups(gpu_rows(outs[i], types), want, types, nkeys=1)
    for o in outs:
        q.release(o)


def test_batch_autotune_and_graph_replay():
    q.autotune_reset()
    # 23M rows: big enough for the autotuner to search (small batches run
    # the defaults).
    sizes = [2_000_000, 100_000, 800_000, 30_000, 1_500_000, 300_000, 1_000_000, 50_000] * 4
    parts = partitions(2, sizes, 30_000)
    prog = q.compile_aggregate(queries.zipf_agg(flags=abi.OUT_DEVICE))
    types = queries.ZIPF_OUT_TYPES
    results = []
    for rep in range(4):
        batch = q.AggregateBatch(prog, len(parts))
        batch.add([q.DeviceRowSet(cols) for cols in parts])
        outs = batch.finish()
        results.append([table(o, types, True) for o in outs])
        for o in outs:
            q.release(o)
    info = q.autotune_info()
    assert info["searches"] == 1 and info["trials"] >= 2, info
    assert info["reused"] >= 3, info
    assert info["graph_replays"] >= 2, info      # captured on the third identical batch
    assert len(info["configs"]) == 1 and info["configs"][0]["threads"] in (512, 1024), info
    for rep in (1, 2, 3):
        for a, b in zip(results[0], results[rep]):
            assert_tables_equal(a, b, types)


def test_batch_lineitem_partitions_char_keys():
    """The Q1-shaped program (two one-byte string keys, 128-bit decimal sums)
    over partitions of a lineitem table: string-offset and validity slices."""
    n = 300_000
    cols = lineitem(n, seed=9)
    spec = queries.lineitem_agg(int(cols[6].max()) - 90)
    prog = q.compile_aggregate(spec)
    bounds = [0, 10, 1000, 50_000, 50_001, 180_000, n]
    parts = [[c[lo:hi] for c in cols] for lo, hi in zip(bounds[:-1], bounds[1:])]
    batch = q.AggregateBatch(prog, len(parts))
    batch.add([q.DeviceRowSet(p) for p in parts])
    outs = batch.finish()
    types = queries.LINEITEM_OUT_TYPES
    for p, o in zip(parts, outs):
        want = O.aggregate(spec, [q.HostRowSet(p)])
        assert_same_groups(gpu_rows(o, types), want, types, nkeys=2)
        q.release(o)


def test_batch_states_without_a_batched_kernel():
    """A nullable input column falls outside the typed shapes: the states
    take the one-state path inside the same call and still match."""
    rng = np.random.default_rng(4)
    parts = partitions(3, [5000, 0, 20_000, 300], 2000)
    masks = [None if i % 2 else [None, rng.random(len(p[0])) > 0.3, None] for i, p in enumerate(parts)]
    e = q.ExprBuilder()
    key, a, x = e.col(0, abi.I64), e.col(1, abi.I64), e.col(2, abi.F64)
    aggs = [(abi.COUNT_STAR, -1), (abi.SUM, a), (abi.MIN, a), (abi.MAX, a), (abi.SUM, x)]
    spec = queries.AggSpec([(abi.I64,), (abi.I64, 0, 1), (abi.F64,)], e, None, [key], aggs)
    prog = q.compile_aggregate(spec)
    types = queries.ZIPF_OUT_TYPES
    batch = q.AggregateBatch(prog, len(parts))
    batch.add([q.DeviceRowSet(p, m) for p, m in zip(parts, masks)])
    outs = batch.finish()
    for p, m, o in zip(parts, masks, outs):
        want = O.aggregate(spec, [q.HostRowSet(p, m)])
        assert_same_groups(gpu_rows(o, types), want, types, nkeys=1)
        q.release(o)


@pytest.mark.parametrize("form", ["filter_literal", "affine_constant"])
def test_same_shape_programs_with_other_literals_do_not_share_a_graph(form):
    """Two programs of one shape that differ only in a literal (a filter
    constant, or the constant of SUM(a + c)) alternate after the launch
    sequence of the first was captured as a graph (three identical batches
    in a row): each batch must give its own program's groups."""
    sizes = [20_000, 3_000, 45_000, 9_000]
    parts = partitions(9, sizes, 5_000)

    def spec(c):
        e = q.ExprBuilder()
        key, a = e.col(0, abi.I64), e.col(1, abi.I64)
        if form == "filter_literal":
            pred = e.op(abi.LT, abi.BOOL, a, e.const(c, abi.I64))
            return queries.AggSpec(queries.ZIPF_COLUMNS, e, pred, [key], [(abi.SUM, a), (abi.COUNT_STAR, -1)])
        val = e.op(abi.ADD, abi.I64, a, e.const(c, abi.I64))
        return queries.AggSpec(queries.ZIPF_COLUMNS, e, None, [key], [(abi.SUM, val), (abi.COUNT_STAR, -1)])

    specs = {c: spec(c) for c in (5, 90_000)}
    progs = {c: q.compile_aggregate(s) for c, s in specs.items()}
    rowsets = [q.DeviceRowSet(p) for p in parts]
    types = [abi.I64, abi.I64, abi.I64]
    want = {c: [O.aggregate(specs[c], [q.HostRowSet(p)]) for p in parts] for c in specs}
    for c in [5, 5, 5, 5, 90_000, 5, 90_000, 90_000, 90_000, 5]:
        batch = q.AggregateBatch(progs[c], len(parts))
        batch.add(rowsets)
        outs = batch.finish()
        for i in range(len(parts)):
            assert_same_groups(gpu_rows(outs[i], types), want[c][i], types, nkeys=1)
        outs.release()


@pytest.mark.parametrize("shape,groups", [("lineitem", 6), ("q6", 1), ("count", 3), ("sum_count", 40),
                                          ("sum_count", 5000)])
def test_batch_low_cardinality_partitions(shape, groups):
    """Uneven partitions (empty, a partial quad, up to 400K rows) of each
    compiled low-cardinality shape in one batched launch of the
    low-cardinality kernel: the first four groups of a work item in
    lane-private accumulators, the next ones in the shared tier, the rest
    (and, with 5000 groups against a hint of 64, the rows the full tables
    turn away) through the tables and the replay.  Two updates per state;
    every partition's groups equal the oracle's."""
    rng = np.random.default_rng(31 + groups)
    sizes = [0, 3, 4, 129, 5000] + [int(x) for x in np.exp(rng.uniform(np.log(1000), np.log(400_000), 27))]
    cols, spec, types = shape_case(shape, groups, sum(sizes), rng)
    bounds = np.concatenate([[0], np.cumsum(sizes)])
    parts = [[c[lo:hi] for c in cols] for lo, hi in zip(bounds[:-1], bounds[1:])]
    halves = ([[c[: len(p[0]) // 2 // 4 * 4] for c in p] for p in parts],
              [[c[len(p[0]) // 2 // 4 * 4:] for c in p] for p in parts])
    prog = q.compile_aggregate(spec)
    before = q.autotune_info()["batched_states"]["low"]
    q.profile(True)
    q.profile_read()
    batch = q.AggregateBatch(prog, len(parts))
    for h in halves:
        batch.add([q.DeviceRowSet(c) for c in h])
    outs = batch.finish()
    names = {k[0] for k in q.profile_read()}
    q.profile(False)
    assert "agg_batch_update_low" in names, names
    assert q.autotune_info()["batched_states"]["low"] - before == 2 * len(parts)
    nkeys = 0 if shape == "q6" else (2 if shape == "lineitem" else 1)
    for p, o in zip(parts, outs):
        want = O.aggregate(spec, [q.HostRowSet(p)])
        assert_same_groups(gpu_rows(o, types), want, types, nkeys=nkeys)
    outs.release()
