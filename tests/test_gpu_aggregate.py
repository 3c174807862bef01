"""Device fused filter -> project -> hash aggregate against the oracle."""
import numpy as np
import pytest

import qumirdb_b200 as q
from oracle import oracle as O
from qumirdb_b200 import abi, queries

from .helpers import assert_same_groups, gpu_rows, lineitem, shape_case, zipf_data

pytestmark = pytest.mark.gpu


def run_gpu(spec, rowsets, initial_capacity=8):
    prog = q.compile_aggregate(spec)
    agg = q.Aggregate(prog, initial_capacity)
    for rs in rowsets:
        agg.add(rs)
    out = agg.finish()
    return out


def out_types(spec):
    return None


@pytest.mark.parametrize("n", [1, 1000, 100_003])
def test_lineitem_host_batches(n):
    cols = lineitem(n, seed=3)
    cutoff = int(cols[6].max()) - 90 if n > 1 else 10**6
    spec = queries.lineitem_agg(cutoff)
    rs = q.HostRowSet(cols)
    out = run_gpu(spec, [rs])
    got = gpu_rows(out, queries.LINEITEM_OUT_TYPES)
    q.release(out)
    want = O.aggregate(spec, [rs])
    assert_same_groups(got, want, queries.LINEITEM_OUT_TYPES, nkeys=2)


def test_lineitem_device_resident_full_size():
    n = 6_001_215
    cols = lineitem(n, seed=0)
    cutoff = int(cols[6].max()) - 90
    spec = queries.lineitem_agg(cutoff)
    drs = q.DeviceRowSet(cols)
    out = run_gpu(spec, [drs])
    got = gpu_rows(out, queries.LINEITEM_OUT_TYPES)
    q.release(out)
    want = O.aggregate(spec, [q.HostRowSet(cols)], lanes=8)
    assert len(got) == 4
    assert_same_groups(got, want, queries.LINEITEM_OUT_TYPES, nkeys=2)


def test_lineitem_general_path_matches_typed_path():
    # Validity masks (all valid) keep the plan off the typed row shape, so the
    # general kernel computes the same query; both must equal the oracle.
    cols = lineitem(80_000, seed=13)
    spec = queries.lineitem_agg(int(cols[6].max()) - 60)
    want = O.aggregate(spec, [q.HostRowSet(cols)])
    typed = run_gpu(spec, [q.HostRowSet(cols)])
    masked = run_gpu(spec, [q.HostRowSet(cols, masks=[np.ones(len(cols[0]), bool)] * len(cols))])
    for out in (typed, masked):
        got = gpu_rows(out, queries.LINEITEM_OUT_TYPES)
        q.release(out)
        assert_same_groups(got, want, queries.LINEITEM_OUT_TYPES, nkeys=2)


def test_lineitem_several_batches_and_selection():
    cols = lineitem(50_000, seed=4)
    cutoff = int(cols[6].max()) - 300
    spec = queries.lineitem_agg(cutoff)
    rng = np.random.default_rng(5)
    batches = []
    for k in range(3):
        part = [c[k * 16_000:(k + 1) * 16_000 + 7] for c in cols]
        sel = rng.integers(0, 2, len(part[0])).astype(np.uint8)
        batches.append(q.HostRowSet(part, selection=sel))
    out = run_gpu(spec, batches)
    got = gpu_rows(out, queries.LINEITEM_OUT_TYPES)
    q.release(out)
    want = O.aggregate(spec, batches)
    assert_same_groups(got, want, queries.LINEITEM_OUT_TYPES, nkeys=2)


@pytest.mark.parametrize("capacity", [8, 1 << 20])
def test_high_cardinality_growth_and_replay(capacity):
    # 300K rows over 200K Zipf ranks from a table of 8 slots: the table grows,
    # rows past the probe bound are deferred and replayed, shared tables spill.
    cols = zipf_data(300_000, 200_000, seed=7)
    spec = queries.zipf_agg(expected_groups=0)
    out = run_gpu(spec, [q.HostRowSet(cols)], initial_capacity=capacity)
    got = gpu_rows(out, queries.ZIPF_OUT_TYPES)
    q.release(out)
    want = O.aggregate(spec, [q.HostRowSet(cols)], lanes=8)
    assert_same_groups(got, want, queries.ZIPF_OUT_TYPES, nkeys=1)


def test_nullable_generic_expressions():
    rng = np.random.default_rng(11)
    n = 20_000
    a = rng.integers(-50, 50, n).astype(np.int64)
    b = rng.integers(0, 5, n).astype(np.int32)
    f = rng.random(n)
    g = rng.integers(0, 7, n).astype(np.int64)
    ma = rng.random(n) > 0.1
    mf = rng.random(n) > 0.2
    cols = [(abi.I64, 0, 1), (abi.I32,), (abi.F64, 0, 1), (abi.I64,)]
    e = q.ExprBuilder()
    ca, cb, cf, cg = e.col(0, abi.I64), e.col(1, abi.I32), e.col(2, abi.F64), e.col(3, abi.I64)
    # WHERE a > -40 OR b = 3  (generic: OR over two columns is still atoms) AND f IS NOT NULL
    pred = e.op(abi.AND, abi.BOOL, e.op(abi.OR, abi.BOOL, e.op(abi.GT, abi.BOOL, ca, e.const(-40, abi.I64)),
                                        e.op(abi.EQ, abi.BOOL, cb, e.const(3, abi.I32))),
                e.op(abi.IS_NOT_NULL, abi.BOOL, cf))
    case = e.op(abi.CASE, abi.I64, e.op(abi.GT, abi.BOOL, cb, e.const(2, abi.I32)), ca, e.const(0, abi.I64))
    mix = e.op(abi.ADD, abi.F64, cf, e.op(abi.CAST, abi.F64, ca))
    key2 = e.op(abi.MOD, abi.I64, cg, e.const(3, abi.I64))
    aggs = [(abi.SUM, case), (abi.MIN, ca), (abi.MAX, mix), (abi.COUNT, ca), (abi.SUM, mix), (abi.COUNT_STAR, -1)]
    spec = queries.AggSpec(cols, e, pred, [cb, key2], aggs)
    types = [abi.I32, abi.I64, abi.I64, abi.I64, abi.F64, abi.I64, abi.F64, abi.I64]
    rs = q.HostRowSet([a, b, f, g], masks=[ma, None, mf, None])
    out = run_gpu(spec, [rs])
    got = gpu_rows(out, types)
    q.release(out)
    want = O.aggregate(spec, [rs])
    assert_same_groups(got, want, types, nkeys=2)


def test_wide_keys_with_decimal_and_nulls():
    rng = np.random.default_rng(12)
    n = 30_000
    d = rng.integers(-10**6, 10**6, n).astype(np.int64)
    k = rng.integers(0, 40, n).astype(np.int64)
    m = rng.integers(0, 3, n).astype(np.int64)
    mm = rng.random(n) > 0.3
    cols = [(abi.I64,), (abi.I64,), (abi.I64, 0, 1)]
    e = q.ExprBuilder()
    c0, c1, c2 = e.col(0, abi.I64), e.col(1, abi.I64), e.col(2, abi.I64)
    dk = e.op(abi.CAST, abi.DECIMAL128, e.op(abi.MOD, abi.I64, c0, e.const(50, abi.I64)), scale=2)
    spec = queries.AggSpec(cols, e, None, [dk, c1, c2], [(abi.COUNT_STAR, -1), (abi.SUM, c0), (abi.MAX, c2)])
    types = [abi.DECIMAL128, abi.I64, abi.I64, abi.I64, abi.I64, abi.I64]
    rs = q.HostRowSet([d, k, m], masks=[None, None, mm])
    out = run_gpu(spec, [rs])
    got = gpu_rows(out, types)
    q.release(out)
    want = O.aggregate(spec, [rs])
    assert_same_groups(got, want, types, nkeys=3)


def test_keyless_aggregate_over_empty_input_has_one_group():
    # COUNT 0 and SUM NULL over no rows (docs/arch/aggregation.md:144-164).
    e = q.ExprBuilder()
    c = e.col(0, abi.I64)
    pred = e.op(abi.GT, abi.BOOL, c, e.const(100, abi.I64))
    spec = queries.AggSpec([(abi.I64,)], e, pred, [], [(abi.COUNT_STAR, -1), (abi.SUM, c), (abi.MIN, c)])
    rs = q.HostRowSet([np.arange(10, dtype=np.int64)])
    out = run_gpu(spec, [rs])
    got = gpu_rows(out, [abi.I64, abi.I64, abi.I64])
    q.release(out)
    assert got == [[0, None, None]]
    assert O.aggregate(spec, [rs]) == got


def test_device_output_stays_resident():
    cols = lineitem(10_000, seed=9)
    spec = queries.lineitem_agg(int(cols[6].max()), flags=abi.OUT_DEVICE)
    out = run_gpu(spec, [q.HostRowSet(cols)])
    assert out.RowCount == 4
    assert q.lib().qdb_gpu_launch_count(0) > 0
    q.release(out)


@pytest.mark.parametrize("groups", [1, 3, 40])
@pytest.mark.parametrize("shape", ["count", "sum_count", "q6", "lineitem"])
def test_shape_kernels(shape, groups):
    """Each compiled query shape of the listed-row kernel, with all groups in
    registers (1 and 3 groups) and with 40 groups (the first four in
    registers, the rest through the shared table); rows in three batches, the
    last ending in a partial tile."""
    rng = np.random.default_rng(7 + groups)
    n = 150_001
    cols, spec, types = shape_case(shape, groups, n, rng)
    bounds = [(0, 70_000), (70_000, 140_000), (140_000, n)]
    q.profile(True)
    q.profile_read()
    out = run_gpu(spec, [q.DeviceRowSet([c[lo:hi] for c in cols]) for lo, hi in bounds])
    names = {kk[0] for kk in q.profile_read()}
    q.profile(False)
    got = gpu_rows(out, types)
    q.release(out)
    assert "agg_update_sig" in names, names
    want = O.aggregate(spec, [q.HostRowSet([c[lo:hi] for c in cols]) for lo, hi in bounds])
    nkeys = 0 if shape == "q6" else (2 if shape == "lineitem" else 1)
    assert_same_groups(got, want, types, nkeys=nkeys)


def test_lineitem_runs_the_signature_kernel():
    """The lineitem query's typed plan has an instantiated state signature:
    its update is the listed-row kernel, with the same groups as the oracle."""
    cols = lineitem(300_000, seed=5)
    spec = queries.lineitem_agg(int(cols[6].max()) - 90)
    q.profile(True)
    q.profile_read()
    out = run_gpu(spec, [q.DeviceRowSet(cols)])
    names = {k[0] for k in q.profile_read()}
    q.profile(False)
    got = gpu_rows(out, queries.LINEITEM_OUT_TYPES)
    q.release(out)
    assert "agg_update_sig" in names, names
    want = O.aggregate(spec, [q.HostRowSet(cols)])
    assert_same_groups(got, want, queries.LINEITEM_OUT_TYPES, nkeys=2)


def test_high_cardinality_heavy_hitter_seeds():
    """An update of at least 16M rows samples its keys and seeds the shared
    tier with the most frequent; a later update (with a selection, and rows
    whose keys include none of some seeds) reuses them.  Rows of key -1 (the
    empty marker) take the table's flag slot.  Every group equals the
    oracle's."""
    n = 17_000_000
    first = zipf_data(n, 200_000, 11)
    first[0][::997] = -1
    second = zipf_data(1_000_000, 400_000, 12)
    sel = (np.random.default_rng(3).random(len(second[0])) > 0.4).astype(np.uint8)
    spec = queries.zipf_agg(expected_groups=200_000)
    q.profile(True)
    q.profile_read()
    out = run_gpu(spec, [q.DeviceRowSet(first), q.DeviceRowSet(second, selection=sel)])
    names = [kk[0] for kk in q.profile_read()]
    q.profile(False)
    got = gpu_rows(out, queries.ZIPF_OUT_TYPES)
    q.release(out)
    assert names.count("agg_seed") == 1 and "agg_update_high" in names, names
    want = O.aggregate(spec, [q.HostRowSet(first), q.HostRowSet(second, selection=sel)])
    assert_same_groups(got, want, queries.ZIPF_OUT_TYPES, nkeys=1)


@pytest.mark.parametrize("shape", ["zipf", "count", "sum_count"])
def test_high_cardinality_shape_kernels(shape):
    """The high-cardinality shape kernel (shared tier for hot keys, global
    table for the rest, typed atomics) on a skewed key stream whose groups
    overflow the initial table (growth and replay of deferred rows)."""
    n = 400_000
    cols = zipf_data(n, 60_000, 4)
    e = q.ExprBuilder()
    key, a, x = e.col(0, abi.I64), e.col(1, abi.I64), e.col(2, abi.F64)
    if shape == "zipf":
        spec = queries.zipf_agg(expected_groups=2000)
        types = queries.ZIPF_OUT_TYPES
    elif shape == "count":
        spec = queries.AggSpec(queries.ZIPF_COLUMNS[:1], e, None, [key], [(abi.COUNT_STAR, -1)], expected_groups=2000)
        cols = cols[:1]
        types = [abi.I64, abi.I64]
    else:
        spec = queries.AggSpec(queries.ZIPF_COLUMNS[:2], e, None, [key], [(abi.SUM, a), (abi.COUNT_STAR, -1)],
                               expected_groups=2000)
        cols = cols[:2]
        types = [abi.I64, abi.I64, abi.I64]
    bounds = [(0, 150_000), (150_000, 300_000), (300_000, n)]
    q.profile(True)
    q.profile_read()
    out = run_gpu(spec, [q.DeviceRowSet([c[lo:hi] for c in cols]) for lo, hi in bounds], initial_capacity=1024)
    names = {kk[0] for kk in q.profile_read()}
    q.profile(False)
    got = gpu_rows(out, types)
    q.release(out)
    assert "agg_update_high" in names, names
    want = O.aggregate(spec, [q.HostRowSet([c[lo:hi] for c in cols]) for lo, hi in bounds])
    assert_same_groups(got, want, types, nkeys=1)


@pytest.mark.parametrize("offset", [0, 1, 4, 129])
def test_low_cardinality_kernels_at_any_column_alignment(offset):
    """Columns that start on a four-value boundary take the four-rows-per-
    thread kernel; a slice starting at another row takes the one-row walk
    (both named agg_update_sig).  Both, over ranges whose CTA tails are
    ragged, equal the oracle."""
    n = 300_007
    cols = lineitem(n + offset, seed=17)
    spec = queries.lineitem_agg(int(cols[6].max()) - 90)
    base = q.DeviceRowSet(cols)
    part = q.SliceRowSet(base, offset, n + offset)
    q.profile(True)
    q.profile_read()
    out = run_gpu(spec, [part])
    names = {kk[0] for kk in q.profile_read()}
    q.profile(False)
    got = gpu_rows(out, queries.LINEITEM_OUT_TYPES)
    q.release(out)
    assert "agg_update_sig" in names, names
    want = O.aggregate(spec, [q.HostRowSet([c[offset:offset + n] for c in cols])])
    assert_same_groups(got, want, queries.LINEITEM_OUT_TYPES, nkeys=2)
