"""Device equi-join build / probe, pair emission, materialize and the fused
join-aggregate against the oracle."""
import numpy as np
import pytest

import qumirdb_b200 as q
from oracle import oracle as O
from qumirdb_b200 import abi, queries

from .helpers import assert_same_groups, gpu_rows, join_data

pytestmark = pytest.mark.gpu


def run_join_sum(b, p, attr_lt=20, device=False):
    jspec, aspec = queries.join_sum(attr_lt)
    prog = q.compile_join_aggregate(jspec, aspec)
    J = q.RowJoin(prog)
    mk = q.DeviceRowSet if device else q.HostRowSet
    J.append(mk(b))
    J.build()
    agg = q.Aggregate(prog)
    J.probe_aggregate(agg, mk(p))
    out = agg.finish()
    rows = gpu_rows(out, [abi.I64, abi.I64])
    q.release(out)
    return rows, jspec, aspec


@pytest.mark.parametrize("build,probe", [(1000, 5000), (200_000, 1_000_000)])
def test_join_sum_matches_oracle(build, probe):
    b, p = join_data(build, probe, int(build * 1.25))
    got, jspec, aspec = run_join_sum(b, p)
    want = O.join_aggregate(jspec, aspec, [q.HostRowSet(b)], [q.HostRowSet(p)])
    assert got == want
    # Plain numpy restatement of the query as a cross-check.
    keep = b[2] < 20
    lookup = dict(zip(b[0][keep].tolist(), b[1][keep].tolist()))
    s = c = 0
    for fk, v in zip(p[0].tolist(), p[1].tolist()):
        if fk in lookup:
            s += lookup[fk] * v
            c += 1
    assert got == [[s, c]]


def test_join_sum_full_size_device_resident():
    b, p = join_data(2_000_000, 120_000_000, 2_500_000)
    got, jspec, aspec = run_join_sum(b, p, device=True)
    keep = b[2] < 20
    pay = np.zeros(2_500_001, dtype=np.int64)
    hit = np.zeros(2_500_001, dtype=bool)
    pay[b[0][keep]] = b[1][keep]
    hit[b[0][keep]] = True
    m = hit[p[0]]
    want_sum = int((pay[p[0]][m].astype(np.int64) * p[1][m]).sum())
    assert got == [[want_sum, int(m.sum())]]


def test_duplicate_build_keys_and_null_keys():
    rng = np.random.default_rng(3)
    bk = rng.integers(0, 50, 3000).astype(np.int64)
    bp = np.arange(3000, dtype=np.int64)
    ba = rng.integers(0, 100, 3000).astype(np.int32)
    pk = rng.integers(-5, 60, 8000).astype(np.int64)
    pv = rng.integers(1, 100, 8000).astype(np.int64)
    bmask = rng.random(3000) > 0.05
    pmask = rng.random(8000) > 0.05
    jspec, aspec = queries.join_sum(50)
    prog = q.compile_join_aggregate(jspec, aspec)
    J = q.RowJoin(prog)
    brs = q.HostRowSet([bk, bp, ba], masks=[bmask, None, None])
    prs = q.HostRowSet([pk, pv], masks=[pmask, None])
    J.append(brs)
    J.build()
    agg = q.Aggregate(prog)
    J.probe_aggregate(agg, prs)
    out = agg.finish()
    got = gpu_rows(out, [abi.I64, abi.I64])
    q.release(out)
    want = O.join_aggregate(jspec, aspec, [brs], [prs])
    assert got == want


@pytest.mark.parametrize("dups", [False, True])
def test_pair_probe_and_materialize(dups):
    """Pairs in the engine's emission order, compared without sorting: probe
    rows ascending, a probe row's build rows in append order (the chain order
    of jr_build_rows / jr_probe_candidates, join_rows.oz:70-197), then
    materialized in 1000-row slices."""
    b, p = join_data(5000, 20_000, 6000)
    if dups:
        rng = np.random.default_rng(4)
        b[0] = rng.integers(1, 800, len(b[0])).astype(np.int64)   # ~6 build rows per key
        b[1] = np.arange(1, len(b[0]) + 1, dtype=np.int64)         # payload names the build row
        p[0][::13] = -1                                              # keys that match nothing
    jspec, _ = queries.join_sum(20)
    prog = q.compile_row_join(jspec)
    J = q.RowJoin(prog)
    brs, prs = q.HostRowSet(b), q.HostRowSet(p)
    J.append(brs)
    J.build()
    n = J.probe(prs)
    want = O.row_join(jspec, [brs], prs)
    assert n == len(want)
    got = []
    start = 0
    while start < n:
        k, out = J.materialize(prs, start, 1000)
        vals, _ = q.read_rowset(out, [abi.I64, abi.I64, abi.I64])
        got.extend(zip(*(v.tolist() for v in vals)))
        q.release(out)
        start += k
    keep = b[2] < 20
    arena_payload = b[1][keep]
    want_rows = [(int(p[0][r]), int(p[1][r]), int(arena_payload[br])) for r, br in want]
    assert got == want_rows


def _shape_aggs(e, name):
    """Aggregates over the joined row (fk, value, payload) for one shape."""
    fk, val, pay = e.col(0, abi.I64), e.col(1, abi.I64), e.col(2, abi.I64)
    mul = lambda a, b: e.op(abi.MUL, abi.I64, a, b)
    add = lambda a, b: e.op(abi.ADD, abi.I64, a, b)
    sub = lambda a, b: e.op(abi.SUB, abi.I64, a, b)
    c = lambda v: e.const(v, abi.I64)
    return {
        "count": [(abi.COUNT_STAR, -1)],
        "sum_pay": [(abi.SUM, pay)],
        "sum_val": [(abi.SUM, val)],
        "sum_val_pay": [(abi.SUM, mul(val, pay))],
        "count_sum": [(abi.COUNT_STAR, -1), (abi.SUM, mul(pay, val))],
        "sum_val_count": [(abi.SUM, val), (abi.COUNT_STAR, -1)],
        "affine": [(abi.SUM, mul(add(pay, c(7)), sub(val, c(3)))), (abi.COUNT_STAR, -1)],
        "sum_val_sq": [(abi.SUM, mul(val, val))],
        "three_states": [(abi.SUM, val), (abi.SUM, pay), (abi.COUNT_STAR, -1)],
        "fk_factor": [(abi.SUM, mul(fk, pay))],
    }[name]


@pytest.mark.parametrize("shape", ["count", "sum_pay", "sum_val", "sum_val_pay", "count_sum", "sum_val_count",
                                   "affine", "sum_val_sq", "three_states", "fk_factor"])
def test_join_aggregate_shapes(shape):
    """Every compile-time state signature of the join-sum kernel, and the
    runtime-interpreted fold, against the oracle on a probe that spans whole
    staged tiles plus a ragged tail."""
    b, p = join_data(300_000, 2_000_000 + 777, 375_000)
    jspec, _ = queries.join_sum(20)
    e = q.ExprBuilder()
    aggs = _shape_aggs(e, shape)
    aspec = queries.AggSpec([(abi.I64,), (abi.I64,), (abi.I64,)], e, None, [], aggs, expected_groups=1)
    prog = q.compile_join_aggregate(jspec, aspec)
    J = q.RowJoin(prog)
    J.append(q.DeviceRowSet(b))
    J.build()
    agg = q.Aggregate(prog)
    J.probe_aggregate(agg, q.DeviceRowSet(p))
    out = agg.finish()
    got = gpu_rows(out, [abi.I64] * len(aggs))
    q.release(out)
    want = O.join_aggregate(jspec, aspec, [q.HostRowSet(b)], [q.HostRowSet(p)])
    assert got == want


@pytest.mark.parametrize("keys", ["dense", "dense_negative", "spans_marker", "sparse", "duplicates"])
def test_join_sum_build_key_layouts(keys):
    """The fused join-sum over build keys that do and do not get the
    direct-address index (unique keys over a dense range; a range holding the
    empty marker -1, sparse 64-bit keys and duplicate keys keep the hashed
    table), each equal to the oracle; probe keys also fall outside the range."""
    rng = np.random.default_rng(40)
    nb, npr = 50_000, 1_500_017
    if keys == "dense":
        bk = rng.permutation(nb).astype(np.int64) + 1000
    elif keys == "dense_negative":
        bk = -(rng.permutation(nb).astype(np.int64) + 2)           # -2 .. -nb-1
    elif keys == "spans_marker":
        bk = rng.permutation(nb).astype(np.int64) - nb // 2         # includes -1
    elif keys == "sparse":
        bk = rng.integers(-2**62, 2**62, nb, dtype=np.int64)
    else:
        bk = rng.integers(1000, 1000 + nb // 3, nb).astype(np.int64)
    b = [bk, rng.integers(1, 10**6, nb).astype(np.int64), rng.integers(0, 100, nb).astype(np.int32)]
    lo, hi = int(bk.min()), int(bk.max())
    span = hi - lo + 1
    other = max(lo - span, -2**63), min(hi + span, 2**63 - 1)
    pk = np.where(rng.random(npr) < 0.7, rng.choice(bk, npr), rng.integers(other[0], other[1], npr)).astype(np.int64)
    p = [pk, rng.integers(1, 10**4, npr).astype(np.int64)]
    jspec, aspec = queries.join_sum(60)
    prog = q.compile_join_aggregate(jspec, aspec)
    J = q.RowJoin(prog)
    J.append(q.DeviceRowSet(b))
    J.build()
    agg = q.Aggregate(prog)
    J.probe_aggregate(agg, q.DeviceRowSet(p))
    out = agg.finish()
    got = gpu_rows(out, [abi.I64, abi.I64])
    q.release(out)
    want = O.join_aggregate(jspec, aspec, [q.HostRowSet(b)], [q.HostRowSet(p)])
    assert got == want


@pytest.mark.parametrize("attr_lt", [20, 100])
def test_join_sum_partitioned_build_and_probe_40m(attr_lt):
    """A 40M-row build whose bucket table is larger than L2 (256 MB with
    attr < 20, 1.3 GB with every row kept): the build is radix-partitioned by
    bucket and inserted slice by slice, the probe rows are partitioned the
    same way and probed one L2-sized slice per launch; the result equals the
    oracle's."""
    b, p = join_data(40_000_000, 20_000_000, 50_000_000, seed=41)
    jspec, aspec = queries.join_sum(attr_lt)
    prog = q.compile_join_aggregate(jspec, aspec)
    J = q.RowJoin(prog)
    J.append(q.DeviceRowSet(b))
    J.build()
    agg = q.Aggregate(prog)
    q.profile(True)
    q.profile_read()
    J.probe_aggregate(agg, q.DeviceRowSet(p))
    names = [k[0] for k in q.profile_read()]
    q.profile(False)
    out = agg.finish()
    got = gpu_rows(out, [abi.I64, abi.I64])
    q.release(out)
    assert "join_part_scatter" in names and names.count("join_agg_probe") > 1, names
    want = O.join_aggregate(jspec, aspec, [q.HostRowSet(b)], [q.HostRowSet(p)])
    assert got == want


def _typed_join_data(seed, nb, np_, nbatches):
    rng = np.random.default_rng(seed)
    bk = rng.integers(0, nb // 3, nb).astype(np.int64)             # ~3 build rows per key
    bp = np.arange(nb, dtype=np.int64) * 7 + 1                      # payload names the build row
    ba = rng.integers(0, 100, nb).astype(np.int32)
    bvalid = rng.random(nb) > 0.04
    pk = rng.integers(-50, nb // 3 + 50, np_).astype(np.int64)
    pv = rng.integers(1, 1000, np_).astype(np.int64)
    pvalid = rng.random(np_) > 0.04
    psel = (rng.random(np_) > 0.1).astype(np.uint8)
    b = [bk, bp, ba]
    p = [pk, pv]
    bounds = [(i * np_ // nbatches, (i + 1) * np_ // nbatches) for i in range(nbatches)]
    return b, bvalid, p, pvalid, psel, bounds


def _canonical(pairs, lo, pvalid):
    """The oracle's pairs in the device's order.  The reference defers a
    probe row whose seek meets a salt collision to a later key pass; the
    device's bucket table has no salts, so within one probe batch the NULL-key
    pads come first (as the collect pass emits them), then rows in row
    order, each row's build rows in chain (build) order.  A stable sort by
    (batch, not a NULL-key pad, row) maps one order onto the other without
    reordering any row's own pairs."""
    def key(lr):
        left, right = lr
        batch, row = left >> 32, left & 0xFFFFFFFF
        pad = right < 0 and not pvalid[lo[batch] + row]
        return (batch, 0 if pad else 1, row)
    return sorted(pairs, key=key)


@pytest.mark.parametrize("join_type,build_is_left", [(abi.JOIN_LEFT, 0), (abi.JOIN_RIGHT, 1)])
def test_outer_join_pairs_against_oracle(join_type, build_is_left):
    """LEFT (right side built) and RIGHT (left side built): every selected
    probe row appears, unmatched and NULL-key rows once with NULL build
    columns; duplicate keys, NULLs on both sides, a build predicate and a
    probe selection, over three probe batches."""
    b, bvalid, p, pvalid, psel, bounds = _typed_join_data(11, 30_000, 120_000, 3)
    jspec, _ = queries.join_sum(60)
    jspec = queries.JoinSpec(queries.JOIN_BUILD_COLUMNS_NULLABLE, queries.JOIN_PROBE_COLUMNS_NULLABLE, [0], [0],
                             [1], out=[(0, 0), (0, 1), (1, 0)], build_eb=jspec.build_eb,
                             build_filter=jspec.struct.build_filter, join_type=join_type,
                             build_is_left=build_is_left)
    brs = q.HostRowSet(b, masks=[bvalid, None, None])
    prs = [q.HostRowSet([c[lo:hi] for c in p], masks=[pvalid[lo:hi], None], selection=psel[lo:hi])
           for lo, hi in bounds]
    want = O.row_join_typed(jspec, [brs], prs).tolist()
    J = q.RowJoin(q.compile_row_join(jspec))
    J.append(brs)
    J.build()
    got = []
    for bi, rs in enumerate(prs):
        n = J.probe(rs)
        start = 0
        while start < n:
            k, out = J.materialize(rs, start, 16384)
            vals, valid = q.read_rowset(out, [abi.I64, abi.I64, abi.I64])
            for r in range(k):
                got.append(tuple(int(vals[c][r]) if valid[c][r] else None for c in range(3)))
            q.release(out)
            start += k
    J.release()
    lo = [b0 for b0, _ in bounds]
    exp = []
    for left, right in _canonical(want, lo, pvalid):
        g = lo[left >> 32] + (left & 0xFFFFFFFF)
        fk = int(p[0][g]) if pvalid[g] else None
        exp.append((fk, int(p[1][g]), None if right < 0 else int(b[1][right])))
    assert len(got) == len(exp)
    assert got == exp
    assert any(r[2] is None and r[0] is None for r in got) and any(r[2] is None and r[0] is not None for r in got)


@pytest.mark.parametrize("join_type", [abi.JOIN_LEFT_SEMI, abi.JOIN_LEFT_ANTI])
def test_semi_anti_join_against_oracle(join_type):
    """LEFT_SEMI / LEFT_ANTI building the left side: probes mark the build
    rows they match across three probe batches; EMIT_BY_MARK lists the
    marked (SEMI) or unmarked (ANTI) rows in build order, then an ANTI join's
    NULL-key rows from its second arena; only build columns come out."""
    b, bvalid, p, pvalid, psel, bounds = _typed_join_data(12, 30_000, 60_000, 3)
    base, _ = queries.join_sum(60)
    jspec = queries.JoinSpec(queries.JOIN_BUILD_COLUMNS_NULLABLE, queries.JOIN_PROBE_COLUMNS_NULLABLE, [0], [0],
                             [1, 0], out=[(1, 0), (1, 1)], build_eb=base.build_eb,
                             build_filter=base.struct.build_filter, join_type=join_type, build_is_left=1)
    brs = q.HostRowSet(b, masks=[bvalid, None, None])
    prs = [q.HostRowSet([c[lo:hi] for c in p], masks=[pvalid[lo:hi], None], selection=psel[lo:hi])
           for lo, hi in bounds]
    want = O.row_join_typed(jspec, [brs], prs).tolist()
    J = q.RowJoin(q.compile_row_join(jspec), keeps_null_keys=join_type == abi.JOIN_LEFT_ANTI)
    J.append(brs)
    J.build()
    for rs in prs:
        assert J.probe(rs) == 0
    n = J.emit_by_mark()
    got = []
    start = 0
    while start < n:
        k, out = J.materialize(None, start, 16384)
        vals, valid = q.read_rowset(out, [abi.I64, abi.I64])
        got.extend((int(vals[0][r]), int(vals[1][r]) if valid[1][r] else None) for r in range(k))
        q.release(out)
        start += k
    J.release()
    exp = [(int(b[1][br]), int(b[0][br]) if bvalid[br] else None) for _, br in want]
    assert got == exp
    if join_type == abi.JOIN_LEFT_ANTI:
        assert any(v is None for _, v in got)   # NULL-key build rows are kept


def test_typed_join_compile_rejects_unserved_shapes():
    base, _ = queries.join_sum(20)
    for jt, left in [(abi.JOIN_FULL, 0), (abi.JOIN_LEFT, 1), (abi.JOIN_RIGHT, 0), (abi.JOIN_LEFT_SEMI, 0),
                     (abi.JOIN_RIGHT_ANTI, 1)]:
        spec = queries.JoinSpec(queries.JOIN_BUILD_COLUMNS, queries.JOIN_PROBE_COLUMNS, [0], [0], [1],
                                out=[(1, 0)], join_type=jt, build_is_left=left)
        with pytest.raises(q.QdbError):
            q.compile_row_join(spec)


@pytest.mark.parametrize("with_selection", [False, True])
def test_batched_joins_match_each_join(with_selection):
    """Many uneven joins of the join-sum program: one batched build and one
    persistent probe launch give every join the oracle's SUM / COUNT (a
    selection on a probe batch takes the one-by-one path, same results)."""
    rng = np.random.default_rng(21)
    jspec, aspec = queries.join_sum(40)
    prog = q.compile_join_aggregate(jspec, aspec)
    n = 200
    jb = q.RowJoinBatch(prog, n)
    builds, probes = [], []
    for i in range(n):
        nb = int(rng.integers(10, 20_000))
        npr = int(rng.integers(1, 200_000))
        b, p = join_data(nb, npr, int(nb * 1.3) + 1)
        if i % 17 == 0:
            b[0][: nb // 3] = b[0][0]            # duplicate build keys
        if i % 23 == 0:
            p[0][::7] = -1                       # the empty-key marker of the table, as a key
        sel = (rng.random(npr) > 0.5).astype(np.uint8) if with_selection and i == 5 else None
        brs, prs = q.HostRowSet(b), q.DeviceRowSet(p, selection=sel)
        if i % 2:
            jb.append(i, brs)
        builds.append(brs)
        probes.append((prs, q.HostRowSet(p, selection=sel)))
    empty = q.HostRowSet([np.empty(0, np.int64), np.empty(0, np.int64), np.empty(0, np.int32)])
    # Even joins take their build rows in one batched append (odd ones were appended one by one).
    jb.append_all([builds[i] if i % 2 == 0 else empty for i in range(n)])
    jb.build()
    jb.probe_aggregate([p for p, _ in probes])
    outs = jb.finish()
    for i, out in enumerate(outs):
        got = gpu_rows(out, [abi.I64, abi.I64])
        q.release(out)
        want = O.join_aggregate(jspec, aspec, [builds[i]], [probes[i][1]])
        assert got == want, i
    jb.release()
