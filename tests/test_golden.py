"""The reference's own regression goldens (test/regtest, collected by
tests/golden/make_golden.py) for the queries this library's operators
serve.  Each query is restated as the operator descriptors the engine's
lowering would hand the kernels (fused filter/aggregate, row join, sort,
top-K); the tables are the suites' fixture tables, split into batches of the
suites' Parquet row-group sizes.  The oracle runs on the CPU (these pin the
oracle); the same plans run through the device path under the gpu marker.

Engine behaviour restated here (not in the kernels): ORDER BY over a
grouped result is applied to the returned groups; string predicates become
selection vectors; a cross product is formed before the aggregate.
"""
from __future__ import annotations

import math
from decimal import Decimal

import numpy as np
import pytest

import qumirdb_b200 as q
from oracle import oracle as O
from qumirdb_b200 import abi, queries

from .golden.golden import Table, assert_rows, case, date_str, expected
from .helpers import gpu_rows

ENGINES = ["oracle", pytest.param("gpu", marks=pytest.mark.gpu)]


# ---------------------------------------------------------------------------
# Row sets over fixture columns.
# ---------------------------------------------------------------------------
def rowsets(cols, bounds, engine, selection=None):
    """cols: [(values, valid|None, (type, scale, nullable))] -> one row set per (lo, hi)."""
    out = []
    for lo, hi in bounds:
        data, masks = [], []
        for vals, valid, ty in cols:
            v = vals[lo:hi]
            if ty[0] == abi.BOOL:
                v = np.packbits(np.asarray(v, dtype=bool), bitorder="little")
            data.append(v)
            masks.append(None if valid is None else valid[lo:hi])
        sel = None if selection is None else selection[lo:hi].astype(np.uint8)
        mk = q.DeviceRowSet if engine == "gpu" else q.HostRowSet
        out.append(mk(data, masks, sel, rows=hi - lo))
    return out


def types_of(cols):
    return [c[2] for c in cols]


def normalize(rows, schema):
    """Engine result cells -> the expected schema's Python values."""
    out = []
    for r in rows:
        row = []
        for v, (_, kind, _, scale) in zip(r, schema):
            if v is None:
                row.append(None)
            elif kind in ("dec64", "dec128"):
                row.append(Decimal(int(v)).scaleb(-scale))
            elif kind in ("f32", "f64"):
                row.append(float(v))
            elif kind == "bool":
                row.append(bool(v))
            else:
                row.append(int(v))
        out.append(row)
    return out


# ---------------------------------------------------------------------------
# Aggregate plans.
# ---------------------------------------------------------------------------
def run_aggregate(engine, spec, out_types, cols, bounds):
    rss = rowsets(cols, bounds, engine)
    if engine == "oracle":
        return O.aggregate(spec, rss)
    agg = q.Aggregate(q.compile_aggregate(spec))
    for rs in rss:
        agg.add(rs)
    out = agg.finish()
    rows = gpu_rows(out, out_types)
    q.release(out)
    return rows


def agg_empty_plan(name, t):
    """count(*), count(n)[, sum(n), min(n), max(n), avg(n)] FROM t [WHERE n > 100]
    and SELECT n, count(*) FROM t GROUP BY n (aggregate_empty/*)."""
    n, valid, ty = t.cols["n"]
    e = q.ExprBuilder()
    col = e.col(0, abi.I64)
    filt = e.op(abi.GT, abi.BOOL, col, e.const(100, abi.I64)) if name.startswith("filter") else None
    if name == "grouped_empty":
        spec = queries.AggSpec([ty], e, None, [col], [(abi.COUNT_STAR, -1)])
        return spec, [abi.I64, abi.I64]
    if name.endswith("count"):
        spec = queries.AggSpec([ty], e, filt, [], [(abi.COUNT_STAR, -1), (abi.COUNT, col)])
        return spec, [abi.I64, abi.I64]
    aggs = [(abi.COUNT_STAR, -1), (abi.COUNT, col), (abi.SUM, col), (abi.MIN, col), (abi.MAX, col)]
    o = q.ExprBuilder()
    c = [o.col(k, abi.I64) for k in range(5)]
    avg = o.op(abi.DIV, abi.F64, c[2], o.op(abi.CAST, abi.F64, c[1]))   # sql_lowering.cpp:799-814
    spec = queries.AggSpec([ty], e, filt, [], aggs, c + [avg], o)
    return spec, [abi.I64] * 5 + [abi.F64]


@pytest.mark.parametrize("engine", ENGINES)
@pytest.mark.parametrize("name", ["empty_count", "empty_mixed", "filter_count", "filter_mixed", "nonempty_mixed",
                                  "split_mixed", "all_null_mixed", "nonnullable_empty", "nonnullable_values",
                                  "grouped_empty"])
def test_aggregate_empty_goldens(engine, name):
    key = f"aggregate_empty/{name}"
    t = Table(case(key)["tables"]["t"])
    spec, out_types = agg_empty_plan(name, t)
    rows = run_aggregate(engine, spec, out_types, [t.cols["n"]], t.batches())
    schema, want = expected(key)
    assert_rows(normalize(rows, schema), want)


@pytest.mark.parametrize("engine", ENGINES)
def test_decimal_multiply_sum(engine):
    """SELECT id % 2 AS g, sum(CAST(a AS DECIMAL(10,2)) * CAST(a AS DECIMAL(10,2))),
    sum(CAST(a AS DECIMAL(10,2)) * (1 - CAST(a AS DECIMAL(10,2)))),
    avg(CAST(a AS DECIMAL(10,2)) * CAST(b AS DECIMAL(19,0))), count(*) FROM t
    GROUP BY id % 2 ORDER BY g — product types by DecimalProductSpec
    (annotate_type.cpp:746-760), the integer operand as DECIMAL(19,0)
    (:834-842), avg of a non-cast argument as sum / double count."""
    key = "decimal_result/multiply_sum"
    t = Table(case(key)["tables"]["t"])
    cols = [t.cols["id"], t.cols["a"], t.cols["b"]]
    e = q.ExprBuilder()
    id_, a, b = e.col(0, abi.I32), e.col(1, abi.I32), e.col(2, abi.I64)
    g = e.op(abi.MOD, abi.I32, id_, e.const(2, abi.I32))
    ca = e.op(abi.CAST, abi.DECIMAL64, a, scale=2)                       # DECIMAL(10,2)
    sq = e.op(abi.MUL, abi.DECIMAL128, ca, ca, scale=4)                  # DECIMAL(21,4)
    om = e.op(abi.SUB, abi.DECIMAL128, e.const(1, abi.I64), ca, scale=2)  # DECIMAL(22,2)
    disc = e.op(abi.MUL, abi.DECIMAL128, ca, om, scale=4)                # DECIMAL(33,4)
    cb = e.op(abi.CAST, abi.DECIMAL128, b, scale=0)                      # DECIMAL(19,0)
    ab = e.op(abi.MUL, abi.DECIMAL128, ca, cb, scale=2)                  # DECIMAL(30,2)
    aggs = [(abi.SUM, sq), (abi.SUM, disc), (abi.SUM, ab), (abi.COUNT, ab), (abi.COUNT_STAR, -1)]
    o = q.ExprBuilder()
    c = [o.col(0, abi.I32), o.col(1, abi.DECIMAL128, 4), o.col(2, abi.DECIMAL128, 4), o.col(3, abi.DECIMAL128, 2),
         o.col(4, abi.I64), o.col(5, abi.I64)]
    m = o.op(abi.DIV, abi.F64, c[3], o.op(abi.CAST, abi.F64, c[4]))
    spec = queries.AggSpec(types_of(cols), e, None, [g], aggs, [c[0], c[1], c[2], m, c[5]], o)
    out_types = [abi.I32, abi.DECIMAL128, abi.DECIMAL128, abi.F64, abi.I64]
    rows = run_aggregate(engine, spec, out_types, cols, t.batches())
    schema, want = expected(key)
    got = sorted(normalize(rows, schema), key=lambda r: r[0])
    assert_rows(got, want)


def cross(tables_cols, predicate_rows=None):
    """Cross product of column dicts: [(prefix, {name: col})] -> {prefix.name: col}."""
    sizes = [len(next(iter(cols.values()))[0]) for _, cols in tables_cols]
    grids = np.meshgrid(*[np.arange(n) for n in sizes], indexing="ij")
    idx = [gr.reshape(-1) for gr in grids]
    out = {}
    for (prefix, cols), ix in zip(tables_cols, idx):
        for name, (vals, valid, ty) in cols.items():
            if ty is None:
                continue
            out[f"{prefix}.{name}"] = (vals[ix], None if valid is None else valid[ix], ty)
    return out, len(idx[0])


@pytest.mark.parametrize("engine", ENGINES)
def test_decimal_storage_sum(engine):
    """SELECT sum(CAST(999999999999999999 AS DECIMAL(18,0))), min(CAST(t1.a AS
    DECIMAL(18,2))), max(CAST(t2.a AS DECIMAL(18,2))), count(*) FROM t t1, t t2:
    a DECIMAL(38,0) sum past the i64 range."""
    key = "decimal_result/storage_sum"
    t = Table(case(key)["tables"]["t"])
    x, n = cross([("t1", t.cols), ("t2", t.cols)])
    cols = [x["t1.a"], x["t2.a"]]
    e = q.ExprBuilder()
    a1, a2 = e.col(0, abi.I32), e.col(1, abi.I32)
    k = e.const(999999999999999999, abi.DECIMAL64)
    aggs = [(abi.SUM, k), (abi.MIN, e.op(abi.CAST, abi.DECIMAL64, a1, scale=2)),
            (abi.MAX, e.op(abi.CAST, abi.DECIMAL64, a2, scale=2)), (abi.COUNT_STAR, -1)]
    spec = queries.AggSpec(types_of(cols), e, None, [], aggs)
    rows = run_aggregate(engine, spec, [abi.DECIMAL128, abi.DECIMAL64, abi.DECIMAL64, abi.I64], cols, [(0, n)])
    schema, want = expected(key)
    assert_rows(normalize(rows, schema), want)


def layout_inner(x, nkeys_variant):
    """Inner GROUP BY of aggregate_row_layout over t x, t y, t z WHERE z.id < 4."""
    names = ["x.id", "x.n", "x.v", "x.f", "y.id", "y.v", "y.f", "z.a", "z.v", "z.f"]
    cols = [x[nm] for nm in names]
    e = q.ExprBuilder()
    xid, xn, xv, xf, yid, yv, yf, za, zv, zf = [e.col(k, ty[0]) for k, (_, _, ty) in enumerate(cols)]
    if nkeys_variant == "checksum":
        d = e.op(abi.CAST, abi.DECIMAL128, xid, scale=2)                  # CAST(x.id AS DECIMAL(20,2))
        keys = [d, yid, xn]
        aggs = [(abi.COUNT_STAR, -1), (abi.COUNT, za), (abi.SUM, e.op(abi.ADD, abi.I64, za, yv)),
                (abi.MIN, e.op(abi.SUB, abi.I64, za, xv)), (abi.MAX, e.op(abi.MUL, abi.I64, za, yv)),
                (abi.SUM, e.op(abi.ADD, abi.I64, e.op(abi.MUL, abi.I64, xv, yv), zv)),
                (abi.MIN, zf), (abi.MAX, e.op(abi.ADD, abi.F64, yf, zf)), (abi.SUM, zf)]
        out_types = [abi.DECIMAL128, abi.I64, abi.I64, abi.I64, abi.I64, abi.I64, abi.I64, abi.I64, abi.I64,
                     abi.F64, abi.F64, abi.F64]
        col_types = [(abi.DECIMAL128, 2, 0), (abi.I64,), (abi.I64, 0, 1), (abi.I64,), (abi.I64,), (abi.I64, 0, 1),
                     (abi.I64, 0, 1), (abi.I64, 0, 1), (abi.I64, 0, 1), (abi.F64, 0, 1), (abi.F64, 0, 1),
                     (abi.F64, 0, 1)]
    else:
        keys = [xid, yid]
        aggs = [(abi.COUNT_STAR, -1), (abi.SUM, za), (abi.MIN, zf), (abi.MAX, e.op(abi.ADD, abi.I64, xv, zv))]
        out_types = [abi.I64, abi.I64, abi.I64, abi.I64, abi.F64, abi.I64]
        col_types = [(abi.I64,), (abi.I64,), (abi.I64,), (abi.I64, 0, 1), (abi.F64, 0, 1), (abi.I64, 0, 1)]
    return queries.AggSpec(types_of(cols), e, None, keys, aggs), out_types, col_types, cols


def layout_outer(variant, col_types):
    e = q.ExprBuilder()
    c = [e.col(k, ty[0], ty[1] if len(ty) > 1 else 0) for k, ty in enumerate(col_types)]
    if variant == "checksum":
        # groups, row_count, sum_d, sum_k, sum_n, count_n, count_a, sum_a, min_a, max_a, sum_v, min_f, max_f, sum_f
        aggs = [(abi.COUNT_STAR, -1), (abi.SUM, c[3]), (abi.SUM, c[0]), (abi.SUM, c[1]), (abi.SUM, c[2]),
                (abi.COUNT, c[2]), (abi.SUM, c[4]), (abi.SUM, c[5]), (abi.MIN, c[6]), (abi.MAX, c[7]),
                (abi.SUM, c[8]), (abi.MIN, c[9]), (abi.MAX, c[10]), (abi.SUM, c[11])]
        out = [abi.I64, abi.I64, abi.DECIMAL128, abi.I64, abi.I64, abi.I64, abi.I64, abi.I64, abi.I64, abi.I64,
               abi.I64, abi.F64, abi.F64, abi.F64]
    else:
        # groups, row_count, sum_i, sum_k, sum_a, min_f, max_v
        aggs = [(abi.COUNT_STAR, -1), (abi.SUM, c[2]), (abi.SUM, c[0]), (abi.SUM, c[1]), (abi.SUM, c[3]),
                (abi.MIN, c[4]), (abi.MAX, c[5])]
        out = [abi.I64, abi.I64, abi.I64, abi.I64, abi.I64, abi.F64, abi.I64]
    return queries.AggSpec(col_types, e, None, [], aggs), out


@pytest.mark.parametrize("engine", ENGINES)
@pytest.mark.parametrize("variant", ["checksum", "estimated_groups"])
def test_aggregate_row_layout(engine, variant):
    """Nested aggregates over a three-way cross product (65,536 groups with
    a DECIMAL(20,2) key and a nullable key; nullable SUM/MIN/MAX of ints
    and doubles), then the checksum aggregate over the groups."""
    key = f"aggregate_row_layout/{variant}"
    t = Table(case(key)["tables"]["t"])
    zmask = t.cols["id"][0] < 4
    zcols = {k: (v[0][zmask], None if v[1] is None else v[1][zmask], v[2]) for k, v in t.cols.items()}
    x, n = cross([("x", t.cols), ("y", t.cols), ("z", zcols)])
    spec, out_types, col_types, cols = layout_inner(x, variant)
    inner = run_aggregate(engine, spec, out_types, cols, [(0, n)])
    # The inner groups become the outer input (one batch).
    gcols = []
    for j, ty in enumerate(col_types):
        vals = [r[j] for r in inner]
        valid = np.array([v is not None for v in vals])
        if ty[0] == abi.F64:
            arr = np.array([v if v is not None else 0.0 for v in vals], dtype=np.float64)
        elif ty[0] == abi.DECIMAL128:
            # One (lo, hi) int64 pair per row, so that a row slice is a pair slice.
            arr = np.zeros((len(vals), 2), dtype=np.int64)
            for i, v in enumerate(vals):
                u = int(v or 0) & ((1 << 128) - 1)
                arr[i, 0] = np.uint64(u & ((1 << 64) - 1)).view(np.int64)
                arr[i, 1] = np.uint64(u >> 64).view(np.int64)
        else:
            arr = np.array([v if v is not None else 0 for v in vals], dtype=np.int64)
        gcols.append((arr, valid if len(ty) > 2 and ty[2] else None, ty))
    ospec, oout = layout_outer(variant, col_types)
    rows = run_aggregate(engine, ospec, oout, gcols, [(0, len(inner))])
    schema, want = expected(key)
    assert_rows(normalize(rows, schema), want)


# ---------------------------------------------------------------------------
# Sort plans: (key columns with (desc, nulls_first)), select list, limit, offset.
# Defaults follow PostgreSQL: ASC NULLS LAST, DESC NULLS FIRST.
# ---------------------------------------------------------------------------
def k(col, desc=False, nulls_first=None):
    return (col, desc, desc if nulls_first is None else nulls_first)


SORTS = {
    "sort_i_asc": ("t", [k("i"), k("id")], ["id", "i"], None, 0),
    "sort_i_desc": ("t", [k("i", True), k("id")], ["id", "i"], None, 0),
    "sort_f_asc": ("t", [k("f"), k("id")], ["id", "f"], None, 0),
    "sort_f_desc": ("t", [k("f", True), k("id")], ["id", "f"], None, 0),
    "sort_b_asc": ("t", [k("b"), k("id")], ["id", "b"], None, 0),
    "sort_b_desc": ("t", [k("b", True), k("id")], ["id", "b"], None, 0),
    "sort_date_asc": ("t", [k("d"), k("id")], ["id", "d"], None, 0),
    "sort_date_desc": ("t", [k("d", True), k("id")], ["id", "d"], None, 0),
    "sort_multi_key_mixed": ("t", [k("g", True), k("i"), k("f", True), k("id")], ["id", "g", "i", "f"], None, 0),
    "sort_nulls_first_asc": ("t", [k("i", False, True), k("id")], ["id", "i"], None, 0),
    "sort_nulls_last_desc": ("t", [k("i", True, False), k("id")], ["id", "i"], None, 0),
    "top_asc": ("t", [k("i"), k("id")], ["id", "i"], 6, 0),
    "top_desc": ("t", [k("i", True), k("id")], ["id", "i"], 3, 0),
    "top_double_asc": ("t", [k("f"), k("id")], ["id", "f"], 7, 0),
    "top_explicit": ("t", [k("i", True, False), k("id")], ["id", "i"], 3, 0),
    "top_multi_key": ("t", [k("g"), k("i", True), k("id")], ["id", "g", "i"], 4, 0),
    "top_offset_asc": ("t", [k("i"), k("id")], ["id", "i"], 3, 4),
    "top_offset_desc": ("t", [k("i", True), k("id")], ["id", "i"], 2, 2),
    "big_sort_f_asc": ("big", [k("f"), k("id")], ["id", "f"], None, 0),
    "big_sort_f_desc": ("big", [k("f", True), k("id")], ["id", "f"], None, 0),
    "big_sort_i_asc": ("big", [k("i"), k("id")], ["id", "i"], None, 0),
    "big_sort_i_desc": ("big", [k("i", True), k("id")], ["id", "i"], None, 0),
    "big_top_i_asc": ("big", [k("i"), k("id")], ["id", "i"], 25, 0),
    "big_top_f_desc_offset": ("big", [k("f", True), k("id")], ["id", "f"], 40, 30),
}


def sort_columns(t, names, date_cols=()):
    cols, index = [], {}
    for nm in names:
        vals, valid, ty = t.cols[nm]
        if nm in date_cols:
            ty = (abi.DATE32, 0, ty[2])
        index[nm] = len(cols)
        cols.append((vals, valid, ty))
    return cols, index


def run_sort(engine, cols, index, keys, select, limit, offset, bounds):
    """Sort (or top-K) over a store of batches; returns the selected columns of
    the rows [offset, offset + limit) of the order."""
    spec = queries.SortSpec(types_of(cols), [(index[c], d, nf) for c, d, nf in keys],
                            out_columns=[index[c] for c in select])
    store = rowsets(cols, bounds, engine)
    ids = np.concatenate([(np.int64(b) << 32) | np.arange(hi - lo, dtype=np.int64)
                          for b, (lo, hi) in enumerate(bounds)]) if bounds[-1][1] else np.empty(0, np.int64)
    n = len(ids)
    end = n if limit is None else min(n, offset + limit)
    results = []
    if engine == "oracle":
        for ordered in (O.sort(spec, store, ids), O.top_k(spec, store, ids, end)):
            sel = ordered[offset:end]
            results.append(sel)
        base = np.array([lo for lo, _ in bounds], dtype=np.int64)
        outs = []
        for sel in results:
            pos = base[sel >> 32] + (sel & 0xffffffff)
            rows = []
            for p in pos:
                row = []
                for c in select:
                    vals, valid, ty = cols[index[c]]
                    row.append(None if valid is not None and not valid[p] else vals[p].item())
                rows.append(row)
            outs.append(rows)
        return outs
    s = q.Sort(q.compile_sort(spec), store)
    full = ids.copy()
    s.sort(full)
    outs = []
    out_types = [cols[index[c]][2][0] for c in select]
    r, rs = s.materialize(full, offset, end - offset)
    outs.append(gpu_rows(rs, out_types) if r > 0 else [])
    if r > 0:
        q.release(rs)
    top = ids.copy()
    kk = s.top_k(top, end)
    sl = top[offset:kk]
    r, rs = s.materialize(sl, 0, len(sl))
    outs.append(gpu_rows(rs, out_types) if r > 0 else [])
    if r > 0:
        q.release(rs)
    return outs


def as_expected(rows, select, cols, index, schema):
    out = []
    for r in rows:
        row = []
        for v, c, (_, kind, _, _) in zip(r, select, schema):
            ty = cols[index[c]][2][0]
            if v is None:
                row.append(None)
            elif ty == abi.DATE32:
                row.append(date_str(v))
            elif kind in ("f32", "f64"):
                row.append(float(v))
            elif kind == "bool":
                row.append(bool(v))
            else:
                row.append(int(v))
        out.append(row)
    return out


@pytest.mark.parametrize("engine", ENGINES)
@pytest.mark.parametrize("name", sorted(SORTS))
def test_null_order_default(engine, name):
    key = f"null_order_default/{name}"
    alias, keys, select, limit, offset = SORTS[name]
    t = Table(case(key)["tables"][alias])
    names = list(dict.fromkeys([c for c, _, _ in keys] + select))
    cols, index = sort_columns(t, names, date_cols=("d",))
    schema, want = expected(key)
    for got in run_sort(engine, cols, index, keys, select, limit, offset, t.batches()):
        assert_rows(as_expected(got, select, cols, index, schema), want, rel=0.0)


def float_table(key):
    t = Table(case(key)["tables"]["t"])
    return t, t.cols["id"], t.cols["d"]


@pytest.mark.parametrize("engine", ENGINES)
@pytest.mark.parametrize("name", ["order_asc", "order_desc"])
def test_float_order(engine, name):
    """SELECT id, CAST(d AS REAL) AS f ... ORDER BY f[, DESC], id[ DESC]: NaN
    above +inf, -0 and +0 peers."""
    key = f"float_sql/{name}"
    t, (ids_, _, idty), (d, dvalid, _) = float_table(key)
    f = d.astype(np.float32)
    cols = [(ids_, None, idty), (f, dvalid, (abi.F32, 0, 1))]
    index = {"id": 0, "f": 1}
    desc = name.endswith("desc")
    keys = [k("f", desc), k("id", desc)]
    schema, want = expected(key)
    for got in run_sort(engine, cols, index, keys, ["id", "f"], None, 0, t.batches()):
        assert_rows(as_expected(got, ["id", "f"], cols, index, schema), want, rel=0.0)


def nan_union(t):
    """SELECT id, d FROM t UNION ALL SELECT id + 10, -d FROM t WHERE id IN (3, 4, 5)."""
    ids_, _, idty = t.cols["id"]
    d, dvalid, dty = t.cols["d"]
    pick = np.isin(ids_, [3, 4, 5])
    uid = np.concatenate([ids_, ids_[pick] + 10]).astype(ids_.dtype)
    ud = np.concatenate([d, -d[pick]])
    uvalid = np.concatenate([dvalid, dvalid[pick]])
    return uid, idty, ud, uvalid, dty


@pytest.mark.parametrize("engine", ENGINES)
def test_float_order_nan_limit(engine):
    key = "float_sql/order_nan_limit"
    t = Table(case(key)["tables"]["t"])
    uid, idty, ud, uvalid, dty = nan_union(t)
    cols = [(uid, None, idty), (ud, uvalid, dty)]
    index = {"id": 0, "d": 1}
    schema, want = expected(key)
    for got in run_sort(engine, cols, index, [k("d", True, False), k("id")], ["id", "d"], 10, 0,
                        [(0, len(uid))]):
        assert_rows(as_expected(got, ["id", "d"], cols, index, schema), want, rel=0.0)


@pytest.mark.parametrize("engine", ENGINES)
def test_float_order_nan(engine):
    """Four copies g = 1..4 of the union, each ordered by d in one of the four
    (direction, NULLS) combinations through CASE keys that are NULL for the
    other copies; the CASE columns are formed before the sort."""
    key = "float_sql/order_nan"
    t = Table(case(key)["tables"]["t"])
    uid, idty, ud, uvalid, dty = nan_union(t)
    m = len(uid)
    g = np.repeat(np.arange(1, 5, dtype=np.int32), m)
    cid = np.tile(uid, 4)
    cd = np.tile(ud, 4)
    cvalid = np.tile(uvalid, 4)
    cols = [(g, None, (abi.I32, 0, 0)), (cid, None, idty), (cd, cvalid, dty)]
    index = {"g": 0, "id": 1, "d": 2}
    for j in range(1, 5):
        cols.append((cd, cvalid & (g == j), (abi.F64, 0, 1)))
        index[f"k{j}"] = len(cols) - 1
    keys = [k("g"), k("k1", False, True), k("k2", False, False), k("k3", True, True), k("k4", True, False), k("id")]
    schema, want = expected(key)
    for got in run_sort(engine, cols, index, keys, ["g", "id", "d"], None, 0, [(0, 4 * m)]):
        assert_rows(as_expected(got, ["g", "id", "d"], cols, index, schema), want, rel=0.0)


# ---------------------------------------------------------------------------
# Join plans: SELECT count(*) FROM t a, t b WHERE <equi keys> AND <side filters>.
# ---------------------------------------------------------------------------
JOINS = {
    # name: (build keys, probe keys, build predicate (column, op, value) | selection, probe selection)
    "join_composite_key_filtered": (["grp", "quad"], ["grp", "quad"], ("id", abi.LT, 10), ("id", ">=", 30)),
    "join_shared_key_range": (["id"], ["quad"], ("grp", abi.EQ, 0), None),
    "join_shared_key_range_independent": (["id"], ["quad"], ("tag", "==", "red"), None),
}


@pytest.mark.parametrize("engine", ENGINES)
@pytest.mark.parametrize("name", sorted(JOINS))
def test_selectivity_joins(engine, name):
    key = f"selectivity/{name}"
    t = Table(case(key)["tables"]["t"])
    bkeys, pkeys, bpred, psel = JOINS[name]
    fixed = [c for c, (_, _, ty) in t.cols.items() if ty is not None]
    cols = [t.cols[c] for c in fixed]
    index = {c: j for j, c in enumerate(fixed)}
    be = q.ExprBuilder()
    bsel = None
    bfilter = None
    if isinstance(bpred[1], int):
        col, op, v = bpred
        ty = cols[index[col]][2][0]
        bfilter = be.op(op, abi.BOOL, be.col(index[col], ty), be.const(v, ty))
    else:   # a string predicate: the selection vector of its filter
        vals = t.cols[bpred[0]][0]
        bsel = np.array([x == bpred[2] for x in vals])
    psel_vec = None
    if psel is not None:
        psel_vec = t.cols[psel[0]][0] >= psel[2]
    # The joined row is the probe row (no build payload): the fused
    # join-aggregate reads the probe columns followed by the payload columns.
    jspec = queries.JoinSpec(types_of(cols), types_of(cols), [index[c] for c in bkeys], [index[c] for c in pkeys],
                             [], out=[(0, j) for j in range(len(cols))],
                             build_eb=be if bfilter is not None else None, build_filter=bfilter)
    e = q.ExprBuilder()
    e.col(index[pkeys[0]], cols[index[pkeys[0]]][2][0])
    aspec = queries.AggSpec(types_of(cols), e, None, [], [(abi.COUNT_STAR, -1)], expected_groups=1)
    build = rowsets(cols, t.batches(), engine, bsel)
    probe = rowsets(cols, t.batches(), engine, psel_vec)
    if engine == "oracle":
        rows = O.join_aggregate(jspec, aspec, build, probe)
    else:
        prog = q.compile_join_aggregate(jspec, aspec)
        J = q.RowJoin(prog)
        for rs in build:
            J.append(rs)
        J.build()
        agg = q.Aggregate(prog)
        for rs in probe:
            J.probe_aggregate(agg, rs)
        out = agg.finish()
        rows = gpu_rows(out, [abi.I64])
        q.release(out)
    schema, want = expected(key)
    assert_rows(normalize(rows, schema), want)


# ---------------------------------------------------------------------------
# Outer, SEMI and ANTI row joins (jr_dispatch + jr_materialize): the pairs
# are materialized into the selected columns, then ORDER BY is applied to
# the output rows (NULLs last, the default for ASC).
# ---------------------------------------------------------------------------
def run_row_join(engine, jspec, bcols, pcols, build, probe, pbounds):
    """Output rows of a row join: oracle pairs read back from the host
    columns, or the device join materialized in 16384-row slices."""
    outs = list(zip(jspec.out_side, jspec.out_col))[: jspec.struct.n_out]
    payload = list(jspec.payload)[: jspec.struct.n_payload]
    marks = jspec.join_type in (abi.JOIN_LEFT_SEMI, abi.JOIN_LEFT_ANTI)
    if engine == "oracle":
        rows = []
        for left, right in O.row_join_typed(jspec, build, probe).tolist():
            row = []
            for side, c in outs:
                if side == 0:
                    b, r = left >> 32, left & 0xFFFFFFFF
                    vals, valid, _ = pcols[c]
                    g = pbounds[b][0] + r
                else:
                    vals, valid, _ = bcols[payload[c]]
                    g = right
                ok = g >= 0 and (valid is None or bool(valid[g]))
                row.append(int(vals[g]) if ok else None)
            rows.append(row)
        return rows
    types = [pcols[c][2][0] if side == 0 else bcols[payload[c]][2][0] for side, c in outs]
    J = q.RowJoin(q.compile_row_join(jspec), keeps_null_keys=jspec.join_type == abi.JOIN_LEFT_ANTI)
    for rs in build:
        J.append(rs)
    J.build()
    rows = []

    def drain(stream, n):
        start = 0
        while start < n:
            k, out = J.materialize(stream, start, 16384)
            rows.extend(gpu_rows(out, types))
            q.release(out)
            start += k

    for rs in probe:
        n = J.probe(rs)
        if not marks:
            drain(rs, n)
    if marks:
        drain(None, J.emit_by_mark())
    J.release()
    return rows


def order_rows(rows, by):
    """ORDER BY columns `by` ascending, NULLs last."""
    return sorted(rows, key=lambda r: tuple((1, 0) if r[j] is None else (0, r[j]) for j in by))


OUTER = {
    # name: (preserved table, build table, probe grp filter, build flag filter, output, ORDER BY)
    "duplicates": ("c", "o", None, None, ["ck", "cv", "ok", "ov"], ["cv", "ov"]),
    "null_keys": ("c", "o", 4, None, ["ck", "cv", "ok", "ov"], ["cv", "ov"]),
    "all_matched": ("c", "o", 1, None, ["ck", "cv", "ok", "ov"], ["cv", "ov"]),
    "none_matched": ("c", "o", 2, None, ["ck", "cv", "ok", "ov"], ["cv", "ov"]),
    "empty_build": ("c", "o", 3, None, ["ck", "cv", "ok", "ov"], ["cv", "ov"]),
    "empty_probe": ("c", "o", None, 2, ["ck", "cv", "ok", "ov"], ["cv", "ov"]),
    "right_join": ("c", "o", None, None, ["ok", "ov", "ck", "cv"], ["cv", "ov"]),
    "preserved_larger": ("o", "c", None, None, ["ok", "ov", "ck", "cv"], ["ov", "cv"]),
}


@pytest.mark.parametrize("engine", ENGINES)
@pytest.mark.parametrize("name", sorted(OUTER))
def test_outer_join_goldens(engine, name):
    """c LEFT JOIN o (o RIGHT JOIN c for right_join): the preserved side
    streams through the probe, the null-supplying side is built; a WHERE on
    the preserved side is its selection, an ON condition on the built side
    is the build predicate."""
    key = f"outer_join/{name}"
    pres, bld, grp, flag, select, order = OUTER[name]
    tp, tb = Table(case(key)["tables"][pres]), Table(case(key)["tables"][bld])
    pnames, bnames = list(tp.cols), list(tb.cols)
    pcols, bcols = [tp.cols[c] for c in pnames], [tb.cols[c] for c in bnames]
    be = q.ExprBuilder()
    bfilter = None
    if flag is not None:
        bfilter = be.op(abi.EQ, abi.BOOL, be.col(bnames.index("flag"), abi.I64), be.const(flag, abi.I64))
    psel = None if grp is None else (tp.cols["grp"][0] == grp)
    out = [(0, pnames.index(c)) if c in pnames else (1, bnames.index(c)) for c in select]
    right = name == "right_join"
    jspec = queries.JoinSpec(types_of(bcols), types_of(pcols), [0], [0], list(range(len(bcols))), out=out,
                             build_eb=be if bfilter is not None else None, build_filter=bfilter,
                             join_type=abi.JOIN_RIGHT if right else abi.JOIN_LEFT, build_is_left=1 if right else 0)
    build = rowsets(bcols, tb.batches(), engine)
    probe = rowsets(pcols, tp.batches(), engine, psel)
    rows = run_row_join(engine, jspec, bcols, pcols, build, probe, tp.batches())
    schema, want = expected(key)
    assert_rows(normalize(order_rows(rows, [select.index(c) for c in order]), schema), want)


@pytest.mark.parametrize("engine", ENGINES)
@pytest.mark.parametrize("kind", ["semi", "anti"])
def test_exists_build_outer_side(engine, kind):
    """SELECT id FROM t WHERE [NOT] EXISTS (SELECT 1 FROM w WHERE w.k = t.a):
    LEFT_SEMI / LEFT_ANTI building t (its NULL key kept by the ANTI join);
    the golden's residual variants are other join programs."""
    key = "anti_join_conditions/exists_build_outer_side"
    t, w = Table(case(key)["tables"]["t"]), Table(case(key)["tables"]["w"])
    tnames = list(t.cols)
    bcols, pcols = [t.cols[c] for c in tnames], [w.cols["k"], w.cols["v"]]
    jt = abi.JOIN_LEFT_SEMI if kind == "semi" else abi.JOIN_LEFT_ANTI
    jspec = queries.JoinSpec(types_of(bcols), types_of(pcols), [tnames.index("a")], [0], [tnames.index("id")],
                             out=[(1, 0)], join_type=jt, build_is_left=1)
    rows = run_row_join(engine, jspec, bcols, pcols, rowsets(bcols, t.batches(), engine),
                        rowsets(pcols, w.batches(), engine), w.batches())
    schema, want = expected(key)
    want = sorted(int(r[1]) for r in want if r[0] == kind)
    assert sorted(r[0] for r in rows) == want


@pytest.mark.parametrize("engine", ENGINES)
def test_not_exists_filter_above(engine):
    """SELECT id FROM t WHERE NOT EXISTS (SELECT 1 FROM s WHERE s.k = t.id
    AND s.v > 4) AND t.b > 15: LEFT_ANTI building t with b > 15 fused into
    Append, probing s with the selection of v > 4."""
    key = "anti_join_conditions/not_exists_filter_above"
    t, s = Table(case(key)["tables"]["t"]), Table(case(key)["tables"]["s"])
    tnames = list(t.cols)
    bcols, pcols = [t.cols[c] for c in tnames], [s.cols["k"], s.cols["v"]]
    be = q.ExprBuilder()
    bfilter = be.op(abi.GT, abi.BOOL, be.col(tnames.index("b"), abi.I64), be.const(15, abi.I64))
    jspec = queries.JoinSpec(types_of(bcols), types_of(pcols), [tnames.index("id")], [0], [tnames.index("id")],
                             out=[(1, 0)], build_eb=be, build_filter=bfilter, join_type=abi.JOIN_LEFT_ANTI,
                             build_is_left=1)
    psel = s.cols["v"][0] > 4
    rows = run_row_join(engine, jspec, bcols, pcols, rowsets(bcols, t.batches(), engine),
                        rowsets(pcols, s.batches(), engine, psel), s.batches())
    schema, want = expected(key)
    assert sorted(r[0] for r in rows) == sorted(int(r[0]) for r in want)
