"""Operator descriptors of the benchmark workloads, as the engine's lowering
would fill them from TOperatorKernelSpec (qdb/kernel/spec.h:65-90).

* lineitem_agg: scan -> filter (shipdate <= cutoff) -> project
  (price*(100-disc), price*(100-disc)*(100+tax)) -> GROUP BY flag, status with
  SUM/AVG/COUNT; AVG lowered to SUM / COUNT (qdb/plan/sql_lowering.cpp:799-814);
  decimal products typed by DecimalProductSpec (qdb/kernel/annotate_type.cpp:746-760).
* join_sum: build (key, payload, attr) filtered by attr < 20, probe (fk, value),
  SELECT SUM(payload * value), COUNT(*).
* zipf_agg: GROUP BY key: COUNT, SUM(a), MIN(a), MAX(a), SUM(x).
"""
from __future__ import annotations

import ctypes as C

from . import abi
from . import ExprBuilder, coltypes, i32s


class AggSpec:
    """qdb_aggregate_spec plus the arrays it points at."""

    def __init__(self, columns, eb: ExprBuilder, filter_node, keys, aggs, outputs=None, out_eb=None, flags=0,
                 expected_groups=0):
        self.columns = coltypes(columns)
        self.eb = eb
        self.nodes = eb.array()
        self.keys = i32s(keys)
        self.aggs = (abi.AggItem * max(1, len(aggs)))()
        for k, (f, a) in enumerate(aggs):
            self.aggs[k].func, self.aggs[k].arg = f, a
        self.outputs = i32s(outputs or [])
        self.out_eb = out_eb
        self.out_nodes = out_eb.array() if out_eb else (abi.Expr * 1)()
        s = abi.AggregateSpec()
        s.n_columns, s.columns = len(columns), self.columns
        s.n_nodes, s.nodes = len(eb.nodes), self.nodes
        s.filter = -1 if filter_node is None else filter_node
        s.n_keys, s.keys = len(keys), self.keys
        s.n_aggs, s.aggs = len(aggs), self.aggs
        s.n_outputs, s.outputs = len(outputs or []), self.outputs
        s.n_output_nodes, s.output_nodes = (len(out_eb.nodes) if out_eb else 0), self.out_nodes
        s.flags = flags
        s.expected_groups = expected_groups
        self.struct = s
        self.column_types = list(columns)


class JoinSpec:
    def __init__(self, build_columns, probe_columns, build_keys, probe_keys, payload, out=(), build_eb=None,
                 build_filter=None, flags=0, join_type=0, build_is_left=0):
        self.bcols = coltypes(build_columns)
        self.pcols = coltypes(probe_columns)
        self.bkeys = i32s(build_keys)
        self.pkeys = i32s(probe_keys)
        self.payload = i32s(payload)
        self.out_side = i32s([s for s, _ in out])
        self.out_col = i32s([c for _, c in out])
        self.build_eb = build_eb
        self.bnodes = build_eb.array() if build_eb else (abi.Expr * 1)()
        s = abi.RowJoinSpec()
        s.join_type = join_type
        s.build_is_left = build_is_left
        s.n_build_columns, s.build_columns = len(build_columns), self.bcols
        s.n_probe_columns, s.probe_columns = len(probe_columns), self.pcols
        s.n_keys, s.build_keys, s.probe_keys = len(build_keys), self.bkeys, self.pkeys
        s.n_payload, s.build_payload = len(payload), self.payload
        s.n_out, s.out_side, s.out_column = len(out), self.out_side, self.out_col
        s.n_build_nodes, s.build_nodes = (len(build_eb.nodes) if build_eb else 0), self.bnodes
        s.build_filter = -1 if build_filter is None else build_filter
        s.flags = flags
        self.struct = s
        self.join_type = join_type


# Column order of the lineitem-shaped table.
LINEITEM_COLUMNS = [(abi.I64,), (abi.DECIMAL64, 2), (abi.I64,), (abi.I64,), (abi.CHAR1,), (abi.CHAR1,),
                    (abi.DATE32,)]
LINEITEM_OUT_TYPES = [abi.CHAR1, abi.CHAR1, abi.I64, abi.DECIMAL128, abi.DECIMAL128, abi.DECIMAL128, abi.F64,
                      abi.DECIMAL128, abi.F64, abi.I64]
LINEITEM_OUT_SCALES = [0, 0, 0, 2, 2, 2, 0, 2, 0, 0]


def lineitem_agg(cutoff: int, flags: int = 0) -> AggSpec:
    """GROUP BY flag, status over rows with shipdate <= cutoff:
    sum_qty, sum_base_price, sum_disc_price, sum_charge, avg_qty, avg_price,
    avg_disc, count_order."""
    e = ExprBuilder()
    qty = e.col(0, abi.I64)
    price = e.col(1, abi.DECIMAL64, 2)
    disc = e.col(2, abi.I64)
    tax = e.col(3, abi.I64)
    flag = e.col(4, abi.CHAR1)
    status = e.col(5, abi.CHAR1)
    ship = e.col(6, abi.DATE32)
    pred = e.op(abi.LE, abi.BOOL, ship, e.const(cutoff, abi.DATE32))
    hundred = e.const(100, abi.I64)
    one_minus = e.op(abi.SUB, abi.I64, hundred, disc)                          # 100 - disc
    disc_price = e.op(abi.MUL, abi.DECIMAL128, price, one_minus, scale=2)      # DECIMAL(34,2)
    one_plus = e.op(abi.ADD, abi.I64, hundred, tax)                            # 100 + tax
    charge = e.op(abi.MUL, abi.DECIMAL128, disc_price, one_plus, scale=2)      # DECIMAL(38,2)
    aggs = [(abi.SUM, qty), (abi.SUM, price), (abi.SUM, disc_price), (abi.SUM, charge),
            (abi.COUNT, qty), (abi.COUNT, price), (abi.SUM, disc), (abi.COUNT, disc), (abi.COUNT_STAR, -1)]
    # Row: flag, status, sum_qty, sum_price, sum_dp, sum_charge, cnt_qty, cnt_price, sum_disc, cnt_disc, cnt.
    o = ExprBuilder()
    c = [o.col(0, abi.CHAR1), o.col(1, abi.CHAR1), o.col(2, abi.I64), o.col(3, abi.DECIMAL128, 2),
         o.col(4, abi.DECIMAL128, 2), o.col(5, abi.DECIMAL128, 2), o.col(6, abi.I64), o.col(7, abi.I64),
         o.col(8, abi.I64), o.col(9, abi.I64), o.col(10, abi.I64)]
    avg_qty = o.op(abi.DIV, abi.F64, c[2], o.op(abi.CAST, abi.F64, c[6]))
    avg_price = o.op(abi.DIV, abi.DECIMAL128, c[3], c[7], scale=2)
    avg_disc = o.op(abi.DIV, abi.F64, c[8], o.op(abi.CAST, abi.F64, c[9]))
    outputs = [c[0], c[1], c[2], c[3], c[4], c[5], avg_qty, avg_price, avg_disc, c[10]]
    return AggSpec(LINEITEM_COLUMNS, e, pred, [flag, status], aggs, outputs, o, flags=flags, expected_groups=8)


JOIN_BUILD_COLUMNS = [(abi.I64,), (abi.I64,), (abi.I32,)]
JOIN_PROBE_COLUMNS = [(abi.I64,), (abi.I64,)]
# The same schemas with nullable key columns.
JOIN_BUILD_COLUMNS_NULLABLE = [(abi.I64, 0, 1), (abi.I64,), (abi.I32,)]
JOIN_PROBE_COLUMNS_NULLABLE = [(abi.I64, 0, 1), (abi.I64,)]


def join_sum(attr_lt: int = 20, flags: int = 0) -> tuple[JoinSpec, AggSpec]:
    """SELECT SUM(b.payload * p.value), COUNT(*) FROM probe p JOIN build b
    ON p.fk = b.key WHERE b.attr < attr_lt (build filter fused into Append)."""
    be = ExprBuilder()
    bf = be.op(abi.LT, abi.BOOL, be.col(2, abi.I32), be.const(attr_lt, abi.I32))
    j = JoinSpec(JOIN_BUILD_COLUMNS, JOIN_PROBE_COLUMNS, [0], [0], [1], out=[(0, 0), (0, 1), (1, 0)],
                 build_eb=be, build_filter=bf, flags=flags)
    e = ExprBuilder()   # joined row: fk, value, payload
    prod = e.op(abi.MUL, abi.I64, e.col(2, abi.I64), e.col(1, abi.I64))
    a = AggSpec([(abi.I64,), (abi.I64,), (abi.I64,)], e, None, [], [(abi.SUM, prod), (abi.COUNT_STAR, -1)],
                flags=flags, expected_groups=1)
    return j, a


ZIPF_COLUMNS = [(abi.I64,), (abi.I64,), (abi.F64,)]
ZIPF_OUT_TYPES = [abi.I64, abi.I64, abi.I64, abi.I64, abi.I64, abi.F64]


def zipf_agg(expected_groups: int = 0, flags: int = 0) -> AggSpec:
    """GROUP BY key: COUNT(*), SUM(a), MIN(a), MAX(a), SUM(x)."""
    e = ExprBuilder()
    key = e.col(0, abi.I64)
    a = e.col(1, abi.I64)
    x = e.col(2, abi.F64)
    aggs = [(abi.COUNT_STAR, -1), (abi.SUM, a), (abi.MIN, a), (abi.MAX, a), (abi.SUM, x)]
    return AggSpec(ZIPF_COLUMNS, e, None, [key], aggs, flags=flags, expected_groups=expected_groups)


class SortSpec:
    """qdb_sort_spec plus the arrays it points at.  keys: (column, desc,
    nulls_first), most significant first."""

    def __init__(self, columns, keys, out_columns=None, flags=0):
        self.columns = coltypes(columns)
        self.keys = (abi.SortKey * max(1, len(keys)))()
        for k, key in enumerate(keys):
            col, desc, nulls_first = (tuple(key) + (0, 0))[:3]
            self.keys[k].column, self.keys[k].desc, self.keys[k].nulls_first = col, int(desc), int(nulls_first)
        outs = list(range(len(columns))) if out_columns is None else list(out_columns)
        self.out = i32s(outs)
        s = abi.SortSpec()
        s.n_columns, s.columns = len(columns), self.columns
        s.n_keys, s.keys = len(keys), self.keys
        s.n_out, s.out_columns = len(outs), self.out
        s.flags = flags
        self.struct = s
        self.column_types = list(columns)
        self.out_columns = outs


SORT_COLUMNS = [(abi.I64,), (abi.I32,), (abi.I64,)]


def sort_k1_desc_k2(flags: int = 0) -> SortSpec:
    """ORDER BY k1 DESC, k2 ASC over (k1 i64, k2 i32, rowid i64); ties keep
    input order."""
    return SortSpec(SORT_COLUMNS, [(0, 1, 0), (1, 0, 0)], flags=flags)


def top_k1(flags: int = 0) -> SortSpec:
    """ORDER BY k1 (the LIMIT is the top-K call's)."""
    return SortSpec(SORT_COLUMNS, [(0, 0, 0)], flags=flags)
