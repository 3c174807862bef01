"""Shared test helpers: result comparison with exact integers and a relative
tolerance for f64 sums (device and host summation orders differ)."""
from __future__ import annotations

import math

import numpy as np

import qumirdb_b200 as q
from qumirdb_b200 import abi, queries

F64_REL = 1e-12


def gpu_rows(rs: abi.RowSet, types) -> list[list]:
    values, valid = q.read_rowset(rs, types)
    n = rs.RowCount
    rows = []
    for r in range(n):
        row = []
        for c, t in enumerate(types):
            if not valid[c][r]:
                row.append(None)
            elif t in (abi.F64, abi.F32):
                row.append(float(values[c][r]))
            else:
                row.append(int(values[c][r]))
        rows.append(row)
    return rows


def _key(row, nkeys):
    return tuple((0, 0) if v is None else (1, v) for v in row[:nkeys])


def assert_same_groups(got: list[list], want: list[list], types, nkeys: int, rel: float = F64_REL) -> None:
    """Equal group sets: exact for integers/decimals, `rel` for doubles."""
    assert len(got) == len(want), f"group count {len(got)} != {len(want)}"
    g = sorted(got, key=lambda r: _key(r, nkeys))
    w = sorted(want, key=lambda r: _key(r, nkeys))
    for rg, rw in zip(g, w):
        for c, t in enumerate(types):
            a, b = rg[c], rw[c]
            if a is None or b is None:
                assert a is None and b is None, f"column {c}: {a} vs {b} in {rg} / {rw}"
            elif t in (abi.F64, abi.F32):
                assert math.isclose(a, b, rel_tol=rel, abs_tol=1e-300) or (math.isnan(a) and math.isnan(b)), \
                    f"column {c}: {a} vs {b}"
            else:
                assert a == b, f"column {c}: {a} vs {b} in {rg} / {rw}"


def lineitem(n: int, seed: int = 0):
    cols = [np.empty(n, np.int64), np.empty(n, np.int64), np.empty(n, np.int64), np.empty(n, np.int64),
            np.empty(n, np.uint8), np.empty(n, np.uint8), np.empty(n, np.int32)]
    q.lib().qdb_gen_lineitem(seed, n, *[c.ctypes.data for c in cols])
    return cols


def join_data(build: int, probe: int, domain: int, seed: int = 1):
    b = [np.empty(build, np.int64), np.empty(build, np.int64), np.empty(build, np.int32)]
    p = [np.empty(probe, np.int64), np.empty(probe, np.int64)]
    q.lib().qdb_gen_join(seed, build, probe, domain, *[x.ctypes.data for x in b + p])
    return b, p


def zipf_data(n: int, distinct: int, seed: int = 2):
    cols = [np.empty(n, np.int64), np.empty(n, np.int64), np.empty(n, np.float64)]
    q.lib().qdb_gen_zipf(seed, n, distinct, 1.1, *[c.ctypes.data for c in cols])
    return cols


def shape_case(shape, groups, n, rng):
    """(columns, spec, output types) of a plan whose shape is compiled in the
    listed-row kernel's catalogue."""
    k = rng.integers(0, groups, n).astype(np.int64) * 1009 + 5
    a = rng.integers(-10**12, 10**12, n).astype(np.int64)
    e = q.ExprBuilder()
    if shape == "count":
        kc = e.col(0, abi.I64)
        spec = queries.AggSpec([(abi.I64,)], e, None, [kc], [(abi.COUNT_STAR, -1)], expected_groups=64)
        return [k], spec, [abi.I64, abi.I64]
    if shape == "sum_count":
        kc, ac = e.col(0, abi.I64), e.col(1, abi.I64)
        spec = queries.AggSpec([(abi.I64,), (abi.I64,)], e, None, [kc], [(abi.SUM, ac), (abi.COUNT_STAR, -1)],
                               expected_groups=64)
        return [k, a], spec, [abi.I64, abi.I64, abi.I64]
    if shape == "q6":
        x = rng.integers(0, 1000, n).astype(np.int64)
        xc, ac = e.col(0, abi.I64), e.col(1, abi.I64)
        filt = e.op(abi.BETWEEN, abi.BOOL, xc, e.const(100, abi.I64), e.const(700, abi.I64))
        spec = queries.AggSpec([(abi.I64,), (abi.I64,)], e, filt, [], [(abi.SUM, e.op(abi.MUL, abi.I64, xc, ac))],
                               expected_groups=1)
        return [x, a], spec, [abi.I64]
    # lineitem shape with `groups` flag codes (two one-byte keys).
    cols = lineitem(n, seed=9)
    cols[4] = (rng.integers(0, groups, n) + 65).astype(np.uint8)
    spec = queries.lineitem_agg(int(cols[6].max()) - 90)
    return cols, spec, queries.LINEITEM_OUT_TYPES
