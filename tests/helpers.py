"""Shared test helpers: result comparison with exact integers and a relative
tolerance for f64 sums (device and host summation orders differ)."""
from __future__ import annotations

import math

import numpy as np

import qumirdb_b200 as q
from qumirdb_b200 import abi

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
