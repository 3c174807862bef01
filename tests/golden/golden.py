"""Reads the reference's regression fixtures (fixtures.json, made by
make_golden.py): table schemas and rows to numpy columns, expected result
rows to Python values, and the comparison of result rows."""
from __future__ import annotations

import datetime
import json
import math
import re
from decimal import Decimal
from pathlib import Path

import numpy as np

from qumirdb_b200 import abi

FIXTURES = json.loads((Path(__file__).resolve().parent / "fixtures.json").read_text())


def parse_schema(schema: str) -> list[tuple[str, str, bool, int]]:
    """'<struct (a i64) (b <named Nullable [<named DECIMAL [38 2]>]>)>' ->
    [(name, kind, nullable, scale)] with kind in i32/i64/f32/f64/bool/string/
    dec64/dec128."""
    body = schema.strip()[len("<struct"):-1]
    fields, depth, start = [], 0, None
    for k, ch in enumerate(body):
        if ch == "(":
            if depth == 0:
                start = k + 1
            depth += 1
        elif ch == ")":
            depth -= 1
            if depth == 0:
                fields.append(body[start:k])
    out = []
    for f in fields:
        name, typ = f.split(" ", 1)
        nullable = "Nullable" in typ
        m = re.search(r"DECIMAL \[(\d+) (\d+)\]", typ)
        if m:
            p, s = int(m.group(1)), int(m.group(2))
            out.append((name, "dec64" if p <= 18 else "dec128", nullable, s))
            continue
        base = re.findall(r"\b(i32|i64|f32|f64|bool|string)\b", typ)
        out.append((name, base[-1] if base else typ, nullable, 0))
    return out


def cell(v, kind: str, scale: int):
    if v is None:
        return None
    if isinstance(v, dict):
        f = v["$float"]
        return {"nan": math.nan, "+inf": math.inf, "-inf": -math.inf, "-0": -0.0}[f]
    if kind in ("f32", "f64"):
        return float(v)
    if kind in ("dec64", "dec128"):
        return Decimal(v)
    if kind == "bool":
        return bool(v)
    if kind == "string" or (isinstance(v, str) and not re.fullmatch(r"-?\d+", v)):
        return v   # strings, and dates printed as ISO text
    return int(v)


NP = {"i32": np.int32, "i64": np.int64, "f32": np.float32, "f64": np.float64, "bool": np.bool_}
QT = {"i32": abi.I32, "i64": abi.I64, "f32": abi.F32, "f64": abi.F64, "bool": abi.BOOL}


class Table:
    """Columns of one fixture table: name -> (values, valid mask, qdb type)."""

    def __init__(self, key: str):
        t = FIXTURES["tables"][key]
        self.schema = parse_schema(t["schema"])
        self.rows = [[cell(v, k, s) for v, (_, k, _, s) in zip(r, self.schema)] for r in t["rows"]]
        self.n = len(self.rows)
        self.group = t.get("row_group_rows") or max(1, self.n)
        self.cols = {}
        for j, (name, kind, nullable, scale) in enumerate(self.schema):
            vals = [r[j] for r in self.rows]
            valid = np.array([v is not None for v in vals], dtype=bool)
            if kind == "string":
                self.cols[name] = (vals, valid, None)
                continue
            dt = NP[kind]
            arr = np.array([(v if v is not None else 0) for v in vals], dtype=dt) if self.n else np.empty(0, dt)
            self.cols[name] = (arr, valid if nullable else None, (QT[kind], 0, 1 if nullable else 0))

    def batches(self) -> list[tuple[int, int]]:
        return [(b, min(self.n, b + self.group)) for b in range(0, self.n, self.group)] or [(0, 0)]


def case(name: str) -> dict:
    return FIXTURES["cases"][name]


def expected(name: str) -> tuple[list[tuple], list[list]]:
    """Expected rows; REAL (f32) cells are rounded to float32, the precision
    the engine holds them in (its printed digits are of the double nearest
    to the shortest float32 text)."""
    e = case(name)["expected"]
    schema = parse_schema(e["schema"])
    rows = [[cell(v, k, s) for v, (_, k, _, s) in zip(r, schema)] for r in e["rows"]]
    for r in rows:
        for j, (_, kind, _, _) in enumerate(schema):
            if kind == "f32" and r[j] is not None:
                r[j] = float(np.float32(r[j]))
    return schema, rows


def date_str(days: int) -> str:
    return (datetime.date(1970, 1, 1) + datetime.timedelta(days=int(days))).isoformat()


def same(a, b, rel: float = 1e-12) -> bool:
    """Result cell equality: exact for integers, decimals, strings and bools;
    floats within `rel` relative error, NaN equal to NaN and the sign of a
    zero significant (the engine prints -0)."""
    if a is None or b is None:
        return a is None and b is None
    if isinstance(a, float) or isinstance(b, float):
        a, b = float(a), float(b)
        if math.isnan(a) or math.isnan(b):
            return math.isnan(a) and math.isnan(b)
        if a == 0.0 and b == 0.0:
            return math.copysign(1, a) == math.copysign(1, b)
        if math.isinf(a) or math.isinf(b):
            return a == b
        return abs(a - b) <= rel * max(abs(a), abs(b))
    return a == b


def assert_rows(got: list[list], want: list[list], rel: float = 1e-12) -> None:
    assert len(got) == len(want), (len(got), len(want), got[:5], want[:5])
    for r, (g, w) in enumerate(zip(got, want)):
        assert len(g) == len(w), (r, g, w)
        for c, (x, y) in enumerate(zip(g, w)):
            assert same(x, y, rel), f"row {r} col {c}: got {x!r} want {y!r} (rows {g} / {w})"
