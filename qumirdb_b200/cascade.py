"""Partial -> shuffle -> final aggregation on the device: the threaded
scheduler's second grouped-aggregate plan (docs/arch/aggregation.md,
"Partial aggregate plan") and its global cascade, over this library's
entries.

    input lanes[N] -> aggregate(partial)[N] -> repartition(group keys, P)
                   -> aggregate(final)[P]

The partial phase is the aggregate program itself with its raw row as output
(keys, then one state per aggregate); a lane flushes its table when it holds
`max_groups` groups (TPartialAggregateProcessor::Add,
qdb/exec/aggregate_exec.cpp:180-215).  The partial states are split by the
engine's key hash with qdb_gpu_shuffle, device to device.  The final phase
combines them as BuildAggregateCombineOperator
(qdb/exec/planner_helpers.cpp:191-209) does: COUNT becomes SUM, SUM / MIN /
MAX stay, each reading its own partial column, and the original output
projection (AVG and the like) runs over the combined row.  A keyless
aggregate gathers its lanes into one final aggregate.
"""
from __future__ import annotations

import ctypes as C

from . import (Aggregate, ExprBuilder, Program, abi, compile_aggregate, compile_hash, release,
               shuffle)
from .queries import AggSpec

_FLOAT = (abi.F32, abi.F64)
_DECIMAL = (abi.DECIMAL64, abi.DECIMAL128)


def _result_type(func: int, t: int, scale: int) -> tuple[int, int]:
    """AggregateResultType (qdb/plan/ops/aggregate.cpp:21-57) of a state."""
    if func in (abi.COUNT_STAR, abi.COUNT):
        return abi.I64, 0
    if t in _FLOAT:
        return abi.F64, 0
    if func == abi.SUM:
        return (abi.DECIMAL128, scale) if t in _DECIMAL else (abi.I64, 0)
    return (t, scale) if t in _DECIMAL else (abi.I64, 0)


def partial_row_types(spec: AggSpec) -> list[tuple]:
    """(type, scale, nullable) of the partial aggregate's raw output row."""
    nodes = spec.eb.nodes
    out = []
    for k in list(spec.keys)[: spec.struct.n_keys]:
        out.append((nodes[k][1], nodes[k][2], 1))
    for j in range(spec.struct.n_aggs):
        f, a = spec.aggs[j].func, spec.aggs[j].arg
        t, s = (abi.I64, 0) if a < 0 else (nodes[a][1], nodes[a][2])
        rt, rs = _result_type(f, t, s)
        out.append((rt, rs, 1))
    return out


def partial_spec(spec: AggSpec) -> AggSpec:
    """The aggregate with its raw row (keys ++ states) as output, on the device."""
    s = spec.struct
    aggs = [(spec.aggs[j].func, spec.aggs[j].arg) for j in range(s.n_aggs)]
    return AggSpec(spec.column_types, spec.eb, None if s.filter < 0 else s.filter, list(spec.keys)[: s.n_keys], aggs,
                   flags=abi.OUT_DEVICE, expected_groups=s.expected_groups)


def combine_spec(spec: AggSpec, flags: int = 0) -> AggSpec:
    """BuildAggregateCombineOperator over the partial row: keys read as
    columns, COUNT -> SUM, SUM / MIN / MAX kept; the original outputs."""
    s = spec.struct
    cols = partial_row_types(spec)
    nk = s.n_keys
    e = ExprBuilder()
    keys = [e.col(j, cols[j][0], cols[j][1]) for j in range(nk)]
    aggs = []
    for j in range(s.n_aggs):
        f = spec.aggs[j].func
        t, sc, _ = cols[nk + j]
        col = e.col(nk + j, t, sc)
        aggs.append((abi.SUM if f in (abi.COUNT_STAR, abi.COUNT) else f, col))
    outputs = list(spec.outputs)[: s.n_outputs] if s.n_outputs else None
    return AggSpec(cols, e, None, keys, aggs, outputs=outputs, out_eb=spec.out_eb if outputs else None,
                   flags=flags)


class _View:
    """A borrowed TRowSet (an output slice) passed back into the library."""

    def __init__(self, rs: abi.RowSet):
        self.rs = rs
        self.ptr = C.byref(rs)


class PartialFinalAggregate:
    """One grouped (or keyless) aggregate run as partial lanes, a device
    shuffle by group key into `partitions`, and final aggregates."""

    def __init__(self, spec: AggSpec, partitions: int = 8, max_groups: int = 1 << 22, flags: int = 0):
        self.keyless = spec.struct.n_keys == 0
        self.partitions = 1 if self.keyless else partitions
        self.max_groups = max_groups
        self._pspec = partial_spec(spec)
        self._fspec = combine_spec(spec, flags)
        self.partial: Program = compile_aggregate(self._pspec)
        self.final: Program = compile_aggregate(self._fspec)
        row = partial_row_types(spec)
        self.hash: Program | None = None if self.keyless else compile_hash(row, list(range(spec.struct.n_keys)))

    def run(self, lanes) -> list[abi.RowSet]:
        """lanes: a list of row-set lists (one per input lane).  Returns the
        final outputs, one row set per partition (release each)."""
        finals = [Aggregate(self.final) for _ in range(self.partitions)]
        pending = []

        def emit(agg: Aggregate) -> None:
            out = agg.finish()
            if self.keyless:
                finals[0].add(_View(out))
            else:
                parts = shuffle(self.hash, _View(out), self.partitions)
                for p in range(self.partitions):
                    if parts[p].RowCount:
                        finals[p].add(_View(parts[p]))
                pending.append(parts)
            release(out)

        for lane in (lanes or [[]]):
            agg = Aggregate(self.partial)
            for batch in lane:
                agg.add(batch)
                if not self.keyless and agg.groups >= self.max_groups:
                    emit(agg)                    # flush: the next add starts a new table
                    agg = Aggregate(self.partial)
            emit(agg)
        outs = [f.finish() for f in finals]
        for parts in pending:
            parts.release()
        return outs
