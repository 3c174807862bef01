"""Serving: a request loop for a mixed stream of SQL queries over
device-resident tables, beside the plain one-query-at-a-time path.

The queries come from the four templates of the hot path — the lineitem
scan-filter-aggregate (GROUP BY flag, status), the build/probe join with its
SUM/COUNT, the high-cardinality GROUP BY key and ORDER BY k1 DESC, k2 LIMIT
1000 (top-K, as the engine runs a small limit) — each
over its own seeded tables, generated once and kept resident in HBM (the
column cache the engine's Parquet scan would fill).

`PlainServer` runs one query at a time on one stream, in arrival order: the
reference's executor shape, one query's operators after another's.

`BatchingServer` is the serving loop:

* admission: a query is admitted when the device memory it needs (its hash
  tables, sort buffers and outputs, estimated from its table sizes) fits the
  HBM budget beside the resident columns and the queries already running;
  the rest wait in arrival order;
* continuous batching: admitted queries run as they come, on a pool of worker
  threads each driving its own CUDA stream, so one query's kernels overlap
  another's host work and kernels; a query that arrives while others run
  takes the next free worker;
* coalescing: small high-cardinality aggregations of one template waiting at
  the same time go to one worker together and run as one batched persistent
  launch (qdb_gpu_agg_dispatch_batch / qdb_gpu_agg_finish_batch).

Each query's latency is measured from its arrival to its result in host
memory; the servers report queries/s and p50/p99.  A query's result is the
same alone and in the mix (integers bit-exact, f64 sums within 1e-12)."""
from __future__ import annotations

import contextlib
import ctypes as C
import gc
import math
import threading
import time
from collections import deque
from dataclasses import dataclass, field

import numpy as np

import qumirdb_b200 as q
from qumirdb_b200 import abi, queries

TEMPLATES = ("lineitem", "join", "zipf", "sort")
TOP_ROWS = 1000            # ORDER BY ... rows returned to the host
JOIN_RATIO = 60            # probe rows per build row (2M build : 120M probe)


def log_uniform_sizes(n: int, lo: int, hi: int, seed: int) -> np.ndarray:
    rng = np.random.default_rng(seed)
    return np.exp(rng.uniform(math.log(lo), math.log(hi), n)).astype(np.int64)


@dataclass
class Table:
    """One query's device-resident seeded tables."""
    template: str
    rows: int
    seed: int
    rowsets: list = field(default_factory=list)
    cutoff: int = 0
    nbytes: int = 0
    ids: object = None        # sort: the packed row ids in input order (device)

    def build(self) -> "Table":
        n, s = self.rows, self.seed
        if self.template == "lineitem":
            cols = [np.empty(n, np.int64), np.empty(n, np.int64), np.empty(n, np.int64), np.empty(n, np.int64),
                    np.empty(n, np.uint8), np.empty(n, np.uint8), np.empty(n, np.int32)]
            q.lib().qdb_gen_lineitem(s, n, *[c.ctypes.data for c in cols])
            self.cutoff = int(cols[6].max()) - 90
            self.rowsets = [q.DeviceRowSet(cols)]
        elif self.template == "join":
            b = max(1, n // JOIN_RATIO)
            bc = [np.empty(b, np.int64), np.empty(b, np.int64), np.empty(b, np.int32)]
            pc = [np.empty(n, np.int64), np.empty(n, np.int64)]
            q.lib().qdb_gen_join(s, b, n, b + b // 4, *[x.ctypes.data for x in bc + pc])
            cols = bc + pc
            self.rowsets = [q.DeviceRowSet(bc), q.DeviceRowSet(pc)]
        elif self.template == "zipf":
            cols = [np.empty(n, np.int64), np.empty(n, np.int64), np.empty(n, np.float64)]
            q.lib().qdb_gen_zipf(s, n, max(1, n // 10), 1.1, *[c.ctypes.data for c in cols])
            self.rowsets = [q.DeviceRowSet(cols)]
        else:
            k1, k2 = np.empty(n, np.int64), np.empty(n, np.int32)
            q.lib().qdb_gen_sort(s, n, k1.ctypes.data, k2.ctypes.data, None)
            rid = np.arange(n, dtype=np.int64)
            cols = [k1, k2, rid]
            self.rowsets = [q.DeviceRowSet(cols)]
            self.ids = q.DeviceBuffer(rid.nbytes).upload(rid)
        self.nbytes = sum(c.nbytes for c in cols) + (self.rows * 8 if self.template == "sort" else 0)
        return self

    def work_bytes(self) -> int:
        """Device memory one query over this table allocates while it runs."""
        n = self.rows
        if self.template == "lineitem":
            return 64 << 20
        if self.template == "join":
            return (n // JOIN_RATIO) * 96 + (64 << 20)
        if self.template == "zipf":
            return int(NextPow2(n // 10 * 3 // 2) * 48 * 2) + (n // 10) * 48 + (64 << 20)
        return n * 48 + (64 << 20)


def NextPow2(v: int) -> int:
    p = 1
    while p < v:
        p <<= 1
    return p


class Programs:
    """The compiled programs of the templates (one per table for lineitem,
    whose cutoff is a constant of the plan)."""

    def __init__(self):
        self.zipf = q.compile_aggregate(queries.zipf_agg())
        j, a = queries.join_sum(20)
        self.join = q.compile_join_aggregate(j, a)
        self.sort = q.compile_sort(queries.sort_k1_desc_k2())
        self._lineitem = {}
        self._mu = threading.Lock()

    def lineitem(self, cutoff: int) -> q.Program:
        with self._mu:
            if cutoff not in self._lineitem:
                self._lineitem[cutoff] = q.compile_aggregate(queries.lineitem_agg(cutoff))
            return self._lineitem[cutoff]


def _agg_result(rs, types, keep: bool):
    """The query's host result: numpy copies when kept, else its row count
    (the row set was in host memory; the client is done with it)."""
    if not keep:
        return rs.RowCount
    vals, valid = q.read_rowset(rs, types)
    return [np.asarray(v) for v in vals], [np.asarray(m) for m in valid]


def run_query(progs: Programs, t: Table, scratch: "Scratch", keep: bool = True):
    """One query alone through the one-state entry points; returns its
    result in host memory (see _agg_result)."""
    if t.template == "lineitem":
        agg = q.Aggregate(progs.lineitem(t.cutoff))
        agg.add(t.rowsets[0])
        out = agg.finish()
        res = _agg_result(out, queries.LINEITEM_OUT_TYPES, keep)
        q.release(out)
        return res
    if t.template == "zipf":
        agg = q.Aggregate(progs.zipf)
        agg.expect_groups(t.rows // 10)      # the planner's estimate from the table's statistics
        agg.add(t.rowsets[0])
        out = agg.finish()
        res = _agg_result(out, queries.ZIPF_OUT_TYPES, keep)
        q.release(out)
        return res
    if t.template == "join":
        J = q.RowJoin(progs.join)
        J.append(t.rowsets[0])
        J.build()
        agg = q.Aggregate(progs.join)
        J.probe_aggregate(agg, t.rowsets[1])
        out = agg.finish()
        res = _agg_result(out, [abi.I64, abi.I64], keep)
        q.release(out)
        J.release()
        return res
    # ORDER BY k1 DESC, k2 LIMIT TOP_ROWS.  The engine takes the heap top-K
    # for a limit of at most 1024 rows and a quarter of the input
    # (qdb/exec/sort_exec.cpp:56-65), else the full sort and a slice.
    ids = scratch.ids(t.rows)
    if q.lib().qdb_gpu_memcpy(ids.ptr, t.ids.ptr, t.rows * 8) != 0:
        raise q.QdbError(q.last_error())
    s = q.Sort(progs.sort, t.rowsets)
    limit = min(TOP_ROWS, t.rows)
    if TOP_ROWS <= 1024 and TOP_ROWS * 4 <= t.rows:
        k = s.top_k(ids, limit, n=t.rows)
    else:
        s.sort(ids, n=t.rows)
        k = limit
    top = np.empty(k, np.int64)
    if k and q.lib().qdb_gpu_memcpy(top.ctypes.data, ids.ptr, top.nbytes) != 0:
        raise q.QdbError(q.last_error())
    q.synchronize()
    return top


def run_agg_batch(progs: Programs, tables: list[Table], keep: bool = True):
    """Several aggregations of one template (and one program) as one batched
    launch; returns their results in order."""
    t0 = tables[0]
    if t0.template == "lineitem":
        prog, types = progs.lineitem(t0.cutoff), queries.LINEITEM_OUT_TYPES
    else:
        prog, types = progs.zipf, queries.ZIPF_OUT_TYPES
    b = q.AggregateBatch(prog, len(tables))
    b.add([t.rowsets[0] for t in tables])
    outs = b.finish()
    res = [_agg_result(o, types, keep) for o in outs]
    outs.release()
    return res


class Scratch:
    """A worker's reusable device buffers (sort row ids), allocated up front
    so that no query waits on a device-wide allocation."""

    def __init__(self, max_rows: int = 0):
        self.buf = q.DeviceBuffer(max_rows * 8) if max_rows else None

    def ids(self, n: int) -> q.DeviceBuffer:
        if self.buf is None or self.buf.nbytes < n * 8:
            self.buf = q.DeviceBuffer(n * 8)
        return self.buf


@dataclass
class Query:
    qid: int
    table: Table
    arrival: float                # seconds from the stream's start
    admitted: float = -1.0
    done: float = -1.0
    result: object = None
    batch: int = 1                # size of the batched launch it ran in


def make_stream(tables: list[Table], rate: float, count: int, seed: int) -> list[Query]:
    """Poisson arrivals at `rate` queries/s; each query picks one of the
    tables uniformly (so templates are drawn uniformly when the tables are)."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for i in range(count):
        t += rng.exponential(1.0 / rate)
        out.append(Query(i, tables[int(rng.integers(0, len(tables)))], t))
    return out


def latency_stats(qs: list[Query], wall: float) -> dict:
    lat = np.array([x.done - x.arrival for x in qs]) * 1e3
    wait = np.array([x.admitted - x.arrival for x in qs]) * 1e3
    run = np.array([x.done - x.admitted for x in qs]) * 1e3
    return {"queries": len(qs), "queries_per_s": len(qs) / wall if wall > 0 else None,
            "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
            "max_ms": float(lat.max()), "wait_p50_ms": float(np.percentile(wait, 50)),
            "run_p50_ms": float(np.percentile(run, 50)), "run_p99_ms": float(np.percentile(run, 99)),
            "wall_s": wall}


class _Clock:
    def __init__(self):
        self.t0 = time.perf_counter()

    def now(self) -> float:
        return time.perf_counter() - self.t0

    def wait_until(self, t: float) -> None:
        d = t - self.now()
        if d > 0:
            time.sleep(d)


@contextlib.contextmanager
def _no_gc():
    """While a stream is served: the collector paused (a full collection
    stops every worker thread mid-query; it runs once afterwards) and the
    interpreter's thread switch interval short, so that a worker whose
    library call returned gets the interpreter back within a fraction of a
    query instead of after the default 5 ms."""
    import sys
    was = gc.isenabled()
    interval = sys.getswitchinterval()
    gc.disable()
    sys.setswitchinterval(1e-4)
    try:
        yield
    finally:
        sys.setswitchinterval(interval)
        if was:
            gc.enable()
            gc.collect()


def _bind_stream():
    """A CUDA stream of the calling worker thread for the library's calls."""
    import torch
    s = torch.cuda.Stream()
    q.lib().qdb_gpu_set_stream(C.c_void_p(s.cuda_stream))
    return s


class PlainServer:
    """One query at a time, in arrival order, on one stream."""

    def __init__(self, progs: Programs, max_sort_rows: int = 0, keep_results: bool = True):
        self.progs = progs
        self.keep = keep_results
        self.scratch = Scratch(max_sort_rows)

    def run(self, stream: list[Query]) -> dict:
        clock = _Clock()
        scratch = self.scratch
        with _no_gc():
            for x in stream:
                clock.wait_until(x.arrival)
                x.admitted = clock.now()
                x.result = run_query(self.progs, x.table, scratch, self.keep)
                x.done = clock.now()
            wall = clock.now()
        return latency_stats(stream, wall)


class _DeviceExecutor:
    """The serving loop's queries on the device: a CUDA stream per worker."""

    def __init__(self, server: "BatchingServer"):
        self.server = server

    def bind(self) -> None:
        _bind_stream()

    def scratch(self) -> "Scratch":
        return Scratch(self.server.max_sort_rows)

    def one(self, table: Table, scratch: "Scratch"):
        return run_query(self.server.progs, table, scratch, self.server.keep)

    def batch(self, tables: list[Table]):
        return run_agg_batch(self.server.progs, tables, self.server.keep)


class BatchingServer:
    """Admission by HBM budget, continuous batching over worker streams and
    coalescing of small aggregations into one batched launch.  The workers
    (each a host thread with its own CUDA stream and scratch) live as long as
    the server: close() ends them."""

    def __init__(self, progs: Programs, budget_bytes: int, resident_bytes: int, workers: int = 4,
                 small_rows: int = 8 << 20, max_batch: int = 16, max_sort_rows: int = 0,
                 keep_results: bool = True, executor=None):
        self.progs = progs
        self.keep = keep_results
        # What runs the queries: the device by default; tests of the loop's
        # own logic give an executor with bind(), scratch(), one(table,
        # scratch) and batch(tables).
        self.executor = executor or _DeviceExecutor(self)
        self.max_sort_rows = max_sort_rows
        self.budget = budget_bytes
        self.resident = resident_bytes
        self.workers = workers
        self.small_rows = small_rows
        self.max_batch = max_batch
        self._cv = threading.Condition()
        self._pending: deque[Query] = deque()
        self._clock = None
        self._left = 0
        self._error = None
        self._stop = False
        self.in_use = 0
        self.peak_in_use = 0
        self.batches = 0
        self.coalesced = 0
        self._threads = [threading.Thread(target=self._worker, daemon=True) for _ in range(workers)]
        for t in self._threads:
            t.start()

    def close(self) -> None:
        with self._cv:
            self._stop = True
            self._cv.notify_all()
        for t in self._threads:
            t.join()

    def _coalescable(self, x: Query) -> bool:
        # Small high-cardinality aggregations: the batched kernel's shapes.
        # (Coalescing the lineitem template too, through the low-cardinality
        # batched kernel, stalled the serving stream for hundreds of
        # milliseconds at every rate measured, so it is left out.)
        return x.table.template == "zipf" and x.table.rows <= self.small_rows

    def _key(self, x: Query):
        return (x.table.template, x.table.cutoff)

    def _take(self) -> list[Query] | None:
        """Under the lock: the oldest query that fits the budget, with the
        small aggregations of its template and program queued behind it;
        None when the server stops."""
        while True:
            if self._stop:
                return None
            if self._pending and self._error is None:
                head = self._pending[0]
                need = head.table.work_bytes()
                if self.resident + self.in_use + need <= self.budget or self.in_use == 0:
                    group = [self._pending.popleft()]
                    if self._coalescable(head):
                        key = self._key(head)
                        keep = deque()
                        while self._pending and len(group) < self.max_batch:
                            y = self._pending.popleft()
                            yneed = y.table.work_bytes()
                            if (self._coalescable(y) and self._key(y) == key and
                                    self.resident + self.in_use + need + yneed <= self.budget):
                                group.append(y)
                                need += yneed
                            else:
                                keep.append(y)
                        keep.extend(self._pending)
                        self._pending = keep
                    self.in_use += need
                    self.peak_in_use = max(self.peak_in_use, self.in_use)
                    now = self._clock.now()
                    for y in group:
                        y.admitted = now
                    return group
            self._cv.wait(timeout=0.05)

    def _worker(self) -> None:
        ex = self.executor
        try:
            ex.bind()
            scratch = ex.scratch()
        except Exception as e:
            with self._cv:
                self._error = e
                self._cv.notify_all()
            return
        while True:
            with self._cv:
                group = self._take()
            if group is None:
                return
            try:
                if len(group) > 1:
                    results = ex.batch([y.table for y in group])
                else:
                    results = [ex.one(group[0].table, scratch)]
            except Exception as e:
                with self._cv:
                    self._error = e
                    self._left = 0
                    self._cv.notify_all()
                continue
            with self._cv:
                now = self._clock.now()
                for y, r in zip(group, results):
                    y.result = r
                    y.done = now
                    y.batch = len(group)
                self.in_use -= sum(y.table.work_bytes() for y in group)
                if len(group) > 1:
                    self.batches += 1
                    self.coalesced += len(group)
                self._left -= len(group)
                self._cv.notify_all()

    def warm(self, tables: list[Table], rounds: int = 2) -> None:
        """Bursts of every table's query on all workers at once, so that the
        device memory pool and the pinned output pool hold what concurrent
        queries need before any latency is measured (growing either stalls
        every stream while the driver maps or page-locks memory)."""
        for r in range(rounds):
            burst = [Query(i, t, 0.0) for i, t in enumerate(sorted(tables, key=lambda t: -t.rows) * self.workers)]
            self.run(burst)
            small = [t for t in tables if self._coalescable(Query(0, t, 0.0))]
            if small:   # coalesced batches on every worker
                self.run([Query(i, t, 0.0) for i, t in enumerate(small * self.max_batch * self.workers)])

    def run(self, stream: list[Query]) -> dict:
        """Serves one stream of queries (arrivals at their `arrival` times)
        and returns its latency statistics."""
        with self._cv:
            self._clock = _Clock()
            self._left = len(stream)
            self._error = None
            self.batches = self.coalesced = 0
            self.peak_in_use = self.in_use
        with _no_gc():
            for x in stream:
                self._clock.wait_until(x.arrival)
                with self._cv:
                    self._pending.append(x)
                    self._cv.notify_all()
            with self._cv:
                while self._left > 0 and self._error is None:
                    self._cv.wait(timeout=0.05)
                if self._error is not None:
                    self._pending.clear()
                    raise self._error
                wall = self._clock.now()
        out = latency_stats(stream, wall)
        out.update({"workers": self.workers, "batched_launches": self.batches, "coalesced_queries": self.coalesced,
                    "peak_work_bytes": self.peak_in_use, "budget_bytes": self.budget,
                    "resident_bytes": self.resident})
        return out


def same_result(a, b, rel: float = 1e-12) -> bool:
    """Equal query results: integers exactly, doubles within `rel`; group
    order is free (rows compared sorted by their key columns)."""
    if isinstance(a, np.ndarray):
        return np.array_equal(a, b)
    (va, ma), (vb, mb) = a, b
    if len(va[0]) != len(vb[0]):
        return False

    def order(v):
        keys = [np.asarray(c) for c in v[:2] if np.asarray(c).dtype != object]
        return np.lexsort(keys[::-1]) if keys else np.arange(len(v[0]))

    oa, ob = order(va), order(vb)
    for x, y, mx, my in zip(va, vb, ma, mb):
        x, y, mx, my = np.asarray(x)[oa], np.asarray(y)[ob], np.asarray(mx)[oa], np.asarray(my)[ob]
        if not np.array_equal(mx, my):
            return False
        x, y = x[mx], y[my]
        if x.dtype.kind == "f":
            if not np.allclose(x, y, rtol=rel, atol=0, equal_nan=True):
                return False
        elif not np.array_equal(x, y):
            return False
    return True
