"""The serving loop's own logic on the CPU, with an executor that stands in
for the device: every query served once, admission never lets the admitted
work exceed the HBM budget (except one query alone), waiting small
high-cardinality aggregations of one program coalesce, others never do, and
arrival order is kept for what cannot run yet."""
import threading
import time
from dataclasses import dataclass

import pytest

from qumirdb_b200 import serving


@dataclass(eq=False)
class FakeTable:
    template: str
    rows: int
    work: int
    cutoff: int = 0

    def work_bytes(self) -> int:
        return self.work


class FakeExecutor:
    def __init__(self, server_ref, delay=0.002):
        self.server_ref = server_ref
        self.delay = delay
        self.mu = threading.Lock()
        self.batches = []
        self.max_in_use = 0

    def bind(self):
        pass

    def scratch(self):
        return None

    def _check(self):
        srv = self.server_ref[0]
        with self.mu:
            self.max_in_use = max(self.max_in_use, srv.in_use)

    def one(self, table, scratch):
        self._check()
        time.sleep(self.delay)
        return ("one", id(table))

    def batch(self, tables):
        self._check()
        with self.mu:
            self.batches.append([t.template for t in tables])
        time.sleep(self.delay)
        return [("batch", id(t)) for t in tables]


def make(tables_spec):
    return [FakeTable(*t) for t in tables_spec]


@pytest.mark.parametrize("workers", [1, 3])
def test_every_query_once_and_budget_kept(workers):
    tables = make([("zipf", 1000, 10), ("zipf", 2000, 10), ("sort", 10**6, 40), ("join", 10**5, 30),
                   ("lineitem", 500, 5), ("zipf", 10**7, 50)])
    ref = [None]
    ex = FakeExecutor(ref)
    budget_work = 60
    srv = serving.BatchingServer(None, budget_bytes=100 + budget_work, resident_bytes=100, workers=workers,
                                 small_rows=5000, max_batch=8, executor=ex)
    ref[0] = srv
    try:
        stream = serving.make_stream(tables, rate=5000.0, count=200, seed=1)
        stats = srv.run(stream)
    finally:
        srv.close()
    assert stats["queries"] == 200
    for x in stream:
        assert x.result is not None and x.result[1] == id(x.table)
        assert x.done >= x.admitted >= x.arrival - 1e-6
    # Admitted work stays inside the budget (a single query larger than the
    # budget would run alone; none is here).
    assert srv.peak_in_use <= budget_work
    assert srv.in_use == 0


def test_only_small_zipf_coalesce_and_by_program():
    small = FakeTable("zipf", 1000, 1)
    big = FakeTable("zipf", 10**7, 1)
    li = FakeTable("lineitem", 1000, 1)
    ref = [None]
    ex = FakeExecutor(ref, delay=0.01)
    srv = serving.BatchingServer(None, budget_bytes=10**6, resident_bytes=0, workers=1, small_rows=5000,
                                 max_batch=4, executor=ex)
    ref[0] = srv
    try:
        # A burst: while the first query runs, the rest queue up.
        stream = [serving.Query(i, t, 0.0) for i, t in enumerate([big, small, li, small, small, big, small, small])]
        srv.run(stream)
    finally:
        srv.close()
    for b in ex.batches:
        assert set(b) == {"zipf"} and 2 <= len(b) <= 4
    batched = [x for x in stream if x.batch > 1]
    assert all(x.table is small for x in batched) and len(batched) >= 2
    assert all(x.batch == 1 for x in stream if x.table is not small)


def test_fifo_for_what_cannot_coalesce():
    tables = [FakeTable("join", 10**5, 1), FakeTable("sort", 10**6, 1)]
    ref = [None]
    ex = FakeExecutor(ref, delay=0.001)
    srv = serving.BatchingServer(None, budget_bytes=10**6, resident_bytes=0, workers=1, small_rows=0,
                                 executor=ex)
    ref[0] = srv
    try:
        stream = [serving.Query(i, tables[i % 2], 0.0) for i in range(20)]
        srv.run(stream)
    finally:
        srv.close()
    order = sorted(stream, key=lambda x: x.admitted)
    assert [x.qid for x in order] == list(range(20))


def test_latency_stats_shape():
    qs = [serving.Query(i, None, 0.001 * i, admitted=0.001 * i, done=0.001 * i + 0.002) for i in range(100)]
    st = serving.latency_stats(qs, 0.2)
    assert st["queries"] == 100 and abs(st["p50_ms"] - 2.0) < 1e-6 and st["queries_per_s"] == 500
