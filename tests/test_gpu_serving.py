"""The serving loop: every query's result is the same alone and in the mix
(integers bit-exact, f64 sums within 1e-12 relative), admission keeps the
in-flight work inside the HBM budget, and small aggregations waiting together
run as one batched launch."""
import numpy as np
import pytest

import qumirdb_b200 as q
from oracle import oracle as O
from qumirdb_b200 import abi, queries, serving

from .helpers import assert_same_groups

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def setup():
    q.init(0)
    sizes = serving.log_uniform_sizes(16, 100_000, 3_000_000, seed=1)
    tables = [serving.Table(serving.TEMPLATES[i % 4], int(n), seed=10 + i).build() for i, n in enumerate(sizes)]
    progs = serving.Programs()
    scratch = serving.Scratch(max(t.rows for t in tables))
    alone = [serving.run_query(progs, t, scratch) for t in tables]
    return tables, progs, alone


def _rows(res, types):
    vals, valid = res
    return [[None if not valid[c][r] else (float(vals[c][r]) if t == abi.F64 else int(vals[c][r]))
             for c, t in enumerate(types)] for r in range(len(vals[0]))]


def _download(rs):
    out = []
    for k, w in enumerate(rs.widths):
        raw = np.empty(rs.rows * w, np.uint8)
        q.lib().qdb_gpu_memcpy(raw.ctypes.data, rs.cols[k].Data, raw.nbytes)
        q.synchronize()
        out.append(raw.view({1: np.uint8, 4: np.int32, 8: np.int64}[w]))
    return out


def test_alone_results_match_the_oracle(setup):
    """The smallest lineitem and Zipf queries of the mix against the oracle."""
    tables, progs, alone = setup
    for tmpl in ("lineitem", "zipf"):
        i = min((i for i, t in enumerate(tables) if t.template == tmpl), key=lambda i: tables[i].rows)
        t = tables[i]
        cols = _download(t.rowsets[0])
        if tmpl == "lineitem":
            spec, types, nk = queries.lineitem_agg(t.cutoff), queries.LINEITEM_OUT_TYPES, 2
        else:
            cols[2] = cols[2].view(np.float64)
            spec, types, nk = queries.zipf_agg(), queries.ZIPF_OUT_TYPES, 1
        want = O.aggregate(spec, [q.HostRowSet(cols)])
        assert_same_groups(_rows(alone[i], types), want, types, nkeys=nk)


@pytest.mark.parametrize("workers", [1, 4])
def test_mix_equals_alone(setup, workers):
    tables, progs, alone = setup
    resident = sum(t.nbytes for t in tables)
    # A budget that holds about two queries' work at a time: admission waits.
    work = sorted(t.work_bytes() for t in tables)
    budget = resident + work[-1] + work[-2]
    server = serving.BatchingServer(progs, budget, resident, workers=workers, small_rows=1 << 21,
                                    max_sort_rows=max(t.rows for t in tables))
    # A burst: the queue builds up behind the workers, so waiting small
    # aggregations meet and coalesce whatever the host's speed.
    stream = serving.make_stream(tables, rate=1e6, count=80, seed=3)
    try:
        stats = server.run(stream)
    finally:
        server.close()
    assert stats["queries"] == 80
    for x in stream:
        i = tables.index(x.table)
        assert serving.same_result(x.result, alone[i]), (x.qid, x.table.template, x.batch)
        assert x.done >= x.admitted >= x.arrival - 1e-3
    assert server.peak_in_use <= budget - resident or server.peak_in_use == work[-1]
    assert stats["coalesced_queries"] >= 2, stats


def test_plain_server_matches(setup):
    tables, progs, alone = setup
    server = serving.PlainServer(progs, max_sort_rows=max(t.rows for t in tables))
    stream = serving.make_stream(tables, rate=500.0, count=24, seed=4)
    stats = server.run(stream)
    assert stats["queries"] == 24 and stats["p99_ms"] >= stats["p50_ms"] > 0
    for x in stream:
        assert serving.same_result(x.result, alone[tables.index(x.table)])
