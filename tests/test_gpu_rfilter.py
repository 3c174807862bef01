"""Runtime join filter on the device against the oracle: the same host logic
(qumirdb_b200.rfilter) over device storage and qdb_gpu_rf_* versus host
storage and the CPU restatement.  Contributions (key order, Bloom words,
overflow), published filters (kind, exact key count and table size, Bloom
words and set bits) and probe answers must be identical; exact tables are
compared by the answers they give, since concurrent inserts place keys in
other slots of the same linear-probing table."""
import numpy as np
import pytest

import qumirdb_b200 as q
from oracle import oracle as O
from qumirdb_b200 import abi, queries
from qumirdb_b200 import rfilter as RF

from . import rf_cases as R

pytestmark = pytest.mark.gpu

HOST = O.HostStorage()


@pytest.fixture(scope="module")
def dev():
    return RF.DeviceStorage()


def same_filter(dev, a, b, probes):
    assert a.ready == b.ready and a.kind == b.kind
    assert a.stats == b.stats
    if a.kind == RF.KIND_BLOOM:
        assert R.published(dev, a)[1] == R.published(HOST, b)[1]
    if a.kind == RF.KIND_EXACT:
        assert a.word_count == b.word_count
    assert (R.probe(dev, a, probes) == R.probe(HOST, b, probes)).all()


def test_bloom_layout_and_compaction(dev):
    assert R.bloom_layout(dev) == R.bloom_layout(HOST)
    assert R.compaction_order(dev) == R.compaction_order(HOST)


def test_batch_boundaries_and_selections(dev):
    cap, inputs = R.batch_boundary_inputs()
    for h in inputs:
        for rows in (1, 7, 129, len(h)):
            assert R.build_partial(dev, cap, 512, h, rows)[2] == R.build_partial(HOST, cap, 512, h, rows)[2]
        for sel in R.selections(len(h)):
            assert R.build_partial(dev, cap, 512, h, 129, sel)[2] == R.build_partial(HOST, cap, 512, h, 129, sel)[2]


def test_publication_cases(dev):
    probes = R.hashes(20000, 99)
    a = R.duplicate_heavy_then_new(dev)
    b = R.duplicate_heavy_then_new(HOST)
    assert a[:2] == b[:2]
    same_filter(dev, a[2], b[2], np.concatenate([probes, a[3], a[4]]))
    for count in (0, 1, 8, 200, 4096, 5000):
        fa, keys, pr = R.exact_key_set(dev, count)
        fb, _, _ = R.exact_key_set(HOST, count)
        same_filter(dev, fa, fb, pr)
        for sel in R.selections(len(pr)):
            assert (R.probe(dev, fa, pr, sel) == R.probe(HOST, fb, pr, sel)).all()
    fa, ka, oa = R.several_producers(dev)
    fb, kb, ob = R.several_producers(HOST)
    assert oa == ob
    same_filter(dev, fa, fb, np.concatenate([probes, ka]))
    for (fa, ka, ba), (fb, kb, bb) in zip(R.capped_count_cases(dev), R.capped_count_cases(HOST)):
        same_filter(dev, fa, fb, np.concatenate([probes, ka]))


@pytest.mark.parametrize("distinct,bloom", [(16_000, False), (300_000, True)])
def test_build_side_scale(dev, distinct, bloom):
    """A 2M-row build side in 2^18-row batches (the engine's scan batch) with
    a selection: 16K distinct hashes stay exact, 300K become a 2 MB Bloom
    filter; 8M probe hashes give the same answers."""
    rng = np.random.default_rng(distinct)
    pool = rng.integers(0, 2**63, distinct, dtype=np.uint64) * 2 + 1
    keys = pool[rng.integers(0, distinct, 2_000_000)]
    sel = (rng.random(len(keys)) > 0.2).astype(np.uint8)
    filters = []
    for st in (dev, HOST):
        filt = RF.RuntimeFilter(st)
        b = filt.make_builder()
        kb, sb = st.upload(keys), st.upload(sel)
        for row in range(0, len(keys), 1 << 18):
            n = min(1 << 18, len(keys) - row)
            b.add(st.ptr(kb) + 8 * row, n, st.ptr(sb) + row, int(sel[row:row + n].sum()))
        filt.finish_producer(b.take_partial())
        filters.append(filt)
    assert filters[0].uses_bloom == bloom
    probes = np.concatenate([pool, rng.integers(0, 2**64 - 1, 8_000_000, dtype=np.uint64)])
    same_filter(dev, filters[0], filters[1], probes)


def test_probe_side_scan_fused_with_the_hash(dev):
    """Build keys -> qdb_gpu_hash -> filter; the probe side's rows are then
    tested by qdb_gpu_rf_probe_rowset (hash and probe in one kernel), equal to
    the oracle's hash followed by the oracle's probe, NULL keys and a
    selection included."""
    rng = np.random.default_rng(5)
    nb, npr = 50_000, 1_000_000
    bkey = rng.integers(0, 400_000, nb).astype(np.int64)
    pkey = rng.integers(0, 1_000_000, npr).astype(np.int64)
    pvalid = rng.random(npr) > 0.05
    psel = (rng.random(npr) > 0.1).astype(np.uint8)
    cols = [(abi.I64, 0, 1)]
    hprog = q.compile_hash(cols, [0])
    bdev = q.DeviceRowSet([bkey])
    hb = dev.alloc(nb * 8)
    q.hash_rows(hprog, bdev, hb.ptr)
    host_h = O.hash_rows(cols, [0], q.HostRowSet([bkey]))
    assert (dev.read_u64(hb, nb) == host_h.astype(np.uint64)).all()
    for max_keys in (RF.DEFAULT_MAX_KEYS, 100_000):
        fd = RF.RuntimeFilter(dev, max_keys)
        b = fd.make_builder()
        b.add(hb.ptr, nb)
        fd.finish_producer(b.take_partial())
        fh = RF.RuntimeFilter(HOST, max_keys)
        R.publish_keys(HOST, fh, host_h.astype(np.uint64))
        assert fd.kind == fh.kind
        prs = q.DeviceRowSet([pkey], masks=[pvalid], selection=psel)
        out = dev.alloc(npr)
        k = RF.probe_rowset(fd, hprog, prs, out.ptr)
        got = dev.read_u8(out, npr)
        ph = O.hash_rows(cols, [0], q.HostRowSet([pkey], masks=[pvalid]))
        want = R.probe(HOST, fh, ph.astype(np.uint64), psel)
        assert (got == want).all() and k == int(want.sum())
        assert k < int(psel.sum())   # the filter drops probe rows
