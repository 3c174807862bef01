"""Runtime join filter on the CPU: the oracle's restatement of
qdb/kernel/join/runtime_filter.oz driven by the host logic of
qumirdb_b200.rfilter (TRuntimeFilterBuilder / TRuntimeFilter), pinned by the
expectations of the reference's own tests (test/test_runtime_filter.cpp)."""
import numpy as np
import pytest

from oracle import oracle as O
from qumirdb_b200 import rfilter as RF

from . import rf_cases as R

ST = O.HostStorage()


def test_bloom_layout_is_stable():
    """BloomLayoutIsStable: fragments merge by OR, so the bit positions are
    part of the format; the reference's golden words."""
    hashes_, words, overflowed, _ = R.bloom_layout(ST)
    assert overflowed
    assert [w for w in words] == [
        0x0000800000004000, 0x0000000000402000, 0x0000000020800000, 0x0800000010000000,
        0x0200000040000000, 0x0020010000000000, 0x0000000101000000, 0x0000000400800000,
        0x0000000100020000, 0x0000100000000200, 0x000000A000000000, 0x0000000008800000,
        0x0080000000000040, 0x0002000080000000, 0x0000000002000002, 0x0000011000000000]
    assert hashes_ == []


def test_compaction_sorts_and_later_keys_keep_their_order():
    early = sorted(set(int(x) for x in R.hashes(38, 51)) | {0, 0xFFFFFFFFFFFFFFFF})
    late = [int(x) for x in R.hashes(10, 53)]
    hashes_, _, overflowed, rows = R.compaction_order(ST)
    assert not overflowed
    assert hashes_ == early + late
    assert rows == 128 + 30


def test_builder_result_does_not_depend_on_batch_boundaries():
    cap, inputs = R.batch_boundary_inputs()
    flags = [R.build_partial(ST, cap, 512, h, 1)[2][2] for h in inputs[:4]]
    assert flags == [False, True, False, True]
    assert len(R.build_partial(ST, cap, 512, inputs[2], 1)[2][0]) == 50
    for h in inputs:
        row_by_row = R.build_partial(ST, cap, 512, h, 1)[2]
        for rows in (7, 128, 129, len(h)):
            assert R.build_partial(ST, cap, 512, h, rows)[2] == row_by_row
        for sel in R.selections(len(h)):
            picked = h[sel != 0]
            assert R.build_partial(ST, cap, 512, h, 129, sel)[2] == R.build_partial(ST, cap, 512, picked, 1)[2]


def test_promotes_after_duplicate_heavy_build_gets_new_key():
    before, after, filt, keys, batch = R.duplicate_heavy_then_new(ST)
    assert not before and after
    assert filt.uses_bloom
    assert R.probe(ST, filt, keys).all() and R.probe(ST, filt, batch).all()


def test_never_rejects_a_key_and_handles_zero_hash():
    filt = RF.RuntimeFilter(ST)
    keys = R.hashes(5000, 1)
    R.publish_keys(ST, filt, keys)
    assert filt.ready and not filt.uses_bloom
    assert R.probe(ST, filt, keys).all()
    # 0 and 8 share a home slot in the smallest table, so one is displaced.
    for keys in ([0, 7], [8, 0]):
        filt = RF.RuntimeFilter(ST)
        R.publish_keys(ST, filt, np.array(keys, np.uint64))
        got = R.probe(ST, filt, np.array(keys + [9, 16], np.uint64))
        assert [bool(x) for x in got] == [True, True, False, False]


@pytest.mark.parametrize("count", [0, 1, 8, 200, 4096, 5000])
def test_exact_filter_matches_the_key_set(count):
    filt, keys, probes = R.exact_key_set(ST, count)
    assert not filt.uses_bloom and filt.stats["exact_keys"] == count
    expected = set(int(k) for k in keys)
    for sel in R.selections(len(probes)) + [None]:
        out = R.probe(ST, filt, probes, sel)
        want = [(sel is None or s != 0) and int(p) in expected
                for p, s in zip(probes, sel if sel is not None else [1] * len(probes))]
        assert [bool(x) for x in out] == want


def test_cap_is_enforced_at_publication():
    for distinct in (8, 9):
        filt = RF.RuntimeFilter(ST, 8, 512)
        keys = R.hashes(distinct, 13)
        b = filt.make_builder()
        buf = ST.upload(keys)
        b.add(ST.ptr(buf), len(keys))
        assert not b.overflowed
        filt.finish_producer(b.take_partial())
        assert filt.uses_bloom == (distinct > 8)
        assert filt.stats["exact_keys"] == (0 if distinct > 8 else 8)
        assert R.probe(ST, filt, keys).all()


def test_capped_count_at_publication_keeps_the_filter():
    probes = R.hashes(2000, 64)
    for filt, allk, bloom in R.capped_count_cases(ST):
        assert filt.uses_bloom == bloom
        assert R.probe(ST, filt, allk).all()
        if not bloom:
            assert filt.stats["exact_keys"] == 8
            continue
        direct = RF.RuntimeFilter(ST, 8, 4096)
        p, _, _ = R.build_partial(ST, 0, 4096, allk, len(allk))
        direct.finish_producer(p)
        assert filt.stats["bloom_set_bits"] == direct.stats["bloom_set_bits"]
        assert (R.probe(ST, filt, probes) == R.probe(ST, direct, probes)).all()


def test_bloom_fragments_merge_from_several_producers():
    filt, allkeys, overflowed = R.several_producers(ST)
    assert all(overflowed) and filt.uses_bloom
    single = RF.RuntimeFilter(ST, 32, 4096)
    p, _, (_, words, _, _) = R.build_partial(ST, 32, 4096, allkeys, len(allkeys))
    single.finish_producer(p)
    bits = sum(bin(w).count("1") for w in words)
    assert filt.stats["build_rows"] == 400 and filt.stats["bloom_bytes"] == 4096
    assert filt.stats["bloom_set_bits"] == bits == single.stats["bloom_set_bits"]
    assert R.probe(ST, filt, allkeys).all()
    probes = R.hashes(20000, 99)
    got = R.probe(ST, filt, probes)
    assert (got == R.probe(ST, single, probes)).all()
    assert int(got.sum()) < 2000


def test_merges_exact_empty_and_bloom_contributions_without_losing_zero_hash():
    filt = RF.RuntimeFilter(ST, 8, 1000, producers=3)
    R.publish_keys(ST, filt, np.array([0, 1], np.uint64))
    filt.finish_producer(filt.make_builder().take_partial())
    keys = R.hashes(200, 71)
    R.publish_keys(ST, filt, keys)
    assert filt.uses_bloom and filt.stats["bloom_bytes"] == 512 and filt.stats["build_rows"] == 202
    assert R.probe(ST, filt, np.array([0, 1], np.uint64)).all() and R.probe(ST, filt, keys).all()


def test_incompatible_or_saturated_bloom_passes_everything():
    filt = RF.RuntimeFilter(ST, 8, 512)
    b = RF.RuntimeFilterBuilder(ST, 8, 64)
    keys = R.hashes(64, 72)
    buf = ST.upload(keys)
    b.add(ST.ptr(buf), len(keys))
    filt.finish_producer(b.take_partial())
    assert filt.ready and filt.stats["bloom_disabled"] and not filt.answers()
    sat = RF.RuntimeFilter(ST, 8, 64)
    R.publish_keys(ST, sat, R.hashes(10000, 88))
    assert sat.stats["bloom_disabled"] and not sat.uses_bloom


def test_repeated_keys_do_not_consume_the_cap():
    filt = RF.RuntimeFilter(ST, 64)
    keys = R.hashes(50, 7)
    b = filt.make_builder()
    buf = ST.upload(keys)
    for _ in range(1000):
        b.add(ST.ptr(buf), len(keys))
    assert not b.overflowed
    filt.finish_producer(b.take_partial())
    assert not filt.uses_bloom and filt.stats["exact_keys"] == 50
    many = RF.RuntimeFilter(ST, 64, producers=20)
    keys = R.hashes(50, 8)
    for _ in range(20):
        R.publish_keys(ST, many, keys)
    assert not many.uses_bloom and many.stats["exact_keys"] == 50
    assert int(R.probe(ST, many, R.hashes(1000, 9)).sum()) < 2
