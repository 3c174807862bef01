"""Runtime join filter scenarios over a storage backend (the oracle's host
storage, or the device's): each returns plain values, so the CPU suite can
check them against the reference's own test expectations
(test/test_runtime_filter.cpp) and the GPU suite can check the device
against the oracle on the same inputs."""
from __future__ import annotations

import numpy as np

from oracle import oracle as O
from qumirdb_b200 import rfilter as RF


def hashes(n: int, seed: int) -> np.ndarray:
    """Hashes(count, seed) of the reference's tests: std::mt19937_64 draws."""
    return O.mt19937_64(seed, n)


def build_partial(st, max_keys, bloom_bytes, keys, batch_rows, selection=None):
    """BuildPartial: one builder fed `keys` in batches of batch_rows; returns
    (partial, builder, (hashes, bloom words, overflowed, build rows))."""
    keys = np.ascontiguousarray(keys, dtype=np.uint64)
    b = RF.RuntimeFilterBuilder(st, max_keys, bloom_bytes)
    hbuf = st.upload(keys) if len(keys) else None
    sbuf = None if selection is None else st.upload(np.ascontiguousarray(selection, dtype=np.uint8))
    for row in range(0, len(keys), batch_rows):
        n = min(batch_rows, len(keys) - row)
        sel = None if sbuf is None else st.ptr(sbuf) + row
        nsel = None if selection is None else int(np.count_nonzero(selection[row:row + n]))
        b.add(st.ptr(hbuf) + 8 * row, n, sel, nsel)
    p = b.take_partial()
    bloom = st.read_u64(p.bloom, p.bloom_words) if p.bloom is not None else np.empty(0, np.uint64)
    return p, b, (b.partial_hashes().tolist(), bloom.tolist(), p.overflowed, p.build_rows)


def publish_keys(st, filt, keys):
    """PublishKeys: one builder with every key, finished as one producer."""
    b = filt.make_builder()
    keys = np.ascontiguousarray(keys, dtype=np.uint64)
    if len(keys):
        buf = st.upload(keys)
        b.add(st.ptr(buf), len(keys))
    filt.finish_producer(b.take_partial())


def probe(st, filt, probes, selection=None) -> np.ndarray:
    """ProbeRuntimeFilter: one output byte per hash, as a consumer probes
    (an unpublished or pass-all filter keeps every selected row)."""
    probes = np.ascontiguousarray(probes, dtype=np.uint64)
    n = len(probes)
    if not filt.answers():
        out = np.ones(n, dtype=np.uint8)
        if selection is not None:
            out &= (np.asarray(selection) != 0).astype(np.uint8)
        return out
    hb = st.upload(probes)
    ob = st.alloc(n)
    sb = None if selection is None else st.upload(np.ascontiguousarray(selection, dtype=np.uint8))
    k = filt.may_contain_batch(st.ptr(hb), st.ptr(ob), n, None if sb is None else st.ptr(sb))
    out = st.read_u8(ob, n)
    assert k == int(np.count_nonzero(out))
    return out


def published(st, filt):
    """The published filter as values: kind, words (exact tables compared by
    key set elsewhere), and the stats."""
    words = st.read_u64(filt.words, filt.word_count).tolist() if filt.words is not None else []
    return filt.kind, words, dict(filt.stats)


def selections(rows: int):
    """Every row selected, none, every third, and a random half."""
    rng = np.random.default_rng(rows)
    return [np.full(rows, 0xFF, np.uint8), np.zeros(rows, np.uint8),
            np.where(np.arange(rows) % 3 == 0, 0xFF, 0).astype(np.uint8),
            rng.integers(0, 2, rows).astype(np.uint8)]


# ---------------------------------------------------------------------------
# Scenarios (each restates one test of test/test_runtime_filter.cpp).
# ---------------------------------------------------------------------------
def bloom_layout(st):
    keys = np.array([0, 1, 2, 0xFEDCBA9876543210], dtype=np.uint64)
    return build_partial(st, 0, 128, keys, len(keys))[2]


def compaction_order(st):
    cap = 64
    early = list(hashes(38, 51)) + [0, 0xFFFFFFFFFFFFFFFF]
    inp = early * 3 + early[:8]
    rng = np.random.default_rng(52)
    inp = [inp[i] for i in rng.permutation(len(inp))]
    late = hashes(10, 53)
    for k in late:
        inp += [int(k), early[int(k) % len(early)], int(k)]
    return build_partial(st, cap, 512, np.array(inp, dtype=np.uint64), len(inp))[2]


def batch_boundary_inputs():
    cap = 64
    late = hashes(30, 41)

    def repeated(distinct, times, tail):
        keys = list(hashes(distinct, distinct))
        return np.array(keys * times + list(tail), dtype=np.uint64)

    return cap, [hashes(100, 42), hashes(cap * 2, 43), repeated(40, 4, late[:10]), repeated(cap, 10, late),
                 hashes(1000, 44)]


def duplicate_heavy_then_new(st):
    cap = 64
    filt = RF.RuntimeFilter(st, cap, 512)
    keys = hashes(cap, 21)
    b = filt.make_builder()
    kb = st.upload(keys)
    for _ in range(100):
        b.add(st.ptr(kb), len(keys))
    before = b.overflowed
    batch = np.concatenate([keys[:10], np.array([0xFEDCBA9876543210], np.uint64), hashes(50, 22)])
    bb = st.upload(batch)
    b.add(st.ptr(bb), len(batch))
    after = b.overflowed
    filt.finish_producer(b.take_partial())
    return before, after, filt, keys, batch


def exact_key_set(st, count):
    keys = hashes(count, count + 21)
    probes = np.concatenate([hashes(10000, count + 22), keys, np.array([0], np.uint64)])
    filt = RF.RuntimeFilter(st, 8192, 512)
    publish_keys(st, filt, keys)
    return filt, keys, probes


def several_producers(st, producers=4):
    filt = RF.RuntimeFilter(st, 32, 4096, producers=producers)
    allkeys = []
    overflowed = []
    for i in range(producers):
        part = hashes(100, i + 70)
        allkeys.append(part)
        b = filt.make_builder()
        pb = st.upload(part)
        b.add(st.ptr(pb), len(part))
        p = b.take_partial()
        overflowed.append(p.overflowed)
        filt.finish_producer(p)
    return filt, np.concatenate(allkeys), overflowed


def capped_count_cases(st):
    cap = 8
    k = hashes(cap + 1, 60)
    cases = [
        ([hashes(cap + 4, 61), hashes(cap + 4, 62), hashes(cap + 4, 63)], True),
        ([[k[0], k[1], k[2], k[0]], [k[1], k[3], k[4], k[5]], [k[6], k[7], k[2], k[7]]], False),
        ([[k[0], k[1], k[2], k[3]], [k[4], k[5], k[6], k[7], k[0]], [k[3], k[cap]]], True),
    ]
    out = []
    for parts, bloom in cases:
        filt = RF.RuntimeFilter(st, cap, 4096, producers=len(parts))
        allk = []
        for keys in parts:
            keys = np.array(keys, dtype=np.uint64)
            allk.append(keys)
            publish_keys(st, filt, keys)
        out.append((filt, np.concatenate(allk), bloom))
    return out
