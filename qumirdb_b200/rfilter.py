"""Runtime join filter, host side: the storage and publication policy of
TRuntimeFilterBuilder / TRuntimeFilter (qdb/exec/runtime_filter.cpp,
runtime_filter.h) over the device entries qdb_gpu_rf_build / _publish /
_probe / _merge, whose state structs point at device arrays.

A join's build side feeds its key hashes (qdb_gpu_hash of the join keys, in
device memory) to a builder per producer; the filter publishes once every
producer has finished, as an exact set of at most MaxKeys hashes or a
blocked Bloom filter, and the probe side's scan asks it which rows may match
(`may_contain_batch` over hashes, or `probe_rowset`, which hashes the probe
keys and tests them in one kernel).  Filters may return false positives,
never false negatives; a filter that cannot answer passes every row.

The storage protocol is pluggable (DeviceStorage here), so the same host
logic can drive another implementation of the four entries over host memory.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import abi

DEFAULT_MAX_KEYS = 1 << 14          # TRuntimeFilter::DefaultMaxKeys
DEFAULT_BLOOM_BYTES = 2 << 20       # TRuntimeFilter::DefaultBloomBytes
BLOOM_BYTES_PER_BLOCK = 64

MODE_COLLECTING, MODE_DEDUPLICATING, MODE_OVERFLOWING, MODE_BLOOM = 0, 1, 2, 3
WANT_NOTHING, WANT_COMPACTION, WANT_BLOOM = 0, 1, 2
KIND_PASS_ALL, KIND_EXACT, KIND_BLOOM = 0, 1, 2


def normalize_bloom_bytes(n: int) -> int:
    """A Bloom filter is a power-of-two number of 64-byte blocks."""
    return 0 if n < BLOOM_BYTES_PER_BLOCK else 1 << (n.bit_length() - 1)


def set_capacity(keys: int) -> int:
    """A dedup set of keys + 1 hashes at most half full, whole swiss groups."""
    need = max(16, (keys + 1) * 2)
    return 1 << (need - 1).bit_length()


class DeviceStorage:
    """Device arrays (qdb_gpu_alloc) and the device entries."""

    def __init__(self):
        from . import lib, _ensure_init
        _ensure_init()
        self.lib = lib()

    def alloc(self, nbytes: int):
        from . import DeviceBuffer
        return DeviceBuffer(max(8, nbytes))

    @staticmethod
    def ptr(buf) -> int:
        return buf.ptr

    def zero(self, buf, nbytes: int) -> None:
        self.lib.qdb_gpu_memset(buf.ptr, 0, max(0, nbytes))

    def copy(self, dst, src, nbytes: int) -> None:
        if nbytes > 0:
            self.lib.qdb_gpu_memcpy(dst.ptr, src.ptr, nbytes)

    def read_u64(self, buf, n: int) -> np.ndarray:
        return buf.download(np.uint64, n) if n else np.empty(0, np.uint64)

    def upload(self, arr: np.ndarray):
        buf = self.alloc(arr.nbytes)
        if arr.nbytes:
            buf.upload(arr)
        return buf

    def read_u8(self, buf, n: int) -> np.ndarray:
        return buf.download(np.uint8, n) if n else np.empty(0, np.uint8)

    def build(self, state, hashes, sel, n) -> int:
        return self.lib.qdb_gpu_rf_build(C.byref(state), hashes, sel, n)

    def publish(self, state, partials, n) -> int:
        return self.lib.qdb_gpu_rf_publish(C.byref(state), partials, n)

    def probe(self, data, hashes, sel, out, n) -> int:
        return self.lib.qdb_gpu_rf_probe(C.byref(data), hashes, sel, out, n, 0, None, None)

    def merge(self, target, source, n) -> None:
        if self.lib.qdb_gpu_rf_merge(target, source, n) != 0:
            raise RuntimeError(self.error())

    def error(self) -> str:
        return self.lib.qdb_gpu_last_error().decode()


class Partial:
    """TRuntimeFilterPartial: the value-only contribution of producers."""

    def __init__(self, hashes, hash_count, bloom, bloom_words, overflowed, build_rows, producers=1):
        self.hashes = hashes              # storage buffer or None
        self.hash_count = hash_count
        self.bloom = bloom                # storage buffer or None
        self.bloom_words = bloom_words
        self.overflowed = overflowed
        self.build_rows = build_rows
        self.producers = producers


class RuntimeFilterBuilder:
    """TRuntimeFilterBuilder: one producer's contribution (task-local)."""

    def __init__(self, storage, max_keys: int, bloom_bytes: int):
        self.st = storage
        self.bloom_bytes = normalize_bloom_bytes(bloom_bytes)
        self.state = abi.RfBuildState()
        self.state.MaxKeys = max_keys
        self.state.BloomWords = -1
        self.keys = None
        self.keys_cap = 0
        self.set_ctrl = self.set_slots = self.sort_order = self.sort_keys = self.bloom = None
        self.build_rows = 0

    def add(self, hashes, n: int, selection=None, selected: int | None = None) -> None:
        """Adds n hashes (a storage pointer) with an optional selection
        pointer; `selected` is the number of selected rows (n when none)."""
        self.build_rows += n if selection is None else int(selected)
        row = 0
        while True:
            self._provide_storage(n - row)
            sel = None if selection is None else selection + row
            got = self.st.build(self.state, hashes + 8 * row, sel, n - row)
            if got < 0:
                raise RuntimeError(f"rf_build failed: {self.st.error()}")
            row += got
            if self.state.Want == WANT_NOTHING:
                break

    def _provide_storage(self, rows: int) -> None:
        s = self.state
        if s.Want == WANT_COMPACTION:
            keys = s.KeyCount
            self.sort_order = self.st.alloc((2 * keys + 256) * 4)
            self.sort_keys = self.st.alloc(keys * 8)
            cap = set_capacity(s.MaxKeys)
            self.set_ctrl = self.st.alloc(cap)
            self.set_slots = self.st.alloc(cap * 8)
            s.SetCapacity = cap
        elif s.Want == WANT_BLOOM:
            words = self.bloom_bytes // 8
            self.bloom = self.st.alloc(words * 8)
            self.st.zero(self.bloom, words * 8)
            s.BloomWords = words
        room = s.KeyCount + rows
        if s.Mode != MODE_BLOOM and self.keys_cap < room:
            grown = self.st.alloc(room * 8)
            if self.keys is not None:
                self.st.copy(grown, self.keys, s.KeyCount * 8)
            self.keys, self.keys_cap = grown, room
        ptr = lambda b: None if b is None else self.st.ptr(b)  # noqa: E731
        s.Keys, s.SetCtrl, s.SetSlots = ptr(self.keys), ptr(self.set_ctrl), ptr(self.set_slots)
        s.SortOrder, s.SortKeys, s.Bloom = ptr(self.sort_order), ptr(self.sort_keys), ptr(self.bloom)

    @property
    def overflowed(self) -> bool:
        return self.state.Mode == MODE_BLOOM

    def take_partial(self) -> Partial:
        s = self.state
        bloom = self.bloom if self.bloom is not None and s.BloomWords > 0 else None
        return Partial(self.keys if s.KeyCount else None, s.KeyCount, bloom,
                       s.BloomWords if bloom is not None else 0, self.overflowed, self.build_rows)

    def partial_hashes(self) -> np.ndarray:
        return self.st.read_u64(self.keys, self.state.KeyCount) if self.state.KeyCount else np.empty(0, np.uint64)


class RuntimeFilter:
    """TRuntimeFilter: merges the producers' partials and answers probes."""

    def __init__(self, storage, max_keys: int = DEFAULT_MAX_KEYS, bloom_bytes: int = DEFAULT_BLOOM_BYTES,
                 producers: int = 1):
        self.st = storage
        self.max_keys = max_keys
        self.bloom_bytes = normalize_bloom_bytes(bloom_bytes)
        self.pending = producers
        self.partials: list[Partial] = []
        self.ready = False
        self.kind = KIND_PASS_ALL
        self.words = None
        self.word_count = 0
        self.stats = {"build_rows": 0, "exact_keys": 0, "bloom_bytes": 0, "bloom_set_bits": 0,
                      "bloom_disabled": False}

    def make_builder(self) -> RuntimeFilterBuilder:
        return RuntimeFilterBuilder(self.st, self.max_keys, self.bloom_bytes)

    def finish_producer(self, partial: Partial) -> None:
        self.partials.append(partial)
        self.pending -= partial.producers
        if self.pending == 0:
            self._publish()
            self.partials = []
            self.ready = True

    def _publish(self) -> None:
        # TRuntimeFilter::BuildPublishedData (qdb/exec/runtime_filter.cpp).
        words_full = self.bloom_bytes // 8
        exact_hashes = 0
        incomplete = False
        for p in self.partials:
            self.stats["build_rows"] += p.build_rows
            exact_hashes += p.hash_count
            incomplete |= p.overflowed and p.bloom is None
            incomplete |= p.bloom is not None and p.bloom_words != words_full
        if incomplete:
            self.stats["bloom_disabled"] = True   # a missing contribution must never reject a key
            return
        state = abi.RfPublishState()
        state.MaxKeys = self.max_keys
        bloom = table = None
        seeded = None
        for p in self.partials:
            if p.bloom is not None:
                seeded = p
                bloom = p.bloom
                state.BloomSeeded = 1
                break
        if seeded is None:
            exact_keys = min(exact_hashes, self.max_keys)
            size = 1 << (max(8, exact_keys * 2) - 1).bit_length()
            table = self.st.alloc(size * 8)
            self.st.zero(table, size * 8)
            if exact_hashes > self.max_keys and words_full > 0:
                bloom = self.st.alloc(words_full * 8)
                self.st.zero(bloom, words_full * 8)
        views = (abi.RfPartial * max(1, len(self.partials)))()
        for i, p in enumerate(self.partials):
            views[i].Keys = None if p.hashes is None else self.st.ptr(p.hashes)
            views[i].KeyCount = p.hash_count
            if p is not seeded and p.bloom is not None:
                views[i].Bloom = self.st.ptr(p.bloom)
                views[i].BloomWords = p.bloom_words
        state.Table = None if table is None else self.st.ptr(table)
        state.Bloom = None if bloom is None else self.st.ptr(bloom)
        state.BloomWords = 0 if bloom is None else words_full
        if self.st.publish(state, views, len(self.partials)) != 0:
            raise RuntimeError(f"rf_publish failed: {self.st.error()}")
        if state.Kind == KIND_EXACT:
            self.kind, self.words, self.word_count = KIND_EXACT, table, state.TableSize
            self.stats["exact_keys"] = state.ExactKeys
            return
        if state.Kind != KIND_BLOOM:
            self.stats["bloom_disabled"] = True   # more keys than the exact set holds, no Bloom storage
            return
        self.stats["bloom_bytes"] = words_full * 8
        self.stats["bloom_set_bits"] = state.BloomSetBits
        # At this density the false-positive rate approaches 50%.
        if state.BloomSetBits * 10 >= words_full * 64 * 9:
            self.stats["bloom_disabled"] = True
            return
        self.kind, self.words, self.word_count = KIND_BLOOM, bloom, words_full

    @property
    def uses_bloom(self) -> bool:
        return self.ready and self.kind == KIND_BLOOM

    def data(self) -> abi.RfData:
        d = abi.RfData()
        d.Kind = self.kind
        d.Words = None if self.words is None else self.st.ptr(self.words)
        d.WordCount = self.word_count
        return d

    def answers(self) -> bool:
        """False when every row passes (unpublished, or PassAll)."""
        return self.ready and self.kind != KIND_PASS_ALL

    def may_contain_batch(self, hashes, out, n: int, selection=None) -> int:
        """rf_probe over n hashes (storage pointers); the kept count.  The
        caller passes every selected row when `answers()` is False."""
        k = self.st.probe(self.data(), hashes, selection, out, n)
        if k < 0:
            raise RuntimeError(f"rf_probe failed: {self.st.error()}")
        return k


def probe_rowset(filt: RuntimeFilter, hash_program, batch, out_ptr: int) -> int:
    """The probe-side scan fused with the filter: out[i] = 1 for batch rows
    whose join-key hash the filter may hold (qdb_gpu_rf_probe_rowset)."""
    from . import lib, last_error
    k = lib().qdb_gpu_rf_probe_rowset(hash_program.handle, C.byref(filt.data()), batch.ptr, out_ptr)
    if k < 0:
        raise RuntimeError(f"rf_probe_rowset failed: {last_error()}")
    return k
