"""Device ORDER BY over packed row ids (qdb_sort_run), slice materialize and
top-K (qdb_top_k_select) against the oracle's restatement of the engine's
LSD sort and heap top-K."""
import numpy as np
import pytest

import qumirdb_b200 as q
from oracle import oracle as O
from qumirdb_b200 import abi, queries

pytestmark = pytest.mark.gpu


def packed_ids(sizes, order=None):
    ids = np.concatenate([(np.int64(b) << 32) | np.arange(n, dtype=np.int64) for b, n in enumerate(sizes)])
    return ids if order is None else ids[order]


def split(cols, sizes, masks=None, device=False):
    """Row sets of consecutive slices of the columns (one per batch size)."""
    out, at = [], 0
    mk = q.DeviceRowSet if device else q.HostRowSet
    for n in sizes:
        m = None if masks is None else [None if x is None else x[at:at + n] for x in masks]
        out.append(mk([c[at:at + n] for c in cols], m))
        at += n
    return out


def sort_case(n, seed, k1_range=None):
    rng = np.random.default_rng(seed)
    k1 = rng.integers(-2**63, 2**63 - 1, n, dtype=np.int64) if k1_range is None else \
        rng.integers(0, k1_range, n, dtype=np.int64)
    k2 = rng.integers(0, 100_000, n, dtype=np.int32)
    rowid = np.arange(n, dtype=np.int64)
    return [k1, k2, rowid]


@pytest.mark.parametrize("n,k1_range", [(1000, None), (150_000, None), (150_000, 50), (300_007, 1000)])
def test_sort_k1_desc_k2_matches_oracle(n, k1_range):
    cols = sort_case(n, 3, k1_range)
    sizes = [n // 3, 0, n // 3, n - 2 * (n // 3)]
    spec = queries.sort_k1_desc_k2()
    prog = q.compile_sort(spec)
    store = split(cols, sizes, device=True)
    ids = packed_ids(sizes)
    want = O.sort(spec, split(cols, sizes), ids)
    got = ids.copy()
    q.Sort(prog, store).sort(got)
    assert np.array_equal(got, want)


def typed_columns(n, seed):
    rng = np.random.default_rng(seed)
    f = rng.normal(size=n)
    f[rng.random(n) < 0.05] = np.nan
    f[rng.random(n) < 0.05] = 0.0
    f[rng.random(n) < 0.05] = -0.0
    f[rng.random(n) < 0.02] = np.inf
    f[rng.random(n) < 0.02] = -np.inf
    f32 = f.astype(np.float32)
    bools = rng.random(n) < 0.5
    cols = [
        rng.integers(-128, 128, n).astype(np.int8),
        rng.integers(-5, 5, n).astype(np.int16),
        rng.integers(0, 7, n).astype(np.uint16),
        rng.integers(-3, 3, n).astype(np.int32),
        f,
        f32,
        rng.integers(0, 2**64 - 1, n, dtype=np.uint64) >> rng.integers(0, 60, n).astype(np.uint64),
        rng.integers(-10, 10, n).astype(np.int32),      # DATE32
        rng.integers(-50, 50, n).astype(np.int64),      # DECIMAL64
        rng.integers(0, 3, n).astype(np.uint8),         # CHAR1 codes
    ]
    types = [(abi.I8,), (abi.I16,), (abi.U16,), (abi.I32, 0, 1), (abi.F64, 0, 1), (abi.F32,), (abi.U64,),
             (abi.DATE32, 0, 1), (abi.DECIMAL64, 2, 1), (abi.CHAR1,)]
    masks = [None, None, None, rng.random(n) > 0.1, rng.random(n) > 0.1, None, None, rng.random(n) > 0.2,
             rng.random(n) > 0.3, None]
    return cols, types, masks, bools


KEY_SETS = [
    [(3, 0, 0), (0, 1, 0)],
    [(4, 0, 1), (1, 1, 0)],
    [(4, 1, 0), (2, 0, 0)],
    [(5, 0, 0), (7, 1, 1), (8, 0, 0)],
    [(6, 1, 0)],
    [(9, 0, 0), (8, 1, 1), (3, 0, 1)],
    [(1, 0, 0), (2, 1, 0), (3, 1, 1), (4, 0, 0)],
]


@pytest.mark.parametrize("keys", KEY_SETS)
def test_sort_types_nulls_directions(keys):
    n = 40_000
    cols, types, masks, _ = typed_columns(n, 11)
    sizes = [10_000, 17_000, 13_000]
    rng = np.random.default_rng(5)
    order = rng.permutation(n)[: n - 3000]          # a permuted subset of the rows
    ids = packed_ids(sizes, order)
    spec = queries.SortSpec(types, keys)
    prog = q.compile_sort(spec)
    want = O.sort(spec, split(cols, sizes, masks), ids)
    for device in (False, True):
        got = ids.copy()
        q.Sort(prog, split(cols, sizes, masks, device=device)).sort(got)
        assert np.array_equal(got, want), device


def test_sort_override_arrays_and_bool_keys():
    n = 30_000
    cols, types, masks, bools = typed_columns(n, 12)
    bitmap = np.packbits(bools, bitorder="little")
    # One batch holding a bit-packed BOOL column beside the others.
    spec = queries.SortSpec(types + [(abi.BOOL,)], [(10, 0, 0), (0, 0, 0), (3, 0, 0)])
    prog = q.compile_sort(spec)
    store = [q.HostRowSet(cols + [bitmap], masks + [None], rows=n)]
    ids = packed_ids([n])[::-1].copy()
    descs, nfs = [True, False, True], [False, False, True]
    want = O.sort(spec, store, ids, descs, nfs)
    got = ids.copy()
    q.Sort(prog, store).sort(got, descs, nfs)
    assert np.array_equal(got, want)


def test_sort_all_equal_keeps_order_and_tiny_inputs():
    spec = queries.SortSpec([(abi.I64,), (abi.I32,)], [(0, 1, 0), (1, 0, 0)])
    prog = q.compile_sort(spec)
    n = 9000
    store = [q.HostRowSet([np.full(n, 7, np.int64), np.full(n, -1, np.int32)])]
    ids = packed_ids([n])[np.random.default_rng(1).permutation(n)]
    got = ids.copy()
    q.Sort(prog, store).sort(got)
    assert np.array_equal(got, ids)
    for m in (0, 1):
        one = ids[:m].copy()
        q.Sort(prog, store).sort(one, n=m)
        assert np.array_equal(one, ids[:m])


def test_sort_device_row_ids_and_materialize_slices():
    n = 70_001
    cols = sort_case(n, 8, 100)
    sizes = [30_000, 40_001]
    spec = queries.sort_k1_desc_k2()
    prog = q.compile_sort(spec)
    store = split(cols, sizes, device=True)
    ids = packed_ids(sizes)
    want = O.sort(spec, split(cols, sizes), ids)
    dids = q.DeviceBuffer(ids.nbytes).upload(ids)
    s = q.Sort(prog, store)
    s.sort(dids)
    assert np.array_equal(dids.download(np.int64, n), want)
    # Slices of the sorted order (sort_exec.cpp:454-490): rows, then 0 at the end.
    full = np.concatenate(cols[:1]), np.concatenate(cols[1:2]), np.concatenate(cols[2:3])
    pos = (want >> 32) * sizes[0] + (want & 0xffffffff)
    at = 0
    for limit in (16384, 16384, 30_000, 16384):
        r, out = s.materialize(dids, at, limit)
        assert r == min(limit, n - at)
        vals, valid = q.read_rowset(out, [abi.I64, abi.I32, abi.I64])
        q.release(out)
        sl = pos[at:at + r]
        for c in range(3):
            assert np.array_equal(vals[c], full[c][sl])
            assert valid[c].all()
        at += r
    r, _ = s.materialize(dids, at, 1024)
    assert r == 0


@pytest.mark.parametrize("n,k,k1_range,desc", [(1_000_000, 1000, None, 0), (200_000, 1000, 20, 0),
                                               (100_000, 257, None, 1), (5000, 10_000, None, 0), (50_000, 1, 7, 1)])
def test_top_k_matches_oracle(n, k, k1_range, desc):
    cols = sort_case(n, 21, k1_range)
    sizes = [n // 2, n - n // 2]
    spec = queries.SortSpec(queries.SORT_COLUMNS, [(0, desc, 0), (1, 0, 0)])
    prog = q.compile_sort(spec)
    ids = packed_ids(sizes)[np.random.default_rng(2).permutation(n)]
    want = O.top_k(spec, split(cols, sizes), ids, k)
    got = ids.copy()
    kk = q.Sort(prog, split(cols, sizes, device=True)).top_k(got, k)
    assert kk == len(want)
    assert np.array_equal(got[:kk], want)


def test_top_k_nullable_float_key():
    n = 60_000
    cols, types, masks, _ = typed_columns(n, 31)
    spec = queries.SortSpec(types, [(4, 0, 1), (0, 1, 0)])
    prog = q.compile_sort(spec)
    sizes = [n]
    ids = packed_ids(sizes)
    for k in (1, 100, 4000):
        want = O.top_k(spec, split(cols, sizes, masks), ids, k)
        got = ids.copy()
        kk = q.Sort(prog, split(cols, sizes, masks)).top_k(got, k)
        assert np.array_equal(got[:kk], want)


def test_sort_50m_rows_order_property():
    """At a size the oracle is not run on: the output is a permutation of the
    input and ordered by (k1 DESC, k2 ASC, input position)."""
    n = 50_000_000
    k1 = np.empty(n, np.int64)
    k2 = np.empty(n, np.int32)
    q.lib().qdb_gen_sort(3, n, k1.ctypes.data, k2.ctypes.data, None)
    k1 //= 1 << 40                                   # ties on k1, so k2 and stability matter
    rowid = np.arange(n, dtype=np.int64)
    sizes = [1 << 24, 1 << 24, n - 2 * (1 << 24)]
    spec = queries.sort_k1_desc_k2()
    prog = q.compile_sort(spec)
    store = split([k1, k2, rowid], sizes, device=True)
    ids = packed_ids(sizes)
    dids = q.DeviceBuffer(ids.nbytes).upload(ids)
    q.Sort(prog, store).sort(dids)
    got = dids.download(np.int64, n)
    pos = (got >> 32) * (1 << 24) + (got & 0xffffffff)
    assert np.array_equal(np.sort(pos), rowid)
    a1, a2 = k1[pos], k2[pos]
    d1 = np.diff(a1)
    assert (d1 <= 0).all()
    same1 = d1 == 0
    d2 = np.diff(a2.astype(np.int64))
    assert (d2[same1] >= 0).all()
    same2 = same1 & (d2 == 0)
    assert (np.diff(pos)[same2] > 0).all()


@pytest.mark.parametrize("case,k,desc", [("random", 1000, 0), ("random", 5000, 1), ("random", 300_000, 0),
                                         ("by_position", 1000, 0), ("by_position", 777, 1),
                                         ("three_values", 1000, 0), ("two_values", 1000, 0)])
def test_top_k_sampled_threshold(case, k, desc):
    """Inputs above the candidate buffer (3M rows): the threshold comes from
    an evenly spread sample; keys ordered by position, and ties so heavy that
    the rows at or below the sampled threshold overflow the buffer (the radix
    select takes over), give the same rows as the oracle."""
    n = 3_000_000
    rng = np.random.default_rng(41)
    if case == "random":
        k1 = rng.integers(-2**63, 2**63 - 1, n, dtype=np.int64)
    elif case == "by_position":
        k1 = np.arange(n, dtype=np.int64) * 3 - 10**6
    else:
        k1 = rng.integers(0, 3 if case == "three_values" else 2, n, dtype=np.int64)
    cols = [k1, rng.integers(0, 100_000, n, dtype=np.int32), np.arange(n, dtype=np.int64)]
    sizes = [1 << 20, 1 << 20, n - 2 * (1 << 20)]
    spec = queries.SortSpec(queries.SORT_COLUMNS, [(0, desc, 0), (1, 0, 0)])
    prog = q.compile_sort(spec)
    ids = packed_ids(sizes)
    want = O.top_k(spec, split(cols, sizes), ids, k)
    dids = q.DeviceBuffer(ids.nbytes).upload(ids)
    kk = q.Sort(prog, split(cols, sizes, device=True)).top_k(dids, k)
    assert kk == k
    assert np.array_equal(dids.download(np.int64, kk), want)


def test_top_k_sampled_key_types():
    """The sampled path over every cell width (1, 2, 4 and 8 bytes), nullable
    keys with NULLs first and last, both directions."""
    n = 2_500_000
    cols, types, masks, _ = typed_columns(n, 43)
    sizes = [n // 2, n - n // 2]
    ids = packed_ids(sizes)
    host, dev = split(cols, sizes, masks), split(cols, sizes, masks, device=True)
    for key, desc, first, k in ((4, 0, 1, 1000), (4, 1, 0, 20_000), (0, 0, 0, 1000), (1, 1, 0, 3000),
                                (3, 0, 1, 1000), (5, 1, 0, 1000), (9, 0, 0, 100), (6, 1, 0, 1000)):
        spec = queries.SortSpec(types, [(key, desc, first), (8, 1, 0)])
        prog = q.compile_sort(spec)
        want = O.top_k(spec, host, ids, k)
        got = ids.copy()
        kk = q.Sort(prog, dev).top_k(got, k)
        assert np.array_equal(got[:kk], want), (key, desc, first, k)
