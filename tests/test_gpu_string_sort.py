"""ORDER BY a string column (QDB_TYPE_STRING, Arrow layout) through
qdb_sort_run: the row ids end in the order of the engine's string sort
(sort_string_rowids / _nullable, qdb/kernel/sort/sort_rowids.oz:594-1060:
bytes compared, shorter first on a common prefix, stable, DESC, NULLs first
or last), equal to the oracle's — alone, under an integer key and above one,
over host and device batches, utf8 and large_utf8 offsets, strings sharing
long prefixes and strings up to 300 bytes; a sort whose longest string
needs more stages than are served is refused, as are string keys in the
top-K entries."""
import numpy as np
import pytest

import qumirdb_b200 as q
from oracle import oracle as O
from qumirdb_b200 import abi, queries

pytestmark = pytest.mark.gpu

PER = 4000
BATCHES = 3


def values(n, seed, maxlen=40):
    rng = np.random.default_rng(seed)
    pool = [b"", b"a", b"a\x00", b"ab", b"abcdefgh", b"abcdefgh\x00", b"abcdefghi", b"abcdefgh" * 3,
            b"https://example.org/a", b"https://example.org/b", b"https://example.org/", b"\xff", b"\x00",
            b"x" * 250, b"x" * 250 + b"y", b"x" * 251]
    out = []
    for _ in range(n):
        r = rng.random()
        if r < 0.4:
            out.append(pool[rng.integers(len(pool))])
        elif r < 0.7:
            out.append(b"https://example.org/" + bytes(rng.integers(97, 100, int(rng.integers(0, 12)),
                                                                   dtype=np.uint8)))
        else:
            out.append(bytes(rng.integers(0, 4, int(rng.integers(0, maxlen)), dtype=np.uint8) + 97))
    return out


def store(vals, k, valid, nullable, device, large):
    out = []
    for b in range(BATCHES):
        lo, hi = b * PER, (b + 1) * PER
        cols = [q.StringColumn.of(vals[lo:hi], large=large), k[lo:hi]]
        masks = [valid[lo:hi] if nullable else None, None]
        out.append(q.DeviceRowSet(cols, masks=masks) if device else q.HostRowSet(cols, masks=masks))
    return out


def ids_shuffled(seed):
    ids = np.concatenate([(np.int64(b) << 32) | np.arange(PER, dtype=np.int64) for b in range(BATCHES)])
    np.random.default_rng(seed).shuffle(ids)
    return ids


@pytest.mark.parametrize("device", [False, True])
@pytest.mark.parametrize("large", [False, True])
@pytest.mark.parametrize("nullable", [False, True])
@pytest.mark.parametrize("desc,nulls_first", [(0, 0), (1, 1), (1, 0)])
def test_string_sort_matches_oracle(device, large, nullable, desc, nulls_first):
    n = PER * BATCHES
    vals = values(n, 11 + desc)
    rng = np.random.default_rng(4)
    valid = rng.random(n) > 0.2 if nullable else np.ones(n, bool)
    k = rng.integers(0, 5, n).astype(np.int64)
    types = [(abi.STRING, 0, 1 if nullable else 0), (abi.I64,)]
    st = store(vals, k, valid, nullable, device, large)
    host = store(vals, k, valid, nullable, False, large)
    for keys in ([(0, desc, nulls_first)], [(1, 0, 0), (0, desc, nulls_first)], [(0, desc, nulls_first), (1, 1, 0)]):
        spec = queries.SortSpec(types, keys, out_columns=[1])
        ids = ids_shuffled(7)
        want = O.sort(spec, host, ids)
        got = ids.copy()
        q.Sort(q.compile_sort(spec), st).sort(got)
        np.testing.assert_array_equal(got, want, err_msg=str(keys))


def test_longest_string_beyond_the_stage_budget_is_refused():
    n = PER * BATCHES
    vals = values(n, 3)
    vals[5] = b"z" * 2000
    k = np.zeros(n, np.int64)
    spec = queries.SortSpec([(abi.STRING,), (abi.I64,)], [(0, 0, 0)], out_columns=[1])
    prog = q.compile_sort(spec)
    ids = ids_shuffled(1)
    before = ids.copy()
    with pytest.raises(q.QdbError, match="stages"):
        q.Sort(prog, store(vals, k, np.ones(n, bool), False, False, False)).sort(ids)
    np.testing.assert_array_equal(ids, before)
    with pytest.raises(q.QdbError, match="string keys"):
        q.Sort(prog, store(vals, k, np.ones(n, bool), False, False, False)).top_k(ids, 10)
