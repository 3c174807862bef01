"""The oracle's string sort (sort_string_rowids / _nullable,
qdb/kernel/sort/sort_rowids.oz:594-1060: prefix passes, then equal-prefix runs
ordered by the full comparison) against an independent statement of the
order it must produce: a stable sort by bytes (shorter first on a common
prefix), ASC or DESC, NULLs first or last, alone and under an integer key."""
import numpy as np
import pytest

import qumirdb_b200 as q
from oracle import oracle as O
from qumirdb_b200 import abi, queries


def values(n, seed):
    rng = np.random.default_rng(seed)
    pool = [b"", b"a", b"a\x00", b"ab", b"abcdefgh", b"abcdefgh\x00", b"abcdefghi", b"abcdefgh" * 3,
            b"https://example.org/a", b"https://example.org/b", b"https://example.org/", b"\xff", b"\x00"]
    out = []
    for _ in range(n):
        if rng.random() < 0.5:
            out.append(pool[rng.integers(len(pool))])
        else:
            m = int(rng.integers(0, 30))
            out.append(bytes(rng.integers(0, 4, m, dtype=np.uint8) + 97))
    return out


def store(vals, k2, valid, nullable, per=1000):
    """Batches of `per` rows: (string, i64) columns."""
    out = []
    for lo in range(0, len(vals), per):
        out.append(q.HostRowSet([q.StringColumn.of(vals[lo:lo + per]), k2[lo:lo + per]],
                                masks=[valid[lo:lo + per] if nullable else None, None]))
    return out


@pytest.mark.parametrize("desc", [0, 1])
@pytest.mark.parametrize("nulls_first", [0, 1])
@pytest.mark.parametrize("nullable", [False, True])
def test_string_sort_order(desc, nulls_first, nullable):
    n = 3000
    vals = values(n, 3 + desc + 2 * nulls_first)
    rng = np.random.default_rng(9)
    valid = rng.random(n) > 0.2 if nullable else np.ones(n, bool)
    k2 = rng.integers(0, 4, n).astype(np.int64)
    types = [(abi.STRING, 0, 1 if nullable else 0), (abi.I64,)]
    batches = store(vals, k2, valid, nullable)
    ids = np.concatenate([(np.int64(b) << 32) | np.arange(1000, dtype=np.int64) for b in range(3)])
    rng.shuffle(ids)

    def cell(i):
        j = (int(i) >> 32) * 1000 + (int(i) & 0xffffffff)
        return vals[j], bool(valid[j]), int(k2[j])

    # One string key: Python's sort is stable in both directions.
    spec = queries.SortSpec(types, [(0, desc, nulls_first)], out_columns=[1])
    got = O.sort(spec, batches, ids)
    nulls = [i for i in ids if not cell(i)[1]]
    good = sorted([i for i in ids if cell(i)[1]], key=lambda i: cell(i)[0], reverse=bool(desc))
    want = nulls + good if nulls_first else good + nulls
    assert list(got) == want
    # Under an integer key (most significant), the string second.
    spec2 = queries.SortSpec(types, [(1, 0, 0), (0, desc, nulls_first)], out_columns=[1])
    assert list(O.sort(spec2, batches, ids)) == sorted(want, key=lambda i: cell(i)[2])
