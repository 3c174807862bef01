"""Device hash shuffle (qdb_gpu_shuffle) against the oracle's routing of
THashShuffleTask (hash % P, or a route table): each output holds exactly
its rows, in input order, with every column, validity and hash."""
import numpy as np
import pytest

import qumirdb_b200 as q
from oracle import oracle as O
from qumirdb_b200 import abi

pytestmark = pytest.mark.gpu

COLS = [(abi.I64, 0, 1), (abi.I32,), (abi.F64, 0, 1), (abi.DECIMAL128, 2), (abi.CHAR1,)]


def _data(n, seed):
    rng = np.random.default_rng(seed)
    key = rng.integers(-1000, 1000, n).astype(np.int64)
    a = rng.integers(-50, 50, n).astype(np.int32)
    x = rng.random(n)
    d = rng.integers(0, 2**62, 2 * n, dtype=np.int64)
    c = rng.integers(65, 70, n).astype(np.uint8)
    kv = rng.random(n) > 0.05
    xv = rng.random(n) > 0.1
    sel = (rng.random(n) > 0.2).astype(np.uint8)
    return [key, a, x, d, c], [kv, None, xv, None, None], sel


def _check(outs, cols, masks, sel, hashes, routes, nout):
    dest = O.route(hashes, sel, routes, nout)
    assert dest is not None
    for p in range(nout):
        rows = np.nonzero(dest == p)[0]
        o = outs[p]
        assert o.RowCount == len(rows)
        vals, valid = q.read_rowset(o, [c[0] for c in COLS], on_device=True)
        for k, (col, m) in enumerate(zip(cols, masks)):
            want = col.reshape(-1, 2)[rows] if COLS[k][0] == abi.DECIMAL128 else col[rows]
            got = vals[k]
            if COLS[k][0] == abi.DECIMAL128:
                got = np.array([[int(v) & (2**64 - 1), (int(v) >> 64) & (2**64 - 1)] for v in got],
                               dtype=np.uint64).view(np.int64).reshape(-1, 2)
            wm = np.ones(len(rows), bool) if m is None else m[rows]
            assert (valid[k] == wm).all()
            assert (np.asarray(got)[wm] == want[wm]).all()
        h = q._fetch(o.Hash, 8 * o.RowCount, True).view(np.uint64) if o.RowCount else np.empty(0, np.uint64)
        assert (h == hashes[rows]).all()


@pytest.mark.parametrize("nout,routes", [(1, None), (7, None), (300, None), (4, [3, 0, 2, 1, 1, 3, 0, 2])])
def test_shuffle_matches_routing(nout, routes):
    n = 200_000
    cols, masks, sel = _data(n, nout)
    prog = q.compile_hash(COLS, [0])
    hashes = O.hash_rows(COLS, [0], q.HostRowSet(cols, masks)).astype(np.uint64)
    for mk in (q.HostRowSet, q.DeviceRowSet):
        outs = q.shuffle(prog, mk(cols, masks, sel), nout, routes)
        _check(outs, cols, masks, sel, hashes, routes, nout)
        outs.release()


def test_shuffle_uses_the_batch_hash_and_rejects_unrouted_rows():
    n = 10_000
    cols, masks, sel = _data(n, 3)
    prog = q.compile_hash(COLS, [0])
    rs = q.HostRowSet(cols, masks, sel)
    given = np.arange(n, dtype=np.uint64) * 0x9E3779B97F4A7C15
    rs.rs.Hash = given.ctypes.data
    outs = q.shuffle(prog, rs, 5)
    _check(outs, cols, masks, sel, given, None, 5)
    outs.release()
    with pytest.raises(q.QdbError):
        q.shuffle(prog, q.HostRowSet(cols, masks), 2, [0, 1, 2])   # route 2 of 2 outputs
