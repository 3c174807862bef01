"""qdb_gpu_hash over string key columns (QDB_TYPE_STRING, Arrow layout):
bit-exact with the engine's key hash — qdb_string_hash_bytes of each string
(qdb/modules/qumirdb_runtime.cpp:270-300: the short-string mix up to 16
bytes, XXH3-64 with the engine's secret above) as a struct field
(qdb/kernel/gen.cpp:233-379) — for every length branch, NULL strings,
utf8 and large_utf8 offsets, host and device row sets, a selection, and
string keys beside integer keys; and the runtime-filter probe of a row set
keyed by a string."""
import ctypes as C

import numpy as np
import pytest

import qumirdb_b200 as q
from oracle import oracle as O
from qumirdb_b200 import abi

pytestmark = pytest.mark.gpu

N = 20_000


def strings(n, seed):
    rng = np.random.default_rng(seed)
    lens = rng.choice([0, 1, 2, 3, 4, 7, 8, 9, 15, 16, 17, 31, 33, 64, 65, 97, 128, 129, 200, 240, 241, 575, 577,
                       1200, 3000], n)
    lens = np.where(rng.random(n) < 0.5, rng.integers(0, 40, n), lens)
    prefix = b"https://example.org/path/"
    out = []
    for i, m in enumerate(lens):
        body = rng.integers(32, 127, int(m), dtype=np.uint8).tobytes()
        out.append((prefix + body)[:int(m)] if i % 3 == 0 else body)
    return out


def run(cols, schema, keys, masks=None, sel=None, where="host"):
    ct = q.coltypes(schema)
    kc = q.i32s(keys)
    err = C.create_string_buffer(512)
    h = q.lib().qdb_gpu_compile_hash(len(schema), ct, len(keys), kc, err, 512)
    assert h, err.value.decode()
    prog = q.Program(h, keep=(ct, kc))
    want = np.full(N, 0xABCD, np.uint64)
    hrs = q.HostRowSet(cols, masks=masks, selection=sel)
    assert O.lib().oracle_hash(len(schema), C.cast(ct, C.c_void_p), len(keys), C.cast(kc, C.c_void_p), hrs.ptr,
                               want.ctypes.data, err, 512) == 0, err.value
    if where == "host":
        got = np.full(N, 0xABCD, np.uint64)
        assert q.lib().qdb_gpu_hash(prog.handle, hrs.ptr, got.ctypes.data), q.last_error()
    else:
        drs = q.DeviceRowSet(cols, masks=masks, selection=sel)
        buf = q.DeviceBuffer(N * 8).upload(np.full(N, 0xABCD, np.uint64))
        assert q.lib().qdb_gpu_hash(prog.handle, drs.ptr, buf.ptr), q.last_error()
        got = buf.download(np.uint64, N)
    return got, want


@pytest.mark.parametrize("where", ["host", "device"])
@pytest.mark.parametrize("large", [False, True])
def test_string_key_hash_is_bit_exact(where, large):
    vals = strings(N, 5)
    got, want = run([q.StringColumn.of(vals, large=large)], [(abi.STRING,)], [0], where=where)
    np.testing.assert_array_equal(got, want)
    # One non-null field: the struct hash is the string hash plus the
    # combine constant (pinned against XXH3 in tests/test_string_hash.py).
    M = (1 << 64) - 1
    for i in range(0, N, 97):
        assert int(want[i]) == (O.string_hash(vals[i]) + 0x9E3779B97F4A7C15) & M, i


@pytest.mark.parametrize("where", ["host", "device"])
def test_nullable_string_beside_integer_keys_with_selection(where):
    rng = np.random.default_rng(8)
    s = q.StringColumn.of(strings(N, 6))
    k = rng.integers(-10**12, 10**12, N)
    valid = rng.random(N) > 0.15
    sel = (rng.random(N) > 0.3).astype(np.uint8)
    schema = [(abi.I64,), (abi.STRING, 0, 1)]
    for keys in ([1], [0, 1], [1, 0]):
        got, want = run([k, s], schema, keys, masks=[None, valid], sel=sel, where=where)
        np.testing.assert_array_equal(got[sel != 0], want[sel != 0])
        np.testing.assert_array_equal(got[sel == 0], np.full(int((sel == 0).sum()), 0xABCD, np.uint64))


def test_runtime_filter_probe_of_string_keyed_rows():
    """A runtime filter built from the hashes of a build side's string keys;
    the probe side's string-keyed rows tested by qdb_gpu_rf_probe_rowset
    (hash and probe in one kernel) equal the oracle's hash then probe."""
    from qumirdb_b200 import rfilter as RF

    from . import rf_cases as R
    HOST = O.HostStorage()
    dev = RF.DeviceStorage()
    build_vals = [b"key-%06d/" % i + b"x" * (i % 300) for i in range(3000)]
    probe_vals = [build_vals[i % 3000] if i % 4 == 0 else b"other-%d/" % i + b"y" * (i % 250) for i in range(N)]
    cols = [(abi.STRING,)]
    hprog = q.compile_hash(cols, [0])
    bdev = q.DeviceRowSet([q.StringColumn.of(build_vals)])
    hb = dev.alloc(len(build_vals) * 8)
    q.hash_rows(hprog, bdev, hb.ptr)
    host_h = O.hash_rows(cols, [0], q.HostRowSet([q.StringColumn.of(build_vals)])).astype(np.uint64)
    assert (dev.read_u64(hb, len(build_vals)) == host_h).all()
    fd = RF.RuntimeFilter(dev, RF.DEFAULT_MAX_KEYS)
    b = fd.make_builder()
    b.add(hb.ptr, len(build_vals))
    fd.finish_producer(b.take_partial())
    fh = RF.RuntimeFilter(HOST, RF.DEFAULT_MAX_KEYS)
    R.publish_keys(HOST, fh, host_h)
    prs = q.DeviceRowSet([q.StringColumn.of(probe_vals)])
    out = dev.alloc(N)
    kept = RF.probe_rowset(fd, hprog, prs, out.ptr)
    got = dev.read_u8(out, N)
    ph = O.hash_rows(cols, [0], q.HostRowSet([q.StringColumn.of(probe_vals)])).astype(np.uint64)
    want = R.probe(HOST, fh, ph, None)
    assert (got == want).all() and kept == int(want.sum())
    assert kept >= N // 4   # every row whose string the build side holds passes
