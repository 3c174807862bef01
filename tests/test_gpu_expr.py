"""The engine's filter, project and shuffle-hash kernel contracts on the device
(TFilterDispatch, TProjectDispatch and the hash dispatch,
qdb/kernel/compiler.h:426-438, :488-520) against the oracle, called through
the C ABI (qdb_gpu_filter / qdb_gpu_project / qdb_gpu_hash) on host and
device row sets, with input selections, NULLs and every expression functor
the lowering selects (compare, arithmetic, date range, IN-list, CASE, CAST,
MOD, IS NULL)."""
import ctypes as C

import numpy as np
import pytest

import qumirdb_b200 as q
from oracle import oracle as O
from qumirdb_b200 import abi

pytestmark = pytest.mark.gpu

N = 50_003

# Schema of the test table: (type, scale, nullable).
SCHEMA = [(abi.I64, 0, 1), (abi.I32,), (abi.F64, 0, 1), (abi.DATE32,), (abi.DECIMAL64, 2), (abi.CHAR1,),
          (abi.DECIMAL128, 2, 1), (abi.I16,), (abi.U8,)]


def table(n=N, seed=31):
    rng = np.random.default_rng(seed)
    cols = [rng.integers(-10**6, 10**6, n).astype(np.int64),
            rng.integers(-100, 100, n).astype(np.int32),
            rng.normal(0, 100, n),
            rng.integers(10_000, 12_000, n).astype(np.int32),
            rng.integers(-10**9, 10**9, n).astype(np.int64),
            rng.choice(np.frombuffer(b"ANRFO", np.uint8), n),
            np.zeros((n, 2), np.int64),
            rng.integers(-30_000, 30_000, n).astype(np.int16),
            rng.integers(0, 256, n).astype(np.uint8)]
    wide = rng.integers(-2**62, 2**62, n)
    cols[6][:, 0] = wide
    cols[6][:, 1] = np.where(wide < 0, -1, 0) + rng.integers(-3, 3, n)
    # Doubles with the hash's canonical cases: -0.0, +0.0 and NaN.
    cols[2][::97] = -0.0
    cols[2][1::97] = 0.0
    cols[2][2::101] = np.nan
    masks = [rng.random(n) > 0.1, None, rng.random(n) > 0.2, None, None, None, rng.random(n) > 0.15, None, None]
    return cols, masks


def rowsets(cols, masks, selection=None):
    host = q.HostRowSet(cols, masks=masks, selection=selection)
    dev = q.DeviceRowSet(cols, masks=masks, selection=selection)
    return host, dev


def predicates():
    """(name, builder, predicate node) over SCHEMA."""
    out = []

    def case(name, fn):
        e = q.ExprBuilder()
        c = [e.col(k, t[0], (t + (0,))[1]) for k, t in enumerate(SCHEMA)]
        out.append((name, e, fn(e, c)))

    case("lt_i64", lambda e, c: e.op(abi.LT, abi.BOOL, c[0], e.const(1000, abi.I64)))
    case("between_i32", lambda e, c: e.op(abi.BETWEEN, abi.BOOL, c[1], e.const(-10, abi.I32), e.const(40, abi.I32)))
    case("date_range", lambda e, c: e.op(abi.AND, abi.BOOL, e.op(abi.GE, abi.BOOL, c[3], e.const(10_500, abi.DATE32)),
                                         e.op(abi.LT, abi.BOOL, c[3], e.const(11_000, abi.DATE32))))
    case("in_list_i32", lambda e, c: e.in_list(c[1], [-7, 0, 3, 11, 99]))
    case("in_list_char", lambda e, c: e.in_list(c[5], [ord("A"), ord("R")]))
    case("in_list_i64_or_null", lambda e, c: e.op(abi.OR, abi.BOOL, e.in_list(c[0], list(range(-500_000, 500_000, 16_661))),
                                                  e.op(abi.IS_NULL, abi.BOOL, c[2])))
    case("not_f64", lambda e, c: e.op(abi.NOT, abi.BOOL, e.op(abi.GT, abi.BOOL, c[2], e.const(0.5, abi.F64))))
    case("decimal_vs_int", lambda e, c: e.op(abi.GE, abi.BOOL, c[4], e.const(12345, abi.I64)))
    case("case_in_pred", lambda e, c: e.op(abi.EQ, abi.BOOL,
                                           e.op(abi.CASE, abi.I64, e.op(abi.GT, abi.BOOL, c[1], e.const(0, abi.I32)),
                                                e.op(abi.MOD, abi.I64, c[0], e.const(3, abi.I64)), e.const(1, abi.I64)),
                                           e.const(1, abi.I64)))
    case("col_cmp_and_is_not_null", lambda e, c: e.op(abi.AND, abi.BOOL,
                                                      e.op(abi.LT, abi.BOOL, c[7], e.op(abi.CAST, abi.I16, c[1])),
                                                      e.op(abi.IS_NOT_NULL, abi.BOOL, c[6])))
    return out


def compile_filter(eb, pred):
    ct = q.coltypes(SCHEMA)
    nodes = eb.array()
    err = C.create_string_buffer(512)
    h = q.lib().qdb_gpu_compile_filter(len(SCHEMA), ct, len(eb.nodes), nodes, pred, err, 512)
    assert h, err.value.decode()
    return q.Program(h, keep=(ct, nodes, eb))


@pytest.mark.parametrize("where", ["host", "device"])
@pytest.mark.parametrize("name,eb,pred", predicates(), ids=[p[0] for p in predicates()])
def test_filter_matches_oracle(name, eb, pred, where):
    cols, masks = table()
    rng = np.random.default_rng(5)
    insel = (rng.random(N) > 0.3).astype(np.uint8)
    host, dev = rowsets(cols, masks)
    rs = host if where == "host" else dev
    prog = compile_filter(eb, pred)
    for input_sel in (None, insel):
        want = O.filter_rows(SCHEMA, eb, pred, q.HostRowSet(cols, masks=masks, selection=input_sel))
        if where == "host":
            out = np.full(N, 7, np.uint8)
            rs.rs.Selection = out.ctypes.data
            isel = None if input_sel is None else input_sel.ctypes.data
            q.lib().qdb_gpu_filter(prog.handle, rs.ptr, isel)
            got = out
        else:
            out = q.DeviceBuffer(N)
            rs.rs.Selection = out.ptr
            isel_buf = None if input_sel is None else q.DeviceBuffer(N).upload(input_sel)
            q.lib().qdb_gpu_filter(prog.handle, rs.ptr, None if isel_buf is None else isel_buf.ptr)
            got = out.download(np.uint8, N)
        rs.rs.Selection = None
        assert q.last_error() == ""
        np.testing.assert_array_equal(got, want)
        assert 0 < want.sum() < N


def projections():
    e = q.ExprBuilder()
    c = [e.col(k, t[0], (t + (0,))[1]) for k, t in enumerate(SCHEMA)]
    exprs = [
        (e.op(abi.ADD, abi.I64, c[0], e.op(abi.CAST, abi.I64, c[1])), abi.I64),
        (e.op(abi.MUL, abi.I64, c[0], c[0]), abi.I64),                                 # wraps in 64 bits
        (e.op(abi.MUL, abi.DECIMAL128, c[4], e.op(abi.SUB, abi.I64, e.const(100, abi.I64), c[0]), scale=2),
         abi.DECIMAL128),                                                               # decimal * int
        (e.op(abi.ADD, abi.DECIMAL128, c[6], c[4], scale=2), abi.DECIMAL128),            # nullable decimal128
        (e.op(abi.DIV, abi.DECIMAL64, c[4], e.const(7, abi.I64), scale=2), abi.DECIMAL64),  # truncating
        (e.op(abi.MOD, abi.I64, c[0], e.const(13, abi.I64)), abi.I64),                 # sign of the dividend
        (e.op(abi.ADD, abi.F64, c[2], e.op(abi.CAST, abi.F64, c[4])), abi.F64),
        (e.op(abi.CASE, abi.I32, e.in_list(c[5], [ord("A"), ord("N")]), c[1], e.op(abi.NEG, abi.I32, c[1])), abi.I32),
        (e.op(abi.LT, abi.BOOL, c[3], e.const(11_111, abi.DATE32)), abi.BOOL),
        (e.op(abi.ADD, abi.I16, c[7], e.op(abi.CAST, abi.I16, c[8])), abi.I16),         # wraps in 16 bits
    ]
    return e, [x for x, _ in exprs], [t for _, t in exprs]


@pytest.mark.parametrize("where", ["host", "device"])
def test_project_matches_oracle(where):
    cols, masks = table(seed=32)
    eb, exprs, types = projections()
    ct = q.coltypes(SCHEMA)
    nodes = eb.array()
    ex = q.i32s(exprs)
    err = C.create_string_buffer(512)
    h = q.lib().qdb_gpu_compile_project(len(SCHEMA), ct, len(eb.nodes), nodes, len(exprs), ex, err, 512)
    assert h, err.value.decode()
    prog = q.Program(h, keep=(ct, nodes, ex, eb))
    rng = np.random.default_rng(6)
    sel = (rng.random(N) > 0.25).astype(np.uint8)
    host, dev = rowsets(cols, masks)
    rs = host if where == "host" else dev
    widths = [abi.WIDTH[t] for t in types]
    # Oracle: values plus validity.
    want = [np.zeros(N * w, np.uint8) for w in widths]
    valid = [np.zeros(N, np.uint8) for _ in widths]
    wp = (C.c_void_p * len(types))(*[a.ctypes.data for a in want])
    vp = (C.c_void_p * len(types))(*[a.ctypes.data for a in valid])
    hrs = q.HostRowSet(cols, masks=masks, selection=sel)
    assert O.lib().oracle_project(len(SCHEMA), C.cast(ct, C.c_void_p), len(eb.nodes), C.cast(nodes, C.c_void_p),
                                  len(exprs), C.cast(ex, C.c_void_p), hrs.ptr, wp, vp, err, 512) == 0, err.value
    if where == "host":
        got = [np.zeros(N * w, np.uint8) for w in widths]
        ptrs = (C.c_void_p * len(types))(*[a.ctypes.data for a in got])
        q.lib().qdb_gpu_project(prog.handle, rs.ptr, ptrs, None, sel.ctypes.data)
    else:
        bufs = [q.DeviceBuffer(N * w) for w in widths]
        for b in bufs:
            q.lib().qdb_gpu_memset(b.ptr, 0, b.nbytes)
        dsel = q.DeviceBuffer(N).upload(sel)
        ptrs = (C.c_void_p * len(types))(*[b.ptr for b in bufs])
        q.lib().qdb_gpu_project(prog.handle, rs.ptr, ptrs, None, dsel.ptr)
        got = [b.download(np.uint8, N * w) for b, w in zip(bufs, widths)]
    assert q.last_error() == ""
    for k, w in enumerate(widths):
        on = (sel != 0) & (valid[k] != 0)
        g = got[k].reshape(N, w)[on]
        x = want[k].reshape(N, w)[on]
        np.testing.assert_array_equal(g, x, err_msg=f"projection {k} (type {types[k]})")


HASH_CASES = {
    "i64": [0],
    "char1": [5],
    "f64_nullable": [2],
    "decimal128_nullable": [6],
    "date32": [3],
    "i32_char1_i64": [1, 5, 0],
    "decimal64_u8_i16": [4, 8, 7],
    "nullable_mix": [0, 5, 2, 6],
}


@pytest.mark.parametrize("where", ["host", "device"])
@pytest.mark.parametrize("case", list(HASH_CASES))
def test_hash_is_bit_exact_with_the_engine(case, where):
    """qdb_gpu_hash must route rows exactly as the engine's hash % P: the
    struct rh_hash of HashKeyValue (qdb/kernel/gen.cpp:233-379), NULL keys and
    validity fields included; rows the selection rejects keep what the
    caller left in their slot."""
    keys = HASH_CASES[case]
    cols, masks = table(seed=33)
    rng = np.random.default_rng(7)
    sel = (rng.random(N) > 0.2).astype(np.uint8)
    ct = q.coltypes(SCHEMA)
    kc = q.i32s(keys)
    err = C.create_string_buffer(512)
    h = q.lib().qdb_gpu_compile_hash(len(SCHEMA), ct, len(keys), kc, err, 512)
    assert h, err.value.decode()
    prog = q.Program(h, keep=(ct, kc))
    host, dev = rowsets(cols, masks, selection=sel)
    want = np.full(N, 0xABCD, np.uint64)
    O_rs = q.HostRowSet(cols, masks=masks, selection=sel)
    assert O.lib().oracle_hash(len(SCHEMA), C.cast(ct, C.c_void_p), len(keys), C.cast(kc, C.c_void_p), O_rs.ptr,
                               want.ctypes.data, err, 512) == 0, err.value
    if where == "host":
        got = np.full(N, 0xABCD, np.uint64)
        assert q.lib().qdb_gpu_hash(prog.handle, host.ptr, got.ctypes.data)
    else:
        buf = q.DeviceBuffer(N * 8).upload(np.full(N, 0xABCD, np.uint64))
        assert q.lib().qdb_gpu_hash(prog.handle, dev.ptr, buf.ptr)
        got = buf.download(np.uint64, N)
    np.testing.assert_array_equal(got, want)
    # Routing as THashShuffleTask does (hash % P).
    for parts in (3, 16, 64):
        np.testing.assert_array_equal(got[sel != 0] % parts, want[sel != 0] % parts)


def test_in_list_longer_than_a_device_plan_is_rejected_at_compile():
    """A plan holds at most 64 IN-list constants; a longer list is refused
    when the program is compiled (there is no CPU fallback to take it)."""
    e = q.ExprBuilder()
    c0 = e.col(0, abi.I64)
    pred = e.in_list(c0, list(range(100)))
    ct = q.coltypes(SCHEMA)
    nodes = e.array()
    err = C.create_string_buffer(512)
    assert not q.lib().qdb_gpu_compile_filter(len(SCHEMA), ct, len(e.nodes), nodes, pred, err, 512)
    assert "IN list" in err.value.decode()
