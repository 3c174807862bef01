"""The C-ABI library: loads without a GPU, exports every declared entry,
mirrors the engine's struct layouts, and its lowering accepts the workload
descriptors and rejects what the device kernels do not serve (no compute)."""
import ctypes as C

import pytest

import qumirdb_b200 as q
from qumirdb_b200 import abi, queries


def test_library_exports_every_declared_symbol():
    lib = q.lib()
    declared = abi.header_symbols(q.HEADER)
    assert len(declared) >= 30
    missing = [s for s in declared if not hasattr(lib, s)]
    assert not missing, missing
    assert set(declared) <= set(abi.SIGNATURES), set(declared) - set(abi.SIGNATURES)


def test_rowset_layout_matches_the_engine():
    # TColumn / TRowSet (qdb/io/io.h:17-39): 48 and 64 bytes.
    assert C.sizeof(abi.Column) == 48
    assert C.sizeof(abi.RowSet) == 64
    assert abi.RowSet.RowCount.offset == 16
    assert abi.RowSet.Selection.offset == 24


def test_state_sizes_match_the_engine():
    assert abi.HASH_TABLE_SIZE == 304
    assert (abi.ROW_ARENA_SIZE, abi.ROW_TABLE_SIZE, abi.ROW_SCRATCH_SIZE, abi.PAIR_BUFFER_SIZE) == (56, 48, 64, 24)


def test_workload_descriptors_compile():
    q.compile_aggregate(queries.lineitem_agg(9000))
    q.compile_aggregate(queries.zipf_agg(1000))
    j, a = queries.join_sum()
    q.compile_join_aggregate(j, a)
    q.compile_row_join(j)


def test_unserved_aggregate_is_rejected_at_compile_time():
    e = q.ExprBuilder()
    d = e.col(0, abi.DECIMAL128, 2)
    spec = queries.AggSpec([(abi.DECIMAL128, 2)], e, None, [], [(abi.MIN, d)])
    with pytest.raises(q.QdbError, match="DECIMAL128"):
        q.compile_aggregate(spec)


def test_bad_node_order_is_rejected():
    e = q.ExprBuilder()
    e.op(abi.ADD, abi.I64, 1, 2)   # operands after their user
    e.col(0, abi.I64)
    e.col(0, abi.I64)
    spec = queries.AggSpec([(abi.I64,)], e, None, [], [(abi.SUM, 0)])
    with pytest.raises(q.QdbError, match="precede"):
        q.compile_aggregate(spec)
