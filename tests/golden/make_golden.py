"""Collects the reference's regression fixtures that pin the hot path into
fixtures.json (tables + expected results, copied verbatim).

The reference's SQL regression suites (test/regtest/cases/<suite>/ with
suite.json, tables/*.json and the .sql file; expected rows in
test/regtest/goldens/<suite>/<case>.result.json) are the only result
goldens it has for aggregation, sort and join.  test_golden.py restates each
listed query as this library's operator descriptors and compares the oracle
(CPU) and the device path (GPU) with the expected rows.

usage: python tests/golden/make_golden.py REFERENCE_REGTEST_DIR
(the test/regtest directory of a checkout of the reference)
"""
from __future__ import annotations

import json
import re
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent

CASES = {
    "aggregate_empty": ["empty_count", "empty_mixed", "filter_count", "filter_mixed", "nonempty_mixed",
                        "split_mixed", "all_null_mixed", "nonnullable_empty", "nonnullable_values",
                        "grouped_empty"],
    "decimal_result": ["multiply_sum", "storage_sum"],
    "aggregate_row_layout": ["checksum", "estimated_groups"],
    "float_sql": ["order_asc", "order_desc", "order_nan", "order_nan_limit"],
    "null_order_default": ["sort_i_asc", "sort_i_desc", "sort_f_asc", "sort_f_desc", "sort_b_asc", "sort_b_desc",
                           "sort_date_asc", "sort_date_desc", "sort_multi_key_mixed", "sort_nulls_first_asc",
                           "sort_nulls_last_desc", "top_asc", "top_desc", "top_double_asc", "top_explicit",
                           "top_multi_key", "top_offset_asc", "top_offset_desc", "big_sort_f_asc",
                           "big_sort_f_desc", "big_sort_i_asc", "big_sort_i_desc", "big_top_i_asc",
                           "big_top_f_desc_offset"],
    "selectivity": ["join_composite_key_filtered", "join_shared_key_range", "join_shared_key_range_independent"],
    "outer_join": ["duplicates", "null_keys", "all_matched", "none_matched", "empty_build", "empty_probe",
                   "right_join", "preserved_larger"],
    "anti_join_conditions": ["exists_build_outer_side", "not_exists_filter_above"],
}


def main() -> None:
    if len(sys.argv) != 2:
        sys.exit("usage: make_golden.py REFERENCE_REGTEST_DIR")
    root = Path(sys.argv[1])
    out = {"source": "test/regtest of the reference (cases/<suite>/tables, goldens/<suite>/<case>.result.json)",
           "tables": {}, "cases": {}}
    for suite, cases in CASES.items():
        manifest = json.loads((root / "cases" / suite / "suite.json").read_text())
        for case in cases:
            entry = manifest["cases"].get(case + ".sql", {})
            aliases = dict(manifest.get("tables", {}))
            aliases.update(entry.get("tables", {}))
            sql = (root / "cases" / suite / (case + ".sql")).read_text()
            used = {}
            for alias, fixture in aliases.items():
                if not re.search(rf"\b{re.escape(alias)}\b", sql):
                    continue
                key = f"{suite}/{fixture}"
                if key not in out["tables"]:
                    fx = manifest["fixtures"][fixture]
                    table = json.loads((root / "cases" / suite / fx["json"]).read_text())
                    if "parquet" in fx:
                        table["row_group_rows"] = fx["parquet"]["row_group_rows"]
                    out["tables"][key] = table
                used[alias] = key
            expected = json.loads((root / "goldens" / suite / (case + ".result.json")).read_text())
            out["cases"][f"{suite}/{case}"] = {"sql": sql, "tables": used, "expected": expected}
    (HERE / "fixtures.json").write_text(json.dumps(out, indent=1, sort_keys=True) + "\n")
    print(f"wrote {len(out['cases'])} cases and {len(out['tables'])} tables to {HERE / 'fixtures.json'}")


if __name__ == "__main__":
    main()
