// lower.h — host lowering of qdb_gpu.h descriptors into device plans.
//
// The lowering selects, per expression, one of the hand-written device
// functors of eval.h: conjunctions of comparison / range / IN-list / NULL
// atoms for predicates, sums of products of affine factors for values, and
// the generic per-row program for every other tree (CASE, OR-of-ANDs, mixed
// widths, f64 trees whose rounding order the fast form would change).
#pragma once

#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/qdb_gpu.h"
#include "plan.h"

namespace qdb {

struct LowerError : std::runtime_error {
    using std::runtime_error::runtime_error;
};

struct TypeInfo {
    uint8_t load;       // LoadKind
    uint8_t width;      // bytes (0 for bit-packed booleans)
    uint8_t dom;        // GDomain
    uint8_t wrap_bits;
    uint8_t is_unsigned;
    uint8_t key_bits;   // bits of a packed group key
};

TypeInfo InfoOf(int type);
int StorageWidth(int type);   // bytes per value of a device output column

// Maps the input columns a plan reads onto plan column slots.
struct ColumnMap {
    std::vector<int> slot_of;     // input column -> slot (-1 unused)
    std::vector<int> input_of;    // slot -> input column
};

// Output description of the finalize projection of an aggregate.
struct OutputPlan {
    int32_t n = 0;                // output columns
    int32_t row_cols = 0;         // keys ++ aggregates
    uint8_t roots[kMaxCols + kMaxAggs];
    int32_t out_type[kMaxCols + kMaxAggs];
    int32_t out_scale[kMaxCols + kMaxAggs];
    uint8_t row_dom[kMaxCols + kMaxAggs];     // GDomain of each row column
    int16_t row_scale[kMaxCols + kMaxAggs];
    int32_t root_max = -1;
    GProg prog;
    int64_t list[kMaxList];
    bool identity = true;         // output = the aggregate row
};

struct AggLowering {
    AggPlan plan;
    ColumnMap cols;
    OutputPlan out;
    std::vector<int> row_types;   // keys ++ aggregates
    std::vector<int> row_scales;
    bool any_generic = false;
};

// `probe_cols` >= 0 marks a fused join: input columns >= probe_cols are
// build payload columns.  `first_inputs` are mapped to slots 0.. first (the
// probe key columns of a fused join).
AggLowering LowerAggregate(const qdb_aggregate_spec& s, int probe_cols = -1,
                           const std::vector<int>& first_inputs = {});

// Filter / project plans reuse AggPlan's predicate and value sections.
struct ExprLowering {
    AggPlan plan;
    ColumnMap cols;
    std::vector<int> value_src;   // per project output: VS_SOP / VS_GENERIC
    std::vector<int> value_idx;
    std::vector<int> out_types;
};

ExprLowering LowerFilter(int ncols, const qdb_column_type* columns, int nnodes,
                         const qdb_expr* nodes, int predicate);
ExprLowering LowerProject(int ncols, const qdb_column_type* columns, int nnodes,
                          const qdb_expr* nodes, int nexprs, const int32_t* exprs);

}  // namespace qdb
