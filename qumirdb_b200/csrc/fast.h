// fast.h — shapes served by the typed fast kernels of fast.cu, and the
// matchers that recognise them in a lowered plan.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "kernels.h"
#include "plan.h"

namespace qdb {

constexpr int kJsMaxStates = 4;

struct JsFactor {
    int32_t side;            // 0 probe column, 1 bucket payload word, 2 build column, 3 staged probe column
    int32_t pad;
    const int64_t* data;     // probe column (row 0 of the batch) or build column
    int64_t c;               // factor = c + d * x
    int64_t d;
};

struct JsState {
    int32_t nf;              // 0: COUNT(*)
    int32_t word;            // state word in the group's slot
    JsFactor f[2];
};

struct JoinSumShape {
    int32_t nstates;
    int32_t need_pay;
    int32_t need_row;        // a factor reads a build column through the arena row
    int32_t pad;
    const int64_t* probe_key;
    const uint8_t* selection;
    JsState states[kJsMaxStates];
};

// Fills `out` when the resolved fused join-aggregate plan has the join-sum
// shape (see fast.cu).
bool MatchJoinSum(const AggPlan& plan, const JoinKeyPlan& jk, int inline_slot, JoinSumShape& out);

// Fills `F` when a resolved (non-join) aggregate plan has the typed row
// shape of FastPlan (plan.h).
bool MatchFast(const AggPlan& plan, FastPlan& F);

void JoinSumRun(const JoinSumShape& shape, const JTableDev& jt, int64_t nrows, uint64_t* group_states,
                AggCounters* counters, cudaStream_t s);

// The probe column every probe factor reads (nullptr: none); false when the
// factors read two probe columns or a build column through the arena row.
bool JoinSumProbeColumn(const JoinSumShape& shape, const int64_t*& vcol);

// One join of a batched join-sum probe.
struct JsBatchJoin {
    JTableDev jt;
    const int64_t* key;             // probe key column
    const int64_t* vcol;            // the probe column the factors read (side 3), or nullptr
    uint64_t* states;               // state words of the join's keyless group
    unsigned long long* matched;    // the join's matched-row counter
};
// Probes many joins of one program in one persistent launch: warps pull work
// items (join, probe-row range) from `next` (zeroed); `shape`'s factors read
// the bucket payload (side 1) or the join's vcol (side 3) only.  joins,
// items and next are device memory.
void JoinSumBatchRun(const JoinSumShape& shape, const JsBatchJoin* joins, const JoinBatchItem* items,
                     int64_t nitems, unsigned* next, cudaStream_t s);

}  // namespace qdb
