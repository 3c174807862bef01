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

}  // namespace qdb
