// runtime.h — host runtime shared by the C ABI translation units.
#pragma once

#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "../../include/qdb_gpu.h"
#include "kernels.h"
#include "lower.h"

namespace qdb {

extern thread_local std::string t_error;
void SetErr(const char* fmt, ...);
bool CudaOk(cudaError_t e, const char* what);
cudaStream_t CurStream();
void* DevAlloc(size_t bytes, cudaStream_t s);
void DevFree(void* p, cudaStream_t s);
struct AggCounters;
AggCounters* PinnedCountersGet();
// Host output buffers: pinned (page-locked) memory from a size-class pool,
// so output copies run at full link speed; returned to the pool on free.
void* HostOutAlloc(size_t bytes);
void HostOutFree(void* p);
void PinnedCountersPut(AggCounters* c);
bool IsDevicePtr(const void* p);
int64_t NextPow2(int64_t v);

// Device copies of host buffers for the duration of one call.
struct Staging {
    explicit Staging(cudaStream_t st) : s(st) {}
    ~Staging();
    const void* Device(const void* p, size_t bytes);
    cudaStream_t s;
    std::vector<void*> owned;
    // Device allocations met during this call: a pointer inside one needs no
    // driver query (many row sets of a batch slice the same columns).
    std::vector<std::pair<uintptr_t, uintptr_t>> dev_ranges;
};

bool ResolveColumns(AggPlan& P, const ColumnMap& cm, const qdb_column_type* types, const qdb_rowset* rs,
                    Staging& st);
AggPlan OffsetPlan(const AggPlan& P, int64_t begin);

// Device memory shared by the tables of a batch of aggregate states; freed
// with the last state that uses it.
struct AggArena {
    void* p = nullptr;
    int64_t refs = 0;
    cudaStream_t s = nullptr;
};
void AggArenaRelease(AggArena* a);

constexpr uint32_t kAggMagic = 0x51444741;   // 'QDGA'
constexpr int64_t kChunkRows = int64_t(64) << 20;

// Device state behind an aggregate's caller-owned HashTable buffer.
struct AggTableState {
    uint32_t magic = kAggMagic;
    cudaStream_t s = nullptr;
    GTableDev t;
    AggCounters* dc = nullptr;      // device counters
    AggCounters* hc = nullptr;      // pinned host mirror
    int64_t groups = 0;
    int64_t expected = 0;
    int64_t* deferred[2] = {nullptr, nullptr};
    int64_t deferred_cap = 0;
    uint64_t* spill = nullptr;
    int64_t spill_cap = 0;
    int smem_slots = 2048;
    int64_t matched = 0;
    AggArena* arena = nullptr;      // batch-created: table and counters may live here
    bool table_in_arena = false;
    bool dc_in_arena = false;
    uint64_t* seeds = nullptr;      // heavy-hitter keys of the shared tier (device), then their count
    bool seeded = false;            // sampled once, from the first large update
};

AggTableState* StateOf(void* ht);
int SlotWords(const AggPlan& p, bool wide);
bool AllocTable(const AggPlan& p, int64_t capacity, cudaStream_t s, GTableDev& t);
bool Grow(AggTableState* st, const AggPlan& p, int64_t min_groups);
bool EnsureBuffers(AggTableState* st, const AggPlan& p, int64_t rows);
bool ReadCounters(AggTableState* st);
void ResetCounters(AggTableState* st);
void MirrorHeader(void* ht, const AggTableState* st, const AggPlan& p);
// Grows the table and replays `ndef` deferred rows (st->deferred[0], as
// (row, build row) pairs) and `nspill` spilled entries (st->spill) of an
// update described by `a`, until none is left.
bool AggReplay(AggTableState* st, const AggPlan& plan, const AggUpdateArgs& a, int64_t ndef, int64_t nspill);
AggTableState* AggStateCreate(const AggPlan& p, int64_t capacity_hint, int64_t expected, cudaStream_t s);
void AggStateDestroy(AggTableState* st);
bool AggRun(AggTableState* st, const AggPlan& plan, int64_t rows, const JoinKeyPlan* jk, const JTableDev* jt,
            int inline_slot = -1);
int64_t AggFinish(AggTableState* st, const AggLowering& lw, uint32_t flags, qdb_rowset* out);
struct JoinSumShape;
bool AggRunJoinSum(AggTableState* st, const JoinSumShape& shape, const JTableDev& jt, int64_t nrows);
// Batched join-sum: the keyless group's state words and matched counter of a
// state (its counters reset on its stream); once the batch has run, Fetch
// queues the counters' read-back on stream s and, after s has drained,
// Commit adds the matched rows.
void AggJoinSumTargets(AggTableState* st, uint64_t** states, unsigned long long** matched);
void AggJoinSumFetch(AggTableState* st, cudaStream_t s);
bool AggJoinSumCommit(AggTableState* st);
int64_t AggStateGroups(const AggTableState* st);
int64_t AggStateMatched(const AggTableState* st);
AggTableState* AggStateOf(void* ht);
void AggMirrorHeader(void* ht, const AggTableState* st, const AggPlan& p);

// Output columns of `rows` rows.  With `blk` (and validity) they are carved
// from one device block: data, then string offsets, then the validity words
// of all columns side by side, cleared by one memset (so runs of never-NULL
// columns are preset by one memset each); EmitRowset given the same block
// hands it to the row set whole, or copies it to the host in one transfer.
struct OutBlock {
    void* p = nullptr;
    size_t bytes = 0;
};
bool AllocOutputCols(const std::vector<int>& types, int64_t rows, bool with_valid, std::vector<AggOutputCol>& cols,
                     cudaStream_t s, OutBlock* blk = nullptr);
bool EmitRowset(std::vector<AggOutputCol>& cols, const std::vector<int>& types, int64_t rows, bool on_device,
                cudaStream_t s, qdb_rowset* out, const OutBlock* blk = nullptr);

struct JoinProgram {
    int32_t build_is_left = 0;
    int32_t join_type = QDB_JOIN_INNER;
    bool emit_unmatched = false;      // outer join streaming its preserved side
    bool marks_build = false;         // LEFT_SEMI / LEFT_ANTI building the left side
    bool keeps_null_keys = false;     // LEFT_ANTI: NULL-key build rows in a second arena
    std::vector<qdb_column_type> build_columns;
    std::vector<qdb_column_type> probe_columns;
    std::vector<int> build_keys;
    std::vector<int> probe_keys;
    std::vector<int> payload;
    std::vector<int> out_side;
    std::vector<int> out_column;
    bool has_build_filter = false;
    ExprLowering build_filter;        // over the build schema (filter + key NULL rejection)
    JoinKeyPlan build_jk;             // col = build input column
    JoinKeyPlan probe_jk;             // col = probe input column
    JoinKeyPlan agg_jk;               // col = fused plan slot of the probe key
};

struct SortProgram {
    std::vector<qdb_column_type> columns;
    std::vector<qdb_sort_key> keys;
    std::vector<int> out_columns;
};

}  // namespace qdb

struct qdb_gpu_program {
    int kind = 0;
    uint32_t flags = 0;
    int64_t expected_groups = 0;
    std::vector<qdb_column_type> columns;     // scan / probe / aggregate input schema
    qdb::AggLowering agg;
    qdb::ExprLowering expr;
    qdb::JoinProgram join;
    qdb::SortProgram sort;
};

namespace qdb {
// The struct rh_hash of a hash program's key slots over nrows rows (the
// plan's columns resolved for the batch).
void HashArgs(const qdb_gpu_program* prog, const AggPlan& plan, int64_t nrows, ExprArgs& a);
}  // namespace qdb


namespace qdb {
enum ProgramKind { PK_AGG = 1, PK_FILTER, PK_PROJECT, PK_HASH, PK_JOIN, PK_JOIN_AGG, PK_SORT };
}
