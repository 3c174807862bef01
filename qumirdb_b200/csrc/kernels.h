// kernels.h — host-side launchers of the device kernels (implemented in the
// .cu files), called by the runtime that serves the C ABI.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <string>

#include "plan.h"

namespace qdb {

constexpr uint64_t kEmptyKey = ~0ull;

// Device-resident counters of one table state.
struct AggCounters {
    unsigned long long new_groups;
    unsigned long long deferred;
    unsigned long long spilled;
    unsigned long long matched;     // fused join: joined rows folded in
    int error;
    unsigned next_chunk;            // work queue head of the listed-row kernel (zeroed with the rest)
};

// Global open-addressing group table in HBM: capacity slots plus one slot for
// the one-word key that equals kEmptyKey.  Slot = [status?][key][states].
struct GTableDev {
    uint64_t* slots = nullptr;
    int64_t capacity = 0;          // power of two
    int32_t slot_words = 0;
    int32_t key_off = 0;           // 1 when the slot leads with a status word
    int32_t state_off = 0;
    int32_t wide = 0;              // multi-word keys claimed by status word
};

// Packed equi-join key over up to four columns (one word).
struct JoinKeyPlan {
    int32_t n = 0;
    int32_t full64 = 0;            // the packed key may equal kEmptyKey
    uint8_t col[4] = {};           // plan column slots (probe) / input columns (build)
    uint8_t bits[4] = {};
    uint8_t shift[4] = {};
    uint8_t is_float[4] = {};
};

// Built join table: buckets of two slots, one 32-byte sector each: words
// [4b, 4b+1] the packed keys of slots 2b, 2b+1 and words [4b+2, 4b+3] their
// first payload words; rows[2b + j] is the arena row of slot 2b + j.  EMPTY
// key = kEmptyKey.  A bucket fills slot 0 before slot 1, and a key only lands
// in a later bucket when both slots of the earlier ones were taken, so a probe
// stops at the first empty slot.  Rows whose key equals kEmptyKey are listed
// separately as (arena row, payload word).
struct JTableDev {
    const uint64_t* buckets = nullptr;
    uint64_t bmask = 0;                               // bucket count - 1
    const int64_t* rows = nullptr;
    const int64_t* special_rows = nullptr;
    const unsigned long long* nspecial = nullptr;   // device count of special rows
    // Blocked Bloom filter over the table's keys (one 32-bit word per key,
    // two bits set), small enough for a CTA's shared memory; nullptr: none.
    const uint32_t* bloom = nullptr;
    int32_t bloom_words = 0;
    // Direct-address index, built when the table has one integer key whose
    // build values are unique and span a dense range (nullptr: none).  Entry
    // key - dense_min holds {key, first 8-byte payload word} ({kEmptyKey, 0}
    // when absent); a presence bitmap over the range, each bit covering
    // 2^dense_shift keys, fits a CTA's shared memory.
    const ulonglong2* dense = nullptr;
    int64_t dense_min = 0;
    uint64_t dense_range = 0;
    const uint32_t* dense_bits = nullptr;
    int32_t dense_words = 0;
    int32_t dense_shift = 0;
};
constexpr int32_t kMaxBloomWords = 32768;   // 128 KB

// Bloom filter word and bits of a mixed key hash h (shared by build and probe).
__host__ __device__ __forceinline__ uint32_t BloomWord(uint64_t h, int32_t nwords) {
    return uint32_t((uint64_t(uint32_t(h >> 32)) * uint32_t(nwords)) >> 32);
}
__host__ __device__ __forceinline__ uint32_t BloomBits(uint64_t h) {
    return (1u << (h & 31)) | (1u << ((h >> 5) & 31));
}
void JoinBuildBloom(const JTableDev& jt, uint32_t* bloom, int32_t nwords, cudaStream_t s);

struct AggUpdateArgs {
    const AggPlan* plan = nullptr;
    int64_t nrows = 0;
    const int64_t* index = nullptr;   // index mode: (row, build row) pairs
    int64_t nindex = 0;
    GTableDev table;
    AggCounters* counters = nullptr;
    int64_t* deferred = nullptr;       // (row, build row) pairs
    int64_t deferred_cap = 0;
    uint64_t* spill = nullptr;
    int64_t spill_cap = 0;
    int32_t smem_slots = 0;            // 0 disables the shared-memory tier
    bool priv = false;                 // lane-private accumulators for the first groups
    const FastPlan* fast = nullptr;    // typed row shape, when the plan has one
    int32_t inline_slot = -1;          // fused join: slot served by the entry's payload word
    bool join = false;
    JoinKeyPlan jkey;
    JTableDev jt;
    const uint64_t* seeds = nullptr;  // high-cardinality kernel: shared-tier seeds (device)
    const int* nseed = nullptr;       // their count (device)
};

struct AggOutputCol {
    int32_t type;
    char* data;           // device, rows * width
    int32_t* offsets;     // CHAR1 outputs: rows + 1 i32 string offsets
    uint32_t* valid;      // validity bitmap (words) or nullptr
};

// Launch geometry chosen per device.
int DeviceSMs();
size_t MaxSmemOptin();

void AggInitTable(const AggPlan& p, const GTableDev& t, cudaStream_t s);
// Returns the shared-memory slots actually used by the launch.
void AggUpdate(const AggUpdateArgs& a, cudaStream_t s);
// Heavy-hitter seeds of a high-cardinality typed plan (a key column and a
// COUNT state): the up-to-k most frequent keys of an evenly strided sample of
// its rows (filter and selection aside) go to seeds[0, *nseed) on stream s (`scratch`: device,
// AggSeedScratch() bytes, free once s has passed the call).  The
// high-cardinality kernel pre-loads them into its shared tier.
bool AggHighSeedable(const AggPlan& p, const FastPlan& f);
size_t AggSeedScratch();
bool AggSeedHeavy(const AggPlan& p, const FastPlan& f, int64_t nrows, uint64_t* seeds, int* nseed, int k,
                  void* scratch, cudaStream_t s);
void AggRehash(const AggPlan& p, const GTableDev& from, const GTableDev& to, AggCounters* c,
               cudaStream_t s);
void AggMergeSpill(const AggPlan& p, const uint64_t* spill, int64_t n, const GTableDev& t,
                   AggCounters* c, cudaStream_t s);
// Writes every group of `t` into `cols`; `scratch` holds >= AggFinalizeScratch
// bytes.  `out` describes the output projection (see lower.h OutputPlan).
// `packed`: the columns' validity words were carved side by side from one
// allocation (AllocOutputCols with a block), so abutting masks are preset by
// one memset.
struct OutputPlan;
size_t AggFinalizeScratch(const GTableDev& t);
void AggFinalize(const AggPlan& p, const OutputPlan& out, const GTableDev& t, AggOutputCol* cols,
                 int ncols, int64_t groups, void* scratch, int* err, cudaStream_t s, bool packed = false);

// One whole aggregate in the file-scope scratch array of agg.cu (no device
// allocation): returns the group count, or -1 with `err` set.
constexpr size_t kNoAllocScratchBytes = size_t(16) << 20;
int64_t AggRunNoAlloc(const AggPlan& plan, const OutputPlan& out, int64_t nrows, AggOutputCol* cols, int ncols,
                      int64_t out_capacity, bool priv, cudaStream_t s, std::string& err);

// ---- join ----
struct JoinBuildArgs {
    // Build columns (device): key columns per JoinKeyPlan.col (input index).
    const char* key_data[4];
    const uint8_t* key_mask[4];
    int64_t key_mask_off[4];
    uint8_t key_width[4];
    uint8_t key_signed[4];
    JoinKeyPlan jkey;
    int64_t nrows;
    const int64_t* pay0;    // first 8-byte payload column (stored in the bucket) or nullptr
    uint64_t* buckets;      // (bmask + 1) * 4 words
    uint64_t bmask;
    int64_t* rows;          // (bmask + 1) * 2 arena rows
    int64_t* special_rows;
    unsigned long long* nspecial;
    int64_t row_base;       // arena row of build row 0
};
void JoinInitTable(uint64_t* buckets, int64_t nbuckets, cudaStream_t s);
void JoinBuild(const JoinBuildArgs& a, cudaStream_t s);
// Work item of a launch over many tables: table `join`, range [lo, hi).
struct JoinBatchItem {
    int32_t join;
    int32_t pad;
    int64_t lo;
    int64_t hi;
};
// Many tables in one launch (args and items in device memory): with init,
// item ranges are bucket ranges to clear; otherwise arena-row ranges to insert.
void JoinBuildBatch(const JoinBuildArgs* args, const JoinBatchItem* items, int64_t nitems, bool init,
                    cudaStream_t s);
// Radix partitioning of join rows for tables larger than L2: partition =
// home bucket (Fmix64(key) & bmask) >> part_shift, so partition p's rows
// touch only bucket slice p (and the slot after a full bucket).
// Build rows (packed keys, the first 8-byte payload word, the arena row):
// counts[p] += rows of partition p; then each row goes to cursor[p]++.
void JoinPartCountBuild(const JoinBuildArgs& a, int part_shift, int nparts, unsigned long long* counts,
                        cudaStream_t s);
void JoinPartScatterBuild(const JoinBuildArgs& a, int part_shift, int nparts, unsigned long long* cursor,
                          uint64_t* keys, int64_t* pays, int64_t* rows, cudaStream_t s);
// Inserts n partitioned build rows (as JoinBuild, from the arrays).
void JoinBuildRows(const JoinBuildArgs& a, const uint64_t* keys, const int64_t* pays, const int64_t* rows, int64_t n,
                   cudaStream_t s);
// Probe rows of an 8-byte key column (and one 8-byte value column, or none).
void JoinPartCountProbe(const int64_t* key, int64_t n, uint64_t bmask, int part_shift, int nparts,
                        unsigned long long* counts, cudaStream_t s);
void JoinPartScatterProbe(const int64_t* key, const int64_t* val, int64_t n, uint64_t bmask, int part_shift,
                          int nparts, unsigned long long* cursor, int64_t* out_key, int64_t* out_val, cudaStream_t s);
constexpr int kMaxJoinParts = 256;
// Bucket tables above this size are built and probed by partition: a slice
// of at most kJoinSliceBytes is what one partition's rows touch, so it stays
// in the 126 MB L2 beside the streamed rows.
constexpr int64_t kJoinPartitionBytes = int64_t(48) << 20;
constexpr int64_t kJoinSliceBytes = int64_t(24) << 20;
// Partitions for a table of nbuckets 32-byte buckets (1: none) and the
// shift from a bucket index to its partition.
inline int JoinPartsFor(int64_t nbuckets, int& part_shift) {
    part_shift = 0;
    if (nbuckets * 32 <= kJoinPartitionBytes) return 1;
    int parts = 1;
    while (nbuckets * 32 / parts > kJoinSliceBytes && parts < kMaxJoinParts) parts *= 2;
    int lb = 0;
    while ((int64_t(1) << lb) < nbuckets) ++lb;
    int lp = 0;
    while ((1 << lp) < parts) ++lp;
    part_shift = lb - lp;
    return parts;
}

// Smallest and largest key of the build rows (a single integer key): out[0]
// and out[1] as int64, preset to INT64_MAX / INT64_MIN by the caller.
void JoinKeyRange(const JoinBuildArgs& a, long long* out, cudaStream_t s);
// Fills the direct-address index of the build rows over [kmin, kmin + range):
// entries (preset here), the presence bitmap (words of 32 bits, each bit for
// 2^shift keys) and *dup, the count of keys met twice.
void JoinDenseBuild(const JoinBuildArgs& a, ulonglong2* dense, int64_t kmin, uint64_t range, uint32_t* bits,
                    int32_t words, int32_t shift, unsigned long long* dup, cudaStream_t s);

struct JoinProbeArgs {
    const char* key_data[4];
    const uint8_t* key_mask[4];
    int64_t key_mask_off[4];
    uint8_t key_width[4];
    uint8_t key_signed[4];
    const uint8_t* selection;
    JoinKeyPlan jkey;
    JTableDev jt;
    int64_t nrows;
    int64_t* pairs;          // (probe row, build row)
    int64_t pair_cap;
    int64_t pair_base;       // pairs already written before this probe's
    int32_t emit_unmatched;  // outer join: a valid-key row with no match pairs with -1
    int* err;
};
// The pair probe in two passes: per-row match counts plus per-chunk totals
// (JoinPairChunks(nrows) of them), then, after an exclusive scan of the
// totals, the pairs themselves at their offsets (probe rows ascending, a
// row's build rows in append order).  Pairs past pair_cap are not written.
int64_t JoinPairChunks(int64_t nrows);
void JoinProbeCount(const JoinProbeArgs& a, uint32_t* counts, unsigned long long* chunk_tot, cudaStream_t s);
void JoinProbeWrite(const JoinProbeArgs& a, const uint32_t* counts, const unsigned long long* chunk_off,
                    cudaStream_t s);
// flags[r] = 1 for a selected probe row whose key is NULL (an outer join
// pads those first, as jr_probe_batch's collect pass does).
void JoinNullKeyFlags(const JoinProbeArgs& a, uint8_t* flags, cudaStream_t s);
// SEMI / ANTI probe: marks[arena row] = 1 for every build row a selected
// valid-key probe row matches.
void JoinMarkProbe(const JoinProbeArgs& a, uint8_t* marks, cudaStream_t s);
// flags[i] = (marks[i] != 0) == want over arena rows; every row when marks
// is null.
void JoinMarkFlags(const uint8_t* marks, int64_t n, int want, uint8_t* flags, cudaStream_t s);
// Pair rows from compacted indices: mode 0 (idx, -1) a padded probe row;
// mode 1 (-1, idx) a build row of the arena; mode 2 (-1, -(idx + 2)) a row
// of the NULL-key arena.
void JoinWritePairs(const int64_t* idx, int64_t n, int64_t* out, int mode, cudaStream_t s);

// Gathers rows: out[i] = src[idx[i]] for `width`-byte values (idx < 0 -> 0;
// with src2, idx <= -2 reads src2[-idx - 2]).
void GatherColumn(const char* src, int width, const int64_t* idx, int idx_stride, int64_t n, char* out,
                  cudaStream_t s, const char* src2 = nullptr);
// Sets bit (out_bit_off + i) of out_words (pre-zeroed) for every valid
// gathered row i (idx == -1 is NULL; idx <= -2 reads mask2 when has2).
void GatherValidity(const uint8_t* mask, int64_t mask_off, const int64_t* idx, int idx_stride, int64_t n,
                    uint32_t* out_words, int64_t out_bit_off, cudaStream_t s, bool has2 = false,
                    const uint8_t* mask2 = nullptr);

// In-place exclusive scan of n counters (one block; n up to a few million).
void ExclusiveScanU64(unsigned long long* counts, int64_t n, cudaStream_t s);

// ---- filter / project / hash over one row set ----
struct ExprArgs {
    const AggPlan* plan = nullptr;   // filter and value sections, columns resolved
    int64_t nrows = 0;
    // Filter: writes out_sel[r] (selected input rows that pass); also rows
    // whose `null_reject` slots are NULL fail (join keys).
    uint8_t* out_sel = nullptr;
    int32_t n_null_reject = 0;
    uint8_t null_reject[4] = {};
    // Set: the other way round, a selected row passes only when one of the
    // null_reject slots IS NULL (the NULL-key rows an ANTI join keeps).
    int32_t null_keys_only = 0;
    // Project: output k = value (src, idx) stored with type out_type[k].
    int32_t nout = 0;
    uint8_t out_src[kMaxCols] = {};
    uint8_t out_idx[kMaxCols] = {};
    int32_t out_type[kMaxCols] = {};
    void* out_ptr[kMaxCols] = {};
    // Hash: struct rh_hash over key slots with their qdb types.
    int32_t nhash = 0;
    uint8_t hash_slot[kMaxKeyParts] = {};
    int32_t hash_type[kMaxKeyParts] = {};
    uint8_t hash_nullable[kMaxKeyParts] = {};   // the key struct has a validity field
    uint64_t* hashes = nullptr;
    // With rf_out, the hash kernel writes rf_out[r] = 1 for a selected row
    // whose hash the runtime filter (rf_kind 1 exact / 2 Bloom over
    // rf_words[0, rf_nwords)) may contain, else 0, and counts those rows in
    // *rf_kept, instead of writing the hash.
    uint8_t* rf_out = nullptr;
    const uint64_t* rf_words = nullptr;
    int64_t rf_kind = 0;
    int64_t rf_nwords = 0;
    unsigned long long* rf_kept = nullptr;
    int* err = nullptr;
};
void FilterRows(const ExprArgs& a, cudaStream_t s);
void ProjectRows(const ExprArgs& a, cudaStream_t s);
void HashRows(const ExprArgs& a, cudaStream_t s);
// Indices (ascending) of the rows with flags[r] != 0; returns nothing on the
// host: the count lands in *d_count (device).  `scratch` >= CompactScratch(n).
size_t CompactScratch(int64_t n);
void CompactFlags(const uint8_t* flags, int64_t n, int64_t* out_idx, unsigned long long* d_count, void* scratch,
                  cudaStream_t s);

// ---- batched aggregate: many aggregates of one program per launch ----
// One aggregate of a batched launch: its columns (the program's typed shape
// columns, at the aggregate's row 0), selection, rows and global table.
struct HighTask {
    const char* cols[kFastCols];
    const uint8_t* sel;
    int64_t nrows;
    GTableDev T;
};
// A work item: rows [row0, row0 + nrows) of one aggregate.
struct HighItem {
    int32_t task;
    int32_t nrows;
    int64_t row0;
};
struct BatchCounters {
    unsigned long long next_item;   // work queue head
    unsigned long long ndeferred;
    unsigned long long nspill;
    int error;
    int pad;
};
struct HighBatch {
    const HighTask* tasks;
    const HighItem* items;
    int64_t nitems;
    unsigned long long* new_groups;   // per aggregate
    BatchCounters* counters;
    int64_t* deferred;                // (row, aggregate) pairs
    int64_t deferred_cap;
    uint64_t* spill;                  // [key, states..., aggregate] records
    int64_t spill_cap;
};
// The program's batched kernel exists when its typed shape was compiled in
// for its cardinality class (`low`: a few groups per aggregate, folded into
// lane-private accumulators; else a shared tier in front of the table).  The
// low-cardinality kernel has a fixed block shape (threads and shared-tier
// slots are ignored) and wants every task's columns on a four-value boundary
// and its selection on a four-byte one.
bool AggBatchSupported(const AggPlan& p, const FastPlan& f, bool low);
// A name of the program's typed shape and class (the autotuner's key).
std::string AggBatchShapeKey(const AggPlan& p, const FastPlan& f, bool low);
// Resident CTAs per SM of the batched kernel at this block shape.
int AggBatchOccupancy(const AggPlan& p, const FastPlan& f, int threads, int smem_slots, bool low);
void AggBatchUpdate(const AggPlan& p, const FastPlan& f, const HighBatch& b, int threads, int smem_slots, int grid,
                    cudaStream_t s, bool low);
void AggBatchReplay(const AggPlan& p, const FastPlan& f, const HighBatch& b, const int64_t* pairs, int64_t n,
                    cudaStream_t s, bool low);
void AggBatchSpill(const AggPlan& p, const HighBatch& b, const uint64_t* recs, int64_t n, cudaStream_t s);
// Initialises `total` slots laid out like the tables of `tasks` (contiguous
// tables of one slot layout), then marks each table's one-word-key flag slot
// (and, keyless, its group at key 0).
void AggBatchInitTables(const AggPlan& p, const GTableDev& all, const HighTask* tasks, int ntasks,
                        cudaStream_t s);
// Batched finalize: block b covers slots [chunk * kFinChunkSlots, ...) of
// table `task`; its groups land in the task's output slice that starts at
// row slice0 (delta: unused, kept for the descriptor's layout).
struct FinBlock {
    int32_t task;
    int32_t chunk;
    int64_t delta;
    int64_t slice0;
};
constexpr int64_t kFinChunkSlots = 4096;
// Per-aggregate row counters: at least one word per aggregate.
size_t AggFinalizeBatchScratch(int64_t nblocks);
// `layout`: any of the tables (all share one slot layout).
void AggFinalizeBatch(const AggPlan& p, const OutputPlan& out, const GTableDev& layout, const GTableDev* tables,
                      const FinBlock* blocks, int64_t nblocks, AggOutputCol* cols, int ncols, int64_t out_rows,
                      void* scratch, int* err, cudaStream_t s);

// Raises a kernel's dynamic shared memory limit to `bytes` when it is
// below (runtime.cpp): the attribute only grows, and an unchanged kernel is
// not touched again (a change can wait on the kernel's launches in flight
// on every stream).
void EnsureSmemLimit(const void* fn, size_t bytes);

// Kernel timing hooks (runtime.cpp).
bool ProfileOn();
void ProfileBegin(cudaStream_t s, const char* name, int64_t units);
void ProfileEnd(cudaStream_t s);
void CountLaunch(int n = 1);

}  // namespace qdb
