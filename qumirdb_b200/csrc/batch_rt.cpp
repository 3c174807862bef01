// batch_rt.cpp — batched aggregation: many independent aggregate states of
// one program (the partitions of a partitioned GROUP BY, or the small
// aggregations of many queries of one template) updated by one persistent
// launch and finished by one batched finalize.
//
// The engine runs one aggregate task per partition and calls agg_dispatch
// (Update) on each task's HashTable (qdb/exec/aggregate_exec.cpp:104-117,
// qdb/kernel/compiler.h:207-230); agg_finish_rowset then turns each table
// into a row set (compiler.h:232-242, aggregate_exec.cpp:119-136).  Here a
// list of such (HashTable, batch) pairs becomes one work queue: fresh
// states get their tables carved from one device arena and initialised by
// one kernel, the rows of all states are cut into work items that the CTAs
// of one launch pull until the queue is empty, and the whole sequence
// (descriptor upload, counter reset, launch, counter read-back) is captured
// once as a CUDA graph and replayed while the batch keeps its structure.
//
// Block shape (threads per CTA, shared-tier slots) and work item size come
// from an autotuner that times candidates on a sample of the batch in
// scratch tables the first time a program meets a batch of a given size
// class; table capacities come from the groups-per-row ratio it has seen for
// states of the same size class (a state that outgrows its table defers its
// rows, and the host grows that table and replays them).
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

#include "common.cuh"
#include "fast.h"
#include "runtime.h"

namespace qdb {
namespace {

struct BatchConfig {
    int threads = 1024;
    int smem_slots = 2048;
    int64_t chunk_rows = int64_t(1) << 17;
};

// The low-cardinality kernel's block shape is fixed: 256 threads, a 64-slot
// shared tier.
BatchConfig DefaultConfig(bool low) {
    BatchConfig c;
    if (low) {
        c.threads = 256;
        c.smem_slots = 64;
    }
    return c;
}

constexpr int64_t kTuneMinRows = int64_t(16) << 20;   // rows in a batch worth a search

int SizeClass(int64_t rows) {
    int c = 0;
    while (c < 40 && (int64_t(1) << (c + 1)) <= rows) ++c;
    return c;
}

// Process-wide tuning state, keyed by the program's shape.
struct Tuner {
    std::mutex mu;
    std::map<std::tuple<std::string, int, int>, BatchConfig> best;   // (shape, rows class, states class)
    std::map<std::pair<std::string, int>, double> ratio;             // groups per row seen, by rows class
    int64_t tuned = 0;      // searches run
    int64_t trials = 0;     // candidate launches timed
    int64_t reused = 0;     // batches served from a stored choice
    int64_t resized = 0;    // launches run again with tables for one group per row
    int64_t states_low = 0;   // states updated by the low-cardinality batched kernel
    int64_t states_high = 0;  // ... and by the high-cardinality one
};

Tuner& Tune() {
    static Tuner t;
    return t;
}

bool TuningEnabled() {
    const char* e = std::getenv("QDB_AUTOTUNE");
    return !(e && e[0] == '0');
}

// QDB_BATCH_GRAPHS=0 runs every batched launch sequence eagerly.
bool GraphsEnabled() {
    static const bool on = [] {
        const char* e = std::getenv("QDB_BATCH_GRAPHS");
        return !(e && e[0] == '0');
    }();
    return on;
}

// Device buffers and pinned staging of one host thread's batched launches;
// they only grow, so a captured graph stays valid while its key holds.
struct BatchContext {
    HighTask* d_tasks = nullptr;
    HighItem* d_items = nullptr;
    unsigned long long* d_new = nullptr;
    BatchCounters* d_counters = nullptr;
    int64_t* d_deferred = nullptr;
    uint64_t* d_spill = nullptr;
    int64_t task_cap = 0, item_cap = 0, deferred_cap = 0, spill_cap = 0;
    HighTask* h_tasks = nullptr;
    HighItem* h_items = nullptr;
    unsigned long long* h_new = nullptr;
    BatchCounters* h_counters = nullptr;
    cudaStream_t s = nullptr;
    // Graph of the launch sequence and the key it was captured for.  A key is
    // captured the third time in a row it comes: batches of changing makeup
    // (a serving mix) run eagerly, since capturing and instantiating a graph
    // holds up the launches of other threads.
    cudaGraphExec_t exec = nullptr;
    std::string graph_key;
    std::string last_key;
    int repeats = 0;
    int64_t graph_launches = 0;
    int64_t graph_replays = 0;

    ~BatchContext() = default;   // one per host thread, kept until exit

    template <class T>
    static bool GrowDev(T*& p, int64_t& cap, int64_t need, cudaStream_t s) {
        if (need <= cap) return true;
        const int64_t n = std::max<int64_t>(need, cap * 2);
        if (p) DevFree(p, s);
        p = static_cast<T*>(DevAlloc(size_t(n) * sizeof(T), s));
        cap = p ? n : 0;
        return p != nullptr;
    }
    // Pinned staging comes from the library's page-locked output pool:
    // page-locking fresh memory while other streams run stalls them all.
    template <class T>
    static bool GrowPinned(T*& p, int64_t cap_before, int64_t n) {
        if (p && n <= cap_before) return true;
        HostOutFree(p);
        p = static_cast<T*>(HostOutAlloc(size_t(std::max<int64_t>(n, 1)) * sizeof(T)));
        return p != nullptr;
    }

    bool Reserve(int64_t ntasks, int64_t nitems, int64_t deferred, int64_t spill_words, cudaStream_t st) {
        s = st;
        const int64_t tcap = task_cap, icap = item_cap;
        if (!GrowDev(d_tasks, task_cap, ntasks, st)) return false;
        if (task_cap != tcap) {
            int64_t c = tcap;
            if (!GrowDev(d_new, c, task_cap, st)) return false;
            if (!GrowPinned(h_tasks, 0, task_cap) || !GrowPinned(h_new, 0, task_cap)) return false;
        }
        if (!GrowDev(d_items, item_cap, nitems, st)) return false;
        if (item_cap != icap && !GrowPinned(h_items, 0, item_cap)) return false;
        if (!d_counters) {
            d_counters = static_cast<BatchCounters*>(DevAlloc(sizeof(BatchCounters), st));
            if (!d_counters || !GrowPinned(h_counters, 0, 1)) return false;
        }
        if (!GrowDev(d_deferred, deferred_cap, deferred * 2, st)) return false;
        if (!GrowDev(d_spill, spill_cap, spill_words, st)) return false;
        return true;
    }

    HighBatch Desc(int64_t nitems) const {
        HighBatch b;
        b.tasks = d_tasks;
        b.items = d_items;
        b.nitems = nitems;
        b.new_groups = d_new;
        b.counters = d_counters;
        b.deferred = d_deferred;
        b.deferred_cap = deferred_cap / 2;
        b.spill = d_spill;
        b.spill_cap = 0;   // set by the caller from the record width
        return b;
    }
};

BatchContext& Ctx() {
    static thread_local BatchContext c;
    return c;
}

// Work items: each state's rows cut into chunks, states biggest first.
void BuildItems(const std::vector<int64_t>& rows, const std::vector<int>& order, int64_t chunk,
                std::vector<HighItem>& items) {
    items.clear();
    for (int t : order) {
        for (int64_t r0 = 0; r0 < rows[size_t(t)]; r0 += chunk) {
            HighItem it;
            it.task = t;
            it.nrows = int32_t(std::min<int64_t>(chunk, rows[size_t(t)] - r0));
            it.row0 = r0;
            items.push_back(it);
        }
    }
}

// Work items for a launch of `grid` CTAs: about `target` items in all, each
// state's share of them in proportion to its rows (largest remainders round
// up), a state's items of equal size on four-row boundaries, and the queue
// ordered biggest item first.  With a target that is a multiple of the grid,
// every CTA draws the same number of near-equal items and none waits out a
// partial last wave, which a fixed item size leaves whenever a state's rows
// are not a multiple of it.
void BuildItemsBalanced(const std::vector<int64_t>& rows, int64_t target, std::vector<HighItem>& items) {
    items.clear();
    const size_t m = rows.size();
    int64_t total = 0;
    for (int64_t r : rows) total += r;
    if (total == 0) return;
    std::vector<int64_t> n(m, 0);
    std::vector<std::pair<double, int>> frac;
    int64_t given = 0;
    for (size_t t = 0; t < m; ++t) {
        if (rows[t] == 0) continue;
        const double want = double(target) * double(rows[t]) / double(total);
        n[t] = std::max<int64_t>(1, int64_t(want));
        given += n[t];
        frac.push_back({want - double(int64_t(want)), int(t)});
    }
    std::stable_sort(frac.begin(), frac.end(), [](const std::pair<double, int>& a, const std::pair<double, int>& b) {
        return a.first > b.first;
    });
    for (size_t k = 0; k < frac.size() && given < target; ++k, ++given) n[size_t(frac[k].second)]++;
    for (size_t t = 0; t < m; ++t) {
        if (rows[t] == 0) continue;
        const int64_t q = ((rows[t] + n[t] - 1) / n[t] + 3) & ~int64_t(3);
        for (int64_t r0 = 0; r0 < rows[t]; r0 += q) {
            HighItem it;
            it.task = int32_t(t);
            it.nrows = int32_t(std::min<int64_t>(q, rows[t] - r0));
            it.row0 = r0;
            items.push_back(it);
        }
    }
    std::stable_sort(items.begin(), items.end(), [](const HighItem& a, const HighItem& b) { return a.nrows > b.nrows; });
}

int GridFor(const AggPlan& p, const FastPlan& f, const BatchConfig& c, int64_t nitems, bool low) {
    const int occ = std::max(1, AggBatchOccupancy(p, f, c.threads, c.smem_slots, low));
    return int(std::max<int64_t>(1, std::min<int64_t>(nitems, int64_t(DeviceSMs()) * occ)));
}

// Runs one batched update of `nitems` items whose tasks and items are
// already in the context's device buffers.
void LaunchUpdate(BatchContext& cx, const AggPlan& p, const FastPlan& f, const BatchConfig& c, int64_t ntasks,
                  int64_t nitems, int grid, cudaStream_t s, bool low) {
    HighBatch b = cx.Desc(nitems);
    b.spill_cap = cx.spill_cap / (2 + p.state_words);
    cudaMemsetAsync(cx.d_counters, 0, sizeof(BatchCounters), s);
    cudaMemsetAsync(cx.d_new, 0, size_t(ntasks) * 8, s);
    AggBatchUpdate(p, f, b, c.threads, c.smem_slots, grid, s, low);
}

// Chooses the block shape and item size for a batch: coordinate search
// over item size, shared-tier slots and threads per CTA (item size only for
// the low-cardinality kernel, whose block shape is fixed), each candidate
// timed (best of two) on a sample of the batch's states folded into
// scratch tables sized like theirs.
BatchConfig Search(const AggPlan& p, const FastPlan& f, const std::vector<HighTask>& tasks,
                   const std::vector<int64_t>& caps, cudaStream_t s, bool low) {
    BatchConfig best = DefaultConfig(low);
    // Sample: states spread over the size order, up to 64 states / 32M rows.
    std::vector<int> order(tasks.size());
    for (size_t i = 0; i < order.size(); ++i) order[i] = int(i);
    std::sort(order.begin(), order.end(), [&](int a, int b) { return tasks[size_t(a)].nrows > tasks[size_t(b)].nrows; });
    std::vector<int> pick;
    const size_t want = std::min<size_t>(64, order.size());
    int64_t total = 0;
    for (size_t k = 0; k < want; ++k) {
        const int t = order[k * order.size() / want];
        if (tasks[size_t(t)].nrows == 0) continue;
        if (total > 0 && total + tasks[size_t(t)].nrows > (int64_t(32) << 20)) continue;
        pick.push_back(t);
        total += tasks[size_t(t)].nrows;
    }
    if (pick.empty()) return best;
    const int sw = SlotWords(p, false);
    std::vector<HighTask> st(pick.size());
    std::vector<int64_t> off(pick.size());
    int64_t slots = 0;
    for (size_t k = 0; k < pick.size(); ++k) {
        off[k] = slots;
        slots += (caps[size_t(pick[k])] + 1 + 15) / 16 * 16;
    }
    uint64_t* arena = static_cast<uint64_t*>(DevAlloc(size_t(slots) * sw * 8, s));
    if (!arena) {
        cudaGetLastError();
        return best;
    }
    std::vector<int64_t> rows(pick.size());
    for (size_t k = 0; k < pick.size(); ++k) {
        st[k] = tasks[size_t(pick[k])];
        st[k].T.slots = arena + off[k] * sw;
        st[k].T.capacity = caps[size_t(pick[k])];
        rows[k] = st[k].nrows;
    }
    std::vector<int> so(pick.size());
    for (size_t k = 0; k < so.size(); ++k) so[k] = int(k);
    BatchContext& cx = Ctx();
    GTableDev all;
    all.slots = arena;
    all.capacity = slots - 1;
    all.slot_words = sw;
    all.key_off = 0;
    all.state_off = 1;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    auto trial = [&](const BatchConfig& c) -> float {
        std::vector<HighItem> items;
        BuildItems(rows, so, c.chunk_rows, items);
        const int64_t spill_words = int64_t(DeviceSMs()) * 4 * c.smem_slots * (2 + p.state_words);
        if (!cx.Reserve(int64_t(st.size()), int64_t(items.size()), std::max<int64_t>(total / 4, 1 << 20), spill_words, s))
            return 1e30f;
        cudaMemcpyAsync(cx.d_tasks, st.data(), st.size() * sizeof(HighTask), cudaMemcpyHostToDevice, s);
        cudaMemcpyAsync(cx.d_items, items.data(), items.size() * sizeof(HighItem), cudaMemcpyHostToDevice, s);
        float bestms = 1e30f;
        for (int rep = 0; rep < 2; ++rep) {
            AggBatchInitTables(p, all, cx.d_tasks, int(st.size()), s);
            cudaEventRecord(e0, s);
            LaunchUpdate(cx, p, f, c, int64_t(st.size()), int64_t(items.size()),
                         GridFor(p, f, c, int64_t(items.size()), low), s, low);
            cudaEventRecord(e1, s);
            cudaEventSynchronize(e1);
            float ms = 0.f;
            cudaEventElapsedTime(&ms, e0, e1);
            bestms = std::min(bestms, ms);
            Tune().trials++;
        }
        return bestms;
    };
    float cur = trial(best);
    for (int64_t chunk : {int64_t(1) << 15, int64_t(1) << 19}) {
        BatchConfig c = best;
        c.chunk_rows = chunk;
        const float ms = trial(c);
        if (ms < cur) {
            cur = ms;
            best = c;
        }
    }
    for (int S : {1024, 4096}) {
        if (low) break;
        BatchConfig c = best;
        c.smem_slots = S;
        if (AggBatchOccupancy(p, f, c.threads, S, low) < 1) continue;
        const float ms = trial(c);
        if (ms < cur) {
            cur = ms;
            best = c;
        }
    }
    if (!low) {
        BatchConfig c = best;
        c.threads = 512;
        if (AggBatchOccupancy(p, f, c.threads, c.smem_slots, low) >= 1) {
            const float ms = trial(c);
            if (ms < cur) best = c;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    DevFree(arena, s);
    cudaStreamSynchronize(s);
    return best;
}

// FNV-1a over a plan's bytes.
uint64_t PlanBytesHash(const void* p, size_t n, uint64_t h = 1469598103934665603ull) {
    // Eight bytes a step (plans run to kilobytes and are hashed per dispatch);
    // each step's product is folded back so every input bit reaches all 64.
    const auto* b = static_cast<const unsigned char*>(p);
    size_t i = 0;
    for (; i + 8 <= n; i += 8) {
        uint64_t w;
        std::memcpy(&w, b + i, 8);
        h = (h ^ w) * 0x9e3779b97f4a7c15ull;
        h ^= h >> 29;
    }
    for (; i < n; ++i) h = (h ^ b[i]) * 1099511628211ull;
    return h;
}

// Identity of a recorded launch sequence.  A captured graph holds the
// launch's AggLaunch by value: the resolved plan (filter literals, affine
// constants, IN-lists) and the typed shape's constants.  Two programs of one
// shape that differ only in a literal must not share a graph, so the key
// covers both plans' bytes besides the batch structure and the context's
// buffers.
std::string ConfigKey(const std::string& shape, const AggPlan& plan, const FastPlan& fast, int64_t ntasks,
                      int64_t nitems, const BatchConfig& c, const BatchContext& cx) {
    // The batched kernel reads every row set's columns from its task (uploaded
    // on each replay); the plan's own column and selection pointers (those
    // of the first row set) are not part of the identity.
    AggPlan bare = plan;
    for (int c = 0; c < kMaxCols; ++c) {
        bare.cols[c].data = nullptr;
        bare.cols[c].mask = nullptr;
        bare.cols[c].mask_off = 0;
        bare.cols[c].bit_off = 0;
    }
    bare.selection = nullptr;
    bare.has_selection = 0;
    const uint64_t h = PlanBytesHash(&fast, sizeof(fast), PlanBytesHash(&bare, sizeof(bare)));
    char buf[320];
    std::snprintf(buf, sizeof(buf), "|%016llx|%lld|%lld|%d|%d|%lld|%p|%p|%p|%p|%p", (unsigned long long)h,
                  (long long)ntasks, (long long)nitems, c.threads, c.smem_slots, (long long)c.chunk_rows,
                  (void*)cx.d_tasks, (void*)cx.d_items, (void*)cx.d_new, (void*)cx.d_deferred, (void*)cx.d_spill);
    return shape + buf;
}

}  // namespace

using RatioTable = std::array<double, 64>;

// The groups-per-row ratios seen for a shape, by size class (0: none yet).
RatioTable RatiosOf(const std::string& shape) {
    RatioTable r{};
    Tuner& t = Tune();
    std::lock_guard<std::mutex> lk(t.mu);
    for (auto it = t.ratio.lower_bound({shape, 0}); it != t.ratio.end() && it->first.first == shape; ++it) {
        if (it->first.second >= 0 && it->first.second < int(r.size())) r[size_t(it->first.second)] = it->second;
    }
    return r;
}

// Estimated groups of a state of `rows` rows: the largest groups-per-row
// ratio seen for its size class (half the rows before any was seen), with
// a quarter of headroom, never above the rows or the program's hint.
int64_t EstimateGroups(const RatioTable& ratios, int64_t rows, int64_t expected) {
    const double seen = ratios[size_t(SizeClass(rows))];
    const double r = seen > 0 ? std::min(1.0, seen * 1.25) : 0.5;
    int64_t est = int64_t(std::ceil(r * double(rows))) + 64;
    est = std::min(est, std::max<int64_t>(rows, 1));
    if (expected > 0) est = std::min(est, expected);
    return est;
}

// The typed shape's columns of one row set (the batched kernel's task),
// resolved against the program's first resolved plan: false when a column
// has a validity bitmap (outside the typed shapes) or no data.
bool ResolveShapeColumns(const AggPlan& P0, const FastPlan& F, const ColumnMap& cm, const qdb_column_type* types,
                         const qdb_rowset* rs, Staging& st, HighTask& t) {
    std::memset(&t, 0, sizeof(t));
    const int64_t n = rs->RowCount;
    for (int c = 0; c < F.ncols && c < kFastCols; ++c) {
        const int slot = F.col_slot[c];
        const int input = cm.input_of[slot];
        if (input >= rs->ColumnCount || types[input].type == QDB_TYPE_BOOL) return false;
        const qdb_column& col = rs->Columns[input];
        if (col.Mask) return false;
        t.cols[c] = static_cast<const char*>(st.Device(col.Data, size_t(n) * P0.cols[slot].width));
        if (n > 0 && !t.cols[c]) return false;
    }
    t.sel = rs->Selection ? static_cast<const uint8_t*>(st.Device(rs->Selection, size_t(n))) : nullptr;
    if (n > 0 && rs->Selection && !t.sel) return false;
    t.nrows = n;
    return true;
}

}  // namespace qdb

using namespace qdb;

namespace {

// Per-aggregate output slices of the combined finalize buffers; the buffers
// go when the last slice is destroyed.
struct BatchOutputs {
    std::vector<void*> dev;
    std::vector<void*> host;
    cudaStream_t s = nullptr;
    ~BatchOutputs() {
        for (void* p : host) HostOutFree(p);
        for (void* p : dev) DevFree(p, s);
    }
};

struct SliceRowset {
    std::shared_ptr<BatchOutputs> owner;
    std::vector<qdb_column> cols;
};

void DestroySlice(qdb_rowset* rs) {
    if (!rs || !rs->Private) return;
    delete static_cast<SliceRowset*>(rs->Private);
    rs->Private = nullptr;
    rs->Columns = nullptr;
}

}  // namespace

namespace {
int64_t DispatchBatch(const qdb_gpu_program* prog, void* const* hts, qdb_rowset* const* batches, int64_t n,
                      bool every_row_a_group);

// Pinned staging of one host thread's batched finalize (its block list and
// table descriptors up, its error word down); it only grows, and each use
// ends with a stream synchronise before the next can write it.
char* FinishStaging(size_t bytes) {
    thread_local char* p = nullptr;
    thread_local size_t cap = 0;
    if (bytes > cap) {
        HostOutFree(p);
        cap = std::max(bytes, cap * 2);
        p = static_cast<char*>(HostOutAlloc(cap));
        if (!p) cap = 0;
    }
    return p;
}
}

extern "C" {

int64_t qdb_gpu_agg_dispatch_batch(const qdb_gpu_program* prog, void* const* hts, qdb_rowset* const* batches,
                                   int64_t n) {
    t_error.clear();
    return DispatchBatch(prog, hts, batches, n, false);
}

}  // extern "C"

namespace {

// The batched update.  Fresh tables are sized from the groups-per-row ratio
// seen so far for the program's shape; with every_row_a_group they are sized
// for one group per row instead (no insert can then run out of room).
int64_t DispatchBatch(const qdb_gpu_program* prog, void* const* hts, qdb_rowset* const* batches, int64_t n,
                      bool every_row_a_group) {
    if (!prog || prog->kind != PK_AGG || (n > 0 && (!hts || !batches))) {
        SetErr("agg_dispatch_batch: not an aggregate program, or no states");
        return -1;
    }
    if (n == 0) return 0;
    const AggLowering& lw = prog->agg;
    cudaStream_t s = CurStream();
    Staging stg(s);
    std::vector<int64_t> rows(static_cast<size_t>(n));
    std::vector<char> typed(static_cast<size_t>(n), 0);
    std::vector<HighTask> resolved(static_cast<size_t>(n));
    // The first row set resolves the whole plan and finds the batched
    // kernel; the others only resolve the typed shape's columns (a plan copy
    // per row set would cost more host time than the launch saves).
    FastPlan fast{};
    bool have_fast = false;
    AggPlan P0 = lw.plan;
    // A few groups per aggregate (the planner's hint, or none at all): the
    // low-cardinality kernel, whose typed columns must start on a boundary of
    // four values (and a selection on one of four bytes).
    const bool low = lw.plan.nkeyparts == 0 || (prog->expected_groups > 0 && prog->expected_groups <= 64);
    auto typed_ok = [&](const HighTask& t) {
        if (!low) return true;
        for (int c = 0; c < fast.ncols && c < kFastCols; ++c) {
            const int w = int(P0.cols[fast.col_slot[c]].width);
            if (reinterpret_cast<uintptr_t>(t.cols[c]) % uintptr_t(std::min(16, 4 * w))) return false;
        }
        return (reinterpret_cast<uintptr_t>(t.sel) & 3) == 0;
    };
    for (int64_t i = 0; i < n; ++i) {
        if (!hts[i] || !batches[i]) {
            SetErr("agg_dispatch_batch: state or batch %lld is NULL", (long long)i);
            return -1;
        }
        rows[size_t(i)] = batches[i]->RowCount;
        if (have_fast) {
            typed[size_t(i)] = ResolveShapeColumns(P0, fast, lw.cols, prog->columns.data(), batches[i], stg,
                                                   resolved[size_t(i)]) && typed_ok(resolved[size_t(i)]) ? 1 : 0;
            continue;
        }
        AggPlan pi = lw.plan;
        if (!ResolveColumns(pi, lw.cols, prog->columns.data(), batches[i], stg)) return -1;
        FastPlan fi{};
        if (MatchFast(pi, fi) && AggBatchSupported(pi, fi, low)) {
            fast = fi;
            have_fast = true;
            P0 = pi;
            typed[size_t(i)] = ResolveShapeColumns(P0, fast, lw.cols, prog->columns.data(), batches[i], stg,
                                                   resolved[size_t(i)]) && typed_ok(resolved[size_t(i)]) ? 1 : 0;
        }
    }
    // States outside the batched kernel (no compiled shape, nullable columns)
    // take the one-state path.
    std::vector<int> members;
    for (int64_t i = 0; i < n; ++i) {
        if (typed[size_t(i)]) {
            members.push_back(int(i));
            continue;
        }
        AggTableState* st = StateOf(hts[i]);
        if (!st) {
            st = AggStateCreate(lw.plan, rows[size_t(i)], prog->expected_groups, s);
            *static_cast<AggTableState**>(hts[i]) = st;
            if (!st) return -1;
        }
        AggPlan pi = lw.plan;
        if (!ResolveColumns(pi, lw.cols, prog->columns.data(), batches[i], stg)) return -1;
        if (!AggRun(st, pi, rows[size_t(i)], nullptr, nullptr)) return -1;
        MirrorHeader(hts[i], st, lw.plan);
    }
    if (members.empty()) return n;
    const std::string shape = AggBatchShapeKey(P0, fast, low);
    {
        Tuner& tn = Tune();
        std::lock_guard<std::mutex> lk(tn.mu);
        (low ? tn.states_low : tn.states_high) += int64_t(members.size());
    }
    const int sw = SlotWords(lw.plan, false);
    const int64_t m = int64_t(members.size());

    // Fresh states: tables (and device counters) carved from one arena.
    std::vector<int> fresh;
    std::vector<int64_t> caps(static_cast<size_t>(m));
    const RatioTable ratios = RatiosOf(shape);
    for (int64_t k = 0; k < m; ++k) {
        const int i = members[size_t(k)];
        AggTableState* st = StateOf(hts[i]);
        if (st) {
            caps[size_t(k)] = st->t.capacity;
            continue;
        }
        fresh.push_back(int(k));
        const int64_t est = every_row_a_group ? std::max<int64_t>(rows[size_t(i)], 1)
                                              : EstimateGroups(ratios, rows[size_t(i)], prog->expected_groups);
        caps[size_t(k)] = std::max<int64_t>(1024, NextPow2(est + est / 4));
    }
    std::vector<HighTask> tasks(static_cast<size_t>(m));
    AggArena* arena = nullptr;
    GTableDev all;
    if (!fresh.empty()) {
        std::vector<int64_t> off(fresh.size());
        int64_t slots = 0;
        for (size_t j = 0; j < fresh.size(); ++j) {
            off[j] = slots;
            slots += (caps[size_t(fresh[j])] + 1 + 15) / 16 * 16;
        }
        const size_t table_bytes = size_t(slots) * sw * 8;
        const size_t counter_bytes = fresh.size() * sizeof(AggCounters);
        arena = new AggArena();
        arena->s = s;
        arena->p = DevAlloc(table_bytes + counter_bytes, s);
        if (!arena->p) {
            delete arena;
            SetErr("agg_dispatch_batch: device allocation of %zu bytes failed", table_bytes + counter_bytes);
            return -1;
        }
        auto* base = static_cast<uint64_t*>(arena->p);
        auto* counters = reinterpret_cast<AggCounters*>(static_cast<char*>(arena->p) + table_bytes);
        cudaMemsetAsync(counters, 0, counter_bytes, s);
        all.slots = base;
        all.capacity = slots - 1;
        all.slot_words = sw;
        all.key_off = 0;
        all.state_off = 1;
        for (size_t j = 0; j < fresh.size(); ++j) {
            const int k = fresh[j];
            const int i = members[size_t(k)];
            auto* st = new AggTableState();
            st->s = s;
            st->expected = prog->expected_groups;
            st->t.slots = base + off[j] * sw;
            st->t.capacity = caps[size_t(k)];
            st->t.slot_words = sw;
            st->t.key_off = 0;
            st->t.state_off = 1;
            st->t.wide = 0;
            st->table_in_arena = true;
            st->dc = counters + j;
            st->dc_in_arena = true;
            st->hc = PinnedCountersGet();
            st->arena = arena;
            arena->refs++;
            st->groups = lw.plan.nkeyparts == 0 ? 1 : 0;
            *static_cast<AggTableState**>(hts[i]) = st;
            if (!st->hc) {
                SetErr("pinned allocation failed");
                return -1;
            }
        }
    }
    for (int64_t k = 0; k < m; ++k) {
        const int i = members[size_t(k)];
        tasks[size_t(k)] = resolved[size_t(i)];
        tasks[size_t(k)].T = StateOf(hts[i])->t;
    }

    // Block shape and item size.
    int64_t total_rows = 0;
    for (int64_t r : rows) total_rows += r;
    const int rows_class = SizeClass(total_rows / std::max<int64_t>(m, 1));
    const int states_class = SizeClass(m);
    // Batches too small to pay for a search run the defaults.
    const bool worth_tuning = total_rows >= kTuneMinRows;
    // A stored choice for this shape and size class; else the choice of the
    // nearest size class of the shape (a search costs tens of launches, so
    // a shape is searched once and its later batches, of whatever mix, reuse
    // the nearest choice); a shape never searched is searched now.
    BatchConfig cfg = DefaultConfig(low);
    bool found = false;
    {
        Tuner& tn = Tune();
        std::lock_guard<std::mutex> lk(tn.mu);
        auto it = tn.best.find({shape, rows_class, states_class});
        if (it == tn.best.end()) {
            int best_d = 1 << 30;
            for (auto j = tn.best.begin(); j != tn.best.end(); ++j) {
                if (std::get<0>(j->first) != shape) continue;
                const int d = std::abs(std::get<1>(j->first) - rows_class) * 4 + std::abs(std::get<2>(j->first) - states_class);
                if (d < best_d) {
                    best_d = d;
                    it = j;
                }
            }
        }
        if (it != tn.best.end()) {
            cfg = it->second;
            found = true;
            tn.reused++;
        }
    }
    BatchContext& cx = Ctx();
    if (!found && TuningEnabled() && worth_tuning) {
        // Fresh tables must be initialised before the search reuses the
        // context's device buffers; it runs on scratch tables of its own.
        cfg = Search(P0, fast, tasks, caps, s, low);
        Tuner& tn = Tune();
        std::lock_guard<std::mutex> lk(tn.mu);
        tn.best[{shape, rows_class, states_class}] = cfg;
        tn.tuned++;
    }

    std::vector<int64_t> task_rows(static_cast<size_t>(m));
    for (int64_t k = 0; k < m; ++k) task_rows[size_t(k)] = tasks[size_t(k)].nrows;
    std::vector<HighItem> items;
    if (!found && low) {
        // Untuned low-cardinality batches: two items per resident CTA while
        // they stay above 8K rows (an item's claim, clear and merge cost a
        // few microseconds), up to about 128K rows each for long batches;
        // tiny batches take fewer CTAs.
        const int64_t grid = int64_t(DeviceSMs()) *
                             std::max(1, AggBatchOccupancy(P0, fast, cfg.threads, cfg.smem_slots, true));
        const int64_t min_rows = int64_t(1) << 13;
        int64_t target = total_rows / min_rows;
        if (target >= 2 * grid) {
            const int64_t k = std::max<int64_t>(2, (total_rows / grid + (int64_t(1) << 17) - 1) >> 17);
            target = k * grid;
        }
        BuildItemsBalanced(task_rows, std::max<int64_t>(target, 1), items);
    } else {
        std::vector<int> order(static_cast<size_t>(m));
        for (int64_t k = 0; k < m; ++k) order[size_t(k)] = int(k);
        std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return task_rows[size_t(a)] > task_rows[size_t(b)]; });
        BuildItems(task_rows, order, cfg.chunk_rows, items);
    }
    const int64_t nitems = int64_t(items.size());
    const int64_t spill_words = int64_t(DeviceSMs()) * 4 * cfg.smem_slots * (2 + lw.plan.state_words);
    const int64_t defer_cap = std::max<int64_t>(total_rows / 4, int64_t(1) << 20);
    if (!cx.Reserve(m, std::max<int64_t>(nitems, 1), defer_cap, spill_words, s)) {
        SetErr("agg_dispatch_batch: device allocation failed");
        return -1;
    }
    std::memcpy(cx.h_tasks, tasks.data(), size_t(m) * sizeof(HighTask));
    if (nitems) std::memcpy(cx.h_items, items.data(), size_t(nitems) * sizeof(HighItem));
    if (!fresh.empty() && fresh.size() == size_t(m)) {
        // Every state fresh: the tables are initialised and their flag slots
        // marked from the tasks uploaded from pinned staging, in stream order
        // before the update (no wait on the host).
        cudaMemcpyAsync(cx.d_tasks, cx.h_tasks, size_t(m) * sizeof(HighTask), cudaMemcpyHostToDevice, s);
        AggBatchInitTables(lw.plan, all, cx.d_tasks, int(m), s);
    } else if (!fresh.empty()) {
        // The fresh tables' flag slots are marked through the uploaded tasks
        // of the fresh states only.
        std::vector<HighTask> ft(fresh.size());
        for (size_t j = 0; j < fresh.size(); ++j) ft[j] = tasks[size_t(fresh[j])];
        HighTask* d_ft = static_cast<HighTask*>(DevAlloc(ft.size() * sizeof(HighTask), s));
        if (!d_ft) return -1;
        cudaMemcpyAsync(d_ft, ft.data(), ft.size() * sizeof(HighTask), cudaMemcpyHostToDevice, s);
        AggBatchInitTables(lw.plan, all, d_ft, int(ft.size()), s);
        DevFree(d_ft, s);
        cudaStreamSynchronize(s);   // `ft` is pageable host memory
    }

    // The launch sequence: as a replayed graph while the batch's structure
    // holds, else eagerly (and always eagerly while kernels are timed).
    const int grid = GridFor(P0, fast, cfg, nitems, low);
    auto record = [&](cudaStream_t st) {
        cudaMemcpyAsync(cx.d_tasks, cx.h_tasks, size_t(m) * sizeof(HighTask), cudaMemcpyHostToDevice, st);
        if (nitems) cudaMemcpyAsync(cx.d_items, cx.h_items, size_t(nitems) * sizeof(HighItem), cudaMemcpyHostToDevice, st);
        LaunchUpdate(cx, P0, fast, cfg, m, nitems, grid, st, low);
        cudaMemcpyAsync(cx.h_new, cx.d_new, size_t(m) * 8, cudaMemcpyDeviceToHost, st);
        cudaMemcpyAsync(cx.h_counters, cx.d_counters, sizeof(BatchCounters), cudaMemcpyDeviceToHost, st);
    };
    const std::string gkey = ConfigKey(shape, P0, fast, m, nitems, cfg, cx);
    bool ran = false;
    cx.repeats = gkey == cx.last_key ? cx.repeats + 1 : 1;
    cx.last_key = gkey;
    const bool repeat = cx.repeats >= 3;
    if (GraphsEnabled() && !ProfileOn() && s != nullptr && (repeat || (cx.exec && cx.graph_key == gkey))) {
        if (cx.exec && cx.graph_key != gkey) {
            cudaGraphExecDestroy(cx.exec);
            cx.exec = nullptr;
        }
        if (!cx.exec) {
            cudaGraph_t g = nullptr;
            const int64_t before = qdb_gpu_launch_count(0);
            if (cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal) == cudaSuccess) {
                record(s);
                if (cudaStreamEndCapture(s, &g) == cudaSuccess && g) {
                    if (cudaGraphInstantiate(&cx.exec, g, 0) != cudaSuccess) cx.exec = nullptr;
                    cudaGraphDestroy(g);
                }
            }
            cudaGetLastError();
            cx.graph_launches = qdb_gpu_launch_count(0) - before;
            if (cx.exec) {
                cx.graph_key = gkey;
                // The captured launches ran nothing yet: they count per replay.
                CountLaunch(int(-cx.graph_launches));
            }
        }
        if (cx.exec && cudaGraphLaunch(cx.exec, s) == cudaSuccess) {
            CountLaunch(int(cx.graph_launches));
            cx.graph_replays++;
            ran = true;
        } else {
            cudaGetLastError();
        }
    }
    if (!ran) record(s);
    if (!CudaOk(cudaStreamSynchronize(s), "batched aggregate update")) return -1;
    const BatchCounters bc = *cx.h_counters;
    if (bc.error) {
        // More rows were turned away than the replay buffers hold: the tables
        // were sized from a ratio that these row sets do not follow.  When
        // every state of the launch was created by this call, its tables are
        // dropped and the launch runs again with tables sized for one group
        // per row.
        const bool overflow = bc.error == qdb::DE_SPILL_FULL || bc.error == qdb::DE_DEFER_FULL;
        if (overflow && !every_row_a_group && fresh.size() == size_t(m)) {
            std::vector<void*> mh;
            std::vector<qdb_rowset*> mb;
            for (int64_t k = 0; k < m; ++k) {
                const int i = members[size_t(k)];
                AggStateDestroy(StateOf(hts[i]));
                std::memset(hts[i], 0, QDB_HASH_TABLE_SIZE);
                mh.push_back(hts[i]);
                mb.push_back(batches[i]);
            }
            {
                std::lock_guard<std::mutex> lk(Tune().mu);
                Tune().resized++;
            }
            return DispatchBatch(prog, mh.data(), mb.data(), m, true) < 0 ? -1 : n;
        }
        SetErr("batched aggregate kernel reported device error %d", bc.error);
        return -1;
    }
    for (int64_t k = 0; k < m; ++k) StateOf(hts[members[size_t(k)]])->groups += int64_t(cx.h_new[k]);

    // Rows a full table turned away, and shared-tier entries it could not
    // take: per state, grow its table and replay them.
    if (bc.ndeferred || bc.nspill) {
        std::vector<int64_t> pairs(size_t(bc.ndeferred) * 2);
        const int rw = 2 + lw.plan.state_words;
        std::vector<uint64_t> recs(size_t(bc.nspill) * size_t(rw));
        if (bc.ndeferred)
            cudaMemcpyAsync(pairs.data(), cx.d_deferred, pairs.size() * 8, cudaMemcpyDeviceToHost, s);
        if (bc.nspill) cudaMemcpyAsync(recs.data(), cx.d_spill, recs.size() * 8, cudaMemcpyDeviceToHost, s);
        if (!CudaOk(cudaStreamSynchronize(s), "batched aggregate replay read-back")) return -1;
        std::vector<std::vector<int64_t>> dpairs(static_cast<size_t>(m));
        std::vector<std::vector<uint64_t>> srecs(static_cast<size_t>(m));
        for (uint64_t j = 0; j < bc.ndeferred; ++j) {
            const int64_t t = pairs[2 * j + 1];
            dpairs[size_t(t)].push_back(pairs[2 * j]);
            dpairs[size_t(t)].push_back(0);
        }
        for (uint64_t j = 0; j < bc.nspill; ++j) {
            const uint64_t* r = &recs[j * size_t(rw)];
            const int64_t t = int64_t(r[rw - 1]);
            srecs[size_t(t)].insert(srecs[size_t(t)].end(), r, r + rw - 1);
        }
        for (int64_t k = 0; k < m; ++k) {
            if (dpairs[size_t(k)].empty() && srecs[size_t(k)].empty()) continue;
            const int i = members[size_t(k)];
            AggTableState* st = StateOf(hts[i]);
            AggPlan pi = lw.plan;
            if (!ResolveColumns(pi, lw.cols, prog->columns.data(), batches[i], stg)) return -1;
            const int64_t nd = int64_t(dpairs[size_t(k)].size() / 2);
            const int64_t ns = int64_t(srecs[size_t(k)].size()) / (1 + lw.plan.state_words);
            if (!EnsureBuffers(st, pi, std::max(rows[size_t(i)], nd))) return -1;
            if (st->spill_cap < ns) {
                DevFree(st->spill, s);
                st->spill = static_cast<uint64_t*>(DevAlloc(size_t(ns) * (1 + lw.plan.state_words) * 8, s));
                st->spill_cap = st->spill ? ns : 0;
            }
            if (st->deferred_cap < nd || st->spill_cap < ns) {
                SetErr("agg_dispatch_batch: replay buffers too small");
                return -1;
            }
            if (nd) cudaMemcpyAsync(st->deferred[0], dpairs[size_t(k)].data(), size_t(nd) * 16, cudaMemcpyHostToDevice, s);
            if (ns)
                cudaMemcpyAsync(st->spill, srecs[size_t(k)].data(), srecs[size_t(k)].size() * 8, cudaMemcpyHostToDevice, s);
            cudaStreamSynchronize(s);
            FastPlan fi{};
            const bool fi_ok = MatchFast(pi, fi);
            AggUpdateArgs a;
            a.plan = &pi;
            a.nrows = rows[size_t(i)];
            a.table = st->t;
            a.counters = st->dc;
            a.deferred = st->deferred[0];
            a.deferred_cap = st->deferred_cap;
            a.spill = st->spill;
            a.spill_cap = st->spill_cap;
            a.smem_slots = st->smem_slots;
            a.fast = fi_ok ? &fi : nullptr;
            if (!AggReplay(st, pi, a, nd, ns)) return -1;
        }
    }
    // Tables over half full grow now, as after a one-state update; the ratio
    // of groups to rows is remembered per size class for later batches.
    {
        RatioTable seen{};
        for (int64_t k = 0; k < m; ++k) {
            const int i = members[size_t(k)];
            AggTableState* st = StateOf(hts[i]);
            // Batch tables run fuller than one-state tables (sized from the
            // learned ratio): grown past 85% load.
            if (st->groups * 20 > st->t.capacity * 17 && !Grow(st, lw.plan, st->groups)) return -1;
            MirrorHeader(hts[i], st, lw.plan);
            if (rows[size_t(i)] >= 1024) {
                double& v = seen[size_t(SizeClass(rows[size_t(i)]))];
                v = std::max(v, double(st->groups) / double(rows[size_t(i)]));
            }
        }
        Tuner& tn = Tune();
        std::lock_guard<std::mutex> lk(tn.mu);
        for (size_t c = 0; c < seen.size(); ++c) {
            if (seen[c] <= 0) continue;
            double& v = tn.ratio[{shape, int(c)}];
            v = std::max(v, seen[c]);
        }
    }
    return n;
}

}  // namespace

extern "C" {

int64_t qdb_gpu_agg_finish_batch(const qdb_gpu_program* prog, void* const* hts, int64_t n, qdb_rowset* outs) {
    t_error.clear();
    if (!prog || (prog->kind != PK_AGG && prog->kind != PK_JOIN_AGG) || (n > 0 && (!hts || !outs))) {
        SetErr("agg_finish_batch: not an aggregate program, or no states");
        return -1;
    }
    if (n == 0) return 0;
    const AggLowering& lw = prog->agg;
    cudaStream_t s = CurStream();
    std::vector<AggTableState*> sts(static_cast<size_t>(n));
    for (int64_t i = 0; i < n; ++i) {
        sts[size_t(i)] = StateOf(hts[i]);
        if (!sts[size_t(i)]) {
            SetErr("agg_finish_batch: state %lld was never initialised", (long long)i);
            return -1;
        }
    }
    // Aggregate i's groups go to rows [pad_i, pad_i + groups_i) of combined
    // output columns; slices start on 64-row boundaries so each slice's
    // validity words are its own.
    std::vector<int64_t> pad(static_cast<size_t>(n));
    int64_t out_rows = 0, total = 0;
    std::vector<FinBlock> blocks;
    std::vector<GTableDev> tables(static_cast<size_t>(n));
    for (int64_t i = 0; i < n; ++i) {
        const AggTableState* st = sts[size_t(i)];
        pad[size_t(i)] = out_rows;
        tables[size_t(i)] = st->t;
        const int64_t nb = (st->t.capacity + 1 + kFinChunkSlots - 1) / kFinChunkSlots;
        for (int64_t c = 0; c < nb; ++c) {
            FinBlock fb;
            fb.task = int32_t(i);
            fb.chunk = int32_t(c);
            fb.delta = out_rows - total;
            fb.slice0 = out_rows;
            blocks.push_back(fb);
        }
        total += st->groups;
        out_rows += (st->groups + 63) / 64 * 64;
    }
    std::vector<int> types;
    for (int k = 0; k < lw.out.n; ++k) types.push_back(lw.out.out_type[k]);
    std::vector<AggOutputCol> cols;
    OutBlock blk;
    if (!AllocOutputCols(types, std::max<int64_t>(out_rows, 64), true, cols, s, &blk)) {
        SetErr("output allocation failed");
        return -1;
    }
    auto owner = std::make_shared<BatchOutputs>();
    owner->s = s;
    owner->dev.push_back(blk.p);
    const int64_t nblocks = int64_t(blocks.size());
    const size_t scratch_bytes = AggFinalizeBatchScratch(nblocks);
    const size_t up_bytes = blocks.size() * sizeof(FinBlock) + tables.size() * sizeof(GTableDev);
    char* h_up = FinishStaging(up_bytes + 16);
    if (!h_up) {
        SetErr("pinned allocation failed");
        return -1;
    }
    std::memcpy(h_up, blocks.data(), blocks.size() * sizeof(FinBlock));
    std::memcpy(h_up + blocks.size() * sizeof(FinBlock), tables.data(), tables.size() * sizeof(GTableDev));
    char* dev = static_cast<char*>(DevAlloc(scratch_bytes + blocks.size() * sizeof(FinBlock) +
                                                tables.size() * sizeof(GTableDev) + 16, s));
    if (!dev) return -1;
    auto* d_blocks = reinterpret_cast<FinBlock*>(dev + scratch_bytes);
    auto* d_tables = reinterpret_cast<GTableDev*>(dev + scratch_bytes + blocks.size() * sizeof(FinBlock));
    int* d_err = reinterpret_cast<int*>(dev + scratch_bytes + blocks.size() * sizeof(FinBlock) +
                                        tables.size() * sizeof(GTableDev));
    // Blocks and tables sit side by side on both ends: one upload.
    cudaMemcpyAsync(d_blocks, h_up, up_bytes, cudaMemcpyHostToDevice, s);
    cudaMemsetAsync(d_err, 0, sizeof(int), s);
    AggFinalizeBatch(lw.plan, lw.out, tables[0], d_tables, d_blocks, nblocks, cols.data(), int(cols.size()),
                     out_rows, dev, d_err, s);
    int* h_err = reinterpret_cast<int*>(h_up + ((up_bytes + 7) & ~size_t(7)));
    cudaMemcpyAsync(h_err, d_err, sizeof(int), cudaMemcpyDeviceToHost, s);
    if (!CudaOk(cudaStreamSynchronize(s), "batched finalize")) return -1;
    const int herr = *h_err;
    DevFree(dev, s);
    if (herr) {
        SetErr("batched finalize reported device error %d", herr);
        return -1;
    }
    const bool on_device = (prog->flags & QDB_OUT_DEVICE) != 0;
    std::vector<char*> base(cols.size());
    std::vector<uint32_t*> vbase(cols.size());
    std::vector<int32_t*> obase(cols.size());
    for (size_t k = 0; k < cols.size(); ++k) {
        base[k] = cols[k].data;
        vbase[k] = cols[k].valid;
        obase[k] = cols[k].offsets;
    }
    if (!on_device) {
        // One copy of the whole block to the host; the slices point there, at
        // the same offsets.
        auto host = std::make_shared<BatchOutputs>();
        char* h = static_cast<char*>(HostOutAlloc(std::max<size_t>(blk.bytes, 16)));
        if (!h) {
            SetErr("pinned allocation failed");
            return -1;
        }
        host->host.push_back(h);
        cudaMemcpyAsync(h, blk.p, blk.bytes, cudaMemcpyDeviceToHost, s);
        const char* b = static_cast<const char*>(blk.p);
        for (size_t k = 0; k < cols.size(); ++k) {
            base[k] = h + (cols[k].data - b);
            if (cols[k].valid) vbase[k] = reinterpret_cast<uint32_t*>(h + (reinterpret_cast<const char*>(cols[k].valid) - b));
            if (cols[k].offsets) obase[k] = reinterpret_cast<int32_t*>(h + (reinterpret_cast<const char*>(cols[k].offsets) - b));
        }
        if (!CudaOk(cudaStreamSynchronize(s), "batched finalize read-back")) return -1;
        owner = host;   // the device block goes back to the pool now
    }
    for (int64_t i = 0; i < n; ++i) {
        auto* sl = new SliceRowset();
        sl->owner = owner;
        sl->cols.resize(cols.size());
        for (size_t k = 0; k < cols.size(); ++k) {
            qdb_column& c = sl->cols[k];
            std::memset(&c, 0, sizeof(c));
            const size_t w = size_t(StorageWidth(types[k]));
            c.Data = base[k] + size_t(pad[size_t(i)]) * w;
            if (obase[k]) {
                c.Offsets = obase[k] + pad[size_t(i)];   // counted from the slice start
                c.OffsetWidth = 4;
            }
            if (vbase[k]) c.Mask = reinterpret_cast<const uint8_t*>(vbase[k] + pad[size_t(i)] / 32);
        }
        qdb_rowset& o = outs[i];
        std::memset(&o, 0, sizeof(o));
        o.Columns = sl->cols.data();
        o.ColumnCount = int64_t(cols.size());
        o.RowCount = sts[size_t(i)]->groups;
        o.Destroy = DestroySlice;
        o.Private = sl;
        o.RefCount = 1;
    }
    for (int64_t i = 0; i < n; ++i) {
        AggStateDestroy(sts[size_t(i)]);
        std::memset(hts[i], 0, QDB_HASH_TABLE_SIZE);
    }
    return total;
}

void qdb_gpu_release_rowsets(qdb_rowset* rs, int64_t n) {
    for (int64_t i = 0; rs && i < n; ++i) {
        if (rs[i].Destroy) rs[i].Destroy(&rs[i]);
    }
}

int64_t qdb_gpu_autotune_info(char* buf, int64_t cap) {
    Tuner& t = Tune();
    std::lock_guard<std::mutex> lk(t.mu);
    std::string js = "{\"searches\": " + std::to_string(t.tuned) + ", \"trials\": " + std::to_string(t.trials) +
                     ", \"reused\": " + std::to_string(t.reused) +
                     ", \"resized\": " + std::to_string(t.resized) +
                     ", \"graph_replays\": " + std::to_string(Ctx().graph_replays) +
                     ", \"batched_states\": {\"low\": " + std::to_string(t.states_low) +
                     ", \"high\": " + std::to_string(t.states_high) + "}, \"configs\": [";
    bool first = true;
    for (auto& kv : t.best) {
        char e[256];
        const bool low = std::get<0>(kv.first).rfind("low:", 0) == 0;
        std::snprintf(e, sizeof(e), "%s{\"class\": \"%s\", \"rows_class\": %d, \"states_class\": %d, \"threads\": %d, "
                                    "\"smem_slots\": %d, \"chunk_rows\": %lld}",
                      first ? "" : ", ", low ? "low" : "high", std::get<1>(kv.first), std::get<2>(kv.first), kv.second.threads,
                      kv.second.smem_slots, (long long)kv.second.chunk_rows);
        js += e;
        first = false;
    }
    js += "]}";
    if (buf && cap > 0) {
        const size_t k = std::min<size_t>(size_t(cap - 1), js.size());
        std::memcpy(buf, js.data(), k);
        buf[k] = 0;
    }
    return int64_t(js.size());
}

void qdb_gpu_autotune_reset(void) {
    Tuner& t = Tune();
    std::lock_guard<std::mutex> lk(t.mu);
    t.best.clear();
    t.ratio.clear();
    t.tuned = t.trials = t.reused = t.resized = 0;
    t.states_low = t.states_high = 0;
}

}  // extern "C"
