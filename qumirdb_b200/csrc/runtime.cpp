// runtime.cpp — the C ABI of include/qdb_gpu.h: programs, per-task device
// states behind the engine's caller-owned state buffers, staging of row sets
// into device memory, the table growth / replay loop, kernel timing.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <atomic>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/qdb_gpu.h"
#include "fast.h"
#include "kernels.h"
#include "lower.h"
#include "runtime.h"

namespace qdb {

// ---------------------------------------------------------------------------
// Errors, streams, memory.
// ---------------------------------------------------------------------------
thread_local std::string t_error;

void SetErr(const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    std::vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    t_error = buf;
}

bool CudaOk(cudaError_t e, const char* what) {
    if (e == cudaSuccess) return true;
    SetErr("%s: %s", what, cudaGetErrorString(e));
    return false;
}

namespace {

std::mutex g_mu;
cudaStream_t g_lib_stream = nullptr;
thread_local cudaStream_t t_stream = nullptr;
thread_local bool t_stream_set = false;
std::atomic<int64_t> g_launches{0};

// Kernel timing.
struct ProfRec {
    std::string name;
    int64_t units;
    cudaEvent_t a;
    cudaEvent_t b;
};
std::mutex g_prof_mu;
std::vector<ProfRec> g_prof;
std::atomic<bool> g_prof_on{false};
thread_local int64_t t_prof_open = -1;

}  // namespace

cudaStream_t CurStream() {
    if (t_stream_set) return t_stream;
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_lib_stream) {
        cudaStreamCreateWithFlags(&g_lib_stream, cudaStreamNonBlocking);
        cudaMemPool_t pool;
        int dev = 0;
        cudaGetDevice(&dev);
        if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
            uint64_t threshold = UINT64_MAX;
            cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &threshold);
            // Memory freed on one stream is not handed to another stream's
            // allocation with a wait on the first stream's work behind it:
            // concurrent queries on their own streams must not serialise
            // through the pool (it grows instead).
            int no = 0;
            cudaMemPoolSetAttribute(pool, cudaMemPoolReuseAllowInternalDependencies, &no);
        }
    }
    return g_lib_stream;
}

bool ProfileOn() { return g_prof_on.load(std::memory_order_relaxed); }

void EnsureSmemLimit(const void* fn, size_t bytes) {
    static std::mutex mu;
    static std::vector<std::pair<const void*, size_t>> limits;
    std::lock_guard<std::mutex> lk(mu);
    for (auto& l : limits) {
        if (l.first != fn) continue;
        if (l.second >= bytes) return;
        if (cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, int(bytes)) == cudaSuccess) {
            l.second = bytes;
        } else {
            cudaGetLastError();
        }
        return;
    }
    if (cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, int(bytes)) == cudaSuccess) {
        limits.emplace_back(fn, bytes);
    } else {
        cudaGetLastError();
    }
}

void ProfileBegin(cudaStream_t s, const char* name, int64_t units) {
    if (!g_prof_on.load(std::memory_order_relaxed)) return;
    ProfRec r;
    r.name = name;
    r.units = units;
    cudaEventCreate(&r.a);
    cudaEventCreate(&r.b);
    cudaEventRecord(r.a, s);
    std::lock_guard<std::mutex> lk(g_prof_mu);
    g_prof.push_back(r);
    t_prof_open = int64_t(g_prof.size()) - 1;
}

void ProfileEnd(cudaStream_t s) {
    if (t_prof_open < 0) return;
    std::lock_guard<std::mutex> lk(g_prof_mu);
    if (t_prof_open < int64_t(g_prof.size())) cudaEventRecord(g_prof[t_prof_open].b, s);
    t_prof_open = -1;
}

void CountLaunch(int n) { g_launches.fetch_add(n, std::memory_order_relaxed); }

void* DevAlloc(size_t bytes, cudaStream_t s) {
    void* p = nullptr;
    if (bytes == 0) bytes = 16;
    if (cudaMallocAsync(&p, bytes, s) != cudaSuccess) {
        cudaGetLastError();
        SetErr("device allocation of %zu bytes failed", bytes);
        return nullptr;
    }
    return p;
}

void DevFree(void* p, cudaStream_t s) {
    if (p) cudaFreeAsync(p, s);
}

// Pinned host mirrors of the per-state counters, carved from slabs pinned
// once per process: pinning or unpinning a page synchronises the device and
// costs milliseconds, far more than the query steps that use the mirrors.
namespace {
std::mutex g_pin_mu;
std::vector<AggCounters*> g_pin_free;
}  // namespace

AggCounters* PinnedCountersGet() {
    std::lock_guard<std::mutex> lk(g_pin_mu);
    if (g_pin_free.empty()) {
        constexpr int kSlab = 256;
        void* slab = nullptr;
        if (cudaMallocHost(&slab, sizeof(AggCounters) * kSlab) != cudaSuccess) {
            cudaGetLastError();
            return nullptr;
        }
        for (int i = kSlab - 1; i >= 0; --i) g_pin_free.push_back(static_cast<AggCounters*>(slab) + i);
    }
    AggCounters* c = g_pin_free.back();
    g_pin_free.pop_back();
    return c;
}

namespace {

std::mutex g_host_mu;
std::vector<std::vector<void*>> g_host_free(64);     // by power-of-two size class
std::vector<std::pair<void*, int>> g_host_class;     // live buffer -> class (sorted by address)
char* g_host_arena = nullptr;                        // page-locked once, carved by size class
size_t g_host_arena_size = 0;
size_t g_host_arena_used = 0;

int HostClass(size_t bytes) {
    int c = 16;   // 64 KiB and up
    while (c < 63 && (size_t(1) << c) < bytes) ++c;
    return c;
}

// Bytes of page-locked memory reserved for host outputs at the first output
// (QDB_PINNED_OUTPUT_MB, default 4 GiB): page-locking later, while queries
// run, would hold the driver and stall every stream.
size_t HostArenaBytes() {
    const char* e = std::getenv("QDB_PINNED_OUTPUT_MB");
    const long long mb = e ? std::atoll(e) : 4096;
    return size_t(std::max<long long>(mb, 0)) << 20;
}

}  // namespace

void* HostOutAlloc(size_t bytes) {
    const int c = HostClass(std::max<size_t>(bytes, 1));
    const size_t size = size_t(1) << c;
    std::lock_guard<std::mutex> lk(g_host_mu);
    if (!g_host_free[size_t(c)].empty()) {
        void* p = g_host_free[size_t(c)].back();
        g_host_free[size_t(c)].pop_back();
        return p;
    }
    if (!g_host_arena && g_host_arena_size == 0) {
        g_host_arena_size = HostArenaBytes();
        void* a = nullptr;
        if (g_host_arena_size && cudaMallocHost(&a, g_host_arena_size) == cudaSuccess) {
            g_host_arena = static_cast<char*>(a);
        } else {
            cudaGetLastError();
            g_host_arena_size = 1;   // not again
        }
    }
    void* p = nullptr;
    int tag = c;
    if (g_host_arena && g_host_arena_used + size <= g_host_arena_size) {
        p = g_host_arena + g_host_arena_used;
        g_host_arena_used += size;
    } else {
        p = std::malloc(size);   // pageable once the page-locked arena is used up
        if (!p) return nullptr;
        tag = -c;
    }
    auto it = std::lower_bound(g_host_class.begin(), g_host_class.end(), std::make_pair(p, INT32_MIN));
    g_host_class.insert(it, std::make_pair(p, tag));
    return p;
}

void HostOutFree(void* p) {
    if (!p) return;
    std::lock_guard<std::mutex> lk(g_host_mu);
    auto it = std::lower_bound(g_host_class.begin(), g_host_class.end(), std::make_pair(p, INT32_MIN));
    if (it == g_host_class.end() || it->first != p) return;
    if (it->second < 0) {   // pageable
        std::free(p);
        g_host_class.erase(it);
        return;
    }
    g_host_free[size_t(it->second)].push_back(p);
}

void PinnedCountersPut(AggCounters* c) {
    if (!c) return;
    std::lock_guard<std::mutex> lk(g_pin_mu);
    g_pin_free.push_back(c);
}

bool IsDevicePtr(const void* p) {
    if (!p) return false;
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

// Device copy of `bytes` at `p` (host or device); adds owned buffers to st.
namespace {

// cuMemGetAddressRange through the runtime's driver entry point (no link
// against the driver library).
using AddrRangeFn = int (*)(unsigned long long*, size_t*, unsigned long long);

AddrRangeFn AddrRange() {
    static AddrRangeFn fn = [] {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuMemGetAddressRange", &f, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess) {
            cudaGetLastError();
            return AddrRangeFn(nullptr);
        }
        return reinterpret_cast<AddrRangeFn>(f);
    }();
    return fn;
}

}  // namespace

// Live allocations of qdb_gpu_alloc, [begin, end) by begin: a column inside
// one is on the device without a driver query (a batch of many row sets meets
// hundreds of distinct buffers, and two driver queries per buffer cost more
// host time than the batched launch saves).
namespace {
std::mutex g_alloc_mu;
std::map<uintptr_t, uintptr_t> g_allocs;

bool InOwnAllocation(uintptr_t a, size_t bytes) {
    std::lock_guard<std::mutex> lk(g_alloc_mu);
    auto it = g_allocs.upper_bound(a);
    if (it == g_allocs.begin()) return false;
    --it;
    return a + bytes <= it->second;
}
}  // namespace

const void* Staging::Device(const void* p, size_t bytes) {
    if (!p) return nullptr;
    const uintptr_t a = reinterpret_cast<uintptr_t>(p);
    for (const auto& r : dev_ranges) {
        if (a >= r.first && a + bytes <= r.second) return p;
    }
    if (InOwnAllocation(a, bytes)) return p;
    if (IsDevicePtr(p)) {
        unsigned long long base = 0;
        size_t size = 0;
        if (AddrRangeFn fn = AddrRange()) {
            if (fn(&base, &size, static_cast<unsigned long long>(a)) == 0 && size) {
                if (dev_ranges.size() >= 16) dev_ranges.erase(dev_ranges.begin());
                dev_ranges.emplace_back(uintptr_t(base), uintptr_t(base) + size);
            }
        }
        return p;
    }
    void* d = DevAlloc(bytes, s);
    if (!d) return nullptr;
    cudaMemcpyAsync(d, p, bytes, cudaMemcpyHostToDevice, s);
    owned.push_back(d);
    return d;
}

Staging::~Staging() {
    for (void* p : owned) DevFree(p, s);
}

// Resolves the plan's probe/scan column slots against a row set.
// A string column's offsets and bytes on the device.  Host offsets give the
// byte count to stage; device offsets need device bytes.
bool ResolveStrings(ColDesc& cd, const qdb_column& c, int64_t n, Staging& st, int input) {
    const int ow = c.OffsetWidth;
    if ((ow != 4 && ow != 8) || (n > 0 && (!c.Offsets || !c.Data))) {
        SetErr("string column %d needs offsets of width 4 or 8 and data", input);
        return false;
    }
    cd.offset_width = ow;
    if (n == 0) {
        cd.offsets = nullptr;
        cd.data = nullptr;
        return true;
    }
    if (IsDevicePtr(c.Offsets)) {
        if (!IsDevicePtr(c.Data)) {
            SetErr("string column %d: device offsets with host bytes", input);
            return false;
        }
        cd.offsets = static_cast<const char*>(c.Offsets);
        cd.data = c.Data;
        return true;
    }
    // Host offsets are checked here (non-decreasing from a non-negative
    // start), so that the kernel reads only the staged bytes; device offsets
    // are taken as Arrow guarantees them.
    int64_t prev = 0, end = 0;
    for (int64_t r = 0; r <= n; ++r) {
        const int64_t o = ow == 8 ? static_cast<const int64_t*>(c.Offsets)[r] : static_cast<const int32_t*>(c.Offsets)[r];
        if (o < prev) {
            SetErr("string column %d: offsets decrease at row %lld", input, (long long)r);
            return false;
        }
        prev = end = o;
    }
    cd.offsets = static_cast<const char*>(st.Device(c.Offsets, size_t(n + 1) * size_t(ow)));
    // No bytes at all (every string empty): no byte is ever read.
    cd.data = end > 0 ? static_cast<const char*>(st.Device(c.Data, size_t(end))) : cd.offsets;
    return cd.offsets != nullptr && cd.data != nullptr;
}

bool ResolveColumns(AggPlan& P, const ColumnMap& cm, const qdb_column_type* types, const qdb_rowset* rs,
                    Staging& st) {
    const int64_t n = rs->RowCount;
    for (int slot = 0; slot < P.ncols; ++slot) {
        ColDesc& cd = P.cols[slot];
        if (cd.build) continue;
        const int input = cm.input_of[slot];
        if (input >= rs->ColumnCount) {
            SetErr("row set has %lld columns, the program reads column %d", (long long)rs->ColumnCount, input);
            return false;
        }
        const qdb_column& c = rs->Columns[input];
        const int t = types[input].type;
        cd.offsets = nullptr;
        cd.offset_width = 0;
        if (t == QDB_TYPE_STRING) {
            if (!ResolveStrings(cd, c, n, st, input)) return false;
        } else if (t == QDB_TYPE_BOOL) {
            const size_t bytes = size_t((c.DataBitOffset + n + 7) / 8);
            cd.data = static_cast<const char*>(st.Device(c.Data, bytes));
            cd.bit_off = c.DataBitOffset;
        } else {
            cd.data = static_cast<const char*>(st.Device(c.Data, size_t(n) * cd.width));
        }
        if (n > 0 && !cd.data) {
            if (t_error.empty()) SetErr("column %d has no data", input);
            return false;
        }
        cd.mask = nullptr;
        cd.mask_off = 0;
        if (c.Mask) {
            cd.mask = static_cast<const uint8_t*>(st.Device(c.Mask, size_t((c.MaskBitOffset + n + 7) / 8)));
            cd.mask_off = c.MaskBitOffset;
        }
    }
    P.selection = rs->Selection ? static_cast<const uint8_t*>(st.Device(rs->Selection, size_t(n))) : nullptr;
    P.has_selection = P.selection != nullptr;
    return true;
}

// Offsets every scan column of a resolved plan by `begin` rows.
AggPlan OffsetPlan(const AggPlan& P, int64_t begin) {
    AggPlan q = P;
    for (int slot = 0; slot < q.ncols; ++slot) {
        ColDesc& cd = q.cols[slot];
        if (cd.build) continue;
        if (cd.offset_width) {
            if (cd.offsets) cd.offsets += begin * cd.offset_width;   // the offsets index the bytes from 0
        } else if (cd.kind == LK_BOOLBIT) {
            cd.bit_off += begin;
        } else {
            cd.data += begin * cd.width;
        }
        if (cd.mask) cd.mask_off += begin;
    }
    if (q.selection) q.selection += begin;
    return q;
}

int64_t NextPow2(int64_t v) {
    int64_t p = 1;
    while (p < v) p <<= 1;
    return p;
}

// ---------------------------------------------------------------------------
// Aggregate table state.
// ---------------------------------------------------------------------------
void AggArenaRelease(AggArena* a) {
    if (!a || --a->refs > 0) return;
    DevFree(a->p, a->s);
    delete a;
}

// Slots are 16-byte aligned; a 48-byte slot still spans two 32-byte sectors.
int SlotWords(const AggPlan& p, bool wide) {
    const int w = (wide ? 1 + p.key_words : 1) + p.state_words;
    return (w + 1) & ~1;
}

bool AllocTable(const AggPlan& p, int64_t capacity, cudaStream_t s, GTableDev& t) {
    t.wide = p.key_words > 1 ? 1 : 0;
    t.capacity = capacity;
    t.slot_words = SlotWords(p, t.wide);
    t.key_off = t.wide ? 1 : 0;
    t.state_off = t.wide ? 1 + p.key_words : 1;
    t.slots = static_cast<uint64_t*>(DevAlloc(size_t(capacity + 1) * t.slot_words * 8, s));
    if (!t.slots) return false;
    AggInitTable(p, t, s);
    return true;
}

AggTableState* StateOf(void* ht) {
    if (!ht) return nullptr;
    AggTableState* st = *static_cast<AggTableState**>(ht);
    if (!st || st->magic != kAggMagic) return nullptr;
    return st;
}

void MirrorHeader(void* ht, const AggTableState* st, const AggPlan& p) {
    int64_t* w = static_cast<int64_t*>(ht);
    w[8] = st ? st->t.capacity : 0;     // Capacity
    w[9] = st ? st->groups : 0;         // Size
    w[10] = p.naggs;                    // NumAggs
    w[11] = p.nkeyparts;                // NumKeys
    w[12] = p.key_words * 8;            // KeySize
}

bool ReadCounters(AggTableState* st) {
    cudaMemcpyAsync(st->hc, st->dc, sizeof(AggCounters), cudaMemcpyDeviceToHost, st->s);
    if (!CudaOk(cudaStreamSynchronize(st->s), "aggregate update")) return false;
    if (st->hc->error) {
        SetErr("aggregate kernel reported device error %d", st->hc->error);
        return false;
    }
    return true;
}

void ResetCounters(AggTableState* st) { cudaMemsetAsync(st->dc, 0, sizeof(AggCounters), st->s); }

bool Grow(AggTableState* st, const AggPlan& p, int64_t min_groups) {
    int64_t cap = st->t.capacity;
    while (cap < 2 * min_groups) cap <<= 1;
    if (cap == st->t.capacity) cap <<= 1;
    GTableDev nt;
    if (!AllocTable(p, cap, st->s, nt)) return false;
    AggRehash(p, st->t, nt, st->dc, st->s);
    if (!st->table_in_arena) DevFree(st->t.slots, st->s);
    st->table_in_arena = false;
    st->t = nt;
    return true;
}

bool EnsureBuffers(AggTableState* st, const AggPlan& p, int64_t rows) {
    const int64_t need = std::min<int64_t>(std::max<int64_t>(rows, 1), kChunkRows);
    if (st->deferred_cap < need) {
        for (int j = 0; j < 2; ++j) {
            DevFree(st->deferred[j], st->s);
            st->deferred[j] = static_cast<int64_t*>(DevAlloc(size_t(need) * 16, st->s));
            if (!st->deferred[j]) return false;
        }
        st->deferred_cap = need;
    }
    const int64_t spill = int64_t(DeviceSMs()) * st->smem_slots;
    if (st->spill_cap < spill) {
        DevFree(st->spill, st->s);
        st->spill = static_cast<uint64_t*>(DevAlloc(size_t(spill) * (1 + p.state_words) * 8, st->s));
        if (!st->spill) return false;
        st->spill_cap = spill;
    }
    return true;
}

AggTableState* AggStateCreate(const AggPlan& p, int64_t capacity_hint, int64_t expected, cudaStream_t s) {
    auto* st = new AggTableState();
    st->s = s;
    st->expected = expected;
    // A high-cardinality hint gets the larger shared tier (4096 slots: the
    // more of a skewed stream's hot keys stay out of the global table).
    if (expected > (int64_t(1) << 16)) st->smem_slots = 4096;
    int64_t cap = std::max<int64_t>(1024, NextPow2(std::max<int64_t>(capacity_hint, 1)));
    if (expected > 0) cap = std::max(cap, NextPow2(expected + expected / 2));
    st->hc = PinnedCountersGet();
    if (!st->hc) {
        delete st;
        SetErr("pinned allocation failed");
        return nullptr;
    }
    st->dc = static_cast<AggCounters*>(DevAlloc(sizeof(AggCounters), s));
    if (!st->dc || !AllocTable(p, cap, s, st->t)) {
        DevFree(st->dc, s);
        PinnedCountersPut(st->hc);
        delete st;
        return nullptr;
    }
    ResetCounters(st);
    // A keyless aggregate has its group before any row arrives: key 0 is
    // all-zero bytes in its home slot.
    if (p.nkeyparts == 0) {
        const int64_t slot = int64_t(Fmix64(0) & uint64_t(cap - 1));
        cudaMemsetAsync(st->t.slots + slot * st->t.slot_words + st->t.key_off, 0, 8, s);
        st->groups = 1;
    }
    return st;
}

// Fused join + keyless aggregate through the join-sum fast kernel: folds into
// the keyless group's slot (created with the table at key 0).
bool AggRunJoinSum(AggTableState* st, const JoinSumShape& shape, const JTableDev& jt, int64_t nrows) {
    const int64_t slot = int64_t(Fmix64(0) & uint64_t(st->t.capacity - 1));
    uint64_t* states = st->t.slots + slot * st->t.slot_words + st->t.state_off;
    ResetCounters(st);
    JoinSumRun(shape, jt, nrows, states, st->dc, st->s);
    if (!ReadCounters(st)) return false;
    st->matched += int64_t(st->hc->matched);
    return true;
}

void AggJoinSumTargets(AggTableState* st, uint64_t** states, unsigned long long** matched) {
    const int64_t slot = int64_t(Fmix64(0) & uint64_t(st->t.capacity - 1));
    *states = st->t.slots + slot * st->t.slot_words + st->t.state_off;
    *matched = &st->dc->matched;
    ResetCounters(st);
}

void AggJoinSumFetch(AggTableState* st, cudaStream_t s) {
    cudaMemcpyAsync(st->hc, st->dc, sizeof(AggCounters), cudaMemcpyDeviceToHost, s);
}

bool AggJoinSumCommit(AggTableState* st) {
    if (st->hc->error) {
        SetErr("aggregate kernel reported device error %d", st->hc->error);
        return false;
    }
    st->matched += int64_t(st->hc->matched);
    return true;
}

int64_t AggStateGroups(const AggTableState* st) { return st ? st->groups : 0; }
int64_t AggStateMatched(const AggTableState* st) { return st ? st->matched : 0; }
AggTableState* AggStateOf(void* ht) { return StateOf(ht); }
void AggMirrorHeader(void* ht, const AggTableState* st, const AggPlan& p) { MirrorHeader(ht, st, p); }

void AggStateDestroy(AggTableState* st) {
    if (!st) return;
    if (!st->table_in_arena) DevFree(st->t.slots, st->s);
    if (!st->dc_in_arena) DevFree(st->dc, st->s);
    AggArenaRelease(st->arena);
    DevFree(st->deferred[0], st->s);
    DevFree(st->deferred[1], st->s);
    DevFree(st->spill, st->s);
    DevFree(st->seeds, st->s);
    // Every readback into the mirror was synchronised when it was read.
    PinnedCountersPut(st->hc);
    st->magic = 0;
    delete st;
}

constexpr int64_t kSeedMinRows = int64_t(16) << 20;  // updates worth a heavy-hitter sample (~60 us)
constexpr int kSeedKeys = 2048;                        // seeds kept (the tier takes up to half its slots)

// Runs the fused kernel over `rows` rows of a resolved plan, then replays
// deferred rows and spilled entries after growing the table.
bool AggRun(AggTableState* st, const AggPlan& plan, int64_t rows, const JoinKeyPlan* jk, const JTableDev* jt,
            int inline_slot) {
    if (!EnsureBuffers(st, plan, rows)) return false;
    // Few expected groups (or none): fold the first groups of each CTA into
    // lane-private accumulators.
    const bool priv = plan.nkeyparts == 0 || (st->expected > 0 && st->expected <= 64);
    FastPlan fast;
    const bool use_fast = jk == nullptr && MatchFast(plan, fast);
    // The table is grown before a chunk that could overfill it (a full
    // table turns every new group's rows into replays): the chunk's new
    // groups are projected from the groups per row this call has seen so
    // far, or, with no planner hint, from a first chunk of kProbeRows rows
    // that the table is grown to hold whole.
    constexpr int64_t kProbeRows = int64_t(1) << 20;
    int64_t seen_rows = 0, seen_groups = 0;
    for (int64_t begin = 0, n = 0; begin < rows; begin += n) {
        n = std::min<int64_t>(kChunkRows, rows - begin);
        if (plan.nkeyparts > 0 && jk == nullptr) {
            int64_t add;
            if (seen_rows > 0) {
                const double r = double(seen_groups) / double(seen_rows);
                add = std::min<int64_t>(n, int64_t(std::ceil(r * 1.25 * double(n))) + 1024);
            } else if (st->expected > 0) {
                add = std::min<int64_t>(n, std::max<int64_t>(0, st->expected - st->groups));
            } else {
                n = std::min<int64_t>(n, kProbeRows);
                add = n;
            }
            if (double(st->groups + add) > 0.85 * double(st->t.capacity) && !Grow(st, plan, st->groups + add))
                return false;
        }
        const int64_t groups_before = st->groups;
        const AggPlan chunk = OffsetPlan(plan, begin);
        // A large high-cardinality update samples its keys once; the most
        // frequent seed the kernel's shared tier from then on.
        if (!priv && use_fast && !st->seeded && rows >= kSeedMinRows && AggHighSeedable(chunk, fast)) {
            st->seeded = true;
            st->seeds = static_cast<uint64_t*>(DevAlloc(size_t(kSeedKeys) * 8 + 16, st->s));
            void* scratch = st->seeds ? DevAlloc(AggSeedScratch(), st->s) : nullptr;
            if (!scratch || !AggSeedHeavy(chunk, fast, n, st->seeds, reinterpret_cast<int*>(st->seeds + kSeedKeys),
                                          kSeedKeys, scratch, st->s)) {
                DevFree(st->seeds, st->s);
                st->seeds = nullptr;
            }
            DevFree(scratch, st->s);
            cudaGetLastError();
        }
        AggUpdateArgs a;
        a.plan = &chunk;
        a.nrows = n;
        a.table = st->t;
        a.counters = st->dc;
        a.deferred = st->deferred[0];
        a.deferred_cap = st->deferred_cap;
        a.spill = st->spill;
        a.spill_cap = st->spill_cap;
        a.smem_slots = st->smem_slots;
        a.priv = priv;
        a.fast = use_fast ? &fast : nullptr;
        if (st->seeds && !priv) {
            a.seeds = st->seeds;
            a.nseed = reinterpret_cast<const int*>(st->seeds + kSeedKeys);
        }
        if (jk) {
            a.join = true;
            a.jkey = *jk;
            a.jt = *jt;
            a.inline_slot = inline_slot;
        }
        ResetCounters(st);
        AggUpdate(a, st->s);
        if (!ReadCounters(st)) return false;
        st->groups += int64_t(st->hc->new_groups);
        st->matched += int64_t(st->hc->matched);
        if (!AggReplay(st, plan, a, int64_t(st->hc->deferred), int64_t(st->hc->spilled))) return false;
        seen_rows += n;
        seen_groups += st->groups - groups_before;
    }
    return true;
}

bool AggReplay(AggTableState* st, const AggPlan& plan, const AggUpdateArgs& a, int64_t ndef, int64_t nspill) {
    int cur = 0;
    for (int round = 0; (ndef > 0 || nspill > 0); ++round) {
        if (round > 16) {
            SetErr("aggregate replay did not converge");
            return false;
        }
        if (!Grow(st, plan, st->groups + ndef + nspill)) return false;
        ResetCounters(st);
        AggMergeSpill(plan, st->spill, nspill, st->t, st->dc, st->s);
        // Replay deferred rows into the grown table; new deferrals go to the other buffer.
        AggUpdateArgs r = a;
        r.table = st->t;
        r.counters = st->dc;
        r.index = st->deferred[cur];
        r.nindex = ndef;
        r.deferred = st->deferred[cur ^ 1];
        r.deferred_cap = st->deferred_cap;
        r.spill = st->spill;
        r.spill_cap = st->spill_cap;
        AggUpdate(r, st->s);
        cur ^= 1;
        if (!ReadCounters(st)) return false;
        st->groups += int64_t(st->hc->new_groups);
        ndef = int64_t(st->hc->deferred);
        nspill = int64_t(st->hc->spilled);
    }
    if (st->groups * 2 > st->t.capacity) {
        if (!Grow(st, plan, st->groups)) return false;
    }
    return true;
}

// ---------------------------------------------------------------------------
// Output row sets.
// ---------------------------------------------------------------------------
struct OwnedRowset {
    std::vector<void*> host;
    std::vector<void*> dev;
    std::vector<qdb_column> cols;
    cudaStream_t s = nullptr;   // device buffers are released in this stream's order
};

// Device outputs go back to the stream-ordered pool on the library stream:
// a caller that read them on another stream synchronises that stream first.
void DestroyOwned(qdb_rowset* rs) {
    if (!rs || !rs->Private) return;
    auto* o = static_cast<OwnedRowset*>(rs->Private);
    for (void* p : o->host) HostOutFree(p);
    for (void* p : o->dev) DevFree(p, o->s);
    delete o;
    rs->Private = nullptr;
    rs->Columns = nullptr;
}

// Moves device output columns into `out` (copying to host unless on_device).
bool EmitRowset(std::vector<AggOutputCol>& cols, const std::vector<int>& types, int64_t rows, bool on_device,
                cudaStream_t s, qdb_rowset* out, const OutBlock* blk) {
    auto* o = new OwnedRowset();
    o->s = s;
    o->cols.resize(cols.size());
    if (blk && blk->p) {
        // One block: the rowset owns it on the device, or one copy of it
        // (columns at the same offsets) on the host.
        char* h = nullptr;
        if (on_device) {
            o->dev.push_back(blk->p);
        } else {
            h = static_cast<char*>(HostOutAlloc(std::max<size_t>(blk->bytes, 16)));
            if (!h) {
                delete o;
                SetErr("pinned allocation failed");
                return false;
            }
            o->host.push_back(h);
            cudaMemcpyAsync(h, blk->p, blk->bytes, cudaMemcpyDeviceToHost, s);
        }
        char* b = static_cast<char*>(blk->p);
        auto at = [&](void* d) -> char* { return on_device ? static_cast<char*>(d) : h + (static_cast<char*>(d) - b); };
        for (size_t k = 0; k < cols.size(); ++k) {
            qdb_column& c = o->cols[k];
            std::memset(&c, 0, sizeof(c));
            c.Data = at(cols[k].data);
            if (cols[k].valid) c.Mask = reinterpret_cast<const uint8_t*>(at(cols[k].valid));
            if (cols[k].offsets) {
                c.Offsets = at(cols[k].offsets);
                c.OffsetWidth = 4;
            }
        }
        if (!CudaOk(cudaStreamSynchronize(s), "output")) {
            for (void* p : o->host) HostOutFree(p);
            delete o;
            return false;
        }
        if (!on_device) DevFree(blk->p, s);
        std::memset(out, 0, sizeof(*out));
        out->Columns = o->cols.data();
        out->ColumnCount = int64_t(cols.size());
        out->RowCount = rows;
        out->Destroy = DestroyOwned;
        out->Private = o;
        out->RefCount = 1;
        return true;
    }
    for (size_t k = 0; k < cols.size(); ++k) {
        qdb_column& c = o->cols[k];
        std::memset(&c, 0, sizeof(c));
        const size_t w = size_t(StorageWidth(types[k]));
        const size_t dbytes = std::max<size_t>(1, size_t(rows) * w);
        const size_t mbytes = size_t((rows + 31) / 32) * 4;
        if (on_device) {
            c.Data = cols[k].data;
            o->dev.push_back(cols[k].data);
            if (cols[k].valid) {
                c.Mask = reinterpret_cast<const uint8_t*>(cols[k].valid);
                o->dev.push_back(cols[k].valid);
            }
            if (cols[k].offsets) {
                c.Offsets = cols[k].offsets;
                c.OffsetWidth = 4;
                o->dev.push_back(cols[k].offsets);
            }
        } else {
            void* h = HostOutAlloc(dbytes);
            cudaMemcpyAsync(h, cols[k].data, size_t(rows) * w, cudaMemcpyDeviceToHost, s);
            c.Data = static_cast<char*>(h);
            o->host.push_back(h);
            if (cols[k].valid) {
                void* m = HostOutAlloc(std::max<size_t>(4, mbytes));
                cudaMemcpyAsync(m, cols[k].valid, mbytes, cudaMemcpyDeviceToHost, s);
                c.Mask = static_cast<const uint8_t*>(m);
                o->host.push_back(m);
            }
            if (cols[k].offsets) {
                void* off = HostOutAlloc(size_t(rows + 1) * 4);
                cudaMemcpyAsync(off, cols[k].offsets, size_t(rows + 1) * 4, cudaMemcpyDeviceToHost, s);
                c.Offsets = off;
                c.OffsetWidth = 4;
                o->host.push_back(off);
            }
        }
    }
    // The host copies have landed once the stream drains; only then do the
    // device buffers go back to the pool.
    if (!CudaOk(cudaStreamSynchronize(s), "output")) {
        for (void* p : o->host) HostOutFree(p);
        delete o;
        return false;
    }
    if (!on_device) {
        for (auto& c : cols) {
            DevFree(c.data, s);
            DevFree(c.valid, s);
            DevFree(c.offsets, s);
        }
    }
    std::memset(out, 0, sizeof(*out));
    out->Columns = o->cols.data();
    out->ColumnCount = int64_t(cols.size());
    out->RowCount = rows;
    out->Destroy = DestroyOwned;
    out->Private = o;
    out->RefCount = 1;
    return true;
}

namespace {
bool AllocOutputBlock(const std::vector<int>& types, int64_t rows, std::vector<AggOutputCol>& cols, cudaStream_t s,
                      OutBlock& blk) {
    cols.resize(types.size());
    for (auto& c : cols) std::memset(&c, 0, sizeof(c));
    const size_t words = size_t((std::max<int64_t>(rows, 1) + 31) / 32);
    auto up = [](size_t b) { return (b + 255) & ~size_t(255); };
    size_t data_bytes = 0, off_bytes = 0;
    for (int t : types) {
        data_bytes += up(std::max<size_t>(16, size_t(rows) * size_t(StorageWidth(t))));
        if (t == QDB_TYPE_CHAR1) off_bytes += up(size_t(rows + 1) * 4);
    }
    const size_t valid_bytes = types.size() * words * 4;
    blk.bytes = data_bytes + off_bytes + valid_bytes;
    char* block = static_cast<char*>(DevAlloc(blk.bytes + 16, s));
    blk.p = block;
    if (!block) return false;
    char* d = block;
    char* o = block + data_bytes;
    auto* v = reinterpret_cast<uint32_t*>(block + data_bytes + off_bytes);
    for (size_t k = 0; k < types.size(); ++k) {
        AggOutputCol& c = cols[k];
        c.type = types[k];
        c.data = d;
        d += up(std::max<size_t>(16, size_t(rows) * size_t(StorageWidth(types[k]))));
        c.valid = v + k * words;
        if (types[k] == QDB_TYPE_CHAR1) {
            c.offsets = reinterpret_cast<int32_t*>(o);
            o += up(size_t(rows + 1) * 4);
            cudaMemsetAsync(c.offsets, 0, 4, s);
        }
    }
    cudaMemsetAsync(v, 0, valid_bytes, s);
    return true;
}
}  // namespace


bool AllocOutputCols(const std::vector<int>& types, int64_t rows, bool with_valid, std::vector<AggOutputCol>& cols,
                     cudaStream_t s, OutBlock* blk) {
    if (blk && with_valid) return AllocOutputBlock(types, rows, cols, s, *blk);
    cols.resize(types.size());
    for (auto& c : cols) std::memset(&c, 0, sizeof(c));
    auto fail = [&]() {
        for (auto& c : cols) {
            DevFree(c.data, s);
            DevFree(c.valid, s);
            DevFree(c.offsets, s);
        }
        return false;
    };
    for (size_t k = 0; k < types.size(); ++k) {
        AggOutputCol& c = cols[k];
        c.type = types[k];
        const size_t w = size_t(StorageWidth(types[k]));
        c.data = static_cast<char*>(DevAlloc(std::max<size_t>(16, size_t(rows) * w), s));
        if (!c.data) return fail();
        if (with_valid) {
            const size_t mb = std::max<size_t>(4, size_t((rows + 31) / 32) * 4);
            c.valid = static_cast<uint32_t*>(DevAlloc(mb, s));
            if (!c.valid) return fail();
            cudaMemsetAsync(c.valid, 0, mb, s);
        }
        if (types[k] == QDB_TYPE_CHAR1) {
            c.offsets = static_cast<int32_t*>(DevAlloc(size_t(rows + 1) * 4, s));
            if (!c.offsets) return fail();
            cudaMemsetAsync(c.offsets, 0, 4, s);
        }
    }
    return true;
}

int64_t AggFinish(AggTableState* st, const AggLowering& lw, uint32_t flags, qdb_rowset* out) {
    const int64_t groups = st->groups;
    std::vector<int> types;
    for (int k = 0; k < lw.out.n; ++k) types.push_back(lw.out.out_type[k]);
    std::vector<AggOutputCol> cols;
    OutBlock blk;
    if (!AllocOutputCols(types, groups, true, cols, st->s, &blk)) {
        SetErr("output allocation failed");
        return -1;
    }
    void* scratch = DevAlloc(AggFinalizeScratch(st->t), st->s);
    if (!scratch) return -1;
    ResetCounters(st);
    AggFinalize(lw.plan, lw.out, st->t, cols.data(), int(cols.size()), groups, scratch, &st->dc->error, st->s,
                true);
    DevFree(scratch, st->s);
    if (!ReadCounters(st)) return -1;
    if (!EmitRowset(cols, types, groups, (flags & QDB_OUT_DEVICE) != 0, st->s, out, &blk)) return -1;
    return groups;
}

}  // namespace qdb

// ===========================================================================
// C ABI
// ===========================================================================
using namespace qdb;

namespace {

void Fill(char* err, size_t len, const char* msg) {
    if (err && len) std::snprintf(err, len, "%s", msg);
    t_error = msg;
}

}  // namespace

namespace qdb {

void HashArgs(const qdb_gpu_program* prog, const AggPlan& plan, int64_t nrows, ExprArgs& a) {
    a.plan = &plan;
    a.nrows = nrows;
    a.nhash = int(prog->expr.out_types.size());
    for (int j = 0; j < a.nhash; ++j) {
        a.hash_slot[j] = uint8_t(prog->expr.value_idx[j]);
        a.hash_type[j] = prog->expr.out_types[j];
        a.hash_nullable[j] = plan.cols[a.hash_slot[j]].nullable;
    }
}

}  // namespace qdb

extern "C" {

int qdb_gpu_init(int device) {
    if (!CudaOk(cudaSetDevice(device), "cudaSetDevice")) return -1;
    if (!CudaOk(cudaFree(nullptr), "context")) return -1;
    CurStream();
    return 0;
}

const char* qdb_gpu_last_error(void) { return t_error.c_str(); }

void qdb_gpu_set_stream(void* stream) {
    t_stream = static_cast<cudaStream_t>(stream);
    t_stream_set = stream != nullptr;
}

void* qdb_gpu_get_stream(void) { return CurStream(); }

int qdb_gpu_synchronize(void) { return CudaOk(cudaStreamSynchronize(CurStream()), "synchronize") ? 0 : -1; }

void* qdb_gpu_alloc(size_t bytes) {
    void* p = nullptr;
    bytes = std::max<size_t>(bytes, 16);
    if (!CudaOk(cudaMalloc(&p, bytes), "cudaMalloc")) return nullptr;
    std::lock_guard<std::mutex> lk(g_alloc_mu);
    g_allocs[reinterpret_cast<uintptr_t>(p)] = reinterpret_cast<uintptr_t>(p) + bytes;
    return p;
}

void qdb_gpu_free(void* ptr) {
    if (!ptr) return;
    {
        std::lock_guard<std::mutex> lk(g_alloc_mu);
        g_allocs.erase(reinterpret_cast<uintptr_t>(ptr));
    }
    cudaFree(ptr);
}

void* qdb_gpu_host_alloc(size_t bytes) {
    void* p = nullptr;
    if (!CudaOk(cudaMallocHost(&p, std::max<size_t>(bytes, 16)), "cudaMallocHost")) return nullptr;
    return p;
}

void qdb_gpu_host_free(void* ptr) {
    if (ptr) cudaFreeHost(ptr);
}

int qdb_gpu_memcpy(void* dst, const void* src, size_t bytes) {
    return CudaOk(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDefault, CurStream()), "memcpy") ? 0 : -1;
}

int qdb_gpu_memset(void* dst, int value, size_t bytes) {
    return CudaOk(cudaMemsetAsync(dst, value, bytes, CurStream()), "memset") ? 0 : -1;
}

void qdb_gpu_profile_enable(int on) { g_prof_on.store(on != 0); }

int64_t qdb_gpu_profile_read(qdb_gpu_kernel_time* out, int64_t cap) {
    std::lock_guard<std::mutex> lk(g_prof_mu);
    int64_t n = 0;
    for (auto& r : g_prof) {
        cudaEventSynchronize(r.b);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, r.a, r.b);
        if (out && n < cap) {
            std::snprintf(out[n].name, sizeof(out[n].name), "%s", r.name.c_str());
            out[n].ms = ms;
            out[n].units = r.units;
        }
        ++n;
        cudaEventDestroy(r.a);
        cudaEventDestroy(r.b);
    }
    g_prof.clear();
    return std::min(n, cap);
}

int64_t qdb_gpu_launch_count(int reset) {
    return reset ? g_launches.exchange(0) : g_launches.load();
}

qdb_gpu_program* qdb_gpu_compile_aggregate(const qdb_aggregate_spec* spec, char* err, size_t err_len) {
    try {
        auto* p = new qdb_gpu_program();
        p->kind = PK_AGG;
        p->flags = spec->flags;
        p->columns.assign(spec->columns, spec->columns + spec->n_columns);
        p->agg = LowerAggregate(*spec);
        p->agg.plan.key_words = std::max(1, p->agg.plan.key_words);
        p->expected_groups = spec->expected_groups;
        return p;
    } catch (const std::exception& e) {
        Fill(err, err_len, e.what());
        return nullptr;
    }
}

qdb_gpu_program* qdb_gpu_compile_filter(int32_t n_columns, const qdb_column_type* columns, int32_t n_nodes,
                                        const qdb_expr* nodes, int32_t predicate, char* err, size_t err_len) {
    try {
        auto* p = new qdb_gpu_program();
        p->kind = PK_FILTER;
        p->columns.assign(columns, columns + n_columns);
        p->expr = LowerFilter(n_columns, columns, n_nodes, nodes, predicate);
        return p;
    } catch (const std::exception& e) {
        Fill(err, err_len, e.what());
        return nullptr;
    }
}

qdb_gpu_program* qdb_gpu_compile_project(int32_t n_columns, const qdb_column_type* columns, int32_t n_nodes,
                                         const qdb_expr* nodes, int32_t n_exprs, const int32_t* exprs, char* err,
                                         size_t err_len) {
    try {
        if (n_exprs > kMaxCols) throw LowerError("too many projections for one device plan");
        auto* p = new qdb_gpu_program();
        p->kind = PK_PROJECT;
        p->columns.assign(columns, columns + n_columns);
        p->expr = LowerProject(n_columns, columns, n_nodes, nodes, n_exprs, exprs);
        return p;
    } catch (const std::exception& e) {
        Fill(err, err_len, e.what());
        return nullptr;
    }
}

qdb_gpu_program* qdb_gpu_compile_hash(int32_t n_columns, const qdb_column_type* columns, int32_t n_keys,
                                      const int32_t* key_columns, char* err, size_t err_len) {
    try {
        if (n_keys < 1 || n_keys > kMaxKeyParts) throw LowerError("hash needs 1..6 key columns");
        if (n_columns < 1 || !columns) throw LowerError("hash needs an input schema");
        // A string key is lowered as a 64-bit slot (its offsets and bytes are
        // resolved per batch from the true schema kept on the program), and
        // the hash kernel reads it as a string.
        std::vector<qdb_column_type> lowered(columns, columns + n_columns);
        for (qdb_column_type& ct : lowered) {
            if (ct.type == QDB_TYPE_STRING) ct.type = QDB_TYPE_U64;
        }
        std::vector<qdb_expr> nodes(n_keys);
        std::vector<int32_t> exprs(n_keys);
        for (int j = 0; j < n_keys; ++j) {
            if (key_columns[j] < 0 || key_columns[j] >= n_columns) throw LowerError("key column out of range");
            const qdb_column_type& ct = lowered[size_t(key_columns[j])];
            std::memset(&nodes[j], 0, sizeof(qdb_expr));
            nodes[j].op = QDB_EXPR_COLUMN;
            nodes[j].type = ct.type;
            nodes[j].scale = ct.scale;
            nodes[j].column = key_columns[j];
            exprs[j] = j;
        }
        auto* p = new qdb_gpu_program();
        p->kind = PK_HASH;
        p->columns.assign(columns, columns + n_columns);
        p->expr = LowerProject(n_columns, lowered.data(), n_keys, nodes.data(), n_keys, exprs.data());
        for (int j = 0; j < n_keys; ++j) {
            p->expr.value_idx[j] = p->expr.cols.slot_of[key_columns[j]];
            p->expr.out_types[j] = columns[key_columns[j]].type;
        }
        return p;
    } catch (const std::exception& e) {
        Fill(err, err_len, e.what());
        return nullptr;
    }
}

void qdb_gpu_program_destroy(qdb_gpu_program* program) { delete program; }

int64_t qdb_gpu_agg_dispatch(const qdb_gpu_program* prog, void* ht, qdb_rowset* batch, int64_t arg, int64_t op) {
    t_error.clear();
    if (!prog || (prog->kind != PK_AGG && prog->kind != PK_JOIN_AGG) || !ht) {
        SetErr("agg_dispatch: not an aggregate program");
        return op == QDB_AGG_OP_UPDATE ? -1 : 0;
    }
    const AggLowering& lw = prog->agg;
    cudaStream_t s = CurStream();
    switch (op) {
        case QDB_AGG_OP_INIT:
        case QDB_AGG_OP_INIT_ROWS: {
            if (StateOf(ht)) AggStateDestroy(StateOf(ht));
            const int64_t hint = op == QDB_AGG_OP_INIT ? arg : arg * 2;
            AggTableState* st = AggStateCreate(lw.plan, hint, prog->expected_groups, s);
            *static_cast<AggTableState**>(ht) = st;
            if (!st) return 0;
            MirrorHeader(ht, st, lw.plan);
            return 1;
        }
        case QDB_AGG_OP_SWITCH_TO_ROWS_AT:
            // The device table already keeps key and states in one row slot.
            return StateOf(ht) ? 1 : 0;
        case QDB_AGG_OP_EXPECT_ROW_GROUPS: {
            AggTableState* st = StateOf(ht);
            if (!st) return 0;
            st->expected = std::max<int64_t>(st->expected, arg);
            if (arg * 2 > st->t.capacity && !Grow(st, lw.plan, arg)) return 0;
            MirrorHeader(ht, st, lw.plan);
            return 1;
        }
        case QDB_AGG_OP_UPDATE: {
            AggTableState* st = StateOf(ht);
            if (!st) {
                SetErr("agg_dispatch(Update) before Init");
                return -1;
            }
            if (prog->kind != PK_AGG) {
                SetErr("a fused join-aggregate is updated through qdb_gpu_join_aggregate_probe");
                return -1;
            }
            if (!batch) return st->groups;
            AggPlan plan = lw.plan;
            Staging stg(st->s);
            if (!ResolveColumns(plan, lw.cols, prog->columns.data(), batch, stg)) return -1;
            if (!AggRun(st, plan, batch->RowCount, nullptr, nullptr)) return -1;
            MirrorHeader(ht, st, lw.plan);
            return st->groups;
        }
        default:
            return 0;
    }
}

void qdb_gpu_agg_release(void* ht) {
    if (!ht) return;
    AggStateDestroy(StateOf(ht));
    std::memset(ht, 0, QDB_HASH_TABLE_SIZE);
}

int64_t qdb_gpu_agg_finish_rowset(const qdb_gpu_program* prog, void* ht, qdb_rowset* out) {
    t_error.clear();
    if (!prog || !ht || !out) {
        SetErr("agg_finish_rowset: bad arguments");
        return -1;
    }
    AggTableState* st = StateOf(ht);
    if (!st) {
        SetErr("agg_finish_rowset before Init");
        return -1;
    }
    const int64_t n = AggFinish(st, prog->agg, prog->flags, out);
    AggStateDestroy(st);
    std::memset(ht, 0, QDB_HASH_TABLE_SIZE);
    return n;
}

void qdb_gpu_filter(const qdb_gpu_program* prog, qdb_rowset* rs, const uint8_t* input_selection) {
    t_error.clear();
    if (!prog || prog->kind != PK_FILTER || !rs || !rs->Selection) {
        SetErr("filter: bad arguments (the caller owns rs->Selection)");
        return;
    }
    cudaStream_t s = CurStream();
    AggPlan plan = prog->expr.plan;
    Staging stg(s);
    qdb_rowset view = *rs;
    view.Selection = const_cast<uint8_t*>(input_selection);
    if (!ResolveColumns(plan, prog->expr.cols, prog->columns.data(), &view, stg)) return;
    const bool dev_out = IsDevicePtr(rs->Selection);
    uint8_t* out = dev_out ? rs->Selection : static_cast<uint8_t*>(DevAlloc(size_t(rs->RowCount), s));
    int* derr = static_cast<int*>(DevAlloc(sizeof(int), s));
    cudaMemsetAsync(derr, 0, sizeof(int), s);
    ExprArgs a;
    a.plan = &plan;
    a.nrows = rs->RowCount;
    a.out_sel = out;
    a.err = derr;
    FilterRows(a, s);
    int herr = 0;
    cudaMemcpyAsync(&herr, derr, sizeof(int), cudaMemcpyDeviceToHost, s);
    if (!dev_out) cudaMemcpyAsync(rs->Selection, out, size_t(rs->RowCount), cudaMemcpyDeviceToHost, s);
    cudaStreamSynchronize(s);
    if (herr) SetErr("filter: device error %d", herr);
    if (!dev_out) DevFree(out, s);
    DevFree(derr, s);
}

void qdb_gpu_project(const qdb_gpu_program* prog, qdb_rowset* in, void** out_buffers, void* arena,
                     const uint8_t* input_selection) {
    (void)arena;
    t_error.clear();
    if (!prog || prog->kind != PK_PROJECT || !in || !out_buffers) {
        SetErr("project: bad arguments");
        return;
    }
    cudaStream_t s = CurStream();
    AggPlan plan = prog->expr.plan;
    Staging stg(s);
    qdb_rowset view = *in;
    view.Selection = const_cast<uint8_t*>(input_selection);
    if (!ResolveColumns(plan, prog->expr.cols, prog->columns.data(), &view, stg)) return;
    const int nout = int(prog->expr.out_types.size());
    ExprArgs a;
    a.plan = &plan;
    a.nrows = in->RowCount;
    a.nout = nout;
    std::vector<void*> dev(nout, nullptr);
    std::vector<bool> staged(nout, false);
    for (int k = 0; k < nout; ++k) {
        a.out_src[k] = uint8_t(prog->expr.value_src[k]);
        a.out_idx[k] = uint8_t(prog->expr.value_idx[k]);
        a.out_type[k] = prog->expr.out_types[k];
        if (IsDevicePtr(out_buffers[k])) {
            dev[k] = out_buffers[k];
        } else {
            dev[k] = DevAlloc(size_t(in->RowCount) * StorageWidth(a.out_type[k]), s);
            staged[k] = true;
        }
        a.out_ptr[k] = dev[k];
    }
    int* derr = static_cast<int*>(DevAlloc(sizeof(int), s));
    cudaMemsetAsync(derr, 0, sizeof(int), s);
    a.err = derr;
    ProjectRows(a, s);
    int herr = 0;
    cudaMemcpyAsync(&herr, derr, sizeof(int), cudaMemcpyDeviceToHost, s);
    for (int k = 0; k < nout; ++k) {
        if (staged[k]) {
            cudaMemcpyAsync(out_buffers[k], dev[k], size_t(in->RowCount) * StorageWidth(a.out_type[k]),
                            cudaMemcpyDeviceToHost, s);
        }
    }
    cudaStreamSynchronize(s);
    if (herr) SetErr("project: device error %d", herr);
    for (int k = 0; k < nout; ++k) {
        if (staged[k]) DevFree(dev[k], s);
    }
    DevFree(derr, s);
}

int64_t qdb_gpu_rf_probe_rowset(const qdb_gpu_program* prog, const qdb_rf_data* data, qdb_rowset* batch,
                                uint8_t* output) {
    t_error.clear();
    if (!prog || prog->kind != PK_HASH || !data || !batch || (batch->RowCount > 0 && !output) ||
        (data->Kind != 1 && data->Kind != 2)) {
        SetErr("rf_probe_rowset: bad arguments (a hash program, and Kind 1 exact or 2 Bloom)");
        return -1;
    }
    if (!IsDevicePtr(output) || !IsDevicePtr(data->Words)) {
        SetErr("rf_probe_rowset: the output and the filter's words must be in device memory");
        return -1;
    }
    if (batch->RowCount == 0) return 0;
    cudaStream_t s = CurStream();
    AggPlan plan = prog->expr.plan;
    Staging stg(s);
    if (!ResolveColumns(plan, prog->expr.cols, prog->columns.data(), batch, stg)) return -1;
    ExprArgs a;
    HashArgs(prog, plan, batch->RowCount, a);
    auto* kept = static_cast<unsigned long long*>(DevAlloc(8, s));
    if (!kept) return -1;
    cudaMemsetAsync(kept, 0, 8, s);
    a.rf_out = output;
    a.rf_words = data->Words;
    a.rf_kind = data->Kind;
    a.rf_nwords = data->WordCount;
    a.rf_kept = kept;
    HashRows(a, s);
    unsigned long long k = 0;
    cudaMemcpyAsync(&k, kept, 8, cudaMemcpyDeviceToHost, s);
    const bool ok = CudaOk(cudaStreamSynchronize(s), "rf_probe_rowset");
    DevFree(kept, s);
    return ok ? int64_t(k) : -1;
}

bool qdb_gpu_hash(const qdb_gpu_program* prog, qdb_rowset* batch, uint64_t* hashes) {
    t_error.clear();
    if (!prog || prog->kind != PK_HASH || !batch || !hashes) {
        SetErr("hash: bad arguments");
        return false;
    }
    cudaStream_t s = CurStream();
    AggPlan plan = prog->expr.plan;
    Staging stg(s);
    if (!ResolveColumns(plan, prog->expr.cols, prog->columns.data(), batch, stg)) return false;
    ExprArgs a;
    HashArgs(prog, plan, batch->RowCount, a);
    const bool dev_out = IsDevicePtr(hashes);
    uint64_t* out = dev_out ? hashes : static_cast<uint64_t*>(DevAlloc(size_t(batch->RowCount) * 8, s));
    if (!dev_out && batch->Selection) {
        cudaMemcpyAsync(out, hashes, size_t(batch->RowCount) * 8, cudaMemcpyHostToDevice, s);
    }
    a.hashes = out;
    HashRows(a, s);
    if (!dev_out) cudaMemcpyAsync(hashes, out, size_t(batch->RowCount) * 8, cudaMemcpyDeviceToHost, s);
    const bool ok = CudaOk(cudaStreamSynchronize(s), "hash");
    if (!dev_out) DevFree(out, s);
    return ok;
}

}  // extern "C"
