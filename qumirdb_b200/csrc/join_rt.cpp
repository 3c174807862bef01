// join_rt.cpp — row join entries of the C ABI: jr_dispatch (Init / Append /
// Build / Probe), jr_materialize and the fused join-aggregate probe.
//
// The caller-owned state buffers keep the engine's layouts where the engine
// reads them (qdb/exec/row_join_exec.h:63-101): arena.Rows (offset 40),
// table.Capacity (8) / Rows (32) / Keys (40), pairs.Count (0).  Word 0 of the
// arena and table buffers holds this library's device state.
#include <algorithm>
#include <climits>
#include <cstring>
#include <memory>

#include "fast.h"
#include "runtime.h"

namespace qdb {

namespace {

constexpr uint32_t kArenaMagic = 0x5144414a;   // 'QDAJ'
constexpr uint32_t kTableMagic = 0x5144544a;   // 'QDTJ'

struct ArenaCol {
    char* data = nullptr;        // device, capacity rows
    uint32_t* valid = nullptr;   // device bitmap (capacity bits), or nullptr
    int width = 0;
    int type = 0;
};

// Build rows in append order: the key columns, then the payload columns.
struct ArenaState {
    uint32_t magic = kArenaMagic;
    cudaStream_t s = nullptr;
    int64_t rows = 0;
    int64_t capacity = 0;
    std::vector<ArenaCol> keys;
    std::vector<ArenaCol> payload;
    bool want_marks = false;       // SEMI / ANTI: one mark byte per row
    uint8_t* marks = nullptr;      // device, capacity bytes, zeroed
    bool null_keys = false;        // the NULL-key arena of an ANTI join
};

struct TableState {
    uint32_t magic = kTableMagic;
    cudaStream_t s = nullptr;
    uint64_t* buckets = nullptr;   // two-slot buckets, 32 bytes each
    int64_t* rows = nullptr;       // arena row per slot
    int64_t slots = 0;             // power of two, >= 2 * rows
    int64_t* special = nullptr;
    unsigned long long* nspecial_d = nullptr;   // device count of special rows
    uint32_t* bloom = nullptr;
    int32_t bloom_words = 0;
    ulonglong2* dense = nullptr;   // direct-address index (see JTableDev)
    int64_t dense_min = 0;
    uint64_t dense_range = 0;
    uint32_t* dense_bits = nullptr;
    int32_t dense_words = 0;
    int32_t dense_shift = 0;
    JTableDev dev() const {
        JTableDev j;
        j.buckets = buckets;
        j.bmask = uint64_t(slots / 2 - 1);
        j.rows = rows;
        j.special_rows = special;
        j.nspecial = nspecial_d;
        j.bloom = bloom;
        j.bloom_words = bloom_words;
        j.dense = dense;
        j.dense_min = dense_min;
        j.dense_range = dense_range;
        j.dense_bits = dense_bits;
        j.dense_words = dense_words;
        j.dense_shift = dense_shift;
        return j;
    }
};

// Blocked Bloom filter size: about 8 bits per key, within a CTA's shared
// memory next to the probe's staging buffers (kMaxBloomWords); tiny tables
// get none.
int32_t BloomWordsFor(int64_t rows) {
    if (rows < 4096) return 0;
    return int32_t(std::min<int64_t>(kMaxBloomWords, std::max<int64_t>(1024, rows / 4)) & ~int64_t(3));
}

constexpr uint32_t kPairMagic = 0x51445050;   // 'QDPP'

// The engine reads only PairBuffer.Count; Data points at this host record of
// the device pairs and of the arena their build rows index.
struct PairState {
    uint32_t magic = kPairMagic;
    int64_t* dev = nullptr;        // (probe row, arena row) pairs
    int64_t cap = 0;
    ArenaState* arena = nullptr;
    ArenaState* arena2 = nullptr;  // NULL-key arena (pairs name its rows -(r + 2))
    cudaStream_t s = nullptr;
};

struct PairBuf {
    int64_t count;
    int64_t capacity;
    PairState* state;
};

ArenaState* ArenaOf(void* arena) {
    auto* a = *static_cast<ArenaState**>(arena);
    return (a && a->magic == kArenaMagic) ? a : nullptr;
}

TableState* TableOf(void* table) {
    auto* t = *static_cast<TableState**>(table);
    return (t && t->magic == kTableMagic) ? t : nullptr;
}

int Width(int type) { return StorageWidth(type); }

bool IsFloat(int t) { return t == QDB_TYPE_F32 || t == QDB_TYPE_F64; }
bool IsSigned(int t) {
    return t != QDB_TYPE_U8 && t != QDB_TYPE_U16 && t != QDB_TYPE_U32 && t != QDB_TYPE_U64 && t != QDB_TYPE_CHAR1;
}

// Packs up to four key columns into one word.  Both sides must agree on the
// key types (the planner casts join keys to a common type).
JoinKeyPlan MakeKeyPlan(const std::vector<qdb_column_type>& bcols, const std::vector<int>& bkeys,
                        const std::vector<qdb_column_type>& pcols, const std::vector<int>& pkeys) {
    JoinKeyPlan k;
    const int n = int(bkeys.size());
    if (n < 1 || n > 4) throw LowerError("row join needs 1..4 key columns");
    k.n = n;
    int shift = 0;
    for (int j = 0; j < n; ++j) {
        const int bt = bcols.at(bkeys[j]).type, pt = pcols.at(pkeys[j]).type;
        if (bt == QDB_TYPE_BOOL || pt == QDB_TYPE_BOOL || bt == QDB_TYPE_DECIMAL128 || pt == QDB_TYPE_DECIMAL128) {
            throw LowerError("boolean and DECIMAL128 join keys are not served");
        }
        if (IsFloat(bt) != IsFloat(pt)) throw LowerError("join keys mix float and integer types");
        if ((bt == QDB_TYPE_DECIMAL64) != (pt == QDB_TYPE_DECIMAL64) ||
            (bt == QDB_TYPE_DECIMAL64 && bcols[bkeys[j]].scale != pcols[pkeys[j]].scale)) {
            throw LowerError("decimal join keys must share a scale");
        }
        k.is_float[j] = IsFloat(bt) ? 1 : 0;
        const int bits = n == 1 ? 64 : std::max(InfoOf(bt).key_bits, InfoOf(pt).key_bits);
        if (n > 1 && InfoOf(bt).key_bits != InfoOf(pt).key_bits) {
            throw LowerError("multi-column join keys must have equal widths on both sides");
        }
        k.bits[j] = uint8_t(bits);
        k.shift[j] = uint8_t(shift);
        shift += bits;
    }
    if (shift > 64) throw LowerError("join key wider than 64 bits is not served");
    k.full64 = (n == 1 && !k.is_float[0]) || shift >= 64 ? 1 : 0;
    return k;
}

bool GrowArena(ArenaState* a, int64_t need) {
    if (need <= a->capacity) return true;
    int64_t cap = std::max<int64_t>(1024, a->capacity);
    while (cap < need) cap *= 2;
    auto grow = [&](ArenaCol& c) -> bool {
        char* d = static_cast<char*>(DevAlloc(size_t(cap) * c.width, a->s));
        if (!d) return false;
        if (c.data) cudaMemcpyAsync(d, c.data, size_t(a->rows) * c.width, cudaMemcpyDeviceToDevice, a->s);
        DevFree(c.data, a->s);
        c.data = d;
        if (c.valid || c.type < 0) {
            uint32_t* v = static_cast<uint32_t*>(DevAlloc(size_t((cap + 31) / 32) * 4, a->s));
            if (!v) return false;
            cudaMemsetAsync(v, 0, size_t((cap + 31) / 32) * 4, a->s);
            if (c.valid) cudaMemcpyAsync(v, c.valid, size_t((a->rows + 31) / 32) * 4, cudaMemcpyDeviceToDevice, a->s);
            DevFree(c.valid, a->s);
            c.valid = v;
            if (c.type < 0) c.type = -c.type;
        }
        return true;
    };
    for (auto& c : a->keys) {
        if (!grow(c)) return false;
    }
    for (auto& c : a->payload) {
        if (!grow(c)) return false;
    }
    if (a->want_marks) {
        auto* m = static_cast<uint8_t*>(DevAlloc(size_t(cap), a->s));
        if (!m) return false;
        cudaMemsetAsync(m, 0, size_t(cap), a->s);
        if (a->marks) cudaMemcpyAsync(m, a->marks, size_t(a->rows), cudaMemcpyDeviceToDevice, a->s);
        DevFree(a->marks, a->s);
        a->marks = m;
    }
    a->capacity = cap;
    return true;
}

void DestroyArena(ArenaState* a) {
    for (auto& c : a->keys) {
        DevFree(c.data, a->s);
        DevFree(c.valid, a->s);
    }
    for (auto& c : a->payload) {
        DevFree(c.data, a->s);
        DevFree(c.valid, a->s);
    }
    DevFree(a->marks, a->s);
    a->magic = 0;
    delete a;
}

void DestroyTable(TableState* t) {
    DevFree(t->dense, t->s);
    DevFree(t->dense_bits, t->s);
    DevFree(t->bloom, t->s);
    DevFree(t->buckets, t->s);
    DevFree(t->rows, t->s);
    DevFree(t->special, t->s);
    DevFree(t->nspecial_d, t->s);
    t->magic = 0;
    delete t;
}

// One Append in two halves, so that a batch of appends waits on the device
// once: Start filters and compacts the batch's rows and queues the read-back
// of their count; Finish (after the stream has drained) grows the arena and
// gathers the rows.
struct AppendJob {
    ArenaState* a = nullptr;
    std::unique_ptr<Staging> stg;
    AggPlan plan;
    int64_t n = 0;
    uint8_t* flags = nullptr;
    int64_t* idx = nullptr;
    unsigned long long* dcount = nullptr;
    void* scratch = nullptr;
    int* derr = nullptr;
    unsigned long long* hcount = nullptr;   // page-locked: count, then error
    void Free() {
        cudaStream_t s = a->s;
        DevFree(flags, s);
        DevFree(idx, s);
        DevFree(dcount, s);
        DevFree(scratch, s);
        DevFree(derr, s);
        flags = nullptr;
        idx = nullptr;
        dcount = nullptr;
        scratch = nullptr;
        derr = nullptr;
    }
};

bool AppendStart(const qdb_gpu_program* prog, ArenaState* a, qdb_rowset* batch, bool null_keys, AppendJob& job,
                 unsigned long long* hcount) {
    const JoinProgram& J = prog->join;
    job.a = a;
    job.n = batch->RowCount;
    job.hcount = hcount;
    hcount[0] = 0;
    hcount[1] = 0;
    if (job.n == 0) return true;
    cudaStream_t s = a->s;
    job.stg.reset(new Staging(s));
    job.plan = J.build_filter.plan;
    if (!ResolveColumns(job.plan, J.build_filter.cols, J.build_columns.data(), batch, *job.stg)) return false;
    const int64_t n = job.n;
    job.flags = static_cast<uint8_t*>(DevAlloc(size_t(n), s));
    job.idx = static_cast<int64_t*>(DevAlloc(size_t(n) * 8, s));
    job.dcount = static_cast<unsigned long long*>(DevAlloc(8, s));
    job.scratch = DevAlloc(CompactScratch(n), s);
    job.derr = static_cast<int*>(DevAlloc(sizeof(int), s));
    if (!job.flags || !job.idx || !job.dcount || !job.scratch || !job.derr) return false;
    cudaMemsetAsync(job.derr, 0, sizeof(int), s);
    ExprArgs ea;
    ea.plan = &job.plan;
    ea.nrows = n;
    ea.out_sel = job.flags;
    ea.err = job.derr;
    ea.n_null_reject = int(J.build_keys.size());
    for (size_t j = 0; j < J.build_keys.size(); ++j) {
        ea.null_reject[j] = uint8_t(J.build_filter.cols.slot_of[J.build_keys[j]]);
    }
    ea.null_keys_only = null_keys ? 1 : 0;
    FilterRows(ea, s);
    CompactFlags(job.flags, n, job.idx, job.dcount, job.scratch, s);
    cudaMemcpyAsync(hcount, job.dcount, 8, cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(hcount + 1, job.derr, sizeof(int), cudaMemcpyDeviceToHost, s);
    return true;
}

bool AppendFinish(const qdb_gpu_program* prog, AppendJob& job) {
    if (job.n == 0) return true;
    const JoinProgram& J = prog->join;
    ArenaState* a = job.a;
    cudaStream_t s = a->s;
    const unsigned long long selected = job.hcount[0];
    const int herr = int(job.hcount[1]);
    bool ok = herr == 0;
    if (!ok) SetErr("row join append: device error %d", herr);
    if (ok && selected > 0) {
        ok = GrowArena(a, a->rows + int64_t(selected));
        auto gather = [&](ArenaCol& c, int input) {
            const ColDesc& cd = job.plan.cols[J.build_filter.cols.slot_of[input]];
            GatherColumn(cd.data, c.width, job.idx, 1, int64_t(selected), c.data + a->rows * c.width, s);
            if (c.valid) GatherValidity(cd.mask, cd.mask_off, job.idx, 1, int64_t(selected), c.valid, a->rows, s);
        };
        for (size_t j = 0; ok && j < J.build_keys.size(); ++j) gather(a->keys[j], J.build_keys[j]);
        for (size_t j = 0; ok && j < J.payload.size(); ++j) gather(a->payload[j], J.payload[j]);
        a->rows += int64_t(selected);
    }
    job.Free();
    return ok;
}

// Append: selected rows that pass the build predicate and have valid keys,
// in input order (GenRowJoinAppendAst, qdb/kernel/join_gen.cpp:2063-2160);
// with null_keys, the rows whose key has a NULL field instead (the
// jr_append_null_keys variant, nullKeys = true).
bool Append(const qdb_gpu_program* prog, ArenaState* a, qdb_rowset* batch, bool null_keys = false) {
    unsigned long long* hc = static_cast<unsigned long long*>(HostOutAlloc(16));
    if (!hc) return false;
    AppendJob job;
    bool ok = AppendStart(prog, a, batch, null_keys, job, hc) && CudaOk(cudaStreamSynchronize(a->s), "row join append");
    if (ok) {
        ok = AppendFinish(prog, job);
    } else if (job.a) {
        job.Free();
    }
    HostOutFree(hc);
    return ok;
}

// A table larger than L2: the arena rows are radix-partitioned by the high
// bits of their home bucket, then inserted partition by partition, so the
// inserts of one pass stay inside one L2-sized slice of the buckets.
bool BuildPartitioned(const ArenaState* a, const JoinBuildArgs& b, int parts, int part_shift, cudaStream_t s) {
    const int64_t n = a->rows;
    auto* counts = static_cast<unsigned long long*>(DevAlloc(size_t(parts) * 8 * 2, s));
    auto* keys = static_cast<uint64_t*>(DevAlloc(size_t(std::max<int64_t>(n, 1)) * 8, s));
    auto* pays = static_cast<int64_t*>(DevAlloc(size_t(std::max<int64_t>(n, 1)) * 8, s));
    auto* rows = static_cast<int64_t*>(DevAlloc(size_t(std::max<int64_t>(n, 1)) * 8, s));
    auto cleanup = [&] {
        DevFree(counts, s);
        DevFree(keys, s);
        DevFree(pays, s);
        DevFree(rows, s);
    };
    if (!counts || !keys || !pays || !rows) {
        cleanup();
        return false;
    }
    unsigned long long* cursor = counts + parts;
    cudaMemsetAsync(counts, 0, size_t(parts) * 8, s);
    JoinPartCountBuild(b, part_shift, parts, counts, s);
    std::vector<unsigned long long> cnt(static_cast<size_t>(parts)), off(static_cast<size_t>(parts));
    cudaMemcpyAsync(cnt.data(), counts, size_t(parts) * 8, cudaMemcpyDeviceToHost, s);
    if (!CudaOk(cudaStreamSynchronize(s), "row join partition count")) {
        cleanup();
        return false;
    }
    unsigned long long run = 0;
    for (int p = 0; p < parts; ++p) {
        off[size_t(p)] = run;
        run += cnt[size_t(p)];
    }
    cudaMemcpyAsync(cursor, off.data(), size_t(parts) * 8, cudaMemcpyHostToDevice, s);
    JoinPartScatterBuild(b, part_shift, parts, cursor, keys, pays, rows, s);
    for (int p = 0; p < parts; ++p) {
        const size_t o = size_t(off[size_t(p)]);
        JoinBuildRows(b, keys + o, pays + o, rows + o, int64_t(cnt[size_t(p)]), s);
    }
    const bool ok = CudaOk(cudaStreamSynchronize(s), "row join partitioned build");
    cleanup();
    return ok;
}

// Entries of the direct-address index at most: 48 MB of entries (so the
// index stays in L2) and eight per build row (plus 64K), so a sparse key set
// keeps the hashed table alone.
constexpr uint64_t kDenseMaxRange = uint64_t(kJoinPartitionBytes) / 16;

// The direct-address index beside the bucket table, for one integer key
// (signed, or unsigned of at most 32 bits) whose build values are unique
// and dense: a probe of it is a subtraction, a bit test in shared memory and
// at most one 16-byte read, with no hashing.  Any duplicate key, a range too
// wide, or the empty marker inside the range leaves the table without it.
// Returns false only on a device failure.
bool BuildDense(const JoinProgram& J, const ArenaState* a, const JoinBuildArgs& b, TableState* t) {
    if (J.build_jk.n != 1 || J.build_jk.is_float[0] || a->rows < 4096) return true;
    const int ty = J.build_columns[J.build_keys[0]].type;
    if (ty == QDB_TYPE_U64) return true;
    auto* buf = static_cast<long long*>(DevAlloc(24, t->s));
    if (!buf) return false;
    const long long init[3] = {LLONG_MAX, LLONG_MIN, 0};
    cudaMemcpyAsync(buf, init, 24, cudaMemcpyHostToDevice, t->s);
    JoinKeyRange(b, buf, t->s);
    long long mm[3] = {0, 0, 0};
    cudaMemcpyAsync(mm, buf, 24, cudaMemcpyDeviceToHost, t->s);
    if (!CudaOk(cudaStreamSynchronize(t->s), "row join key range")) {
        DevFree(buf, t->s);
        return false;
    }
    const long long kmin = mm[0], kmax = mm[1];
    const uint64_t range = kmin <= kmax ? uint64_t(kmax) - uint64_t(kmin) + 1 : 0;
    const uint64_t limit = std::min<uint64_t>(kDenseMaxRange, uint64_t(a->rows) * 8 + (uint64_t(1) << 16));
    const bool marker_inside = kmin <= -1 && kmax >= -1;   // kEmptyKey as int64
    if (range == 0 || range > limit || marker_inside) {
        DevFree(buf, t->s);
        return true;
    }
    int32_t shift = 0;
    while ((((range - 1) >> shift) + 1) > uint64_t(kMaxBloomWords) * 32 - 96) ++shift;
    // Bitmap words, a multiple of four (the probe copies it in 16-byte loads).
    const int32_t words = int32_t(((((range - 1) >> shift) + 32) / 32 + 3) & ~uint64_t(3));
    t->dense = static_cast<ulonglong2*>(DevAlloc(size_t(range) * 16, t->s));
    t->dense_bits = static_cast<uint32_t*>(DevAlloc(size_t(words) * 4, t->s));
    if (!t->dense || !t->dense_bits) {
        DevFree(buf, t->s);
        return false;
    }
    auto* dup = reinterpret_cast<unsigned long long*>(buf + 2);
    JoinDenseBuild(b, t->dense, kmin, range, t->dense_bits, words, shift, dup, t->s);
    unsigned long long ndup = 0;
    cudaMemcpyAsync(&ndup, dup, 8, cudaMemcpyDeviceToHost, t->s);
    const bool ok = CudaOk(cudaStreamSynchronize(t->s), "row join direct index");
    DevFree(buf, t->s);
    if (!ok) return false;
    if (ndup) {
        DevFree(t->dense, t->s);
        DevFree(t->dense_bits, t->s);
        t->dense = nullptr;
        t->dense_bits = nullptr;
        return true;
    }
    t->dense_min = kmin;
    t->dense_range = range;
    t->dense_words = words;
    t->dense_shift = shift;
    return true;
}

// Sizes and allocates the bucket table of arena `a` (not yet initialised)
// and fills its build arguments; nullptr on an allocation failure.
TableState* NewTable(const JoinProgram& J, const ArenaState* a, JoinBuildArgs& b) {
    auto* t = new TableState();
    t->s = a->s;
    // Slots: a power of two >= 2x the rows; >= 4x while the buckets stay
    // within 32 MB, so that few probes find their first bucket full.
    int64_t cap = 1024;
    while (cap < a->rows * 2) cap *= 2;
    if (cap * 2 * 16 <= (int64_t(32) << 20)) cap *= 2;
    t->slots = cap;
    t->buckets = static_cast<uint64_t*>(DevAlloc(size_t(cap / 2) * 32, t->s));
    t->rows = static_cast<int64_t*>(DevAlloc(size_t(cap) * 8, t->s));
    t->special = static_cast<int64_t*>(DevAlloc(size_t(std::max<int64_t>(a->rows, 1)) * 16, t->s));
    t->nspecial_d = static_cast<unsigned long long*>(DevAlloc(8, t->s));
    if (!t->buckets || !t->rows || !t->special || !t->nspecial_d) {
        DestroyTable(t);
        return nullptr;
    }
    cudaMemsetAsync(t->nspecial_d, 0, 8, t->s);
    std::memset(&b, 0, sizeof(b));
    for (size_t j = 0; j < J.build_keys.size(); ++j) {
        const int ty = J.build_columns[J.build_keys[j]].type;
        b.key_data[j] = a->keys[j].data;
        b.key_mask[j] = nullptr;   // the arena only holds rows with valid keys
        b.key_width[j] = uint8_t(Width(ty));
        b.key_signed[j] = IsSigned(ty) ? 1 : 0;
    }
    b.jkey = J.build_jk;
    b.nrows = a->rows;
    // The first 8-byte payload column rides in the bucket: a probe reads one
    // 32-byte sector for the keys and those values.
    b.pay0 = (!a->payload.empty() && a->payload[0].width == 8) ? reinterpret_cast<const int64_t*>(a->payload[0].data)
                                                                : nullptr;
    b.buckets = t->buckets;
    b.bmask = uint64_t(cap / 2 - 1);
    b.rows = t->rows;
    b.special_rows = t->special;
    b.nspecial = t->nspecial_d;
    b.row_base = 0;
    return t;
}

void PublishTable(void* table, TableState* t, int64_t rows) {
    *static_cast<TableState**>(table) = t;
    int64_t* w = static_cast<int64_t*>(table);
    w[1] = t->slots;   // Capacity
    w[4] = rows;       // Rows
    w[5] = rows;       // Keys (rows indexed)
}

bool Build(const qdb_gpu_program* prog, ArenaState* a, void* table) {
    const JoinProgram& J = prog->join;
    TableState* old = TableOf(table);
    if (old) DestroyTable(old);
    JoinBuildArgs b;
    TableState* t = NewTable(J, a, b);
    if (!t) return false;
    const int64_t cap = t->slots;
    JoinInitTable(t->buckets, cap / 2, t->s);
    int part_shift = 0;
    const int parts = JoinPartsFor(cap / 2, part_shift);
    if (parts == 1) {
        JoinBuild(b, t->s);
    } else if (!BuildPartitioned(a, b, parts, part_shift, t->s)) {
        DestroyTable(t);
        return false;
    }
    t->bloom_words = BloomWordsFor(a->rows);
    if (t->bloom_words > 0) {
        t->bloom = static_cast<uint32_t*>(DevAlloc(size_t(t->bloom_words) * 4, t->s));
        if (!t->bloom) {
            DestroyTable(t);
            return false;
        }
        JoinBuildBloom(t->dev(), t->bloom, t->bloom_words, t->s);
    }
    if (!BuildDense(J, a, b, t)) {
        DestroyTable(t);
        return false;
    }
    if (!CudaOk(cudaGetLastError(), "row join build")) {
        DestroyTable(t);
        return false;
    }
    PublishTable(table, t, a->rows);
    return true;
}

// Resolves the probe key columns of a batch into JoinProbeArgs.
bool ProbeKeyArgs(const JoinProgram& J, qdb_rowset* batch, Staging& stg, JoinProbeArgs& p) {
    const int64_t n = batch->RowCount;
    for (size_t j = 0; j < J.probe_keys.size(); ++j) {
        const int input = J.probe_keys[j];
        if (input >= batch->ColumnCount) {
            SetErr("probe batch has too few columns");
            return false;
        }
        const int ty = J.probe_columns[input].type;
        const qdb_column& c = batch->Columns[input];
        p.key_data[j] = static_cast<const char*>(stg.Device(c.Data, size_t(n) * Width(ty)));
        p.key_width[j] = uint8_t(Width(ty));
        p.key_signed[j] = IsSigned(ty) ? 1 : 0;
        if (c.Mask) {
            p.key_mask[j] = static_cast<const uint8_t*>(stg.Device(c.Mask, size_t((c.MaskBitOffset + n + 7) / 8)));
            p.key_mask_off[j] = c.MaskBitOffset;
        }
    }
    p.selection = batch->Selection ? static_cast<const uint8_t*>(stg.Device(batch->Selection, size_t(n))) : nullptr;
    return true;
}

PairState* PairsOf(PairBuf* pairs, cudaStream_t s) {
    if (!pairs->state || pairs->state->magic != kPairMagic) {
        pairs->state = new PairState();
        pairs->state->s = s;
    }
    return pairs->state;
}

// Room for `need` pairs; the first `keep` are kept.
bool ReservePairs(PairState* ps, int64_t need, int64_t keep, cudaStream_t s) {
    if (ps->cap >= need && ps->dev) return true;
    const int64_t cap = std::max<int64_t>(need, std::max<int64_t>(1024, ps->cap * 2));
    auto* d = static_cast<int64_t*>(DevAlloc(size_t(cap) * 16, s));
    if (!d) return false;
    if (keep > 0) cudaMemcpyAsync(d, ps->dev, size_t(keep) * 16, cudaMemcpyDeviceToDevice, s);
    DevFree(ps->dev, s);
    ps->dev = d;
    ps->cap = cap;
    return true;
}

// Compacts flags[0, n) into ascending indices; returns their count, < 0 on
// a device failure.  idx has room for n entries.
int64_t CompactCount(const uint8_t* flags, int64_t n, int64_t* idx, cudaStream_t s) {
    if (n == 0) return 0;
    auto* dcount = static_cast<unsigned long long*>(DevAlloc(8, s));
    void* scratch = DevAlloc(CompactScratch(n), s);
    if (!dcount || !scratch) {
        DevFree(dcount, s);
        DevFree(scratch, s);
        return -1;
    }
    CompactFlags(flags, n, idx, dcount, scratch, s);
    unsigned long long k = 0;
    cudaMemcpyAsync(&k, dcount, 8, cudaMemcpyDeviceToHost, s);
    const bool ok = CudaOk(cudaStreamSynchronize(s), "row join compaction");
    DevFree(dcount, s);
    DevFree(scratch, s);
    return ok ? int64_t(k) : -1;
}

bool Probe(const qdb_gpu_program* prog, ArenaState* a, TableState* t, PairBuf* pairs, qdb_rowset* batch) {
    const JoinProgram& J = prog->join;
    const int64_t n = batch->RowCount;
    cudaStream_t s = a->s;
    Staging stg(s);
    JoinProbeArgs p;
    std::memset(&p, 0, sizeof(p));
    if (!ProbeKeyArgs(J, batch, stg, p)) return false;
    p.jkey = J.probe_jk;
    p.jt = t->dev();
    p.nrows = n;
    PairState* ps = PairsOf(pairs, s);
    ps->arena = a;
    if (J.marks_build) {
        // SEMI / ANTI: mark the matched build rows; no pairs (jt_probe_and_mark).
        JoinMarkProbe(p, a->marks, s);
        pairs->count = 0;
        pairs->capacity = ps->cap;
        return CudaOk(cudaStreamSynchronize(s), "row join mark probe");
    }
    // An outer join pads its NULL-key rows first, in row order, as the
    // collect pass of jr_probe_batch does (join_gen.cpp:2206-2230).
    int64_t nnull = 0;
    int64_t* null_idx = nullptr;
    if (J.emit_unmatched && n > 0) {
        auto* flags = static_cast<uint8_t*>(DevAlloc(size_t(n), s));
        null_idx = static_cast<int64_t*>(DevAlloc(size_t(n) * 8, s));
        if (!flags || !null_idx) {
            DevFree(flags, s);
            DevFree(null_idx, s);
            return false;
        }
        JoinNullKeyFlags(p, flags, s);
        nnull = CompactCount(flags, n, null_idx, s);
        DevFree(flags, s);
        if (nnull < 0) {
            DevFree(null_idx, s);
            return false;
        }
        p.emit_unmatched = 1;
    }
    // Count pass, scan of the chunk totals (the last entry becomes the
    // total), then the write pass into a buffer of exactly that size.
    const int64_t nch = JoinPairChunks(n);
    auto* counts = static_cast<uint32_t*>(DevAlloc(size_t(std::max<int64_t>(n, 1)) * 4, s));
    auto* off = static_cast<unsigned long long*>(DevAlloc(size_t(nch + 1) * 8, s));
    auto free_scratch = [&]() {
        DevFree(counts, s);
        DevFree(off, s);
        DevFree(null_idx, s);
    };
    auto fail = [&]() {
        free_scratch();
        return false;
    };
    if (!counts || !off) return fail();
    cudaMemsetAsync(off, 0, size_t(nch + 1) * 8, s);
    JoinProbeCount(p, counts, off, s);
    ExclusiveScanU64(off, nch + 1, s);
    unsigned long long matched = 0;
    cudaMemcpyAsync(&matched, off + nch, 8, cudaMemcpyDeviceToHost, s);
    if (!CudaOk(cudaStreamSynchronize(s), "row join probe count")) return fail();
    const int64_t total = nnull + int64_t(matched);
    if (!ReservePairs(ps, total, 0, s)) return fail();
    JoinWritePairs(null_idx, nnull, ps->dev, 0, s);
    p.pairs = ps->dev;
    p.pair_cap = ps->cap;
    p.pair_base = nnull;
    JoinProbeWrite(p, counts, off, s);
    free_scratch();
    pairs->count = total;
    pairs->capacity = ps->cap;
    return CudaOk(cudaStreamSynchronize(s), "row join probe");
}

// jr_emit_by_mark (qdb/kernel/join/join_rows.oz:199-224): appends (NULL,
// build row) for every arena row whose mark is `marked`, in build order.  The
// NULL-key arena of an ANTI join has no marks: all its rows are emitted.
bool EmitByMark(const JoinProgram& J, ArenaState* a, PairBuf* pairs) {
    cudaStream_t s = a->s;
    PairState* ps = PairsOf(pairs, s);
    const bool second = a->null_keys;
    if (second) {
        ps->arena2 = a;
    } else {
        ps->arena = a;
    }
    const int64_t have = pairs->count;
    const int64_t n = a->rows;
    if (n == 0) return true;
    auto* flags = static_cast<uint8_t*>(DevAlloc(size_t(n), s));
    auto* idx = static_cast<int64_t*>(DevAlloc(size_t(n) * 8, s));
    if (!flags || !idx) {
        DevFree(flags, s);
        DevFree(idx, s);
        return false;
    }
    const bool semi = J.join_type == QDB_JOIN_LEFT_SEMI;
    JoinMarkFlags(second ? nullptr : a->marks, n, semi ? 1 : 0, flags, s);
    const int64_t k = CompactCount(flags, n, idx, s);
    bool ok = k >= 0 && ReservePairs(ps, have + k, have, s);
    if (ok) {
        JoinWritePairs(idx, k, ps->dev + 2 * have, second ? 2 : 1, s);
        pairs->count = have + k;
        pairs->capacity = ps->cap;
        ok = CudaOk(cudaStreamSynchronize(s), "row join emit by mark");
    }
    DevFree(flags, s);
    DevFree(idx, s);
    return ok;
}

}  // namespace

}  // namespace qdb

using namespace qdb;

extern "C" {

qdb_gpu_program* qdb_gpu_compile_row_join(const qdb_row_join_spec* spec, char* err, size_t err_len) {
    try {
        // CompileRowJoin (qdb/kernel/compiler.cpp:3134-3148): an outer join
        // streams its preserved side, so it builds the other one; a SEMI/ANTI
        // join builds its left side and marks the rows it matches.
        const int jt = spec->join_type;
        const bool streams_preserved = spec->build_is_left ? jt == QDB_JOIN_RIGHT : jt == QDB_JOIN_LEFT;
        const bool marks_build = spec->build_is_left && (jt == QDB_JOIN_LEFT_SEMI || jt == QDB_JOIN_LEFT_ANTI);
        if (jt != QDB_JOIN_INNER && !streams_preserved && !marks_build) {
            throw LowerError("only inner joins, outer joins that build their null-supplying side and "
                             "semi/anti joins that build their left side are served");
        }
        if (marks_build) {
            for (int k = 0; k < spec->n_out; ++k) {
                if (spec->out_side[k] != 1) throw LowerError("a SEMI/ANTI join outputs build columns only");
            }
        }
        auto* p = new qdb_gpu_program();
        p->kind = PK_JOIN;
        p->flags = spec->flags;
        JoinProgram& J = p->join;
        J.join_type = jt;
        J.emit_unmatched = streams_preserved;
        J.marks_build = marks_build;
        J.keeps_null_keys = marks_build && jt == QDB_JOIN_LEFT_ANTI;
        J.build_is_left = spec->build_is_left;
        J.build_columns.assign(spec->build_columns, spec->build_columns + spec->n_build_columns);
        J.probe_columns.assign(spec->probe_columns, spec->probe_columns + spec->n_probe_columns);
        J.build_keys.assign(spec->build_keys, spec->build_keys + spec->n_keys);
        J.probe_keys.assign(spec->probe_keys, spec->probe_keys + spec->n_keys);
        J.payload.assign(spec->build_payload, spec->build_payload + spec->n_payload);
        J.out_side.assign(spec->out_side, spec->out_side + spec->n_out);
        J.out_column.assign(spec->out_column, spec->out_column + spec->n_out);
        for (int c : J.build_keys) {
            if (c < 0 || c >= spec->n_build_columns) throw LowerError("build key column out of range");
        }
        for (int c : J.probe_keys) {
            if (c < 0 || c >= spec->n_probe_columns) throw LowerError("probe key column out of range");
        }
        for (int c : J.payload) {
            if (c < 0 || c >= spec->n_build_columns) throw LowerError("payload column out of range");
        }
        for (size_t k = 0; k < J.out_side.size(); ++k) {
            const int lim = J.out_side[k] == 0 ? spec->n_probe_columns : spec->n_payload;
            if (J.out_column[k] < 0 || J.out_column[k] >= lim) throw LowerError("output column out of range");
        }
        J.build_jk = MakeKeyPlan(J.build_columns, J.build_keys, J.probe_columns, J.probe_keys);
        J.probe_jk = J.build_jk;
        // The build predicate program also maps every key and payload column
        // so that Append can gather them.
        std::vector<qdb_expr> nodes(spec->build_nodes, spec->build_nodes + spec->n_build_nodes);
        int predicate = spec->build_filter;
        if (predicate < 0) {
            // A constant-true predicate: 1 = 1.
            qdb_expr one;
            std::memset(&one, 0, sizeof(one));
            one.op = QDB_EXPR_CONST;
            one.type = QDB_TYPE_I64;
            one.imm_lo = 1;
            nodes.push_back(one);
            qdb_expr eq;
            std::memset(&eq, 0, sizeof(eq));
            eq.op = QDB_EXPR_EQ;
            eq.type = QDB_TYPE_BOOL;
            eq.args[0] = int(nodes.size()) - 1;
            eq.args[1] = int(nodes.size()) - 1;
            nodes.push_back(eq);
            predicate = int(nodes.size()) - 1;
        }
        J.build_filter = LowerFilter(spec->n_build_columns, spec->build_columns, int(nodes.size()), nodes.data(),
                                     predicate);
        J.has_build_filter = spec->build_filter >= 0;
        // Map key and payload columns into the filter plan's slots.
        {
            std::vector<int> need(J.build_keys);
            need.insert(need.end(), J.payload.begin(), J.payload.end());
            for (int c : need) {
                if (J.build_filter.cols.slot_of[c] >= 0) continue;
                const int slot = int(J.build_filter.cols.input_of.size());
                if (slot >= kMaxCols) throw LowerError("too many build columns");
                J.build_filter.cols.slot_of[c] = slot;
                J.build_filter.cols.input_of.push_back(c);
                ColDesc& cd = J.build_filter.plan.cols[slot];
                std::memset(&cd, 0, sizeof(cd));
                const TypeInfo ti = InfoOf(J.build_columns[c].type);
                cd.width = ti.width;
                cd.kind = ti.load;
                cd.nullable = J.build_columns[c].nullable ? 1 : 0;
                cd.scale = J.build_columns[c].type == QDB_TYPE_DECIMAL64 || J.build_columns[c].type == QDB_TYPE_DECIMAL128
                               ? J.build_columns[c].scale : 0;
                J.build_filter.plan.ncols = slot + 1;
            }
        }
        return p;
    } catch (const std::exception& e) {
        if (err && err_len) std::snprintf(err, err_len, "%s", e.what());
        t_error = e.what();
        return nullptr;
    }
}

qdb_gpu_program* qdb_gpu_compile_join_aggregate(const qdb_row_join_spec* join, const qdb_aggregate_spec* agg,
                                                char* err, size_t err_len) {
    qdb_gpu_program* p = qdb_gpu_compile_row_join(join, err, err_len);
    if (!p) return nullptr;
    try {
        if (join->join_type != QDB_JOIN_INNER) throw LowerError("a fused join-aggregate is an inner join");
        if (agg->n_columns != join->n_probe_columns + join->n_payload) {
            throw LowerError("aggregate input must be the probe columns followed by the payload columns");
        }
        p->kind = PK_JOIN_AGG;
        p->flags = agg->flags;
        p->expected_groups = agg->expected_groups;
        p->columns.assign(agg->columns, agg->columns + agg->n_columns);
        std::vector<int> first(join->probe_keys, join->probe_keys + join->n_keys);
        p->agg = LowerAggregate(*agg, join->n_probe_columns, first);
        p->agg.plan.key_words = std::max(1, p->agg.plan.key_words);
        p->join.agg_jk = p->join.probe_jk;
        for (int j = 0; j < join->n_keys; ++j) p->join.agg_jk.col[j] = uint8_t(p->agg.cols.slot_of[join->probe_keys[j]]);
        return p;
    } catch (const std::exception& e) {
        if (err && err_len) std::snprintf(err, err_len, "%s", e.what());
        t_error = e.what();
        delete p;
        return nullptr;
    }
}

bool qdb_gpu_jr_dispatch(const qdb_gpu_program* prog, void* arena, void* table, void* scratch, void* pairs,
                         qdb_rowset* batch, int64_t op) {
    (void)scratch;
    t_error.clear();
    if (!prog || (prog->kind != PK_JOIN && prog->kind != PK_JOIN_AGG) || !arena) {
        SetErr("jr_dispatch: not a row join program");
        return false;
    }
    const JoinProgram& J = prog->join;
    switch (op) {
        case QDB_JR_OP_INIT: {
            if (ArenaOf(arena)) DestroyArena(ArenaOf(arena));
            auto* a = new ArenaState();
            a->s = CurStream();
            for (int c : J.build_keys) {
                ArenaCol col;
                col.type = J.build_columns[c].type;
                col.width = Width(col.type);
                a->keys.push_back(col);
            }
            for (int c : J.payload) {
                ArenaCol col;
                col.type = J.build_columns[c].nullable ? -J.build_columns[c].type : J.build_columns[c].type;
                col.width = Width(J.build_columns[c].type);
                a->payload.push_back(col);
            }
            a->want_marks = J.marks_build;
            *static_cast<ArenaState**>(arena) = a;
            static_cast<int64_t*>(arena)[5] = 0;
            return GrowArena(a, 1024);
        }
        case QDB_JR_OP_APPEND_NULL_KEYS: {
            ArenaState* a = ArenaOf(arena);
            if (!J.keeps_null_keys) {
                SetErr("jr_dispatch(AppendNullKeys) is only served for LEFT_ANTI joins");
                return false;
            }
            if (!a || !batch) {
                SetErr("jr_dispatch(AppendNullKeys) before Init");
                return false;
            }
            a->null_keys = true;
            if (!Append(prog, a, batch, true)) return false;
            static_cast<int64_t*>(arena)[5] = a->rows;
            return true;
        }
        case QDB_JR_OP_EMIT_BY_MARK: {
            ArenaState* a = ArenaOf(arena);
            if (!J.marks_build) {
                SetErr("jr_dispatch(EmitByMark) is only served for LEFT_SEMI / LEFT_ANTI joins");
                return false;
            }
            if (!a || !pairs) {
                SetErr("jr_dispatch(EmitByMark) before Init");
                return false;
            }
            return EmitByMark(J, a, static_cast<PairBuf*>(pairs));
        }
        case QDB_JR_OP_APPEND: {
            ArenaState* a = ArenaOf(arena);
            if (!a || !batch) {
                SetErr("jr_dispatch(Append) before Init");
                return false;
            }
            if (!Append(prog, a, batch)) return false;
            static_cast<int64_t*>(arena)[5] = a->rows;
            return true;
        }
        case QDB_JR_OP_BUILD: {
            ArenaState* a = ArenaOf(arena);
            if (!a || !table) {
                SetErr("jr_dispatch(Build) before Init");
                return false;
            }
            return Build(prog, a, table);
        }
        case QDB_JR_OP_PROBE: {
            ArenaState* a = ArenaOf(arena);
            TableState* t = table ? TableOf(table) : nullptr;
            if (!a || !t || !pairs || !batch) {
                SetErr("jr_dispatch(Probe) before Build");
                return false;
            }
            return Probe(prog, a, t, static_cast<PairBuf*>(pairs), batch);
        }
        default:
            SetErr("jr_dispatch: op %lld is not served", (long long)op);
            return false;
    }
}

void qdb_gpu_jr_release(void* arena, void* table, void* scratch, void* pairs) {
    (void)scratch;
    if (pairs) {
        auto* pb = static_cast<PairBuf*>(pairs);
        PairState* ps = pb->state;
        if (ps && ps->magic == kPairMagic) {
            DevFree(ps->dev, ps->s);
            ps->magic = 0;
            delete ps;
        }
        std::memset(pairs, 0, QDB_PAIR_BUFFER_SIZE);
    }
    if (table) {
        if (TableState* t = TableOf(table)) DestroyTable(t);
        std::memset(table, 0, QDB_ROW_TABLE_SIZE);
    }
    if (arena) {
        if (ArenaState* a = ArenaOf(arena)) DestroyArena(a);
        std::memset(arena, 0, QDB_ROW_ARENA_SIZE);
    }
}

int64_t qdb_gpu_jr_materialize(const qdb_gpu_program* prog, void* pairs_v, qdb_rowset* stream, int64_t start,
                               int64_t limit, qdb_rowset* out) {
    t_error.clear();
    if (!prog || !pairs_v || !out || (prog->kind != PK_JOIN && prog->kind != PK_JOIN_AGG)) {
        SetErr("jr_materialize: bad arguments");
        return -1;
    }
    auto* pairs = static_cast<PairBuf*>(pairs_v);
    const JoinProgram& J = prog->join;
    const int64_t n = std::max<int64_t>(0, std::min(limit, pairs->count - start));
    if (n == 0) return 0;
    cudaStream_t s = CurStream();
    PairState* ps = pairs->state;
    const bool probe_cols = std::find(J.out_side.begin(), J.out_side.end(), 0) != J.out_side.end();
    if (!ps || ps->magic != kPairMagic || (!ps->arena && !ps->arena2) || (probe_cols && !stream)) {
        SetErr("jr_materialize: the pair buffer holds no probe result");
        return -1;
    }
    ArenaState* a = ps->arena ? ps->arena : ps->arena2;
    ArenaState* a2 = ps->arena2;
    Staging stg(s);
    std::vector<int> types;
    for (size_t k = 0; k < J.out_side.size(); ++k) {
        types.push_back(J.out_side[k] == 0 ? J.probe_columns[J.out_column[k]].type
                                           : J.build_columns[J.payload[J.out_column[k]]].type);
    }
    std::vector<AggOutputCol> cols;
    OutBlock blk;
    if (!AllocOutputCols(types, n, true, cols, s, &blk)) {
        SetErr("jr_materialize: allocation failed");
        return -1;
    }
    const int64_t* base = ps->dev + 2 * start;
    for (size_t k = 0; k < J.out_side.size(); ++k) {
        const int w = Width(types[k]);
        if (J.out_side[k] == 0) {
            const qdb_column& c = stream->Columns[J.out_column[k]];
            const char* d = static_cast<const char*>(stg.Device(c.Data, size_t(stream->RowCount) * w));
            GatherColumn(d, w, base, 2, n, cols[k].data, s);
            const uint8_t* m = c.Mask ? static_cast<const uint8_t*>(stg.Device(
                                            c.Mask, size_t((c.MaskBitOffset + stream->RowCount + 7) / 8)))
                                      : nullptr;
            GatherValidity(m, c.MaskBitOffset, base, 2, n, cols[k].valid, 0, s);
        } else {
            // Build row -1 is an outer join's NULL row; -(r + 2) row r of the
            // NULL-key arena.
            const ArenaCol& ac = a->payload[J.out_column[k]];
            const ArenaCol* ac2 = a2 ? &a2->payload[J.out_column[k]] : nullptr;
            GatherColumn(ac.data, w, base + 1, 2, n, cols[k].data, s, ac2 ? ac2->data : nullptr);
            GatherValidity(reinterpret_cast<const uint8_t*>(ac.valid), 0, base + 1, 2, n, cols[k].valid, 0, s,
                           ac2 != nullptr, ac2 ? reinterpret_cast<const uint8_t*>(ac2->valid) : nullptr);
        }
    }
    if (!EmitRowset(cols, types, n, (prog->flags & QDB_OUT_DEVICE) != 0, s, out, &blk)) return -1;
    return n;
}

int64_t qdb_gpu_join_aggregate_probe(const qdb_gpu_program* prog, void* arena, void* table, void* ht,
                                     qdb_rowset* batch) {
    t_error.clear();
    if (!prog || prog->kind != PK_JOIN_AGG || !arena || !table || !ht || !batch) {
        SetErr("join_aggregate_probe: bad arguments");
        return -1;
    }
    ArenaState* a = ArenaOf(arena);
    TableState* t = TableOf(table);
    AggTableState* st = AggStateOf(ht);
    if (!a || !t || !st) {
        SetErr("join_aggregate_probe: arena, table and aggregate state must be initialised and built");
        return -1;
    }
    const JoinProgram& J = prog->join;
    AggPlan plan = prog->agg.plan;
    Staging stg(CurStream());
    if (!ResolveColumns(plan, prog->agg.cols, prog->columns.data(), batch, stg)) return -1;
    const int np = int(J.probe_columns.size());
    for (int slot = 0; slot < plan.ncols; ++slot) {
        ColDesc& cd = plan.cols[slot];
        if (!cd.build) continue;
        const ArenaCol& ac = a->payload[prog->agg.cols.input_of[slot] - np];
        cd.data = ac.data;
        cd.mask = reinterpret_cast<const uint8_t*>(ac.valid);
        cd.mask_off = 0;
        cd.bit_off = 0;
    }
    // The slot of the first payload column reads the entry's payload word.
    int inline_slot = -1;
    if (!J.payload.empty() && a->payload[0].width == 8) {
        const int s0 = prog->agg.cols.slot_of[np];
        if (s0 >= 0 && (plan.cols[s0].kind == LK_SIGNED || plan.cols[s0].kind == LK_F64)) inline_slot = s0;
    }
    const int64_t before = AggStateMatched(st);
    const JTableDev jt = t->dev();
    JoinSumShape shape;
    if (MatchJoinSum(plan, J.agg_jk, inline_slot, shape)) {
        // Typed fast kernel for a keyless SUM / COUNT over 8-byte columns.
        shape.selection = nullptr;
        if (!AggRunJoinSum(st, shape, jt, batch->RowCount)) return -1;
    } else if (!AggRun(st, plan, batch->RowCount, &J.agg_jk, &jt, inline_slot)) {
        return -1;
    }
    AggMirrorHeader(ht, st, prog->agg.plan);
    return AggStateMatched(st) - before;
}

}  // extern "C"

namespace qdb {

namespace {

// Rows per work item of the batched launches: enough items to keep every
// warp of the persistent probe busy on a partitioned 120M-row probe.
constexpr int64_t kBatchItemRows = 16384;

void AddItems(std::vector<JoinBatchItem>& items, int32_t join, int64_t n) {
    for (int64_t lo = 0; lo < n; lo += kBatchItemRows) {
        JoinBatchItem it;
        it.join = join;
        it.pad = 0;
        it.lo = lo;
        it.hi = std::min(n, lo + kBatchItemRows);
        items.push_back(it);
    }
}

// Device copy of a host vector on stream s (freed by the caller).
template <class T>
T* ToDevice(const std::vector<T>& v, cudaStream_t s) {
    auto* d = static_cast<T*>(DevAlloc(std::max<size_t>(v.size(), 1) * sizeof(T), s));
    if (d && !v.empty()) cudaMemcpyAsync(d, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, s);
    return d;
}

// The fused join-aggregate plan of one probe batch (as
// qdb_gpu_join_aggregate_probe resolves it) and its join-sum shape; false
// when it has none (then `plan` is still resolved).
bool ResolveJoinSum(const qdb_gpu_program* prog, const ArenaState* a, qdb_rowset* batch, Staging& stg,
                    AggPlan& plan, int& inline_slot, JoinSumShape& shape, bool& is_sum) {
    const JoinProgram& J = prog->join;
    plan = prog->agg.plan;
    if (!ResolveColumns(plan, prog->agg.cols, prog->columns.data(), batch, stg)) return false;
    const int np = int(J.probe_columns.size());
    for (int slot = 0; slot < plan.ncols; ++slot) {
        ColDesc& cd = plan.cols[slot];
        if (!cd.build) continue;
        const ArenaCol& ac = a->payload[prog->agg.cols.input_of[slot] - np];
        cd.data = ac.data;
        cd.mask = reinterpret_cast<const uint8_t*>(ac.valid);
        cd.mask_off = 0;
        cd.bit_off = 0;
    }
    inline_slot = -1;
    if (!J.payload.empty() && a->payload[0].width == 8) {
        const int s0 = prog->agg.cols.slot_of[np];
        if (s0 >= 0 && (plan.cols[s0].kind == LK_SIGNED || plan.cols[s0].kind == LK_F64)) inline_slot = s0;
    }
    std::memset(&shape, 0, sizeof(shape));
    is_sum = MatchJoinSum(plan, J.agg_jk, inline_slot, shape);
    return true;
}

}  // namespace

}  // namespace qdb

extern "C" {

bool qdb_gpu_jr_build_batch(const qdb_gpu_program* prog, void* const* arenas, void* const* tables, int64_t n) {
    t_error.clear();
    if (!prog || (prog->kind != PK_JOIN && prog->kind != PK_JOIN_AGG) || n < 0 || (n > 0 && (!arenas || !tables))) {
        SetErr("jr_build_batch: bad arguments");
        return false;
    }
    const JoinProgram& J = prog->join;
    cudaStream_t s = CurStream();
    std::vector<JoinBuildArgs> args;
    std::vector<JoinBatchItem> init_items, build_items;
    std::vector<std::pair<TableState*, int64_t>> made;   // table, index
    std::vector<cudaStream_t> streams;
    for (int64_t i = 0; i < n; ++i) {
        ArenaState* a = ArenaOf(arenas[i]);
        if (!a || !tables[i]) {
            SetErr("jr_build_batch: state %lld is not initialised", (long long)i);
            return false;
        }
        if (TableState* old = TableOf(tables[i])) DestroyTable(old);
        int64_t cap = 1024;   // NewTable's slot count
        while (cap < a->rows * 2) cap *= 2;
        if (cap * 2 * 16 <= (int64_t(32) << 20)) cap *= 2;
        int part_shift = 0;
        if (JoinPartsFor(cap / 2, part_shift) > 1) {   // a table larger than L2 takes the partitioned build
            if (!Build(prog, a, tables[i])) return false;
            continue;
        }
        JoinBuildArgs b;
        TableState* t = NewTable(J, a, b);
        if (!t) return false;
        if (std::find(streams.begin(), streams.end(), t->s) == streams.end()) streams.push_back(t->s);
        AddItems(init_items, int32_t(args.size()), t->slots / 2);
        AddItems(build_items, int32_t(args.size()), a->rows);
        args.push_back(b);
        made.emplace_back(t, i);
    }
    // Appends and allocations ran on the arenas' streams.
    for (cudaStream_t st : streams) {
        if (st != s && !CudaOk(cudaStreamSynchronize(st), "jr_build_batch")) return false;
    }
    auto* dargs = ToDevice(args, s);
    auto* dinit = ToDevice(init_items, s);
    auto* dbuild = ToDevice(build_items, s);
    bool ok = dargs && dinit && dbuild;
    if (ok) {
        JoinBuildBatch(dargs, dinit, int64_t(init_items.size()), true, s);
        JoinBuildBatch(dargs, dbuild, int64_t(build_items.size()), false, s);
        ok = CudaOk(cudaStreamSynchronize(s), "jr_build_batch");
    }
    DevFree(dargs, s);
    DevFree(dinit, s);
    DevFree(dbuild, s);
    for (auto& m : made) {
        if (ok) {
            PublishTable(tables[m.second], m.first, ArenaOf(arenas[m.second])->rows);
        } else {
            DestroyTable(m.first);
        }
    }
    return ok;
}

int64_t qdb_gpu_join_aggregate_probe_batch(const qdb_gpu_program* prog, void* const* arenas, void* const* tables,
                                           void* const* hts, qdb_rowset* const* batches, int64_t n) {
    t_error.clear();
    if (!prog || prog->kind != PK_JOIN_AGG || n < 0 || (n > 0 && (!arenas || !tables || !hts || !batches))) {
        SetErr("join_aggregate_probe_batch: bad arguments");
        return -1;
    }
    cudaStream_t s = CurStream();
    Staging stg(s);
    std::vector<JsBatchJoin> joins;
    std::vector<JoinBatchItem> items;
    std::vector<AggTableState*> sts;
    std::vector<cudaStream_t> streams;
    JoinSumShape common;
    bool batched = true;
    for (int64_t i = 0; i < n && batched; ++i) {
        ArenaState* a = ArenaOf(arenas[i]);
        TableState* t = TableOf(tables[i]);
        AggTableState* st = AggStateOf(hts[i]);
        if (!a || !t || !st || !batches[i]) {
            SetErr("join_aggregate_probe_batch: state %lld is not initialised and built", (long long)i);
            return -1;
        }
        AggPlan plan;
        int inline_slot = -1;
        JoinSumShape shape;
        bool is_sum = false;
        if (!ResolveJoinSum(prog, a, batches[i], stg, plan, inline_slot, shape, is_sum)) return -1;
        const int64_t* vcol = nullptr;
        // The batched kernel reads the bucket payload and one probe column.
        batched = is_sum && !batches[i]->Selection && JoinSumProbeColumn(shape, vcol);
        if (!batched) break;
        for (int k = 0; k < shape.nstates; ++k) {
            for (int f = 0; f < shape.states[k].nf; ++f) {
                JsFactor& jf = shape.states[k].f[f];
                if (jf.side == 0) jf.side = 3;
                jf.data = nullptr;
            }
        }
        if (i == 0) {
            common = shape;
        } else if (std::memcmp(common.states, shape.states, sizeof(shape.states)) != 0 ||
                   common.nstates != shape.nstates || common.need_pay != shape.need_pay) {
            batched = false;
            break;
        }
        JsBatchJoin j;
        std::memset(&j, 0, sizeof(j));
        j.jt = t->dev();
        j.key = shape.probe_key;
        j.vcol = vcol;
        AggJoinSumTargets(st, &j.states, &j.matched);
        if (std::find(streams.begin(), streams.end(), st->s) == streams.end()) streams.push_back(st->s);
        AddItems(items, int32_t(joins.size()), batches[i]->RowCount);
        joins.push_back(j);
        sts.push_back(st);
    }
    if (!batched) {
        // Another shape (a grouped aggregate, a selection): one by one.
        int64_t total = 0;
        for (int64_t i = 0; i < n; ++i) {
            const int64_t m = qdb_gpu_join_aggregate_probe(prog, arenas[i], tables[i], hts[i], batches[i]);
            if (m < 0) return -1;
            total += m;
        }
        return total;
    }
    // Biggest joins' items first: the tail of the launch is small items.
    std::stable_sort(items.begin(), items.end(), [&](const JoinBatchItem& x, const JoinBatchItem& y) {
        return batches[x.join]->RowCount > batches[y.join]->RowCount;
    });
    for (cudaStream_t st : streams) {
        if (st != s && !CudaOk(cudaStreamSynchronize(st), "join_aggregate_probe_batch")) return -1;
    }
    auto* djoins = ToDevice(joins, s);
    auto* ditems = ToDevice(items, s);
    auto* next = static_cast<unsigned*>(DevAlloc(4, s));
    bool ok = djoins && ditems && next;
    if (ok) {
        cudaMemsetAsync(next, 0, 4, s);
        JoinSumBatchRun(common, djoins, ditems, int64_t(items.size()), next, s);
        for (AggTableState* st : sts) AggJoinSumFetch(st, s);
        ok = CudaOk(cudaStreamSynchronize(s), "join_aggregate_probe_batch");
    }
    DevFree(djoins, s);
    DevFree(ditems, s);
    DevFree(next, s);
    if (!ok) return -1;
    int64_t total = 0;
    for (int64_t i = 0; i < n; ++i) {
        const int64_t before = AggStateMatched(sts[size_t(i)]);
        if (!AggJoinSumCommit(sts[size_t(i)])) return -1;
        AggMirrorHeader(hts[i], sts[size_t(i)], prog->agg.plan);
        total += AggStateMatched(sts[size_t(i)]) - before;
    }
    return total;
}

bool qdb_gpu_jr_append_batch(const qdb_gpu_program* prog, void* const* arenas, qdb_rowset* const* batches,
                             int64_t n) {
    t_error.clear();
    if (!prog || (prog->kind != PK_JOIN && prog->kind != PK_JOIN_AGG) || n < 0 || (n > 0 && (!arenas || !batches))) {
        SetErr("jr_append_batch: bad arguments");
        return false;
    }
    auto* hc = static_cast<unsigned long long*>(HostOutAlloc(size_t(std::max<int64_t>(n, 1)) * 16));
    if (!hc) return false;
    std::vector<AppendJob> jobs(static_cast<size_t>(n));
    std::vector<cudaStream_t> streams;
    bool ok = true;
    for (int64_t i = 0; i < n && ok; ++i) {
        ArenaState* a = ArenaOf(arenas[i]);
        if (!a || !batches[i]) {
            SetErr("jr_append_batch: arena %lld is not initialised", (long long)i);
            ok = false;
            break;
        }
        ok = AppendStart(prog, a, batches[i], false, jobs[size_t(i)], hc + 2 * i);
        if (std::find(streams.begin(), streams.end(), a->s) == streams.end()) streams.push_back(a->s);
    }
    for (cudaStream_t st : streams) ok = CudaOk(cudaStreamSynchronize(st), "jr_append_batch") && ok;
    for (int64_t i = 0; i < n; ++i) {
        AppendJob& job = jobs[size_t(i)];
        if (!job.a) continue;
        if (ok) {
            ok = AppendFinish(prog, job);
            static_cast<int64_t*>(arenas[i])[5] = job.a->rows;
        } else {
            job.Free();
        }
    }
    HostOutFree(hc);
    return ok;
}

}  // extern "C"
