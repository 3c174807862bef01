// sort_rt.cpp — sort entries of the C ABI: qdb_sort_run (sort + slice
// materialize, BuildSortRunWrapperAst, qdb/kernel/compiler.cpp:1165-1218),
// qdb_top_k_select (THeapTopKDispatch, qdb/kernel/compiler.h:585-596) and
// qdb_top_sort_update (TTopSortDispatch, compiler.h:570-583; the update of
// BuildTopSortUpdateAst, compiler.cpp:881-975).
//
// The store is the engine's array of retained batches (TSortProcessor::Add,
// qdb/exec/sort_exec.cpp:427-440) addressed by packed row ids; the number of
// batches a call touches is the largest batch index among its row ids plus
// one.  Columns may live in host or device memory; host columns are staged
// for the call.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include "runtime.h"
#include "sort.h"

namespace qdb {

namespace {

// Rows the top-K threshold is estimated from.
constexpr int64_t kTopKSamples = 32768;

// Device pointer tables of `cols` (store column indexes) over nbatches batches.
struct StoreView {
    StoreTable t;
    std::vector<int> cols;   // slot -> store column
    std::vector<int> owidth; // slot -> string offset bytes (0: not a string column)
    void* dev = nullptr;     // one allocation holding the five tables
    cudaStream_t s = nullptr;
    ~StoreView() { DevFree(dev, s); }
    int Slot(int col) const {
        for (size_t i = 0; i < cols.size(); ++i) {
            if (cols[i] == col) return int(i);
        }
        return -1;
    }
};

// A batch's string column on the device: its offsets and bytes (host
// offsets are checked to be non-decreasing, so that only staged bytes are
// read); every batch of a column must use one offset width.
bool StageStrings(const qdb_column& c, int64_t rows, Staging& stg, int64_t b, int col, int& owidth,
                  const char*& data, const char*& offs) {
    const int ow = c.OffsetWidth;
    if ((ow != 4 && ow != 8) || (owidth && owidth != ow) || (rows > 0 && (!c.Offsets || !c.Data))) {
        SetErr("sort: string column %d of batch %lld needs offsets of one width (4 or 8) and data", col, (long long)b);
        return false;
    }
    owidth = ow;
    data = offs = nullptr;
    if (rows == 0) return true;
    if (IsDevicePtr(c.Offsets)) {
        if (!IsDevicePtr(c.Data)) {
            SetErr("sort: string column %d of batch %lld has device offsets and host bytes", col, (long long)b);
            return false;
        }
        offs = static_cast<const char*>(c.Offsets);
        data = c.Data;
        return true;
    }
    int64_t prev = 0;
    for (int64_t r = 0; r <= rows; ++r) {
        const int64_t o = ow == 8 ? static_cast<const int64_t*>(c.Offsets)[r] : static_cast<const int32_t*>(c.Offsets)[r];
        if (o < prev) {
            SetErr("sort: string column %d of batch %lld: offsets decrease at row %lld", col, (long long)b,
                   (long long)r);
            return false;
        }
        prev = o;
    }
    offs = static_cast<const char*>(stg.Device(c.Offsets, size_t(rows + 1) * size_t(ow)));
    data = prev > 0 ? static_cast<const char*>(stg.Device(c.Data, size_t(prev))) : offs;
    return offs != nullptr && data != nullptr;
}

bool BuildStoreView(const SortProgram& P, const qdb_rowset* store, int64_t nbatches, Staging& stg, StoreView& v) {
    v.s = stg.s;
    const int nc = int(v.cols.size());
    const size_t cells = size_t(nbatches) * nc;
    std::vector<const char*> data(cells), offs(cells, nullptr);
    std::vector<const uint8_t*> mask(cells);
    std::vector<int64_t> dbit(cells), mbit(cells);
    v.owidth.assign(size_t(nc), 0);
    for (int64_t b = 0; b < nbatches; ++b) {
        const qdb_rowset& rs = store[b];
        for (int j = 0; j < nc; ++j) {
            const int col = v.cols[j];
            if (col >= rs.ColumnCount) {
                SetErr("sort: batch %lld has %lld columns, column %d is needed", (long long)b,
                       (long long)rs.ColumnCount, col);
                return false;
            }
            const qdb_column& c = rs.Columns[col];
            const int type = P.columns[col].type;
            const size_t i = size_t(b) * nc + j;
            const int64_t rows = rs.RowCount;
            size_t bytes;
            if (type == QDB_TYPE_STRING) {
                if (!StageStrings(c, rows, stg, b, col, v.owidth[size_t(j)], data[i], offs[i])) return false;
                bytes = 0;
            } else if (type == QDB_TYPE_BOOL) {
                bytes = size_t((c.DataBitOffset + rows + 7) / 8);
            } else {
                bytes = size_t(rows) * size_t(type == QDB_TYPE_DECIMAL128 ? 16 : SortKeyBits(type) / 8);
            }
            if (type != QDB_TYPE_STRING)
                data[i] = rows > 0 ? static_cast<const char*>(stg.Device(c.Data, std::max<size_t>(bytes, 1))) : nullptr;
            mask[i] = (c.Mask && rows > 0)
                          ? static_cast<const uint8_t*>(stg.Device(c.Mask, size_t((c.MaskBitOffset + rows + 7) / 8)))
                          : nullptr;
            dbit[i] = c.DataBitOffset;
            mbit[i] = c.MaskBitOffset;
            if (rows > 0 && !data[i]) return false;
        }
    }
    const size_t part = std::max<size_t>(cells, 1) * 8;
    v.dev = DevAlloc(5 * part, stg.s);
    if (!v.dev) return false;
    char* base = static_cast<char*>(v.dev);
    if (cells) {
        cudaMemcpyAsync(base, data.data(), cells * 8, cudaMemcpyHostToDevice, stg.s);
        cudaMemcpyAsync(base + part, mask.data(), cells * 8, cudaMemcpyHostToDevice, stg.s);
        cudaMemcpyAsync(base + 2 * part, dbit.data(), cells * 8, cudaMemcpyHostToDevice, stg.s);
        cudaMemcpyAsync(base + 3 * part, mbit.data(), cells * 8, cudaMemcpyHostToDevice, stg.s);
        cudaMemcpyAsync(base + 4 * part, offs.data(), cells * 8, cudaMemcpyHostToDevice, stg.s);
    }
    v.t.offsets = reinterpret_cast<const char* const*>(base + 4 * part);
    v.t.data = reinterpret_cast<const char* const*>(base);
    v.t.mask = reinterpret_cast<const uint8_t* const*>(base + part);
    v.t.data_bit = reinterpret_cast<const int64_t*>(base + 2 * part);
    v.t.mask_bit = reinterpret_cast<const int64_t*>(base + 3 * part);
    v.t.ncols = nc;
    v.t.nbatches = int32_t(nbatches);
    return true;
}

// Scratch owned by one call, freed in stream order.
struct Scratch {
    explicit Scratch(cudaStream_t st) : s(st) {}
    ~Scratch() {
        for (void* p : owned) DevFree(p, s);
    }
    void* Get(size_t bytes) {
        void* p = DevAlloc(std::max<size_t>(bytes, 16), s);
        if (p) owned.push_back(p);
        return p;
    }
    cudaStream_t s;
    std::vector<void*> owned;
};

// Number of batches the row ids touch (largest batch index + 1).  With
// `tiles`, also their dense-run marks and the number of tiles that are not
// dense (*sparse).
bool BatchCount(const int64_t* ids, int64_t n, Scratch& sc, int64_t& nbatches, int64_t* tiles = nullptr,
                int64_t* sparse = nullptr) {
    auto* d = static_cast<unsigned long long*>(sc.Get(16));
    if (!d) return false;
    SortMaxBatch(ids, n, d, tiles, sc.s);
    unsigned long long m[2] = {0, 0};
    cudaMemcpyAsync(m, d, tiles ? 16 : 8, cudaMemcpyDeviceToHost, sc.s);
    if (!CudaOk(cudaStreamSynchronize(sc.s), "sort: batch count")) return false;
    nbatches = n > 0 ? int64_t(m[0]) + 1 : 0;
    if (sparse) *sparse = int64_t(m[1]);
    return true;
}

// Dense-run marks of n row ids (one word per kSortIdTile ids).
int64_t* TileMarks(int64_t n, Scratch& sc) {
    return static_cast<int64_t*>(sc.Get(size_t((n + kSortIdTile - 1) / kSortIdTile) * 8));
}

bool ReadError(int* derr, cudaStream_t s, const char* what) {
    int herr = 0;
    cudaMemcpyAsync(&herr, derr, sizeof(int), cudaMemcpyDeviceToHost, s);
    if (!CudaOk(cudaStreamSynchronize(s), what)) return false;
    if (herr) {
        SetErr("%s: device error %d", what, herr);
        return false;
    }
    return true;
}

// Stages of an ORDER BY, least significant first: key k from the last to the
// first (compiler.cpp:595-599), a 64-bit nullable key followed by its NULL
// rank.  With `id_first`, the packed row id is the least significant stage.
// `chunks[k]`: 8-byte chunks of string key k (its longest string, rounded
// up), known once the store view is built; without it a string key gets its
// length stage only (enough to register its column in the view).
std::vector<SortStage> MakeStages(const SortProgram& P, const bool* descs, const bool* nulls_firsts, bool id_first,
                                  StoreView& v, const std::vector<int>* chunks = nullptr) {
    std::vector<SortStage> st;
    if (id_first) {
        SortStage g;
        g.src = SS_ROW_ID;
        g.wide = 1;
        st.push_back(g);
    }
    for (int k = int(P.keys.size()) - 1; k >= 0; --k) {
        const int col = P.keys[k].column;
        const qdb_column_type& ct = P.columns[col];
        int slot = v.Slot(col);
        if (slot < 0) {
            v.cols.push_back(col);
            slot = int(v.cols.size()) - 1;
        }
        SortStage g;
        g.src = SS_KEY;
        g.tcol = slot;
        g.type = ct.type;
        g.desc = descs ? descs[k] : P.keys[k].desc;
        g.nulls_first = nulls_firsts ? nulls_firsts[k] : P.keys[k].nulls_first;
        g.nullable = ct.nullable ? 1 : 0;
        if (ct.type == QDB_TYPE_STRING) {
            // Least significant first: the length, then the chunks from the
            // last to the first, then the NULL rank.
            g.wide = 1;
            g.owidth = size_t(slot) < v.owidth.size() ? v.owidth[size_t(slot)] : 0;
            SortStage len = g;
            len.src = SS_STR_LEN;
            st.push_back(len);
            const int nch = chunks ? (*chunks)[size_t(k)] : 0;
            for (int c = nch - 1; c >= 0; --c) {
                SortStage ch = g;
                ch.src = SS_STR_CHUNK;
                ch.chunk = c;
                st.push_back(ch);
            }
            if (g.nullable) {
                SortStage r = g;
                r.src = SS_NULL_RANK;
                r.wide = 0;
                st.push_back(r);
            }
            continue;
        }
        const int bits = SortKeyBits(ct.type);
        g.wide = (bits > 32 || g.nullable) ? 1 : 0;
        st.push_back(g);
        if (g.nullable && bits == 64) {
            SortStage r = g;
            r.src = SS_NULL_RANK;
            r.wide = 0;
            st.push_back(r);
        }
    }
    return st;
}

// Sorts n device row ids in place by the stages (stable).  `id_tiles`: the
// ids' dense-run marks (or nullptr), `sparse`: how many tiles are not dense.
bool SortIds(int64_t* ids, int64_t n, const std::vector<SortStage>& stages, const StoreTable& table, Scratch& sc,
             const int64_t* id_tiles = nullptr, int64_t sparse = 1) {
    cudaStream_t s = sc.s;
    const int ns = int(stages.size());
    if (n <= 1 || ns == 0) return true;
    if (ns > kMaxSortStagesTotal) {
        SetErr("sort: at most %d key stages are served (a string key takes one per 8 bytes of its longest value)",
               kMaxSortStagesTotal);
        return false;
    }
    bool any_wide = false;
    std::vector<void*> keys(ns);
    for (int i = 0; i < ns; ++i) {
        keys[i] = sc.Get(size_t(n) * (stages[i].wide ? 8 : 4));
        if (!keys[i]) return false;
        any_wide = any_wide || stages[i].wide;
    }
    const size_t nh = size_t(ns) * kSortDigits * 256;
    auto* hist = static_cast<unsigned long long*>(sc.Get(nh * 8));
    int* derr = static_cast<int*>(sc.Get(sizeof(int)));
    if (!hist || !derr) return false;
    cudaMemsetAsync(hist, 0, nh * 8, s);
    cudaMemsetAsync(derr, 0, sizeof(int), s);
    SortExtract(ids, n, table, stages.data(), ns, keys.data(), hist, derr, s);
    std::vector<unsigned long long> h(nh);
    cudaMemcpyAsync(h.data(), hist, nh * 8, cudaMemcpyDeviceToHost, s);
    if (!ReadError(derr, s, "sort: key extraction")) return false;

    // Pass plan: every digit that is not the same for all rows.
    struct Pass {
        int stage;
        int digit;
    };
    std::vector<Pass> plan;
    std::vector<unsigned long long> bases;
    for (int i = 0; i < ns; ++i) {
        const int nd = stages[i].wide ? 8 : 4;
        for (int d = 0; d < nd; ++d) {
            const unsigned long long* c = &h[(size_t(i) * kSortDigits + d) * 256];
            bool constant = false;
            unsigned long long run = 0;
            std::vector<unsigned long long> b(256);
            for (int x = 0; x < 256; ++x) {
                if (int64_t(c[x]) == n) constant = true;
                b[x] = run;
                run += c[x];
            }
            if (constant) continue;
            plan.push_back({i, d});
            bases.insert(bases.end(), b.begin(), b.end());
        }
    }
    if (plan.empty()) return true;   // every key is the same for all rows: the order stays

    const int64_t tiles = (n + kSortTile - 1) / kSortTile;
    auto* dbases = static_cast<unsigned long long*>(sc.Get(bases.size() * 8));
    auto* status = static_cast<unsigned long long*>(sc.Get(size_t(tiles) * 256 * 8));
    auto* counter = static_cast<unsigned int*>(sc.Get(sizeof(unsigned int)));
    void* kbuf[2] = {sc.Get(size_t(n) * (any_wide ? 8 : 4)), sc.Get(size_t(n) * (any_wide ? 8 : 4))};
    uint32_t* ibuf[2] = {static_cast<uint32_t*>(sc.Get(size_t(n) * 4)), static_cast<uint32_t*>(sc.Get(size_t(n) * 4))};
    // The ids are rewritten in place at the end: keep the originals unless
    // every one of them follows from its tile's mark.
    const bool keep = !(id_tiles && sparse == 0);
    int64_t* orig = keep ? static_cast<int64_t*>(sc.Get(size_t(n) * 8)) : nullptr;
    if (!dbases || !status || !counter || !kbuf[0] || !kbuf[1] || !ibuf[0] || !ibuf[1] || (keep && !orig)) return false;
    cudaMemcpyAsync(dbases, bases.data(), bases.size() * 8, cudaMemcpyHostToDevice, s);
    cudaMemsetAsync(status, 0, size_t(tiles) * 256 * 8, s);
    if (keep) cudaMemcpyAsync(orig, ids, size_t(n) * 8, cudaMemcpyDeviceToDevice, s);

    const uint32_t* idx = nullptr;   // identity
    int cur = 0;
    int prev_stage = -1;
    const void* kin = nullptr;
    for (size_t p = 0; p < plan.size(); ++p) {
        const int st = plan[p].stage;
        const bool first_of_stage = st != prev_stage;
        const bool gather = first_of_stage && idx != nullptr;
        if (first_of_stage) kin = keys[st];
        SortPass(stages[st].wide != 0, kin, idx, gather, kbuf[cur], ibuf[cur], n, 8 * plan[p].digit,
                 dbases + p * 256, status, uint32_t(p + 1), counter, derr, s);
        kin = kbuf[cur];
        idx = ibuf[cur];
        cur ^= 1;
        prev_stage = st;
    }
    SortGatherIds(orig, idx, n, id_tiles, ids, s);
    return ReadError(derr, s, "sort: radix passes");
}

bool HasStringKey(const SortProgram& P) {
    for (const qdb_sort_key& k : P.keys) {
        if (P.columns[k.column].type == QDB_TYPE_STRING) return true;
    }
    return false;
}

// 8-byte chunks of every string key (of its longest value among the rows);
// 0 for other keys.
bool StringChunks(const SortProgram& P, const int64_t* ids, int64_t n, const StoreView& v, Scratch& sc,
                  std::vector<int>& chunks) {
    chunks.assign(P.keys.size(), 0);
    auto* dmax = static_cast<unsigned long long*>(sc.Get(P.keys.size() * 8));
    int* derr = static_cast<int*>(sc.Get(sizeof(int)));
    if (!dmax || !derr) return false;
    cudaMemsetAsync(dmax, 0, P.keys.size() * 8, sc.s);
    cudaMemsetAsync(derr, 0, sizeof(int), sc.s);
    for (size_t k = 0; k < P.keys.size(); ++k) {
        const int col = P.keys[k].column;
        if (P.columns[col].type != QDB_TYPE_STRING) continue;
        const int slot = v.Slot(col);
        SortStringMaxLen(ids, n, v.t, slot, v.owidth[size_t(slot)], dmax + k, derr, sc.s);
    }
    std::vector<unsigned long long> h(P.keys.size());
    cudaMemcpyAsync(h.data(), dmax, h.size() * 8, cudaMemcpyDeviceToHost, sc.s);
    if (!ReadError(derr, sc.s, "sort: string lengths")) return false;
    for (size_t k = 0; k < h.size(); ++k) chunks[k] = int((h[k] + 7) / 8);
    return true;
}

// Materializes the out columns of ids[0, rows) into `out`.
int64_t Materialize(const qdb_gpu_program* prog, qdb_rowset* store, const int64_t* ids, int64_t rows, Scratch& sc,
                    Staging& stg, qdb_rowset* out) {
    const SortProgram& P = prog->sort;
    int64_t nbatches = 0;
    if (!BatchCount(ids, rows, sc, nbatches)) return -1;
    StoreView v;
    v.cols = P.out_columns;
    if (!BuildStoreView(P, store, nbatches, stg, v)) return -1;
    std::vector<int> types;
    for (int c : P.out_columns) types.push_back(P.columns[c].type);
    std::vector<AggOutputCol> cols;
    OutBlock blk;
    if (!AllocOutputCols(types, rows, true, cols, sc.s, &blk)) {
        SetErr("sort materialize: allocation failed");
        return -1;
    }
    int* derr = static_cast<int*>(sc.Get(sizeof(int)));
    if (!derr) return -1;
    cudaMemsetAsync(derr, 0, sizeof(int), sc.s);
    for (size_t j = 0; j < P.out_columns.size(); ++j) {
        SortMaterialize(v.t, int(j), types[j], ids, rows, cols[j].data, cols[j].valid, derr, sc.s);
    }
    if (!ReadError(derr, sc.s, "sort materialize")) return -1;
    if (!EmitRowset(cols, types, rows, (prog->flags & QDB_OUT_DEVICE) != 0, sc.s, out, &blk)) return -1;
    return rows;
}

// The first k row ids of the order (the keys, then the packed row id as the
// tie break, compiler.h:135-148) among the `size` device row ids `ids`,
// left in ids[0, k); returns k, or -1.
int64_t TopKDevice(const qdb_gpu_program* prog, qdb_rowset* store, int64_t* ids, int64_t size, int64_t k,
                   Scratch& sc, Staging& stg) {
    cudaStream_t s = sc.s;
    // Runs of consecutive rows (a scan's row ids) are fetched without their ids.
    int64_t* tiles = TileMarks(size, sc);
    if (!tiles) return -1;
    int64_t nbatches = 0;
    if (!BatchCount(ids, size, sc, nbatches, tiles)) return -1;
    StoreView v;
    // Exact order: row id first (the tie break, compiler.h:135-148), then the keys.
    const std::vector<SortStage> stages = MakeStages(prog->sort, nullptr, nullptr, true, v);
    if (!BuildStoreView(prog->sort, store, nbatches, stg, v)) return -1;
    const SortStage primary = stages.back().src == SS_NULL_RANK ? stages[stages.size() - 2] : stages.back();
    int* derr = static_cast<int*>(sc.Get(sizeof(int)));
    auto* counts = static_cast<unsigned long long*>(sc.Get(4096 * 8));
    if (!derr || !counts) return -1;
    cudaMemsetAsync(derr, 0, sizeof(int), s);

    if (SortKeyWidth(primary.type) < 0) {
        SetErr("top-k: the first key's type is not a sort key type");
        return -1;
    }
    const int64_t cap = std::max<int64_t>(4 * k, int64_t(1) << 20);
    int64_t* cand = nullptr;
    int64_t take = -1;

    // Sampled threshold: the r-th smallest primary key of ns rows spread
    // evenly over the input has about r * size / ns rows at or below it
    // (spread sqrt(r) * size / ns).  r is chosen so that count is at least K
    // with a margin of six spreads and is expected to fit the candidate
    // buffer.  The sample, the selection of its r-th key and the pass that
    // collects every row at or below it run back to back on the device; the
    // host reads only the count.  The result is exact whatever the sample
    // says: a count below K or above the buffer falls through to the radix
    // select.
    if (size > cap) {
        const int64_t ns = std::min<int64_t>(kTopKSamples, size);
        const double per = double(size) / double(ns);
        const double mk = double(k) / per;
        const int64_t r = int64_t(std::ceil(mk + 6.0 * std::sqrt(mk) + 8.0));
        if (r <= ns && (double(r) + 6.0 * std::sqrt(double(r))) * per <= double(cap)) {
            auto* skeys = static_cast<uint64_t*>(sc.Get(size_t(ns) * 8));
            auto* tau = static_cast<uint64_t*>(sc.Get(8));
            cand = static_cast<int64_t*>(sc.Get(size_t(cap) * 8));
            auto* ccount = static_cast<unsigned long long*>(sc.Get(8));
            if (!skeys || !tau || !cand || !ccount) return -1;
            TopKThreshold(ids, size, v.t, primary, skeys, ns, r, tau, derr, s);
            TopKCollect(ids, size, v.t, primary, 0, 64, tau, cand, cap, ccount, tiles, derr, s);
            unsigned long long got = 0;
            cudaMemcpyAsync(&got, ccount, 8, cudaMemcpyDeviceToHost, s);
            if (!ReadError(derr, s, "top-k: collect")) return -1;
            if (int64_t(got) >= k && int64_t(got) <= cap) take = int64_t(got);
        }
    }

    // Radix select on the primary key: narrow the bucket holding the K-th
    // row until the rows at or below it are few enough to order exactly.
    if (take < 0) {
        uint64_t prefix = 0;
        int pbits = 0;
        int64_t below = 0;
        take = size;
        std::vector<unsigned long long> h(4096);
        while (pbits < 64) {
            const int dbits = std::min(12, 64 - pbits);
            TopKHistogram(ids, size, v.t, primary, 64 - pbits - dbits, dbits, prefix, pbits, counts, derr, s);
            cudaMemcpyAsync(h.data(), counts, 4096 * 8, cudaMemcpyDeviceToHost, s);
            if (!ReadError(derr, s, "top-k: histogram")) return -1;
            int64_t run = below;
            int b = 0;
            for (; b < (1 << dbits) - 1; ++b) {
                if (run + int64_t(h[b]) >= k) break;
                run += int64_t(h[b]);
            }
            below = run;
            prefix = (prefix << dbits) | uint64_t(b);
            pbits += dbits;
            take = below + int64_t(h[b]);
            if (take <= cap) break;
        }
        if (!cand || take > cap) cand = static_cast<int64_t*>(sc.Get(size_t(take) * 8));
        auto* ccount = static_cast<unsigned long long*>(sc.Get(8));
        if (!cand || !ccount) return -1;
        TopKCollect(ids, size, v.t, primary, prefix, pbits, nullptr, cand, take, ccount, tiles, derr, s);
        unsigned long long got = 0;
        cudaMemcpyAsync(&got, ccount, 8, cudaMemcpyDeviceToHost, s);
        if (!ReadError(derr, s, "top-k: collect")) return -1;
        if (int64_t(got) != take) {
            SetErr("top-k: collected %llu rows, expected %lld", got, (long long)take);
            return -1;
        }
    }
    if (!SortIds(cand, take, stages, v.t, sc)) return -1;
    if (cand != ids) cudaMemcpyAsync(ids, cand, size_t(k) * 8, cudaMemcpyDeviceToDevice, s);
    return k;
}

const qdb_gpu_program* SortProgramOf(const qdb_gpu_program* p) {
    if (!p || p->kind != PK_SORT) {
        SetErr("not a sort program");
        return nullptr;
    }
    return p;
}

}  // namespace

}  // namespace qdb

using namespace qdb;

extern "C" {

qdb_gpu_program* qdb_gpu_compile_sort(const qdb_sort_spec* spec, char* err, size_t err_len) {
    auto fail = [&](const char* msg) -> qdb_gpu_program* {
        if (err && err_len) std::snprintf(err, err_len, "%s", msg);
        t_error = msg;
        return nullptr;
    };
    if (!spec || spec->n_columns <= 0 || spec->n_keys <= 0) return fail("sort: a schema and at least one key are needed");
    auto* p = new qdb_gpu_program();
    p->kind = PK_SORT;
    p->flags = spec->flags;
    SortProgram& P = p->sort;
    P.columns.assign(spec->columns, spec->columns + spec->n_columns);
    P.keys.assign(spec->keys, spec->keys + spec->n_keys);
    P.out_columns.assign(spec->out_columns, spec->out_columns + spec->n_out);
    for (const qdb_sort_key& k : P.keys) {
        if (k.column < 0 || k.column >= spec->n_columns) {
            delete p;
            return fail("sort: key column out of range");
        }
        if (SortKeyBits(P.columns[k.column].type) == 0 && P.columns[k.column].type != QDB_TYPE_STRING) {
            delete p;
            return fail("sort: key type is not served (fixed-width integer, decimal64, date, float, bool, char1, "
                        "string)");
        }
    }
    for (int c : P.out_columns) {
        if (c < 0 || c >= spec->n_columns) {
            delete p;
            return fail("sort: output column out of range");
        }
        const int t = P.columns[c].type;
        if (SortKeyBits(t) == 0 && t != QDB_TYPE_DECIMAL128) {
            delete p;
            return fail("sort: output column type is not served");
        }
    }
    // Stages: every key plus a NULL rank per nullable 64-bit key, plus the row
    // id stage top-K adds.
    // (A string key's stages depend on its longest value: checked per sort.)
    int stages = 1;
    for (const qdb_sort_key& k : P.keys) {
        const int t = P.columns[k.column].type;
        stages += 1 + ((P.columns[k.column].nullable && (SortKeyBits(t) == 64 || t == QDB_TYPE_STRING)) ? 1 : 0);
    }
    if (stages > kMaxSortStagesTotal) {
        delete p;
        return fail("sort: too many keys");
    }
    return p;
}

int64_t qdb_gpu_sort_run(const qdb_gpu_program* program, qdb_rowset* store, int64_t* row_ids, int64_t* work,
                         uint32_t* counts, int64_t n, bool* descs, bool* nulls_firsts, bool do_sort, int64_t start,
                         int64_t limit, qdb_rowset* out) {
    (void)work;
    (void)counts;
    t_error.clear();
    const qdb_gpu_program* prog = SortProgramOf(program);
    if (!prog) return -1;
    if (n > 0 && (!store || !row_ids)) {
        SetErr("sort: store and row ids are needed");
        return -1;
    }
    if (n > int64_t(UINT32_MAX)) {
        SetErr("sort: more than 2^32 rows");   // TSortProcessor::TryRadixSort's bound
        return -1;
    }
    cudaStream_t s = CurStream();
    const bool dev_ids = IsDevicePtr(row_ids);
    if (do_sort && n > 1) {
        Scratch sc(s);
        Staging stg(s);
        int64_t* ids = row_ids;
        if (!dev_ids) {
            ids = static_cast<int64_t*>(sc.Get(size_t(n) * 8));
            if (!ids) return -1;
            cudaMemcpyAsync(ids, row_ids, size_t(n) * 8, cudaMemcpyHostToDevice, s);
        }
        int64_t* tiles = TileMarks(n, sc);
        if (!tiles) return -1;
        int64_t nbatches = 0, sparse = 0;
        if (!BatchCount(ids, n, sc, nbatches, tiles, &sparse)) return -1;
        StoreView v;
        std::vector<SortStage> stages = MakeStages(prog->sort, descs, nulls_firsts, false, v);
        if (!BuildStoreView(prog->sort, store, nbatches, stg, v)) return -1;
        if (HasStringKey(prog->sort)) {
            std::vector<int> chunks;
            if (!StringChunks(prog->sort, ids, n, v, sc, chunks)) return -1;
            stages = MakeStages(prog->sort, descs, nulls_firsts, false, v, &chunks);
        }
        if (!SortIds(ids, n, stages, v.t, sc, tiles, sparse)) return -1;
        if (!dev_ids) {
            cudaMemcpyAsync(row_ids, ids, size_t(n) * 8, cudaMemcpyDeviceToHost, s);
            if (!CudaOk(cudaStreamSynchronize(s), "sort: row ids")) return -1;
        }
    }
    if (limit <= 0 || !out) return 0;
    const int64_t rows = std::min(limit, n - start);
    if (start < 0 || rows <= 0) {
        std::memset(out, 0, sizeof(*out));
        return 0;
    }
    Scratch sc(s);
    Staging stg(s);
    const int64_t* ids = row_ids + start;
    if (!dev_ids) {
        int64_t* d = static_cast<int64_t*>(sc.Get(size_t(rows) * 8));
        if (!d) return -1;
        cudaMemcpyAsync(d, row_ids + start, size_t(rows) * 8, cudaMemcpyHostToDevice, s);
        ids = d;
    }
    return Materialize(prog, store, ids, rows, sc, stg, out);
}

int64_t qdb_gpu_top_k_select(const qdb_gpu_program* program, qdb_rowset* store, int64_t* row_ids, int64_t size,
                             int64_t limit) {
    t_error.clear();
    const qdb_gpu_program* prog = SortProgramOf(program);
    if (!prog) return -1;
    if (HasStringKey(prog->sort)) {
        SetErr("top-K: string keys are served by qdb_sort_run (then a slice), not by the top-K entries");
        return -1;
    }
    const int64_t k = std::min(limit, size);
    if (k <= 0) return 0;
    if (!store || !row_ids) {
        SetErr("top-k: store and row ids are needed");
        return -1;
    }
    if (size > int64_t(UINT32_MAX)) {
        SetErr("top-k: more than 2^32 rows");
        return -1;
    }
    cudaStream_t s = CurStream();
    Scratch sc(s);
    Staging stg(s);
    const bool dev_ids = IsDevicePtr(row_ids);
    int64_t* ids = row_ids;
    if (!dev_ids) {
        ids = static_cast<int64_t*>(sc.Get(size_t(size) * 8));
        if (!ids) return -1;
        cudaMemcpyAsync(ids, row_ids, size_t(size) * 8, cudaMemcpyHostToDevice, s);
    }
    if (TopKDevice(prog, store, ids, size, k, sc, stg) < 0) return -1;
    if (!dev_ids) cudaMemcpyAsync(row_ids, ids, size_t(k) * 8, cudaMemcpyDeviceToHost, s);
    if (!CudaOk(cudaStreamSynchronize(s), "top-k")) return -1;
    return k;
}

// Writes n int64 values to `dst`, host or device memory.
static bool PutI64(int64_t* dst, const int64_t* src, int64_t n, cudaStream_t s) {
    if (n <= 0) return true;
    if (IsDevicePtr(dst)) return CudaOk(cudaMemcpyAsync(dst, src, size_t(n) * 8, cudaMemcpyHostToDevice, s), "copy");
    std::memcpy(dst, src, size_t(n) * 8);
    return true;
}

int64_t qdb_gpu_top_sort_update(const qdb_gpu_program* program, qdb_rowset* state, qdb_rowset* batch,
                                int64_t* row_ids, int64_t* work, uint32_t* counts, int64_t n, bool sort_input,
                                uint8_t* pick_src, uint32_t* pick_idx, int64_t limit, qdb_rowset* out) {
    (void)work;
    (void)counts;
    t_error.clear();
    const qdb_gpu_program* prog = SortProgramOf(program);
    if (!prog) return -1;
    if (HasStringKey(prog->sort)) {
        SetErr("top-K: string keys are served by qdb_sort_run (then a slice), not by the top-K entries");
        return -1;
    }
    const SortProgram& P = prog->sort;
    if (!state || !batch || !out || (n > 0 && !row_ids) || n < 0) {
        SetErr("top-sort: state, batch, output and row ids are needed");
        return -1;
    }
    // The state is this call's output of the previous call: it must have the
    // batch's schema, so the program materializes every column in order.
    bool identity = P.out_columns.size() == P.columns.size();
    for (size_t c = 0; identity && c < P.out_columns.size(); ++c) identity = P.out_columns[c] == int(c);
    if (!identity) {
        SetErr("top-sort: the program must materialize every input column in order (the state keeps the schema)");
        return -1;
    }
    if (n > int64_t(UINT32_MAX)) {
        SetErr("top-sort: more than 2^32 rows");
        return -1;
    }
    const int64_t state_n = std::max<int64_t>(0, state->RowCount);
    if (limit <= 0) {
        std::memset(out, 0, sizeof(*out));
        return 0;
    }
    cudaStream_t s = CurStream();
    Scratch sc(s);
    Staging stg(s);

    // 1. The batch's first k rows of the order (sort_input: sort them here,
    // stable in row-id order; else they arrive ordered, e.g. by top-K).
    const int64_t k = std::min(n, limit);
    std::vector<int64_t> temp(size_t(std::max<int64_t>(k, 0)));
    if (k > 0) {
        int64_t* ids = row_ids;
        if (!IsDevicePtr(row_ids)) {
            ids = static_cast<int64_t*>(sc.Get(size_t(n) * 8));
            if (!ids) return -1;
            cudaMemcpyAsync(ids, row_ids, size_t(n) * 8, cudaMemcpyHostToDevice, s);
        }
        if (sort_input && n > 1) {
            int64_t nbatches = 0;
            if (!BatchCount(ids, n, sc, nbatches)) return -1;
            if (nbatches > 1) {
                SetErr("top-sort: the batch's row ids must name batch 0");
                return -1;
            }
            qdb_rowset one[1] = {*batch};
            if (k < n) {
                if (TopKDevice(prog, one, ids, n, k, sc, stg) < 0) return -1;
            } else {
                StoreView v;
                const std::vector<SortStage> stages = MakeStages(P, nullptr, nullptr, false, v);
                if (!BuildStoreView(P, one, 1, stg, v)) return -1;
                if (!SortIds(ids, n, stages, v.t, sc)) return -1;
            }
        }
        cudaMemcpyAsync(temp.data(), ids, size_t(k) * 8, cudaMemcpyDeviceToHost, s);
        if (!CudaOk(cudaStreamSynchronize(s), "top-sort: batch order")) return -1;
    }

    // 2. Merge with the state (top_sort_merge_picks, qdb/kernel/sort/top_sort.oz:15-57):
    // a stable sort of the state rows followed by the batch rows keeps the
    // state row first on equal keys, as the merge does.  Row ids name the
    // store [state, batch].
    const int64_t m = state_n + k;
    const int64_t out_count = std::min(limit, m);
    std::vector<int64_t> comb(size_t(std::max<int64_t>(m, 1)));
    for (int64_t i = 0; i < state_n; ++i) comb[size_t(i)] = i;
    for (int64_t j = 0; j < k; ++j) comb[size_t(state_n + j)] = (int64_t(1) << 32) | int64_t(uint32_t(temp[size_t(j)]));
    qdb_rowset two[2] = {*state, *batch};
    int64_t* dcomb = static_cast<int64_t*>(sc.Get(size_t(std::max<int64_t>(m, 1)) * 8));
    if (!dcomb) return -1;
    if (state_n > 0 && k > 0) {
        cudaMemcpyAsync(dcomb, comb.data(), size_t(m) * 8, cudaMemcpyHostToDevice, s);
        StoreView v;
        const std::vector<SortStage> stages = MakeStages(P, nullptr, nullptr, false, v);
        if (!BuildStoreView(P, two, 2, stg, v)) return -1;
        if (!SortIds(dcomb, m, stages, v.t, sc)) return -1;
        cudaMemcpyAsync(comb.data(), dcomb, size_t(out_count) * 8, cudaMemcpyDeviceToHost, s);
        if (!CudaOk(cudaStreamSynchronize(s), "top-sort: merge")) return -1;
    }

    // 3. The picks, and row_ids[i] = (pick_src << 32) | pick_idx as the
    // reference leaves them.
    for (int64_t i = 0; i < out_count; ++i) {
        const int64_t id = comb[size_t(i)];
        if (pick_src && !IsDevicePtr(pick_src)) pick_src[i] = uint8_t(id >> 32);
        if (pick_idx && !IsDevicePtr(pick_idx)) pick_idx[i] = uint32_t(id);
    }
    if (pick_src && IsDevicePtr(pick_src)) {
        std::vector<uint8_t> ps(static_cast<size_t>(out_count));
        for (int64_t i = 0; i < out_count; ++i) ps[size_t(i)] = uint8_t(comb[size_t(i)] >> 32);
        cudaMemcpyAsync(pick_src, ps.data(), ps.size(), cudaMemcpyHostToDevice, s);
        if (!CudaOk(cudaStreamSynchronize(s), "top-sort: picks")) return -1;
    }
    if (pick_idx && IsDevicePtr(pick_idx)) {
        std::vector<uint32_t> pi(static_cast<size_t>(out_count));
        for (int64_t i = 0; i < out_count; ++i) pi[size_t(i)] = uint32_t(comb[size_t(i)]);
        cudaMemcpyAsync(pick_idx, pi.data(), pi.size() * 4, cudaMemcpyHostToDevice, s);
        if (!CudaOk(cudaStreamSynchronize(s), "top-sort: picks")) return -1;
    }
    if (out_count > 0 && row_ids && !PutI64(row_ids, comb.data(), out_count, s)) return -1;
    if (out_count <= 0) {
        std::memset(out, 0, sizeof(*out));
        return 0;
    }

    // 4. Materialize the kept rows from [state, batch] (just the batch when
    // the state is empty).
    qdb_rowset* store = two;
    if (state_n == 0) {
        for (int64_t i = 0; i < out_count; ++i) comb[size_t(i)] &= 0xffffffffll;
        store = two + 1;
    }
    cudaMemcpyAsync(dcomb, comb.data(), size_t(out_count) * 8, cudaMemcpyHostToDevice, s);
    const int64_t r = Materialize(prog, store, dcomb, out_count, sc, stg, out);
    if (r >= 0 && !CudaOk(cudaStreamSynchronize(s), "top-sort")) return -1;
    return r;
}

}  // extern "C"
