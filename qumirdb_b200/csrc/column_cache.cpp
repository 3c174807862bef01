// column_cache.cpp — device column cache between the engine's scan sources
// and the kernels.  TParquetSource::Next (qdb/io/parquet/source.h:89) hands
// out host row sets of 2^18 rows (qdb/io/parquet/source.cpp:333); every
// query over the same file would copy them to the device again.  This cache
// keeps each column of each batch resident in HBM under (source, batch,
// column), up to a byte budget, and hands out device row sets over them.
//
// Copies from pageable host memory go through two pinned staging buffers:
// the host fills one while the DMA engine drains the other (an event per
// buffer orders the reuse), so a cold batch moves at PCIe speed without
// page-locking the engine's buffers.  Page-locked host columns are copied
// directly.  Entries in use by a handed-out row set are pinned; the least
// recently used unpinned ones are evicted to make room.
#include <algorithm>
#include <cstring>
#include <list>
#include <mutex>
#include <unordered_map>
#include <vector>

#include "runtime.h"

namespace qdb {

namespace {

struct CacheKey {
    uint64_t source;
    int64_t batch;
    int32_t column;
    bool operator==(const CacheKey& o) const {
        return source == o.source && batch == o.batch && column == o.column;
    }
};

struct CacheKeyHash {
    size_t operator()(const CacheKey& k) const {
        uint64_t h = k.source * 0x9E3779B97F4A7C15ull;
        h ^= uint64_t(k.batch) + 0x632BE59BD9B4E019ull + (h << 6) + (h >> 2);
        h ^= uint64_t(uint32_t(k.column)) + 0x85EBCA77C2B2AE63ull + (h << 6) + (h >> 2);
        return size_t(h);
    }
};

struct CacheEntry {
    CacheKey key;
    void* data = nullptr;        // device, rows * width bytes
    uint8_t* mask = nullptr;     // device validity bitmap, bit offset 0 (or null)
    int64_t rows = 0;
    size_t bytes = 0;
    int32_t pins = 0;
    std::list<CacheEntry*>::iterator lru;   // position in the LRU list (front = most recent)
};

}  // namespace

}  // namespace qdb

struct qdb_gpu_column_cache {
    std::mutex mu;
    cudaStream_t s = nullptr;
    size_t budget = 0;
    size_t staging = 0;
    char* pinned[2] = {nullptr, nullptr};
    cudaEvent_t drained[2] = {nullptr, nullptr};
    int next = 0;
    std::unordered_map<qdb::CacheKey, qdb::CacheEntry*, qdb::CacheKeyHash> map;
    std::list<qdb::CacheEntry*> lru;
    qdb_gpu_cache_stats st{};
};

namespace qdb {

namespace {

// What one handed-out row set holds: its columns and the pinned entries.
struct CacheRowset {
    qdb_gpu_column_cache* cache;
    std::vector<CacheEntry*> entries;
    std::vector<qdb_column> cols;
    void* selection = nullptr;
};

bool IsPinnedHost(const void* p) {
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeHost;
}

// Host -> device copy of `bytes` on the cache's stream: direct from
// page-locked memory, else through the two pinned staging buffers.
bool CopyIn(qdb_gpu_column_cache* c, void* dst, const void* src, size_t bytes) {
    if (bytes == 0) return true;
    if (IsPinnedHost(src)) {
        return CudaOk(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, c->s), "cache copy");
    }
    size_t done = 0;
    while (done < bytes) {
        const int b = c->next;
        c->next ^= 1;
        // The buffer's previous copy must have drained before it is refilled.
        if (!CudaOk(cudaEventSynchronize(c->drained[b]), "cache staging")) return false;
        const size_t n = std::min(c->staging, bytes - done);
        std::memcpy(c->pinned[b], static_cast<const char*>(src) + done, n);
        if (!CudaOk(cudaMemcpyAsync(static_cast<char*>(dst) + done, c->pinned[b], n, cudaMemcpyHostToDevice, c->s),
                    "cache copy") ||
            !CudaOk(cudaEventRecord(c->drained[b], c->s), "cache staging")) {
            return false;
        }
        done += n;
    }
    return true;
}

void FreeEntry(qdb_gpu_column_cache* c, CacheEntry* e) {
    DevFree(e->data, c->s);
    DevFree(e->mask, c->s);
    c->st.resident_bytes -= int64_t(e->bytes);
    c->st.entries -= 1;
    delete e;
}

// Evicts least recently used unpinned entries until `need` more bytes fit.
bool MakeRoom(qdb_gpu_column_cache* c, size_t need) {
    auto it = c->lru.end();
    while (size_t(c->st.resident_bytes) + need > c->budget && it != c->lru.begin()) {
        --it;
        CacheEntry* e = *it;
        if (e->pins > 0) continue;
        it = c->lru.erase(it);
        c->map.erase(e->key);
        FreeEntry(c, e);
        c->st.evictions += 1;
    }
    return size_t(c->st.resident_bytes) + need <= c->budget;
}

void Touch(qdb_gpu_column_cache* c, CacheEntry* e) {
    c->lru.erase(e->lru);
    c->lru.push_front(e);
    e->lru = c->lru.begin();
}

void Unpin(qdb_gpu_column_cache* c, CacheEntry* e) {
    e->pins -= 1;
    if (e->pins == 0) c->st.pinned_bytes -= int64_t(e->bytes);
}

void DestroyCacheRowset(qdb_rowset* rs) {
    if (!rs || !rs->Private) return;
    auto* r = static_cast<CacheRowset*>(rs->Private);
    {
        std::lock_guard<std::mutex> g(r->cache->mu);
        for (CacheEntry* e : r->entries) Unpin(r->cache, e);
        DevFree(r->selection, r->cache->s);
    }
    delete r;
    rs->Private = nullptr;
    rs->Columns = nullptr;
    rs->Selection = nullptr;
}

}  // namespace

}  // namespace qdb

using namespace qdb;

extern "C" {

qdb_gpu_column_cache* qdb_gpu_cache_create(size_t budget_bytes, size_t staging_bytes) {
    t_error.clear();
    auto* c = new qdb_gpu_column_cache();
    c->s = CurStream();
    c->budget = budget_bytes;
    c->staging = staging_bytes ? staging_bytes : (size_t(8) << 20);
    for (int b = 0; b < 2; ++b) {
        if (!CudaOk(cudaMallocHost(reinterpret_cast<void**>(&c->pinned[b]), c->staging), "cache staging") ||
            !CudaOk(cudaEventCreateWithFlags(&c->drained[b], cudaEventDisableTiming), "cache staging")) {
            qdb_gpu_cache_destroy(c);
            return nullptr;
        }
    }
    return c;
}

void qdb_gpu_cache_destroy(qdb_gpu_column_cache* c) {
    if (!c) return;
    {
        std::lock_guard<std::mutex> g(c->mu);
        for (CacheEntry* e : c->lru) FreeEntry(c, e);
        c->lru.clear();
        c->map.clear();
        cudaStreamSynchronize(c->s);
        for (int b = 0; b < 2; ++b) {
            if (c->drained[b]) cudaEventDestroy(c->drained[b]);
            if (c->pinned[b]) cudaFreeHost(c->pinned[b]);
        }
    }
    delete c;
}

int64_t qdb_gpu_cache_get(qdb_gpu_column_cache* c, uint64_t source_id, int64_t batch_index, const qdb_rowset* host,
                          const qdb_column_type* types, const int32_t* columns, int32_t n, qdb_rowset* out) {
    t_error.clear();
    if (!c || !host || !out || n < 0 || (n > 0 && (!types || !columns))) {
        SetErr("cache_get: bad arguments");
        return -1;
    }
    const int64_t rows = host->RowCount;
    auto* r = new CacheRowset();
    r->cache = c;
    r->cols.resize(size_t(std::max(n, 1)));
    std::lock_guard<std::mutex> g(c->mu);
    auto fail = [&]() {
        for (CacheEntry* e : r->entries) Unpin(c, e);
        DevFree(r->selection, c->s);
        delete r;
        return int64_t(-1);
    };
    bool copied = false;
    for (int32_t j = 0; j < n; ++j) {
        const int32_t ci = columns[j];
        if (ci < 0 || ci >= host->ColumnCount) {
            SetErr("cache_get: column %d outside the batch", ci);
            return fail();
        }
        const qdb_column& hc = host->Columns[ci];
        const int type = types[ci].type;
        const CacheKey key{source_id, batch_index, ci};
        CacheEntry* e = nullptr;
        auto it = c->map.find(key);
        if (it != c->map.end()) {
            e = it->second;
            if (e->rows != rows) {
                SetErr("cache_get: batch %lld of source %llu has %lld rows, not %lld as cached",
                       (long long)batch_index, (unsigned long long)source_id, (long long)rows, (long long)e->rows);
                return fail();
            }
            Touch(c, e);
            c->st.hits += 1;
        } else {
            // BOOL is bit-packed from DataBitOffset; masks from MaskBitOffset:
            // both are copied whole bytes from bit 0 and keep their offsets.
            const size_t dbytes = type == QDB_TYPE_BOOL ? size_t((hc.DataBitOffset + rows + 7) / 8)
                                                        : size_t(rows) * size_t(StorageWidth(type));
            const size_t mbytes = hc.Mask ? size_t((hc.MaskBitOffset + rows + 7) / 8) : 0;
            const size_t bytes = dbytes + mbytes;
            if (bytes > c->budget) {
                SetErr("cache_get: a column of %zu bytes exceeds the cache budget of %zu", bytes, c->budget);
                return fail();
            }
            if (!MakeRoom(c, bytes)) {
                SetErr("cache_get: columns in use fill the cache budget");
                return fail();
            }
            e = new CacheEntry();
            e->key = key;
            e->rows = rows;
            e->bytes = bytes;
            e->data = DevAlloc(std::max<size_t>(dbytes, 16), c->s);
            e->mask = mbytes ? static_cast<uint8_t*>(DevAlloc(mbytes, c->s)) : nullptr;
            if (!e->data || (mbytes && !e->mask) || !CopyIn(c, e->data, hc.Data, dbytes) ||
                (mbytes && !CopyIn(c, e->mask, hc.Mask, mbytes))) {
                DevFree(e->data, c->s);
                DevFree(e->mask, c->s);
                delete e;
                return fail();
            }
            c->lru.push_front(e);
            e->lru = c->lru.begin();
            c->map.emplace(key, e);
            c->st.resident_bytes += int64_t(bytes);
            c->st.entries += 1;
            c->st.misses += 1;
            c->st.h2d_bytes += int64_t(bytes);
            copied = true;
        }
        if (e->pins++ == 0) c->st.pinned_bytes += int64_t(e->bytes);
        r->entries.push_back(e);
        qdb_column& oc = r->cols[size_t(j)];
        std::memset(&oc, 0, sizeof(oc));
        oc.Data = static_cast<char*>(e->data);
        oc.DataBitOffset = type == QDB_TYPE_BOOL ? hc.DataBitOffset : 0;
        oc.Mask = e->mask;
        oc.MaskBitOffset = e->mask ? hc.MaskBitOffset : 0;
    }
    if (host->Selection && rows > 0) {
        r->selection = DevAlloc(size_t(rows), c->s);
        if (!r->selection || !CopyIn(c, r->selection, host->Selection, size_t(rows))) return fail();
        copied = true;
    }
    if (copied && !CudaOk(cudaStreamSynchronize(c->s), "cache copy")) return fail();
    std::memset(out, 0, sizeof(*out));
    out->Columns = r->cols.data();
    out->ColumnCount = n;
    out->RowCount = rows;
    out->Selection = static_cast<uint8_t*>(r->selection);
    out->Destroy = DestroyCacheRowset;
    out->Private = r;
    out->RefCount = 1;
    return 0;
}

int64_t qdb_gpu_cache_invalidate(qdb_gpu_column_cache* c, uint64_t source_id) {
    if (!c) return 0;
    std::lock_guard<std::mutex> g(c->mu);
    int64_t dropped = 0;
    for (auto it = c->lru.begin(); it != c->lru.end();) {
        CacheEntry* e = *it;
        if (e->key.source == source_id && e->pins == 0) {
            it = c->lru.erase(it);
            c->map.erase(e->key);
            FreeEntry(c, e);
            ++dropped;
        } else {
            ++it;
        }
    }
    return dropped;
}

void qdb_gpu_cache_get_stats(qdb_gpu_column_cache* c, qdb_gpu_cache_stats* st) {
    if (!c || !st) return;
    std::lock_guard<std::mutex> g(c->mu);
    *st = c->st;
}

}  // extern "C"
