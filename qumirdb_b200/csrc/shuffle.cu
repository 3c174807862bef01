// shuffle.cu — the hash shuffle on the device (sm_100a): THashShuffleTask's
// scatter of one batch (qdb/scheduler/tasks/runtime_adapter.cpp:998-1112)
// into partition-contiguous device buffers, so that threaded plans can feed
// GPU partitions (a partial aggregate's states to the final aggregates of
// their key partitions, a join side to its build partitions) without a host
// gather.
//
// Every selected row goes to output routes[hash % n_routes], or hash %
// n_outputs without routes; hash is the batch's precomputed Hash column when
// it has one, else the program's rh_hash of its key columns.  Outputs keep
// input row order.  On the device: one pass hashes and routes the rows and
// counts each output's rows; the selected rows are compacted; a stable
// counting sort on the output index (the onesweep passes of sort.cu, one per
// non-constant byte) orders them; every column, its validity and the hashes
// are then gathered once into buffers that the outputs slice.
#include <algorithm>
#include <cstring>
#include <memory>
#include <vector>

#include "common.cuh"
#include "kernels.h"
#include "runtime.h"
#include "sort.h"

namespace qdb {

namespace {

constexpr int kMaxOutputs = 1 << 16;

// dst[r] = output of selected row r (flags[r] = 1), counts[dst] += 1; a
// route outside [0, n_outputs) sets *err to 1.
__global__ void __launch_bounds__(256) RouteKernel(const uint64_t* hashes, const uint8_t* sel, int64_t n,
                                                   const int32_t* routes, int64_t n_routes, int64_t n_outputs,
                                                   uint32_t* dst, uint8_t* flags, unsigned long long* counts,
                                                   int* err) {
    for (int64_t r = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; r < n; r += int64_t(gridDim.x) * blockDim.x) {
        const bool selected = sel == nullptr || sel[r] != 0;
        flags[r] = selected ? 1 : 0;
        if (!selected) continue;
        const uint64_t h = hashes[r];
        int64_t d = routes ? int64_t(routes[h % uint64_t(n_routes)]) : int64_t(h % uint64_t(n_outputs));
        if (d < 0 || d >= n_outputs) {
            atomicExch(err, 1);
            d = 0;
        }
        dst[r] = uint32_t(d);
        atomicAdd(&counts[d], 1ull);
    }
}

// keys[i] = dst[rows[i]].
__global__ void __launch_bounds__(256) GatherDstKernel(const uint32_t* dst, const int64_t* rows, int64_t m,
                                                       uint32_t* keys) {
    for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < m; i += int64_t(gridDim.x) * blockDim.x) {
        keys[i] = dst[rows[i]];
    }
}

// out[i] = rows[perm[i]] (perm null: the identity).
__global__ void __launch_bounds__(256) PermuteRowsKernel(const int64_t* rows, const uint32_t* perm, int64_t m,
                                                         int64_t* out) {
    for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < m; i += int64_t(gridDim.x) * blockDim.x) {
        out[i] = rows[perm ? perm[i] : i];
    }
}

__global__ void __launch_bounds__(256) GatherU64Kernel(const uint64_t* src, const int64_t* rows, int64_t m,
                                                       uint64_t* out) {
    for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < m; i += int64_t(gridDim.x) * blockDim.x) {
        out[i] = src[rows[i]];
    }
}

__global__ void __launch_bounds__(256) IotaI32Kernel(int32_t* out, int64_t n) {
    for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
        out[i] = int32_t(i);
    }
}

int Grid(int64_t n) {
    return int(std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, int64_t(DeviceSMs()) * 16)));
}

struct CallScratch {
    cudaStream_t s;
    std::vector<void*> held;
    explicit CallScratch(cudaStream_t st) : s(st) {}
    ~CallScratch() {
        for (void* p : held) DevFree(p, s);
    }
    template <class T>
    T* Get(int64_t count) {
        void* p = DevAlloc(size_t(std::max<int64_t>(count, 1)) * sizeof(T), s);
        if (p) held.push_back(p);
        return static_cast<T*>(p);
    }
};

// Device buffers shared by the outputs of one shuffle; freed with the last.
struct ShuffleOutputs {
    std::vector<void*> dev;
    cudaStream_t s = nullptr;
    ~ShuffleOutputs() {
        for (void* p : dev) DevFree(p, s);
    }
};

struct ShuffleSlice {
    std::shared_ptr<ShuffleOutputs> owner;
    std::vector<qdb_column> cols;
};

void DestroyShuffleSlice(qdb_rowset* rs) {
    if (!rs || !rs->Private) return;
    delete static_cast<ShuffleSlice*>(rs->Private);
    rs->Private = nullptr;
    rs->Columns = nullptr;
    rs->Hash = nullptr;
}

// Stable order of m u32 keys below n_outputs: perm (positions into the
// keys) from the onesweep passes over the non-constant bytes, whose digit
// counts follow from the per-output counts.  perm = nullptr when the keys
// are already in order (one output).
bool StableOrder(const uint32_t* keys, int64_t m, const std::vector<unsigned long long>& counts, uint32_t** perm,
                 CallScratch& sc) {
    *perm = nullptr;
    const int64_t nout = int64_t(counts.size());
    if (m <= 1 || nout <= 1) return true;
    std::vector<int> digits;
    std::vector<unsigned long long> bases;
    for (int d = 0; d < 4 && (int64_t(1) << (8 * d)) < nout; ++d) {
        std::vector<unsigned long long> h(256, 0);
        for (int64_t o = 0; o < nout; ++o) h[(o >> (8 * d)) & 255] += counts[size_t(o)];
        if (std::find(h.begin(), h.end(), (unsigned long long)m) != h.end()) continue;   // constant byte
        digits.push_back(d);
        unsigned long long run = 0;
        for (int x = 0; x < 256; ++x) {
            bases.push_back(run);
            run += h[x];
        }
    }
    if (digits.empty()) return true;
    cudaStream_t s = sc.s;
    const int64_t tiles = (m + kSortTile - 1) / kSortTile;
    auto* dbases = sc.Get<unsigned long long>(int64_t(bases.size()));
    auto* status = sc.Get<unsigned long long>(tiles * 256);
    auto* counter = sc.Get<unsigned int>(1);
    auto* derr = sc.Get<int>(1);
    uint32_t* kbuf[2] = {sc.Get<uint32_t>(m), sc.Get<uint32_t>(m)};
    uint32_t* ibuf[2] = {sc.Get<uint32_t>(m), sc.Get<uint32_t>(m)};
    if (!dbases || !status || !counter || !derr || !kbuf[0] || !kbuf[1] || !ibuf[0] || !ibuf[1]) return false;
    cudaMemcpyAsync(dbases, bases.data(), bases.size() * 8, cudaMemcpyHostToDevice, s);
    cudaMemsetAsync(status, 0, size_t(tiles) * 256 * 8, s);
    cudaMemsetAsync(derr, 0, sizeof(int), s);
    const void* kin = keys;
    const uint32_t* idx = nullptr;
    int cur = 0;
    for (size_t p = 0; p < digits.size(); ++p) {
        SortPass(false, kin, idx, false, kbuf[cur], ibuf[cur], m, 8 * digits[p], dbases + p * 256, status,
                 uint32_t(p + 1), counter, derr, s);
        kin = kbuf[cur];
        idx = ibuf[cur];
        cur ^= 1;
    }
    int herr = 0;
    cudaMemcpyAsync(&herr, derr, sizeof(int), cudaMemcpyDeviceToHost, s);
    if (!CudaOk(cudaStreamSynchronize(s), "shuffle order")) return false;
    if (herr) {
        SetErr("shuffle order: device error %d", herr);
        return false;
    }
    *perm = const_cast<uint32_t*>(idx);
    return true;
}

}  // namespace

}  // namespace qdb

using namespace qdb;

extern "C" {

int64_t qdb_gpu_shuffle(const qdb_gpu_program* prog, qdb_rowset* batch, const int64_t* routes, int64_t n_routes,
                        int64_t n_outputs, qdb_rowset* outs) {
    t_error.clear();
    if (!prog || prog->kind != PK_HASH || !batch || !outs || n_outputs < 1 || n_outputs > kMaxOutputs ||
        n_routes < 0 || n_routes > kMaxOutputs || (n_routes > 0 && !routes)) {
        SetErr("shuffle: bad arguments (a hash program, 1..%d outputs, at most as many routes)", kMaxOutputs);
        return -1;
    }
    const std::vector<qdb_column_type>& types = prog->columns;
    const int ncols = int(types.size());
    if (batch->ColumnCount < ncols) {
        SetErr("shuffle: the batch has %lld columns, the program's schema %d", (long long)batch->ColumnCount, ncols);
        return -1;
    }
    for (const qdb_column_type& t : types) {
        if (t.type == QDB_TYPE_BOOL) {
            SetErr("shuffle: bit-packed BOOL columns are not served");
            return -1;
        }
        if (t.type == QDB_TYPE_STRING) {
            SetErr("shuffle: string columns are hashed (qdb_gpu_hash) but not gathered");
            return -1;
        }
    }
    const int64_t n = batch->RowCount;
    cudaStream_t s = CurStream();
    Staging stg(s);
    CallScratch sc(s);

    // Hashes: the batch's own, or the key hash.
    const uint64_t* hashes = nullptr;
    if (batch->Hash) {
        hashes = static_cast<const uint64_t*>(stg.Device(batch->Hash, size_t(n) * 8));
    } else if (n > 0) {
        AggPlan plan = prog->expr.plan;
        if (!ResolveColumns(plan, prog->expr.cols, types.data(), batch, stg)) return -1;
        auto* h = sc.Get<uint64_t>(n);
        if (!h) return -1;
        ExprArgs a;
        HashArgs(prog, plan, n, a);
        a.hashes = h;
        HashRows(a, s);
        hashes = h;
    }
    const uint8_t* sel = batch->Selection ? static_cast<const uint8_t*>(stg.Device(batch->Selection, size_t(n)))
                                          : nullptr;
    int32_t* droutes = nullptr;
    if (n_routes > 0) {
        std::vector<int32_t> r32(static_cast<size_t>(n_routes));
        for (int64_t i = 0; i < n_routes; ++i) {
            r32[size_t(i)] = (routes[i] < 0 || routes[i] >= n_outputs) ? -1 : int32_t(routes[i]);
        }
        droutes = sc.Get<int32_t>(n_routes);
        if (!droutes) return -1;
        cudaMemcpyAsync(droutes, r32.data(), size_t(n_routes) * 4, cudaMemcpyHostToDevice, s);
    }
    auto* dst = sc.Get<uint32_t>(n);
    auto* flags = sc.Get<uint8_t>(n);
    auto* dcounts = sc.Get<unsigned long long>(n_outputs);
    auto* derr = sc.Get<int>(1);
    auto* sel_rows = sc.Get<int64_t>(n);
    auto* dcount = sc.Get<unsigned long long>(1);
    auto* cscratch = sc.Get<char>(int64_t(CompactScratch(std::max<int64_t>(n, 1))));
    if (!dst || !flags || !dcounts || !derr || !sel_rows || !dcount || !cscratch) return -1;
    cudaMemsetAsync(dcounts, 0, size_t(n_outputs) * 8, s);
    cudaMemsetAsync(derr, 0, sizeof(int), s);
    ProfileBegin(s, "shuffle_route", n);
    if (n > 0) {
        RouteKernel<<<Grid(n), 256, 0, s>>>(hashes, sel, n, droutes, n_routes, n_outputs, dst, flags, dcounts, derr);
        CountLaunch();
    }
    ProfileEnd(s);
    CompactFlags(flags, n, sel_rows, dcount, cscratch, s);
    std::vector<unsigned long long> counts(static_cast<size_t>(n_outputs));
    unsigned long long m = 0;
    int herr = 0;
    cudaMemcpyAsync(counts.data(), dcounts, size_t(n_outputs) * 8, cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(&m, dcount, 8, cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(&herr, derr, sizeof(int), cudaMemcpyDeviceToHost, s);
    if (!CudaOk(cudaStreamSynchronize(s), "shuffle route")) return -1;
    if (herr) {
        SetErr("shuffle: a row's partition is routed nowhere (route outside [0, %lld))", (long long)n_outputs);
        return -1;
    }
    const int64_t rows = int64_t(m);

    // Rows in output order, stable in input order.
    auto* keys = sc.Get<uint32_t>(rows);
    auto* order = sc.Get<int64_t>(rows);
    if (!keys || !order) return -1;
    if (rows > 0) {
        GatherDstKernel<<<Grid(rows), 256, 0, s>>>(dst, sel_rows, rows, keys);
        CountLaunch();
    }
    uint32_t* perm = nullptr;
    if (!StableOrder(keys, rows, counts, &perm, sc)) return -1;
    if (rows > 0) {
        PermuteRowsKernel<<<Grid(rows), 256, 0, s>>>(sel_rows, perm, rows, order);
        CountLaunch();
    }

    // One gather per column into buffers the outputs slice.
    auto owner = std::make_shared<ShuffleOutputs>();
    owner->s = s;
    std::vector<int> otypes;
    for (const qdb_column_type& t : types) otypes.push_back(t.type);
    std::vector<AggOutputCol> cols;
    if (!AllocOutputCols(otypes, std::max<int64_t>(rows, 1), true, cols, s)) {
        SetErr("shuffle: allocation failed");
        return -1;
    }
    for (auto& c : cols) {
        owner->dev.push_back(c.data);
        if (c.valid) owner->dev.push_back(c.valid);
        if (c.offsets) owner->dev.push_back(c.offsets);
    }
    auto* hout = static_cast<uint64_t*>(DevAlloc(size_t(std::max<int64_t>(rows, 1)) * 8, s));
    if (!hout) return -1;
    owner->dev.push_back(hout);
    ProfileBegin(s, "shuffle_gather", rows);
    for (int k = 0; k < ncols; ++k) {
        const qdb_column& c = batch->Columns[k];
        const int w = StorageWidth(types[size_t(k)].type);
        const char* d = static_cast<const char*>(stg.Device(c.Data, size_t(n) * w));
        if (n > 0 && !d) {
            if (t_error.empty()) SetErr("shuffle: column %d has no data", k);
            return -1;
        }
        GatherColumn(d, w, order, 1, rows, cols[size_t(k)].data, s);
        const uint8_t* mk =
            c.Mask ? static_cast<const uint8_t*>(stg.Device(c.Mask, size_t((c.MaskBitOffset + n + 7) / 8))) : nullptr;
        GatherValidity(mk, c.MaskBitOffset, order, 1, rows, cols[size_t(k)].valid, 0, s);
        if (cols[size_t(k)].offsets) {
            IotaI32Kernel<<<Grid(rows + 1), 256, 0, s>>>(cols[size_t(k)].offsets, rows + 1);
            CountLaunch();
        }
    }
    if (rows > 0) {
        GatherU64Kernel<<<Grid(rows), 256, 0, s>>>(hashes, order, rows, hout);
        CountLaunch();
    }
    ProfileEnd(s);
    if (!CudaOk(cudaStreamSynchronize(s), "shuffle gather")) return -1;

    int64_t off = 0;
    for (int64_t p = 0; p < n_outputs; ++p) {
        auto* sl = new ShuffleSlice();
        sl->owner = owner;
        sl->cols.resize(size_t(ncols));
        for (int k = 0; k < ncols; ++k) {
            qdb_column& c = sl->cols[size_t(k)];
            std::memset(&c, 0, sizeof(c));
            const AggOutputCol& oc = cols[size_t(k)];
            c.Data = oc.data + size_t(off) * StorageWidth(otypes[size_t(k)]);
            if (types[size_t(k)].nullable || batch->Columns[k].Mask) {
                c.Mask = reinterpret_cast<const uint8_t*>(oc.valid);
                c.MaskBitOffset = int32_t(off);
            }
            if (oc.offsets) {
                // Absolute positions: a reader subtracts Offsets[0].
                c.Offsets = oc.offsets + off;
                c.OffsetWidth = 4;
            }
        }
        qdb_rowset& o = outs[p];
        std::memset(&o, 0, sizeof(o));
        o.Columns = sl->cols.data();
        o.ColumnCount = ncols;
        o.RowCount = int64_t(counts[size_t(p)]);
        o.Hash = hout + off;
        o.Destroy = DestroyShuffleSlice;
        o.Private = sl;
        o.RefCount = 1;
        off += int64_t(counts[size_t(p)]);
    }
    return rows;
}

}  // extern "C"
