// sort.cu — ORDER BY over packed row ids and top-K selection for sm_100a.
//
// The engine sorts row ids key by key from the last key to the first with a
// stable 8-bit LSD over (radix key, row id), skipping passes whose digit is
// the same for every row (sort_rowids.oz:63-228, compiler.cpp:595-599).  The
// device keeps that pass plan and its stability but reorganises the data:
//
// * one extraction pass reads every row id once, loads each key of the row
//   from the store's batches, writes the stage keys in input order and adds
//   the digit histograms of every pass (an LSD digit's histogram does not
//   depend on the order, so all are known before the first pass and constant
//   digits are skipped up front);
// * every pass is one onesweep kernel: a tile of 4096 (key, u32 position)
//   pairs is ranked in shared memory (warp match + per-warp counters, stable
//   in input order), its per-digit counts are published at once and its
//   global offsets come from a decoupled look-back over earlier tiles; the
//   tile is reordered by digit in shared memory and written out in coalesced
//   runs.  Tiles are taken from an atomic counter, so a tile only ever waits
//   on tiles already running, and every wait is bounded;
// * a stage's first pass gathers its keys through the positions left by the
//   previous stage; the last pass's positions gather the row ids.
//
// Top-K selects a threshold on the first key's order-preserving "primary"
// key by 12-bit radix select (histogram passes), collects the rows at or
// below it and orders only those exactly.
#include <algorithm>

#include "../../include/qdb_gpu.h"
#include "common.cuh"
#include "kernels.h"
#include "sort.h"

namespace qdb {

namespace {

__device__ __forceinline__ bool BitAt(const uint8_t* m, int64_t bit) { return (m[bit >> 3] >> (bit & 7)) & 1; }

// Order-preserving unsigned key of a cell (qumir_radix_key,
// qdb/kernel/sort/radix.oz:4-64): signed integers flip the sign bit; floats
// order as PostgreSQL does (NaN above every number, -0 == +0).  Returns false
// for NULL (key 0).
__device__ __forceinline__ bool CellRadix(const StoreTable& st, int tcol, int type, int64_t id, uint64_t& key,
                                          int* err) {
    key = 0;
    const uint32_t batch = uint32_t(uint64_t(id) >> 32);
    const int64_t row = int64_t(uint32_t(uint64_t(id)));
    if (batch >= uint32_t(st.nbatches)) {
        SetError(err, DE_BAD_ROW_ID);
        return false;
    }
    const int64_t c = int64_t(batch) * st.ncols + tcol;
    const uint8_t* m = st.mask[c];
    if (m && !BitAt(m, st.mask_bit[c] + row)) return false;
    const char* d = st.data[c];
    switch (type) {
        case QDB_TYPE_BOOL: key = BitAt(reinterpret_cast<const uint8_t*>(d), st.data_bit[c] + row); break;
        case QDB_TYPE_I8: key = uint8_t(reinterpret_cast<const int8_t*>(d)[row]) ^ 0x80u; break;
        case QDB_TYPE_U8:
        case QDB_TYPE_CHAR1: key = reinterpret_cast<const uint8_t*>(d)[row]; break;
        case QDB_TYPE_I16: key = uint16_t(reinterpret_cast<const int16_t*>(d)[row]) ^ 0x8000u; break;
        case QDB_TYPE_U16: key = reinterpret_cast<const uint16_t*>(d)[row]; break;
        case QDB_TYPE_I32:
        case QDB_TYPE_DATE32: key = uint32_t(reinterpret_cast<const int32_t*>(d)[row]) ^ 0x80000000u; break;
        case QDB_TYPE_U32: key = reinterpret_cast<const uint32_t*>(d)[row]; break;
        case QDB_TYPE_I64:
        case QDB_TYPE_DECIMAL64: key = uint64_t(reinterpret_cast<const int64_t*>(d)[row]) ^ (1ull << 63); break;
        case QDB_TYPE_U64: key = reinterpret_cast<const uint64_t*>(d)[row]; break;
        case QDB_TYPE_F32: {
            uint32_t b = reinterpret_cast<const uint32_t*>(d)[row];
            const uint32_t mag = b & 0x7fffffffu;
            if (mag > 0x7f800000u) {
                key = 0xffffffffu;
            } else {
                if (mag == 0) b = 0;
                key = (b >> 31) ? uint32_t(~b) : (b ^ 0x80000000u);
            }
            break;
        }
        case QDB_TYPE_F64: {
            uint64_t b = reinterpret_cast<const uint64_t*>(d)[row];
            const uint64_t mag = b & 0x7fffffffffffffffull;
            if (mag > 0x7ff0000000000000ull) {
                key = ~0ull;
            } else {
                if (mag == 0) b = 0;
                key = (b >> 63) ? ~b : (b ^ (1ull << 63));
            }
            break;
        }
        default: SetError(err, DE_BAD_ROW_ID); return false;
    }
    return true;
}

__device__ __forceinline__ uint64_t KeyMask(int bits) { return bits >= 64 ? ~0ull : ((1ull << bits) - 1); }

// The key one stage sorts on.
__device__ __forceinline__ uint64_t StageKey(const StoreTable& st, const SortStage& sg, int64_t id, int* err) {
    if (sg.src == SS_ROW_ID) return uint64_t(id);
    uint64_t k;
    const bool valid = CellRadix(st, sg.tcol, sg.type, id, k, err);
    const uint64_t rank = sg.nulls_first ? (valid ? 1 : 0) : (valid ? 0 : 1);
    if (sg.src == SS_NULL_RANK) return rank;
    const int bits = SortKeyBits(sg.type);
    if (valid && sg.desc) k = ~k & KeyMask(bits);
    if (sg.nullable && bits <= 32) k |= rank << 32;
    return k;
}

// First-key primary order for top-K: the stage key left-aligned to 64 bits
// with the NULL rank on top.  Non-decreasing along the true order, so the
// rows at or below the K-th smallest primary key contain the true top K.
__device__ __forceinline__ uint64_t PrimaryKey(const StoreTable& st, const SortStage& sg, int64_t id, int* err) {
    uint64_t k;
    const bool valid = CellRadix(st, sg.tcol, sg.type, id, k, err);
    const int bits = SortKeyBits(sg.type);
    if (valid && sg.desc) k = ~k & KeyMask(bits);
    const uint64_t aligned = bits >= 64 ? k : (k << (64 - bits));
    if (!sg.nullable) return aligned;
    const uint64_t rank = sg.nulls_first ? (valid ? 1 : 0) : (valid ? 0 : 1);
    return (rank << 63) | (aligned >> 1);
}

// ---------------------------------------------------------------------------
// Extraction + upfront histograms.
// ---------------------------------------------------------------------------
struct ExtractLaunch {
    const int64_t* ids;
    int64_t n;
    StoreTable st;
    int32_t nstages;
    int32_t pad;
    SortStage stages[kMaxSortStages];
    void* keys[kMaxSortStages];
    unsigned long long* hist;
    int* err;
};

constexpr int kExtractThreads = 256;

__global__ void __launch_bounds__(kExtractThreads) SortExtractKernel(const __grid_constant__ ExtractLaunch a) {
    extern __shared__ unsigned int sh[];   // nstages * kSortDigits * 256
    const int nh = a.nstages * kSortDigits * 256;
    for (int i = threadIdx.x; i < nh; i += blockDim.x) sh[i] = 0;
    __syncthreads();
    const int lane = LaneId();
    const int64_t stride = int64_t(gridDim.x) * blockDim.x;
    for (int64_t base = int64_t(blockIdx.x) * blockDim.x; base < a.n; base += stride) {
        const int64_t i = base + threadIdx.x;
        const bool ok = i < a.n;
        const unsigned act = __ballot_sync(kFull, ok);
        const int64_t id = ok ? a.ids[i] : 0;
        for (int s = 0; s < a.nstages; ++s) {
            const SortStage& sg = a.stages[s];
            const uint64_t k = ok ? StageKey(a.st, sg, id, a.err) : 0;
            if (ok) {
                if (sg.wide) static_cast<uint64_t*>(a.keys[s])[i] = k;
                else static_cast<uint32_t*>(a.keys[s])[i] = uint32_t(k);
            }
            const int nd = sg.wide ? 8 : 4;
            if (ok) {
                for (int d = 0; d < nd; ++d) {
                    const unsigned dig = unsigned(k >> (8 * d)) & 255u;
                    const unsigned peers = __match_any_sync(act, dig);
                    if (lane == __ffs(peers) - 1) {
                        atomicAdd(&sh[(s * kSortDigits + d) * 256 + dig], unsigned(__popc(peers)));
                    }
                }
            }
        }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < nh; i += blockDim.x) {
        if (sh[i]) atomicAdd(&a.hist[i], (unsigned long long)sh[i]);
    }
}

// ---------------------------------------------------------------------------
// Onesweep pass.
// ---------------------------------------------------------------------------
constexpr int kPassThreads = 512;
constexpr int kPassItems = kSortTile / kPassThreads;
constexpr int kPassWarps = kPassThreads / 32;
constexpr unsigned long long kFlagAgg = 1ull << 62;
constexpr unsigned long long kFlagInc = 2ull << 62;
constexpr unsigned long long kValueMask = (1ull << 40) - 1;
constexpr uint32_t kEpochMask = 0x3fffff;

template <typename K>
struct PassLaunch {
    const K* keys_in;
    const uint32_t* idx_in;
    K* keys_out;
    uint32_t* idx_out;
    int64_t n;
    int32_t shift;
    int32_t gather;
    uint32_t epoch;
    int32_t pad;
    const unsigned long long* base;   // 256 bucket bases of this digit
    unsigned long long* status;       // per tile and digit: flag | epoch | count
    unsigned int* tile_counter;
    int* err;
};

__device__ __forceinline__ void StoreVolatile(unsigned long long* p, unsigned long long v) {
    *reinterpret_cast<volatile unsigned long long*>(p) = v;
}
__device__ __forceinline__ unsigned long long LoadVolatile(const unsigned long long* p) {
    return *reinterpret_cast<const volatile unsigned long long*>(p);
}

template <typename K>
__global__ void __launch_bounds__(kPassThreads, 2) SortPassKernel(const __grid_constant__ PassLaunch<K> a) {
    extern __shared__ __align__(16) unsigned char dyn[];
    K* skeys = reinterpret_cast<K*>(dyn);
    uint32_t* sidx = reinterpret_cast<uint32_t*>(dyn + size_t(kSortTile) * sizeof(K));
    __shared__ uint32_t whist[kPassWarps][256];
    __shared__ uint32_t local_off[256];
    __shared__ unsigned long long gbase[256];
    __shared__ uint32_t wsum[8];
    __shared__ uint32_t tile_s;
    const int tid = threadIdx.x;
    const int lane = tid & 31;
    const int w = tid >> 5;
    if (tid == 0) tile_s = atomicAdd(a.tile_counter, 1u);
    for (int i = tid; i < kPassWarps * 256; i += kPassThreads) (&whist[0][0])[i] = 0;
    __syncthreads();
    const int64_t tile = tile_s;
    const int64_t t0 = tile * kSortTile;
    const int tile_n = int(min((long long)kSortTile, (long long)(a.n - t0)));

    K key[kPassItems];
    uint32_t idx[kPassItems];
    uint32_t rank[kPassItems];
#pragma unroll
    for (int j = 0; j < kPassItems; ++j) {
        const int lp = w * (32 * kPassItems) + j * 32 + lane;
        const int64_t p = t0 + lp;
        const bool ok = lp < tile_n;
        idx[j] = ok ? (a.idx_in ? a.idx_in[p] : uint32_t(p)) : 0u;
        key[j] = ok ? (a.gather ? a.keys_in[idx[j]] : a.keys_in[p]) : K(0);
    }
    // Stable rank of every key among the equal digits of its warp's segment.
#pragma unroll
    for (int j = 0; j < kPassItems; ++j) {
        const int lp = w * (32 * kPassItems) + j * 32 + lane;
        const bool ok = lp < tile_n;
        const unsigned act = __ballot_sync(kFull, ok);
        rank[j] = 0;
        if (ok) {
            const unsigned d = unsigned(uint64_t(key[j]) >> a.shift) & 255u;
            const unsigned peers = __match_any_sync(act, d);
            const int leader = __ffs(peers) - 1;
            uint32_t old = 0;
            if (lane == leader) {
                old = whist[w][d];
                whist[w][d] = old + uint32_t(__popc(peers));
            }
            old = __shfl_sync(act, old, leader);
            rank[j] = old + uint32_t(__popc(peers & ((1u << lane) - 1u)));
        }
        __syncwarp();
    }
    __syncthreads();
    if (tid < 256) {
        // Warp prefixes in place, then publish this tile's count at once.
        uint32_t cnt = 0;
        for (int ww = 0; ww < kPassWarps; ++ww) {
            const uint32_t c = whist[ww][tid];
            whist[ww][tid] = cnt;
            cnt += c;
        }
        const unsigned long long ep = (unsigned long long)(a.epoch & kEpochMask) << 40;
        unsigned long long* mine = a.status + tile * 256 + tid;
        StoreVolatile(mine, (tile == 0 ? kFlagInc : kFlagAgg) | ep | cnt);
        // Exclusive scan of the digit counts within the tile (threads 0-255).
        uint32_t v = cnt;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t t = __shfl_up_sync(kFull, v, o);
            if (lane >= o) v += t;
        }
        if (lane == 31) wsum[w] = v;
        asm volatile("bar.sync 1, 256;" ::: "memory");
        uint32_t off = v - cnt;
        for (int ww = 0; ww < w; ++ww) off += wsum[ww];
        local_off[tid] = off;
        // Decoupled look-back: sum earlier tiles' counts until an inclusive one.
        unsigned long long excl = 0;
        if (tile > 0) {
            int64_t t = tile - 1;
            const long long start = clock64();
            while (t >= 0) {
                const unsigned long long s = LoadVolatile(a.status + t * 256 + tid);
                const unsigned flag = unsigned(s >> 62);
                if (flag == 0 || uint32_t((s >> 40) & kEpochMask) != (a.epoch & kEpochMask)) {
                    if (clock64() - start > kSpinCycles) {
                        SetError(a.err, DE_LOOKBACK_TIMEOUT);
                        break;
                    }
                    continue;
                }
                excl += s & kValueMask;
                if (flag == 2) break;
                --t;
            }
            StoreVolatile(mine, kFlagInc | ep | (excl + cnt));
        }
        gbase[tid] = a.base[tid] + excl;
    }
    __syncthreads();
    // Reorder the tile by digit in shared memory, then write coalesced runs.
#pragma unroll
    for (int j = 0; j < kPassItems; ++j) {
        const int lp = w * (32 * kPassItems) + j * 32 + lane;
        if (lp < tile_n) {
            const unsigned d = unsigned(uint64_t(key[j]) >> a.shift) & 255u;
            const uint32_t pos = local_off[d] + whist[w][d] + rank[j];
            if (pos < uint32_t(kSortTile)) {
                skeys[pos] = key[j];
                sidx[pos] = idx[j];
            }
        }
    }
    __syncthreads();
    for (int p = tid; p < tile_n; p += kPassThreads) {
        const K k = skeys[p];
        const unsigned d = unsigned(uint64_t(k) >> a.shift) & 255u;
        const unsigned long long g = gbase[d] + uint64_t(p - int(local_off[d]));
        if (g < (unsigned long long)a.n) {   // only a timed-out look-back can break this
            a.keys_out[g] = k;
            a.idx_out[g] = sidx[p];
        }
    }
}

__global__ void SortGatherIdsKernel(const int64_t* ids, const uint32_t* idx, int64_t n, int64_t* out) {
    for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
        out[i] = ids[idx[i]];
    }
}

__global__ void SortMaxBatchKernel(const int64_t* ids, int64_t n, unsigned long long* out) {
    unsigned long long m = 0;
    for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
        m = max(m, (unsigned long long)(uint64_t(ids[i]) >> 32));
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_xor_sync(kFull, m, o));
    if (LaneId() == 0 && m) atomicMax(out, m);
}

struct MaterializeLaunch {
    StoreTable st;
    int32_t tcol;
    int32_t type;
    int32_t width;
    int32_t pad;
    const int64_t* ids;
    int64_t n;
    char* out;
    uint32_t* valid;
    int* err;
};

__global__ void __launch_bounds__(256) SortMaterializeKernel(const __grid_constant__ MaterializeLaunch a) {
    const int64_t stride = int64_t(gridDim.x) * blockDim.x;
    for (int64_t base = int64_t(blockIdx.x) * blockDim.x; base < a.n; base += stride) {
        const int64_t i = base + threadIdx.x;
        bool ok = false;
        if (i < a.n) {
            const int64_t id = a.ids[i];
            const uint32_t batch = uint32_t(uint64_t(id) >> 32);
            const int64_t row = int64_t(uint32_t(uint64_t(id)));
            char* o = a.out + i * a.width;
            if (batch >= uint32_t(a.st.nbatches)) {
                SetError(a.err, DE_BAD_ROW_ID);
            } else {
                const int64_t c = int64_t(batch) * a.st.ncols + a.tcol;
                const uint8_t* m = a.st.mask[c];
                ok = !m || BitAt(m, a.st.mask_bit[c] + row);
                const char* d = a.st.data[c];
                if (a.type == QDB_TYPE_BOOL) {
                    *o = ok ? char(BitAt(reinterpret_cast<const uint8_t*>(d), a.st.data_bit[c] + row)) : 0;
                } else {
                    switch (a.width) {
                        case 1: *o = ok ? d[row] : 0; break;
                        case 2:
                            *reinterpret_cast<int16_t*>(o) = ok ? reinterpret_cast<const int16_t*>(d)[row] : 0;
                            break;
                        case 4:
                            *reinterpret_cast<int32_t*>(o) = ok ? reinterpret_cast<const int32_t*>(d)[row] : 0;
                            break;
                        case 8:
                            *reinterpret_cast<int64_t*>(o) = ok ? reinterpret_cast<const int64_t*>(d)[row] : 0;
                            break;
                        default: {
                            const int64_t* src = reinterpret_cast<const int64_t*>(d) + 2 * row;
                            reinterpret_cast<int64_t*>(o)[0] = ok ? src[0] : 0;
                            reinterpret_cast<int64_t*>(o)[1] = ok ? src[1] : 0;
                        }
                    }
                }
            }
        }
        // Base is a multiple of 32: one lane writes each validity word.
        const unsigned bits = __ballot_sync(kFull, ok);
        if (LaneId() == 0 && i < a.n) a.valid[i >> 5] = bits;
    }
}

// ---------------------------------------------------------------------------
// Top-K radix select.
// ---------------------------------------------------------------------------
constexpr int kTopKBins = 4096;

struct TopKLaunch {
    const int64_t* ids;
    int64_t n;
    StoreTable st;
    SortStage stage;
    int32_t shift;
    int32_t dbits;
    uint64_t prefix;
    int32_t prefix_bits;
    int32_t pad;
    unsigned long long* counts;
    int64_t* out;
    int64_t out_cap;
    int* err;
};

__device__ __forceinline__ bool UnderPrefix(uint64_t p, uint64_t prefix, int prefix_bits, bool le) {
    if (prefix_bits == 0) return true;
    const uint64_t top = p >> (64 - prefix_bits);
    return le ? top <= prefix : top == prefix;
}

__global__ void __launch_bounds__(256) TopKHistogramKernel(const __grid_constant__ TopKLaunch a) {
    __shared__ unsigned int sh[kTopKBins];
    for (int i = threadIdx.x; i < kTopKBins; i += blockDim.x) sh[i] = 0;
    __syncthreads();
    const int lane = LaneId();
    const uint64_t dmask = (1ull << a.dbits) - 1;
    const int64_t stride = int64_t(gridDim.x) * blockDim.x;
    for (int64_t base = int64_t(blockIdx.x) * blockDim.x; base < a.n; base += stride) {
        const int64_t i = base + threadIdx.x;
        bool in = false;
        unsigned dig = 0;
        if (i < a.n) {
            const uint64_t p = PrimaryKey(a.st, a.stage, a.ids[i], a.err);
            in = UnderPrefix(p, a.prefix, a.prefix_bits, false);
            dig = unsigned((p >> a.shift) & dmask);
        }
        const unsigned act = __ballot_sync(kFull, in);
        if (in) {
            const unsigned peers = __match_any_sync(act, dig);
            if (lane == __ffs(peers) - 1) atomicAdd(&sh[dig], unsigned(__popc(peers)));
        }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < kTopKBins; i += blockDim.x) {
        if (sh[i]) atomicAdd(&a.counts[i], (unsigned long long)sh[i]);
    }
}

__global__ void __launch_bounds__(256) TopKCollectKernel(const __grid_constant__ TopKLaunch a) {
    const int lane = LaneId();
    const int64_t stride = int64_t(gridDim.x) * blockDim.x;
    for (int64_t base = int64_t(blockIdx.x) * blockDim.x; base < a.n; base += stride) {
        const int64_t i = base + threadIdx.x;
        bool in = false;
        int64_t id = 0;
        if (i < a.n) {
            id = a.ids[i];
            in = UnderPrefix(PrimaryKey(a.st, a.stage, id, a.err), a.prefix, a.prefix_bits, true);
        }
        const unsigned m = __ballot_sync(kFull, in);
        if (m == 0) continue;
        unsigned long long at = 0;
        if (lane == __ffs(m) - 1) at = atomicAdd(a.counts, (unsigned long long)__popc(m));
        at = __shfl_sync(kFull, at, __ffs(m) - 1);
        const unsigned long long slot = at + __popc(m & ((1u << lane) - 1u));
        if (in && int64_t(slot) < a.out_cap) a.out[slot] = id;
    }
}

int Blocks(int64_t n, int threads, int per_sm) {
    return int(std::max<int64_t>(1, std::min<int64_t>((n + threads - 1) / threads, int64_t(DeviceSMs()) * per_sm)));
}

}  // namespace

void SortExtract(const int64_t* ids, int64_t n, const StoreTable& st, const SortStage* stages, int nstages,
                 void* const* keys, unsigned long long* hist, int* err, cudaStream_t s) {
    if (n == 0 || nstages == 0) return;
    static thread_local ExtractLaunch L;
    L = ExtractLaunch{};
    L.ids = ids;
    L.n = n;
    L.st = st;
    L.nstages = nstages;
    for (int i = 0; i < nstages; ++i) {
        L.stages[i] = stages[i];
        L.keys[i] = keys[i];
    }
    L.hist = hist;
    L.err = err;
    const size_t smem = size_t(nstages) * kSortDigits * 256 * 4;
    EnsureSmemLimit(reinterpret_cast<const void*>(SortExtractKernel), smem);
    ProfileBegin(s, "sort_extract", n);
    SortExtractKernel<<<Blocks(n, kExtractThreads, 4), kExtractThreads, smem, s>>>(L);
    ProfileEnd(s);
    CountLaunch();
}

void SortPass(bool wide, const void* keys_in, const uint32_t* idx_in, bool gather, void* keys_out, uint32_t* idx_out,
              int64_t n, int shift, const unsigned long long* bucket_base, unsigned long long* status, uint32_t epoch,
              unsigned int* tile_counter, int* err, cudaStream_t s) {
    if (n == 0) return;
    const int64_t tiles = (n + kSortTile - 1) / kSortTile;
    cudaMemsetAsync(tile_counter, 0, sizeof(unsigned int), s);
    auto launch = [&](auto tag) {
        using K = decltype(tag);
        PassLaunch<K> L{};
        L.keys_in = static_cast<const K*>(keys_in);
        L.idx_in = idx_in;
        L.keys_out = static_cast<K*>(keys_out);
        L.idx_out = idx_out;
        L.n = n;
        L.shift = shift;
        L.gather = gather ? 1 : 0;
        L.epoch = epoch;
        L.base = bucket_base;
        L.status = status;
        L.tile_counter = tile_counter;
        L.err = err;
        const size_t smem = size_t(kSortTile) * (sizeof(K) + 4);
        EnsureSmemLimit(reinterpret_cast<const void*>(SortPassKernel<K>), smem);
        ProfileBegin(s, wide ? "sort_pass_u64" : "sort_pass_u32", n);
        SortPassKernel<K><<<int(tiles), kPassThreads, smem, s>>>(L);
        ProfileEnd(s);
        CountLaunch();
    };
    if (wide) launch(uint64_t{});
    else launch(uint32_t{});
}

void SortGatherIds(const int64_t* ids, const uint32_t* idx, int64_t n, int64_t* out, cudaStream_t s) {
    if (n == 0) return;
    ProfileBegin(s, "sort_gather_ids", n);
    SortGatherIdsKernel<<<Blocks(n, 256, 8), 256, 0, s>>>(ids, idx, n, out);
    ProfileEnd(s);
    CountLaunch();
}

void SortMaxBatch(const int64_t* ids, int64_t n, unsigned long long* out, cudaStream_t s) {
    cudaMemsetAsync(out, 0, sizeof(unsigned long long), s);
    if (n == 0) return;
    SortMaxBatchKernel<<<Blocks(n, 256, 8), 256, 0, s>>>(ids, n, out);
    CountLaunch();
}

void SortMaterialize(const StoreTable& st, int tcol, int type, const int64_t* ids, int64_t n, char* out,
                     uint32_t* valid, int* err, cudaStream_t s) {
    if (n == 0) return;
    MaterializeLaunch L{};
    L.st = st;
    L.tcol = tcol;
    L.type = type;
    L.width = type == QDB_TYPE_BOOL ? 1 : std::max(1, SortKeyBits(type) / 8);
    if (type == QDB_TYPE_DECIMAL128) L.width = 16;
    L.ids = ids;
    L.n = n;
    L.out = out;
    L.valid = valid;
    L.err = err;
    ProfileBegin(s, "sort_materialize", n);
    SortMaterializeKernel<<<Blocks(n, 256, 8), 256, 0, s>>>(L);
    ProfileEnd(s);
    CountLaunch();
}

void TopKHistogram(const int64_t* ids, int64_t n, const StoreTable& st, const SortStage& stage, int shift,
                   int dbits, uint64_t prefix, int prefix_bits, unsigned long long* counts, int* err, cudaStream_t s) {
    cudaMemsetAsync(counts, 0, sizeof(unsigned long long) * kTopKBins, s);
    if (n == 0) return;
    TopKLaunch L{};
    L.ids = ids;
    L.n = n;
    L.st = st;
    L.stage = stage;
    L.shift = shift;
    L.dbits = dbits;
    L.prefix = prefix;
    L.prefix_bits = prefix_bits;
    L.counts = counts;
    L.err = err;
    ProfileBegin(s, "topk_histogram", n);
    TopKHistogramKernel<<<Blocks(n, 256, 8), 256, 0, s>>>(L);
    ProfileEnd(s);
    CountLaunch();
}

void TopKCollect(const int64_t* ids, int64_t n, const StoreTable& st, const SortStage& stage, uint64_t prefix,
                 int prefix_bits, int64_t* out, int64_t out_cap, unsigned long long* count, int* err,
                 cudaStream_t s) {
    cudaMemsetAsync(count, 0, sizeof(unsigned long long), s);
    if (n == 0) return;
    TopKLaunch L{};
    L.ids = ids;
    L.n = n;
    L.st = st;
    L.stage = stage;
    L.prefix = prefix;
    L.prefix_bits = prefix_bits;
    L.counts = count;
    L.out = out;
    L.out_cap = out_cap;
    L.err = err;
    ProfileBegin(s, "topk_collect", n);
    TopKCollectKernel<<<Blocks(n, 256, 8), 256, 0, s>>>(L);
    ProfileEnd(s);
    CountLaunch();
}

}  // namespace qdb
