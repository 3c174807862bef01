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
// Top-K picks a threshold on the first key's order-preserving "primary" key
// from an evenly spread sample (or, when the sample misses, by 12-bit radix
// select over histogram passes), collects the rows at or below it in one
// pass and orders only those exactly.
#include <algorithm>

#include "../../include/qdb_gpu.h"
#include "common.cuh"
#include "kernels.h"
#include "sort.h"

namespace qdb {

namespace {

__device__ __forceinline__ bool BitAt(const uint8_t* m, int64_t bit) { return (m[bit >> 3] >> (bit & 7)) & 1; }

// Order-preserving images of float bits (NaN above every number, -0 == +0).
__device__ __forceinline__ uint64_t F32Radix(uint64_t raw) {
    uint32_t b = uint32_t(raw);
    const uint32_t mag = b & 0x7fffffffu;
    b = mag == 0 ? 0u : b;
    const uint32_t k = (b >> 31) ? ~b : (b ^ 0x80000000u);
    return mag > 0x7f800000u ? 0xffffffffu : k;
}

__device__ __forceinline__ uint64_t F64Radix(uint64_t b) {
    const uint64_t mag = b & 0x7fffffffffffffffull;
    b = mag == 0 ? 0ull : b;
    const uint64_t k = (b >> 63) ? ~b : (b ^ (1ull << 63));
    return mag > 0x7ff0000000000000ull ? ~0ull : k;
}


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
// Loads the cell of `row` from column data `d` (W bytes, 0 = one bit at
// data_bit + row).
template <int W>
__device__ __forceinline__ uint64_t LoadCell(const char* d, int64_t data_bit, int64_t row) {
    if constexpr (W == 0) return BitAt(reinterpret_cast<const uint8_t*>(d), data_bit + row);
    if constexpr (W == 1) return reinterpret_cast<const uint8_t*>(d)[row];
    if constexpr (W == 2) return reinterpret_cast<const uint16_t*>(d)[row];
    if constexpr (W == 4) return reinterpret_cast<const uint32_t*>(d)[row];
    if constexpr (W == 8) return reinterpret_cast<const uint64_t*>(d)[row];
    return 0;
}

// StageKey arithmetic on host-derived constants: a key stage is
// valid ? (image ^ dmask) | rank_valid : rank_null, where the image is the
// cell's bits ^ flip (or a float image), dmask inverts the key bits for DESC
// and the rank words carry the NULL rank above keys of <= 32 bits; a NULL-rank
// stage is rank_valid / rank_null alone; a row-id stage is the id.
struct StageCodec {
    uint64_t flip;
    uint64_t dmask;
    uint64_t rank_valid;
    uint64_t rank_null;
    int32_t width;   // cell bytes, 0 = one bit
    int32_t flt;     // 0: integer image, 4: F32, 8: F64
};

struct ExtractLaunch {
    const int64_t* ids;
    int64_t n;
    StoreTable st;
    int32_t nstages;
    int32_t pad;
    SortStage stages[kMaxSortStages];
    StageCodec codec[kMaxSortStages];
    void* keys[kMaxSortStages];
    unsigned long long* hist;
    int* err;
};

constexpr int kExtractThreads = 256;
constexpr int kExtractUnroll = 4;

template <int W, int U>
__device__ __forceinline__ void LoadCells(const char* const (&d)[U], const int64_t (&db)[U], const int64_t (&row)[U],
                                          const bool (&valid)[U], uint64_t (&raw)[U]) {
#pragma unroll
    for (int u = 0; u < U; ++u) raw[u] = valid[u] ? LoadCell<W>(d[u], db[u], row[u]) : 0;
}

// The stage keys of U rows: every row's batch pointers, validity bits and
// cells are loaded before any is used.  A row id outside the store sets
// `bad` and reads nothing (key of a NULL), as CellRadix does.
template <int U>
__device__ __forceinline__ void StageKeys(const StoreTable& st, const SortStage& sg, const StageCodec& sc,
                                          const int64_t (&id)[U], const bool (&live)[U], uint64_t (&k)[U],
                                          bool& bad) {
    if (sg.src == SS_ROW_ID) {
#pragma unroll
        for (int u = 0; u < U; ++u) k[u] = uint64_t(id[u]);
        return;
    }
    bool valid[U];
    int64_t row[U], c[U], db[U];
    const char* d[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
        const uint32_t batch = uint32_t(uint64_t(id[u]) >> 32);
        const bool ok = live[u] && batch < uint32_t(st.nbatches);
        bad = bad || (live[u] && !ok);
        row[u] = int64_t(uint32_t(uint64_t(id[u])));
        c[u] = ok ? int64_t(batch) * st.ncols + sg.tcol : -1;
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
        const uint8_t* m = c[u] >= 0 ? st.mask[c[u]] : nullptr;
        valid[u] = c[u] >= 0 && (m == nullptr || BitAt(m, st.mask_bit[c[u]] + row[u]));
        d[u] = c[u] >= 0 ? st.data[c[u]] : nullptr;
        db[u] = (sc.width == 0 && c[u] >= 0) ? st.data_bit[c[u]] : 0;
    }
    uint64_t raw[U];
    if (sg.src == SS_STR_CHUNK || sg.src == SS_STR_LEN) {
        // NULL strings take key 0: their order is the NULL rank stage's.
#pragma unroll
        for (int u = 0; u < U; ++u) {
            uint64_t key = 0;
            if (valid[u]) {
                const char* off = st.offsets[c[u]];
                int64_t b, e;
                if (sc.width == 8) {
                    b = reinterpret_cast<const int64_t*>(off)[row[u]];
                    e = reinterpret_cast<const int64_t*>(off)[row[u] + 1];
                } else {
                    b = reinterpret_cast<const int32_t*>(off)[row[u]];
                    e = reinterpret_cast<const int32_t*>(off)[row[u] + 1];
                }
                const int64_t len = e - b;
                if (sg.src == SS_STR_LEN) {
                    key = uint64_t(len);
                } else {
                    // The chunk's bytes inside the string (0..8 of them);
                    // every load reads one of the string's own bytes, and
                    // the bytes past its end are masked to zero.
                    const int64_t at = 8 * int64_t(sg.chunk);
                    const int64_t nb = min(int64_t(8), len - at);
                    if (nb > 0) {
                        const uint8_t* p = reinterpret_cast<const uint8_t*>(d[u]) + b + at;
#pragma unroll
                        for (int j = 0; j < 8; ++j) {
                            const uint64_t byte = uint64_t(p[min(int64_t(j), nb - 1)]);
                            const uint64_t keep = j < nb ? 0xffull : 0ull;
                            key |= (byte & keep) << (56 - 8 * j);
                        }
                    }
                }
                key ^= sc.dmask;
            }
            k[u] = key;
        }
        return;
    }
    if (sg.src == SS_NULL_RANK) {
#pragma unroll
        for (int u = 0; u < U; ++u) k[u] = valid[u] ? sc.rank_valid : sc.rank_null;
        return;
    }
    switch (sc.width) {
        case 0: LoadCells<0, U>(d, db, row, valid, raw); break;
        case 1: LoadCells<1, U>(d, db, row, valid, raw); break;
        case 2: LoadCells<2, U>(d, db, row, valid, raw); break;
        case 4: LoadCells<4, U>(d, db, row, valid, raw); break;
        default: LoadCells<8, U>(d, db, row, valid, raw); break;
    }
    if (sc.flt == 4) {
#pragma unroll
        for (int u = 0; u < U; ++u) raw[u] = F32Radix(raw[u]);
    } else if (sc.flt == 8) {
#pragma unroll
        for (int u = 0; u < U; ++u) raw[u] = F64Radix(raw[u]);
    } else {
#pragma unroll
        for (int u = 0; u < U; ++u) raw[u] ^= sc.flip;
    }
#pragma unroll
    for (int u = 0; u < U; ++u) k[u] = valid[u] ? ((raw[u] ^ sc.dmask) | sc.rank_valid) : sc.rank_null;
}

// One row's digit into a shared histogram: a warp whose live lanes share the
// digit (constant high digits) adds once, otherwise each lane adds its own.
__device__ __forceinline__ void HistAdd(unsigned int* bins, unsigned dig, bool live, unsigned act, int lane) {
    const int lead = __ffs(act) - 1;
    const unsigned d0 = __shfl_sync(kFull, dig, lead);
    if (__all_sync(kFull, !live || dig == d0)) {
        if (lane == lead) atomicAdd(&bins[d0], unsigned(__popc(act)));
    } else if (live) {
        atomicAdd(&bins[dig], 1u);
    }
}

__global__ void __launch_bounds__(kExtractThreads) SortExtractKernel(const __grid_constant__ ExtractLaunch a) {
    constexpr int U = kExtractUnroll;
    extern __shared__ unsigned int sh[];   // nstages * kSortDigits * 256
    const int nh = a.nstages * kSortDigits * 256;
    for (int i = threadIdx.x; i < nh; i += blockDim.x) sh[i] = 0;
    __syncthreads();
    const int lane = LaneId();
    const int64_t stride = int64_t(gridDim.x) * blockDim.x * U;
    bool bad = false;
    for (int64_t base = int64_t(blockIdx.x) * blockDim.x * U; base < a.n; base += stride) {
        int64_t id[U];
        bool live[U];
        unsigned act[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int64_t i = base + int64_t(u) * blockDim.x + threadIdx.x;
            live[u] = i < a.n;
            id[u] = live[u] ? a.ids[i] : 0;
            act[u] = __ballot_sync(kFull, live[u]);
        }
        for (int s = 0; s < a.nstages; ++s) {
            const SortStage& sg = a.stages[s];
            uint64_t k[U];
            StageKeys<U>(a.st, sg, a.codec[s], id, live, k, bad);
#pragma unroll
            for (int u = 0; u < U; ++u) {
                if (!live[u]) continue;
                const int64_t i = base + int64_t(u) * blockDim.x + threadIdx.x;
                if (sg.wide) static_cast<uint64_t*>(a.keys[s])[i] = k[u];
                else static_cast<uint32_t*>(a.keys[s])[i] = uint32_t(k[u]);
            }
            const int nd = sg.wide ? 8 : 4;
            unsigned int* hs = sh + s * kSortDigits * 256;
#pragma unroll
            for (int u = 0; u < U; ++u) {
                if (act[u] == 0) continue;
                for (int dg = 0; dg < nd; ++dg) HistAdd(hs + dg * 256, unsigned(k[u] >> (8 * dg)) & 255u, live[u], act[u], lane);
            }
        }
    }
    if (bad) SetError(a.err, DE_BAD_ROW_ID);
    __syncthreads();
    for (int i = threadIdx.x; i < nh; i += blockDim.x) {
        if (sh[i]) atomicAdd(&a.hist[i], (unsigned long long)sh[i]);
    }
}

// ---------------------------------------------------------------------------
// Onesweep pass.
// ---------------------------------------------------------------------------
constexpr int kPassThreads = 256;   // 16 keys per thread; three CTAs per SM
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

// Earlier tiles' states one look-back round trip reads.
constexpr int kLookWindow = 4;

// Shared state of one onesweep tile.
struct PassShared {
    uint32_t whist[kPassWarps][256];
    uint32_t local_off[256];
    unsigned long long gbase[256];
    uint32_t wsum[8];
    uint32_t tile;
};

// One tile of the pass.  FULL: the tile holds kSortTile keys, so no key
// needs a bounds check.
template <typename K, bool FULL>
__device__ __forceinline__ void PassTile(const PassLaunch<K>& a, PassShared& sh, K* skeys, uint32_t* sidx,
                                         int64_t tile, int tile_n) {
    const int tid = threadIdx.x;
    const int lane = tid & 31;
    const int w = tid >> 5;
    const int64_t t0 = tile * kSortTile;

    K key[kPassItems];
    uint32_t idx[kPassItems];
    uint32_t rank[kPassItems];
#pragma unroll
    for (int j = 0; j < kPassItems; ++j) {
        const int lp = w * (32 * kPassItems) + j * 32 + lane;
        const int64_t p = t0 + lp;
        const bool ok = FULL || lp < tile_n;
        idx[j] = ok ? (a.idx_in ? a.idx_in[p] : uint32_t(p)) : 0u;
        key[j] = ok ? (a.gather ? a.keys_in[idx[j]] : a.keys_in[p]) : K(0);
    }
    // Stable rank of every key among the equal digits of its warp's segment.
    // The lanes sharing a digit come from one ballot per digit bit: lane i
    // keeps the ballot where its bit is set and the complement where not.
#pragma unroll
    for (int j = 0; j < kPassItems; ++j) {
        const int lp = w * (32 * kPassItems) + j * 32 + lane;
        const bool ok = FULL || lp < tile_n;
        const unsigned d = unsigned(uint64_t(key[j]) >> a.shift) & 255u;
        const unsigned act = FULL ? kFull : __ballot_sync(kFull, ok);
        unsigned peers = act;
#pragma unroll
        for (int bt = 0; bt < 8; ++bt) {
            const unsigned bit = (d >> bt) & 1u;
            const unsigned set = __ballot_sync(kFull, bit);
            peers &= set ^ (bit - 1u);
        }
        rank[j] = 0;
        if (ok) {
            const int leader = __ffs(peers) - 1;
            uint32_t old = 0;
            if (lane == leader) {
                old = sh.whist[w][d];
                sh.whist[w][d] = old + uint32_t(__popc(peers));
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
#pragma unroll
        for (int ww = 0; ww < kPassWarps; ++ww) {
            const uint32_t c = sh.whist[ww][tid];
            sh.whist[ww][tid] = cnt;
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
        if (lane == 31) sh.wsum[w] = v;
        asm volatile("bar.sync 1, 256;" ::: "memory");
        uint32_t off = v - cnt;
        for (int ww = 0; ww < w; ++ww) off += sh.wsum[ww];
        sh.local_off[tid] = off;
        // Decoupled look-back: sum earlier tiles' counts until an inclusive
        // one, reading a window of kLookWindow earlier tiles per round trip
        // (tile 0 publishes an inclusive count, so no walk passes it).
        unsigned long long excl = 0;
        if (tile > 0) {
            int64_t t = tile - 1;
            const long long start = clock64();
            bool done = false;
            while (!done) {
                unsigned long long st[kLookWindow];
#pragma unroll
                for (int q = 0; q < kLookWindow; ++q) st[q] = t - q >= 0 ? LoadVolatile(a.status + (t - q) * 256 + tid) : 0;
                int used = 0;
#pragma unroll
                for (int q = 0; q < kLookWindow; ++q) {
                    if (done || used < q) break;
                    const unsigned flag = unsigned(st[q] >> 62);
                    if (flag == 0 || uint32_t((st[q] >> 40) & kEpochMask) != (a.epoch & kEpochMask)) break;
                    excl += st[q] & kValueMask;
                    used = q + 1;
                    done = flag == 2;
                }
                t -= used;
                if (!done && used == 0 && clock64() - start > kSpinCycles) {
                    SetError(a.err, DE_LOOKBACK_TIMEOUT);
                    break;
                }
            }
            StoreVolatile(mine, kFlagInc | ep | (excl + cnt));
        }
        sh.gbase[tid] = a.base[tid] + excl;
    }
    __syncthreads();
    // Reorder the tile by digit in shared memory, then write coalesced runs.
#pragma unroll
    for (int j = 0; j < kPassItems; ++j) {
        const int lp = w * (32 * kPassItems) + j * 32 + lane;
        if (FULL || lp < tile_n) {
            const unsigned d = unsigned(uint64_t(key[j]) >> a.shift) & 255u;
            const uint32_t pos = sh.local_off[d] + sh.whist[w][d] + rank[j];
            if (pos < uint32_t(kSortTile)) {
                skeys[pos] = key[j];
                sidx[pos] = idx[j];
            }
        }
    }
    __syncthreads();
#pragma unroll
    for (int j = 0; j < kPassItems; ++j) {
        const int p = tid + j * kPassThreads;
        if (FULL || p < tile_n) {
            const K k = skeys[p];
            const unsigned d = unsigned(uint64_t(k) >> a.shift) & 255u;
            const unsigned long long g = sh.gbase[d] + uint64_t(p - int(sh.local_off[d]));
            if (g < (unsigned long long)a.n) {   // only a timed-out look-back can break this
                a.keys_out[g] = k;
                a.idx_out[g] = sidx[p];
            }
        }
    }
}

template <typename K>
__global__ void __launch_bounds__(kPassThreads, 3) SortPassKernel(const __grid_constant__ PassLaunch<K> a) {
    extern __shared__ __align__(16) unsigned char dyn[];
    K* skeys = reinterpret_cast<K*>(dyn);
    uint32_t* sidx = reinterpret_cast<uint32_t*>(dyn + size_t(kSortTile) * sizeof(K));
    __shared__ PassShared sh;
    const int tid = threadIdx.x;
    if (tid == 0) sh.tile = atomicAdd(a.tile_counter, 1u);
    for (int i = tid; i < kPassWarps * 256; i += kPassThreads) (&sh.whist[0][0])[i] = 0;
    __syncthreads();
    const int64_t tile = sh.tile;
    const int tile_n = int(min((long long)kSortTile, (long long)(a.n - tile * kSortTile)));
    if (tile_n == kSortTile) PassTile<K, true>(a, sh, skeys, sidx, tile, tile_n);
    else PassTile<K, false>(a, sh, skeys, sidx, tile, tile_n);
}

// out[i] = ids[idx[i]], four rows per thread per step with every position
// and then every id load in flight together.  With `tiles` (dense-run marks
// of ids), an id in a dense tile is its tile's first id plus its offset; ids
// is read only for the other tiles (and may be null when there are none).
__global__ void __launch_bounds__(256) SortGatherIdsKernel(const int64_t* ids, const uint32_t* idx, int64_t n,
                                                           const int64_t* tiles, int64_t* out) {
    constexpr int U = 4;
    const int64_t stride = int64_t(gridDim.x) * blockDim.x * U;
    for (int64_t base = int64_t(blockIdx.x) * blockDim.x * U; base < n; base += stride) {
        uint32_t pos[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int64_t i = base + int64_t(u) * blockDim.x + threadIdx.x;
            pos[u] = i < n ? idx[i] : 0;
        }
        int64_t v[U];
        if (tiles) {
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const int64_t i = base + int64_t(u) * blockDim.x + threadIdx.x;
                v[u] = i < n ? tiles[pos[u] / kSortIdTile] : 0;
            }
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const int64_t i = base + int64_t(u) * blockDim.x + threadIdx.x;
                if (i < n) v[u] = v[u] >= 0 ? v[u] + int64_t(pos[u] % kSortIdTile) : ids[pos[u]];
            }
        } else {
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const int64_t i = base + int64_t(u) * blockDim.x + threadIdx.x;
                v[u] = i < n ? ids[pos[u]] : 0;
            }
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int64_t i = base + int64_t(u) * blockDim.x + threadIdx.x;
            if (i < n) out[i] = v[u];
        }
    }
}

// Row ids per warp tile of the id scans: lane l holds positions
// tile * kIdTile + u * 32 + l, u < kIdTile / 32.
constexpr int kIdTile = kSortIdTile;

// Largest batch index among the row ids.  With TILES, also marks every full
// warp tile whose ids are consecutive rows of one batch: tiles[t] = its first
// id, else -1.
template <bool TILES>
__global__ void __launch_bounds__(256) SortMaxBatchKernel(const int64_t* ids, int64_t n, unsigned long long* out,
                                                          int64_t* tiles) {
    constexpr int U = kIdTile / 32;
    const int lane = LaneId();
    const int64_t ntiles = (n + kIdTile - 1) / kIdTile;
    const int64_t warps = int64_t(gridDim.x) * (blockDim.x / 32);
    unsigned long long m = 0, sparse = 0;
    for (int64_t t = int64_t(blockIdx.x) * (blockDim.x / 32) + threadIdx.x / 32; t < ntiles; t += warps) {
        const int64_t base = t * kIdTile;
        int64_t v[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int64_t i = base + u * 32 + lane;
            v[u] = i < n ? ids[i] : 0;
        }
#pragma unroll
        for (int u = 0; u < U; ++u) m = max(m, (unsigned long long)(uint64_t(v[u]) >> 32));
        if constexpr (TILES) {
            const uint64_t first = uint64_t(__shfl_sync(kFull, v[0], 0));
            bool dense = base + kIdTile <= n && int64_t(first) >= 0 &&
                         uint64_t(uint32_t(first)) + (kIdTile - 1) <= 0xffffffffull;
#pragma unroll
            for (int u = 0; u < U; ++u) dense = dense && uint64_t(v[u]) == first + uint64_t(u * 32 + lane);
            dense = __all_sync(kFull, dense);
            if (lane == 0) tiles[t] = dense ? int64_t(first) : -1;
            sparse += dense ? 0 : 1;
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_xor_sync(kFull, m, o));
    if (lane == 0 && m) atomicMax(out, m);
    if (TILES && lane == 0 && sparse) atomicAdd(out + 1, sparse);
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

// PrimaryKey of a loaded cell as straight-line arithmetic on constants the
// host derives from the stage: k = raw ^ flip (integers; floats map their
// bits), DESC xors all key bits, the key is left-aligned by lsh and, when
// nullable, shifted down one bit under its NULL rank.
struct KeyCodec {
    uint64_t flip;
    uint64_t dmask;
    uint64_t rank_valid;   // bit 63 set when a valid cell's NULL rank is 1 (nullable keys)
    uint64_t rank_null;
    int32_t lsh;
    int32_t nsh;
};

struct TopKLaunch {
    const int64_t* ids;
    int64_t n;
    StoreTable st;
    SortStage stage;
    KeyCodec kc;
    int32_t shift;
    int32_t dbits;
    uint64_t hmask;        // histogram: rows with (p & hmask) == hval
    uint64_t hval;
    uint64_t limit;        // collect: rows with p <= limit, or <= *limit_dev when set
    const uint64_t* limit_dev;
    unsigned long long* counts;
    int64_t* out;
    int64_t out_cap;
    const int64_t* tiles;  // dense-run marks of the ids (SortMaxBatch)
    int* err;
};

// PrimaryKey from a cell's validity and raw bits (zero extended); FLT: a
// float cell of W bytes.
template <int W, bool FLT>
__device__ __forceinline__ uint64_t PrimaryOf(const KeyCodec& kc, bool valid, uint64_t raw) {
    uint64_t k;
    if constexpr (FLT) k = W == 4 ? F32Radix(raw) : F64Radix(raw);
    else k = raw ^ kc.flip;
    k = valid ? (k ^ kc.dmask) : 0;
    return ((k << kc.lsh) >> kc.nsh) | (valid ? kc.rank_valid : kc.rank_null);
}

// PrimaryKey of U rows at once: every row's batch pointers, then every row's
// validity bit, then every row's cell are loaded before any is used, so a
// thread keeps U row fetches in flight instead of one dependent chain.  A
// row id outside the store sets `bad` and reads nothing (key 0, NULL), as
// CellRadix does; a NULL cell's data is not read.
template <int W, bool FLT, int U>
__device__ __forceinline__ void PrimaryKeys(const StoreTable& st, const SortStage& sg, const KeyCodec& kc,
                                            const int64_t (&id)[U], const bool (&live)[U], uint64_t (&p)[U],
                                            bool& bad) {
    bool ok[U];
    int64_t row[U], c[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
        const uint32_t batch = uint32_t(uint64_t(id[u]) >> 32);
        ok[u] = live[u] && batch < uint32_t(st.nbatches);
        bad = bad || (live[u] && !ok[u]);
        row[u] = int64_t(uint32_t(uint64_t(id[u])));
        c[u] = ok[u] ? int64_t(batch) * st.ncols + sg.tcol : 0;
    }
    const char* d[U];
    const uint8_t* m[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
        d[u] = ok[u] ? st.data[c[u]] : nullptr;
        m[u] = ok[u] ? st.mask[c[u]] : nullptr;
    }
    bool valid[U];
#pragma unroll
    for (int u = 0; u < U; ++u) valid[u] = ok[u] && (m[u] == nullptr || BitAt(m[u], st.mask_bit[c[u]] + row[u]));
    uint64_t raw[U];
#pragma unroll
    for (int u = 0; u < U; ++u) raw[u] = valid[u] ? LoadCell<W>(d[u], W == 0 ? st.data_bit[c[u]] : 0, row[u]) : 0;
#pragma unroll
    for (int u = 0; u < U; ++u) p[u] = PrimaryOf<W, FLT>(kc, valid[u], raw[u]);
}

// PrimaryKeys of the U rows a lane holds in a dense tile: rows
// row0 + u * 32 + lane of the batch of `first`, whose pointers are looked up
// once.  The caller has checked the batch.
template <int W, bool FLT, int U>
__device__ __forceinline__ void DenseKeys(const StoreTable& st, const SortStage& sg, const KeyCodec& kc,
                                          int64_t first, int lane, uint64_t (&p)[U]) {
    const int64_t c = int64_t(uint64_t(first) >> 32) * st.ncols + sg.tcol;
    const int64_t row0 = int64_t(uint32_t(uint64_t(first))) + lane;
    const char* d = st.data[c];
    const uint8_t* m = st.mask[c];
    const int64_t db = W == 0 ? st.data_bit[c] : 0;
    uint64_t raw[U];
    if (m == nullptr) {
#pragma unroll
        for (int u = 0; u < U; ++u) raw[u] = LoadCell<W>(d, db, row0 + u * 32);
#pragma unroll
        for (int u = 0; u < U; ++u) p[u] = PrimaryOf<W, FLT>(kc, true, raw[u]);
    } else {
        const int64_t mb = st.mask_bit[c] + row0;
        bool valid[U];
#pragma unroll
        for (int u = 0; u < U; ++u) valid[u] = BitAt(m, mb + u * 32);
#pragma unroll
        for (int u = 0; u < U; ++u) raw[u] = valid[u] ? LoadCell<W>(d, db, row0 + u * 32) : 0;
#pragma unroll
        for (int u = 0; u < U; ++u) p[u] = PrimaryOf<W, FLT>(kc, valid[u], raw[u]);
    }
}

// Rows per thread per step of the top-K passes.
constexpr int kTopKUnroll = 4;

// Row ids of one step: thread t takes rows base + u * blockDim.x + t.
template <int U>
__device__ __forceinline__ void TopKIds(const TopKLaunch& a, int64_t base, int64_t (&id)[U], bool (&live)[U]) {
#pragma unroll
    for (int u = 0; u < U; ++u) {
        const int64_t i = base + int64_t(u) * blockDim.x + threadIdx.x;
        live[u] = i < a.n;
        id[u] = live[u] ? a.ids[i] : 0;
    }
}

template <int W, bool FLT>
__global__ void __launch_bounds__(256) TopKHistogramKernel(const __grid_constant__ TopKLaunch a) {
    constexpr int U = kTopKUnroll;
    __shared__ unsigned int sh[kTopKBins];
    for (int i = threadIdx.x; i < kTopKBins; i += blockDim.x) sh[i] = 0;
    __syncthreads();
    const int lane = LaneId();
    const uint64_t dmask = (1ull << a.dbits) - 1;
    const int64_t stride = int64_t(gridDim.x) * blockDim.x * U;
    bool bad = false;
    for (int64_t base = int64_t(blockIdx.x) * blockDim.x * U; base < a.n; base += stride) {
        int64_t id[U];
        bool live[U];
        uint64_t p[U];
        TopKIds<U>(a, base, id, live);
        PrimaryKeys<W, FLT, U>(a.st, a.stage, a.kc, id, live, p, bad);
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const bool in = live[u] && (p[u] & a.hmask) == a.hval;
            const unsigned dig = unsigned((p[u] >> a.shift) & dmask);
            const unsigned act = __ballot_sync(kFull, in);
            if (in) {
                const unsigned peers = __match_any_sync(act, dig);
                if (lane == __ffs(peers) - 1) atomicAdd(&sh[dig], unsigned(__popc(peers)));
            }
        }
    }
    if (bad) SetError(a.err, DE_BAD_ROW_ID);
    __syncthreads();
    for (int i = threadIdx.x; i < kTopKBins; i += blockDim.x) {
        if (sh[i]) atomicAdd(&a.counts[i], (unsigned long long)sh[i]);
    }
}

// Appends the row ids of the lanes with `in` to a.out (first a.out_cap
// slots) and counts them in *a.counts.
__device__ __forceinline__ void TopKAppend(const TopKLaunch& a, bool in, int64_t id, int lane) {
    const unsigned m = __ballot_sync(kFull, in);
    if (m == 0) return;
    unsigned long long at = 0;
    if (lane == __ffs(m) - 1) at = atomicAdd(a.counts, (unsigned long long)__popc(m));
    at = __shfl_sync(kFull, at, __ffs(m) - 1);
    const unsigned long long slot = at + __popc(m & ((1u << lane) - 1u));
    if (in && int64_t(slot) < a.out_cap) a.out[slot] = id;
}

// Collects the rows at or below the threshold, one warp tile of the ids at a
// time.  A tile of consecutive rows of one batch (a.tiles) reads no ids and
// looks its column up once, so each lane's U cells are independent loads;
// the next tile's mark is loaded while this one's cells are in flight, and
// a tile with no row at or below the threshold (nearly all of them) costs
// one vote.  Any other tile takes the general fetch, H rows per lane at a
// time.
template <int W, bool FLT>
__global__ void __launch_bounds__(256, 4) TopKCollectKernel(const __grid_constant__ TopKLaunch a) {
    constexpr int U = kIdTile / 32;
    constexpr int H = 2;
    const int lane = LaneId();
    const int64_t ntiles = (a.n + kIdTile - 1) / kIdTile;
    const int64_t warps = int64_t(gridDim.x) * (blockDim.x / 32);
    const uint64_t limit = a.limit_dev ? *a.limit_dev : a.limit;
    bool bad = false;
    int64_t t = int64_t(blockIdx.x) * (blockDim.x / 32) + threadIdx.x / 32;
    int64_t next = t < ntiles ? a.tiles[t] : -1;
    for (; t < ntiles; t += warps) {
        const int64_t first = next;
        next = t + warps < ntiles ? a.tiles[t + warps] : -1;
        if (first >= 0 && uint32_t(uint64_t(first) >> 32) < uint32_t(a.st.nbatches)) {
            uint64_t p[U];
            DenseKeys<W, FLT, U>(a.st, a.stage, a.kc, first, lane, p);
            bool any = false;
#pragma unroll
            for (int u = 0; u < U; ++u) any = any || p[u] <= limit;
            if (__any_sync(kFull, any)) {
#pragma unroll
                for (int u = 0; u < U; ++u) TopKAppend(a, p[u] <= limit, first + u * 32 + lane, lane);
            }
        } else {
#pragma unroll
            for (int h = 0; h < U; h += H) {
                int64_t id[H];
                bool live[H];
                uint64_t p[H];
#pragma unroll
                for (int u = 0; u < H; ++u) {
                    const int64_t i = t * kIdTile + (h + u) * 32 + lane;
                    live[u] = i < a.n;
                    id[u] = live[u] ? a.ids[i] : 0;
                }
                PrimaryKeys<W, FLT, H>(a.st, a.stage, a.kc, id, live, p, bad);
#pragma unroll
                for (int u = 0; u < H; ++u) TopKAppend(a, live[u] && p[u] <= limit, id[u], lane);
            }
        }
    }
    if (bad) SetError(a.err, DE_BAD_ROW_ID);
}

__global__ void TopKSampleKernel(const __grid_constant__ TopKLaunch a, uint64_t* keys, int64_t ns) {
    const int64_t j = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (j >= ns) return;
    keys[j] = PrimaryKey(a.st, a.stage, a.ids[j * a.n / ns], a.err);
}

// The r-th smallest (1-based) of keys[0, ns) into *out, by one block of
// 1024 threads: eight rounds of an 8-bit radix select, most significant
// digit first, each a shared histogram of the keys still under the prefix
// and a one-warp scan for the digit holding the r-th key.
__global__ void __launch_bounds__(1024) TopKSelectKernel(const uint64_t* keys, int64_t ns, int64_t r,
                                                          uint64_t* out) {
    __shared__ unsigned int hist[256];
    __shared__ uint64_t s_prefix;
    __shared__ unsigned long long s_need;
    if (threadIdx.x == 0) {
        s_prefix = 0;
        s_need = (unsigned long long)r;
    }
    uint64_t mask = 0;
    for (int shift = 56; shift >= 0; shift -= 8) {
        for (int i = threadIdx.x; i < 256; i += blockDim.x) hist[i] = 0;
        __syncthreads();
        const uint64_t prefix = s_prefix;
        for (int64_t i = threadIdx.x; i < ns; i += blockDim.x) {
            const uint64_t k = keys[i];
            if ((k & mask) == prefix) atomicAdd(&hist[(k >> shift) & 255], 1u);
        }
        __syncthreads();
        if (threadIdx.x < 32) {
            const int lane = threadIdx.x;
            unsigned long long c[8], own = 0;
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                c[j] = hist[lane * 8 + j];
                own += c[j];
            }
            unsigned long long incl = own;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const unsigned long long v = __shfl_up_sync(kFull, incl, o);
                if (lane >= o) incl += v;
            }
            const unsigned long long need = s_need;
            const unsigned long long before = incl - own;
            const unsigned hit = __ballot_sync(kFull, incl >= need);
            if (hit && lane == __ffs(hit) - 1) {
                unsigned long long run = before;
                int j = 0;
                for (; j < 7; ++j) {
                    if (run + c[j] >= need) break;
                    run += c[j];
                }
                s_need = need - run;
                s_prefix = prefix | (uint64_t(lane * 8 + j) << shift);
            }
        }
        mask |= 0xffull << shift;
        __syncthreads();
    }
    if (threadIdx.x == 0) *out = s_prefix;
}

using TopKKernel = void (*)(const TopKLaunch);

// Kernel instances for the first key's type: cell width, and float or not.
TopKKernel TopKHistogramFor(int type) {
    switch (type) {
        case QDB_TYPE_F32: return TopKHistogramKernel<4, true>;
        case QDB_TYPE_F64: return TopKHistogramKernel<8, true>;
        default: break;
    }
    switch (SortKeyWidth(type)) {
        case 0: return TopKHistogramKernel<0, false>;
        case 1: return TopKHistogramKernel<1, false>;
        case 2: return TopKHistogramKernel<2, false>;
        case 4: return TopKHistogramKernel<4, false>;
        case 8: return TopKHistogramKernel<8, false>;
        default: return nullptr;
    }
}

TopKKernel TopKCollectFor(int type) {
    switch (type) {
        case QDB_TYPE_F32: return TopKCollectKernel<4, true>;
        case QDB_TYPE_F64: return TopKCollectKernel<8, true>;
        default: break;
    }
    switch (SortKeyWidth(type)) {
        case 0: return TopKCollectKernel<0, false>;
        case 1: return TopKCollectKernel<1, false>;
        case 2: return TopKCollectKernel<2, false>;
        case 4: return TopKCollectKernel<4, false>;
        case 8: return TopKCollectKernel<8, false>;
        default: return nullptr;
    }
}

// The codec of a stage's primary key (PrimaryKey's arithmetic).
KeyCodec CodecOf(const SortStage& sg) {
    KeyCodec kc{};
    const int bits = SortKeyBits(sg.type);
    switch (sg.type) {
        case QDB_TYPE_I8: kc.flip = 0x80u; break;
        case QDB_TYPE_I16: kc.flip = 0x8000u; break;
        case QDB_TYPE_I32:
        case QDB_TYPE_DATE32: kc.flip = 0x80000000u; break;
        case QDB_TYPE_I64:
        case QDB_TYPE_DECIMAL64: kc.flip = 1ull << 63; break;
        default: kc.flip = 0; break;
    }
    kc.dmask = sg.desc ? (bits >= 64 ? ~0ull : ((1ull << bits) - 1)) : 0;
    kc.lsh = 64 - bits;
    kc.nsh = sg.nullable ? 1 : 0;
    if (sg.nullable) {
        kc.rank_valid = sg.nulls_first ? (1ull << 63) : 0;
        kc.rank_null = sg.nulls_first ? 0 : (1ull << 63);
    }
    return kc;
}

// The codec of a stage (StageKey's arithmetic).
StageCodec StageCodecOf(const SortStage& sg) {
    StageCodec c{};
    if (sg.src == SS_STR_CHUNK || sg.src == SS_STR_LEN) {
        c.width = sg.owidth;
        c.dmask = sg.desc ? ~0ull : 0ull;
        return c;
    }
    const int bits = SortKeyBits(sg.type);
    c.width = SortKeyWidth(sg.type) < 0 ? 8 : SortKeyWidth(sg.type);
    c.flt = sg.type == QDB_TYPE_F32 ? 4 : (sg.type == QDB_TYPE_F64 ? 8 : 0);
    switch (sg.type) {
        case QDB_TYPE_I8: c.flip = 0x80u; break;
        case QDB_TYPE_I16: c.flip = 0x8000u; break;
        case QDB_TYPE_I32:
        case QDB_TYPE_DATE32: c.flip = 0x80000000u; break;
        case QDB_TYPE_I64:
        case QDB_TYPE_DECIMAL64: c.flip = 1ull << 63; break;
        default: c.flip = 0; break;
    }
    c.dmask = sg.desc ? (bits >= 64 ? ~0ull : ((1ull << bits) - 1)) : 0;
    const uint64_t rv = sg.nulls_first ? 1 : 0, rn = sg.nulls_first ? 0 : 1;
    if (sg.src == SS_NULL_RANK) {
        c.rank_valid = rv;
        c.rank_null = rn;
    } else if (sg.nullable && bits <= 32) {
        c.rank_valid = rv << 32;
        c.rank_null = rn << 32;
    }
    return c;
}

int Blocks(int64_t n, int threads, int per_sm) {
    return int(std::max<int64_t>(1, std::min<int64_t>((n + threads - 1) / threads, int64_t(DeviceSMs()) * per_sm)));
}

}  // namespace

__global__ void __launch_bounds__(256) SortStringMaxLenKernel(const int64_t* ids, int64_t n, StoreTable st, int tcol,
                                                              int owidth, unsigned long long* out, int* err) {
    unsigned long long m = 0;
    bool bad = false;
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
        const uint32_t batch = uint32_t(uint64_t(ids[i]) >> 32);
        const int64_t row = int64_t(uint32_t(uint64_t(ids[i])));
        if (batch >= uint32_t(st.nbatches)) {
            bad = true;
            continue;
        }
        const char* off = st.offsets[int64_t(batch) * st.ncols + tcol];
        const int64_t len = owidth == 8 ? reinterpret_cast<const int64_t*>(off)[row + 1] -
                                              reinterpret_cast<const int64_t*>(off)[row]
                                        : int64_t(reinterpret_cast<const int32_t*>(off)[row + 1]) -
                                              int64_t(reinterpret_cast<const int32_t*>(off)[row]);
        m = max(m, (unsigned long long)max(len, int64_t(0)));
    }
    m = WarpMaxU64(m);
    if (LaneId() == 0 && m) atomicMax(out, m);
    if (bad) SetError(err, DE_BAD_ROW_ID);
}

void SortStringMaxLen(const int64_t* ids, int64_t n, const StoreTable& st, int tcol, int owidth,
                      unsigned long long* out, int* err, cudaStream_t s) {
    if (n == 0) return;
    ProfileBegin(s, "sort_string_len", n);
    SortStringMaxLenKernel<<<Blocks(n, 256, 4), 256, 0, s>>>(ids, n, st, tcol, owidth, out, err);
    ProfileEnd(s);
    CountLaunch();
}

void SortExtract(const int64_t* ids, int64_t n, const StoreTable& st, const SortStage* stages, int nstages,
                 void* const* keys, unsigned long long* hist, int* err, cudaStream_t s) {
    if (n == 0 || nstages == 0) return;
    // At most kMaxSortStages stages per launch (their histograms live in
    // shared memory); more go in further launches.
    if (nstages > kMaxSortStages) {
        for (int g = 0; g < nstages; g += kMaxSortStages) {
            const int m = std::min(kMaxSortStages, nstages - g);
            SortExtract(ids, n, st, stages + g, m, keys + g, hist + size_t(g) * kSortDigits * 256, err, s);
        }
        return;
    }
    static thread_local ExtractLaunch L;
    L = ExtractLaunch{};
    L.ids = ids;
    L.n = n;
    L.st = st;
    L.nstages = nstages;
    for (int i = 0; i < nstages; ++i) {
        L.stages[i] = stages[i];
        L.codec[i] = StageCodecOf(stages[i]);
        L.keys[i] = keys[i];
    }
    L.hist = hist;
    L.err = err;
    const size_t smem = size_t(nstages) * kSortDigits * 256 * 4;
    EnsureSmemLimit(reinterpret_cast<const void*>(SortExtractKernel), smem);
    ProfileBegin(s, "sort_extract", n);
    SortExtractKernel<<<Blocks((n + kExtractUnroll - 1) / kExtractUnroll, kExtractThreads, 4), kExtractThreads, smem,
                        s>>>(L);
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

void SortGatherIds(const int64_t* ids, const uint32_t* idx, int64_t n, const int64_t* tiles, int64_t* out,
                   cudaStream_t s) {
    if (n == 0) return;
    ProfileBegin(s, "sort_gather_ids", n);
    SortGatherIdsKernel<<<Blocks((n + 3) / 4, 256, 8), 256, 0, s>>>(ids, idx, n, tiles, out);
    ProfileEnd(s);
    CountLaunch();
}

void SortMaxBatch(const int64_t* ids, int64_t n, unsigned long long* out, int64_t* tiles, cudaStream_t s) {
    cudaMemsetAsync(out, 0, sizeof(unsigned long long) * (tiles ? 2 : 1), s);
    if (n == 0) return;
    ProfileBegin(s, "sort_max_batch", n);
    const int64_t threads = (n + kIdTile - 1) / kIdTile * 32;
    if (tiles)
        SortMaxBatchKernel<true><<<Blocks(threads, 256, 8), 256, 0, s>>>(ids, n, out, tiles);
    else
        SortMaxBatchKernel<false><<<Blocks(threads, 256, 8), 256, 0, s>>>(ids, n, out, nullptr);
    ProfileEnd(s);
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

void TopKThreshold(const int64_t* ids, int64_t n, const StoreTable& st, const SortStage& stage, uint64_t* keys,
                   int64_t n_samples, int64_t r, uint64_t* out, int* err, cudaStream_t s) {
    if (n == 0 || n_samples == 0) return;
    TopKLaunch L{};
    L.ids = ids;
    L.n = n;
    L.st = st;
    L.stage = stage;
    L.err = err;
    ProfileBegin(s, "topk_sample", n_samples);
    TopKSampleKernel<<<int((n_samples + 255) / 256), 256, 0, s>>>(L, keys, n_samples);
    ProfileEnd(s);
    CountLaunch();
    ProfileBegin(s, "topk_select", n_samples);
    TopKSelectKernel<<<1, 1024, 0, s>>>(keys, n_samples, r, out);
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
    L.kc = CodecOf(stage);
    L.shift = shift;
    L.dbits = dbits;
    L.hmask = prefix_bits == 0 ? 0 : (~0ull << (64 - prefix_bits));
    L.hval = prefix_bits == 0 ? 0 : (prefix << (64 - prefix_bits));
    L.counts = counts;
    L.err = err;
    ProfileBegin(s, "topk_histogram", n);
    TopKHistogramFor(stage.type)<<<Blocks((n + kTopKUnroll - 1) / kTopKUnroll, 256, 4), 256, 0, s>>>(L);
    ProfileEnd(s);
    CountLaunch();
}

void TopKCollect(const int64_t* ids, int64_t n, const StoreTable& st, const SortStage& stage, uint64_t prefix,
                 int prefix_bits, const uint64_t* limit_dev, int64_t* out, int64_t out_cap,
                 unsigned long long* count, const int64_t* tiles, int* err, cudaStream_t s) {
    cudaMemsetAsync(count, 0, sizeof(unsigned long long), s);
    if (n == 0) return;
    TopKLaunch L{};
    L.ids = ids;
    L.n = n;
    L.st = st;
    L.stage = stage;
    L.kc = CodecOf(stage);
    // p >> (64 - prefix_bits) <= prefix  <=>  p <= prefix followed by ones.
    L.limit = prefix_bits == 0 ? ~0ull
                               : (prefix_bits == 64 ? prefix : ((prefix << (64 - prefix_bits)) | (~0ull >> prefix_bits)));
    L.limit_dev = limit_dev;
    L.counts = count;
    L.out = out;
    L.out_cap = out_cap;
    L.tiles = tiles;
    L.err = err;
    ProfileBegin(s, "topk_collect", n);
    TopKCollectFor(stage.type)<<<Blocks((n + kIdTile - 1) / kIdTile * 32, 256, 4), 256, 0, s>>>(L);
    ProfileEnd(s);
    CountLaunch();
}

}  // namespace qdb
