// join.cu — equi-join hash build and pair-emitting probe for sm_100a.
//
// The build side (the row arena, in append order) is indexed by an
// open-addressing multi-map of two-slot buckets, one 32-byte sector each
// (keys, first payload words; layout in kernels.h JTableDev): every arena row
// claims its own slot with one 64-bit CAS, so equal keys occupy several slots
// along one bucket sequence.  Slots are a power of two of at least twice the
// rows (load <= 1/2, as the row table sizes itself,
// qdb/kernel/row_table.oz:140-166); a config-sized build of ~400K rows is a
// 16 MB bucket array that stays resident in the 126 MB L2 while the probe
// streams, and almost every probe reads exactly one sector.  A probe row
// walks its bucket sequence until an empty slot and emits one (probe row,
// arena row) pair per equal key (jr_probe_candidates,
// qdb/kernel/join/join_rows.oz:146-197); NULL keys match nothing.  Pairs
// come out in the engine's order: probe rows ascending, a row's build rows
// in append order (a count pass, a scan, then a write pass).
#include <algorithm>
#include <climits>

#include "common.cuh"
#include "eval.h"
#include "jtable.cuh"
#include "kernels.h"

namespace qdb {

namespace {

__device__ __forceinline__ i128 LoadKeyValue(const char* data, int width, bool is_signed, int64_t r) {
    switch (width) {
        case 1: return is_signed ? i128(reinterpret_cast<const int8_t*>(data)[r]) : i128(reinterpret_cast<const uint8_t*>(data)[r]);
        case 2: return is_signed ? i128(reinterpret_cast<const int16_t*>(data)[r]) : i128(reinterpret_cast<const uint16_t*>(data)[r]);
        case 4: return is_signed ? i128(reinterpret_cast<const int32_t*>(data)[r]) : i128(reinterpret_cast<const uint32_t*>(data)[r]);
        default: return is_signed ? i128(reinterpret_cast<const int64_t*>(data)[r]) : i128(reinterpret_cast<const uint64_t*>(data)[r]);
    }
}

__device__ __forceinline__ bool MaskValid(const uint8_t* mask, int64_t off, int64_t r) {
    if (!mask) return true;
    const int64_t bit = off + r;
    return (mask[bit >> 3] >> (bit & 7)) & 1;
}

// Packs the key of row r exactly as the fused probe's PackJoinKey does.
template <class A>
__device__ __forceinline__ uint64_t PackKeyCols(const A& a, int64_t r, bool& null) {
    null = false;
    uint64_t k = 0;
    for (int j = 0; j < a.jkey.n; ++j) {
        if (!MaskValid(a.key_mask[j], a.key_mask_off[j], r)) {
            null = true;
            return 0;
        }
        uint64_t v;
        if (a.jkey.is_float[j]) {
            double f = a.key_width[j] == 4 ? double(reinterpret_cast<const float*>(a.key_data[j])[r])
                                           : reinterpret_cast<const double*>(a.key_data[j])[r];
            v = CanonF64(f);
        } else {
            v = uint64_t(u128(LoadKeyValue(a.key_data[j], a.key_width[j], a.key_signed[j], r)));
        }
        if (a.jkey.n == 1 && !a.jkey.is_float[0]) return v;
        if (a.jkey.bits[j] < 64) v &= (1ull << a.jkey.bits[j]) - 1;
        k |= v << a.jkey.shift[j];
    }
    return k;
}

__global__ void JoinInitKernel(uint64_t* buckets, int64_t nbuckets) {
    for (int64_t b = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; b < nbuckets; b += int64_t(gridDim.x) * blockDim.x) {
        reinterpret_cast<ulonglong2*>(buckets)[2 * b] = make_ulonglong2(kEmptyKey, kEmptyKey);
        reinterpret_cast<ulonglong2*>(buckets)[2 * b + 1] = make_ulonglong2(0, 0);
    }
}

// Inserts arena row r: one slot of its key's bucket sequence claimed by CAS.
__device__ __forceinline__ void BuildRow(const JoinBuildArgs& a, int64_t r) {
    bool null = false;
    const uint64_t key = PackKeyCols(a, r, null);
    if (null) return;
    const uint64_t pay = a.pay0 ? uint64_t(a.pay0[r]) : 0;
    if (a.jkey.full64 && key == kEmptyKey) {
        const unsigned long long k = atomicAdd(a.nspecial, 1ull);
        a.special_rows[2 * k] = a.row_base + r;
        a.special_rows[2 * k + 1] = int64_t(pay);
        return;
    }
    uint64_t b = Fmix64(key) & a.bmask;
    for (uint64_t p = 0; p <= a.bmask; ++p) {
        for (int j = 0; j < 2; ++j) {
            auto* kp = reinterpret_cast<unsigned long long*>(&a.buckets[4 * b + j]);
            if (*reinterpret_cast<volatile unsigned long long*>(kp) == kEmptyKey &&
                atomicCAS(kp, kEmptyKey, key) == kEmptyKey) {
                a.buckets[4 * b + 2 + j] = pay;
                a.rows[2 * b + j] = a.row_base + r;
                return;
            }
        }
        b = (b + 1) & a.bmask;
    }
}

__global__ void __launch_bounds__(256) JoinBuildKernel(const __grid_constant__ JoinBuildArgs a) {
    for (int64_t r = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; r < a.nrows; r += int64_t(gridDim.x) * blockDim.x) {
        BuildRow(a, r);
    }
}

// Many tables in one launch: item = (table, range); `init` clears bucket
// ranges, otherwise arena-row ranges are inserted.
__global__ void __launch_bounds__(256) JoinBatchKernel(const JoinBuildArgs* args, const JoinBatchItem* items,
                                                       int64_t nitems, int init) {
    for (int64_t it = blockIdx.x; it < nitems; it += gridDim.x) {
        const JoinBatchItem item = items[it];
        const JoinBuildArgs& a = args[item.join];
        for (int64_t r = item.lo + threadIdx.x; r < item.hi; r += blockDim.x) {
            if (init) {
                reinterpret_cast<ulonglong2*>(a.buckets)[2 * r] = make_ulonglong2(kEmptyKey, kEmptyKey);
                reinterpret_cast<ulonglong2*>(a.buckets)[2 * r + 1] = make_ulonglong2(0, 0);
            } else {
                BuildRow(a, r);
            }
        }
    }
}

// Calls emit(arena row) for every build row whose key equals probe row r's
// (none for an unselected row or a NULL key) and returns their number.
template <class F>
__device__ __forceinline__ unsigned ProbeRowMatches(const JoinProbeArgs& a, int64_t r, F&& emit) {
    if (a.selection != nullptr && a.selection[r] == 0) return 0;
    bool null = false;
    const uint64_t key = PackKeyCols(a, r, null);
    if (null) return 0;
    if (a.jkey.full64 && key == kEmptyKey) {
        const int64_t nspecial = int64_t(*a.jt.nspecial);
        for (int64_t sp = 0; sp < nspecial; ++sp) emit(a.jt.special_rows[2 * sp]);
        return unsigned(nspecial);
    }
    const uint64_t b = Fmix64(key) & a.jt.bmask;
    return VisitMatches(a.jt, key, b, BucketKeys(a.jt, b),
                        [&](uint64_t slot, uint64_t, int) { emit(a.jt.rows[slot]); });
}

// A selected probe row with no NULL key field.
__device__ __forceinline__ bool RowHasValidKey(const JoinProbeArgs& a, int64_t r) {
    if (a.selection != nullptr && a.selection[r] == 0) return false;
    bool null = false;
    PackKeyCols(a, r, null);
    return !null;
}

// Rows of one chunk of the pair probe (one block per chunk).
constexpr int kPairChunk = 2048;
constexpr int kPairThreads = 256;

// Pass 1: every row's match count, and the chunk's total.
__global__ void __launch_bounds__(kPairThreads) JoinPairCountKernel(const __grid_constant__ JoinProbeArgs a,
                                                                    uint32_t* counts,
                                                                    unsigned long long* chunk_tot) {
    __shared__ unsigned long long warp_sum[kPairThreads / 32];
    const int64_t begin = int64_t(blockIdx.x) * kPairChunk;
    const int64_t end = min(a.nrows, begin + kPairChunk);
    unsigned long long local = 0;
    for (int64_t r = begin + threadIdx.x; r < end; r += kPairThreads) {
        unsigned c = ProbeRowMatches(a, r, [](int64_t) {});
        if (c == 0 && a.emit_unmatched && RowHasValidKey(a, r)) c = 1;   // padded with a NULL build row
        counts[r] = c;
        local += c;
    }
    local = WarpSumU64(local);
    if (LaneId() == 0) warp_sum[threadIdx.x >> 5] = local;
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long t = 0;
        for (int w = 0; w < kPairThreads / 32; ++w) t += warp_sum[w];
        chunk_tot[blockIdx.x] = t;
    }
}

// Pass 2: row r's pairs go to [off(r), off(r) + counts[r]), off = the
// chunk's offset plus the counts of the chunk's earlier rows, so pairs list
// probe rows in order; a row's own pairs are then put in arena (build
// append) order, the order of the engine's chains (jr_build_rows links the
// table last -> first, qdb/kernel/join/join_rows.oz:70-113).
__global__ void __launch_bounds__(kPairThreads) JoinPairWriteKernel(const __grid_constant__ JoinProbeArgs a,
                                                                    const uint32_t* counts,
                                                                    const unsigned long long* chunk_off) {
    __shared__ unsigned long long warp_sum[kPairThreads / 32];
    const int64_t begin = int64_t(blockIdx.x) * kPairChunk;
    const int64_t end = min(a.nrows, begin + kPairChunk);
    unsigned long long base = chunk_off[blockIdx.x];
    for (int64_t t0 = begin; t0 < end; t0 += kPairThreads) {
        const int64_t r = t0 + threadIdx.x;
        const unsigned long long c = r < end ? counts[r] : 0;
        // Block-wide exclusive scan of the tile's counts.
        unsigned long long incl = c;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const unsigned long long y = __shfl_up_sync(kFull, incl, d);
            if (LaneId() >= d) incl += y;
        }
        if (LaneId() == 31) warp_sum[threadIdx.x >> 5] = incl;
        __syncthreads();
        unsigned long long before = 0, tile = 0;
        for (int w = 0; w < kPairThreads / 32; ++w) {
            const unsigned long long v = warp_sum[w];
            if (w < int(threadIdx.x >> 5)) before += v;
            tile += v;
        }
        __syncthreads();
        const unsigned long long off = a.pair_base + base + before + incl - c;
        base += tile;
        if (c == 0 || int64_t(off + c) > a.pair_cap) continue;
        int64_t* out = a.pairs + 2 * off;
        unsigned k = 0;
        ProbeRowMatches(a, r, [&](int64_t brow) {
            if (k < c) {
                out[2 * k] = r;
                out[2 * k + 1] = brow;
            }
            ++k;
        });
        if (k == 0) {   // an outer join's unmatched row (its count is 1)
            out[0] = r;
            out[1] = -1;
            continue;
        }
        // Arena order within the row (insertion sort; chains are short).
        for (unsigned x = 1; x < c; ++x) {
            const int64_t v = out[2 * x + 1];
            unsigned y = x;
            while (y > 0 && out[2 * (y - 1) + 1] > v) {
                out[2 * y + 1] = out[2 * (y - 1) + 1];
                --y;
            }
            out[2 * y + 1] = v;
        }
    }
}

__global__ void __launch_bounds__(256) JoinNullKeyFlagsKernel(const __grid_constant__ JoinProbeArgs a, uint8_t* flags) {
    for (int64_t r = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; r < a.nrows; r += int64_t(gridDim.x) * blockDim.x) {
        bool null = false;
        if (a.selection == nullptr || a.selection[r] != 0) PackKeyCols(a, r, null);
        flags[r] = null ? 1 : 0;
    }
}

// Marks every build row a probe row matches; rows matched by many probe rows
// take the same plain byte store, so no atomics are needed.
__global__ void __launch_bounds__(256) JoinMarkKernel(const __grid_constant__ JoinProbeArgs a, uint8_t* marks) {
    for (int64_t r = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; r < a.nrows; r += int64_t(gridDim.x) * blockDim.x) {
        ProbeRowMatches(a, r, [&](int64_t brow) {
            if (marks[brow] == 0) marks[brow] = 1;
        });
    }
}

__global__ void __launch_bounds__(256) JoinMarkFlagsKernel(const uint8_t* marks, int64_t n, int want, uint8_t* flags) {
    for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
        flags[i] = marks == nullptr ? 1 : uint8_t((marks[i] != 0) == (want != 0));
    }
}

__global__ void __launch_bounds__(256) JoinWritePairsKernel(const int64_t* idx, int64_t n, int64_t* out, int mode) {
    for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
        const int64_t j = idx[i];
        out[2 * i] = mode == 0 ? j : -1;
        out[2 * i + 1] = mode == 0 ? -1 : (mode == 1 ? j : -j - 2);
    }
}

__global__ void __launch_bounds__(256) JoinKeyRangeKernel(const __grid_constant__ JoinBuildArgs a, long long* out) {
    long long lo = LLONG_MAX, hi = LLONG_MIN;
    for (int64_t r = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; r < a.nrows; r += int64_t(gridDim.x) * blockDim.x) {
        bool null = false;
        const long long k = (long long)PackKeyCols(a, r, null);
        if (null) continue;
        lo = min(lo, k);
        hi = max(hi, k);
    }
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) {
        lo = min(lo, __shfl_xor_sync(kFull, lo, d));
        hi = max(hi, __shfl_xor_sync(kFull, hi, d));
    }
    if (LaneId() == 0) {
        atomicMin(&out[0], lo);
        atomicMax(&out[1], hi);
    }
}

__global__ void __launch_bounds__(256) JoinDenseInitKernel(ulonglong2* dense, uint64_t range, uint32_t* bits,
                                                           int32_t words) {
    const int64_t stride = int64_t(gridDim.x) * blockDim.x;
    for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < int64_t(range); i += stride) {
        dense[i] = make_ulonglong2(kEmptyKey, 0);
    }
    for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < words; i += stride) bits[i] = 0;
}

__global__ void __launch_bounds__(256) JoinDenseBuildKernel(const __grid_constant__ JoinBuildArgs a, ulonglong2* dense,
                                                            int64_t kmin, uint64_t range, uint32_t* bits, int32_t shift,
                                                            unsigned long long* dup) {
    for (int64_t r = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; r < a.nrows; r += int64_t(gridDim.x) * blockDim.x) {
        bool null = false;
        const uint64_t key = PackKeyCols(a, r, null);
        if (null) continue;
        const uint64_t d = key - uint64_t(kmin);
        if (d >= range) {   // outside the measured range: cannot happen; counted as a duplicate (no index)
            atomicAdd(dup, 1ull);
            continue;
        }
        auto* kp = reinterpret_cast<unsigned long long*>(&dense[d].x);
        if (atomicCAS(kp, kEmptyKey, key) != kEmptyKey) {
            atomicAdd(dup, 1ull);
            continue;
        }
        dense[d].y = a.pay0 ? uint64_t(a.pay0[r]) : 0ull;
        const uint64_t bit = d >> shift;
        atomicOr(&bits[bit >> 5], 1u << (bit & 31));
    }
}

// Partition of a packed key: the high bits of its home bucket.
__device__ __forceinline__ int PartOf(uint64_t key, uint64_t bmask, int part_shift) {
    return int((Fmix64(key) & bmask) >> part_shift);
}

// Per-CTA histogram in shared memory, then one global add per partition.
template <class KeyAt>
__device__ __forceinline__ void PartCount(KeyAt key_at, int64_t n, uint64_t bmask, int part_shift, int nparts,
                                          unsigned long long* counts) {
    __shared__ unsigned hist[kMaxJoinParts];
    for (int i = threadIdx.x; i < nparts; i += blockDim.x) hist[i] = 0;
    __syncthreads();
    for (int64_t r = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; r < n; r += int64_t(gridDim.x) * blockDim.x) {
        bool skip = false;
        const uint64_t k = key_at(r, skip);
        if (!skip) atomicAdd(&hist[PartOf(k, bmask, part_shift)], 1u);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < nparts; i += blockDim.x) {
        if (hist[i]) atomicAdd(&counts[i], (unsigned long long)hist[i]);
    }
}

// Rows of a block-sized tile reserve their places per partition with one
// global add per (tile, partition), then write.
template <class KeyAt, class Write>
__device__ __forceinline__ void PartScatter(KeyAt key_at, Write write, int64_t n, uint64_t bmask, int part_shift,
                                            int nparts, unsigned long long* cursor) {
    __shared__ unsigned hist[kMaxJoinParts];
    __shared__ unsigned long long base[kMaxJoinParts];
    for (int64_t t0 = int64_t(blockIdx.x) * blockDim.x; t0 < n; t0 += int64_t(gridDim.x) * blockDim.x) {
        for (int i = threadIdx.x; i < nparts; i += blockDim.x) hist[i] = 0;
        __syncthreads();
        const int64_t r = t0 + threadIdx.x;
        bool skip = r >= n;
        uint64_t k = 0;
        if (!skip) k = key_at(r, skip);
        const int p = skip ? 0 : PartOf(k, bmask, part_shift);
        const unsigned rank = skip ? 0u : atomicAdd(&hist[p], 1u);
        __syncthreads();
        for (int i = threadIdx.x; i < nparts; i += blockDim.x) {
            base[i] = hist[i] ? atomicAdd(&cursor[i], (unsigned long long)hist[i]) : 0ull;
        }
        __syncthreads();
        if (!skip) write(r, k, int64_t(base[p] + rank));
        __syncthreads();
    }
}

__global__ void __launch_bounds__(256) JoinPartCountBuildKernel(const __grid_constant__ JoinBuildArgs a, int part_shift,
                                                                int nparts, unsigned long long* counts) {
    PartCount([&](int64_t r, bool& skip) { return PackKeyCols(a, r, skip); }, a.nrows, a.bmask, part_shift, nparts,
              counts);
}

__global__ void __launch_bounds__(256) JoinPartScatterBuildKernel(const __grid_constant__ JoinBuildArgs a,
                                                                  int part_shift, int nparts,
                                                                  unsigned long long* cursor, uint64_t* keys,
                                                                  int64_t* pays, int64_t* rows) {
    PartScatter([&](int64_t r, bool& skip) { return PackKeyCols(a, r, skip); },
                [&](int64_t r, uint64_t k, int64_t at) {
                    keys[at] = k;
                    pays[at] = a.pay0 ? a.pay0[r] : 0;
                    rows[at] = a.row_base + r;
                },
                a.nrows, a.bmask, part_shift, nparts, cursor);
}

// JoinBuildKernel's insert over partitioned rows.
__global__ void __launch_bounds__(256) JoinBuildRowsKernel(const __grid_constant__ JoinBuildArgs a,
                                                           const uint64_t* keys, const int64_t* pays,
                                                           const int64_t* rows, int64_t n) {
    for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
        const uint64_t key = keys[i];
        const uint64_t pay = uint64_t(pays[i]);
        if (a.jkey.full64 && key == kEmptyKey) {
            const unsigned long long k = atomicAdd(a.nspecial, 1ull);
            a.special_rows[2 * k] = rows[i];
            a.special_rows[2 * k + 1] = int64_t(pay);
            continue;
        }
        uint64_t b = Fmix64(key) & a.bmask;
        bool placed = false;
        for (uint64_t p = 0; p <= a.bmask && !placed; ++p) {
            for (int j = 0; j < 2; ++j) {
                auto* kp = reinterpret_cast<unsigned long long*>(&a.buckets[4 * b + j]);
                if (*reinterpret_cast<volatile unsigned long long*>(kp) == kEmptyKey &&
                    atomicCAS(kp, kEmptyKey, key) == kEmptyKey) {
                    a.buckets[4 * b + 2 + j] = pay;
                    a.rows[2 * b + j] = rows[i];
                    placed = true;
                    break;
                }
            }
            b = (b + 1) & a.bmask;
        }
    }
}

__global__ void __launch_bounds__(256) JoinPartCountProbeKernel(const int64_t* key, int64_t n, uint64_t bmask,
                                                                int part_shift, int nparts,
                                                                unsigned long long* counts) {
    PartCount([&](int64_t r, bool&) { return uint64_t(__ldcs(&key[r])); }, n, bmask, part_shift, nparts, counts);
}

__global__ void __launch_bounds__(256) JoinPartScatterProbeKernel(const int64_t* key, const int64_t* val, int64_t n,
                                                                  uint64_t bmask, int part_shift, int nparts,
                                                                  unsigned long long* cursor, int64_t* out_key,
                                                                  int64_t* out_val) {
    PartScatter([&](int64_t r, bool&) { return uint64_t(__ldcs(&key[r])); },
                [&](int64_t r, uint64_t k, int64_t at) {
                    out_key[at] = int64_t(k);
                    if (val) out_val[at] = __ldcs(&val[r]);
                },
                n, bmask, part_shift, nparts, cursor);
}

// Sets the Bloom bits of every occupied slot's key.
__global__ void __launch_bounds__(256) JoinBloomKernel(const uint64_t* buckets, int64_t nbuckets, uint32_t* bloom,
                                                       int32_t nwords) {
    for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < 2 * nbuckets; i += int64_t(gridDim.x) * blockDim.x) {
        const uint64_t k = buckets[4 * (i >> 1) + (i & 1)];
        if (k == kEmptyKey) continue;
        const uint64_t h = Fmix64(k);
        atomicOr(&bloom[BloomWord(h, nwords)], BloomBits(h));
    }
}

int Blocks(int64_t n, int threads) {
    return int(std::max<int64_t>(1, std::min<int64_t>((n + threads - 1) / threads, int64_t(DeviceSMs()) * 16)));
}

}  // namespace

void JoinInitTable(uint64_t* buckets, int64_t nbuckets, cudaStream_t s) {
    ProfileBegin(s, "join_init_table", nbuckets);
    JoinInitKernel<<<Blocks(nbuckets, 256), 256, 0, s>>>(buckets, nbuckets);
    ProfileEnd(s);
    CountLaunch();
}

void JoinBuild(const JoinBuildArgs& a, cudaStream_t s) {
    if (a.nrows == 0) return;
    ProfileBegin(s, "join_build", a.nrows);
    JoinBuildKernel<<<Blocks(a.nrows, 256), 256, 0, s>>>(a);
    ProfileEnd(s);
    CountLaunch();
}

void JoinPartCountBuild(const JoinBuildArgs& a, int part_shift, int nparts, unsigned long long* counts,
                        cudaStream_t s) {
    if (a.nrows == 0) return;
    ProfileBegin(s, "join_part_count", a.nrows);
    JoinPartCountBuildKernel<<<Blocks(a.nrows, 256), 256, 0, s>>>(a, part_shift, nparts, counts);
    ProfileEnd(s);
    CountLaunch();
}

void JoinPartScatterBuild(const JoinBuildArgs& a, int part_shift, int nparts, unsigned long long* cursor,
                          uint64_t* keys, int64_t* pays, int64_t* rows, cudaStream_t s) {
    if (a.nrows == 0) return;
    ProfileBegin(s, "join_part_scatter", a.nrows);
    JoinPartScatterBuildKernel<<<Blocks(a.nrows, 256), 256, 0, s>>>(a, part_shift, nparts, cursor, keys, pays, rows);
    ProfileEnd(s);
    CountLaunch();
}

void JoinBuildRows(const JoinBuildArgs& a, const uint64_t* keys, const int64_t* pays, const int64_t* rows, int64_t n,
                   cudaStream_t s) {
    if (n == 0) return;
    ProfileBegin(s, "join_build", n);
    JoinBuildRowsKernel<<<Blocks(n, 256), 256, 0, s>>>(a, keys, pays, rows, n);
    ProfileEnd(s);
    CountLaunch();
}

void JoinPartCountProbe(const int64_t* key, int64_t n, uint64_t bmask, int part_shift, int nparts,
                        unsigned long long* counts, cudaStream_t s) {
    if (n == 0) return;
    ProfileBegin(s, "join_part_count", n);
    JoinPartCountProbeKernel<<<Blocks(n, 256), 256, 0, s>>>(key, n, bmask, part_shift, nparts, counts);
    ProfileEnd(s);
    CountLaunch();
}

void JoinPartScatterProbe(const int64_t* key, const int64_t* val, int64_t n, uint64_t bmask, int part_shift,
                          int nparts, unsigned long long* cursor, int64_t* out_key, int64_t* out_val, cudaStream_t s) {
    if (n == 0) return;
    ProfileBegin(s, "join_part_scatter", n);
    JoinPartScatterProbeKernel<<<Blocks(n, 256), 256, 0, s>>>(key, val, n, bmask, part_shift, nparts, cursor, out_key,
                                                               out_val);
    ProfileEnd(s);
    CountLaunch();
}

void JoinKeyRange(const JoinBuildArgs& a, long long* out, cudaStream_t s) {
    if (a.nrows == 0) return;
    ProfileBegin(s, "join_key_range", a.nrows);
    JoinKeyRangeKernel<<<Blocks(a.nrows, 256), 256, 0, s>>>(a, out);
    ProfileEnd(s);
    CountLaunch();
}

void JoinDenseBuild(const JoinBuildArgs& a, ulonglong2* dense, int64_t kmin, uint64_t range, uint32_t* bits,
                    int32_t words, int32_t shift, unsigned long long* dup, cudaStream_t s) {
    ProfileBegin(s, "join_dense_build", int64_t(range));
    JoinDenseInitKernel<<<Blocks(int64_t(range), 256), 256, 0, s>>>(dense, range, bits, words);
    if (a.nrows > 0) JoinDenseBuildKernel<<<Blocks(a.nrows, 256), 256, 0, s>>>(a, dense, kmin, range, bits, shift, dup);
    ProfileEnd(s);
    CountLaunch(a.nrows > 0 ? 2 : 1);
}

void JoinBuildBloom(const JTableDev& jt, uint32_t* bloom, int32_t nwords, cudaStream_t s) {
    const int64_t nbuckets = int64_t(jt.bmask) + 1;
    cudaMemsetAsync(bloom, 0, size_t(nwords) * 4, s);
    ProfileBegin(s, "join_bloom", 2 * nbuckets);
    JoinBloomKernel<<<Blocks(2 * nbuckets, 256), 256, 0, s>>>(jt.buckets, nbuckets, bloom, nwords);
    ProfileEnd(s);
    CountLaunch();
}

int64_t JoinPairChunks(int64_t nrows) { return (nrows + kPairChunk - 1) / kPairChunk; }

void JoinProbeCount(const JoinProbeArgs& a, uint32_t* counts, unsigned long long* chunk_tot, cudaStream_t s) {
    if (a.nrows == 0) return;
    ProfileBegin(s, "join_probe_count", a.nrows);
    JoinPairCountKernel<<<unsigned(JoinPairChunks(a.nrows)), kPairThreads, 0, s>>>(a, counts, chunk_tot);
    ProfileEnd(s);
    CountLaunch();
}

void JoinProbeWrite(const JoinProbeArgs& a, const uint32_t* counts, const unsigned long long* chunk_off,
                    cudaStream_t s) {
    if (a.nrows == 0) return;
    ProfileBegin(s, "join_probe_pairs", a.nrows);
    JoinPairWriteKernel<<<unsigned(JoinPairChunks(a.nrows)), kPairThreads, 0, s>>>(a, counts, chunk_off);
    ProfileEnd(s);
    CountLaunch();
}

void JoinNullKeyFlags(const JoinProbeArgs& a, uint8_t* flags, cudaStream_t s) {
    if (a.nrows == 0) return;
    JoinNullKeyFlagsKernel<<<Blocks(a.nrows, 256), 256, 0, s>>>(a, flags);
    CountLaunch();
}

void JoinMarkProbe(const JoinProbeArgs& a, uint8_t* marks, cudaStream_t s) {
    if (a.nrows == 0) return;
    ProfileBegin(s, "join_mark_probe", a.nrows);
    JoinMarkKernel<<<Blocks(a.nrows, 256), 256, 0, s>>>(a, marks);
    ProfileEnd(s);
    CountLaunch();
}

void JoinMarkFlags(const uint8_t* marks, int64_t n, int want, uint8_t* flags, cudaStream_t s) {
    if (n == 0) return;
    JoinMarkFlagsKernel<<<Blocks(n, 256), 256, 0, s>>>(marks, n, want, flags);
    CountLaunch();
}

void JoinWritePairs(const int64_t* idx, int64_t n, int64_t* out, int mode, cudaStream_t s) {
    if (n == 0) return;
    JoinWritePairsKernel<<<Blocks(n, 256), 256, 0, s>>>(idx, n, out, mode);
    CountLaunch();
}

void JoinBuildBatch(const JoinBuildArgs* args, const JoinBatchItem* items, int64_t nitems, bool init,
                    cudaStream_t s) {
    if (nitems == 0) return;
    ProfileBegin(s, init ? "join_init_batch" : "join_build_batch", nitems);
    JoinBatchKernel<<<int(std::min<int64_t>(nitems, int64_t(DeviceSMs()) * 8)), 256, 0, s>>>(args, items, nitems,
                                                                                            init ? 1 : 0);
    ProfileEnd(s);
    CountLaunch();
}

}  // namespace qdb
