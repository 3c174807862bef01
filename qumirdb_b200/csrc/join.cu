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
// qdb/kernel/join/join_rows.oz:146-197); NULL keys match nothing.
#include <algorithm>

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

__global__ void __launch_bounds__(256) JoinBuildKernel(const __grid_constant__ JoinBuildArgs a) {
    for (int64_t r = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; r < a.nrows; r += int64_t(gridDim.x) * blockDim.x) {
        bool null = false;
        const uint64_t key = PackKeyCols(a, r, null);
        if (null) continue;
        const uint64_t pay = a.pay0 ? uint64_t(a.pay0[r]) : 0;
        if (a.jkey.full64 && key == kEmptyKey) {
            const unsigned long long k = atomicAdd(a.nspecial, 1ull);
            a.special_rows[2 * k] = a.row_base + r;
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
                    a.rows[2 * b + j] = a.row_base + r;
                    placed = true;
                    break;
                }
            }
            b = (b + 1) & a.bmask;
        }
    }
}

__global__ void __launch_bounds__(256) JoinProbePairsKernel(const __grid_constant__ JoinProbeArgs a) {
    const int64_t warps = int64_t(gridDim.x) * (blockDim.x / 32);
    for (int64_t base = (int64_t(blockIdx.x) * (blockDim.x / 32) + (threadIdx.x >> 5)) * 32; base < a.nrows;
         base += warps * 32) {
        const int64_t r = base + LaneId();
        bool act = r < a.nrows && (a.selection == nullptr || a.selection[r] != 0);
        bool null = false;
        uint64_t key = 0;
        if (act) key = PackKeyCols(a, r, null);
        act = act && !null;
        const bool special = act && a.jkey.full64 && key == kEmptyKey;
        uint64_t b = act ? (Fmix64(key) & a.jt.bmask) : 0;
        int j = 0;                      // next slot of bucket b to look at
        ulonglong2 kk = make_ulonglong2(kEmptyKey, kEmptyKey);
        if (act && !special) kk = BucketKeys(a.jt, b);
        int64_t sp = special ? 0 : -1;
        const int64_t nspecial = special ? int64_t(*a.jt.nspecial) : 0;
        uint64_t buckets_seen = 0;
        // Walk the bucket sequence; emit a pair per equal key.
        while (true) {
            int64_t brow = -1;
            if (act && !special) {
                while (true) {
                    if (j == 2) {
                        if (++buckets_seen > a.jt.bmask) {
                            act = false;
                            break;
                        }
                        b = (b + 1) & a.jt.bmask;
                        j = 0;
                        kk = BucketKeys(a.jt, b);
                    }
                    const uint64_t k = j == 0 ? kk.x : kk.y;
                    const int jj = j++;
                    if (k == kEmptyKey) {
                        act = false;
                        break;
                    }
                    if (k == key) {
                        brow = a.jt.rows[2 * b + jj];
                        break;
                    }
                }
            } else if (special) {
                if (sp < nspecial) brow = a.jt.special_rows[2 * sp++];
                else act = false;
            }
            const bool emit = brow >= 0;
            const unsigned m = __ballot_sync(kFull, emit);
            if (m == 0 && !__any_sync(kFull, act)) break;
            if (m) {
                unsigned long long at = 0;
                if (LaneId() == __ffs(m) - 1) at = atomicAdd(a.npairs, (unsigned long long)__popc(m));
                at = __shfl_sync(kFull, at, __ffs(m) - 1);
                if (emit) {
                    const unsigned long long slot = at + __popc(m & ((1u << LaneId()) - 1));
                    if (int64_t(slot) < a.pair_cap) {
                        a.pairs[2 * slot] = r;
                        a.pairs[2 * slot + 1] = brow;
                    }
                }
            }
            if (!__any_sync(kFull, act)) break;
        }
    }
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

void JoinBuildBloom(const JTableDev& jt, uint32_t* bloom, int32_t nwords, cudaStream_t s) {
    const int64_t nbuckets = int64_t(jt.bmask) + 1;
    cudaMemsetAsync(bloom, 0, size_t(nwords) * 4, s);
    ProfileBegin(s, "join_bloom", 2 * nbuckets);
    JoinBloomKernel<<<Blocks(2 * nbuckets, 256), 256, 0, s>>>(jt.buckets, nbuckets, bloom, nwords);
    ProfileEnd(s);
    CountLaunch();
}

void JoinProbePairs(const JoinProbeArgs& a, cudaStream_t s) {
    if (a.nrows == 0) return;
    ProfileBegin(s, "join_probe_pairs", a.nrows);
    JoinProbePairsKernel<<<Blocks(a.nrows, 256), 256, 0, s>>>(a);
    ProfileEnd(s);
    CountLaunch();
}

}  // namespace qdb
