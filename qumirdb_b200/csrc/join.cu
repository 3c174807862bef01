// join.cu — equi-join hash build and pair-emitting probe for sm_100a.
//
// The build side (the row arena, in append order) is indexed by an
// open-addressing multi-map of 16-byte entries (packed key, arena row): every
// arena row claims its own entry with one 64-bit CAS, so equal keys occupy
// several entries along one probe sequence.  Capacity is a power of two of at
// least twice the rows (load <= 1/2, as the row table sizes itself,
// qdb/kernel/row_table.oz:140-166); a config-sized build of ~400K rows is a
// 16 MB table that stays resident in the 126 MB L2 while the probe streams.
// A probe row walks its sequence until an empty entry and emits one
// (probe row, arena row) pair per equal key (jr_probe_candidates,
// qdb/kernel/join/join_rows.oz:146-197); NULL keys match nothing.
#include <algorithm>

#include "common.cuh"
#include "eval.h"
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

__global__ void JoinInitKernel(uint64_t* entries, int64_t capacity) {
    for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < capacity; i += int64_t(gridDim.x) * blockDim.x) {
        reinterpret_cast<ulonglong2*>(entries)[2 * i] = make_ulonglong2(kEmptyKey, 0);
        reinterpret_cast<ulonglong2*>(entries)[2 * i + 1] = make_ulonglong2(0, 0);
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
        uint64_t i = Fmix64(key) & a.mask;
        for (uint64_t p = 0; p <= a.mask; ++p) {
            auto* kp = reinterpret_cast<unsigned long long*>(&a.entries[4 * i]);
            if (*reinterpret_cast<volatile unsigned long long*>(kp) == kEmptyKey &&
                atomicCAS(kp, kEmptyKey, key) == kEmptyKey) {
                a.entries[4 * i + 1] = uint64_t(a.row_base + r);
                a.entries[4 * i + 2] = pay;
                break;
            }
            i = (i + 1) & a.mask;
        }
    }
}

__global__ void __launch_bounds__(256) JoinProbePairsKernel(const __grid_constant__ JoinProbeArgs a) {
    const int64_t warps = int64_t(gridDim.x) * (blockDim.x / 32);
    for (int64_t b = (int64_t(blockIdx.x) * (blockDim.x / 32) + (threadIdx.x >> 5)) * 32; b < a.nrows; b += warps * 32) {
        const int64_t r = b + LaneId();
        bool act = r < a.nrows && (a.selection == nullptr || a.selection[r] != 0);
        bool null = false;
        uint64_t key = 0;
        if (act) key = PackKeyCols(a, r, null);
        act = act && !null;
        const bool special = act && a.jkey.full64 && key == kEmptyKey;
        int64_t pos = -1;
        uint64_t i = act ? (Fmix64(key) & a.jt.mask) : 0;
        int64_t sp = special ? 0 : -1;
        int64_t probes = 0;
        // Walk the probe sequence; emit a pair per equal key.
        while (true) {
            int64_t brow = -1;
            if (act && !special) {
                while (probes <= int64_t(a.jt.mask)) {
                    const ulonglong2 e = *reinterpret_cast<const ulonglong2*>(&a.jt.entries[4 * i]);
                    ++probes;
                    if (e.x == kEmptyKey) {
                        act = false;
                        break;
                    }
                    const uint64_t here = i;
                    i = (i + 1) & a.jt.mask;
                    if (e.x == key) {
                        brow = int64_t(e.y);
                        pos = int64_t(here);
                        break;
                    }
                }
                if (probes > int64_t(a.jt.mask)) act = false;
            } else if (special) {
                if (sp < a.jt.nspecial) brow = a.jt.special_rows[2 * sp++];
                else act = false;
            }
            const bool emit = brow >= 0;
            const unsigned m = __ballot_sync(kFull, emit);
            if (m == 0 && !__any_sync(kFull, act)) break;
            if (m) {
                unsigned long long base = 0;
                if (LaneId() == __ffs(m) - 1) base = atomicAdd(a.npairs, (unsigned long long)__popc(m));
                base = __shfl_sync(kFull, base, __ffs(m) - 1);
                if (emit) {
                    const unsigned long long slot = base + __popc(m & ((1u << LaneId()) - 1));
                    if (int64_t(slot) < a.pair_cap) {
                        a.pairs[2 * slot] = r;
                        a.pairs[2 * slot + 1] = brow;
                    }
                }
            }
            if (!__any_sync(kFull, act)) break;
        }
        (void)pos;
    }
}

int Blocks(int64_t n, int threads) {
    return int(std::max<int64_t>(1, std::min<int64_t>((n + threads - 1) / threads, int64_t(DeviceSMs()) * 16)));
}

}  // namespace

void JoinInitTable(uint64_t* entries, int64_t capacity, cudaStream_t s) {
    ProfileBegin(s, "join_init_table", capacity);
    JoinInitKernel<<<Blocks(capacity, 256), 256, 0, s>>>(entries, capacity);
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

void JoinProbePairs(const JoinProbeArgs& a, cudaStream_t s) {
    if (a.nrows == 0) return;
    ProfileBegin(s, "join_probe_pairs", a.nrows);
    JoinProbePairsKernel<<<Blocks(a.nrows, 256), 256, 0, s>>>(a);
    ProfileEnd(s);
    CountLaunch();
}

}  // namespace qdb
