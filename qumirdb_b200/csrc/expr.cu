// expr.cu — row-parallel filter, project, shuffle hash, compaction and gather
// kernels (the engine's filter / project / hash kernel contracts,
// qdb/kernel/compiler.h:488-520), built on the functors of eval.h.
#include <algorithm>

#include "../../include/qdb_gpu.h"
#include "common.cuh"
#include "eval.h"
#include "hash.h"
#include "kernels.h"
#include "rfilter.cuh"

namespace qdb {

namespace {

struct GlobalAcc {
    const AggPlan* P;
    int64_t row;
    __device__ __forceinline__ const char* Ptr(int c) const { return P->cols[c].data + row * P->cols[c].width; }
    __device__ __forceinline__ i128 Int(int c) const {
        const ColDesc& cd = P->cols[c];
        if (cd.kind == LK_BOOLBIT) {
            const int64_t bit = cd.bit_off + row;
            return (reinterpret_cast<const uint8_t*>(cd.data)[bit >> 3] >> (bit & 7)) & 1;
        }
        const char* p = Ptr(c);
        const bool u = cd.kind == LK_UNSIGNED;
        switch (cd.width) {
            case 1: return u ? i128(*reinterpret_cast<const uint8_t*>(p)) : i128(*reinterpret_cast<const int8_t*>(p));
            case 2: return u ? i128(*reinterpret_cast<const uint16_t*>(p)) : i128(*reinterpret_cast<const int16_t*>(p));
            case 4: return u ? i128(*reinterpret_cast<const uint32_t*>(p)) : i128(*reinterpret_cast<const int32_t*>(p));
            case 8: return u ? i128(*reinterpret_cast<const uint64_t*>(p)) : i128(*reinterpret_cast<const int64_t*>(p));
            default: {
                const uint64_t* q = reinterpret_cast<const uint64_t*>(p);
                return i128((u128(q[1]) << 64) | q[0]);
            }
        }
    }
    __device__ __forceinline__ double F64(int c) const {
        const ColDesc& cd = P->cols[c];
        if (cd.kind == LK_F64) return *reinterpret_cast<const double*>(Ptr(c));
        if (cd.kind == LK_F32) return double(*reinterpret_cast<const float*>(Ptr(c)));
        const i128 v = Int(c);
        return cd.scale ? double(v) / Pow10F(cd.scale) : double(v);
    }
    __device__ __forceinline__ bool Null(int c) const {
        const ColDesc& cd = P->cols[c];
        if (!cd.mask) return false;
        const int64_t bit = cd.mask_off + row;
        return !((cd.mask[bit >> 3] >> (bit & 7)) & 1);
    }
};

struct ExprLaunch {
    AggPlan P;
    ExprArgs A;
};

// The NULL tests of the key slots: normally every key must be valid; with
// null_keys_only at least one must be NULL.
__device__ __forceinline__ bool KeyNullsPass(const ExprArgs& A, const GlobalAcc& acc) {
    if (A.null_keys_only) {
        bool any = false;
        for (int j = 0; j < A.n_null_reject; ++j) any |= acc.Null(A.null_reject[j]);
        return any;
    }
    for (int j = 0; j < A.n_null_reject; ++j) {
        if (acc.Null(A.null_reject[j])) return false;
    }
    return true;
}

// Filters without a generic expression (selection, NULL rejects, atoms): no
// evaluation stack, so it keeps a full SM of warps where FilterKernel's
// generic evaluator (154 registers, a 1.7 KB stack) holds eight.
__global__ void __launch_bounds__(256) FilterAtomsKernel(const __grid_constant__ ExprLaunch L) {
    const AggPlan& P = L.P;
    for (int64_t r = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; r < L.A.nrows;
         r += int64_t(gridDim.x) * blockDim.x) {
        bool pass = P.selection == nullptr || P.selection[r] != 0;
        GlobalAcc acc{&P, r};
        if (pass) pass = KeyNullsPass(L.A, acc);
        if (pass && P.filter_kind == 1) pass = AtomsPass(P, acc);
        L.A.out_sel[r] = pass ? 1 : 0;
    }
}

__global__ void __launch_bounds__(256) FilterKernel(const __grid_constant__ ExprLaunch L) {
    const AggPlan& P = L.P;
    for (int64_t r = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; r < L.A.nrows;
         r += int64_t(gridDim.x) * blockDim.x) {
        bool pass = P.selection == nullptr || P.selection[r] != 0;
        GlobalAcc acc{&P, r};
        if (pass) pass = KeyNullsPass(L.A, acc);
        if (pass && P.filter_kind == 1) {
            pass = AtomsPass(P, acc);
        } else if (pass && P.filter_kind == 2) {
            GVal gv[kMaxGNodes];
            uint64_t gn = 0;
            if (!EvalGeneric(P.prog, P.filter_node, P.list, acc, gv, gn)) {
                SetError(L.A.err, DE_DIV_ZERO);
                pass = false;
            } else {
                pass = !((gn >> P.filter_node) & 1) && gv[P.filter_node].i != 0;
            }
        }
        L.A.out_sel[r] = pass ? 1 : 0;
    }
}

__device__ __forceinline__ void StoreTyped(void* base, int type, int64_t r, i128 iv, double fv) {
    char* p = static_cast<char*>(base);
    switch (type) {
        case QDB_TYPE_F64: reinterpret_cast<double*>(p)[r] = fv; break;
        case QDB_TYPE_F32: reinterpret_cast<float*>(p)[r] = float(fv); break;
        case QDB_TYPE_DECIMAL128:
            reinterpret_cast<uint64_t*>(p)[2 * r] = uint64_t(u128(iv));
            reinterpret_cast<uint64_t*>(p)[2 * r + 1] = uint64_t(u128(iv) >> 64);
            break;
        case QDB_TYPE_I64: case QDB_TYPE_U64: case QDB_TYPE_DECIMAL64:
            reinterpret_cast<int64_t*>(p)[r] = int64_t(iv);
            break;
        case QDB_TYPE_I32: case QDB_TYPE_U32: case QDB_TYPE_DATE32:
            reinterpret_cast<int32_t*>(p)[r] = int32_t(iv);
            break;
        case QDB_TYPE_I16: case QDB_TYPE_U16: reinterpret_cast<int16_t*>(p)[r] = int16_t(iv); break;
        default: reinterpret_cast<uint8_t*>(p)[r] = uint8_t(iv); break;
    }
}

__global__ void __launch_bounds__(256) ProjectKernel(const __grid_constant__ ExprLaunch L) {
    const AggPlan& P = L.P;
    for (int64_t r = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; r < L.A.nrows;
         r += int64_t(gridDim.x) * blockDim.x) {
        if (P.selection && !P.selection[r]) continue;
        GlobalAcc acc{&P, r};
        GVal gv[kMaxGNodes];
        uint64_t gn = 0;
        if (P.generic_root >= 0 && !EvalGeneric(P.prog, P.generic_root, P.list, acc, gv, gn)) {
            SetError(L.A.err, DE_DIV_ZERO);
            continue;
        }
        for (int k = 0; k < L.A.nout; ++k) {
            i128 iv = 0;
            double fv = 0.0;
            const int idx = L.A.out_idx[k];
            if (L.A.out_src[k] == VS_SOP) {
                const SopValue& v = P.values[idx];
                if (!SopNull(v, acc)) {
                    if (v.kind == VK_F64) fv = SopF64(v, acc);
                    else iv = SopInt(v, acc);
                }
            } else if (!((gn >> idx) & 1)) {
                iv = gv[idx].i;
                fv = gv[idx].f;
                if (P.prog.nodes[idx].dom == GD_F64) iv = 0;
            }
            StoreTyped(L.A.out_ptr[k], L.A.out_type[k], r, iv, fv);
        }
    }
}

// ---------------------------------------------------------------------------
// qdb_string_hash_bytes (qdb/modules/qumirdb_runtime.cpp:270-300) on the
// device: the engine's short-string mix up to 16 bytes, XXH3-64 (xxHash
// 0.8, seed 0) with the engine's 136-byte secret above.  A restatement of
// the published XXH3 steps; bytes are read one at a time (a string starts
// anywhere).
// ---------------------------------------------------------------------------
__constant__ uint8_t kStrSecret[136] = {
    0xe7, 0x8b, 0x13, 0xf9, 0xfc, 0xb5, 0x8e, 0xef, 0x81, 0x48, 0x2c, 0xbf, 0xf9, 0x9f,
    0xc1, 0x1e, 0x43, 0x6d, 0xbf, 0xa6, 0x6d, 0xb5, 0x72, 0xbc, 0x97, 0xd8, 0x61, 0x24,
    0x0f, 0x12, 0xe3, 0x05, 0x21, 0xf7, 0x5c, 0x66, 0x67, 0xa5, 0x65, 0x03, 0x96, 0x26,
    0x69, 0xd8, 0x29, 0x20, 0xf8, 0xc7, 0xb0, 0x3d, 0xdd, 0x7d, 0x18, 0xa0, 0x60, 0x75,
    0x92, 0xa4, 0xce, 0xba, 0xc0, 0x77, 0xf4, 0xac, 0xb7, 0x03, 0x53, 0xf0, 0x98, 0xce,
    0xe6, 0x2b, 0x20, 0xc7, 0x82, 0x91, 0xab, 0xbf, 0x68, 0x5c, 0x62, 0x4d, 0x33, 0xa3,
    0xe1, 0xb3, 0xff, 0x97, 0x54, 0x4c, 0x44, 0x34, 0xb5, 0xb9, 0x32, 0x4c, 0x75, 0x42,
    0x89, 0x53, 0x94, 0xd4, 0x9f, 0x2b, 0x76, 0x4d, 0x4e, 0xe6, 0xfa, 0x15, 0x3e, 0xc1,
    0xdb, 0x71, 0x4b, 0x2c, 0x94, 0xf5, 0xfc, 0x8c, 0x89, 0x4b, 0xfb, 0xc1, 0x82, 0xa5,
    0x6a, 0x53, 0xf9, 0x4a, 0xba, 0xce, 0x1f, 0xc0, 0x97, 0x1a,
};
constexpr int kStrSecretBytes = 136;

__device__ __forceinline__ uint64_t StrLe64(const uint8_t* p) {
    uint64_t v = 0;
#pragma unroll
    for (int k = 7; k >= 0; --k) v = (v << 8) | p[k];
    return v;
}

__device__ __forceinline__ uint32_t StrLe32(const uint8_t* p) {
    return uint32_t(p[0]) | (uint32_t(p[1]) << 8) | (uint32_t(p[2]) << 16) | (uint32_t(p[3]) << 24);
}

__device__ __forceinline__ uint64_t XxFold(uint64_t a, uint64_t b) { return a * b ^ __umul64hi(a, b); }

__device__ __forceinline__ uint64_t XxAvalanche(uint64_t h) {
    h ^= h >> 37;
    h *= 0x165667919E3779F9ull;
    return h ^ (h >> 32);
}

__device__ __forceinline__ uint64_t XxMix16(const uint8_t* in, int so) {
    return XxFold(StrLe64(in) ^ StrLe64(kStrSecret + so), StrLe64(in + 8) ^ StrLe64(kStrSecret + so + 8));
}

__device__ __forceinline__ void XxStripe(uint64_t (&acc)[8], const uint8_t* in, int so) {
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        const uint64_t v = StrLe64(in + 8 * i);
        const uint64_t k = v ^ StrLe64(kStrSecret + so + 8 * i);
        acc[i ^ 1] += v;
        acc[i] += (k & 0xffffffffull) * (k >> 32);
    }
}

__device__ __noinline__ uint64_t Xxh3Long(const uint8_t* d, int64_t n) {
    uint64_t acc[8] = {0xC2B2AE3Dull, 0x9E3779B185EBCA87ull, 0xC2B2AE3D27D4EB4Full, 0x165667B19E3779F9ull,
                       0x85EBCA77C2B2AE63ull, 0x85EBCA77ull, 0x27D4EB2F165667C5ull, 0x9E3779B1ull};
    constexpr int kStripes = (kStrSecretBytes - 64) / 8;
    constexpr int64_t kBlock = 64 * kStripes;
    const int64_t blocks = (n - 1) / kBlock;
    for (int64_t b = 0; b < blocks; ++b) {
        for (int s = 0; s < kStripes; ++s) XxStripe(acc, d + b * kBlock + 64 * s, 8 * s);
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            uint64_t a = acc[i];
            a ^= a >> 47;
            a ^= StrLe64(kStrSecret + kStrSecretBytes - 64 + 8 * i);
            acc[i] = a * 0x9E3779B1ull;
        }
    }
    const int64_t tail = ((n - 1) - kBlock * blocks) / 64;
    for (int64_t s = 0; s < tail; ++s) XxStripe(acc, d + blocks * kBlock + 64 * s, int(8 * s));
    XxStripe(acc, d + n - 64, kStrSecretBytes - 64 - 7);
    uint64_t r = uint64_t(n) * 0x9E3779B185EBCA87ull;
#pragma unroll
    for (int i = 0; i < 4; ++i)
        r += XxFold(acc[2 * i] ^ StrLe64(kStrSecret + 11 + 16 * i), acc[2 * i + 1] ^ StrLe64(kStrSecret + 19 + 16 * i));
    return XxAvalanche(r);
}

__device__ __forceinline__ uint64_t StringHashDev(const uint8_t* d, int64_t n) {
    constexpr uint64_t m0 = 11400714785074694791ull, m1 = 14029467366897019727ull;
    if (n == 0) return 1;
    if (n <= 3) {
        const uint32_t x = (uint32_t(n) << 24) ^ (uint32_t(d[0]) << 16) ^ (uint32_t(d[n / 2]) << 8) ^ d[n - 1];
        return ByteSwap64(m0 * x);
    }
    if (n <= 8) return uint64_t(n) ^ ByteSwap64(m0 * StrLe32(d + n - 4)) ^ ByteSwap64(m1 * StrLe32(d));
    if (n <= 16) return uint64_t(n) ^ ByteSwap64(m0 * StrLe64(d + n - 8)) ^ ByteSwap64(m1 * StrLe64(d));
    const uint64_t len = uint64_t(n);
    if (n <= 128) {
        uint64_t acc = len * 0x9E3779B185EBCA87ull;
        if (n > 32) {
            if (n > 64) {
                if (n > 96) {
                    acc += XxMix16(d + 48, 96);
                    acc += XxMix16(d + n - 64, 112);
                }
                acc += XxMix16(d + 32, 64);
                acc += XxMix16(d + n - 48, 80);
            }
            acc += XxMix16(d + 16, 32);
            acc += XxMix16(d + n - 32, 48);
        }
        acc += XxMix16(d, 0);
        acc += XxMix16(d + n - 16, 16);
        return XxAvalanche(acc);
    }
    if (n <= 240) {
        uint64_t acc = len * 0x9E3779B185EBCA87ull;
#pragma unroll
        for (int i = 0; i < 8; ++i) acc += XxMix16(d + 16 * i, 16 * i);
        acc = XxAvalanche(acc);
        const int rounds = int(n / 16);
        for (int i = 8; i < rounds; ++i) acc += XxMix16(d + 16 * i, 16 * (i - 8) + 3);
        acc += XxMix16(d + n - 16, kStrSecretBytes - 17);
        return XxAvalanche(acc);
    }
    return Xxh3Long(d, n);
}

// The string of row r of a string column (offsets of 4 or 8 bytes).
__device__ __forceinline__ uint64_t StringCellHash(const ColDesc& cd, int64_t r) {
    int64_t b, e;
    if (cd.offset_width == 8) {
        b = reinterpret_cast<const int64_t*>(cd.offsets)[r];
        e = reinterpret_cast<const int64_t*>(cd.offsets)[r + 1];
    } else {
        b = reinterpret_cast<const int32_t*>(cd.offsets)[r];
        e = reinterpret_cast<const int32_t*>(cd.offsets)[r + 1];
    }
    return StringHashDev(reinterpret_cast<const uint8_t*>(cd.data) + b, e - b);
}

// STR: some key column is a string (the string hash is compiled in only then,
// so that integer keys keep the lean kernel).
template <bool STR>
__global__ void __launch_bounds__(256) HashKernel(const __grid_constant__ ExprLaunch L) {
    const AggPlan& P = L.P;
    unsigned long long kept = 0;
    for (int64_t r = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; r < L.A.nrows;
         r += int64_t(gridDim.x) * blockDim.x) {
        if (P.selection && !P.selection[r]) {
            if (L.A.rf_out) L.A.rf_out[r] = 0;
            continue;
        }
        GlobalAcc acc{&P, r};
        uint64_t h = 0;
        for (int j = 0; j < L.A.nhash; ++j) {
            const int c = L.A.hash_slot[j];
            const int t = L.A.hash_type[j];
            const bool null = acc.Null(c);
            // A nullable key is two struct fields: its BOOL validity, then the value.
            if (L.A.hash_nullable[j]) h = Combine(h, null ? 0 : LeafHashOf(QDB_TYPE_BOOL, 1, 0.0));
            uint64_t fh = 0;
            if (STR && !null && t == QDB_TYPE_STRING) {
                fh = StringCellHash(P.cols[c], r);
            } else if (!null) {
                const bool fl = t == QDB_TYPE_F32 || t == QDB_TYPE_F64;
                fh = LeafHashOf(t, fl ? i128(0) : acc.Int(c), fl ? acc.F64(c) : 0.0);
            }
            h = Combine(h, fh);
        }
        if (L.A.rf_out) {
            const bool keep = FilterContains(L.A.rf_kind, L.A.rf_words, L.A.rf_nwords, h);
            L.A.rf_out[r] = keep ? 1 : 0;
            kept += keep;
        } else {
            L.A.hashes[r] = h;
        }
    }
    if (L.A.rf_kept) {
        kept = WarpSumU64(kept);
        if (LaneId() == 0 && kept) atomicAdd(L.A.rf_kept, kept);
    }
}

constexpr int kCompactChunk = 4096;

__global__ void __launch_bounds__(256) CountFlagsKernel(const uint8_t* flags, int64_t n, unsigned long long* counts) {
    __shared__ unsigned cnt;
    if (threadIdx.x == 0) cnt = 0;
    __syncthreads();
    const int64_t begin = int64_t(blockIdx.x) * kCompactChunk;
    const int64_t end = begin + kCompactChunk < n ? begin + kCompactChunk : n;
    unsigned local = 0;
    for (int64_t i = begin + threadIdx.x; i < end; i += blockDim.x) local += flags[i] ? 1 : 0;
    atomicAdd(&cnt, local);
    __syncthreads();
    if (threadIdx.x == 0) counts[blockIdx.x] = cnt;
}

__global__ void __launch_bounds__(256) WriteFlagsKernel(const uint8_t* flags, int64_t n,
                                                        const unsigned long long* offsets, int64_t nblocks,
                                                        int64_t* out, unsigned long long* d_count) {
    __shared__ unsigned warp_cnt[8];
    __shared__ unsigned running;
    if (threadIdx.x == 0) running = 0;
    __syncthreads();
    const int64_t begin = int64_t(blockIdx.x) * kCompactChunk;
    const int64_t end = begin + kCompactChunk < n ? begin + kCompactChunk : n;
    const unsigned long long base = offsets[blockIdx.x];
    for (int64_t b = begin; b < end; b += blockDim.x) {
        const int64_t i = b + threadIdx.x;
        const bool on = i < end && flags[i];
        const unsigned m = __ballot_sync(kFull, on);
        if (LaneId() == 0) warp_cnt[threadIdx.x >> 5] = __popc(m);
        __syncthreads();
        unsigned before = running;
        for (int w = 0; w < int(threadIdx.x >> 5); ++w) before += warp_cnt[w];
        before += __popc(m & ((1u << LaneId()) - 1));
        if (on) out[base + before] = i;
        __syncthreads();
        if (threadIdx.x == 0) {
            unsigned tot = 0;
            for (int w = 0; w < 8; ++w) tot += warp_cnt[w];
            running += tot;
        }
        __syncthreads();
    }
    if (blockIdx.x == nblocks - 1 && threadIdx.x == 0) *d_count = base + running;
}

__global__ void __launch_bounds__(256) GatherKernel(const char* src, int width, const int64_t* idx, int stride,
                                                    int64_t n, char* out, const char* src2) {
    for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
        int64_t j = idx[i * stride];
        if (j <= -2 && src2 != nullptr) {
            // A row of the second source (the NULL-key arena of an ANTI join).
            j = -j - 2;
            src = src2;
        }
        switch (width) {
            case 1: out[i] = j < 0 ? 0 : src[j]; break;
            case 2: reinterpret_cast<int16_t*>(out)[i] = j < 0 ? 0 : reinterpret_cast<const int16_t*>(src)[j]; break;
            case 4: reinterpret_cast<int32_t*>(out)[i] = j < 0 ? 0 : reinterpret_cast<const int32_t*>(src)[j]; break;
            case 8: reinterpret_cast<int64_t*>(out)[i] = j < 0 ? 0 : reinterpret_cast<const int64_t*>(src)[j]; break;
            default: {
                const uint64_t* s = reinterpret_cast<const uint64_t*>(src);
                uint64_t* o = reinterpret_cast<uint64_t*>(out);
                o[2 * i] = j < 0 ? 0 : s[2 * j];
                o[2 * i + 1] = j < 0 ? 0 : s[2 * j + 1];
            }
        }
    }
}

__global__ void __launch_bounds__(256) GatherValidityKernel(const uint8_t* mask, int64_t mask_off, const int64_t* idx,
                                                            int stride, int64_t n, uint32_t* out, int64_t out_off,
                                                            bool has2, const uint8_t* mask2) {
    for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
        int64_t j = idx[i * stride];
        const uint8_t* m = mask;
        int64_t moff = mask_off;
        if (j <= -2 && has2) {
            j = -j - 2;
            m = mask2;
            moff = 0;
        }
        bool valid = j >= 0;
        if (valid && m) {
            const int64_t bit = moff + j;
            valid = (m[bit >> 3] >> (bit & 7)) & 1;
        }
        const int64_t o = out_off + i;
        if (valid) atomicOr(&out[o >> 5], 1u << (o & 31));
    }
}

int Blocks(int64_t n, int threads) {
    return int(std::max<int64_t>(1, std::min<int64_t>((n + threads - 1) / threads, int64_t(DeviceSMs()) * 16)));
}

ExprLaunch* ThreadLaunch() {
    static thread_local ExprLaunch* p = nullptr;
    if (!p) p = new ExprLaunch();
    return p;
}

}  // namespace

void FilterRows(const ExprArgs& a, cudaStream_t s) {
    if (a.nrows == 0) return;
    ExprLaunch& L = *ThreadLaunch();
    L.P = *a.plan;
    L.A = a;
    ProfileBegin(s, "filter", a.nrows);
    if (L.P.filter_kind == 2) FilterKernel<<<Blocks(a.nrows, 256), 256, 0, s>>>(L);
    else FilterAtomsKernel<<<Blocks(a.nrows, 256), 256, 0, s>>>(L);
    ProfileEnd(s);
    CountLaunch();
}

void ProjectRows(const ExprArgs& a, cudaStream_t s) {
    if (a.nrows == 0) return;
    ExprLaunch& L = *ThreadLaunch();
    L.P = *a.plan;
    L.A = a;
    ProfileBegin(s, "project", a.nrows);
    ProjectKernel<<<Blocks(a.nrows, 256), 256, 0, s>>>(L);
    ProfileEnd(s);
    CountLaunch();
}

void HashRows(const ExprArgs& a, cudaStream_t s) {
    if (a.nrows == 0) return;
    ExprLaunch& L = *ThreadLaunch();
    L.P = *a.plan;
    L.A = a;
    bool str = false;
    for (int j = 0; j < a.nhash; ++j) str = str || a.hash_type[j] == QDB_TYPE_STRING;
    ProfileBegin(s, "hash", a.nrows);
    if (str) HashKernel<true><<<Blocks(a.nrows, 256), 256, 0, s>>>(L);
    else HashKernel<false><<<Blocks(a.nrows, 256), 256, 0, s>>>(L);
    ProfileEnd(s);
    CountLaunch();
}

size_t CompactScratch(int64_t n) {
    return size_t((n + kCompactChunk - 1) / kCompactChunk + 1) * sizeof(unsigned long long);
}

void CompactFlags(const uint8_t* flags, int64_t n, int64_t* out_idx, unsigned long long* d_count, void* scratch,
                  cudaStream_t s) {
    if (n == 0) {
        cudaMemsetAsync(d_count, 0, sizeof(unsigned long long), s);
        return;
    }
    const int64_t nb = (n + kCompactChunk - 1) / kCompactChunk;
    auto* counts = static_cast<unsigned long long*>(scratch);
    CountFlagsKernel<<<int(nb), 256, 0, s>>>(flags, n, counts);
    ExclusiveScanU64(counts, nb, s);
    WriteFlagsKernel<<<int(nb), 256, 0, s>>>(flags, n, counts, nb, out_idx, d_count);
    CountLaunch(2);
}

void GatherColumn(const char* src, int width, const int64_t* idx, int idx_stride, int64_t n, char* out,
                  cudaStream_t s, const char* src2) {
    if (n == 0) return;
    GatherKernel<<<Blocks(n, 256), 256, 0, s>>>(src, width, idx, idx_stride, n, out, src2);
    CountLaunch();
}

void GatherValidity(const uint8_t* mask, int64_t mask_off, const int64_t* idx, int idx_stride, int64_t n,
                    uint32_t* out_words, int64_t out_bit_off, cudaStream_t s, bool has2, const uint8_t* mask2) {
    if (n == 0) return;
    GatherValidityKernel<<<Blocks(n, 256), 256, 0, s>>>(mask, mask_off, idx, idx_stride, n, out_words, out_bit_off,
                                                         has2, mask2);
    CountLaunch();
}

}  // namespace qdb
