// fast.cu — typed fast kernels the runtime selects when a lowered plan has a
// shape they serve; every other plan runs the general fused kernel (agg.cu).
//
// Join-sum shape: a fused equi-join + keyless aggregate whose inputs are an
// 8-byte probe key and COUNT(*) / SUM(product of up to two 8-byte integer
// factors c + d*x), x a probe column or a build payload column, with no
// NULLs.  One persistent CTA per SM: a producer warp streams tiles of the
// probe key column and of one probe value column into shared memory with
// bulk copies (L2 evict-first, so the build table stays resident in L2),
// three stages deep; thirty-one consumer warps take two rows per thread from
// a stage, reject most of them against the build side's Bloom filter (held in
// shared memory), and issue the bucket reads of the rest together: one
// 32-byte sector carries both keys and both payload words of a bucket, so a
// hit or a miss is one L2 round trip.  Joined rows fold into register
// accumulators; a block reduction and one atomic per state word per CTA end
// the launch.
#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "common.cuh"
#include "fast.h"
#include "jtable.cuh"
#include "kernels.h"
#include "runtime.h"

namespace qdb {

namespace {

// Latency of the bucket reads is hidden by warps: 31 consumer warps and the
// producer fill the CTA's 1,024 threads (0.82 ms for 120M probe rows, against
// 1.21 ms with 16 consumer warps taking four rows per thread).
constexpr int kJsConsumerWarps = 31;
constexpr int kJsConsumers = kJsConsumerWarps * 32;
constexpr int kJsThreads = kJsConsumers + 32;   // + the producer warp
constexpr int kJsTile = kJsConsumers * 2;       // rows per stage (1,984: 15.5 KB per column)
constexpr int kJsStages = 3;
constexpr int kJsRows = kJsTile / kJsConsumers;  // rows per consumer thread per stage
constexpr int kJsBarBytes = 128;                 // barriers and the abort flag

struct JsLaunch {
    JoinSumShape S;
    JTableDev jt;
    int64_t nrows;
    uint64_t* group_states;    // state words of the keyless group in the global table
    AggCounters* counters;
    const int64_t* vcol;       // probe column staged beside the keys, or nullptr
    int64_t staged_tiles;      // leading full tiles that go through the stages
    int32_t bloom_words;       // filter words held in shared memory (0: none)
    int32_t stage_bytes;
};

struct JsAcc {
    uint64_t v[kJsMaxStates];
    unsigned long long matched;
};

// Folds one joined row: probe row `row` with staged value `sv`, bucket
// payload word `pay`, arena row `brow`.
__device__ __forceinline__ void JsFold(const JsLaunch& L, JsAcc& a, int64_t row, int64_t sv, uint64_t pay,
                                       int64_t brow) {
    ++a.matched;
#pragma unroll
    for (int s = 0; s < kJsMaxStates; ++s) {
        if (s >= L.S.nstates) break;
        const JsState& st = L.S.states[s];
        if (st.nf == 0) {
            a.v[s] += 1;
            continue;
        }
        uint64_t v = 1;
#pragma unroll
        for (int f = 0; f < 2; ++f) {
            if (f >= st.nf) break;
            const JsFactor& jf = st.f[f];
            int64_t x;
            switch (jf.side) {
                case 3: x = sv; break;
                case 1: x = int64_t(pay); break;
                case 2: x = jf.data[brow]; break;
                default: x = jf.data[row]; break;
            }
            v *= uint64_t(jf.c) + uint64_t(jf.d) * uint64_t(x);
        }
        a.v[s] += v;
    }
}

// Compile-time state signatures.  A state code names what one state adds
// per joined row: 0 COUNT(*), 1 f(pay), 2 f(sv), 3 f(pay) * g(sv),
// 4 f(pay) * g(pay), 5 f(sv) * g(sv), with f, g the state's affine factors
// (c + d * x, wrapping) over the bucket payload word `pay` and the staged
// probe value `sv`.  NS = 0 selects the runtime interpretation (JsFold).
__device__ __forceinline__ uint64_t Affine(const JsFactor& f, uint64_t x) { return uint64_t(f.c) + uint64_t(f.d) * x; }

template <int C>
__device__ __forceinline__ uint64_t JsTerm(const JsState& st, uint64_t pay, int64_t sv) {
    if constexpr (C == 0) return 1;
    else if constexpr (C == 1) return Affine(st.f[0], pay);
    else if constexpr (C == 2) return Affine(st.f[0], uint64_t(sv));
    else if constexpr (C == 3) return Affine(st.f[0], pay) * Affine(st.f[1], uint64_t(sv));
    else if constexpr (C == 4) return Affine(st.f[0], pay) * Affine(st.f[1], pay);
    else return Affine(st.f[0], uint64_t(sv)) * Affine(st.f[1], uint64_t(sv));
}

template <int NS, int C0, int C1>
__device__ __forceinline__ void JsFoldSlot(const JsLaunch& L, JsAcc& a, int64_t row, int64_t sv, uint64_t pay,
                                           uint64_t slot) {
    if constexpr (NS == 0) {
        JsFold(L, a, row, sv, pay, L.S.need_row ? L.jt.rows[slot] : 0);
    } else {
        ++a.matched;
        a.v[0] += JsTerm<C0>(L.S.states[0], pay, sv);
        if constexpr (NS == 2) a.v[1] += JsTerm<C1>(L.S.states[1], pay, sv);
    }
}

// Probes kJsRows rows of one thread: Bloom test, then every surviving row's
// first bucket read in one batch, then the (rare) longer bucket walks.
template <int NS, int C0, int C1>
__device__ __forceinline__ void JsProbe(const JsLaunch& L, JsAcc& a, const uint32_t* bloom, int32_t nb,
                                        int64_t nspecial, const int64_t (&row)[kJsRows],
                                        const uint64_t (&key)[kJsRows], const int64_t (&sv)[kJsRows],
                                        const bool (&valid)[kJsRows]) {
    const JTableDev& jt = L.jt;
    uint64_t b[kJsRows];
    ulonglong2 k[kJsRows];
    ulonglong2 p[kJsRows];
    bool ok[kJsRows];
#pragma unroll
    for (int j = 0; j < kJsRows; ++j) {
        ok[j] = valid[j] && key[j] != kEmptyKey;
        const uint64_t h = Fmix64(key[j]);
        if (ok[j] && nb) {
            const uint32_t bits = BloomBits(h);
            ok[j] = (bloom[BloomWord(h, nb)] & bits) == bits;
        }
        b[j] = h & jt.bmask;
        k[j] = ok[j] ? BucketKeys(jt, b[j]) : make_ulonglong2(kEmptyKey, kEmptyKey);
        p[j] = (ok[j] && L.S.need_pay) ? BucketPays(jt, b[j]) : make_ulonglong2(0, 0);
    }
#pragma unroll
    for (int j = 0; j < kJsRows; ++j) {
        if (ok[j] && k[j].x != kEmptyKey) {
            if (k[j].x == key[j]) JsFoldSlot<NS, C0, C1>(L, a, row[j], sv[j], p[j].x, 2 * b[j]);
            if (k[j].y != kEmptyKey) {
                if (k[j].y == key[j]) JsFoldSlot<NS, C0, C1>(L, a, row[j], sv[j], p[j].y, 2 * b[j] + 1);
                // Both slots taken: the key's sequence goes on (rare at load <= 1/2).
                const uint64_t nb2 = (b[j] + 1) & jt.bmask;
                const uint64_t kk = key[j];
                const int64_t rr = row[j];
                const int64_t vv = sv[j];
                VisitMatches(jt, kk, nb2, BucketKeys(jt, nb2), [&](uint64_t slot, uint64_t bk, int jj) {
                    const uint64_t pay = L.S.need_pay ? jt.buckets[4 * bk + 2 + jj] : 0;
                    JsFoldSlot<NS, C0, C1>(L, a, rr, vv, pay, slot);
                });
            }
        }
        // The one key equal to the empty marker lives in the side list.
        if (valid[j] && key[j] == kEmptyKey) {
            for (int64_t q = 0; q < nspecial; ++q) {
                if constexpr (NS == 0) {
                    JsFold(L, a, row[j], sv[j], uint64_t(jt.special_rows[2 * q + 1]),
                           L.S.need_row ? jt.special_rows[2 * q] : 0);
                } else {
                    JsFoldSlot<NS, C0, C1>(L, a, row[j], sv[j], uint64_t(jt.special_rows[2 * q + 1]), 0);
                }
            }
        }
    }
}

// Waits for `phase` of `bar`; false when the wait ran out or another warp
// raised the abort flag.
__device__ __forceinline__ bool JsWait(uint64_t* bar, uint32_t phase, const volatile unsigned* abort) {
    if (MbarTryWait(bar, phase)) return true;
    const long long start = clock64();
    while (!MbarTryWait(bar, phase)) {
        if (*abort) return false;
        if (clock64() - start > kSpinCycles) return false;
    }
    return true;
}

// Probes kJsRows rows of one thread against the direct-address index: the
// key's offset in the dense range, the presence bit in shared memory, then
// every surviving row's 16-byte entry {key, payload} in one batch (a folded
// bitmap lets a neighbour's key through; the key compare settles it).
template <int NS, int C0, int C1>
__device__ __forceinline__ void JsProbeDense(const JsLaunch& L, JsAcc& a, const uint32_t* bits,
                                             const int64_t (&row)[kJsRows], const uint64_t (&key)[kJsRows],
                                             const int64_t (&sv)[kJsRows], const bool (&valid)[kJsRows]) {
    const JTableDev& jt = L.jt;
    ulonglong2 e[kJsRows];
    bool ok[kJsRows];
#pragma unroll
    for (int j = 0; j < kJsRows; ++j) {
        const uint64_t d = key[j] - uint64_t(jt.dense_min);
        ok[j] = valid[j] && d < jt.dense_range;
        const uint64_t bit = ok[j] ? (d >> jt.dense_shift) : 0;
        ok[j] = ok[j] && ((bits[bit >> 5] >> (bit & 31)) & 1u);
        e[j] = ok[j] ? __ldg(jt.dense + d) : make_ulonglong2(kEmptyKey, 0);
    }
#pragma unroll
    for (int j = 0; j < kJsRows; ++j) {
        if (ok[j] && e[j].x == key[j]) JsFoldSlot<NS, C0, C1>(L, a, row[j], sv[j], e[j].y, 0);
    }
}

template <int NS, int C0, int C1, bool DENSE>
__global__ void __launch_bounds__(kJsThreads, 1) JoinSumKernel(const __grid_constant__ JsLaunch L) {
    extern __shared__ __align__(128) unsigned char smem[];
    uint64_t* full = reinterpret_cast<uint64_t*>(smem);
    uint64_t* empty = full + kJsStages;
    volatile unsigned* abort = reinterpret_cast<volatile unsigned*>(empty + kJsStages);
    unsigned char* stages = smem + kJsBarBytes;
    uint32_t* bloom = reinterpret_cast<uint32_t*>(stages + size_t(kJsStages) * L.stage_bytes);
    const int tid = threadIdx.x;
    const int warp = tid >> 5;
    const int32_t nb = L.bloom_words;
    // Tiles the producer issued bulk copies for (read only on the abort path).
    __shared__ long long issued_tiles;

    if (tid == 0) {
        for (int s = 0; s < kJsStages; ++s) {
            MbarInit(&full[s], 1);
            MbarInit(&empty[s], kJsConsumerWarps);
        }
        *abort = 0;
        issued_tiles = 0;
        FenceBarrierInit();
    }
    // The build side's Bloom filter (or the direct index's presence bitmap)
    // goes to shared memory: most probe rows miss and are rejected there
    // without touching the table in L2.
    const uint32_t* filter_src = DENSE ? L.jt.dense_bits : L.jt.bloom;
    for (int w = tid * 4; w < nb; w += blockDim.x * 4) {
        *reinterpret_cast<uint4*>(&bloom[w]) = __ldg(reinterpret_cast<const uint4*>(&filter_src[w]));
    }
    __syncthreads();

    const int64_t nspecial = L.jt.nspecial ? int64_t(*L.jt.nspecial) : 0;
    JsAcc acc;
#pragma unroll
    for (int s = 0; s < kJsMaxStates; ++s) acc.v[s] = 0;
    acc.matched = 0;
    bool failed = false;

    if (warp == kJsConsumerWarps) {
        // Producer: one lane streams the CTA's tiles into the stages.
        if ((tid & 31) == 0) {
            const uint64_t pol = EvictFirstPolicy();
            const uint32_t half = uint32_t(kJsTile * 8);
            int64_t k = 0;
            for (;; ++k) {
                const int64_t t = blockIdx.x + k * gridDim.x;
                if (t >= L.staged_tiles) break;
                const int s = int(k % kJsStages);
                if (k >= kJsStages && !JsWait(&empty[s], uint32_t(((k / kJsStages) - 1) & 1), abort)) {
                    failed = true;
                    break;
                }
                unsigned char* st = stages + size_t(s) * L.stage_bytes;
                FenceProxyAsync();
                MbarArriveExpectTx(&full[s], uint32_t(L.stage_bytes));
                BulkG2SHint(st, L.S.probe_key + t * kJsTile, half, &full[s], pol);
                if (L.vcol) BulkG2SHint(st + half, L.vcol + t * kJsTile, half, &full[s], pol);
            }
            issued_tiles = k;
        }
    } else {
        // Consumers: staged tiles, then the rows past the last full tile.
        for (int64_t k = 0;; ++k) {
            const int64_t t = blockIdx.x + k * gridDim.x;
            if (t >= L.staged_tiles) break;
            const int s = int(k % kJsStages);
            if (!JsWait(&full[s], uint32_t((k / kJsStages) & 1), abort)) {
                failed = true;
                break;
            }
            const unsigned char* st = stages + size_t(s) * L.stage_bytes;
            const uint64_t* ks = reinterpret_cast<const uint64_t*>(st);
            const int64_t* vs = reinterpret_cast<const int64_t*>(st + kJsTile * 8);
            int64_t row[kJsRows];
            uint64_t key[kJsRows];
            int64_t sv[kJsRows];
            bool valid[kJsRows];
#pragma unroll
            for (int j = 0; j < kJsRows; ++j) {
                const int rl = tid + j * kJsConsumers;
                row[j] = t * kJsTile + rl;
                key[j] = ks[rl];
                sv[j] = L.vcol ? vs[rl] : 0;
                valid[j] = true;
            }
            // The stage is in registers: hand it back before probing.
            __syncwarp();
            if ((tid & 31) == 0) {
                asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(SmemAddr(&empty[s])) : "memory");
            }
            if constexpr (DENSE) JsProbeDense<NS, C0, C1>(L, acc, bloom, row, key, sv, valid);
            else JsProbe<NS, C0, C1>(L, acc, bloom, nb, nspecial, row, key, sv, valid);
        }
        if (!failed) {
            const int64_t step = int64_t(gridDim.x) * kJsConsumers;
            for (int64_t base = L.staged_tiles * kJsTile + int64_t(blockIdx.x) * kJsConsumers + tid; base < L.nrows;
                 base += step * kJsRows) {
                int64_t row[kJsRows];
                uint64_t key[kJsRows];
                int64_t sv[kJsRows];
                bool valid[kJsRows];
#pragma unroll
                for (int j = 0; j < kJsRows; ++j) {
                    row[j] = base + j * step;
                    valid[j] = row[j] < L.nrows;
                    key[j] = valid[j] ? uint64_t(__ldcs(&L.S.probe_key[row[j]])) : 0;
                    sv[j] = (valid[j] && L.vcol) ? __ldcs(&L.vcol[row[j]]) : 0;
                }
                if constexpr (DENSE) JsProbeDense<NS, C0, C1>(L, acc, bloom, row, key, sv, valid);
                else JsProbe<NS, C0, C1>(L, acc, bloom, nb, nspecial, row, key, sv, valid);
            }
        }
    }
    if (failed) {
        *abort = 1;
        SetError(&L.counters->error, DE_WAIT_TIMEOUT);
    }
    __syncthreads();
    if (*abort) {
        // Copies already issued must land before the CTA's shared memory goes
        // away.  Only the last kJsStages issued tiles can still be in flight
        // (the producer reuses a stage only after its consumers released it,
        // which they do after its copy landed): wait for each of their `full`
        // phases, each wait bounded.
        if (tid == 0) {
            const long long n = issued_tiles;
            for (long long k = n > kJsStages ? n - kJsStages : 0; k < n; ++k) {
                const int s = int(k % kJsStages);
                const uint32_t phase = uint32_t((k / kJsStages) & 1);
                const long long start = clock64();
                while (!MbarTryWait(&full[s], phase)) {
                    if (clock64() - start > kSpinCycles) break;
                }
            }
        }
        __syncthreads();
        return;
    }
    // Block reduction: warp sums, then one atomic per state word per CTA.
    __shared__ uint64_t part[kJsMaxStates + 1][kJsThreads / 32];
#pragma unroll
    for (int s = 0; s < kJsMaxStates; ++s) {
        const uint64_t v = WarpSumU64(acc.v[s]);
        if (LaneId() == 0) part[s][warp] = v;
    }
    {
        const uint64_t v = WarpSumU64(acc.matched);
        if (LaneId() == 0) part[kJsMaxStates][warp] = v;
    }
    __syncthreads();
    if (tid < kJsMaxStates + 1) {
        uint64_t t = 0;
        for (int w = 0; w < kJsThreads / 32; ++w) t += part[tid][w];
        if (tid < kJsMaxStates) {
            if (tid < L.S.nstates && t) {
                atomicAdd(reinterpret_cast<unsigned long long*>(L.group_states + L.S.states[tid].word),
                          (unsigned long long)t);
            }
        } else if (t) {
            atomicAdd(&L.counters->matched, (unsigned long long)t);
        }
    }
}

bool Aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15) == 0; }

// QDB_JOIN_DIRECT=0 keeps the fused probe on the hashed bucket table even
// when the build has a direct-address index (to compare the two paths).
bool DenseDisabled() {
    const char* e = std::getenv("QDB_JOIN_DIRECT");
    return e && e[0] == '0';
}

// State code of `st` (see JsTerm), canonicalising f(sv) * g(pay) to
// g(pay) * f(sv) (wrapping products commute); -1: only the runtime fold.
int StateCode(JsState& st) {
    if (st.nf == 0) return 0;
    auto src = [](const JsFactor& f) { return f.side == 1 ? 1 : f.side == 3 ? 2 : 0; };
    if (st.nf == 1) return src(st.f[0]) == 0 ? -1 : src(st.f[0]);
    const int a = src(st.f[0]);
    const int b = src(st.f[1]);
    if (a == 0 || b == 0) return -1;
    if (a == 2 && b == 1) {
        std::swap(st.f[0], st.f[1]);
        return 3;
    }
    if (a == 1 && b == 2) return 3;
    return a == 1 ? 4 : 5;
}

using JsKernelFn = void (*)(JsLaunch);

// The instantiated signatures: one state of any code, or a SUM of codes 1-3
// beside a COUNT(*) in either order; anything else runs the runtime fold
// (never with the direct index, which carries no arena row).
template <bool DENSE>
JsKernelFn PickKernelOf(JsLaunch& L) {
    int code[kJsMaxStates];
    for (int st = 0; st < L.S.nstates; ++st) {
        code[st] = StateCode(L.S.states[st]);
        if (code[st] < 0 || L.S.need_row) return JoinSumKernel<0, 0, 0, DENSE>;
    }
    if (L.S.nstates == 1) {
        switch (code[0]) {
            case 0: return JoinSumKernel<1, 0, 0, DENSE>;
            case 1: return JoinSumKernel<1, 1, 0, DENSE>;
            case 2: return JoinSumKernel<1, 2, 0, DENSE>;
            case 3: return JoinSumKernel<1, 3, 0, DENSE>;
            default: break;
        }
    } else if (L.S.nstates == 2) {
        const int k = code[0] * 8 + code[1];
        switch (k) {
            case 1 * 8 + 0: return JoinSumKernel<2, 1, 0, DENSE>;
            case 2 * 8 + 0: return JoinSumKernel<2, 2, 0, DENSE>;
            case 3 * 8 + 0: return JoinSumKernel<2, 3, 0, DENSE>;
            case 0 * 8 + 1: return JoinSumKernel<2, 0, 1, DENSE>;
            case 0 * 8 + 2: return JoinSumKernel<2, 0, 2, DENSE>;
            case 0 * 8 + 3: return JoinSumKernel<2, 0, 3, DENSE>;
            default: break;
        }
    }
    return JoinSumKernel<0, 0, 0, DENSE>;
}

}  // namespace

namespace {

void JoinSumLaunch(const JoinSumShape& shape, const JTableDev& jt, int64_t nrows, uint64_t* group_states,
                   AggCounters* counters, cudaStream_t s) {
    if (nrows == 0) return;
    static thread_local JsLaunch L;
    std::memset(&L, 0, sizeof(L));
    L.S = shape;
    L.jt = jt;
    L.nrows = nrows;
    L.group_states = group_states;
    L.counters = counters;
    // The first probe-side factor column is staged with the keys; every
    // factor that reads it takes the staged value.
    for (int st = 0; st < L.S.nstates; ++st) {
        for (int f = 0; f < L.S.states[st].nf; ++f) {
            JsFactor& jf = L.S.states[st].f[f];
            if (jf.side != 0) continue;
            if (!L.vcol) L.vcol = jf.data;
            if (jf.data == L.vcol) jf.side = 3;
        }
    }
    const bool aligned = Aligned16(L.S.probe_key) && (!L.vcol || Aligned16(L.vcol));
    L.stage_bytes = kJsTile * 8 * (L.vcol ? 2 : 1);
    L.staged_tiles = aligned ? nrows / kJsTile : 0;
    const size_t base = size_t(kJsBarBytes) + size_t(kJsStages) * L.stage_bytes;
    const size_t room = MaxSmemOptin() > base + 1024 ? (MaxSmemOptin() - base - 1024) / 4 : 0;
    // The direct index when the table has one and the shape needs no arena
    // row; its presence bitmap takes the Bloom filter's place.
    const bool dense = jt.dense && !L.S.need_row && size_t(jt.dense_words) <= room && !DenseDisabled();
    if (dense) {
        L.bloom_words = (jt.dense_words + 3) & ~3;
    } else {
        L.jt.dense = nullptr;
        L.bloom_words = (jt.bloom && size_t(jt.bloom_words) <= room) ? jt.bloom_words : 0;
    }
    const size_t smem = base + size_t(L.bloom_words) * 4;
    const int64_t tiles = std::max<int64_t>(1, (nrows + kJsTile - 1) / kJsTile);
    const int blocks = int(std::min<int64_t>(tiles, DeviceSMs()));
    const JsKernelFn fn = dense ? PickKernelOf<true>(L) : PickKernelOf<false>(L);
    EnsureSmemLimit(reinterpret_cast<const void*>(fn), smem);
    ProfileBegin(s, "join_agg_probe", nrows);
    fn<<<blocks, kJsThreads, smem, s>>>(L);
    ProfileEnd(s);
    CountLaunch();
}

// The probe-side column every probe factor reads (the one staged beside the
// keys), or nullptr when none does; false when factors read two different
// probe columns or a build column through the arena row.
bool SingleProbeColumn(const JoinSumShape& shape, const int64_t*& vcol) {
    vcol = nullptr;
    if (shape.need_row) return false;
    for (int st = 0; st < shape.nstates; ++st) {
        for (int f = 0; f < shape.states[st].nf; ++f) {
            const JsFactor& jf = shape.states[st].f[f];
            if (jf.side == 2) return false;
            if (jf.side != 0 && jf.side != 3) continue;
            if (vcol && jf.data != vcol) return false;
            vcol = jf.data;
        }
    }
    return true;
}

// A probe of a table larger than L2: the probe rows (key, and the one value
// column the factors read) are radix-partitioned by the high bits of their
// home bucket into 16-row-aligned runs, then each partition is probed by its
// own launch, whose bucket reads stay inside one L2-sized slice.
bool JoinSumPartitioned(const JoinSumShape& shape, const JTableDev& jt, int64_t nrows, uint64_t* group_states,
                        AggCounters* counters, int parts, int part_shift, const int64_t* vcol, cudaStream_t s) {
    const int64_t cap = nrows + int64_t(parts) * 16;
    auto* counts = static_cast<unsigned long long*>(DevAlloc(size_t(parts) * 16, s));
    auto* pkeys = static_cast<int64_t*>(DevAlloc(size_t(cap) * 8, s));
    auto* pvals = vcol ? static_cast<int64_t*>(DevAlloc(size_t(cap) * 8, s)) : nullptr;
    auto cleanup = [&] {
        DevFree(counts, s);
        DevFree(pkeys, s);
        DevFree(pvals, s);
    };
    if (!counts || !pkeys || (vcol && !pvals)) {
        cleanup();
        return false;
    }
    unsigned long long* cursor = counts + parts;
    cudaMemsetAsync(counts, 0, size_t(parts) * 8, s);
    JoinPartCountProbe(shape.probe_key, nrows, jt.bmask, part_shift, parts, counts, s);
    std::vector<unsigned long long> cnt(static_cast<size_t>(parts)), off(static_cast<size_t>(parts));
    cudaMemcpyAsync(cnt.data(), counts, size_t(parts) * 8, cudaMemcpyDeviceToHost, s);
    if (cudaStreamSynchronize(s) != cudaSuccess) {
        cleanup();
        return false;
    }
    unsigned long long run = 0;
    for (int p = 0; p < parts; ++p) {
        off[size_t(p)] = run;
        run += (cnt[size_t(p)] + 15) / 16 * 16;   // each run starts on a 128-byte boundary
    }
    cudaMemcpyAsync(cursor, off.data(), size_t(parts) * 8, cudaMemcpyHostToDevice, s);
    JoinPartScatterProbe(shape.probe_key, vcol, nrows, jt.bmask, part_shift, parts, cursor, pkeys, pvals, s);
    JTableDev pt = jt;
    pt.bloom = nullptr;      // a filter of a table this size rejects little
    pt.bloom_words = 0;
    pt.dense = nullptr;
    for (int p = 0; p < parts; ++p) {
        if (!cnt[size_t(p)]) continue;
        JoinSumShape sp = shape;
        sp.probe_key = pkeys + off[size_t(p)];
        for (int st = 0; st < sp.nstates; ++st) {
            for (int f = 0; f < sp.states[st].nf; ++f) {
                JsFactor& jf = sp.states[st].f[f];
                if ((jf.side == 0 || jf.side == 3) && jf.data == vcol) jf.data = pvals + off[size_t(p)];
            }
        }
        JoinSumLaunch(sp, pt, int64_t(cnt[size_t(p)]), group_states, counters, s);
    }
    cleanup();
    return true;
}

}  // namespace

bool JoinSumProbeColumn(const JoinSumShape& shape, const int64_t*& vcol) { return SingleProbeColumn(shape, vcol); }

void JoinSumRun(const JoinSumShape& shape, const JTableDev& jt, int64_t nrows, uint64_t* group_states,
                AggCounters* counters, cudaStream_t s) {
    if (nrows == 0) return;
    const bool direct = jt.dense && !shape.need_row && !DenseDisabled();
    int part_shift = 0;
    const int parts = direct ? 1 : JoinPartsFor(int64_t(jt.bmask) + 1, part_shift);
    const int64_t* vcol = nullptr;
    if (parts > 1 && SingleProbeColumn(shape, vcol) &&
        JoinSumPartitioned(shape, jt, nrows, group_states, counters, parts, part_shift, vcol, s)) {
        return;
    }
    JoinSumLaunch(shape, jt, nrows, group_states, counters, s);
}

// ---------------------------------------------------------------------------
// Batched join-sum probe: many small joins of one program (the partitions of
// a partitioned join, or the joins of many queries of one template) in one
// persistent launch.  A warp pulls a work item (join, range of at most
// 16K probe rows), probes two rows per lane per step against that
// join's bucket table (left in L2: small tables, no staging or Bloom filter),
// and ends the item with a warp reduction and one atomic add per state word.
// ---------------------------------------------------------------------------
namespace {

constexpr int kJsBatchRows = 2;   // rows per lane per step

struct JsBatchLaunch {
    JoinSumShape S;
    const JsBatchJoin* joins;
    const JoinBatchItem* items;
    int64_t nitems;
    unsigned* next;
};

__device__ __forceinline__ uint64_t JsBatchTerm(const JsState& st, uint64_t pay, int64_t sv) {
    uint64_t v = 1;
#pragma unroll
    for (int f = 0; f < 2; ++f) {
        if (f >= st.nf) break;
        const JsFactor& jf = st.f[f];
        v *= uint64_t(jf.c) + uint64_t(jf.d) * (jf.side == 1 ? pay : uint64_t(sv));
    }
    return v;
}

__global__ void __launch_bounds__(256, 4) JoinSumBatchKernel(const __grid_constant__ JsBatchLaunch L) {
    const int lane = LaneId();
    for (;;) {
        unsigned it = 0;
        if (lane == 0) it = atomicAdd(L.next, 1u);
        it = __shfl_sync(kFull, it, 0);
        if (int64_t(it) >= L.nitems) return;
        const JoinBatchItem item = L.items[it];
        const JsBatchJoin& J = L.joins[item.join];
        const JTableDev& jt = J.jt;
        const int64_t nspecial = int64_t(*jt.nspecial);
        uint64_t v[kJsMaxStates];
#pragma unroll
        for (int s = 0; s < kJsMaxStates; ++s) v[s] = 0;
        unsigned long long matched = 0;
        auto fold = [&](uint64_t pay, int64_t sv) {
            ++matched;
#pragma unroll
            for (int s = 0; s < kJsMaxStates; ++s) {
                if (s < L.S.nstates) v[s] += JsBatchTerm(L.S.states[s], pay, sv);
            }
        };
        // Two coalesced 32-row slabs per step: every lane's key loads, then
        // its bucket reads, are in flight together (two rows per lane keep
        // 60 registers, so that four CTAs fit an SM).
        for (int64_t r0 = item.lo + lane; r0 < item.hi; r0 += 32 * kJsBatchRows) {
            uint64_t key[kJsBatchRows];
            int64_t sv[kJsBatchRows];
            bool on[kJsBatchRows];
#pragma unroll
            for (int j = 0; j < kJsBatchRows; ++j) {
                const int64_t r = r0 + 32 * j;
                on[j] = r < item.hi;
                key[j] = on[j] ? uint64_t(__ldcs(&J.key[r])) : 0;
                sv[j] = (on[j] && J.vcol) ? __ldcs(&J.vcol[r]) : 0;
            }
            uint64_t b[kJsBatchRows];
            ulonglong2 k[kJsBatchRows], p[kJsBatchRows];
#pragma unroll
            for (int j = 0; j < kJsBatchRows; ++j) {
                const bool probe = on[j] && key[j] != kEmptyKey;
                b[j] = Fmix64(key[j]) & jt.bmask;
                k[j] = probe ? BucketKeys(jt, b[j]) : make_ulonglong2(kEmptyKey, kEmptyKey);
                p[j] = (probe && L.S.need_pay) ? BucketPays(jt, b[j]) : make_ulonglong2(0, 0);
            }
#pragma unroll
            for (int j = 0; j < kJsBatchRows; ++j) {
                if (!on[j]) continue;
                if (key[j] == kEmptyKey) {   // the one key equal to the empty marker lives in the side list
                    for (int64_t q = 0; q < nspecial; ++q) fold(uint64_t(jt.special_rows[2 * q + 1]), sv[j]);
                    continue;
                }
                if (k[j].x == kEmptyKey) continue;
                if (k[j].x == key[j]) fold(p[j].x, sv[j]);
                if (k[j].y == kEmptyKey) continue;
                if (k[j].y == key[j]) fold(p[j].y, sv[j]);
                // Both slots taken: the key's sequence goes on.
                const uint64_t nb = (b[j] + 1) & jt.bmask;
                const int64_t v = sv[j];
                VisitMatches(jt, key[j], nb, BucketKeys(jt, nb), [&](uint64_t, uint64_t bk, int jj) {
                    fold(L.S.need_pay ? jt.buckets[4 * bk + 2 + jj] : 0, v);
                });
            }
        }
#pragma unroll
        for (int s = 0; s < kJsMaxStates; ++s) {
            if (s >= L.S.nstates) break;
            const uint64_t t = WarpSumU64(v[s]);
            if (lane == 0 && t) atomicAdd(reinterpret_cast<unsigned long long*>(J.states + L.S.states[s].word), t);
        }
        const uint64_t m = WarpSumU64(matched);
        if (lane == 0 && m) atomicAdd(J.matched, (unsigned long long)m);
    }
}

}  // namespace

void JoinSumBatchRun(const JoinSumShape& shape, const JsBatchJoin* joins, const JoinBatchItem* items,
                     int64_t nitems, unsigned* next, cudaStream_t s) {
    if (nitems == 0) return;
    JsBatchLaunch L;
    std::memset(&L, 0, sizeof(L));
    L.S = shape;
    L.joins = joins;
    L.items = items;
    L.nitems = nitems;
    L.next = next;
    // Four CTAs of eight warps per SM (64 registers each), fewer when there
    // are fewer items than warps.
    const int warps = int(std::min<int64_t>(nitems, int64_t(DeviceSMs()) * 32));
    ProfileBegin(s, "join_agg_probe_batch", nitems);
    JoinSumBatchKernel<<<(warps + 7) / 8, 256, 0, s>>>(L);
    ProfileEnd(s);
    CountLaunch();
}

}  // namespace qdb
