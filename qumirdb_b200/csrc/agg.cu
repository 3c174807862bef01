// agg.cu — fused filter -> project -> hash aggregate for sm_100a.
//
// One persistent CTA per SM streams row tiles of every referenced column
// into shared memory with 1-D bulk copies (cp.async.bulk, completion on an
// mbarrier; several stages in flight), evaluates the predicate, group key and
// aggregate arguments per row from shared memory, and folds rows into
//   (1) a per-CTA shared-memory group table (low cardinality, and the hot
//       head of a skewed key distribution), after a warp-level
//       pre-aggregation (__match_any_sync + butterfly reduction) when a warp
//       holds few distinct groups, and
//   (2) a global open-addressing table in HBM (one cache-line-sized slot per
//       group: key + state words; CAS key claim, atomic state updates).
// At the end each CTA merges its shared table into the global one.  A row
// whose global probe exceeds the probe bound is deferred (row id to a list)
// and a shared entry that cannot be merged is spilled; the host grows the
// table and replays both, so no row is ever lost or double counted.
//
// Semantics match the engine's reducers (qdb/kernel/gen.cpp:3301-3593): i64
// sums wrap, decimal sums are exact i128, COUNT counts non-NULL inputs, MIN /
// MAX fold non-NULL inputs, f64 sums are IEEE additions in device order.
#include <algorithm>
#include <cstdio>
#include <cstring>

#include "common.cuh"
#include "eval.h"
#include "kernels.h"
#include "lower.h"

namespace qdb {

constexpr int kAggThreads = 512;
constexpr int kWarpAggMax = 4;     // leader-loop pre-aggregation up to this many groups per warp
constexpr int kMaxProbe = 256;     // global table probe bound before a row is deferred

__device__ __forceinline__ int64_t Min64(int64_t a, int64_t b) { return a < b ? a : b; }

struct StatesParam {
    StateDesc s[kMaxStates];
    int32_t n;
};

struct AggLaunch {
    AggPlan P;
    int64_t nrows;
    const int64_t* index;
    int64_t nindex;
    int32_t tile_rows;
    int32_t stages;
    int32_t stage_bytes;
    int32_t sel_off;          // selection tile offset inside a stage (-1: not staged)
    int32_t smem_slots;
    int32_t smem_limit;
    int32_t off_bars;
    int32_t off_bases;
    int32_t off_skeys;
    int32_t off_sst;
    int32_t off_misc;
    int32_t any_staged;
    GTableDev T;
    uint64_t cap_mask;
    AggCounters* counters;
    int64_t* deferred;
    int64_t deferred_cap;
    uint64_t* spill;
    int64_t spill_cap;
    int32_t join;
    JoinKeyPlan jk;
    JTableDev jt;
};

// ---------------------------------------------------------------------------
// Row accessor over staged tiles, global columns and gathered build rows.
// ---------------------------------------------------------------------------
struct RowAcc {
    const AggPlan* P;
    const char* const* base;  // tile base per column slot (smem or global), or nullptr
    int r;                    // row inside the tile
    int64_t arow;             // row inside the launch range
    int64_t brow;             // matched build row (fused join)

    __device__ __forceinline__ const char* Ptr(int c) const {
        const ColDesc& cd = P->cols[c];
        if (cd.build) return cd.data + brow * cd.width;
        if (base) return base[c] + int64_t(r) * cd.width;
        return cd.data + arow * cd.width;
    }
    __device__ __forceinline__ i128 Int(int c) const {
        const ColDesc& cd = P->cols[c];
        if (cd.kind == LK_BOOLBIT) {
            const int64_t bit = cd.bit_off + (cd.build ? brow : arow);
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
        const int64_t bit = cd.mask_off + (cd.build ? brow : arow);
        return !((cd.mask[bit >> 3] >> (bit & 7)) & 1);
    }
};

// One-word key of the current row (every part lives in word 0).
__device__ __forceinline__ uint64_t PackKey1(const AggPlan& p, const RowAcc& a, const GVal* gv, uint64_t gn) {
    uint64_t w[kMaxKeyWords];
    PackKey(p, a, gv, gn, w);
    return w[0];
}

// ---------------------------------------------------------------------------
// State inputs and updates.
// ---------------------------------------------------------------------------
struct Contrib {
    uint64_t lo;
    uint64_t hi;
    double f;
    bool has;
};

__device__ __forceinline__ Contrib StateInput(const AggPlan& P, const StateDesc& sd, const RowAcc& acc,
                                              const GVal* gv, uint64_t gn) {
    Contrib c{0, 0, 0.0, true};
    if (sd.src == VS_NONE) {
        c.lo = 1;
        return c;
    }
    bool null;
    i128 iv = 0;
    double fv = 0.0;
    if (sd.src == VS_SOP) {
        const SopValue& v = P.values[sd.idx];
        null = SopNull(v, acc);
        if (!null) {
            if (v.kind == VK_F64) fv = SopF64(v, acc);
            else iv = SopInt(v, acc);
        }
    } else {
        null = (gn >> sd.idx) & 1;
        if (!null) {
            if (P.prog.nodes[sd.idx].dom == GD_F64) fv = gv[sd.idx].f;
            else iv = gv[sd.idx].i;
        }
    }
    if (sd.kind == ST_COUNT) {
        c.lo = null ? 0 : 1;
        c.has = !null;
        return c;
    }
    if (null) {
        c.has = false;
        return c;
    }
    switch (sd.kind) {
        case ST_SUM_I128:
            c.lo = uint64_t(u128(iv));
            c.hi = uint64_t(u128(iv) >> 64);
            break;
        case ST_SUM_F64: c.f = fv; break;
        case ST_MIN_F64: case ST_MAX_F64: c.lo = F64Ordered(fv); break;
        default: c.lo = uint64_t(int64_t(iv)); break;
    }
    return c;
}

__device__ __forceinline__ uint64_t StateIdentity(uint8_t kind) {
    switch (kind) {
        case ST_MIN_I64: return uint64_t(INT64_MAX);
        case ST_MAX_I64: return uint64_t(INT64_MIN);
        case ST_MIN_F64: return ~0ull;
        default: return 0;
    }
}

// Atomic fold into a state word w (and w_hi for 128-bit sums); works on
// shared and global memory.
__device__ __forceinline__ void ApplyState(uint64_t* w, uint64_t* w_hi, uint8_t kind, uint64_t lo, uint64_t hi,
                                           double f) {
    auto* u = reinterpret_cast<unsigned long long*>(w);
    switch (kind) {
        case ST_COUNT:
        case ST_SUM_I64: atomicAdd(u, (unsigned long long)lo); break;
        case ST_SUM_I128: {
            const unsigned long long old = atomicAdd(u, (unsigned long long)lo);
            const unsigned long long carry = (old + lo < old) ? 1ull : 0ull;
            const unsigned long long h = hi + carry;
            if (h) atomicAdd(reinterpret_cast<unsigned long long*>(w_hi), h);
            break;
        }
        case ST_SUM_F64: atomicAdd(reinterpret_cast<double*>(w), f); break;
        case ST_MIN_I64: atomicMin(reinterpret_cast<long long*>(w), (long long)lo); break;
        case ST_MAX_I64: atomicMax(reinterpret_cast<long long*>(w), (long long)lo); break;
        case ST_MIN_F64: atomicMin(u, (unsigned long long)lo); break;
        case ST_MAX_F64: atomicMax(u, (unsigned long long)lo); break;
    }
}

// Butterfly reduction of one contribution over the lanes where `member`.
__device__ __forceinline__ void WarpReduceState(uint8_t kind, bool member, Contrib& c) {
    switch (kind) {
        case ST_COUNT:
        case ST_SUM_I64: c.lo = WarpSumU64(member ? c.lo : 0); break;
        case ST_SUM_I128: {
            uint64_t lo = member ? c.lo : 0, hi = member ? c.hi : 0;
            WarpSumU128(lo, hi);
            c.lo = lo;
            c.hi = hi;
            break;
        }
        case ST_SUM_F64: c.f = WarpSumF64(member ? c.f : 0.0); break;
        case ST_MIN_I64: c.lo = uint64_t(WarpMinI64(member ? (long long)c.lo : INT64_MAX)); break;
        case ST_MAX_I64: c.lo = uint64_t(WarpMaxI64(member ? (long long)c.lo : INT64_MIN)); break;
        case ST_MIN_F64: c.lo = WarpMinU64(member ? c.lo : ~0ull); break;
        case ST_MAX_F64: c.lo = WarpMaxU64(member ? c.lo : 0ull); break;
    }
}

__device__ __forceinline__ bool IsIdentity(uint8_t kind, uint64_t lo, uint64_t hi) {
    switch (kind) {
        case ST_SUM_I128: return lo == 0 && hi == 0;
        default: return lo == StateIdentity(kind);
    }
}

// ---------------------------------------------------------------------------
// Global table probes.
// ---------------------------------------------------------------------------
__device__ __forceinline__ int64_t GlobalFind1(const GTableDev& T, uint64_t mask, uint64_t key, int& is_new) {
    uint64_t i = Fmix64(key) & mask;
    for (int p = 0; p < kMaxProbe; ++p) {
        unsigned long long* kp =
            reinterpret_cast<unsigned long long*>(T.slots + int64_t(i) * T.slot_words + T.key_off);
        const uint64_t cur = *reinterpret_cast<volatile unsigned long long*>(kp);
        if (cur == key) return int64_t(i);
        if (cur == kEmptyKey) {
            const uint64_t old = atomicCAS(kp, kEmptyKey, key);
            if (old == kEmptyKey) {
                is_new = 1;
                return int64_t(i);
            }
            if (old == key) return int64_t(i);
        }
        i = (i + 1) & mask;
    }
    return -1;
}

// Multi-word keys: a status word (0 empty, 1 being written, 2 ready) leads
// the slot; the key words follow.
__device__ int64_t GlobalFindW(const GTableDev& T, uint64_t mask, const uint64_t* key, int kw, int& is_new,
                               int* err) {
    uint64_t h = 0;
    for (int w = 0; w < kw; ++w) h = Fmix64(h ^ key[w] ^ (uint64_t(w) << 56));
    uint64_t i = h & mask;
    for (int p = 0; p < kMaxProbe; ++p) {
        uint64_t* s = T.slots + int64_t(i) * T.slot_words;
        auto* st = reinterpret_cast<unsigned long long*>(s);
        uint64_t cur = *reinterpret_cast<volatile unsigned long long*>(st);
        if (cur == 0) {
            cur = atomicCAS(st, 0ull, 1ull);
            if (cur == 0) {
                for (int w = 0; w < kw; ++w) reinterpret_cast<volatile uint64_t*>(s)[1 + w] = key[w];
                __threadfence();
                atomicExch(st, 2ull);
                is_new = 1;
                return int64_t(i);
            }
        }
        if (cur == 1) {
            const long long start = clock64();
            while ((cur = *reinterpret_cast<volatile unsigned long long*>(st)) == 1) {
                if (clock64() - start > kSpinCycles) {
                    SetError(err, DE_WAIT_TIMEOUT);
                    return -2;
                }
            }
            __threadfence();
        }
        bool eq = true;
        for (int w = 0; w < kw && eq; ++w) eq = reinterpret_cast<volatile uint64_t*>(s)[1 + w] == key[w];
        if (eq) return int64_t(i);
        i = (i + 1) & mask;
    }
    return -1;
}

__device__ __forceinline__ void Defer(const AggLaunch& L, int64_t arow, int64_t brow) {
    const unsigned long long k = atomicAdd(&L.counters->deferred, 1ull);
    if (int64_t(k) < L.deferred_cap) {
        L.deferred[2 * k] = arow;
        L.deferred[2 * k + 1] = brow;
    } else {
        SetError(&L.counters->error, DE_DEFER_FULL);
    }
}

// ---------------------------------------------------------------------------
// Shared-memory tier (one-word keys).
// ---------------------------------------------------------------------------
struct SmemTable {
    uint64_t* keys;       // S keys (kEmptyKey = free)
    uint64_t* st;         // state word w of slot i at st[w * S + i]
    unsigned* count;      // keys inserted
    unsigned* fresh;      // global groups this CTA created
    int S;
    int limit;

    __device__ __forceinline__ int Find(uint64_t key) const {
        uint32_t i = uint32_t(Fmix64(key)) & uint32_t(S - 1);
        for (int p = 0; p < S; ++p) {
            const uint64_t cur = *reinterpret_cast<volatile uint64_t*>(&keys[i]);
            if (cur == key) return int(i);
            if (cur == kEmptyKey) {
                if (*reinterpret_cast<volatile unsigned*>(count) >= unsigned(limit)) return -1;
                const uint64_t old = atomicCAS(reinterpret_cast<unsigned long long*>(&keys[i]), kEmptyKey, key);
                if (old == kEmptyKey) {
                    atomicAdd(count, 1u);
                    return int(i);
                }
                if (old == key) return int(i);
            }
            i = (i + 1) & uint32_t(S - 1);
        }
        return -1;
    }
};

// ---------------------------------------------------------------------------
// Per-row (per-warp) fold of one joined/scanned row.  Warp-uniform.
// ---------------------------------------------------------------------------
template <bool WIDE, bool GEN>
__device__ __forceinline__ void FoldRow(const AggLaunch& L, const SmemTable& sm, bool act, const RowAcc& acc) {
    const AggPlan& P = L.P;
    GVal gv[GEN ? kMaxGNodes : 1];
    uint64_t gn = 0;
    if (GEN && act && P.generic_root >= 0) {
        if (!EvalGeneric(P.prog, P.generic_root, P.list, acc, gv, gn)) {
            SetError(&L.counters->error, DE_DIV_ZERO);
            act = false;
        }
    }
    if (act && P.filter_kind == 1) act = AtomsPass(P, acc);
    else if (GEN && act && P.filter_kind == 2) act = !((gn >> P.filter_node) & 1) && gv[P.filter_node].i != 0;

    int slot = -1;
    int64_t gslot = -1;
    if (!WIDE) {
        uint64_t key = 0;
        if (act) key = PackKey1(P, acc, gv, gn);
        const bool special = act && P.key_full64 && key == kEmptyKey;
        if (act && sm.S > 0 && !special) slot = sm.Find(key);
        if (act && slot < 0) {
            if (special) {
                gslot = L.T.capacity;
                unsigned long long* flag = reinterpret_cast<unsigned long long*>(
                    L.T.slots + L.T.capacity * L.T.slot_words + L.T.key_off);
                if (*reinterpret_cast<volatile unsigned long long*>(flag) == 0 && atomicExch(flag, 1ull) == 0) {
                    atomicAdd(sm.fresh, 1u);
                }
            } else {
                int is_new = 0;
                gslot = GlobalFind1(L.T, L.cap_mask, key, is_new);
                if (is_new) atomicAdd(sm.fresh, 1u);
            }
            if (gslot < 0) {
                Defer(L, acc.arow, acc.brow);
                act = false;
            }
        }
    } else {
        if (act) {
            uint64_t kw[kMaxKeyWords];
            PackKey(P, acc, gv, gn, kw);
            int is_new = 0;
            gslot = GlobalFindW(L.T, L.cap_mask, kw, P.key_words, is_new, &L.counters->error);
            if (is_new) atomicAdd(sm.fresh, 1u);
            if (gslot == -1) Defer(L, acc.arow, acc.brow);
            if (gslot < 0) act = false;
        }
    }

    const unsigned actmask = __ballot_sync(kFull, act);
    if (actmask == 0) return;
    const int grp = (act && slot >= 0) ? slot : -1;
    const unsigned peers = __match_any_sync(kFull, grp);
    const bool leader = grp >= 0 && LaneId() == __ffs(peers) - 1;
    const unsigned leaders = __ballot_sync(kFull, leader);
    const int nlead = __popc(leaders);
    const bool wagg = nlead > 0 && nlead <= kWarpAggMax;
    uint64_t* gbase = gslot >= 0 ? L.T.slots + gslot * L.T.slot_words + L.T.state_off : nullptr;

    for (int s = 0; s < P.nstates; ++s) {
        const StateDesc sd = P.states[s];
        Contrib c{0, 0, 0.0, false};
        if (act) c = StateInput(P, sd, acc, gv, gn);
        if (wagg) {
            unsigned lm = leaders;
            while (lm) {
                const int ld = __ffs(lm) - 1;
                lm &= lm - 1;
                const int lslot = __shfl_sync(kFull, slot, ld);
                Contrib r = c;
                WarpReduceState(sd.kind, act && c.has && slot == lslot, r);
                const bool any = sd.kind == ST_SUM_F64 ? r.f != 0.0 : !IsIdentity(sd.kind, r.lo, r.hi);
                if (LaneId() == ld && any) {
                    uint64_t* w = sm.st + int64_t(sd.word) * sm.S + lslot;
                    ApplyState(w, w + sm.S, sd.kind, r.lo, r.hi, r.f);
                }
            }
        } else if (act && slot >= 0 && c.has) {
            uint64_t* w = sm.st + int64_t(sd.word) * sm.S + slot;
            ApplyState(w, w + sm.S, sd.kind, c.lo, c.hi, c.f);
        }
        if (act && gslot >= 0 && c.has) {
            uint64_t* w = gbase + sd.word;
            ApplyState(w, w + 1, sd.kind, c.lo, c.hi, c.f);
        }
    }
}

// Probes the join table for the first match at or after slot `i`.
__device__ __forceinline__ int64_t JoinNext(const JTableDev& jt, uint64_t key, uint64_t i, int64_t& brow) {
    for (int64_t p = 0; p <= int64_t(jt.mask); ++p) {
        const uint64_t k = jt.entries[2 * i];
        if (k == kEmptyKey) return -1;
        if (k == key) {
            brow = int64_t(jt.entries[2 * i + 1]);
            return int64_t(i);
        }
        i = (i + 1) & jt.mask;
    }
    return -1;
}

__device__ __forceinline__ uint64_t PackJoinKey(const JoinKeyPlan& jk, const RowAcc& a, bool& null) {
    null = false;
    if (jk.n == 1 && !jk.is_float[0]) {
        if (a.Null(jk.col[0])) {
            null = true;
            return 0;
        }
        return uint64_t(int64_t(a.Int(jk.col[0])));
    }
    uint64_t k = 0;
    for (int j = 0; j < jk.n; ++j) {
        if (a.Null(jk.col[j])) {
            null = true;
            return 0;
        }
        uint64_t v = jk.is_float[j] ? CanonF64(a.F64(jk.col[j])) : uint64_t(u128(a.Int(jk.col[j])));
        if (jk.bits[j] < 64) v &= (1ull << jk.bits[j]) - 1;
        k |= v << jk.shift[j];
    }
    return k;
}

// Folds every joined row of probe row `acc` (fused join-aggregate).
template <bool WIDE, bool GEN>
__device__ __forceinline__ void FoldProbeRow(const AggLaunch& L, const SmemTable& sm, bool act, RowAcc acc) {
    bool null = false;
    uint64_t key = 0;
    if (act) key = PackJoinKey(L.jk, acc, null);
    act = act && !null;
    int64_t pos = -1;
    int64_t special_i = -1;
    const bool special = act && L.jk.full64 && key == kEmptyKey;
    if (act && !special) pos = JoinNext(L.jt, key, Fmix64(key) & L.jt.mask, acc.brow);
    if (special && L.jt.nspecial > 0) {
        special_i = 0;
        acc.brow = L.jt.special_rows[0];
    }
    unsigned matched = 0;
    while (__any_sync(kFull, pos >= 0 || special_i >= 0)) {
        const bool has = pos >= 0 || special_i >= 0;
        FoldRow<WIDE, GEN>(L, sm, has, acc);
        matched += has ? 1u : 0u;
        if (pos >= 0) {
            pos = JoinNext(L.jt, key, (uint64_t(pos) + 1) & L.jt.mask, acc.brow);
        } else if (special_i >= 0) {
            ++special_i;
            if (special_i < L.jt.nspecial) acc.brow = L.jt.special_rows[special_i];
            else special_i = -1;
        }
    }
    const unsigned total = __reduce_add_sync(kFull, matched);
    if (LaneId() == 0 && total) atomicAdd(&L.counters->matched, (unsigned long long)total);
}

template <bool WIDE, bool JOIN, bool GEN>
__global__ void __launch_bounds__(kAggThreads, 1) AggUpdateKernel(const __grid_constant__ AggLaunch L) {
    extern __shared__ __align__(128) unsigned char smem[];
    uint64_t* bars = reinterpret_cast<uint64_t*>(smem + L.off_bars);
    const char** sbase = reinterpret_cast<const char**>(smem + L.off_bases);
    unsigned* misc = reinterpret_cast<unsigned*>(smem + L.off_misc);
    SmemTable sm;
    sm.keys = reinterpret_cast<uint64_t*>(smem + L.off_skeys);
    sm.st = reinterpret_cast<uint64_t*>(smem + L.off_sst);
    sm.count = misc;
    sm.fresh = misc + 1;
    sm.S = WIDE ? 0 : L.smem_slots;
    sm.limit = L.smem_limit;
    const AggPlan& P = L.P;
    const int tid = threadIdx.x;

    if (tid == 0) {
        misc[0] = 0;
        misc[1] = 0;
        misc[2] = 0;
        for (int s = 0; s < L.stages; ++s) MbarInit(&bars[s], 1);
        FenceBarrierInit();
    }
    for (int i = tid; i < sm.S; i += blockDim.x) {
        sm.keys[i] = kEmptyKey;
        for (int s = 0; s < P.nstates; ++s) {
            const StateDesc sd = P.states[s];
            sm.st[int64_t(sd.word) * sm.S + i] = StateIdentity(sd.kind);
            if (sd.kind == ST_SUM_I128) sm.st[int64_t(sd.word + 1) * sm.S + i] = 0;
        }
    }
    __syncthreads();

    const int T = L.tile_rows;
    const int64_t ntiles = (L.nrows + T - 1) / T;
    auto tile_full = [&](int64_t t) { return L.any_staged && (t + 1) * int64_t(T) <= L.nrows; };
    auto issue = [&](int64_t t, int s) {
        unsigned char* st = smem + int64_t(s) * L.stage_bytes;
        FenceProxyAsync();
        MbarArriveExpectTx(&bars[s], uint32_t(L.stage_bytes));
        for (int c = 0; c < P.ncols; ++c) {
            const ColDesc& cd = P.cols[c];
            if (!cd.stage) continue;
            BulkG2S(st + cd.smem_off, cd.data + t * T * cd.width, uint32_t(T * cd.width), &bars[s]);
        }
        if (L.sel_off >= 0) BulkG2S(st + L.sel_off, P.selection + t * T, uint32_t(T), &bars[s]);
    };

    if (tid == 0) {
        for (int k = 0; k < L.stages; ++k) {
            const int64_t t = blockIdx.x + int64_t(k) * gridDim.x;
            if (t < ntiles && tile_full(t)) issue(t, k);
        }
    }

    bool aborted = false;
    for (int64_t k = 0;; ++k) {
        const int64_t t = blockIdx.x + k * gridDim.x;
        if (t >= ntiles) break;
        const int s = int(k % L.stages);
        const bool full = tile_full(t);
        const int64_t row0 = t * T;
        if (tid == 0) {
            unsigned char* st = smem + int64_t(s) * L.stage_bytes;
            for (int c = 0; c < P.ncols; ++c) {
                const ColDesc& cd = P.cols[c];
                sbase[c] = (full && cd.stage) ? reinterpret_cast<const char*>(st + cd.smem_off)
                                              : cd.data + row0 * cd.width;
            }
            sbase[kMaxCols] = P.selection == nullptr ? nullptr
                              : (full && L.sel_off >= 0) ? reinterpret_cast<const char*>(st + L.sel_off)
                                                         : reinterpret_cast<const char*>(P.selection + row0);
        }
        __syncthreads();
        if (full) {
            if (!MbarWaitBounded(&bars[s], uint32_t((k / L.stages) & 1))) {
                SetError(&L.counters->error, DE_WAIT_TIMEOUT);
                aborted = true;
            }
        }
        if (__syncthreads_or(aborted)) {
            aborted = true;
            break;
        }
        const int nrows = int(Min64(T, L.nrows - row0));
        const uint8_t* sel = reinterpret_cast<const uint8_t*>(sbase[kMaxCols]);
        for (int rb = (tid & ~31); rb < T; rb += blockDim.x) {
            const int r = rb + LaneId();
            bool act = r < nrows;
            if (act && sel) act = sel[r] != 0;
            RowAcc acc{&P, sbase, r, row0 + r, 0};
            if (JOIN) FoldProbeRow<WIDE, GEN>(L, sm, act, acc);
            else FoldRow<WIDE, GEN>(L, sm, act, acc);
        }
        __syncthreads();
        if (tid == 0) {
            const int64_t nt = t + int64_t(L.stages) * gridDim.x;
            if (nt < ntiles && tile_full(nt)) issue(nt, s);
        }
    }
    if (aborted) {
        // Let copies already issued land before the CTA's memory goes away.
        if (tid == 0) {
            for (int s = 0; s < L.stages; ++s) {
                const long long start = clock64();
                while (clock64() - start < 1000000) {
                }
            }
        }
        __syncthreads();
        return;
    }

    // Merge the shared table into the global table.
    __syncthreads();
    for (int i = tid; i < sm.S; i += blockDim.x) {
        const uint64_t key = sm.keys[i];
        if (key == kEmptyKey) continue;
        int is_new = 0;
        const int64_t g = GlobalFind1(L.T, L.cap_mask, key, is_new);
        if (is_new) atomicAdd(sm.fresh, 1u);
        if (g < 0) {
            const unsigned long long e = atomicAdd(&L.counters->spilled, 1ull);
            if (int64_t(e) >= L.spill_cap) {
                SetError(&L.counters->error, DE_SPILL_FULL);
                continue;
            }
            uint64_t* rec = L.spill + int64_t(e) * (1 + P.state_words);
            rec[0] = key;
            for (int w = 0; w < P.state_words; ++w) rec[1 + w] = sm.st[int64_t(w) * sm.S + i];
            continue;
        }
        uint64_t* gbase = L.T.slots + g * L.T.slot_words + L.T.state_off;
        for (int s = 0; s < P.nstates; ++s) {
            const StateDesc sd = P.states[s];
            const uint64_t lo = sm.st[int64_t(sd.word) * sm.S + i];
            const uint64_t hi = sd.kind == ST_SUM_I128 ? sm.st[int64_t(sd.word + 1) * sm.S + i] : 0;
            if (IsIdentity(sd.kind, lo, hi)) continue;
            double f;
            __builtin_memcpy(&f, &lo, 8);
            ApplyState(gbase + sd.word, gbase + sd.word + 1, sd.kind, lo, hi, f);
        }
    }
    __syncthreads();
    if (tid == 0 && sm.fresh[0]) atomicAdd(&L.counters->new_groups, (unsigned long long)sm.fresh[0]);
}

// Index mode: rows named by (row, build row) pairs, global table only.
template <bool WIDE>
__global__ void __launch_bounds__(256) AggIndexKernel(const __grid_constant__ AggLaunch L) {
    __shared__ unsigned misc[4];
    if (threadIdx.x == 0) misc[1] = 0;
    __syncthreads();
    SmemTable sm{nullptr, nullptr, misc, misc + 1, 0, 0};
    const int64_t warps = int64_t(gridDim.x) * (blockDim.x / 32);
    const int64_t wid = int64_t(blockIdx.x) * (blockDim.x / 32) + (threadIdx.x >> 5);
    for (int64_t b = wid * 32; b < L.nindex; b += warps * 32) {
        const int64_t i = b + LaneId();
        const bool act = i < L.nindex;
        RowAcc acc{&L.P, nullptr, 0, act ? L.index[2 * i] : 0, act ? L.index[2 * i + 1] : 0};
        FoldRow<WIDE, true>(L, sm, act, acc);
    }
    __syncthreads();
    if (threadIdx.x == 0 && misc[1]) atomicAdd(&L.counters->new_groups, (unsigned long long)misc[1]);
}

// ---------------------------------------------------------------------------
// Table maintenance kernels.
// ---------------------------------------------------------------------------
__global__ void AggInitKernel(uint64_t* slots, int64_t capacity, int32_t slot_words, int32_t key_off,
                              int32_t state_off, int32_t wide, const __grid_constant__ StatesParam sp) {
    const int64_t total = (capacity + 1) * slot_words;
    for (int64_t w = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; w < total; w += int64_t(gridDim.x) * blockDim.x) {
        const int64_t slot = w / slot_words;
        const int32_t off = int32_t(w - slot * slot_words);
        uint64_t v = 0;
        if (!wide && off == key_off) {
            v = slot == capacity ? 0 : kEmptyKey;
        } else if (off >= state_off) {
            const int32_t sw = off - state_off;
            for (int s = 0; s < sp.n; ++s) {
                if (sp.s[s].word == sw) v = StateIdentity(sp.s[s].kind);
            }
        }
        slots[w] = v;
    }
}

__global__ void AggRehashKernel(const __grid_constant__ AggLaunch L, GTableDev from) {
    const AggPlan& P = L.P;
    for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i <= from.capacity;
         i += int64_t(gridDim.x) * blockDim.x) {
        const uint64_t* s = from.slots + i * from.slot_words;
        int64_t g;
        if (!from.wide) {
            const uint64_t key = s[from.key_off];
            if (i == from.capacity) {
                if (key == 0) continue;
                g = L.T.capacity;
                L.T.slots[g * L.T.slot_words + L.T.key_off] = 1;
            } else {
                if (key == kEmptyKey) continue;
                int is_new = 0;
                g = GlobalFind1(L.T, L.cap_mask, key, is_new);
            }
        } else {
            if (i == from.capacity || s[0] != 2) continue;
            int is_new = 0;
            g = GlobalFindW(L.T, L.cap_mask, s + 1, P.key_words, is_new, &L.counters->error);
        }
        if (g < 0) {
            SetError(&L.counters->error, DE_PROBE_LIMIT);
            continue;
        }
        for (int w = 0; w < P.state_words; ++w) {
            L.T.slots[g * L.T.slot_words + L.T.state_off + w] = s[from.state_off + w];
        }
    }
}

__global__ void AggMergeSpillKernel(const __grid_constant__ AggLaunch L, const uint64_t* spill, int64_t n) {
    const AggPlan& P = L.P;
    for (int64_t e = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; e < n; e += int64_t(gridDim.x) * blockDim.x) {
        const uint64_t* rec = spill + e * (1 + P.state_words);
        int is_new = 0;
        const int64_t g = GlobalFind1(L.T, L.cap_mask, rec[0], is_new);
        if (is_new) atomicAdd(&L.counters->new_groups, 1ull);
        if (g < 0) {
            SetError(&L.counters->error, DE_PROBE_LIMIT);
            continue;
        }
        uint64_t* gbase = L.T.slots + g * L.T.slot_words + L.T.state_off;
        for (int s = 0; s < P.nstates; ++s) {
            const StateDesc sd = P.states[s];
            const uint64_t lo = rec[1 + sd.word];
            const uint64_t hi = sd.kind == ST_SUM_I128 ? rec[2 + sd.word] : 0;
            if (IsIdentity(sd.kind, lo, hi)) continue;
            double f;
            __builtin_memcpy(&f, &lo, 8);
            ApplyState(gbase + sd.word, gbase + sd.word + 1, sd.kind, lo, hi, f);
        }
    }
}

// ---------------------------------------------------------------------------
// Finalize: compact the occupied slots, in slot order, into output columns.
// ---------------------------------------------------------------------------
constexpr int kFinThreads = 256;
constexpr int kFinChunk = 4096;   // slots per block

struct FinLaunch {
    AggPlan P;
    OutputPlan O;
    GTableDev T;
    AggOutputCol cols[kMaxCols + kMaxAggs];
    int32_t ncols;
    int64_t groups;
    unsigned long long* block_counts;
    int* err;
};

__device__ __forceinline__ bool SlotOccupied(const GTableDev& T, int64_t i) {
    const uint64_t* s = T.slots + i * T.slot_words;
    if (T.wide) return i < T.capacity && s[0] == 2;
    if (i == T.capacity) return s[T.key_off] != 0;
    return s[T.key_off] != kEmptyKey;
}

__global__ void __launch_bounds__(kFinThreads) FinCountKernel(const __grid_constant__ FinLaunch L) {
    __shared__ unsigned cnt;
    if (threadIdx.x == 0) cnt = 0;
    __syncthreads();
    const int64_t begin = int64_t(blockIdx.x) * kFinChunk;
    const int64_t end = Min64(begin + kFinChunk, L.T.capacity + 1);
    unsigned local = 0;
    for (int64_t i = begin + threadIdx.x; i < end; i += blockDim.x) local += SlotOccupied(L.T, i) ? 1 : 0;
    atomicAdd(&cnt, local);
    __syncthreads();
    if (threadIdx.x == 0) L.block_counts[blockIdx.x] = cnt;
}

__global__ void __launch_bounds__(1024) FinScanKernel(unsigned long long* counts, int64_t n) {
    __shared__ unsigned long long carry;
    __shared__ unsigned long long warp_sums[32];
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (int64_t base = 0; base < n; base += blockDim.x) {
        const int64_t i = base + threadIdx.x;
        const unsigned long long v = i < n ? counts[i] : 0;
        unsigned long long x = v;
        for (int d = 1; d < 32; d <<= 1) {
            const unsigned long long y = __shfl_up_sync(kFull, x, d);
            if (LaneId() >= d) x += y;
        }
        if (LaneId() == 31) warp_sums[threadIdx.x >> 5] = x;
        __syncthreads();
        if (threadIdx.x < 32) {
            unsigned long long w = warp_sums[threadIdx.x];
            for (int d = 1; d < 32; d <<= 1) {
                const unsigned long long y = __shfl_up_sync(kFull, w, d);
                if (LaneId() >= d) w += y;
            }
            warp_sums[threadIdx.x] = w;
        }
        __syncthreads();
        const unsigned long long before = (threadIdx.x >= 32 ? warp_sums[(threadIdx.x >> 5) - 1] : 0) + carry;
        if (i < n) counts[i] = before + x - v;   // exclusive
        __syncthreads();
        if (threadIdx.x == blockDim.x - 1) carry = before + x;
        __syncthreads();
    }
}

// Output row accessor for the finalize projection.
struct OutRowAcc {
    const GVal* v;
    uint64_t nulls;
    const OutputPlan* O;
    __device__ i128 Int(int c) const { return v[c].i; }
    __device__ double F64(int c) const {
        if (O->row_dom[c] == GD_F64) return v[c].f;
        return double(v[c].i) / Pow10F(O->row_scale[c]);
    }
    __device__ bool Null(int c) const { return (nulls >> c) & 1; }
};

__device__ __forceinline__ void StoreValue(const AggOutputCol& col, int64_t row, const GVal& v, bool null) {
    if (col.valid && !null) atomicOr(&col.valid[row >> 5], 1u << (row & 31));
    char* p = col.data;
    switch (col.type) {
        case QDB_TYPE_F64: reinterpret_cast<double*>(p)[row] = null ? 0.0 : v.f; break;
        case QDB_TYPE_F32: reinterpret_cast<float*>(p)[row] = null ? 0.0f : float(v.f); break;
        case QDB_TYPE_DECIMAL128:
            reinterpret_cast<uint64_t*>(p)[2 * row] = null ? 0 : uint64_t(u128(v.i));
            reinterpret_cast<uint64_t*>(p)[2 * row + 1] = null ? 0 : uint64_t(u128(v.i) >> 64);
            break;
        case QDB_TYPE_I64: case QDB_TYPE_U64: case QDB_TYPE_DECIMAL64:
            reinterpret_cast<int64_t*>(p)[row] = null ? 0 : int64_t(v.i);
            break;
        case QDB_TYPE_I32: case QDB_TYPE_U32: case QDB_TYPE_DATE32:
            reinterpret_cast<int32_t*>(p)[row] = null ? 0 : int32_t(v.i);
            break;
        case QDB_TYPE_I16: case QDB_TYPE_U16: reinterpret_cast<int16_t*>(p)[row] = null ? 0 : int16_t(v.i); break;
        default:
            reinterpret_cast<uint8_t*>(p)[row] = null ? 0 : uint8_t(v.i);
            if (col.offsets) {
                col.offsets[row + 1] = int32_t(row + 1);
                if (row == 0) col.offsets[0] = 0;
            }
            break;
    }
}

__global__ void __launch_bounds__(kFinThreads) FinWriteKernel(const __grid_constant__ FinLaunch L) {
    __shared__ unsigned warp_off[kFinThreads / 32];
    __shared__ unsigned running;
    const AggPlan& P = L.P;
    const OutputPlan& O = L.O;
    if (threadIdx.x == 0) running = 0;
    __syncthreads();
    const int64_t begin = int64_t(blockIdx.x) * kFinChunk;
    const int64_t end = Min64(begin + kFinChunk, L.T.capacity + 1);
    const unsigned long long block_off = L.block_counts[blockIdx.x];
    for (int64_t b = begin; b < end; b += blockDim.x) {
        const int64_t i = b + threadIdx.x;
        const bool occ = i < end && SlotOccupied(L.T, i);
        const unsigned m = __ballot_sync(kFull, occ);
        if (LaneId() == 0) warp_off[threadIdx.x >> 5] = __popc(m);
        __syncthreads();
        unsigned before = running;
        for (int w = 0; w < int(threadIdx.x >> 5); ++w) before += warp_off[w];
        before += __popc(m & ((1u << LaneId()) - 1));
        __syncthreads();
        if (threadIdx.x == blockDim.x - 1) {
            unsigned tot = 0;
            for (int w = 0; w < kFinThreads / 32; ++w) tot += warp_off[w];
            running += tot;
        }
        if (occ) {
            const int64_t row = int64_t(block_off) + before;
            if (row < L.groups) {
                const uint64_t* s = L.T.slots + i * L.T.slot_words;
                uint64_t kw[kMaxKeyWords];
                if (!L.T.wide && i == L.T.capacity) {
                    kw[0] = kEmptyKey;
                } else {
                    for (int w = 0; w < P.key_words; ++w) kw[w] = s[L.T.key_off + w];
                }
                GVal rowv[kMaxCols + kMaxAggs];
                uint64_t nulls = 0;
                int c = 0;
                for (int j = 0; j < P.nkeyparts; ++j, ++c) {
                    const KeyPart& k = P.keys[j];
                    rowv[c].i = 0;
                    rowv[c].f = 0.0;
                    if (UnpackKeyNull(k, kw)) {
                        nulls |= 1ull << c;
                    } else if (k.is_float) {
                        uint64_t b2 = kw[k.word];
                        double f;
                        __builtin_memcpy(&f, &b2, 8);
                        rowv[c].f = f;
                    } else {
                        rowv[c].i = UnpackKeyInt(k, kw);
                    }
                }
                const uint64_t* st = s + L.T.state_off;
                for (int j = 0; j < P.naggs; ++j, ++c) {
                    const AggOut& ao = P.aggs[j];
                    const StateDesc sd = P.states[ao.state];
                    rowv[c].i = 0;
                    rowv[c].f = 0.0;
                    if (ao.valid_state != 0xFF && st[P.states[ao.valid_state].word] == 0) {
                        nulls |= 1ull << c;
                        continue;
                    }
                    const uint64_t lo = st[sd.word];
                    switch (sd.kind) {
                        case ST_SUM_I128: rowv[c].i = i128((u128(st[sd.word + 1]) << 64) | lo); break;
                        case ST_SUM_F64: {
                            double f;
                            __builtin_memcpy(&f, &lo, 8);
                            rowv[c].f = f;
                            break;
                        }
                        case ST_MIN_F64: case ST_MAX_F64: rowv[c].f = F64FromOrdered(lo); break;
                        default: rowv[c].i = i128(int64_t(lo)); break;
                    }
                }
                if (O.identity) {
                    for (int k = 0; k < L.ncols; ++k) StoreValue(L.cols[k], row, rowv[k], (nulls >> k) & 1);
                } else {
                    GVal gv[kMaxGNodes];
                    uint64_t gn = 0;
                    OutRowAcc oa{rowv, nulls, &O};
                    if (!EvalGeneric(O.prog, O.root_max, O.list, oa, gv, gn)) SetError(L.err, DE_DIV_ZERO);
                    for (int k = 0; k < L.ncols; ++k) {
                        const int rt = O.roots[k];
                        StoreValue(L.cols[k], row, gv[rt], (gn >> rt) & 1);
                    }
                }
            }
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// Host launchers.
// ---------------------------------------------------------------------------
namespace {

int g_sms = 0;
size_t g_smem_optin = 0;

void EnsureDeviceInfo() {
    if (g_sms) return;
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&g_sms, cudaDevAttrMultiProcessorCount, dev);
    int v = 0;
    cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    g_smem_optin = size_t(v);
}

template <class K>
void SetSmem(K kernel, size_t bytes) {
    cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(bytes));
}

int64_t Align(int64_t v, int64_t a) { return (v + a - 1) / a * a; }

}  // namespace

int DeviceSMs() {
    EnsureDeviceInfo();
    return g_sms;
}

size_t MaxSmemOptin() {
    EnsureDeviceInfo();
    return g_smem_optin;
}

void AggInitTable(const AggPlan& p, const GTableDev& t, cudaStream_t s) {
    StatesParam sp;
    std::memcpy(sp.s, p.states, sizeof(sp.s));
    sp.n = p.nstates;
    const int64_t total = (t.capacity + 1) * t.slot_words;
    const int blocks = int(std::min<int64_t>((total + 255) / 256, int64_t(DeviceSMs()) * 16));
    ProfileBegin(s, "agg_init_table", t.capacity);
    AggInitKernel<<<blocks, 256, 0, s>>>(t.slots, t.capacity, t.slot_words, t.key_off, t.state_off, t.wide, sp);
    ProfileEnd(s);
    CountLaunch();
}

static void FillTableArgs(AggLaunch& L, const GTableDev& t) {
    L.T = t;
    L.cap_mask = uint64_t(t.capacity - 1);
}

void AggUpdate(const AggUpdateArgs& a, cudaStream_t s) {
    EnsureDeviceInfo();
    static thread_local AggLaunch* Lp = nullptr;
    if (!Lp) Lp = new AggLaunch();
    AggLaunch& L = *Lp;
    std::memset(&L, 0, sizeof(L));
    L.P = *a.plan;
    L.nrows = a.nrows;
    L.index = a.index;
    L.nindex = a.nindex;
    FillTableArgs(L, a.table);
    L.counters = a.counters;
    L.deferred = a.deferred;
    L.deferred_cap = a.deferred_cap;
    L.spill = a.spill;
    L.spill_cap = a.spill_cap;
    L.join = a.join;
    L.jk = a.jkey;
    L.jt = a.jt;
    const bool wide = a.table.wide != 0;

    if (a.index) {
        if (a.nindex == 0) return;
        const int blocks = int(std::min<int64_t>((a.nindex + 255) / 256, int64_t(g_sms) * 8));
        ProfileBegin(s, "agg_update_index", a.nindex);
        if (wide) AggIndexKernel<true><<<blocks, 256, 0, s>>>(L);
        else AggIndexKernel<false><<<blocks, 256, 0, s>>>(L);
        ProfileEnd(s);
        CountLaunch();
        return;
    }
    if (a.nrows == 0) return;

    // Tile geometry: bulk-stage every aligned, non-build column.
    int bytes_per_row = 0;
    bool any = false;
    for (int c = 0; c < L.P.ncols; ++c) {
        ColDesc& cd = L.P.cols[c];
        const bool aligned = (reinterpret_cast<uintptr_t>(cd.data) & 15) == 0;
        cd.stage = (!cd.build && cd.kind != LK_BOOLBIT && cd.width > 0 && aligned) ? 1 : 0;
        if (cd.stage) {
            bytes_per_row += cd.width;
            any = true;
        }
    }
    const bool sel_staged = L.P.selection && (reinterpret_cast<uintptr_t>(L.P.selection) & 15) == 0;
    if (sel_staged) {
        bytes_per_row += 1;
        any = true;
    }
    int T = 1024;
    if (bytes_per_row > 0) {
        const int target = 40 * 1024;
        T = 256;
        while (T * 2 * bytes_per_row <= target && T < 4096) T *= 2;
    }
    L.tile_rows = T;
    L.stages = 3;
    int off = 0;
    for (int c = 0; c < L.P.ncols; ++c) {
        ColDesc& cd = L.P.cols[c];
        if (!cd.stage) continue;
        cd.smem_off = off;
        off += int(Align(int64_t(T) * cd.width, 16));
    }
    L.sel_off = -1;
    if (sel_staged) {
        L.sel_off = off;
        off += int(Align(T, 16));
    }
    L.stage_bytes = off;
    L.any_staged = any ? 1 : 0;
    if (!any) L.stages = 1;
    L.off_bars = int(Align(int64_t(L.stages) * L.stage_bytes, 16));
    L.off_bases = L.off_bars + 8 * L.stages;
    L.off_bases = int(Align(L.off_bases, 16));
    L.off_misc = L.off_bases + 8 * (kMaxCols + 1);
    L.off_skeys = int(Align(L.off_misc + 16, 128));
    const size_t budget = g_smem_optin - 1024;
    const int sw = L.P.state_words;
    int S = wide ? 0 : a.smem_slots;
    while (S > 0 && size_t(L.off_skeys) + size_t(S) * (1 + sw) * 8 > budget) S >>= 1;
    if (S < 32) S = 0;
    L.smem_slots = S;
    L.smem_limit = S / 2;
    L.off_sst = L.off_skeys + S * 8;
    const size_t smem_bytes = size_t(L.off_sst) + size_t(S) * sw * 8;

    const int64_t ntiles = (a.nrows + T - 1) / T;
    const int grid = int(std::max<int64_t>(1, std::min<int64_t>(ntiles, g_sms)));
    const char* name = a.join ? "join_agg_probe" : "agg_update";
    const bool gen = L.P.generic_root >= 0;
    ProfileBegin(s, name, a.nrows);
    auto launch = [&](auto kernel) {
        SetSmem(kernel, smem_bytes);
        kernel<<<grid, kAggThreads, smem_bytes, s>>>(L);
    };
    const int variant = (wide ? 4 : 0) | (a.join ? 2 : 0) | (gen ? 1 : 0);
    switch (variant) {
        case 0: launch(AggUpdateKernel<false, false, false>); break;
        case 1: launch(AggUpdateKernel<false, false, true>); break;
        case 2: launch(AggUpdateKernel<false, true, false>); break;
        case 3: launch(AggUpdateKernel<false, true, true>); break;
        case 4: launch(AggUpdateKernel<true, false, false>); break;
        case 5: launch(AggUpdateKernel<true, false, true>); break;
        case 6: launch(AggUpdateKernel<true, true, false>); break;
        default: launch(AggUpdateKernel<true, true, true>); break;
    }
    ProfileEnd(s);
    CountLaunch();
}

void AggRehash(const AggPlan& p, const GTableDev& from, const GTableDev& to, AggCounters* c, cudaStream_t s) {
    static thread_local AggLaunch* Lp = nullptr;
    if (!Lp) Lp = new AggLaunch();
    AggLaunch& L = *Lp;
    std::memset(&L, 0, sizeof(L));
    L.P = p;
    FillTableArgs(L, to);
    L.counters = c;
    const int blocks = int(std::min<int64_t>((from.capacity + 256) / 256, int64_t(DeviceSMs()) * 16));
    ProfileBegin(s, "agg_rehash", from.capacity);
    AggRehashKernel<<<blocks, 256, 0, s>>>(L, from);
    ProfileEnd(s);
    CountLaunch();
}

void AggMergeSpill(const AggPlan& p, const uint64_t* spill, int64_t n, const GTableDev& t, AggCounters* c,
                   cudaStream_t s) {
    if (n == 0) return;
    static thread_local AggLaunch* Lp = nullptr;
    if (!Lp) Lp = new AggLaunch();
    AggLaunch& L = *Lp;
    std::memset(&L, 0, sizeof(L));
    L.P = p;
    FillTableArgs(L, t);
    L.counters = c;
    const int blocks = int(std::min<int64_t>((n + 255) / 256, int64_t(DeviceSMs()) * 16));
    ProfileBegin(s, "agg_merge_spill", n);
    AggMergeSpillKernel<<<blocks, 256, 0, s>>>(L, spill, n);
    ProfileEnd(s);
    CountLaunch();
}

void ExclusiveScanU64(unsigned long long* counts, int64_t n, cudaStream_t s) {
    if (n <= 0) return;
    FinScanKernel<<<1, 1024, 0, s>>>(counts, n);
    CountLaunch();
}

size_t AggFinalizeScratch(const GTableDev& t) {
    const int64_t blocks = (t.capacity + 1 + kFinChunk - 1) / kFinChunk;
    return size_t(blocks) * sizeof(unsigned long long);
}

void AggFinalize(const AggPlan& p, const OutputPlan& out, const GTableDev& t, AggOutputCol* cols, int ncols,
                 int64_t groups, void* scratch, int* err, cudaStream_t s) {
    static thread_local FinLaunch* Lp = nullptr;
    if (!Lp) Lp = new FinLaunch();
    FinLaunch& L = *Lp;
    std::memset(&L, 0, sizeof(L));
    L.P = p;
    L.O = out;
    L.T = t;
    for (int k = 0; k < ncols; ++k) L.cols[k] = cols[k];
    L.ncols = ncols;
    L.groups = groups;
    L.block_counts = static_cast<unsigned long long*>(scratch);
    L.err = err;
    const int64_t blocks = (t.capacity + 1 + kFinChunk - 1) / kFinChunk;
    ProfileBegin(s, "agg_finalize", t.capacity);
    FinCountKernel<<<int(blocks), kFinThreads, 0, s>>>(L);
    FinScanKernel<<<1, 1024, 0, s>>>(L.block_counts, blocks);
    FinWriteKernel<<<int(blocks), kFinThreads, 0, s>>>(L);
    ProfileEnd(s);
    CountLaunch(3);
}

}  // namespace qdb
