// agg.cu — fused filter -> project -> hash aggregate for sm_100a.
//
// One persistent CTA per SM streams row tiles of every referenced column
// into shared memory with 1-D bulk copies (cp.async.bulk completing on an
// mbarrier, three stages in flight; warps release a stage through a second
// mbarrier, so no block-wide barrier sits between tiles).  Each lane takes
// one row at a time and evaluates the predicate, the group key and every
// aggregate input from shared memory, then folds the row into
//   (1) lane-private accumulators in shared memory for the first four
//       groups the CTA meets (no atomics, no bank conflicts: word w of
//       group g of thread t lives at ((g * W + w) * blockDim + t)) — the
//       low-cardinality and keyless case,
//   (2) a per-CTA shared-memory group table updated with shared atomics,
//   (3) a global open-addressing table in HBM (one slot per group holding
//       key and state words; CAS key claim, atomic state updates) — the
//       high-cardinality case.
// At the end a CTA reduces (1) into (2) and merges (2) into (3).  A row whose
// global probe exceeds the probe bound is deferred (row id to a list) and a
// shared entry that cannot be merged is spilled; the host grows the table and
// replays both, so no row is lost or counted twice.
//
// The fused join variant probes a built join table (32-byte entries: key,
// arena row, first payload word) for several probe rows per lane at once and
// folds every joined row the same way.
//
// Semantics are the engine's reducers (qdb/kernel/gen.cpp:3301-3593): i64
// sums wrap, decimal sums are exact i128, COUNT counts non-NULL inputs, MIN /
// MAX fold non-NULL inputs, f64 sums are IEEE additions in device order.
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

#include "common.cuh"
#include "eval.h"
#include "jtable.cuh"
#include "kernels.h"
#include "lower.h"

namespace qdb {

constexpr int kAggThreads = 512;
constexpr int kPrivGroups = 4;     // groups per CTA folded into lane-private accumulators
constexpr int kProbeRows = 4;      // fused join: probe rows in flight per lane
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
    int32_t off_bars;         // full barriers, then empty barriers
    int32_t off_misc;
    int32_t off_skeys;
    int32_t off_sst;
    int32_t off_gid;
    int32_t off_pacc;
    int32_t any_staged;
    int32_t priv;
    int32_t inline_slot;      // fused join: plan slot served by the entry's payload word (-1 none)
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
    FastPlan F;               // typed row shape (FAST kernels)
    const uint64_t* seeds;    // high-cardinality kernel: keys pre-loaded into the shared tier
    const int* nseed;         // their count (device), or seeds == nullptr
};

// Launch arguments of the listed-row kernel (AggSigQuadKernel): the typed
// plan and the fields of AggLaunch it reads, under a fifth of AggLaunch's
// bytes — a launch's parameter block travels with it, and ~11 KB of it cost
// about 6 us per launch on B200 against a small block.
struct QuadLaunch {
    FastPlan F;
    const char* cols[kFastCols];   // the typed columns, at row 0
    const uint8_t* selection;
    int64_t nrows;
    GTableDev T;
    uint64_t cap_mask;
    AggCounters* counters;
    int64_t* deferred;
    int64_t deferred_cap;
    uint64_t* spill;
    int64_t spill_cap;
    StateDesc states[kMaxStates];
    int32_t nstates;
    int32_t state_words;
    int32_t nkeyparts;
    int32_t key_full64;
    int32_t smem_slots;
    int32_t smem_limit;
    int32_t off_misc;
    int32_t off_skeys;
    int32_t off_sst;
    int32_t off_gid;
    int32_t off_pacc;
    int64_t list[kMaxList];        // IN-list constants of the filter atoms
};

// ---------------------------------------------------------------------------
// Row accessor over staged tiles, global columns and gathered build rows.
// ---------------------------------------------------------------------------
struct RowAcc {
    const AggPlan* P;
    const unsigned char* stage;   // staged tile of this row, or nullptr (global columns)
    int r;                        // row inside the tile
    int64_t arow;                 // row inside the launch range
    int64_t brow;                 // matched build row (fused join)
    int inl_slot;                 // slot whose value is `inl` (fused join), -1 none
    uint64_t inl;

    __device__ __forceinline__ const char* Ptr(int c) const {
        const ColDesc& cd = P->cols[c];
        if (cd.build) return cd.data + brow * cd.width;
        if (stage && cd.stage) return reinterpret_cast<const char*>(stage + cd.smem_off) + int64_t(r) * cd.width;
        return cd.data + arow * cd.width;
    }
    __device__ __forceinline__ i128 Int(int c) const {
        if (c == inl_slot) return i128(int64_t(inl));
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
        if (c == inl_slot) {
            if (cd.kind == LK_F64) return __longlong_as_double((long long)inl);
            return cd.scale ? double(int64_t(inl)) / Pow10F(cd.scale) : double(int64_t(inl));
        }
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
        null = v.null_cols != 0 && SopNull(v, acc);
        if (!null && sd.kind != ST_COUNT) {
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

// Plain fold into a lane-private accumulator (w_hi: the high word).
__device__ __forceinline__ void PrivFold(uint64_t* w, uint64_t* w_hi, uint8_t kind, uint64_t lo, uint64_t hi,
                                         double f) {
    switch (kind) {
        case ST_COUNT:
        case ST_SUM_I64: *w += lo; break;
        case ST_SUM_I128: {
            const uint64_t o = *w;
            const uint64_t n = o + lo;
            *w = n;
            *w_hi += hi + (n < o ? 1ull : 0ull);
            break;
        }
        case ST_SUM_F64: *reinterpret_cast<double*>(w) += f; break;
        case ST_MIN_I64: if ((long long)lo < (long long)*w) *w = lo; break;
        case ST_MAX_I64: if ((long long)lo > (long long)*w) *w = lo; break;
        case ST_MIN_F64: if (lo < *w) *w = lo; break;
        case ST_MAX_F64: if (lo > *w) *w = lo; break;
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
// Shared-memory tier (one-word keys) with the lane-private group directory.
// ---------------------------------------------------------------------------
struct SmemTable {
    uint64_t* keys;       // S keys (kEmptyKey = free)
    uint64_t* st;         // state word w of slot i at st[w * S + i]
    int* gid;             // slot -> lane-private group (-2 pending, -1 none)
    int* gid_slot;        // lane-private group -> slot
    unsigned* count;      // keys inserted
    unsigned* fresh;      // global groups this CTA created
    unsigned* ngid;       // lane-private groups handed out
    uint64_t* pacc;       // lane-private accumulators
    int S;
    int limit;
    int priv;

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
                    int g = -1;
                    if (priv) {
                        const unsigned k = atomicAdd(ngid, 1u);
                        if (k < unsigned(kPrivGroups)) {
                            g = int(k);
                            gid_slot[k] = int(i);
                        }
                    }
                    *reinterpret_cast<volatile int*>(&gid[i]) = g;
                    return int(i);
                }
                if (old == key) return int(i);
            }
            i = (i + 1) & uint32_t(S - 1);
        }
        return -1;
    }
};

__device__ __forceinline__ unsigned char* DynSmem() {
    extern __shared__ __align__(128) unsigned char qdb_dyn_smem[];
    return qdb_dyn_smem;
}

// The shared-memory tier of this CTA, located by the launch's offsets.
template <class LT>
__device__ __forceinline__ SmemTable MakeSmem(const LT& L, bool wide, bool priv) {
    unsigned char* smem = DynSmem();
    unsigned* misc = reinterpret_cast<unsigned*>(smem + L.off_misc);
    SmemTable sm;
    sm.keys = reinterpret_cast<uint64_t*>(smem + L.off_skeys);
    sm.st = reinterpret_cast<uint64_t*>(smem + L.off_sst);
    sm.gid = reinterpret_cast<int*>(smem + L.off_gid);
    sm.gid_slot = reinterpret_cast<int*>(misc + 8);
    sm.count = misc;
    sm.fresh = misc + 1;
    sm.ngid = misc + 2;
    sm.pacc = reinterpret_cast<uint64_t*>(smem + L.off_pacc);
    sm.S = wide ? 0 : L.smem_slots;
    sm.limit = L.smem_limit;
    sm.priv = priv;
    return sm;
}

// ---------------------------------------------------------------------------
// Per-lane fold of one (joined) row that is selected.  Kept out of line: one
// copy serves every call site, so the kernel stays inside the instruction
// cache.
// ---------------------------------------------------------------------------
template <bool WIDE, bool GEN, bool PRIV>
__device__ __noinline__ void FoldRow(const AggLaunch& L, RowAcc acc) {
    const SmemTable sm = MakeSmem(L, WIDE, PRIV);
    const AggPlan& P = L.P;
    GVal gv[GEN ? kMaxGNodes : 1];
    uint64_t gn = 0;
    if (GEN && P.generic_root >= 0) {
        if (!EvalGeneric(P.prog, P.generic_root, P.list, acc, gv, gn)) {
            SetError(&L.counters->error, DE_DIV_ZERO);
            return;
        }
    }
    if (P.filter_kind == 1) {
        if (!AtomsPass(P, acc)) return;
    } else if (GEN && P.filter_kind == 2) {
        if (((gn >> P.filter_node) & 1) || gv[P.filter_node].i == 0) return;
    }

    int slot = -1;
    int g = -1;
    int64_t gslot = -1;
    if (!WIDE) {
        uint64_t key = 0;
        if (P.nkeyparts) key = PackKey1(P, acc, gv, gn);
        const bool special = P.key_full64 && key == kEmptyKey;
        if (sm.S > 0 && !special) {
            slot = sm.Find(key);
            if (PRIV && slot >= 0) g = *reinterpret_cast<volatile int*>(&sm.gid[slot]);
        }
        if (slot < 0) {
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
                return;
            }
        }
    } else {
        uint64_t kw[kMaxKeyWords];
        PackKey(P, acc, gv, gn, kw);
        int is_new = 0;
        gslot = GlobalFindW(L.T, L.cap_mask, kw, P.key_words, is_new, &L.counters->error);
        if (is_new) atomicAdd(sm.fresh, 1u);
        if (gslot == -1) Defer(L, acc.arow, acc.brow);
        if (gslot < 0) return;
    }

    const int bd = blockDim.x;
    uint64_t* gbase = gslot >= 0 ? L.T.slots + gslot * L.T.slot_words + L.T.state_off : nullptr;
    for (int s = 0; s < P.nstates; ++s) {
        const StateDesc sd = P.states[s];
        const Contrib c = StateInput(P, sd, acc, gv, gn);
        if (!c.has) continue;
        if (PRIV && g >= 0) {
            uint64_t* w = sm.pacc + (int64_t(g) * P.state_words + sd.word) * bd + threadIdx.x;
            PrivFold(w, w + bd, sd.kind, c.lo, c.hi, c.f);
        } else if (slot >= 0) {
            uint64_t* w = sm.st + int64_t(sd.word) * sm.S + slot;
            ApplyState(w, w + sm.S, sd.kind, c.lo, c.hi, c.f);
        } else {
            uint64_t* w = gbase + sd.word;
            ApplyState(w, w + 1, sd.kind, c.lo, c.hi, c.f);
        }
    }
}

// ---------------------------------------------------------------------------
// Typed row fold (FastPlan shape): columns loaded once as int64, 64-bit
// predicates, products in 64 or 128 bits from 64-bit factors.
// ---------------------------------------------------------------------------
__device__ __forceinline__ int64_t LoadI64(const AggPlan& P, const RowAcc& a, int slot) {
    const ColDesc& cd = P.cols[slot];
    const char* p = a.Ptr(slot);
    const bool u = cd.kind == LK_UNSIGNED;
    switch (cd.width) {
        case 1: return u ? int64_t(*reinterpret_cast<const uint8_t*>(p)) : int64_t(*reinterpret_cast<const int8_t*>(p));
        case 2: return u ? int64_t(*reinterpret_cast<const uint16_t*>(p)) : int64_t(*reinterpret_cast<const int16_t*>(p));
        case 4: return u ? int64_t(*reinterpret_cast<const uint32_t*>(p)) : int64_t(*reinterpret_cast<const int32_t*>(p));
        default: return *reinterpret_cast<const int64_t*>(p);
    }
}

__device__ __forceinline__ int64_t Sel(const int64_t (&x)[kFastCols], int k) {
    int64_t v = x[0];
#pragma unroll
    for (int j = 1; j < kFastCols; ++j) v = k == j ? x[j] : v;
    return v;
}

// (hi:lo) * b mod 2^128 with b sign-extended.
__device__ __forceinline__ void Mul128x64(uint64_t& lo, uint64_t& hi, int64_t b) {
    const uint64_t bl = uint64_t(b);
    const uint64_t nlo = lo * bl;
    const uint64_t nhi = __umul64hi(lo, bl) + hi * bl - (b < 0 ? lo : 0);
    lo = nlo;
    hi = nhi;
}

template <bool PRIV>
__device__ __noinline__ void FoldRowFast(const AggLaunch& L, RowAcc acc) {
    const SmemTable sm = MakeSmem(L, false, PRIV);
    const AggPlan& P = L.P;
    const FastPlan& F = L.F;
    int64_t x[kFastCols];
#pragma unroll
    for (int k = 0; k < kFastCols; ++k) x[k] = k < F.ncols ? LoadI64(P, acc, F.col_slot[k]) : 0;
    if (F.natoms) {
        uint32_t held = 0;
        for (int j = 0; j < F.natoms; ++j) {
            const FastAtom& t = F.atoms[j];
            const int64_t v = Sel(x, t.col);
            bool ok;
            if (t.op == AT_BETWEEN) {
                ok = v >= t.c0 && v <= t.c1;
            } else if (t.op == AT_IN) {
                ok = false;
                for (int q = 0; q < t.list_len; ++q) ok = ok || P.list[t.list_off + q] == v;
            } else {
                ok = CmpHolds(t.op, v < t.c0 ? -1 : (v > t.c0 ? 1 : 0));
            }
            if (ok) held |= 1u << t.clause;
        }
        if (held != F.clause_mask) return;
    }
    uint64_t key = 0;
    for (int j = 0; j < F.nkeys; ++j) {
        uint64_t v = uint64_t(Sel(x, F.key_col[j]));
        if (F.key_bits[j] < 64) v &= (1ull << F.key_bits[j]) - 1;
        key |= v << F.key_shift[j];
    }
    int slot = -1;
    int g = -1;
    int64_t gslot = -1;
    const bool special = P.key_full64 && key == kEmptyKey;
    if (sm.S > 0 && !special) {
        slot = sm.Find(key);
        if (PRIV && slot >= 0) g = *reinterpret_cast<volatile int*>(&sm.gid[slot]);
    }
    if (slot < 0) {
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
            return;
        }
    }
    const int bd = blockDim.x;
    uint64_t* gbase = gslot >= 0 ? L.T.slots + gslot * L.T.slot_words + L.T.state_off : nullptr;
    for (int s = 0; s < F.nstates; ++s) {
        const FastState& st = F.states[s];
        uint64_t lo = 1, hi = 0;
        double fv = 0.0;
        if (st.kind == ST_SUM_F64 || st.kind == ST_MIN_F64 || st.kind == ST_MAX_F64) {
            // A double column travels as its raw bits.
            fv = __longlong_as_double((long long)Sel(x, st.f[0].col));
            lo = st.kind == ST_SUM_F64 ? 0 : F64Ordered(fv);
        } else if (st.nf) {
            const FastFactor& f0 = st.f[0];
            const int64_t v0 = int64_t(uint64_t(f0.c) + uint64_t(f0.d) * uint64_t(Sel(x, f0.col)));
            if (!st.wide) {
                uint64_t v = uint64_t(v0);
                for (int j = 1; j < st.nf; ++j) {
                    const FastFactor& f = st.f[j];
                    v *= uint64_t(f.c) + uint64_t(f.d) * uint64_t(Sel(x, f.col));
                }
                lo = v;
                hi = int64_t(v) < 0 ? ~0ull : 0ull;   // a 64-bit value summed in 128 bits
            } else {
                lo = uint64_t(v0);
                hi = v0 < 0 ? ~0ull : 0ull;
                for (int j = 1; j < st.nf; ++j) {
                    const FastFactor& f = st.f[j];
                    Mul128x64(lo, hi, int64_t(uint64_t(f.c) + uint64_t(f.d) * uint64_t(Sel(x, f.col))));
                }
            }
        }
        const uint8_t kind = st.kind;
        if (PRIV && g >= 0) {
            uint64_t* w = sm.pacc + (int64_t(g) * P.state_words + st.word) * bd + threadIdx.x;
            PrivFold(w, w + bd, kind, lo, hi, fv);
        } else if (slot >= 0) {
            uint64_t* w = sm.st + int64_t(st.word) * sm.S + slot;
            ApplyState(w, w + sm.S, kind, lo, hi, fv);
        } else {
            uint64_t* w = gbase + st.word;
            ApplyState(w, w + 1, kind, lo, hi, fv);
        }
    }
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

// Folds every joined row of one probe row whose first bucket b (keys `k`)
// is already loaded.
template <bool WIDE, bool GEN, bool PRIV>
__device__ __forceinline__ unsigned FoldMatches(const AggLaunch& L, RowAcc acc, uint64_t key, uint64_t b,
                                                ulonglong2 k) {
    return VisitMatches(L.jt, key, b, k, [&](uint64_t slot, uint64_t bk, int j) {
        acc.brow = L.jt.rows[slot];
        if (acc.inl_slot >= 0) acc.inl = L.jt.buckets[4 * bk + 2 + j];
        FoldRow<WIDE, GEN, PRIV>(L, acc);
    });
}

template <bool WIDE, bool JOIN, bool GEN, bool PRIV, bool FAST = false>
__global__ void __launch_bounds__(kAggThreads, 1) AggUpdateKernel(const __grid_constant__ AggLaunch L) {
    unsigned char* smem = DynSmem();
    uint64_t* full = reinterpret_cast<uint64_t*>(smem + L.off_bars);
    uint64_t* empty = full + L.stages;
    unsigned* misc = reinterpret_cast<unsigned*>(smem + L.off_misc);
    const SmemTable sm = MakeSmem(L, WIDE, PRIV);
    const AggPlan& P = L.P;
    const int tid = threadIdx.x;
    const int bd = blockDim.x;
    const int nwarps = bd >> 5;
    const int64_t nspecial = (JOIN && L.jt.nspecial) ? int64_t(*L.jt.nspecial) : 0;

    if (tid == 0) {
        misc[0] = 0;
        misc[1] = 0;
        misc[2] = 0;
        misc[3] = 0;   // matched rows (fused join)
        misc[4] = 0;   // abort flag
        for (int s = 0; s < L.stages; ++s) {
            MbarInit(&full[s], 1);
            MbarInit(&empty[s], nwarps);
        }
        FenceBarrierInit();
    }
    for (int i = tid; i < sm.S; i += bd) {
        sm.keys[i] = kEmptyKey;
        sm.gid[i] = -1;
        for (int s = 0; s < P.nstates; ++s) {
            const StateDesc sd = P.states[s];
            sm.st[int64_t(sd.word) * sm.S + i] = StateIdentity(sd.kind);
            if (sd.kind == ST_SUM_I128) sm.st[int64_t(sd.word + 1) * sm.S + i] = 0;
        }
    }
    if (PRIV) {
        for (int g = 0; g < kPrivGroups; ++g) {
            for (int s = 0; s < P.nstates; ++s) {
                const StateDesc sd = P.states[s];
                sm.pacc[(int64_t(g) * P.state_words + sd.word) * bd + tid] = StateIdentity(sd.kind);
                if (sd.kind == ST_SUM_I128) sm.pacc[(int64_t(g) * P.state_words + sd.word + 1) * bd + tid] = 0;
            }
        }
    }
    __syncthreads();
    if (PRIV && P.nkeyparts == 0 && tid == 0 && sm.S > 0) {
        // A keyless aggregate has one group: key 0, lane-private group 0.
        const int i = int(uint32_t(Fmix64(0)) & uint32_t(sm.S - 1));
        sm.keys[i] = 0;
        sm.gid[i] = 0;
        sm.gid_slot[0] = i;
        misc[0] = 1;
        misc[2] = 1;
    }
    __syncthreads();

    const int T = L.tile_rows;
    const int64_t ntiles = (L.nrows + T - 1) / T;
    auto tile_full = [&](int64_t t) { return L.any_staged && (t + 1) * int64_t(T) <= L.nrows; };
    auto issue = [&](int64_t t, int s) {
        unsigned char* st = smem + int64_t(s) * L.stage_bytes;
        FenceProxyAsync();
        MbarArriveExpectTx(&full[s], uint32_t(L.stage_bytes));
        for (int c = 0; c < P.ncols; ++c) {
            const ColDesc& cd = P.cols[c];
            if (!cd.stage) continue;
            BulkG2S(st + cd.smem_off, cd.data + t * T * cd.width, uint32_t(T * cd.width), &full[s]);
        }
        if (L.sel_off >= 0) BulkG2S(st + L.sel_off, P.selection + t * T, uint32_t(T), &full[s]);
    };

    if (tid == 0) {
        for (int k = 0; k < L.stages; ++k) {
            const int64_t t = blockIdx.x + int64_t(k) * gridDim.x;
            if (t < ntiles && tile_full(t)) issue(t, k);
        }
    }

    unsigned matched = 0;
    bool aborted = false;
    for (int64_t k = 0;; ++k) {
        const int64_t t = blockIdx.x + k * gridDim.x;
        if (t >= ntiles) break;
        const int s = int(k % L.stages);
        const uint32_t phase = uint32_t((k / L.stages) & 1);
        const bool full_tile = tile_full(t);
        const int64_t row0 = t * T;
        const unsigned char* stage = full_tile ? smem + int64_t(s) * L.stage_bytes : nullptr;
        if (full_tile && !MbarWaitBounded(&full[s], phase)) {
            SetError(&L.counters->error, DE_WAIT_TIMEOUT);
            aborted = true;
        }
        if (!aborted) {
            const int nrows = int(Min64(T, L.nrows - row0));
            const uint8_t* sel = P.selection == nullptr ? nullptr
                                 : (stage && L.sel_off >= 0) ? stage + L.sel_off : P.selection + row0;
            // Row accessor: staged columns come from the stage, the others
            // (unaligned or tail tiles) from global memory.
            RowAcc acc{&P, stage, 0, 0, 0, L.inline_slot, 0};
            if (!JOIN) {
                for (int r = tid; r < nrows; r += bd) {
                    if (sel && !sel[r]) continue;
                    acc.r = r;
                    acc.arow = row0 + r;
                    if (FAST) FoldRowFast<PRIV>(L, acc);
                    else FoldRow<WIDE, GEN, PRIV>(L, acc);
                }
            } else {
                for (int rb = tid; rb < nrows; rb += bd * kProbeRows) {
                    uint64_t key[kProbeRows];
                    uint64_t slot[kProbeRows];
                    ulonglong2 e[kProbeRows];
                    bool ok[kProbeRows];
#pragma unroll
                    for (int j = 0; j < kProbeRows; ++j) {
                        const int r = rb + j * bd;
                        ok[j] = r < nrows && (!sel || sel[r]);
                        bool null = false;
                        key[j] = 0;
                        if (ok[j]) {
                            acc.r = r;
                            acc.arow = row0 + r;
                            key[j] = PackJoinKey(L.jk, acc, null);
                        }
                        ok[j] = ok[j] && !null && !(L.jk.full64 && key[j] == kEmptyKey);
                        slot[j] = Fmix64(key[j]) & L.jt.bmask;
                        e[j] = make_ulonglong2(kEmptyKey, kEmptyKey);
                        if (ok[j]) e[j] = BucketKeys(L.jt, slot[j]);
                    }
#pragma unroll 1
                    for (int j = 0; j < kProbeRows; ++j) {
                        const int r = rb + j * bd;
                        if (r >= nrows) continue;
                        acc.r = r;
                        acc.arow = row0 + r;
                        if (ok[j]) matched += FoldMatches<WIDE, GEN, PRIV>(L, acc, key[j], slot[j], e[j]);
                        // Keys equal to the empty marker live in a side list.
                        if (L.jk.full64 && nspecial > 0 && (!sel || sel[r])) {
                            bool null = false;
                            const uint64_t k2 = PackJoinKey(L.jk, acc, null);
                            if (!null && k2 == kEmptyKey) {
                                for (int64_t q = 0; q < nspecial; ++q) {
                                    acc.brow = L.jt.special_rows[2 * q];
                                    if (acc.inl_slot >= 0) acc.inl = uint64_t(L.jt.special_rows[2 * q + 1]);
                                    FoldRow<WIDE, GEN, PRIV>(L, acc);
                                    ++matched;
                                }
                            }
                        }
                    }
                }
            }
        }
        // Release the stage; the producer refills it once every warp is done
        // with it, so warps run up to `stages` tiles apart without a
        // block-wide barrier.
        __syncwarp();
        if ((tid & 31) == 0) asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(SmemAddr(&empty[s])) : "memory");
        if (aborted) *reinterpret_cast<volatile unsigned*>(&misc[4]) = 1;
        if (*reinterpret_cast<volatile unsigned*>(&misc[4])) {
            aborted = true;
            break;
        }
        if (tid == 0) {
            const int64_t nt = t + int64_t(L.stages) * gridDim.x;
            if (nt < ntiles && tile_full(nt)) {
                if (!MbarWaitBounded(&empty[s], phase)) {
                    SetError(&L.counters->error, DE_WAIT_TIMEOUT);
                    *reinterpret_cast<volatile unsigned*>(&misc[4]) = 1;
                } else {
                    issue(nt, s);
                }
            }
        }
    }
    __syncthreads();
    if (aborted || *reinterpret_cast<volatile unsigned*>(&misc[4])) {
        // Let copies already issued land before the CTA's memory goes away.
        if (tid == 0) {
            const long long start = clock64();
            while (clock64() - start < 2000000) {
            }
        }
        __syncthreads();
        return;
    }
    if (JOIN && matched) atomicAdd(&misc[3], matched);

    // Lane-private accumulators -> shared table (one warp per group state).
    __syncthreads();
    if (PRIV) {
        const int ng = int(min(*reinterpret_cast<volatile unsigned*>(sm.ngid), unsigned(kPrivGroups)));
        for (int item = tid >> 5; item < ng * P.nstates; item += nwarps) {
            const int g = item / P.nstates;
            const StateDesc sd = P.states[item % P.nstates];
            Contrib c{StateIdentity(sd.kind), 0, 0.0, true};
            for (int t2 = tid & 31; t2 < bd; t2 += 32) {
                const uint64_t* w = sm.pacc + (int64_t(g) * P.state_words + sd.word) * bd + t2;
                const uint64_t lo = w[0];
                switch (sd.kind) {
                    case ST_COUNT: case ST_SUM_I64: c.lo += lo; break;
                    case ST_SUM_I128: {
                        const uint64_t n = c.lo + lo;
                        c.hi += w[bd] + (n < c.lo ? 1ull : 0ull);
                        c.lo = n;
                        break;
                    }
                    case ST_SUM_F64: c.f += __longlong_as_double((long long)lo); break;
                    case ST_MIN_I64: if ((long long)lo < (long long)c.lo) c.lo = lo; break;
                    case ST_MAX_I64: if ((long long)lo > (long long)c.lo) c.lo = lo; break;
                    case ST_MIN_F64: if (lo < c.lo) c.lo = lo; break;
                    case ST_MAX_F64: if (lo > c.lo) c.lo = lo; break;
                }
            }
            WarpReduceState(sd.kind, true, c);
            const bool any = sd.kind == ST_SUM_F64 ? c.f != 0.0 : !IsIdentity(sd.kind, c.lo, c.hi);
            if ((tid & 31) == 0 && any) {
                uint64_t* w = sm.st + int64_t(sd.word) * sm.S + sm.gid_slot[g];
                ApplyState(w, w + sm.S, sd.kind, c.lo, c.hi, c.f);
            }
        }
        __syncthreads();
    }

    // Shared table -> global table.
    for (int i = tid; i < sm.S; i += bd) {
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
    if (tid == 0) {
        if (sm.fresh[0]) atomicAdd(&L.counters->new_groups, (unsigned long long)sm.fresh[0]);
        if (JOIN && misc[3]) atomicAdd(&L.counters->matched, (unsigned long long)misc[3]);
    }
}

// ---------------------------------------------------------------------------
// Scan aggregates specialised by a compile-time query shape (the typed row
// shape of FastPlan): column widths, filter atoms, key columns and every
// state's factor columns are template constants, so each value is one typed
// load at a fixed offset; constants (filter bounds, affine factors, key
// packing) stay runtime-uniform.  The shape machinery below serves the
// low-cardinality kernel (AggSigDirectKernel: lane-private accumulators of
// the first groups a CTA meets) and the high-cardinality kernels
// (AggHighKernel, AggHighBatchKernel: a shared tier and the global table).
// ---------------------------------------------------------------------------
enum SigKind : int {
    SK_COUNT = 0, SK_SUM64 = 1, SK_SUM128_OF64 = 2, SK_SUM128 = 3,
    SK_MIN64 = 4, SK_MAX64 = 5, SK_SUMF64 = 6, SK_MINMAXF64 = 7   // (high-cardinality kernel only)
};

template <int... V>
struct IntList {
    static constexpr int n = int(sizeof...(V));
    __host__ __device__ static constexpr int at(int s) {
        int i = 0, r = 0;
        ((r = (i++ == s ? V : r)), ...);
        return r;
    }
};

// Column code: width in bytes * 2 + 1 when unsigned.  Atom code: AtomOp * 8 +
// column.  State code: kind << 11 | factors << 9 | col0 << 6 | col1 << 3 | col2.
constexpr int ColCode(int width, bool uns) { return width * 2 + (uns ? 1 : 0); }
// Key code: fast column + 8 * bits + 1024 * shift (the key packing of the plan).
constexpr int KeyCode(int col, int bits, int shift) { return col + 8 * bits + 1024 * shift; }
constexpr int AtomCode(int op, int col) { return op * 8 + col; }
// Factor forms (bits 14-19 of a state code, two per factor): 0 x, 1 c + x,
// 2 c - x, 3 c + d * x.
enum FactorForm : int { FF_X = 0, FF_ADD = 1, FF_SUB = 2, FF_AFFINE = 3 };
constexpr int StateCode(int kind, int nf, int c0 = 0, int c1 = 0, int c2 = 0, int f0 = 0, int f1 = 0, int f2 = 0) {
    return (f2 << 18) | (f1 << 16) | (f0 << 14) | (kind << 11) | (nf << 9) | (c0 << 6) | (c1 << 3) | c2;
}

template <class COLS, class ATOMS, class KEYS, class STATES>
struct Shape {
    using Cols = COLS;
    using Atoms = ATOMS;
    using Keys = KEYS;
    using States = STATES;
    static constexpr int n = States::n;
    __host__ __device__ static constexpr int kind(int s) { return (States::at(s) >> 11) & 7; }
    __host__ __device__ static constexpr int form(int s, int j) { return (States::at(s) >> (14 + 2 * j)) & 3; }
    __host__ __device__ static constexpr int nf(int s) { return (States::at(s) >> 9) & 3; }
    __host__ __device__ static constexpr int fcol(int s, int j) { return (States::at(s) >> (6 - 3 * j)) & 7; }
    __host__ __device__ static constexpr int width(int s) {
        return (kind(s) == SK_SUM128_OF64 || kind(s) == SK_SUM128) ? 2 : 1;
    }
    __host__ __device__ static constexpr int off(int s) {
        int o = 0;
        for (int i = 0; i < s; ++i) o += width(i);
        return o;
    }
    static constexpr int words = off(n);
    // Word of the first COUNT state (every folded row adds one), or -1.
    __host__ __device__ static constexpr int count_off() {
        for (int s = 0; s < n; ++s) {
            if (kind(s) == SK_COUNT) return off(s);
        }
        return -1;
    }
    __host__ __device__ static constexpr int cw(int k) { return Cols::at(k) >> 1; }
    __host__ __device__ static constexpr bool cu(int k) { return (Cols::at(k) & 1) != 0; }
};

// 128-bit add through the carry flag (add.cc / addc): no compare and select
// for the carry.
__device__ __forceinline__ void Add128(uint64_t& lo, uint64_t& hi, uint64_t l, uint64_t h) {
    asm("add.cc.u64 %0, %0, %2;\n\taddc.u64 %1, %1, %3;" : "+l"(lo), "+l"(hi) : "l"(l), "l"(h));
}

// Fast column K of tile row r (cb: the tile's column bases).
template <class SH, int K>
__device__ __forceinline__ int64_t ColVal(const char* const* cb, int r) {
    constexpr int w = SH::cw(K);
    constexpr bool u = SH::cu(K);
    const char* p = cb[K] + int64_t(r) * w;
    if constexpr (w == 1) return u ? int64_t(*reinterpret_cast<const uint8_t*>(p)) : int64_t(*reinterpret_cast<const int8_t*>(p));
    else if constexpr (w == 2) return u ? int64_t(*reinterpret_cast<const uint16_t*>(p)) : int64_t(*reinterpret_cast<const int16_t*>(p));
    else if constexpr (w == 4) return u ? int64_t(*reinterpret_cast<const uint32_t*>(p)) : int64_t(*reinterpret_cast<const int32_t*>(p));
    else return *reinterpret_cast<const int64_t*>(p);
}

// Row accessors of the shape helpers: a row of a staged tile (or of the
// launch's global columns) read in place, or a row already in registers.
struct TileRow {
    const char* const* cb;
    int r;
    template <class SH, int K>
    __device__ __forceinline__ int64_t col() const { return ColVal<SH, K>(cb, r); }
};

template <int N>
struct RegRow {
    int64_t v[N > 0 ? N : 1];
    template <class SH, int K>
    __device__ __forceinline__ int64_t col() const { return v[K]; }
};

template <class SH, int S, int J, class A>
__device__ __forceinline__ int64_t ShapeFactor(const FastPlan& F, const A& row) {
    constexpr int FM = SH::form(S, J);
    const FastFactor& f = F.states[S].f[J];
    const int64_t x = row.template col<SH, SH::fcol(S, J)>();
    if constexpr (FM == FF_X) return x;
    else if constexpr (FM == FF_ADD) return int64_t(uint64_t(f.c) + uint64_t(x));
    else if constexpr (FM == FF_SUB) return int64_t(uint64_t(f.c) - uint64_t(x));
    else return int64_t(uint64_t(f.c) + uint64_t(f.d) * uint64_t(x));
}

__device__ __forceinline__ bool Fits32(int64_t v) { return v == int64_t(int32_t(v)); }

// Product of a state's factors: wrapping 64-bit (a, b, c), or exact 128-bit
// when WIDE.  Factors that fit in 32 bits multiply as 32 x 32 -> 64; others
// take the full 64 / 128-bit path (same result).
template <class SH, int S, bool WIDE, class A>
__device__ __forceinline__ void ShapeProduct(const FastPlan& F, const A& row, uint64_t& lo, uint64_t& hi) {
    constexpr int NF = SH::nf(S);
    const int64_t a = ShapeFactor<SH, S, 0>(F, row);
    if constexpr (NF == 1) {
        lo = uint64_t(a);
        hi = a < 0 ? ~0ull : 0ull;
        return;
    } else {
        const int64_t b = ShapeFactor<SH, S, 1>(F, row);
        int64_t c = 1;
        if constexpr (NF > 2) c = ShapeFactor<SH, S, 2>(F, row);
        if (Fits32(a) && Fits32(b) && Fits32(c)) {
            const int64_t ab = int64_t(int32_t(a)) * int32_t(b);
            if (NF == 2 || Fits32(ab)) {
                const int64_t p = NF == 2 ? ab : int64_t(int32_t(ab)) * int32_t(c);
                lo = uint64_t(p);
                hi = p < 0 ? ~0ull : 0ull;
                return;
            }
        }
        if constexpr (WIDE) {
            lo = uint64_t(a);
            hi = a < 0 ? ~0ull : 0ull;
            Mul128x64(lo, hi, b);
            if constexpr (NF > 2) Mul128x64(lo, hi, c);
        } else {
            lo = uint64_t(a) * uint64_t(b) * uint64_t(c);
            hi = int64_t(lo) < 0 ? ~0ull : 0ull;
        }
    }
}

// Folds one row into its group's lane-private accumulators: p points at
// word 0 of the group for this lane; word w lives at p[w * stride].
template <class SH, int STRIDE, int S = 0, class A>
__device__ __forceinline__ void ShapeFoldP(uint64_t* p, const FastPlan& F, const A& row) {
    constexpr int stride = STRIDE;   // compile time: every word is an immediate offset
    if constexpr (S < SH::n) {
        constexpr int K = SH::kind(S);
        constexpr int NF = SH::nf(S);
        constexpr int O = SH::off(S);
        uint64_t lo = 1, hi = 0;
        if constexpr (K != SK_COUNT) ShapeProduct<SH, S, K == SK_SUM128>(F, row, lo, hi);
        (void)NF;
        if constexpr (SH::width(S) == 2) {
            uint64_t a = p[O * stride];
            uint64_t b = p[(O + 1) * stride];
            Add128(a, b, lo, hi);
            p[O * stride] = a;
            p[(O + 1) * stride] = b;
        } else {
            p[O * stride] += lo;
        }
        ShapeFoldP<SH, STRIDE, S + 1>(p, F, row);
    }
}

// Clauses held by the row's filter atoms (AND of OR clauses).
template <class SH, int J = 0, class PL, class A>
__device__ __forceinline__ uint32_t ShapeHeld(const PL& P, const FastPlan& F, const A& row) {
    if constexpr (J < SH::Atoms::n) {
        constexpr int op = SH::Atoms::at(J) >> 3;
        constexpr int col = SH::Atoms::at(J) & 7;
        const FastAtom& t = F.atoms[J];
        const int64_t v = row.template col<SH, col>();
        bool ok;
        if constexpr (op == AT_BETWEEN) {
            ok = v >= t.c0 && v <= t.c1;
        } else if constexpr (op == AT_IN) {
            ok = false;
            for (int q = 0; q < t.list_len; ++q) ok = ok || P.list[t.list_off + q] == v;
        } else if constexpr (op == AT_EQ) {
            ok = v == t.c0;
        } else if constexpr (op == AT_NE) {
            ok = v != t.c0;
        } else if constexpr (op == AT_LT) {
            ok = v < t.c0;
        } else if constexpr (op == AT_LE) {
            ok = v <= t.c0;
        } else if constexpr (op == AT_GT) {
            ok = v > t.c0;
        } else {
            ok = v >= t.c0;
        }
        return (ok ? (1u << t.clause) : 0u) | ShapeHeld<SH, J + 1, PL>(P, F, row);
    } else {
        return 0u;
    }
}

template <class SH, int J = 0, class A>
__device__ __forceinline__ uint64_t ShapeKey(const A& row) {
    if constexpr (J < SH::Keys::n) {
        constexpr int code = SH::Keys::at(J);
        constexpr int col = code & 7;
        constexpr int bits = (code >> 3) & 127;
        constexpr int shift = code >> 10;
        uint64_t v = uint64_t(row.template col<SH, col>());
        // A zero-extended column narrower than its key field needs no mask.
        if constexpr (bits < 64 && !(SH::cu(col) && SH::cw(col) * 8 <= bits)) v &= (1ull << bits) - 1;
        return (v << shift) | ShapeKey<SH, J + 1>(row);
    } else {
        return 0ull;
    }
}

// Sum of a 64- or 128-bit accumulator over the warp.
__device__ __forceinline__ void WarpSum128(uint64_t& lo, uint64_t& hi) {
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) {
        const uint64_t ol = __shfl_xor_sync(kFull, lo, d);
        const uint64_t oh = __shfl_xor_sync(kFull, hi, d);
        Add128(lo, hi, ol, oh);
    }
}

constexpr int kSigThreads = 512;


// ---------------------------------------------------------------------------
// High-cardinality scan aggregate specialised by query shape: typed loads
// from the staged tile, the CTA's shared table for the keys it holds (the
// hot keys of a skewed stream settle there), the global HBM table for the
// rest, and each state's update a typed atomic chosen at compile time.
// ---------------------------------------------------------------------------
// One row's contribution to every state (COUNT 1, sums, min/max values,
// double bits).
template <class SH>
struct ShapeVals {
    uint64_t lo[SH::n];
    uint64_t hi[SH::n];
};

template <class SH, int S = 0, class A>
__device__ __forceinline__ void ShapeRowVals(ShapeVals<SH>& v, const FastPlan& F, const A& row) {
    if constexpr (S < SH::n) {
        constexpr int K = SH::kind(S);
        v.hi[S] = 0;
        if constexpr (K == SK_COUNT) {
            v.lo[S] = 1;
        } else if constexpr (K == SK_SUMF64) {
            v.lo[S] = uint64_t(row.template col<SH, SH::fcol(S, 0)>());
        } else if constexpr (K == SK_MIN64 || K == SK_MAX64) {
            v.lo[S] = uint64_t(ShapeFactor<SH, S, 0>(F, row));
        } else {
            ShapeProduct<SH, S, K == SK_SUM128>(F, row, v.lo[S], v.hi[S]);
        }
        ShapeRowVals<SH, S + 1>(v, F, row);
    }
}

// Folds one row's values into state words w[O * stride] with atomics.
template <class SH, int S = 0>
__device__ __forceinline__ void ShapeAtomics(uint64_t* w, int64_t stride, const ShapeVals<SH>& v) {
    if constexpr (S < SH::n) {
        constexpr int K = SH::kind(S);
        constexpr int O = SH::off(S);
        auto* u = reinterpret_cast<unsigned long long*>(w + O * stride);
        if constexpr (K == SK_SUMF64) {
            atomicAdd(reinterpret_cast<double*>(u), __longlong_as_double((long long)v.lo[S]));
        } else if constexpr (K == SK_MIN64) {
            atomicMin(reinterpret_cast<long long*>(u), (long long)v.lo[S]);
        } else if constexpr (K == SK_MAX64) {
            atomicMax(reinterpret_cast<long long*>(u), (long long)v.lo[S]);
        } else if constexpr (SH::width(S) == 2) {
            const unsigned long long old = atomicAdd(u, (unsigned long long)v.lo[S]);
            const unsigned long long carry = (old + v.lo[S] < old) ? 1ull : 0ull;
            if (v.hi[S] + carry) {
                atomicAdd(reinterpret_cast<unsigned long long*>(w + (O + 1) * stride), v.hi[S] + carry);
            }
        } else {
            atomicAdd(u, (unsigned long long)v.lo[S]);
        }
        ShapeAtomics<SH, S + 1>(w, stride, v);
    }
}

// Shared-memory adds of the high-cardinality kernel.  A 64-bit add goes as
// two native 32-bit adds: the low half's carry (read from the value the
// atomic returned) joins the high half, so the pair sums exactly mod 2^64.
__device__ __forceinline__ void SmemAdd64(uint64_t* p, uint64_t v) {
    unsigned* q = reinterpret_cast<unsigned*>(p);
    const unsigned lo = unsigned(v);
    const unsigned hi = unsigned(v >> 32);
    const unsigned old = atomicAdd(q, lo);
    const unsigned up = hi + (old + lo < old ? 1u : 0u);
    if (up) atomicAdd(q + 1, up);
}

// Folds one row's values into the shared tier's state words w[O * stride].
// MIN/MAX read the word first: once a hot group's extreme has settled, most
// rows change nothing and need no atomic.
template <class SH, int S = 0>
__device__ __forceinline__ void ShapeSmemAtomics(uint64_t* w, int stride, const ShapeVals<SH>& v) {
    if constexpr (S < SH::n) {
        constexpr int K = SH::kind(S);
        constexpr int O = SH::off(S);
        uint64_t* p = w + O * stride;
        if constexpr (K == SK_SUMF64) {
            atomicAdd(reinterpret_cast<double*>(p), __longlong_as_double((long long)v.lo[S]));
        } else if constexpr (K == SK_MIN64) {
            if (int64_t(v.lo[S]) < *reinterpret_cast<volatile int64_t*>(p)) {
                atomicMin(reinterpret_cast<long long*>(p), (long long)v.lo[S]);
            }
        } else if constexpr (K == SK_MAX64) {
            if (int64_t(v.lo[S]) > *reinterpret_cast<volatile int64_t*>(p)) {
                atomicMax(reinterpret_cast<long long*>(p), (long long)v.lo[S]);
            }
        } else if constexpr (SH::width(S) == 2) {
            auto* u = reinterpret_cast<unsigned long long*>(p);
            const unsigned long long old = atomicAdd(u, (unsigned long long)v.lo[S]);
            const unsigned long long carry = (old + v.lo[S] < old) ? 1ull : 0ull;
            if (v.hi[S] + carry) atomicAdd(reinterpret_cast<unsigned long long*>(w + (O + 1) * stride), v.hi[S] + carry);
        } else {
            SmemAdd64(p, v.lo[S]);
        }
        ShapeSmemAtomics<SH, S + 1>(w, stride, v);
    }
}

constexpr int kHighThreads = 1024;
constexpr int kHighSmemProbe = 16;   // shared-tier probes before a row goes to the global table

// Shared tier of the high-cardinality kernel: S one-word keys, the state
// words of slot i at st[w * S + i].  Its index comes from the high bits of
// the key's hash, the global table's from the low bits.
struct HighSmem {
    uint64_t* keys;
    uint64_t* st;
    unsigned* count;    // keys inserted
    unsigned* fresh;    // global groups this CTA created
    int S;
    int limit;

    __device__ __forceinline__ int Find(uint64_t h, uint64_t key) const {
        uint32_t i = uint32_t(h >> 40) & uint32_t(S - 1);
#pragma unroll 1
        for (int p = 0; p < kHighSmemProbe; ++p) {
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

__device__ __forceinline__ int64_t GlobalFindH(const GTableDev& T, uint64_t mask, uint64_t h, uint64_t key,
                                               int& is_new) {
    uint64_t i = h & mask;
#pragma unroll 1
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

// Where a range's rows land: the aggregate's global table, its replay list
// and its spill buffer.  `tag` names the aggregate in a batched launch (-1:
// the launch's only aggregate): it is the second word of a replay pair and
// the last word of a spill record.
struct HighDst {
    GTableDev T;
    uint64_t cap_mask;
    int64_t* deferred;
    int64_t deferred_cap;
    unsigned long long* ndeferred;
    uint64_t* spill;
    int64_t spill_cap;
    unsigned long long* nspill;
    int* error;
    int32_t tag;
};

__device__ __forceinline__ HighDst HighDstOf(const AggLaunch& L) {
    HighDst d;
    d.T = L.T;
    d.cap_mask = L.cap_mask;
    d.deferred = L.deferred;
    d.deferred_cap = L.deferred_cap;
    d.ndeferred = &L.counters->deferred;
    d.spill = L.spill;
    d.spill_cap = L.spill_cap;
    d.nspill = &L.counters->spilled;
    d.error = &L.counters->error;
    d.tag = -1;
    return d;
}

__device__ __forceinline__ void DeferTo(const HighDst& D, int64_t row) {
    const unsigned long long k = atomicAdd(D.ndeferred, 1ull);
    if (int64_t(k) < D.deferred_cap) {
        D.deferred[2 * k] = row;
        D.deferred[2 * k + 1] = D.tag < 0 ? 0 : D.tag;
    } else {
        SetError(D.error, DE_DEFER_FULL);
    }
}

// Shared tier layout inside dynamic shared memory: misc words, keys, then
// the state words.
struct HighLayout {
    int off_keys;
    int off_st;
    int bytes;
};

__host__ __device__ inline HighLayout HighLayoutOf(int S, int state_words) {
    HighLayout h;
    h.off_keys = 128;
    h.off_st = h.off_keys + S * 8;
    h.bytes = h.off_st + S * state_words * 8;
    return h;
}

// Loads the shape's columns of row r into registers (zeros past the end).
template <class SH, int K = 0>
__device__ __forceinline__ void LoadRow(RegRow<SH::Cols::n>& row, const char* const* cb, int r, bool in) {
    if constexpr (K < SH::Cols::n) {
        row.v[K] = in ? ColVal<SH, K>(cb, r) : 0;
        LoadRow<SH, K + 1>(row, cb, r, in);
    }
}

// The probe of `key` from its home slot, whose key word `cur` is already
// loaded (so that two rows' first probes can be in flight together).
__device__ __forceinline__ int64_t GlobalFindFrom(const GTableDev& T, uint64_t mask, uint64_t h, uint64_t key,
                                                  uint64_t cur, int& is_new) {
    uint64_t i = h & mask;
#pragma unroll 1
    for (int p = 0; p < kMaxProbe; ++p) {
        unsigned long long* kp =
            reinterpret_cast<unsigned long long*>(T.slots + int64_t(i) * T.slot_words + T.key_off);
        if (p > 0) cur = *reinterpret_cast<volatile unsigned long long*>(kp);
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

// One row's fold up to the global table: filter, key, values, the shared
// tier.  Returns true when the row still needs the global table.
template <class SH>
__device__ __forceinline__ bool HighRowTier(const AggPlan& P, const FastPlan& F, const HighDst& D,
                                            const HighSmem& sm, const RegRow<SH::Cols::n>& row, bool ok,
                                            int64_t defer_row, uint64_t& key, uint64_t& h, ShapeVals<SH>& v) {
    if (ok && SH::Atoms::n) ok = ShapeHeld<SH>(P, F, row) == F.clause_mask;
    if (!ok) return false;
    key = ShapeKey<SH>(row);
    ShapeRowVals<SH>(v, F, row);
    h = Fmix64(key);
    if (P.key_full64 && key == kEmptyKey) {
        // The one key equal to the empty marker: the table's flag slot.
        unsigned long long* flag =
            reinterpret_cast<unsigned long long*>(D.T.slots + D.T.capacity * D.T.slot_words + D.T.key_off);
        if (*reinterpret_cast<volatile unsigned long long*>(flag) == 0 && atomicExch(flag, 1ull) == 0) {
            atomicAdd(sm.fresh, 1u);
        }
        ShapeAtomics<SH>(D.T.slots + D.T.capacity * D.T.slot_words + D.T.state_off, 1, v);
        return false;
    }
    const int slot = sm.Find(h, key);
    if (slot >= 0) {
        ShapeSmemAtomics<SH>(sm.st + slot, sm.S, v);
        return false;
    }
    (void)defer_row;
    return true;
}

template <class SH>
__device__ __forceinline__ void HighRowGlobal(const HighDst& D, const HighSmem& sm, uint64_t key, uint64_t h,
                                              uint64_t first, const ShapeVals<SH>& v, int64_t defer_row) {
    int is_new = 0;
    const int64_t gslot = GlobalFindFrom(D.T, D.cap_mask, h, key, first, is_new);
    if (is_new) atomicAdd(sm.fresh, 1u);
    if (gslot < 0) {
        DeferTo(D, defer_row);    // replayed after the table grows
    } else {
        ShapeAtomics<SH>(D.T.slots + gslot * D.T.slot_words + D.T.state_off, 1, v);
    }
}

// One range of rows through the tiers.  Each warp takes two groups of 32
// consecutive rows at a time (each lane one row of each), coalesced straight
// from HBM with the next two groups already loading into registers while
// these are folded.  A lane resolves both rows against the shared tier, then
// issues the first global-table probe of each row that missed before it
// waits on either, so two dependent probe chains overlap; the warp
// reconverges before the next rows.  `defer_base` numbers the range's rows
// for the replay list.
template <class SH>
__device__ __forceinline__ void HighRows(const AggPlan& P, const FastPlan& F, const HighDst& D, const HighSmem& sm,
                                         const char* const* cb, const uint8_t* sel, int nrows, int64_t defer_base,
                                         int wid, int nw) {
    const int lane = int(threadIdx.x & 31);
    const int step = nw * 32;
    int r = wid * 32 + lane;
    RegRow<SH::Cols::n> ca, cbr;
    LoadRow<SH>(ca, cb, r, r < nrows);
    LoadRow<SH>(cbr, cb, r + step, r + step < nrows);
    bool sa = r < nrows && (!sel || sel[r]);
    bool sb = r + step < nrows && (!sel || sel[r + step]);
#pragma unroll 1
    for (; r - lane < nrows; r += 2 * step) {
        const int ra = r + 2 * step, rb = r + 3 * step;
        RegRow<SH::Cols::n> na, nb;
        LoadRow<SH>(na, cb, ra, ra < nrows);
        LoadRow<SH>(nb, cb, rb, rb < nrows);
        const bool nsa = ra < nrows && (!sel || sel[ra]);
        const bool nsb = rb < nrows && (!sel || sel[rb]);
        uint64_t ka = 0, ha = 0, kb = 0, hb = 0;
        ShapeVals<SH> va, vb;
        const bool ga = HighRowTier<SH>(P, F, D, sm, ca, sa, defer_base + r, ka, ha, va);
        const bool gb = HighRowTier<SH>(P, F, D, sm, cbr, sb, defer_base + r + step, kb, hb, vb);
        // Both rows' first probes before either is examined.
        const uint64_t fa = ga ? *reinterpret_cast<volatile unsigned long long*>(
                                     D.T.slots + int64_t(ha & D.cap_mask) * D.T.slot_words + D.T.key_off)
                               : 0;
        const uint64_t fb = gb ? *reinterpret_cast<volatile unsigned long long*>(
                                     D.T.slots + int64_t(hb & D.cap_mask) * D.T.slot_words + D.T.key_off)
                               : 0;
        if (ga) HighRowGlobal<SH>(D, sm, ka, ha, fa, va, defer_base + r);
        if (gb) HighRowGlobal<SH>(D, sm, kb, hb, fb, vb, defer_base + r + step);
        ca = na;
        cbr = nb;
        sa = nsa;
        sb = nsb;
        __syncwarp();   // the lanes' paths meet again before the next rows
    }
}

// Typed flush of the shared tier: every occupied slot's states (each
// updated by every row of its key, so none is at its identity) go to the
// global table as the shape's own atomics; with `reset` the tier is cleared
// to the shape's identities for the next range.
template <class SH, int S = 0>
__device__ __forceinline__ void ShapeReadSlot(ShapeVals<SH>& v, const HighSmem& sm, int i) {
    if constexpr (S < SH::n) {
        constexpr int O = SH::off(S);
        v.lo[S] = sm.st[int64_t(O) * sm.S + i];
        v.hi[S] = SH::width(S) == 2 ? sm.st[int64_t(O + 1) * sm.S + i] : 0;
        ShapeReadSlot<SH, S + 1>(v, sm, i);
    }
}

template <class SH, int S = 0>
__device__ __forceinline__ void ShapeClearSlot(const HighSmem& sm, int i) {
    if constexpr (S < SH::n) {
        constexpr int K = SH::kind(S);
        constexpr int O = SH::off(S);
        sm.st[int64_t(O) * sm.S + i] = K == SK_MIN64 ? uint64_t(INT64_MAX) : K == SK_MAX64 ? uint64_t(INT64_MIN) : 0;
        if constexpr (SH::width(S) == 2) sm.st[int64_t(O + 1) * sm.S + i] = 0;
        ShapeClearSlot<SH, S + 1>(sm, i);
    }
}

template <class SH>
__device__ __forceinline__ void ShapeFlush(const AggPlan& P, const HighDst& D, const HighSmem& sm, bool reset) {
    const int rec_words = 1 + P.state_words + (D.tag >= 0 ? 1 : 0);
    for (int i = threadIdx.x; i < sm.S; i += blockDim.x) {
        const uint64_t key = sm.keys[i];
        if (key == kEmptyKey) continue;
        if constexpr (SH::count_off() >= 0) {
            // A seeded slot that no row of the range reached.
            if (sm.st[int64_t(SH::count_off()) * sm.S + i] == 0) {
                if (reset) sm.keys[i] = kEmptyKey;
                continue;
            }
        }
        int is_new = 0;
        const int64_t g = GlobalFindH(D.T, D.cap_mask, Fmix64(key), key, is_new);
        if (is_new) atomicAdd(sm.fresh, 1u);
        if (g < 0) {
            const unsigned long long e = atomicAdd(D.nspill, 1ull);
            if (int64_t(e) >= D.spill_cap) {
                SetError(D.error, DE_SPILL_FULL);
            } else {
                uint64_t* rec = D.spill + int64_t(e) * rec_words;
                rec[0] = key;
                for (int w = 0; w < P.state_words; ++w) rec[1 + w] = sm.st[int64_t(w) * sm.S + i];
                if (D.tag >= 0) rec[1 + P.state_words] = uint64_t(D.tag);
            }
        } else {
            ShapeVals<SH> v;
            ShapeReadSlot<SH>(v, sm, i);
            ShapeAtomics<SH>(D.T.slots + g * D.T.slot_words + D.T.state_off, 1, v);
        }
        if (reset) {
            sm.keys[i] = kEmptyKey;
            ShapeClearSlot<SH>(sm, i);
        }
    }
}

__device__ __forceinline__ HighSmem HighSmemOf(const AggLaunch& L, const HighLayout& hl) {
    unsigned char* smem = DynSmem();
    HighSmem sm;
    sm.count = reinterpret_cast<unsigned*>(smem);
    sm.fresh = sm.count + 1;
    sm.keys = reinterpret_cast<uint64_t*>(smem + hl.off_keys);
    sm.st = reinterpret_cast<uint64_t*>(smem + hl.off_st);
    sm.S = L.smem_slots;
    sm.limit = L.smem_limit;
    return sm;
}

__device__ __forceinline__ void HighInit(const AggLaunch& L, const HighSmem& sm) {
    const AggPlan& P = L.P;
    if (threadIdx.x == 0) {
        sm.count[0] = 0;
        sm.fresh[0] = 0;
    }
    for (int i = threadIdx.x; i < sm.S; i += blockDim.x) {
        sm.keys[i] = kEmptyKey;
        for (int s = 0; s < P.nstates; ++s) {
            const StateDesc sd = P.states[s];
            sm.st[int64_t(sd.word) * sm.S + i] = StateIdentity(sd.kind);
            if (sd.kind == ST_SUM_I128) sm.st[int64_t(sd.word + 1) * sm.S + i] = 0;
        }
    }
}

template <class SH>
__device__ __forceinline__ void HighColumns(const AggLaunch& L, int64_t row0, const char* (&cb)[kFastCols]) {
#pragma unroll
    for (int c = 0; c < kFastCols; ++c) {
        cb[c] = nullptr;
        if (c < SH::Cols::n) cb[c] = L.P.cols[L.F.col_slot[c]].data + row0 * SH::cw(c);
    }
}

// High-cardinality scan aggregate specialised by query shape.  The launch's
// rows are cut into one contiguous range per CTA; the shared tier holds the
// first keys a CTA meets (the hot keys of a skewed stream settle there) and
// goes to the global table once, at the end.
template <class SH>
__global__ void __launch_bounds__(kHighThreads, 1) AggHighKernel(const __grid_constant__ AggLaunch L) {
    const HighLayout hl = HighLayoutOf(L.smem_slots, L.P.state_words);
    const HighSmem sm = HighSmemOf(L, hl);
    HighInit(L, sm);
    __syncthreads();
    if (L.seeds) {
        // The aggregate's most frequent keys take the tier first, so that the
        // rows of the distribution's head fold in shared memory instead of
        // each going to the global table before the tier fills with whatever
        // came first.  A seed that none of this CTA's rows reached has a
        // COUNT of 0 and is skipped at the flush (seeded shapes count rows).
        const int ns = min(*L.nseed, sm.limit);
        for (int i = threadIdx.x; i < ns; i += blockDim.x) {
            const uint64_t key = L.seeds[i];
            sm.Find(Fmix64(key), key);
        }
        __syncthreads();
    }
    const int64_t per = (L.nrows + gridDim.x - 1) / gridDim.x;
    const int64_t row0 = int64_t(blockIdx.x) * per;
    const int n = int(max(int64_t(0), min(per, L.nrows - row0)));
    const char* cb[kFastCols];
    HighColumns<SH>(L, row0, cb);
    const uint8_t* sel = L.P.selection ? L.P.selection + row0 : nullptr;
    const HighDst D = HighDstOf(L);
    HighRows<SH>(L.P, L.F, D, sm, cb, sel, n, row0, threadIdx.x >> 5, blockDim.x >> 5);
    __syncthreads();
    ShapeFlush<SH>(L.P, D, sm, false);
    __syncthreads();
    if (threadIdx.x == 0 && sm.fresh[0]) atomicAdd(&L.counters->new_groups, (unsigned long long)sm.fresh[0]);
}

// ---------------------------------------------------------------------------
// Batched high-cardinality aggregate: many independent aggregates of one
// program (partitions of a table, or small queries of one template) in one
// persistent launch.  Each CTA takes work items (aggregate, row range) from
// a device queue until it runs dry, folds the range through its shared tier
// into that aggregate's own global table, flushes the tier and takes the
// next item.  Items come biggest aggregate first, so the short ones fill the
// tail of the launch.
// ---------------------------------------------------------------------------
template <class SH>
__global__ void __launch_bounds__(kHighThreads, 1) AggHighBatchKernel(const __grid_constant__ AggLaunch L,
                                                                      const __grid_constant__ HighBatch B) {
    const HighLayout hl = HighLayoutOf(L.smem_slots, L.P.state_words);
    const HighSmem sm = HighSmemOf(L, hl);
    __shared__ long long item_at;
    HighInit(L, sm);
    for (;;) {
        __syncthreads();
        if (threadIdx.x == 0) item_at = (long long)atomicAdd(&B.counters->next_item, 1ull);
        __syncthreads();
        const int64_t it = item_at;
        if (it >= B.nitems) break;
        const HighItem item = B.items[it];
        const HighTask& tk = B.tasks[item.task];
        HighDst D;
        D.T = tk.T;
        D.cap_mask = uint64_t(tk.T.capacity - 1);
        D.deferred = B.deferred;
        D.deferred_cap = B.deferred_cap;
        D.ndeferred = &B.counters->ndeferred;
        D.spill = B.spill;
        D.spill_cap = B.spill_cap;
        D.nspill = &B.counters->nspill;
        D.error = &B.counters->error;
        D.tag = item.task;
        const char* cb[kFastCols];
#pragma unroll
        for (int c = 0; c < kFastCols; ++c) {
            cb[c] = nullptr;
            if (c < SH::Cols::n) cb[c] = tk.cols[c] + item.row0 * SH::cw(c);
        }
        const uint8_t* sel = tk.sel ? tk.sel + item.row0 : nullptr;
        HighRows<SH>(L.P, L.F, D, sm, cb, sel, item.nrows, item.row0, threadIdx.x >> 5, blockDim.x >> 5);
        __syncthreads();
        ShapeFlush<SH>(L.P, D, sm, true);
        __syncthreads();
        if (threadIdx.x == 0) {
            if (sm.fresh[0]) atomicAdd(&B.new_groups[item.task], (unsigned long long)sm.fresh[0]);
            sm.fresh[0] = 0;
            sm.count[0] = 0;
        }
    }
}

// Replay of a batched launch's deferred rows, one thread per (row, task)
// pair, into tables grown since: the same typed fold, global table only.
template <class SH>
__global__ void __launch_bounds__(256) AggBatchReplayKernel(const __grid_constant__ AggLaunch L,
                                                            const __grid_constant__ HighBatch B,
                                                            const int64_t* pairs, int64_t n) {
    const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int64_t row = pairs[2 * i];
    const int task = int(pairs[2 * i + 1]);
    const HighTask& tk = B.tasks[task];
    const char* cb[kFastCols];
#pragma unroll
    for (int c = 0; c < kFastCols; ++c) cb[c] = c < SH::Cols::n ? tk.cols[c] : nullptr;
    const TileRow row_acc{cb, int(row)};
    if (SH::Atoms::n && ShapeHeld<SH>(L.P, L.F, row_acc) != L.F.clause_mask) return;
    const uint64_t key = ShapeKey<SH>(row_acc);
    ShapeVals<SH> v;
    ShapeRowVals<SH>(v, L.F, row_acc);
    int64_t gslot;
    int is_new = 0;
    if (L.P.key_full64 && key == kEmptyKey) {
        gslot = tk.T.capacity;
        unsigned long long* flag =
            reinterpret_cast<unsigned long long*>(tk.T.slots + tk.T.capacity * tk.T.slot_words + tk.T.key_off);
        if (*reinterpret_cast<volatile unsigned long long*>(flag) == 0 && atomicExch(flag, 1ull) == 0) is_new = 1;
    } else {
        gslot = GlobalFindH(tk.T, uint64_t(tk.T.capacity - 1), Fmix64(key), key, is_new);
    }
    if (is_new) atomicAdd(&B.new_groups[task], 1ull);
    if (gslot < 0) {
        HighDst D;
        D.deferred = B.deferred;
        D.deferred_cap = B.deferred_cap;
        D.ndeferred = &B.counters->ndeferred;
        D.error = &B.counters->error;
        D.tag = task;
        DeferTo(D, row);
        return;
    }
    ShapeAtomics<SH>(tk.T.slots + gslot * tk.T.slot_words + tk.T.state_off, 1, v);
}

// Spill records [key, states..., task] of a batched launch into the grown
// tables.
__global__ void __launch_bounds__(256) AggBatchSpillKernel(const __grid_constant__ AggLaunch L,
                                                           const __grid_constant__ HighBatch B,
                                                           const uint64_t* recs, int64_t n) {
    const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const AggPlan& P = L.P;
    const uint64_t* rec = recs + i * (2 + P.state_words);
    const int task = int(rec[1 + P.state_words]);
    const HighTask& tk = B.tasks[task];
    const uint64_t key = rec[0];
    int is_new = 0;
    const int64_t g = GlobalFindH(tk.T, uint64_t(tk.T.capacity - 1), Fmix64(key), key, is_new);
    if (is_new) atomicAdd(&B.new_groups[task], 1ull);
    if (g < 0) {
        SetError(&B.counters->error, DE_SPILL_FULL);
        return;
    }
    uint64_t* gbase = tk.T.slots + g * tk.T.slot_words + tk.T.state_off;
    for (int st2 = 0; st2 < P.nstates; ++st2) {
        const StateDesc sd = P.states[st2];
        const uint64_t lo = rec[1 + sd.word];
        const uint64_t hi = sd.kind == ST_SUM_I128 ? rec[2 + sd.word] : 0;
        if (IsIdentity(sd.kind, lo, hi)) continue;
        double f;
        __builtin_memcpy(&f, &lo, 8);
        ApplyState(gbase + sd.word, gbase + sd.word + 1, sd.kind, lo, hi, f);
    }
}

// ---------------------------------------------------------------------------
// Low-cardinality scan aggregate read straight from HBM: the signature
// kernel's folds (lane-private accumulators of the first kPrivGroups groups,
// the shared table, the general typed fold past them) over one contiguous
// row range per CTA, each warp taking 32 consecutive rows at a time with the
// next 32 already loading into registers; no staging, no block barrier
// until the merge.
// ---------------------------------------------------------------------------
template <class SIG>
__global__ void __launch_bounds__(kSigThreads, 1) AggSigDirectKernel(const __grid_constant__ AggLaunch L) {
    unsigned char* smem = DynSmem();
    unsigned* misc = reinterpret_cast<unsigned*>(smem + L.off_misc);
    const SmemTable sm = MakeSmem(L, false, true);
    const AggPlan& P = L.P;
    const FastPlan& F = L.F;
    const int tid = threadIdx.x;
    const int bd = blockDim.x;
    const int lane = tid & 31;

    if (tid == 0) {
        misc[0] = 0;
        misc[1] = 0;
        misc[2] = 0;
        misc[4] = 0;
    }
    for (int i = tid; i < sm.S; i += bd) {
        sm.keys[i] = kEmptyKey;
        sm.gid[i] = -1;
        for (int s = 0; s < P.nstates; ++s) {
            const StateDesc sd = P.states[s];
            sm.st[int64_t(sd.word) * sm.S + i] = StateIdentity(sd.kind);
            if (sd.kind == ST_SUM_I128) sm.st[int64_t(sd.word + 1) * sm.S + i] = 0;
        }
    }
    uint64_t* pacc = reinterpret_cast<uint64_t*>(smem + L.off_pacc);
    for (int i = tid; i < kPrivGroups * SIG::words * bd; i += bd) pacc[i] = 0;
    __syncthreads();
    if (P.nkeyparts == 0 && tid == 0 && sm.S > 0) {
        const int i = int(uint32_t(Fmix64(0)) & uint32_t(sm.S - 1));
        sm.keys[i] = 0;
        sm.gid[i] = 0;
        sm.gid_slot[0] = i;
        misc[0] = 1;
        misc[2] = 1;
    }
    __syncthreads();

    uint64_t ckey[kPrivGroups];
    int cgid[kPrivGroups];
#pragma unroll
    for (int j = 0; j < kPrivGroups; ++j) {
        ckey[j] = kEmptyKey;
        cgid[j] = -1;
    }
    int ncache = 0;
    if (P.nkeyparts == 0) {
        ckey[0] = 0;
        cgid[0] = 0;
        ncache = 1;
    }

    const int64_t per = (L.nrows + gridDim.x - 1) / gridDim.x;
    const int64_t row0 = int64_t(blockIdx.x) * per;
    const int n = int(max(int64_t(0), min(per, L.nrows - row0)));
    const char* cb[kFastCols];
#pragma unroll
    for (int c = 0; c < kFastCols; ++c) {
        cb[c] = nullptr;
        if (c < SIG::Cols::n) cb[c] = P.cols[F.col_slot[c]].data + row0 * SIG::cw(c);
    }
    const uint8_t* sel = P.selection ? P.selection + row0 : nullptr;
    const int step = (bd >> 5) * 32;
    int r = (tid >> 5) * 32 + lane;
    RegRow<SIG::Cols::n> cur;
    LoadRow<SIG>(cur, cb, r, r < n);
    bool cur_sel = r < n && (!sel || sel[r]);
#pragma unroll 1
    for (; r - lane < n; r += step) {
        const int rn = r + step;
        RegRow<SIG::Cols::n> nxt;
        LoadRow<SIG>(nxt, cb, rn, rn < n);
        const bool nxt_sel = rn < n && (!sel || sel[rn]);
        bool ok = cur_sel;
        if (ok && SIG::Atoms::n) ok = ShapeHeld<SIG>(P, F, cur) == F.clause_mask;
        if (ok) {
            const uint64_t key = ShapeKey<SIG>(cur);
            int g = -1;
#pragma unroll
            for (int j = 0; j < kPrivGroups; ++j) g = ckey[j] == key ? cgid[j] : g;
            if (g < 0 && !(P.key_full64 && key == kEmptyKey)) {
                // First row of this group for this thread: the shared table.
                const int slot = sm.Find(key);
                if (slot >= 0) {
                    const int gg = *reinterpret_cast<volatile int*>(&sm.gid[slot]);
                    if (gg >= 0 && gg < kPrivGroups && ncache < kPrivGroups) {
                        g = gg;
#pragma unroll
                        for (int j = 0; j < kPrivGroups; ++j) {
                            if (j == ncache) {
                                ckey[j] = key;
                                cgid[j] = gg;
                            }
                        }
                        ++ncache;
                    }
                }
            }
            if (g >= 0) {
                ShapeFoldP<SIG, kSigThreads>(pacc + g * SIG::words * kSigThreads + tid, F, cur);
            } else {
                RowAcc acc{&P, nullptr, r, row0 + r, 0, -1, 0};
                FoldRowFast<false>(L, acc);
            }
        }
        cur = nxt;
        cur_sel = nxt_sel;
        __syncwarp();
    }
    __syncthreads();

    // Lane-private accumulators -> shared table: one warp per (group,
    // state) sums the lanes, then one shared-memory update.
    const int ng = int(min(*reinterpret_cast<volatile unsigned*>(sm.ngid), unsigned(kPrivGroups)));
    const int nwarps = bd >> 5;
    for (int item = tid >> 5; item < ng * SIG::n; item += nwarps) {
        const int q = item / SIG::n;
        const int st2 = item - q * SIG::n;
        const int o = SIG::off(st2);
        const bool wide2 = SIG::width(st2) == 2;
        uint64_t lo = 0, hi = 0;
        for (int t2 = lane; t2 < bd; t2 += 32) {
            const uint64_t* w = pacc + int64_t(q * SIG::words + o) * bd + t2;
            Add128(lo, hi, w[0], wide2 ? w[bd] : 0ull);
        }
        WarpSum128(lo, hi);
        if (lane == 0 && (lo | hi)) {
            const int slot = *reinterpret_cast<volatile int*>(&sm.gid_slot[q]);
            const StateDesc sd = P.states[st2];
            uint64_t* w = sm.st + int64_t(sd.word) * sm.S + slot;
            ApplyState(w, w + sm.S, sd.kind, lo, hi, 0.0);
        }
    }
    __syncthreads();

    // Shared table -> global table.
    for (int i = tid; i < sm.S; i += bd) {
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
        for (int st2 = 0; st2 < P.nstates; ++st2) {
            const StateDesc sd = P.states[st2];
            const uint64_t lo = sm.st[int64_t(sd.word) * sm.S + i];
            const uint64_t hi = sd.kind == ST_SUM_I128 ? sm.st[int64_t(sd.word + 1) * sm.S + i] : 0;
            if (IsIdentity(sd.kind, lo, hi)) continue;
            ApplyState(gbase + sd.word, gbase + sd.word + 1, sd.kind, lo, hi, 0.0);
        }
    }
    __syncthreads();
    if (tid == 0 && sm.fresh[0]) atomicAdd(&L.counters->new_groups, (unsigned long long)sm.fresh[0]);
}

// ---------------------------------------------------------------------------
// Low-cardinality scan aggregate, four rows per thread: each lane of a warp
// takes four consecutive rows of a 128-row warp tile, loading every column
// of the four with one or two vector loads (8-byte columns 2 x 16 B, 4-byte
// 16 B, 2-byte 8 B, 1-byte 4 B; all coalesced across the warp), so loads and
// their address arithmetic are a quarter of the one-row walk's and four rows'
// loads are in flight per lane.  Rows fold into the same lane-private
// accumulators (the first kPrivGroups groups) as AggSigDirectKernel; two CTAs
// of 256 threads share an SM.  Columns must start on a boundary of four
// values (16 B at most), checked by the host.
// ---------------------------------------------------------------------------
constexpr int kQuadThreads = 256;
constexpr int kQuadRows = 4;

// Column K of the four rows starting at row r4 (nvalid of them inside the
// range; zeros past it).
template <class SH, int K>
__device__ __forceinline__ void LoadQuadCol(int64_t (&out)[kQuadRows], const char* base, int64_t r4, int nvalid) {
    constexpr int w = SH::cw(K);
    constexpr bool u = SH::cu(K);
    const char* p = base + r4 * w;
    if (nvalid == kQuadRows) {
        if constexpr (w == 8) {
            const longlong2 a = __ldcs(reinterpret_cast<const longlong2*>(p));
            const longlong2 b = __ldcs(reinterpret_cast<const longlong2*>(p) + 1);
            out[0] = a.x;
            out[1] = a.y;
            out[2] = b.x;
            out[3] = b.y;
        } else if constexpr (w == 4) {
            const int4 a = __ldcs(reinterpret_cast<const int4*>(p));
            const int32_t v[4] = {a.x, a.y, a.z, a.w};
#pragma unroll
            for (int j = 0; j < 4; ++j) out[j] = u ? int64_t(uint32_t(v[j])) : int64_t(v[j]);
        } else if constexpr (w == 2) {
            const uint2 a = __ldcs(reinterpret_cast<const uint2*>(p));
            const uint32_t v[4] = {a.x & 0xffffu, a.x >> 16, a.y & 0xffffu, a.y >> 16};
#pragma unroll
            for (int j = 0; j < 4; ++j) out[j] = u ? int64_t(v[j]) : int64_t(int16_t(uint16_t(v[j])));
        } else {
            const uint32_t a = __ldcs(reinterpret_cast<const unsigned int*>(p));
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const uint32_t b = (a >> (8 * j)) & 0xffu;
                out[j] = u ? int64_t(b) : int64_t(int8_t(uint8_t(b)));
            }
        }
    } else {
#pragma unroll
        for (int j = 0; j < kQuadRows; ++j) {
            const char* pj = p + j * w;
            int64_t v = 0;
            if (j < nvalid) {
                if constexpr (w == 8) v = *reinterpret_cast<const int64_t*>(pj);
                else if constexpr (w == 4) v = u ? int64_t(*reinterpret_cast<const uint32_t*>(pj))
                                                 : int64_t(*reinterpret_cast<const int32_t*>(pj));
                else if constexpr (w == 2) v = u ? int64_t(*reinterpret_cast<const uint16_t*>(pj))
                                                 : int64_t(*reinterpret_cast<const int16_t*>(pj));
                else v = u ? int64_t(*reinterpret_cast<const uint8_t*>(pj)) : int64_t(*reinterpret_cast<const int8_t*>(pj));
            }
            out[j] = v;
        }
    }
}

template <class SH, int K = 0>
__device__ __forceinline__ void LoadQuad(int64_t (&q)[SH::Cols::n > 0 ? SH::Cols::n : 1][kQuadRows],
                                         const char* const* cb, int64_t r4, int nvalid) {
    if constexpr (K < SH::Cols::n) {
        LoadQuadCol<SH, K>(q[K], cb[K], r4, nvalid);
        LoadQuad<SH, K + 1>(q, cb, r4, nvalid);
    }
}

template <class SH, int K = 0>
__device__ __forceinline__ void QuadRow(RegRow<SH::Cols::n>& row,
                                        const int64_t (&q)[SH::Cols::n > 0 ? SH::Cols::n : 1][kQuadRows], int j) {
    if constexpr (K < SH::Cols::n) {
        row.v[K] = q[K][j];
        QuadRow<SH, K + 1>(row, q, j);
    }
}

// L2 prefetch of 128-row tile `t` of a range of n rows: the tile's w lines
// of a w-byte column (and its selection bytes), one line per lane.  Rows
// past the range are not touched.
constexpr int kQuadChunkTiles = 4;   // tiles a warp takes from the queue at a time

template <class SH, int K = 0>
__device__ __forceinline__ void QuadPrefetchTile(const char* const* cb, const uint8_t* sel, int64_t t, int64_t n,
                                                 int lane) {
    constexpr int kTileRows = 32 * kQuadRows;
    if constexpr (K < SH::Cols::n) {
        constexpr int w = SH::cw(K);
        const int64_t r = t * kTileRows + int64_t(lane) * (128 / w);
        if (lane < w && r < n) asm volatile("prefetch.global.L2 [%0];" ::"l"(cb[K] + r * w));
        QuadPrefetchTile<SH, K + 1>(cb, sel, t, n, lane);
    } else {
        const int64_t r = t * kTileRows;
        if (sel && lane == 0 && r < n) asm volatile("prefetch.global.L2 [%0];" ::"l"(sel + r));
    }
}

// A row of the listed-row kernel that neither the lanes' groups nor the
// shared tier took (the tier is full, or the key is the empty marker): the
// table itself — its flag slot for the marker — or the replay list when the
// table is full.
template <class SIG>
__device__ __forceinline__ void QuadGlobalRow(const QuadLaunch& L, const SmemTable& sm, uint64_t key, bool special,
                                              const ShapeVals<SIG>& v, int64_t row) {
    uint64_t* flag_slot = L.T.slots + L.T.capacity * L.T.slot_words;
    if (special) {
        auto* flag = reinterpret_cast<unsigned long long*>(flag_slot + L.T.key_off);
        if (*reinterpret_cast<volatile unsigned long long*>(flag) == 0 && atomicExch(flag, 1ull) == 0)
            atomicAdd(sm.fresh, 1u);
        ShapeAtomics<SIG>(flag_slot + L.T.state_off, 1, v);
        return;
    }
    int is_new = 0;
    const int64_t g = GlobalFindH(L.T, L.cap_mask, Fmix64(key), key, is_new);
    if (is_new) atomicAdd(sm.fresh, 1u);
    if (g >= 0) {
        ShapeAtomics<SIG>(L.T.slots + g * L.T.slot_words + L.T.state_off, 1, v);
        return;
    }
    const unsigned long long k = atomicAdd(&L.counters->deferred, 1ull);
    if (int64_t(k) < L.deferred_cap) {
        L.deferred[2 * k] = row;
        L.deferred[2 * k + 1] = 0;
    } else {
        SetError(&L.counters->error, DE_DEFER_FULL);
    }
}

template <class SIG>
__global__ void __launch_bounds__(kQuadThreads, 2) AggSigQuadKernel(const __grid_constant__ QuadLaunch L) {
    unsigned char* smem = DynSmem();
    unsigned* misc = reinterpret_cast<unsigned*>(smem + L.off_misc);
    const SmemTable sm = MakeSmem(L, false, true);
    const QuadLaunch& P = L;
    const FastPlan& F = L.F;
    const int tid = threadIdx.x;
    const int lane = tid & 31;
    constexpr int bd = kQuadThreads;

    if (tid == 0) {
        misc[0] = 0;
        misc[1] = 0;
        misc[2] = 0;
        misc[4] = 0;
    }
    for (int i = tid; i < sm.S; i += bd) {
        sm.keys[i] = kEmptyKey;
        sm.gid[i] = -1;
        for (int s = 0; s < P.nstates; ++s) {
            const StateDesc sd = P.states[s];
            sm.st[int64_t(sd.word) * sm.S + i] = StateIdentity(sd.kind);
            if (sd.kind == ST_SUM_I128) sm.st[int64_t(sd.word + 1) * sm.S + i] = 0;
        }
    }
    uint64_t* pacc = reinterpret_cast<uint64_t*>(smem + L.off_pacc);
    for (int i = tid; i < kPrivGroups * SIG::words * bd; i += bd) pacc[i] = 0;
    __syncthreads();
    if (P.nkeyparts == 0 && tid == 0 && sm.S > 0) {
        const int i = int(uint32_t(Fmix64(0)) & uint32_t(sm.S - 1));
        sm.keys[i] = 0;
        sm.gid[i] = 0;
        sm.gid_slot[0] = i;
        misc[0] = 1;
        misc[2] = 1;
    }
    __syncthreads();

    uint64_t ckey[kPrivGroups];
    int cgid[kPrivGroups];
#pragma unroll
    for (int j = 0; j < kPrivGroups; ++j) {
        ckey[j] = kEmptyKey;
        cgid[j] = -1;
    }
    int ncache = 0;
    if (P.nkeyparts == 0) {
        ckey[0] = 0;
        cgid[0] = 0;
        ncache = 1;
    }

    // Every warp of the grid takes chunks of kQuadChunkTiles 128-row tiles
    // from one queue, so that no SM idles at the end while another still has
    // rows (a static split left the slowest SMs 20% behind the median).
    constexpr int kWarpRows = 32 * kQuadRows;
    constexpr int64_t row0 = 0;
    const int64_t n = L.nrows;
    const char* cb[kFastCols];
#pragma unroll
    for (int c = 0; c < kFastCols; ++c) {
        cb[c] = nullptr;
        if (c < SIG::Cols::n) cb[c] = L.cols[c] + row0 * SIG::cw(c);
    }
    const uint8_t* sel = P.selection ? P.selection + row0 : nullptr;
    constexpr int NC = SIG::Cols::n > 0 ? SIG::Cols::n : 1;
    // Each warp asks the L2 for the chunk one round of the grid's warps ahead
    // of the one it takes (every chunk is asked for once), so that the
    // chunk's loads meet it in L2 rather than in HBM.
    const int64_t nchunks = (n + kQuadChunkTiles * kWarpRows - 1) / (kQuadChunkTiles * kWarpRows);
    const int64_t ahead = int64_t(gridDim.x) * (bd >> 5);
#pragma unroll 1
    for (;;) {
        unsigned c = 0;
        if (lane == 0) c = atomicAdd(&L.counters->next_chunk, 1u);
        c = __shfl_sync(0xffffffffu, c, 0);
        if (int64_t(c) >= nchunks) break;
#pragma unroll 1
        for (int k = 0; k < kQuadChunkTiles; ++k)
            QuadPrefetchTile<SIG>(cb, sel, (int64_t(c) + ahead) * kQuadChunkTiles + k, n, lane);
#pragma unroll 1
        for (int k = 0; k < kQuadChunkTiles; ++k) {
            const int64_t r4 = (int64_t(c) * kQuadChunkTiles + k) * kWarpRows + lane * kQuadRows;
            if (r4 >= n) break;
            const int nvalid = int(min(int64_t(kQuadRows), n - r4));
            int64_t q[NC][kQuadRows];
            LoadQuad<SIG>(q, cb, r4, nvalid);
            uint32_t selq = nvalid == kQuadRows ? 0x01010101u : 0u;
            if (nvalid < kQuadRows) {
                for (int j = 0; j < nvalid; ++j) selq |= 1u << (8 * j);
            }
            if (sel) {
                if (nvalid == kQuadRows) {
                    selq = __ldcs(reinterpret_cast<const unsigned int*>(sel + r4));
                } else {
                    uint32_t m = 0;
                    for (int j = 0; j < nvalid; ++j) m |= uint32_t(sel[r4 + j]) << (8 * j);
                    selq = m;
                }
            }
#pragma unroll
            for (int j = 0; j < kQuadRows; ++j) {
                if (((selq >> (8 * j)) & 0xffu) == 0) continue;
                RegRow<SIG::Cols::n> cur;
                QuadRow<SIG>(cur, q, j);
                if (SIG::Atoms::n && ShapeHeld<SIG>(P, F, cur) != F.clause_mask) continue;
                const uint64_t key = ShapeKey<SIG>(cur);
                int g = -1;
#pragma unroll
                for (int k = 0; k < kPrivGroups; ++k) g = ckey[k] == key ? cgid[k] : g;
                const bool special = P.key_full64 && key == kEmptyKey;
                int slot = -1;
                if (g < 0 && !special) {
                    slot = sm.Find(key);
                    if (slot >= 0) {
                        const int gg = *reinterpret_cast<volatile int*>(&sm.gid[slot]);
                        if (gg >= 0 && gg < kPrivGroups && ncache < kPrivGroups) {
                            g = gg;
#pragma unroll
                            for (int k = 0; k < kPrivGroups; ++k) {
                                if (k == ncache) {
                                    ckey[k] = key;
                                    cgid[k] = gg;
                                }
                            }
                            ++ncache;
                        }
                    }
                }
                if (g >= 0) {
                    ShapeFoldP<SIG, kQuadThreads>(pacc + g * SIG::words * kQuadThreads + tid, F, cur);
                } else {
                    ShapeVals<SIG> v;
                    ShapeRowVals<SIG>(v, F, cur);
                    if (slot >= 0) {
                        ShapeSmemAtomics<SIG>(sm.st + slot, sm.S, v);   // a group past the lanes' four
                    } else {
                        QuadGlobalRow<SIG>(L, sm, key, special, v, row0 + r4 + j);
                    }
                }
            }
        }
    }
    __syncthreads();

    // Lane-private accumulators -> shared table -> global table, as in
    // AggSigDirectKernel.
    const int ng = int(min(*reinterpret_cast<volatile unsigned*>(sm.ngid), unsigned(kPrivGroups)));
    constexpr int nwarps = bd >> 5;
    for (int item = tid >> 5; item < ng * SIG::n; item += nwarps) {
        const int qg = item / SIG::n;
        const int st2 = item - qg * SIG::n;
        const int o = SIG::off(st2);
        const bool wide2 = SIG::width(st2) == 2;
        uint64_t lo = 0, hi = 0;
        for (int t2 = lane; t2 < bd; t2 += 32) {
            const uint64_t* w = pacc + int64_t(qg * SIG::words + o) * bd + t2;
            Add128(lo, hi, w[0], wide2 ? w[bd] : 0ull);
        }
        WarpSum128(lo, hi);
        if (lane == 0 && (lo | hi)) {
            const int slot = *reinterpret_cast<volatile int*>(&sm.gid_slot[qg]);
            const StateDesc sd = P.states[st2];
            uint64_t* w = sm.st + int64_t(sd.word) * sm.S + slot;
            ApplyState(w, w + sm.S, sd.kind, lo, hi, 0.0);
        }
    }
    __syncthreads();
    for (int i = tid; i < sm.S; i += bd) {
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
        for (int st2 = 0; st2 < P.nstates; ++st2) {
            const StateDesc sd = P.states[st2];
            const uint64_t lo = sm.st[int64_t(sd.word) * sm.S + i];
            const uint64_t hi = sd.kind == ST_SUM_I128 ? sm.st[int64_t(sd.word + 1) * sm.S + i] : 0;
            if (IsIdentity(sd.kind, lo, hi)) continue;
            ApplyState(gbase + sd.word, gbase + sd.word + 1, sd.kind, lo, hi, 0.0);
        }
    }
    __syncthreads();
    if (tid == 0 && sm.fresh[0]) atomicAdd(&L.counters->new_groups, (unsigned long long)sm.fresh[0]);
}

// ---------------------------------------------------------------------------
// Many low-cardinality aggregates of one program in one persistent launch
// (batched aggregation of the QDB_SHAPE_LIST shapes): a CTA pulls work items
// (aggregate, row range) from the queue; for each it walks the rows four per
// lane as AggSigQuadKernel does, folding the item's first kPrivGroups groups
// into lane-private accumulators and any others into the shared tier, then
// merges both into that aggregate's table — spilling tagged entries when the
// table is full, for the replay into a grown table — and clears them for the
// next item.  A row whose group finds no room in the tier goes to the table
// at once; one that the full table turns away is deferred for the replay.
// ---------------------------------------------------------------------------
template <class SIG>
__global__ void __launch_bounds__(kQuadThreads, 2) AggSigQuadBatchKernel(const __grid_constant__ AggLaunch L,
                                                                         const __grid_constant__ HighBatch B) {
    unsigned char* smem = DynSmem();
    unsigned* misc = reinterpret_cast<unsigned*>(smem + L.off_misc);
    const SmemTable sm = MakeSmem(L, false, true);
    const AggPlan& P = L.P;
    const FastPlan& F = L.F;
    const int tid = threadIdx.x;
    const int lane = tid & 31;
    constexpr int bd = kQuadThreads;
    constexpr int kWarpRows = 32 * kQuadRows;
    constexpr int NC = SIG::Cols::n > 0 ? SIG::Cols::n : 1;
    uint64_t* pacc = reinterpret_cast<uint64_t*>(smem + L.off_pacc);
    __shared__ long long item_at;
    for (;;) {
        // Clear the tiers for the next item.
        if (tid == 0) {
            misc[0] = 0;
            misc[1] = 0;
            misc[2] = 0;
            misc[4] = 0;
            item_at = (long long)atomicAdd(&B.counters->next_item, 1ull);
        }
        for (int i = tid; i < sm.S; i += bd) {
            sm.keys[i] = kEmptyKey;
            sm.gid[i] = -1;
            for (int st = 0; st < P.nstates; ++st) {
                const StateDesc sd = P.states[st];
                sm.st[int64_t(sd.word) * sm.S + i] = StateIdentity(sd.kind);
                if (sd.kind == ST_SUM_I128) sm.st[int64_t(sd.word + 1) * sm.S + i] = 0;
            }
        }
        for (int i = tid; i < kPrivGroups * SIG::words * bd; i += bd) pacc[i] = 0;
        __syncthreads();
        const int64_t it = item_at;
        if (it >= B.nitems) return;
        if (P.nkeyparts == 0 && tid == 0 && sm.S > 0) {
            const int i = int(uint32_t(Fmix64(0)) & uint32_t(sm.S - 1));
            sm.keys[i] = 0;
            sm.gid[i] = 0;
            sm.gid_slot[0] = i;
            misc[0] = 1;
            misc[2] = 1;
        }
        __syncthreads();
        const HighItem item = B.items[it];
        const HighTask& tk = B.tasks[item.task];
        HighDst D;
        D.T = tk.T;
        D.cap_mask = uint64_t(tk.T.capacity - 1);
        D.deferred = B.deferred;
        D.deferred_cap = B.deferred_cap;
        D.ndeferred = &B.counters->ndeferred;
        D.spill = B.spill;
        D.spill_cap = B.spill_cap;
        D.nspill = &B.counters->nspill;
        D.error = &B.counters->error;
        D.tag = item.task;

        uint64_t ckey[kPrivGroups];
        int cgid[kPrivGroups];
#pragma unroll
        for (int j = 0; j < kPrivGroups; ++j) {
            ckey[j] = kEmptyKey;
            cgid[j] = -1;
        }
        int ncache = 0;
        if (P.nkeyparts == 0) {
            ckey[0] = 0;
            cgid[0] = 0;
            ncache = 1;
        }
        const char* cb[kFastCols];
#pragma unroll
        for (int c = 0; c < kFastCols; ++c) {
            cb[c] = nullptr;
            if (c < SIG::Cols::n) cb[c] = tk.cols[c] + item.row0 * SIG::cw(c);
        }
        const uint8_t* sel = tk.sel ? tk.sel + item.row0 : nullptr;
        const int64_t n = item.nrows;
        // Columns of every task start on a four-value boundary and selections
        // on a four-byte one (checked by the host), so full quads take vector
        // loads; items start on a multiple of four rows.
#pragma unroll 1
        for (int64_t r4 = int64_t(tid >> 5) * kWarpRows + lane * kQuadRows; r4 < n; r4 += (bd >> 5) * kWarpRows) {
            const int nvalid = int(min(int64_t(kQuadRows), n - r4));
            int64_t q[NC][kQuadRows];
            LoadQuad<SIG>(q, cb, r4, nvalid);
            uint32_t selq = nvalid == kQuadRows ? 0x01010101u : 0u;
            if (nvalid < kQuadRows) {
                for (int j = 0; j < nvalid; ++j) selq |= 1u << (8 * j);
            }
            if (sel) {
                if (nvalid == kQuadRows) {
                    selq = __ldcs(reinterpret_cast<const unsigned int*>(sel + r4));
                } else {
                    uint32_t m = 0;
                    for (int j = 0; j < nvalid; ++j) m |= uint32_t(sel[r4 + j]) << (8 * j);
                    selq = m;
                }
            }
#pragma unroll
            for (int j = 0; j < kQuadRows; ++j) {
                if (((selq >> (8 * j)) & 0xffu) == 0) continue;
                RegRow<SIG::Cols::n> cur;
                QuadRow<SIG>(cur, q, j);
                if (SIG::Atoms::n && ShapeHeld<SIG>(P, F, cur) != F.clause_mask) continue;
                const uint64_t key = ShapeKey<SIG>(cur);
                int g = -1;
#pragma unroll
                for (int k = 0; k < kPrivGroups; ++k) g = ckey[k] == key ? cgid[k] : g;
                const bool special = P.key_full64 && key == kEmptyKey;
                int slot = -1;
                if (g < 0 && !special) {
                    slot = sm.Find(key);
                    if (slot >= 0) {
                        const int gg = *reinterpret_cast<volatile int*>(&sm.gid[slot]);
                        if (gg >= 0 && gg < kPrivGroups && ncache < kPrivGroups) {
                            g = gg;
#pragma unroll
                            for (int k = 0; k < kPrivGroups; ++k) {
                                if (k == ncache) {
                                    ckey[k] = key;
                                    cgid[k] = gg;
                                }
                            }
                            ++ncache;
                        }
                    }
                }
                if (g >= 0) {
                    ShapeFoldP<SIG, kQuadThreads>(pacc + g * SIG::words * kQuadThreads + tid, F, cur);
                } else if (slot >= 0) {
                    ShapeVals<SIG> v;
                    ShapeRowVals<SIG>(v, F, cur);
                    ShapeSmemAtomics<SIG>(sm.st + slot, sm.S, v);
                } else {
                    // The tier is full, or the key is the empty marker: the
                    // aggregate's own table (its flag slot for the marker).
                    ShapeVals<SIG> v;
                    ShapeRowVals<SIG>(v, F, cur);
                    uint64_t* gw = D.T.slots + D.T.capacity * D.T.slot_words;
                    if (special) {
                        auto* flag = reinterpret_cast<unsigned long long*>(gw + D.T.key_off);
                        if (*reinterpret_cast<volatile unsigned long long*>(flag) == 0 && atomicExch(flag, 1ull) == 0)
                            atomicAdd(sm.fresh, 1u);
                        ShapeAtomics<SIG>(gw + D.T.state_off, 1, v);
                    } else {
                        int is_new = 0;
                        const int64_t gs = GlobalFindH(D.T, D.cap_mask, Fmix64(key), key, is_new);
                        if (is_new) atomicAdd(sm.fresh, 1u);
                        if (gs < 0) {
                            DeferTo(D, item.row0 + r4 + j);   // replayed after the table grows
                        } else {
                            ShapeAtomics<SIG>(D.T.slots + gs * D.T.slot_words + D.T.state_off, 1, v);
                        }
                    }
                }
            }
        }
        __syncthreads();
        // Lane-private accumulators -> shared tier.
        const int ng = int(min(*reinterpret_cast<volatile unsigned*>(sm.ngid), unsigned(kPrivGroups)));
        constexpr int nwarps = bd >> 5;
        for (int w = tid >> 5; w < ng * SIG::n; w += nwarps) {
            const int qg = w / SIG::n;
            const int st2 = w - qg * SIG::n;
            const int o = SIG::off(st2);
            const bool wide2 = SIG::width(st2) == 2;
            uint64_t lo = 0, hi = 0;
            for (int t2 = lane; t2 < bd; t2 += 32) {
                const uint64_t* src = pacc + int64_t(qg * SIG::words + o) * bd + t2;
                Add128(lo, hi, src[0], wide2 ? src[bd] : 0ull);
            }
            WarpSum128(lo, hi);
            if (lane == 0 && (lo | hi)) {
                const int slot = *reinterpret_cast<volatile int*>(&sm.gid_slot[qg]);
                const StateDesc sd = P.states[st2];
                uint64_t* dst = sm.st + int64_t(sd.word) * sm.S + slot;
                ApplyState(dst, dst + sm.S, sd.kind, lo, hi, 0.0);
            }
        }
        __syncthreads();
        // Shared tier -> the aggregate's table (tagged spill when it is full).
        const int rec_words = 2 + P.state_words;
        for (int i = tid; i < sm.S; i += bd) {
            const uint64_t key = sm.keys[i];
            if (key == kEmptyKey) continue;
            int is_new = 0;
            const int64_t g = GlobalFindH(D.T, D.cap_mask, Fmix64(key), key, is_new);
            if (is_new) atomicAdd(sm.fresh, 1u);
            if (g < 0) {
                const unsigned long long e = atomicAdd(D.nspill, 1ull);
                if (int64_t(e) >= D.spill_cap) {
                    SetError(D.error, DE_SPILL_FULL);
                    continue;
                }
                uint64_t* rec = D.spill + int64_t(e) * rec_words;
                rec[0] = key;
                for (int w = 0; w < P.state_words; ++w) rec[1 + w] = sm.st[int64_t(w) * sm.S + i];
                rec[1 + P.state_words] = uint64_t(D.tag);
                continue;
            }
            uint64_t* gbase = D.T.slots + g * D.T.slot_words + D.T.state_off;
            for (int st2 = 0; st2 < P.nstates; ++st2) {
                const StateDesc sd = P.states[st2];
                const uint64_t lo = sm.st[int64_t(sd.word) * sm.S + i];
                const uint64_t hi = sd.kind == ST_SUM_I128 ? sm.st[int64_t(sd.word + 1) * sm.S + i] : 0;
                if (IsIdentity(sd.kind, lo, hi)) continue;
                ApplyState(gbase + sd.word, gbase + sd.word + 1, sd.kind, lo, hi, 0.0);
            }
        }
        __syncthreads();
        if (tid == 0 && sm.fresh[0]) atomicAdd(&B.new_groups[item.task], (unsigned long long)sm.fresh[0]);
    }
}

// ---------------------------------------------------------------------------
// Heavy hitters of a high-cardinality aggregate: its keys counted over an
// evenly strided sample of rows in a scratch table, then the most frequent
// (sampled at least twice, at most k of them) kept as the shared tier's seeds.
// ---------------------------------------------------------------------------
struct SeedSlot {
    unsigned long long key;
    unsigned count;
    unsigned pad;
};

constexpr int kSeedSampleRows = 1 << 16;
constexpr int kSeedTableSlots = 1 << 17;   // twice the sample: at most half full
constexpr int kSeedProbe = 64;
constexpr int kSeedHistBins = 1024;

__global__ void SeedInitKernel(SeedSlot* tab, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        tab[i].key = kEmptyKey;
        tab[i].count = 0;
        tab[i].pad = 0;
    }
}

template <class SH>
__global__ void __launch_bounds__(256) SeedSampleKernel(const __grid_constant__ AggLaunch L, SeedSlot* tab,
                                                        int64_t stride, int64_t nsample) {
    const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= nsample) return;
    const char* cb[kFastCols];
#pragma unroll
    for (int c = 0; c < kFastCols; ++c) cb[c] = c < SH::Cols::n ? L.P.cols[L.F.col_slot[c]].data : nullptr;
    const TileRow row{cb, int(i * stride)};
    const uint64_t key = ShapeKey<SH>(row);
    if (key == kEmptyKey) return;
    uint32_t h = uint32_t(Fmix64(key)) & uint32_t(kSeedTableSlots - 1);
    for (int p = 0; p < kSeedProbe; ++p) {
        auto* kp = &tab[h].key;
        const unsigned long long cur = *reinterpret_cast<volatile unsigned long long*>(kp);
        if (cur == key) {
            atomicAdd(&tab[h].count, 1u);
            return;
        }
        if (cur == kEmptyKey) {
            const unsigned long long old = atomicCAS(kp, kEmptyKey, key);
            if (old == kEmptyKey || old == key) {
                atomicAdd(&tab[h].count, 1u);
                return;
            }
        }
        h = (h + 1) & uint32_t(kSeedTableSlots - 1);
    }
}

// One CTA: a histogram of the sampled counts picks the smallest count c >= 2
// whose keys sampled at least c times number at most k; those keys are the
// seeds (in table order).
__global__ void __launch_bounds__(1024) SeedSelectKernel(const SeedSlot* tab, int k, uint64_t* seeds, int* nseed) {
    __shared__ unsigned hist[kSeedHistBins];
    __shared__ unsigned thr;
    __shared__ unsigned taken;
    for (int i = threadIdx.x; i < kSeedHistBins; i += blockDim.x) hist[i] = 0;
    __syncthreads();
    for (int i = threadIdx.x; i < kSeedTableSlots; i += blockDim.x) {
        const unsigned c = tab[i].count;
        if (c >= 2) atomicAdd(&hist[min(c, unsigned(kSeedHistBins - 1))], 1u);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned cum = 0, t = kSeedHistBins;
        for (int b = kSeedHistBins - 1; b >= 2; --b) {
            if (cum + hist[b] > unsigned(k)) break;
            cum += hist[b];
            t = unsigned(b);
        }
        thr = t;
        taken = 0;
    }
    __syncthreads();
    for (int i = threadIdx.x; i < kSeedTableSlots; i += blockDim.x) {
        const unsigned c = tab[i].count;
        if (c >= 2 && min(c, unsigned(kSeedHistBins - 1)) >= thr) {
            const unsigned at = atomicAdd(&taken, 1u);
            if (at < unsigned(k)) seeds[at] = tab[i].key;
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) *nseed = int(min(taken, unsigned(k)));
}

// The instantiated query shapes.  QDB_C(w, u): a fast column of w bytes
// (u: unsigned); QDB_A(op, col): a filter atom; QDB_S(kind, nf, cols...): a
// state.  A plan whose shape is not listed runs the general typed kernel.
#define QDB_C(w, u) ColCode(w, u)
#define QDB_A(op, c) AtomCode(op, c)
#define QDB_S(...) StateCode(__VA_ARGS__)
#define QDB_SHAPE_LIST(X)                                                                                    \
    /* lineitem (TPC-H Q1 shape): GROUP BY two one-byte codes WHERE date <= c: SUM(qty), SUM(price),       \
       SUM(price*(c-disc)), SUM(price*(c-disc)*(c+tax)), COUNT(*), SUM(disc) */                            \
    X(Shape<IntList<QDB_C(1, 1), QDB_C(1, 1), QDB_C(4, 0), QDB_C(8, 0), QDB_C(8, 0), QDB_C(8, 0), QDB_C(8, 0)>, \
            IntList<QDB_A(AT_LE, 2)>, IntList<KeyCode(0, 8, 0), KeyCode(1, 8, 8)>,                                                         \
            IntList<QDB_S(SK_SUM64, 1, 3), QDB_S(SK_SUM128_OF64, 1, 4),                                       \
                    QDB_S(SK_SUM128, 2, 4, 5, 0, FF_X, FF_SUB),                                                \
                    QDB_S(SK_SUM128, 3, 4, 5, 6, FF_X, FF_SUB, FF_ADD), QDB_S(SK_COUNT, 0),                    \
                    QDB_S(SK_SUM64, 1, 5)>>)                                                                   \
    /* COUNT(*) GROUP BY an 8-byte key */                                                                    \
    X(Shape<IntList<QDB_C(8, 0)>, IntList<>, IntList<KeyCode(0, 64, 0)>, IntList<QDB_S(SK_COUNT, 0)>>)                        \
    /* SUM(x), COUNT(*) GROUP BY an 8-byte key */                                                            \
    X(Shape<IntList<QDB_C(8, 0), QDB_C(8, 0)>, IntList<>, IntList<KeyCode(0, 64, 0)>,                                         \
            IntList<QDB_S(SK_SUM64, 1, 1), QDB_S(SK_COUNT, 0)>>)                                               \
    /* keyless SUM(x * y) WHERE x BETWEEN a AND b over 8-byte columns (a TPC-H Q6 shape) */                  \
    X(Shape<IntList<QDB_C(8, 0), QDB_C(8, 0)>, IntList<QDB_A(AT_BETWEEN, 0)>, IntList<>,                      \
            IntList<QDB_S(SK_SUM64, 2, 0, 1), QDB_S(SK_COUNT, 0)>>)

// Shapes of the high-cardinality kernel (global table, typed atomics).
#define QDB_HIGH_SHAPE_LIST(X)                                                                               \
    /* GROUP BY an 8-byte key: COUNT(*), SUM(a), MIN(a), MAX(a), SUM(double x) */                          \
    X(Shape<IntList<QDB_C(8, 0), QDB_C(8, 0), QDB_C(8, 0)>, IntList<>, IntList<KeyCode(0, 64, 0)>,            \
            IntList<QDB_S(SK_COUNT, 0), QDB_S(SK_SUM64, 1, 1), QDB_S(SK_MIN64, 1, 1), QDB_S(SK_MAX64, 1, 1),    \
                    QDB_S(SK_SUMF64, 1, 2)>>)                                                                 \
    /* COUNT(*) GROUP BY an 8-byte key */                                                                    \
    X(Shape<IntList<QDB_C(8, 0)>, IntList<>, IntList<KeyCode(0, 64, 0)>, IntList<QDB_S(SK_COUNT, 0)>>)        \
    /* SUM(x), COUNT(*) GROUP BY an 8-byte key */                                                            \
    X(Shape<IntList<QDB_C(8, 0), QDB_C(8, 0)>, IntList<>, IntList<KeyCode(0, 64, 0)>,                         \
            IntList<QDB_S(SK_SUM64, 1, 1), QDB_S(SK_COUNT, 0)>>)

// Index mode: rows named by (row, build row) pairs, global table only.
template <bool WIDE>
__global__ void __launch_bounds__(256) AggIndexKernel(const __grid_constant__ AggLaunch L) {
    unsigned* misc = reinterpret_cast<unsigned*>(DynSmem() + L.off_misc);
    if (threadIdx.x == 0) misc[1] = 0;
    __syncthreads();
    for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < L.nindex;
         i += int64_t(gridDim.x) * blockDim.x) {
        RowAcc acc{&L.P, nullptr, 0, L.index[2 * i], L.index[2 * i + 1], -1, 0};
        FoldRow<WIDE, true, false>(L, acc);
    }
    __syncthreads();
    if (threadIdx.x == 0 && misc[1]) atomicAdd(&L.counters->new_groups, (unsigned long long)misc[1]);
}

// ---------------------------------------------------------------------------
// Table maintenance kernels.
// ---------------------------------------------------------------------------
// An empty slot's words are built once per block in shared memory.  With a
// 16-byte aligned table the table is one array of 16-byte vectors, slot_words
// / 2 per slot; blocks hold a multiple of that many threads and the grid
// strides by a multiple too, so each thread always writes the same vector of
// the slot, and consecutive threads consecutive vectors.  The host then
// clears the flag slot's key word (slot_words <= kInitMaxSlotWords: at most
// 1 + kMaxKeyWords + kMaxStates).
constexpr int kInitMaxSlotWords = 64;
static_assert(1 + kMaxKeyWords + kMaxStates <= kInitMaxSlotWords + 1, "slot template too small");

__global__ void AggInitKernel(uint64_t* slots, int64_t capacity, int32_t slot_words, int32_t key_off,
                              int32_t state_off, int32_t wide, int32_t vec16, const __grid_constant__ StatesParam sp) {
    __shared__ __align__(16) uint64_t tmpl[kInitMaxSlotWords];
    for (int off = threadIdx.x; off < slot_words; off += blockDim.x) {
        uint64_t v = 0;
        if (!wide && off == key_off) {
            v = kEmptyKey;
        } else if (off >= state_off) {
            const int32_t sw = off - state_off;
            for (int s = 0; s < sp.n; ++s) {
                if (sp.s[s].word == sw) v = StateIdentity(sp.s[s].kind);
            }
        }
        tmpl[off] = v;
    }
    __syncthreads();
    const int64_t stride = int64_t(gridDim.x) * blockDim.x;
    const int64_t first = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
    if (vec16) {
        const int vec = slot_words / 2;
        const uint4 v = reinterpret_cast<const uint4*>(tmpl)[threadIdx.x % vec];
        uint4* dst = reinterpret_cast<uint4*>(slots);
        const int64_t total = (capacity + 1) * vec;
        for (int64_t i = first; i < total; i += stride) dst[i] = v;
    } else {
        const uint64_t v = tmpl[threadIdx.x % slot_words];
        const int64_t total = (capacity + 1) * slot_words;
        for (int64_t i = first; i < total; i += stride) slots[i] = v;
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
constexpr int64_t kFinChunk = kFinChunkSlots;   // slots per block

struct FinLaunch {
    AggPlan P;
    OutputPlan O;
    GTableDev T;
    AggOutputCol cols[kMaxCols + kMaxAggs];
    int32_t ncols;
    int64_t groups;
    unsigned long long* row_counters;   // per aggregate: output rows claimed so far
    int* err;
    // Batched finalize: block b covers chunk blocks[b].chunk of table
    // tables[blocks[b].task] (nullptr: one table, T).
    const GTableDev* tables;
    const FinBlock* blocks;
    // Copy plan: every output column is one (or, for DECIMAL128, two) slot
    // words stored as they are (copy_n = ncols), else 0.
    int32_t copy_n;
    int8_t copy_word[kMaxCols + kMaxAggs];
    int8_t copy_two[kMaxCols + kMaxAggs];
    int8_t copy_key[kMaxCols + kMaxAggs];
};

// The table and slot range of a finalize block.
__device__ __forceinline__ GTableDev FinBlockTable(const FinLaunch& L, int64_t& begin, int64_t& end, int64_t& delta,
                                                   int64_t& slice0, int& task) {
    GTableDev T = L.T;
    int64_t chunk = blockIdx.x;
    delta = 0;
    slice0 = -1;
    task = 0;
    if (L.blocks) {
        const FinBlock fb = L.blocks[blockIdx.x];
        T = L.tables[fb.task];
        task = fb.task;
        chunk = fb.chunk;
        delta = fb.delta;
        slice0 = fb.slice0;
    }
    begin = chunk * kFinChunk;
    end = Min64(begin + kFinChunk, T.capacity + 1);
    return T;
}

__device__ __forceinline__ bool SlotOccupied(const GTableDev& T, int64_t i) {
    const uint64_t* s = T.slots + i * T.slot_words;
    if (T.wide) return i < T.capacity && s[0] == 2;
    if (i == T.capacity) return s[T.key_off] != 0;
    return s[T.key_off] != kEmptyKey;
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

// slice0 >= 0: the output is cut into per-aggregate slices and `row`'s
// slice starts at row slice0; string offsets count from the slice start and
// each row writes its own start offset too.
__device__ __forceinline__ void StoreValue(const AggOutputCol& col, int64_t row, const GVal& v, bool null,
                                           int64_t slice0 = -1) {
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
                if (slice0 >= 0) {
                    col.offsets[row] = int32_t(row - slice0);
                    col.offsets[row + 1] = int32_t(row + 1 - slice0);
                } else {
                    col.offsets[row + 1] = int32_t(row + 1);
                    if (row == 0) col.offsets[0] = 0;
                }
            }
            break;
    }
}

// The copy-plan finalize: the same one-pass row claiming as FinWriteKernel,
// each output column one (or two) slot words as stored.  Kept apart from the
// general kernel so that its few registers leave room for many warps, the
// only way a pass bound by dependent loads and row claims fills HBM.
__global__ void __launch_bounds__(kFinThreads) FinCopyKernel(const __grid_constant__ FinLaunch L) {
    int64_t begin, end, delta, slice0;
    int task = 0;
    const GTableDev T = FinBlockTable(L, begin, end, delta, slice0, task);
    const int64_t row_base = slice0 < 0 ? 0 : slice0;
    const int lane = LaneId();
    for (int64_t b = begin + (threadIdx.x & ~31); b < end; b += blockDim.x) {
        const int64_t i = b + lane;
        const bool occ = i < end && SlotOccupied(T, i);
        const unsigned m = __ballot_sync(kFull, occ);
        if (!m) continue;
        unsigned long long first = 0;
        if (lane == 0) first = atomicAdd(&L.row_counters[task], (unsigned long long)__popc(m));
        first = __shfl_sync(kFull, first, 0);
        if (!occ) continue;
        const int64_t row = row_base + int64_t(first) + __popc(m & ((1u << lane) - 1));
        if (row >= L.groups) continue;
        const uint64_t* s = T.slots + i * T.slot_words;
        const bool flag_slot = !T.wide && i == T.capacity;
        for (int k = 0; k < L.copy_n; ++k) {
            uint64_t* dst = reinterpret_cast<uint64_t*>(L.cols[k].data);
            const int w = L.copy_word[k];
            if (L.copy_two[k]) {
                dst[2 * row] = s[w];
                dst[2 * row + 1] = s[w + 1];
            } else {
                dst[row] = (L.copy_key[k] && flag_slot) ? kEmptyKey : s[w];
            }
        }
    }
}

// One pass over the table: each warp takes 32 consecutive slots at a time
// and claims output rows for its occupied ones with one atomic on the
// aggregate's row counter (groups come out in no particular order: an
// aggregate's output is a set of groups).
__global__ void __launch_bounds__(kFinThreads) FinWriteKernel(const __grid_constant__ FinLaunch L) {
    const AggPlan& P = L.P;
    const OutputPlan& O = L.O;
    int64_t begin, end, delta, slice0;
    int task = 0;
    const GTableDev T = FinBlockTable(L, begin, end, delta, slice0, task);
    const int64_t row_base = slice0 < 0 ? 0 : slice0;
    const int lane = LaneId();
    for (int64_t b = begin + (threadIdx.x & ~31); b < end; b += blockDim.x) {
        const int64_t i = b + lane;
        const bool occ = i < end && SlotOccupied(T, i);
        const unsigned m = __ballot_sync(kFull, occ);
        if (!m) continue;
        unsigned long long first = 0;
        if (lane == 0) first = atomicAdd(&L.row_counters[task], (unsigned long long)__popc(m));
        first = __shfl_sync(kFull, first, 0);
        const int64_t before = int64_t(first) + __popc(m & ((1u << lane) - 1));
        if (occ && L.copy_n) {
            const int64_t row = row_base + before;
            if (row < L.groups) {
                const uint64_t* s = T.slots + i * T.slot_words;
                const bool flag_slot = !T.wide && i == T.capacity;
                for (int k = 0; k < L.copy_n; ++k) {
                    uint64_t* dst = reinterpret_cast<uint64_t*>(L.cols[k].data);
                    const int w = L.copy_word[k];
                    if (L.copy_two[k]) {
                        dst[2 * row] = s[w];
                        dst[2 * row + 1] = s[w + 1];
                    } else {
                        dst[row] = (L.copy_key[k] && flag_slot) ? kEmptyKey : s[w];
                    }
                }
            }
        } else if (occ) {
            const int64_t row = row_base + before;
            if (row < L.groups) {
                const uint64_t* s = T.slots + i * T.slot_words;
                uint64_t kw[kMaxKeyWords];
                if (!T.wide && i == T.capacity) {
                    kw[0] = kEmptyKey;
                } else {
                    for (int w = 0; w < P.key_words; ++w) kw[w] = s[T.key_off + w];
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
                const uint64_t* st = s + T.state_off;
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
                    for (int k = 0; k < L.ncols; ++k) StoreValue(L.cols[k], row, rowv[k], (nulls >> k) & 1, slice0);
                } else {
                    GVal gv[kMaxGNodes];
                    uint64_t gn = 0;
                    OutRowAcc oa{rowv, nulls, &O};
                    if (!EvalGeneric(O.prog, O.root_max, O.list, oa, gv, gn)) SetError(L.err, DE_DIV_ZERO);
                    for (int k = 0; k < L.ncols; ++k) {
                        const int rt = O.roots[k];
                        StoreValue(L.cols[k], row, gv[rt], (gn >> rt) & 1, slice0);
                    }
                }
            }
        }
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
    EnsureSmemLimit(reinterpret_cast<const void*>(kernel), bytes);
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
    // Threads per block: a multiple of the vectors (or words) per slot.
    const bool vec16 = (reinterpret_cast<uintptr_t>(t.slots) & 15) == 0 && (t.slot_words & 1) == 0;
    const int per_slot = vec16 ? t.slot_words / 2 : t.slot_words;
    const int threads = per_slot * std::max(1, 512 / per_slot);
    const int64_t total = (t.capacity + 1) * per_slot;
    const int blocks = int(std::min<int64_t>((total + threads - 1) / threads, int64_t(DeviceSMs()) * 8));
    ProfileBegin(s, "agg_init_table", t.capacity);
    AggInitKernel<<<blocks, threads, 0, s>>>(t.slots, t.capacity, t.slot_words, t.key_off, t.state_off, t.wide,
                                             vec16 ? 1 : 0, sp);
    if (!t.wide) cudaMemsetAsync(t.slots + t.capacity * t.slot_words + t.key_off, 0, 8, s);   // flag slot: unused
    ProfileEnd(s);
    CountLaunch();
}

static void FillTableArgs(AggLaunch& L, const GTableDev& t) {
    L.T = t;
    L.cap_mask = uint64_t(t.capacity - 1);
}

namespace {

// Shape key of a typed plan: column codes, -1, atom codes, -1, key columns,
// -1, state codes; empty when a state has no compile-time kind.
std::vector<int> ShapeKeyOf(const AggPlan& P, const FastPlan& F) {
    std::vector<int> key;
    for (int c = 0; c < F.ncols; ++c) {
        const ColDesc& cd = P.cols[F.col_slot[c]];
        key.push_back(ColCode(cd.width, cd.kind == LK_UNSIGNED));
    }
    key.push_back(-1);
    for (int j = 0; j < F.natoms; ++j) key.push_back(AtomCode(F.atoms[j].op, F.atoms[j].col));
    key.push_back(-1);
    for (int j = 0; j < F.nkeys; ++j) key.push_back(KeyCode(F.key_col[j], F.key_bits[j], F.key_shift[j]));
    key.push_back(-1);
    for (int s = 0; s < F.nstates; ++s) {
        const FastState& st = F.states[s];
        int kind;
        switch (st.kind) {
            case ST_COUNT: kind = SK_COUNT; break;
            case ST_SUM_I64: kind = SK_SUM64; break;
            case ST_SUM_I128: kind = st.wide ? SK_SUM128 : SK_SUM128_OF64; break;
            case ST_MIN_I64: kind = SK_MIN64; break;
            case ST_MAX_I64: kind = SK_MAX64; break;
            case ST_SUM_F64: kind = SK_SUMF64; break;
            default: return {};
        }
        if ((kind == SK_COUNT) != (st.nf == 0)) return {};
        auto form = [&](int j) {
            if (j >= st.nf || kind == SK_SUMF64) return 0;
            const FastFactor& f = st.f[j];
            if (f.d == 1) return f.c == 0 ? int(FF_X) : int(FF_ADD);
            if (f.d == -1) return int(FF_SUB);
            return int(FF_AFFINE);
        };
        key.push_back(StateCode(kind, st.nf, st.nf > 0 ? st.f[0].col : 0, st.nf > 1 ? st.f[1].col : 0,
                                st.nf > 2 ? st.f[2].col : 0, form(0), form(1), form(2)));
    }
    return key;
}

template <class LIST>
void AppendList(std::vector<int>& key) {
    for (int i = 0; i < LIST::n; ++i) key.push_back(LIST::at(i));
}

// The shape's compile-time state words must be the plan's (the kernels
// address the table's state words by them).
template <class SH>
bool ShapeWordsMatch(const FastPlan& F) {
    if (SH::n != F.nstates) return false;
    for (int s = 0; s < SH::n; ++s) {
        if (SH::off(s) != F.states[s].word) return false;
    }
    return true;
}

template <class SH>
bool ShapeMatches(const std::vector<int>& key) {
    std::vector<int> want;
    AppendList<typename SH::Cols>(want);
    want.push_back(-1);
    AppendList<typename SH::Atoms>(want);
    want.push_back(-1);
    AppendList<typename SH::Keys>(want);
    want.push_back(-1);
    AppendList<typename SH::States>(want);
    return key == want;
}

using SigKernelFn = void (*)(AggLaunch);

SigKernelFn FindHighKernel(const AggPlan& P, const FastPlan& F) {
    const std::vector<int> key = ShapeKeyOf(P, F);
    if (key.empty()) return nullptr;
#define QDB_SHAPE_FIND(...) \
    if (ShapeMatches<__VA_ARGS__>(key) && ShapeWordsMatch<__VA_ARGS__>(F)) return AggHighKernel<__VA_ARGS__>;
    QDB_HIGH_SHAPE_LIST(QDB_SHAPE_FIND)
#undef QDB_SHAPE_FIND
    if (std::getenv("QDB_SHAPE_DEBUG")) {
        std::fprintf(stderr, "qdb: no compiled high-cardinality shape for key");
        for (int v : key) std::fprintf(stderr, " %d", v);
        std::fprintf(stderr, "\n");
    }
    return nullptr;
}

using SeedKernelFn = void (*)(AggLaunch, SeedSlot*, int64_t, int64_t);

SeedKernelFn FindSeedKernel(const AggPlan& P, const FastPlan& F) {
    const std::vector<int> key = ShapeKeyOf(P, F);
    if (key.empty()) return nullptr;
    // Seeds need a COUNT state: the flush skips the seeded slots it is 0 in.
#define QDB_SHAPE_FIND(...)                                                             \
    if (ShapeMatches<__VA_ARGS__>(key) && ShapeWordsMatch<__VA_ARGS__>(F))               \
        return __VA_ARGS__::count_off() >= 0 ? SeedSampleKernel<__VA_ARGS__> : nullptr;
    QDB_HIGH_SHAPE_LIST(QDB_SHAPE_FIND)
#undef QDB_SHAPE_FIND
    return nullptr;
}

using QuadKernelFn = void (*)(QuadLaunch);

QuadKernelFn FindQuadKernel(const AggPlan& P, const FastPlan& F) {
    const std::vector<int> key = ShapeKeyOf(P, F);
    if (key.empty()) return nullptr;
#define QDB_SHAPE_FIND(...) \
    if (ShapeMatches<__VA_ARGS__>(key) && ShapeWordsMatch<__VA_ARGS__>(F)) return AggSigQuadKernel<__VA_ARGS__>;
    QDB_SHAPE_LIST(QDB_SHAPE_FIND)
#undef QDB_SHAPE_FIND
    return nullptr;
}

// The listed-row kernel's arguments, from a launch laid out for it.
void QuadLaunchOf(const AggLaunch& L, QuadLaunch& Q) {
    std::memset(&Q, 0, sizeof(Q));
    Q.F = L.F;
    for (int c = 0; c < L.F.ncols && c < kFastCols; ++c) Q.cols[c] = L.P.cols[L.F.col_slot[c]].data;
    Q.selection = L.P.selection;
    Q.nrows = L.nrows;
    Q.T = L.T;
    Q.cap_mask = L.cap_mask;
    Q.counters = L.counters;
    Q.deferred = L.deferred;
    Q.deferred_cap = L.deferred_cap;
    Q.spill = L.spill;
    Q.spill_cap = L.spill_cap;
    static_assert(sizeof(Q.states) == sizeof(L.P.states), "state table sizes");
    std::memcpy(Q.states, L.P.states, sizeof(Q.states));
    Q.nstates = L.P.nstates;
    Q.state_words = L.P.state_words;
    Q.nkeyparts = L.P.nkeyparts;
    Q.key_full64 = L.P.key_full64;
    Q.smem_slots = L.smem_slots;
    Q.smem_limit = L.smem_limit;
    Q.off_misc = L.off_misc;
    Q.off_skeys = L.off_skeys;
    Q.off_sst = L.off_sst;
    Q.off_gid = L.off_gid;
    Q.off_pacc = L.off_pacc;
    static_assert(sizeof(Q.list) == sizeof(L.P.list), "IN-list sizes");
    std::memcpy(Q.list, L.P.list, sizeof(Q.list));
}

SigKernelFn FindSigKernel(const AggPlan& P, const FastPlan& F) {
    const std::vector<int> key = ShapeKeyOf(P, F);
    if (key.empty()) return nullptr;
#define QDB_SHAPE_FIND(...) \
    if (ShapeMatches<__VA_ARGS__>(key) && ShapeWordsMatch<__VA_ARGS__>(F)) return AggSigDirectKernel<__VA_ARGS__>;
    QDB_SHAPE_LIST(QDB_SHAPE_FIND)
#undef QDB_SHAPE_FIND
    if (std::getenv("QDB_SHAPE_DEBUG")) {
        std::fprintf(stderr, "qdb: no compiled shape for key");
        for (int v : key) std::fprintf(stderr, " %d", v);
        std::fprintf(stderr, "\n");
    }
    return nullptr;
}

}  // namespace

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
    L.inline_slot = a.join ? a.inline_slot : -1;
    L.seeds = a.seeds;
    L.nseed = a.nseed;
    const bool wide = a.table.wide != 0;

    if (a.index) {
        if (a.nindex == 0) return;
        const int blocks = int(std::min<int64_t>((a.nindex + 255) / 256, int64_t(g_sms) * 8));
        // The index kernel keeps only its counters in shared memory.
        L.off_misc = 0;
        L.smem_slots = 0;
        ProfileBegin(s, "agg_update_index", a.nindex);
        if (wide) AggIndexKernel<true><<<blocks, 256, 64, s>>>(L);
        else AggIndexKernel<false><<<blocks, 256, 64, s>>>(L);
        ProfileEnd(s);
        CountLaunch();
        return;
    }
    if (a.nrows == 0) return;

    // Stage every aligned scan column (not build-side ones) through shared memory.
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
    const int sw = L.P.state_words;
    const size_t budget = g_smem_optin - 1024;
    bool priv = a.priv && !wide;
    int S = wide ? 0 : (priv ? 64 : a.smem_slots);
    const size_t pacc_bytes = size_t(kPrivGroups) * sw * kAggThreads * 8;
    auto layout = [&](int T, int stages, int S_) -> size_t {
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
        L.stages = any ? stages : 1;
        L.tile_rows = T;
        L.off_bars = int(Align(int64_t(L.stages) * L.stage_bytes, 16));
        L.off_misc = L.off_bars + 16 * L.stages;
        L.off_skeys = int(Align(L.off_misc + 64, 128));
        L.off_sst = L.off_skeys + S_ * 8;
        L.off_gid = L.off_sst + S_ * sw * 8;
        L.off_pacc = int(Align(L.off_gid + S_ * 4, 16));
        return size_t(L.off_pacc) + (priv ? pacc_bytes : 0);
    };
    int T = 1024, stages = 3;
    if (bytes_per_row > 0) {
        T = 256;
        while (T * 2 * bytes_per_row <= 40 * 1024 && T < 4096) T *= 2;
    }
    // Shrink tiles, then stages, then the private accumulators, until it fits.
    for (;;) {
        if (layout(T, stages, S) <= budget) break;
        if (priv && S > 64) { S >>= 1; continue; }
        if (!priv && S > 256) { S >>= 1; continue; }
        if (T > 256) { T >>= 1; continue; }
        if (stages > 2) { stages--; continue; }
        if (priv) { priv = false; S = a.smem_slots; T = 1024; stages = 3; continue; }
        if (S > 0) { S >>= 1; if (S < 32) S = 0; continue; }
        break;
    }
    if (!priv && !wide) {
        // Grow the shared table into whatever shared memory is left.
        while (S > 0 && S < a.smem_slots && layout(T, stages, S * 2) <= budget) S *= 2;
    }
    const size_t smem_bytes = layout(T, stages, S);
    L.smem_slots = S;
    L.smem_limit = S / 2;
    L.priv = priv;
    L.any_staged = any ? 1 : 0;

    const int64_t ntiles = (a.nrows + T - 1) / T;
    const int grid = int(std::max<int64_t>(1, std::min<int64_t>(ntiles, g_sms)));
    const bool gen = L.P.generic_root >= 0;
    const int variant = (wide ? 8 : 0) | (a.join ? 4 : 0) | (gen ? 2 : 0) | (priv ? 1 : 0);
    if (a.fast && variant == 1) {
        // A typed plan with an instantiated state signature: the listed-row
        // kernels read their columns straight from HBM (nothing is staged).
        // Four rows per thread when every typed column (and the selection)
        // starts on a boundary of four values.
        bool quad = true;
        for (int c = 0; c < a.fast->ncols && quad; ++c) {
            const ColDesc& cd = L.P.cols[a.fast->col_slot[c]];
            quad = (reinterpret_cast<uintptr_t>(cd.data) % uintptr_t(std::min(16, 4 * int(cd.width)))) == 0;
        }
        if (L.P.selection && (reinterpret_cast<uintptr_t>(L.P.selection) & 3)) quad = false;
        if (quad) {
            if (QuadKernelFn fn = FindQuadKernel(L.P, *a.fast)) {
                L.F = *a.fast;
                layout(16, 1, 64);
                const size_t bytes = size_t(L.off_pacc) + size_t(kPrivGroups) * sw * kQuadThreads * 8;
                if (bytes <= budget) {
                    L.smem_slots = 64;
                    L.smem_limit = 32;
                    L.priv = 1;
                    static thread_local QuadLaunch* Qp = nullptr;
                    if (!Qp) Qp = new QuadLaunch();
                    QuadLaunchOf(L, *Qp);
                    SetSmem(fn, bytes);
                    int per_sm = 1;
                    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, kQuadThreads, bytes) != cudaSuccess) {
                        cudaGetLastError();
                        per_sm = 1;
                    }
                    // At least 16K rows per CTA: the merge at the end costs a few
                    // microseconds per CTA.
                    const int64_t nt = (a.nrows + (int64_t(1) << 14) - 1) >> 14;
                    const int g2 = int(std::max<int64_t>(1, std::min<int64_t>(nt, int64_t(g_sms) * std::max(1, per_sm))));
                    ProfileBegin(s, "agg_update_sig", a.nrows);
                    fn<<<g2, kQuadThreads, bytes, s>>>(*Qp);
                    ProfileEnd(s);
                    CountLaunch();
                    return;
                }
                layout(T, stages, S);
            }
        }
        if (SigKernelFn fn = FindSigKernel(L.P, *a.fast)) {
            L.F = *a.fast;
            // The kernel stages nothing: a token stage keeps the layout's offsets.
            layout(16, 1, 64);
            const size_t pacc_sig = size_t(kPrivGroups) * sw * kSigThreads * 8;
            const size_t bytes = size_t(L.off_pacc) + pacc_sig;
            const int Ts = 2048;                   // rows per CTA at least, for the grid size
            if (bytes <= budget) {
                L.smem_slots = 64;
                L.smem_limit = 32;
                L.priv = 1;
                const int64_t nt = (a.nrows + Ts - 1) / Ts;
                const int g2 = int(std::max<int64_t>(1, std::min<int64_t>(nt, g_sms)));
                SetSmem(fn, bytes);
                ProfileBegin(s, "agg_update_sig", a.nrows);
                fn<<<g2, kSigThreads, bytes, s>>>(L);
                ProfileEnd(s);
                CountLaunch();
                return;
            }
            layout(T, stages, S);
        }
    }
    if (a.fast && variant == 0 && any) {
        if (SigKernelFn fn = FindHighKernel(L.P, *a.fast)) {
            // The largest shared tier (up to the state's slot budget) that fits.
            int S2 = std::max(256, a.smem_slots);
            while (S2 > 256 && size_t(HighLayoutOf(S2, sw).bytes) > budget) S2 >>= 1;
            const HighLayout hl = HighLayoutOf(S2, sw);
            if (size_t(hl.bytes) <= budget) {
                L.smem_slots = S2;
                L.smem_limit = S2 / 2;
                L.F = *a.fast;
                const int hgrid = int(std::max<int64_t>(1, std::min<int64_t>((a.nrows + 4095) / 4096, g_sms)));
                SetSmem(fn, size_t(hl.bytes));
                ProfileBegin(s, "agg_update_high", a.nrows);
                fn<<<hgrid, kHighThreads, size_t(hl.bytes), s>>>(L);
                ProfileEnd(s);
                CountLaunch();
                return;
            }
        }
    }
    const char* name = a.join ? "join_agg_probe" : "agg_update";
    ProfileBegin(s, name, a.nrows);
    auto launch = [&](auto kernel) {
        SetSmem(kernel, smem_bytes);
        kernel<<<grid, kAggThreads, smem_bytes, s>>>(L);
    };
    if (a.fast && variant <= 1) {
        L.F = *a.fast;
        if (priv) launch(AggUpdateKernel<false, false, false, true, true>);
        else launch(AggUpdateKernel<false, false, false, false, true>);
        ProfileEnd(s);
        CountLaunch();
        return;
    }
    switch (variant) {
        case 0: launch(AggUpdateKernel<false, false, false, false>); break;
        case 1: launch(AggUpdateKernel<false, false, false, true>); break;
        case 2: launch(AggUpdateKernel<false, false, true, false>); break;
        case 3: launch(AggUpdateKernel<false, false, true, true>); break;
        case 4: launch(AggUpdateKernel<false, true, false, false>); break;
        case 5: launch(AggUpdateKernel<false, true, false, true>); break;
        case 6: launch(AggUpdateKernel<false, true, true, false>); break;
        case 7: launch(AggUpdateKernel<false, true, true, true>); break;
        case 8: case 9: launch(AggUpdateKernel<true, false, false, false>); break;
        case 10: case 11: launch(AggUpdateKernel<true, false, true, false>); break;
        case 12: case 13: launch(AggUpdateKernel<true, true, false, false>); break;
        default: launch(AggUpdateKernel<true, true, true, false>); break;
    }
    ProfileEnd(s);
    CountLaunch();
}

bool AggHighSeedable(const AggPlan& p, const FastPlan& f) {
    return p.nkeyparts > 0 && p.key_words <= 1 && FindHighKernel(p, f) != nullptr && FindSeedKernel(p, f) != nullptr;
}

size_t AggSeedScratch() { return size_t(kSeedTableSlots) * sizeof(SeedSlot); }

bool AggSeedHeavy(const AggPlan& p, const FastPlan& f, int64_t nrows, uint64_t* seeds, int* nseed, int k,
                  void* scratch, cudaStream_t s) {
    const SeedKernelFn fn = FindSeedKernel(p, f);
    if (!fn || nrows <= 0 || k <= 0 || !scratch) return false;
    auto* tab = static_cast<SeedSlot*>(scratch);
    static thread_local AggLaunch* Lp = nullptr;
    if (!Lp) Lp = new AggLaunch();
    AggLaunch& L = *Lp;
    std::memset(&L, 0, sizeof(L));
    L.P = p;
    L.F = f;
    const int64_t nsample = std::min<int64_t>(nrows, kSeedSampleRows);
    const int64_t stride = nrows / nsample;
    ProfileBegin(s, "agg_seed", nsample);
    SeedInitKernel<<<kSeedTableSlots / 256, 256, 0, s>>>(tab, kSeedTableSlots);
    fn<<<int((nsample + 255) / 256), 256, 0, s>>>(L, tab, stride, nsample);
    SeedSelectKernel<<<1, 1024, 0, s>>>(tab, k, seeds, nseed);
    ProfileEnd(s);
    CountLaunch(3);
    return true;
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

// Output columns of an identity output that no group can leave NULL (keys
// and aggregates over non-nullable inputs) get an all-valid bitmap up front
// instead of one atomic per row.
static void PresetValidity(const AggPlan& p, const OutputPlan& out, FinLaunch& L, int64_t rows, cudaStream_t s,
                           bool packed) {
    if (!out.identity) return;
    const size_t words = size_t((rows + 31) / 32);
    // Runs of never-NULL columns whose validity words lie side by side in one
    // packed output block take one memset each.  Only there: the masks of
    // caller-owned outputs may be separate allocations that merely abut, and
    // a memset may not run across an allocation's end.
    uint32_t* run = nullptr;
    size_t run_words = 0;
    for (int k = 0; k < L.ncols; ++k) {
        AggOutputCol& c = L.cols[k];
        if (!c.valid) continue;
        bool never_null;
        if (k < p.nkeyparts) never_null = p.keys[k].null_shift == 0xFF;
        else if (k - p.nkeyparts < p.naggs) never_null = p.aggs[k - p.nkeyparts].valid_state == 0xFF;
        else never_null = false;
        if (!never_null) continue;
        if (packed && run && c.valid == run + run_words) {
            run_words += words;
        } else {
            if (run) cudaMemsetAsync(run, 0xFF, run_words * 4, s);
            run = c.valid;
            run_words = words;
        }
        c.valid = nullptr;
    }
    if (run) cudaMemsetAsync(run, 0xFF, run_words * 4, s);
}

// Copy plan of an identity output whose columns are all never NULL and are
// each one slot word as stored: 64-bit keys unpacked from one word, and
// COUNT / SUM / MIN / MAX of integers, SUM of doubles (bits as summed) and
// 128-bit decimal sums.  `t` gives the slot layout.
static void PlanCopy(const AggPlan& p, const OutputPlan& out, const GTableDev& t, FinLaunch& L) {
    L.copy_n = 0;
    if (!out.identity || t.wide || p.key_words != 1) return;
    for (int k = 0; k < L.ncols; ++k) {
        const AggOutputCol& c = L.cols[k];
        if (c.valid || c.offsets) return;
        const bool i64 = c.type == QDB_TYPE_I64 || c.type == QDB_TYPE_U64 || c.type == QDB_TYPE_DECIMAL64;
        L.copy_two[k] = 0;
        L.copy_key[k] = 0;
        if (k < p.nkeyparts) {
            const KeyPart& kp = p.keys[k];
            if (kp.bits != 64 || kp.shift != 0 || kp.null_shift != 0xFF) return;
            if (!(kp.is_float ? c.type == QDB_TYPE_F64 : i64)) return;
            L.copy_word[k] = int8_t(t.key_off + kp.word);
            L.copy_key[k] = 1;
        } else if (k - p.nkeyparts < p.naggs) {
            const AggOut& ao = p.aggs[k - p.nkeyparts];
            const StateDesc& sd = p.states[ao.state];
            if (ao.valid_state != 0xFF) return;
            const int w = t.state_off + sd.word;
            if (sd.kind == ST_COUNT || sd.kind == ST_SUM_I64 || sd.kind == ST_MIN_I64 || sd.kind == ST_MAX_I64) {
                if (!i64) return;
            } else if (sd.kind == ST_SUM_F64) {
                if (c.type != QDB_TYPE_F64) return;
            } else if (sd.kind == ST_SUM_I128) {
                if (c.type != QDB_TYPE_DECIMAL128) return;
                L.copy_two[k] = 1;
            } else {
                return;
            }
            if (w > 127) return;
            L.copy_word[k] = int8_t(w);
        } else {
            return;
        }
    }
    L.copy_n = L.ncols;
}

size_t AggFinalizeScratch(const GTableDev&) { return sizeof(unsigned long long); }

void AggFinalize(const AggPlan& p, const OutputPlan& out, const GTableDev& t, AggOutputCol* cols, int ncols,
                 int64_t groups, void* scratch, int* err, cudaStream_t s, bool packed) {
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
    L.row_counters = static_cast<unsigned long long*>(scratch);
    L.err = err;
    PresetValidity(p, out, L, groups, s, packed);
    PlanCopy(p, out, t, L);
    const int64_t blocks = (t.capacity + 1 + kFinChunk - 1) / kFinChunk;
    cudaMemsetAsync(L.row_counters, 0, sizeof(unsigned long long), s);
    ProfileBegin(s, "agg_finalize", t.capacity);
    if (L.copy_n) FinCopyKernel<<<int(blocks), kFinThreads, 0, s>>>(L);
    else FinWriteKernel<<<int(blocks), kFinThreads, 0, s>>>(L);
    ProfileEnd(s);
    CountLaunch(1);
}

// ---------------------------------------------------------------------------
// Batched aggregate launchers.
// ---------------------------------------------------------------------------
__global__ void AggBatchMarkKernel(const HighTask* tasks, int ntasks, int keyless) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= ntasks) return;
    const GTableDev& T = tasks[i].T;
    if (!T.wide) T.slots[T.capacity * T.slot_words + T.key_off] = 0;   // flag slot: unused
    if (keyless) T.slots[int64_t(Fmix64(0) & uint64_t(T.capacity - 1)) * T.slot_words + T.key_off] = 0;
}

void AggBatchInitTables(const AggPlan& p, const GTableDev& all, const HighTask* tasks, int ntasks,
                        cudaStream_t s) {
    AggInitTable(p, all, s);
    if (ntasks <= 0) return;
    AggBatchMarkKernel<<<(ntasks + 255) / 256, 256, 0, s>>>(tasks, ntasks, p.nkeyparts == 0 ? 1 : 0);
    CountLaunch();
}

namespace {

struct BatchFns {
    void (*update)(AggLaunch, HighBatch) = nullptr;
    void (*replay)(AggLaunch, HighBatch, const int64_t*, int64_t) = nullptr;
};

// High-cardinality programs take AggHighBatchKernel (a shared tier in front
// of each aggregate's table); low-cardinality ones AggSigQuadBatchKernel,
// whose lane-private accumulators keep a handful of groups from piling every
// row's atomics onto a few shared slots.
BatchFns FindBatchKernels(const AggPlan& P, const FastPlan& F, bool low) {
    BatchFns b;
    const std::vector<int> key = ShapeKeyOf(P, F);
    if (key.empty()) return b;
#define QDB_SHAPE_FIND(KERNEL, ...)                                                   \
    if (!b.update && ShapeMatches<__VA_ARGS__>(key) && ShapeWordsMatch<__VA_ARGS__>(F)) { \
        b.update = KERNEL<__VA_ARGS__>;                                               \
        b.replay = AggBatchReplayKernel<__VA_ARGS__>;                                 \
    }
#define QDB_SHAPE_FIND_HIGH(...) QDB_SHAPE_FIND(AggHighBatchKernel, __VA_ARGS__)
#define QDB_SHAPE_FIND_LOW(...) QDB_SHAPE_FIND(AggSigQuadBatchKernel, __VA_ARGS__)
    if (low) {
        QDB_SHAPE_LIST(QDB_SHAPE_FIND_LOW)
    } else {
        QDB_HIGH_SHAPE_LIST(QDB_SHAPE_FIND_HIGH)
    }
#undef QDB_SHAPE_FIND_LOW
#undef QDB_SHAPE_FIND_HIGH
#undef QDB_SHAPE_FIND
    return b;
}

// Shared memory of AggSigQuadBatchKernel: misc words, the kQuadSlots-slot
// tier (keys, states, group ids), then kPrivGroups groups of lane-private
// words per thread.  Sets the launch's offsets; returns the bytes.
constexpr int kQuadSlots = 64;

size_t QuadBatchLayout(AggLaunch& L) {
    const int S = kQuadSlots;
    L.off_misc = 0;
    L.off_skeys = 128;
    L.off_sst = L.off_skeys + S * 8;
    L.off_gid = L.off_sst + S * L.P.state_words * 8;
    L.off_pacc = int(Align(L.off_gid + S * 4, 16));
    return size_t(L.off_pacc) + size_t(kPrivGroups) * L.P.state_words * kQuadThreads * 8;
}

AggLaunch& BatchLaunchOf(const AggPlan& p, const FastPlan& f, int smem_slots) {
    static thread_local AggLaunch* Lp = nullptr;
    if (!Lp) Lp = new AggLaunch();
    AggLaunch& L = *Lp;
    std::memset(&L, 0, sizeof(L));
    L.P = p;
    L.F = f;
    L.smem_slots = smem_slots;
    L.smem_limit = smem_slots / 2;
    L.inline_slot = -1;
    return L;
}

// The launch's block shape: the low-cardinality kernel has a fixed one.
size_t BatchSmemOf(AggLaunch& L, bool low, int smem_slots, int& threads) {
    if (!low) return size_t(HighLayoutOf(smem_slots, L.P.state_words).bytes);
    threads = kQuadThreads;
    L.smem_slots = kQuadSlots;
    L.smem_limit = kQuadSlots / 2;
    L.priv = 1;
    return QuadBatchLayout(L);
}

}  // namespace

std::string AggBatchShapeKey(const AggPlan& p, const FastPlan& f, bool low) {
    std::string k = low ? "low:" : "high:";
    for (int v : ShapeKeyOf(p, f)) k += std::to_string(v) + ",";
    return k;
}

bool AggBatchSupported(const AggPlan& p, const FastPlan& f, bool low) {
    return p.key_words <= 1 && FindBatchKernels(p, f, low).update != nullptr;
}

int AggBatchOccupancy(const AggPlan& p, const FastPlan& f, int threads, int smem_slots, bool low) {
    EnsureDeviceInfo();
    const BatchFns fns = FindBatchKernels(p, f, low);
    if (!fns.update) return 0;
    AggLaunch& L = BatchLaunchOf(p, f, smem_slots);
    const size_t bytes = BatchSmemOf(L, low, smem_slots, threads) + 64;
    if (bytes > g_smem_optin) return 0;
    // The answer depends only on the kernel and its block shape; the driver
    // query costs microseconds on every batched dispatch, so it is kept.
    static std::mutex mu;
    static std::map<std::tuple<const void*, int, size_t>, int> seen;
    const auto key = std::make_tuple(reinterpret_cast<const void*>(fns.update), threads, bytes);
    {
        std::lock_guard<std::mutex> lk(mu);
        auto it = seen.find(key);
        if (it != seen.end()) return it->second;
    }
    SetSmem(fns.update, bytes);
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, fns.update, threads, bytes) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    std::lock_guard<std::mutex> lk(mu);
    seen[key] = n;
    return n;
}

void AggBatchUpdate(const AggPlan& p, const FastPlan& f, const HighBatch& b, int threads, int smem_slots, int grid,
                    cudaStream_t s, bool low) {
    EnsureDeviceInfo();
    const BatchFns fns = FindBatchKernels(p, f, low);
    AggLaunch& L = BatchLaunchOf(p, f, smem_slots);
    const size_t bytes = BatchSmemOf(L, low, smem_slots, threads);
    SetSmem(fns.update, bytes + 64);
    ProfileBegin(s, low ? "agg_batch_update_low" : "agg_batch_update", b.nitems);
    fns.update<<<grid, threads, bytes, s>>>(L, b);
    ProfileEnd(s);
    CountLaunch();
}

void AggBatchReplay(const AggPlan& p, const FastPlan& f, const HighBatch& b, const int64_t* pairs, int64_t n,
                    cudaStream_t s, bool low) {
    if (n <= 0) return;
    const BatchFns fns = FindBatchKernels(p, f, low);
    AggLaunch& L = BatchLaunchOf(p, f, 0);
    ProfileBegin(s, "agg_batch_replay", n);
    fns.replay<<<int((n + 255) / 256), 256, 0, s>>>(L, b, pairs, n);
    ProfileEnd(s);
    CountLaunch();
}

void AggBatchSpill(const AggPlan& p, const HighBatch& b, const uint64_t* recs, int64_t n, cudaStream_t s) {
    if (n <= 0) return;
    FastPlan f{};
    AggLaunch& L = BatchLaunchOf(p, f, 0);
    ProfileBegin(s, "agg_batch_spill", n);
    AggBatchSpillKernel<<<int((n + 255) / 256), 256, 0, s>>>(L, b, recs, n);
    ProfileEnd(s);
    CountLaunch();
}

size_t AggFinalizeBatchScratch(int64_t nblocks) { return size_t(std::max<int64_t>(nblocks, 1)) * 8; }

void AggFinalizeBatch(const AggPlan& p, const OutputPlan& out, const GTableDev& layout, const GTableDev* tables,
                      const FinBlock* blocks, int64_t nblocks, AggOutputCol* cols, int ncols, int64_t out_rows,
                      void* scratch, int* err, cudaStream_t s) {
    if (nblocks <= 0) return;
    static thread_local FinLaunch* Lp = nullptr;
    if (!Lp) Lp = new FinLaunch();
    FinLaunch& L = *Lp;
    std::memset(&L, 0, sizeof(L));
    L.P = p;
    L.O = out;
    for (int k = 0; k < ncols; ++k) L.cols[k] = cols[k];
    L.ncols = ncols;
    L.groups = out_rows;
    L.row_counters = static_cast<unsigned long long*>(scratch);
    L.err = err;
    L.tables = tables;
    L.blocks = blocks;
    PresetValidity(p, out, L, out_rows, s, true);
    PlanCopy(p, out, layout, L);
    cudaMemsetAsync(L.row_counters, 0, AggFinalizeBatchScratch(nblocks), s);
    ProfileBegin(s, "agg_finalize_batch", nblocks);
    if (L.copy_n) FinCopyKernel<<<int(nblocks), kFinThreads, 0, s>>>(L);
    else FinWriteKernel<<<int(nblocks), kFinThreads, 0, s>>>(L);
    ProfileEnd(s);
    CountLaunch(1);
}

// ---------------------------------------------------------------------------
// Aggregation without device allocation.
//
// Some embedders cannot allocate device memory while a query runs: an engine
// that hands the GPU a fixed memory budget up front and must stay inside it,
// or a process whose device allocator belongs to another runtime.  For them
// one whole aggregate (table init, fused update, finalize) runs in
// this file-scope scratch array instead of cudaMalloc'd buffers.  Every GPU
// that loads the library holds it until the process exits.  All calls share
// it and it keeps the last call's contents, so each call clears the counters
// and the table it uses; two calls whose work overlaps on the GPU (different
// streams, or different host threads) race on it and must be serialised by
// the caller.
// ---------------------------------------------------------------------------
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

namespace {

std::mutex g_noalloc_mu;
void* g_noalloc_addr[64] = {};

// Device address of the scratch array on the current device, looked up once
// per device (the host-side symbol is only a stand-in for it).
void* NoAllocScratch(std::string& err) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) {
        err = "no current CUDA device";
        return nullptr;
    }
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (!g_noalloc_addr[dev]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) {
            err = std::string("cudaGetSymbolAddress of the scratch array failed: ") + cudaGetErrorString(e);
            return nullptr;
        }
        g_noalloc_addr[dev] = p;
    }
    return g_noalloc_addr[dev];
}

}  // namespace

int64_t AggRunNoAlloc(const AggPlan& plan, const OutputPlan& out, int64_t nrows, AggOutputCol* cols, int ncols,
                      int64_t out_capacity, bool priv, cudaStream_t s, std::string& err) {
    EnsureDeviceInfo();
    unsigned char* base = static_cast<unsigned char*>(NoAllocScratch(err));
    if (!base) return -1;
    if (plan.key_words > 1) {
        err = "the no-allocation aggregate serves one-word group keys only";
        return -1;
    }
    // Scratch layout: counters | finalize block counts | spill | table.
    const int sw = plan.state_words;
    const int slot_words = (1 + sw + 1) & ~1;
    const int S = priv ? 64 : 256;
    const int64_t spill_cap = int64_t(g_sms) * S;
    const size_t counters_bytes = 256;
    const size_t spill_bytes = size_t(spill_cap) * (1 + sw) * 8;
    int64_t cap = int64_t(1) << 20;
    auto table_bytes = [&](int64_t c) { return size_t(c + 1) * slot_words * 8; };
    auto fin_bytes = [&](int64_t c) { return size_t((c + 1 + kFinChunk - 1) / kFinChunk) * 8; };
    while (cap > 1024 && counters_bytes + fin_bytes(cap) + spill_bytes + table_bytes(cap) > kNoAllocScratchBytes) {
        cap >>= 1;
    }
    if (counters_bytes + fin_bytes(cap) + spill_bytes + table_bytes(cap) > kNoAllocScratchBytes) {
        err = "aggregate state too wide for the no-allocation scratch of " +
              std::to_string(kNoAllocScratchBytes) + " bytes";
        return -1;
    }
    auto* counters = reinterpret_cast<AggCounters*>(base);
    auto* block_counts = reinterpret_cast<unsigned long long*>(base + counters_bytes);
    auto* spill = reinterpret_cast<uint64_t*>(base + counters_bytes + fin_bytes(cap));
    GTableDev t;
    t.slots = reinterpret_cast<uint64_t*>(base + counters_bytes + fin_bytes(cap) + spill_bytes);
    t.capacity = cap;
    t.slot_words = slot_words;
    t.key_off = 0;
    t.state_off = 1;
    t.wide = 0;

    cudaMemsetAsync(counters, 0, sizeof(AggCounters), s);
    AggInitTable(plan, t, s);
    int64_t groups = 0;
    if (plan.nkeyparts == 0) {
        // The keyless group exists before any row: key 0 at its home slot.
        const int64_t slot = int64_t(Fmix64(0) & uint64_t(cap - 1));
        cudaMemsetAsync(t.slots + slot * t.slot_words + t.key_off, 0, 8, s);
        groups = 1;
    }
    AggUpdateArgs a;
    a.plan = &plan;
    a.nrows = nrows;
    a.table = t;
    a.counters = counters;
    a.deferred = nullptr;   // a row that does not fit is an error here, not a replay
    a.deferred_cap = 0;
    a.spill = spill;
    a.spill_cap = spill_cap;
    a.smem_slots = S;
    a.priv = priv;
    AggUpdate(a, s);
    AggCounters hc;
    cudaMemcpyAsync(&hc, counters, sizeof(hc), cudaMemcpyDeviceToHost, s);
    if (cudaStreamSynchronize(s) != cudaSuccess) {
        err = std::string("no-allocation aggregate: ") + cudaGetErrorString(cudaGetLastError());
        return -1;
    }
    groups += int64_t(hc.new_groups);
    if (hc.deferred || hc.spilled || hc.error == DE_DEFER_FULL || hc.error == DE_SPILL_FULL) {
        err = "more groups than the no-allocation table holds (" + std::to_string(cap / 2) + " at most)";
        return -1;
    }
    if (hc.error) {
        err = "no-allocation aggregate: device error " + std::to_string(hc.error);
        return -1;
    }
    if (groups > cap / 2) {
        err = "more groups than the no-allocation table holds (" + std::to_string(cap / 2) + " at most)";
        return -1;
    }
    if (groups > out_capacity) {
        err = "output capacity " + std::to_string(out_capacity) + " is below the group count " +
              std::to_string(groups);
        return -1;
    }
    AggFinalize(plan, out, t, cols, ncols, groups, block_counts, &counters->error, s);
    int derr = 0;
    cudaMemcpyAsync(&derr, &counters->error, sizeof(int), cudaMemcpyDeviceToHost, s);
    if (cudaStreamSynchronize(s) != cudaSuccess || derr) {
        err = "no-allocation aggregate finalize failed";
        return -1;
    }
    return groups;
}

}  // namespace qdb
