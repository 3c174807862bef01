// eval.h — per-row functors of the fused operator pipeline: column loads,
// predicate atoms, sum-of-products values, the generic expression program and
// group-key packing.  Host+device so that the lowering can be unit-tested on
// the host against the oracle; the kernels instantiate them on the device.
//
// An accessor type `Acc` provides, for the current row:
//   i128 Int(int col)    — integer/decimal value (sign/zero-extended)
//   double F64(int col)  — floating value (integers converted)
//   bool Null(int col)   — validity
#pragma once

#include "plan.h"

namespace qdb {

// Exact powers of ten representable in a double.
QDB_HD inline double Pow10F(int k) {
    constexpr double t[23] = {1e0, 1e1, 1e2, 1e3, 1e4, 1e5, 1e6, 1e7, 1e8, 1e9, 1e10, 1e11,
                              1e12, 1e13, 1e14, 1e15, 1e16, 1e17, 1e18, 1e19, 1e20, 1e21, 1e22};
    double r = 1.0;
    while (k > 22) { r *= 1e22; k -= 22; }
    return r * t[k < 0 ? 0 : k];
}

QDB_HD inline i128 Pow10I(int k) {
    i128 r = 1;
    for (int j = 0; j < k; ++j) r *= 10;
    return r;
}

// Wraps to `bits` bits, sign- or zero-extending.
QDB_HD inline i128 WrapBits(i128 v, int bits, bool is_unsigned) {
    if (bits >= 128) return v;
    const u128 mask = (u128(1) << bits) - 1;
    u128 u = u128(v) & mask;
    if (!is_unsigned && ((u >> (bits - 1)) & 1)) u |= ~mask;
    return i128(u);
}

QDB_HD inline bool CmpHolds(int cmp, int c) {
    switch (cmp) {
        case AT_EQ: return c == 0;
        case AT_NE: return c != 0;
        case AT_LT: return c < 0;
        case AT_LE: return c <= 0;
        case AT_GT: return c > 0;
        default: return c >= 0;
    }
}

QDB_HD inline int Cmp128(i128 x, i128 y) { return x < y ? -1 : (x > y ? 1 : 0); }
QDB_HD inline int CmpF(double x, double y) { return x < y ? -1 : (x > y ? 1 : 0); }

QDB_HD inline double BitsToF64(int64_t b) {
    double f;
    __builtin_memcpy(&f, &b, 8);
    return f;
}

// ---------------------------------------------------------------------------
// Predicate atoms: AND over clauses of OR over atoms.
// ---------------------------------------------------------------------------
template <class Acc>
QDB_HD inline bool AtomHolds(const Atom& t, const int64_t* list, const Acc& a) {
    if (t.op == AT_IS_NULL) return a.Null(t.col);
    if (t.op == AT_IS_NOT_NULL) return !a.Null(t.col);
    if (a.Null(t.col)) return false;
    if (t.op == AT_COL_CMP) {
        if (a.Null(t.col2)) return false;
        if (t.as_f64) {
            const double x = a.F64(t.col), y = a.F64(t.col2);
            if (x != x || y != y) return t.cmp == AT_NE;
            return CmpHolds(t.cmp, CmpF(x, y));
        }
        const i128 x = a.Int(t.col) * Pow10I(t.mul), y = a.Int(t.col2) * Pow10I(t.mul2);
        return CmpHolds(t.cmp, Cmp128(x, y));
    }
    if (t.as_f64) {
        const double x = a.F64(t.col);
        if (t.op == AT_IN) {
            for (int j = 0; j < t.list_len; ++j) {
                if (BitsToF64(list[t.list_off + j]) == x) return true;
            }
            return false;
        }
        const double c0 = BitsToF64(int64_t(t.c0));
        if (x != x || c0 != c0) return t.op == AT_NE;
        if (t.op == AT_BETWEEN) {
            const double c1 = BitsToF64(int64_t(t.c1));
            return x >= c0 && x <= c1;
        }
        return CmpHolds(t.op, CmpF(x, c0));
    }
    const i128 x = t.mul ? a.Int(t.col) * Pow10I(t.mul) : a.Int(t.col);
    if (t.op == AT_IN) {
        for (int j = 0; j < t.list_len; ++j) {
            if (i128(list[t.list_off + j]) == x) return true;
        }
        return false;
    }
    if (t.op == AT_BETWEEN) return x >= t.c0 && x <= t.c1;
    return CmpHolds(t.op, Cmp128(x, t.c0));
}

template <class Acc>
QDB_HD inline bool AtomsPass(const AggPlan& p, const Acc& a) {
    uint32_t held = 0;
    for (int j = 0; j < p.natoms; ++j) {
        const Atom& t = p.atoms[j];
        if (!((held >> t.clause) & 1) && AtomHolds(t, p.list, a)) held |= 1u << t.clause;
    }
    return held == p.clause_mask;
}

// ---------------------------------------------------------------------------
// Sum-of-products values.
// ---------------------------------------------------------------------------
QDB_HD inline int Ctz32(uint32_t m) {
#if defined(__CUDA_ARCH__)
    return __ffs(int(m)) - 1;
#else
    return __builtin_ctz(m);
#endif
}

template <class Acc>
QDB_HD inline bool SopNull(const SopValue& v, const Acc& a) {
    uint32_t m = v.null_cols;
    while (m) {
        const int c = Ctz32(m);
        if (a.Null(c)) return true;
        m &= m - 1;
    }
    return false;
}

template <class Acc>
QDB_HD inline i128 FactorInt(const Factor& f, const Acc& a) {
    if (f.col == 0xFF) return i128(f.c);
    const i128 x = a.Int(f.col);
    if (f.kind == VK_I64) {
        const uint64_t r = uint64_t(f.c) + uint64_t(f.d) * uint64_t(int64_t(x));
        return i128(int64_t(r));
    }
    return i128(u128(i128(f.c)) + u128(i128(f.d)) * u128(x));
}

// A factor without an additive constant is d * x (or x): adding a zero would
// turn -0.0 into +0.0.
template <class Acc>
QDB_HD inline double FactorF64(const Factor& f, const Acc& a) {
    if (f.col == 0xFF) return f.fc;
    const double x = a.F64(f.col);
    const double dx = f.fd == 1.0 ? x : (f.fd == -1.0 ? -x : f.fd * x);
    return f.has_c ? f.fc + dx : dx;
}

template <class Acc>
QDB_HD inline i128 SopInt(const SopValue& v, const Acc& a) {
    if (v.kind == VK_I64) {
        uint64_t sum = 0;
        for (int t = 0; t < v.nterms; ++t) {
            const Term& tm = v.t[t];
            uint64_t prod = 1;
            for (int j = 0; j < tm.nf; ++j) prod *= uint64_t(int64_t(FactorInt(tm.f[j], a)));
            sum = tm.sign < 0 ? sum - prod : sum + prod;
        }
        return i128(int64_t(sum));
    }
    u128 sum = 0;
    for (int t = 0; t < v.nterms; ++t) {
        const Term& tm = v.t[t];
        u128 prod = 1;
        for (int j = 0; j < tm.nf; ++j) prod *= u128(FactorInt(tm.f[j], a));
        sum = tm.sign < 0 ? sum - prod : sum + prod;
    }
    return i128(sum);
}

template <class Acc>
QDB_HD inline double SopF64(const SopValue& v, const Acc& a) {
    double sum = 0.0;
    for (int t = 0; t < v.nterms; ++t) {
        const Term& tm = v.t[t];
        double prod = FactorF64(tm.f[0], a);
        for (int j = 1; j < tm.nf; ++j) prod = prod * FactorF64(tm.f[j], a);
        if (t == 0) sum = tm.sign < 0 ? -prod : prod;
        else sum = tm.sign < 0 ? sum - prod : sum + prod;
    }
    return sum;
}

// ---------------------------------------------------------------------------
// Generic expression program (operand-before-user nodes, one row).
// ---------------------------------------------------------------------------
struct GVal {
    i128 i;
    double f;
};

QDB_HD inline double GToF64(const GNode& n, const GVal& v) {
    if (n.dom == GD_F64) return v.f;
    return double(v.i) / Pow10F(n.scale);
}

// Integer operand aligned to `target` scale.
QDB_HD inline i128 GAtScale(const GNode& n, const GVal& v, int target) {
    if (target >= n.scale) return v.i * Pow10I(target - n.scale);
    return v.i / Pow10I(n.scale - target);
}

QDB_HD inline int GCmp(const GNode& na, const GVal& a, const GNode& nb, const GVal& b, bool& nan) {
    nan = false;
    if (na.dom == GD_F64 || nb.dom == GD_F64) {
        const double x = GToF64(na, a), y = GToF64(nb, b);
        nan = x != x || y != y;
        return CmpF(x, y);
    }
    const int s = na.scale > nb.scale ? na.scale : nb.scale;
    return Cmp128(GAtScale(na, a, s), GAtScale(nb, b, s));
}

// Evaluates nodes [0, root].  Returns false on a row error (division by
// zero); `nulls` gets one bit per node.
template <class Acc>
QDB_HD QDB_NOINLINE bool EvalGeneric(const GProg& g, int root, const int64_t* list, const Acc& acc,
                                     GVal* v, uint64_t& nulls) {
    nulls = 0;
    for (int k = 0; k <= root; ++k) {
        const GNode& n = g.nodes[k];
        GVal r{0, 0.0};
        bool isnull = false;
        const bool na = (nulls >> n.a) & 1, nb = (nulls >> n.b) & 1, nc = (nulls >> n.c) & 1;
        switch (n.op) {
            case G_COL:
                isnull = acc.Null(n.col);
                if (!isnull) {
                    if (n.dom == GD_F64) r.f = acc.F64(n.col);
                    else r.i = acc.Int(n.col);
                }
                break;
            case G_CONST:
                if (n.dom == GD_F64) r.f = BitsToF64(n.imm_lo);
                else r.i = i128((u128(uint64_t(n.imm_hi)) << 64) | uint64_t(n.imm_lo));
                break;
            case G_NULL: isnull = true; break;
            case G_ADD: case G_SUB: case G_MUL: case G_DIV: {
                if (na || nb) { isnull = true; break; }
                const GNode& A = g.nodes[n.a];
                const GNode& B = g.nodes[n.b];
                if (n.dom == GD_F64) {
                    const double x = GToF64(A, v[n.a]), y = GToF64(B, v[n.b]);
                    r.f = n.op == G_ADD ? x + y : n.op == G_SUB ? x - y : n.op == G_MUL ? x * y : x / y;
                    if (n.wrap_bits == 32) r.f = double(float(r.f));
                    break;
                }
                if (n.op == G_ADD || n.op == G_SUB) {
                    const i128 x = GAtScale(A, v[n.a], n.scale), y = GAtScale(B, v[n.b], n.scale);
                    r.i = WrapBits(n.op == G_ADD ? i128(u128(x) + u128(y)) : i128(u128(x) - u128(y)),
                                   n.wrap_bits, n.is_unsigned);
                } else if (n.op == G_MUL) {
                    i128 p = i128(u128(v[n.a].i) * u128(v[n.b].i));
                    const int extra = n.scale - A.scale - B.scale;
                    if (extra > 0) p = i128(u128(p) * u128(Pow10I(extra)));
                    r.i = WrapBits(p, n.wrap_bits, n.is_unsigned);
                } else {
                    if (v[n.b].i == 0) return false;
                    const int up = n.scale - A.scale + B.scale;
                    const i128 x = v[n.a].i * Pow10I(up > 0 ? up : 0);
                    r.i = WrapBits(x / v[n.b].i, n.wrap_bits, n.is_unsigned);
                }
                break;
            }
            case G_MOD: {
                if (na || nb) { isnull = true; break; }
                const i128 x = GAtScale(g.nodes[n.a], v[n.a], n.scale), y = GAtScale(g.nodes[n.b], v[n.b], n.scale);
                if (y == 0) return false;
                r.i = WrapBits(x % y, n.wrap_bits, n.is_unsigned);
                break;
            }
            case G_NEG: {
                if (na) { isnull = true; break; }
                if (n.dom == GD_F64) r.f = -GToF64(g.nodes[n.a], v[n.a]);
                else r.i = WrapBits(i128(u128(0) - u128(v[n.a].i)), n.wrap_bits, n.is_unsigned);
                break;
            }
            case G_CAST: {
                if (na) { isnull = true; break; }
                const GNode& A = g.nodes[n.a];
                if (n.dom == GD_F64) {
                    r.f = GToF64(A, v[n.a]);
                    if (n.wrap_bits == 32) r.f = double(float(r.f));
                } else if (A.dom == GD_F64) {
                    r.i = WrapBits(i128(int64_t(v[n.a].f)), n.wrap_bits, n.is_unsigned);
                } else {
                    r.i = WrapBits(GAtScale(A, v[n.a], n.scale), n.wrap_bits, n.is_unsigned);
                }
                break;
            }
            case G_EQ: case G_NE: case G_LT: case G_LE: case G_GT: case G_GE: {
                if (na || nb) { isnull = true; break; }
                bool nan = false;
                const int c = GCmp(g.nodes[n.a], v[n.a], g.nodes[n.b], v[n.b], nan);
                const int cmp = n.op - G_EQ;   // AT_EQ..AT_GE order
                r.i = nan ? (n.op == G_NE) : CmpHolds(cmp, c);
                break;
            }
            case G_AND: {
                const bool fa = !na && v[n.a].i == 0, fb = !nb && v[n.b].i == 0;
                if (fa || fb) r.i = 0;
                else if (na || nb) isnull = true;
                else r.i = 1;
                break;
            }
            case G_OR: {
                const bool ta = !na && v[n.a].i != 0, tb = !nb && v[n.b].i != 0;
                if (ta || tb) r.i = 1;
                else if (na || nb) isnull = true;
                else r.i = 0;
                break;
            }
            case G_NOT:
                if (na) isnull = true; else r.i = v[n.a].i ? 0 : 1;
                break;
            case G_BETWEEN: {
                if (na || nb || nc) { isnull = true; break; }
                bool n1 = false, n2 = false;
                const int c1 = GCmp(g.nodes[n.a], v[n.a], g.nodes[n.b], v[n.b], n1);
                const int c2 = GCmp(g.nodes[n.a], v[n.a], g.nodes[n.c], v[n.c], n2);
                r.i = (!n1 && !n2 && c1 >= 0 && c2 <= 0) ? 1 : 0;
                break;
            }
            case G_IN: {
                if (na) { isnull = true; break; }
                const GNode& A = g.nodes[n.a];
                bool found = false;
                for (int j = 0; j < n.list_len && !found; ++j) {
                    if (A.dom == GD_F64) found = BitsToF64(list[n.list_off + j]) == v[n.a].f;
                    else found = i128(list[n.list_off + j]) == v[n.a].i;
                }
                r.i = found;
                break;
            }
            case G_CASE: {
                const bool take = !na && v[n.a].i != 0;
                const int src = take ? n.b : n.c;
                const GNode& S = g.nodes[src];
                isnull = (nulls >> src) & 1;
                if (!isnull) {
                    if (n.dom == GD_F64) r.f = GToF64(S, v[src]);
                    else r.i = WrapBits(GAtScale(S, v[src], n.scale), n.wrap_bits, n.is_unsigned);
                }
                break;
            }
            case G_IS_NULL: r.i = na ? 1 : 0; break;
            case G_IS_NOT_NULL: r.i = na ? 0 : 1; break;
            default: return false;
        }
        v[k] = r;
        if (isnull) nulls |= 1ull << k;
    }
    return true;
}

// Canonical bits of a double key (-0 -> +0, NaN -> one quiet NaN).
QDB_HD inline uint64_t CanonF64(double f) {
    if (f == 0.0) return 0;
    if (f != f) return 0x7ff8000000000000ull;
    uint64_t b;
    __builtin_memcpy(&b, &f, 8);
    return b;
}

// Packs the group key of the current row into `words` (zeroed first).
template <class Acc>
QDB_HD inline void PackKey(const AggPlan& p, const Acc& a, const GVal* gv, uint64_t gnulls,
                           uint64_t* words) {
    for (int w = 0; w < p.key_words; ++w) words[w] = 0;
    for (int j = 0; j < p.nkeyparts; ++j) {
        const KeyPart& k = p.keys[j];
        bool null;
        i128 iv = 0;
        double fv = 0.0;
        if (k.src == KS_COLUMN) {
            null = a.Null(k.idx);
            if (!null) {
                if (k.is_float) fv = a.F64(k.idx); else iv = a.Int(k.idx);
            }
        } else if (k.src == KS_SOP) {
            const SopValue& sv = p.values[k.idx];
            null = SopNull(sv, a);
            if (!null) {
                if (k.is_float) fv = SopF64(sv, a); else iv = SopInt(sv, a);
            }
        } else {
            null = (gnulls >> k.idx) & 1;
            if (!null) {
                if (k.is_float) fv = gv[k.idx].f; else iv = gv[k.idx].i;
            }
        }
        if (null) {
            if (k.null_shift != 0xFF) words[k.null_word] |= 1ull << k.null_shift;
            continue;
        }
        if (k.is_float) {
            words[k.word] |= CanonF64(fv);
        } else if (k.bits == 128) {
            words[k.word] = uint64_t(u128(iv));
            words[k.word + 1] = uint64_t(u128(iv) >> 64);
        } else {
            const uint64_t mask = k.bits >= 64 ? ~0ull : ((1ull << k.bits) - 1);
            words[k.word] |= (uint64_t(u128(iv)) & mask) << k.shift;
        }
    }
}

// Value of key part `k` unpacked from a packed key.
QDB_HD inline i128 UnpackKeyInt(const KeyPart& k, const uint64_t* words) {
    if (k.bits == 128) return i128((u128(words[k.word + 1]) << 64) | words[k.word]);
    const uint64_t mask = k.bits >= 64 ? ~0ull : ((1ull << k.bits) - 1);
    const uint64_t raw = (words[k.word] >> k.shift) & mask;
    return WrapBits(i128(raw), k.bits, !k.is_signed);
}

QDB_HD inline bool UnpackKeyNull(const KeyPart& k, const uint64_t* words) {
    return k.null_shift != 0xFF && ((words[k.null_word] >> k.null_shift) & 1);
}

}  // namespace qdb
