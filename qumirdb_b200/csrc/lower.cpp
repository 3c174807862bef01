// lower.cpp — host lowering of operator descriptors into device plans.
//
// Result typing follows the descriptor's annotated types (the engine's
// AnnotateExprType, qdb/kernel/annotate_type.cpp:725-945) and aggregate result
// types follow AggregateResultType (qdb/plan/ops/aggregate.cpp:21-57).
#include "lower.h"

#include <algorithm>
#include <cstring>
#include <map>

namespace qdb {

namespace {

bool IsDecimalType(int t) { return t == QDB_TYPE_DECIMAL64 || t == QDB_TYPE_DECIMAL128; }
bool IsFloatType(int t) { return t == QDB_TYPE_F32 || t == QDB_TYPE_F64; }

int Arity(int op) {
    switch (op) {
        case QDB_EXPR_COLUMN: case QDB_EXPR_CONST: case QDB_EXPR_NULL: return 0;
        case QDB_EXPR_NEG: case QDB_EXPR_CAST: case QDB_EXPR_NOT: case QDB_EXPR_IN_LIST:
        case QDB_EXPR_IS_NULL: case QDB_EXPR_IS_NOT_NULL: return 1;
        case QDB_EXPR_BETWEEN: case QDB_EXPR_CASE: return 3;
        default: return 2;
    }
}

int ScaleOf(const qdb_expr& n) { return IsDecimalType(n.type) ? n.scale : 0; }

i128 ConstInt(const qdb_expr& n) {
    if (n.type == QDB_TYPE_DECIMAL128) return i128((u128(uint64_t(n.imm_hi)) << 64) | uint64_t(n.imm_lo));
    return i128(n.imm_lo);
}

double ConstF64(const qdb_expr& n) {
    if (IsFloatType(n.type)) {
        double f;
        std::memcpy(&f, &n.imm_lo, 8);
        return f;
    }
    double p = 1.0;
    for (int j = 0; j < ScaleOf(n); ++j) p *= 10.0;
    return double(ConstInt(n)) / p;
}

int64_t F64Bits(double f) {
    int64_t b;
    std::memcpy(&b, &f, 8);
    return b;
}

bool FitsI64(i128 v) { return v >= i128(INT64_MIN) && v <= i128(INT64_MAX); }

i128 P10(int k) {
    i128 r = 1;
    for (int j = 0; j < k; ++j) r *= 10;
    return r;
}

class Lowerer {
public:
    Lowerer(const qdb_column_type* cols, int ncols, const qdb_expr* nodes, int nnodes, AggPlan& plan,
            ColumnMap& map)
        : cols_(cols), ncols_(ncols), nodes_(nodes), nnodes_(nnodes), plan_(plan), map_(map) {
        map_.slot_of.assign(ncols, -1);
        map_.input_of.clear();
    }

    const qdb_expr& N(int k) const {
        if (k < 0 || k >= nnodes_) throw LowerError("expression node index out of range");
        return nodes_[k];
    }

    void CheckTree(int root) const {
        const qdb_expr& n = N(root);
        for (int j = 0; j < Arity(n.op); ++j) {
            if (n.args[j] < 0 || n.args[j] >= root) throw LowerError("operand must precede its user");
            CheckTree(n.args[j]);
        }
        if (n.op == QDB_EXPR_COLUMN && (n.column < 0 || n.column >= ncols_)) {
            throw LowerError("column index out of range");
        }
    }

    int Slot(int input) {
        if (input < 0 || input >= ncols_) throw LowerError("column index out of range");
        if (map_.slot_of[input] >= 0) return map_.slot_of[input];
        const int slot = int(map_.input_of.size());
        if (slot >= kMaxCols) throw LowerError("too many input columns for one device plan");
        map_.slot_of[input] = slot;
        map_.input_of.push_back(input);
        const TypeInfo ti = InfoOf(cols_[input].type);
        ColDesc& cd = plan_.cols[slot];
        std::memset(&cd, 0, sizeof(cd));
        cd.width = ti.width;
        cd.kind = ti.load;
        cd.nullable = cols_[input].nullable ? 1 : 0;
        cd.scale = IsDecimalType(cols_[input].type) ? cols_[input].scale : 0;
        plan_.ncols = int32_t(map_.input_of.size());
        return slot;
    }

    // ---- predicates ----------------------------------------------------
    bool TryAtoms(int root) {
        std::vector<std::vector<int>> clauses;
        if (!CollectClauses(root, clauses)) return false;
        if (int(clauses.size()) > kMaxClauses) return false;
        std::vector<Atom> atoms;
        std::vector<int64_t> list(plan_.list, plan_.list + list_used_);
        int list_used = list_used_;
        for (size_t c = 0; c < clauses.size(); ++c) {
            for (int leaf : clauses[c]) {
                Atom a;
                std::memset(&a, 0, sizeof(a));
                if (!MakeAtom(leaf, a, list, list_used)) return false;
                a.clause = uint8_t(c);
                atoms.push_back(a);
            }
        }
        if (int(atoms.size()) > kMaxAtoms) return false;
        // Commit (slots were already assigned by MakeAtom; harmless if unused).
        plan_.natoms = int32_t(atoms.size());
        for (size_t j = 0; j < atoms.size(); ++j) plan_.atoms[j] = atoms[j];
        for (int j = list_used_; j < list_used; ++j) plan_.list[j] = list[j];
        list_used_ = list_used;
        plan_.clause_mask = clauses.size() >= 32 ? ~0u : ((1u << clauses.size()) - 1);
        return true;
    }

    // ---- values: sums of products ------------------------------------------
    struct FBuild {
        Factor f;
        int scale;
    };
    struct TBuild {
        std::vector<FBuild> f;
        int sign;
    };

    static int KindOfType(int t) {
        switch (t) {
            case QDB_TYPE_I64: case QDB_TYPE_DECIMAL64: return VK_I64;
            case QDB_TYPE_DECIMAL128: return VK_I128;
            case QDB_TYPE_F64: return VK_F64;
            default: return -1;
        }
    }

    // A value kind for a bare column: narrower signed ints widen exactly.
    static int KindForColumn(int t) {
        switch (t) {
            case QDB_TYPE_I8: case QDB_TYPE_I16: case QDB_TYPE_I32: case QDB_TYPE_I64:
            case QDB_TYPE_U8: case QDB_TYPE_U16: case QDB_TYPE_U32: case QDB_TYPE_DATE32:
            case QDB_TYPE_DECIMAL64: case QDB_TYPE_CHAR1: return VK_I64;
            case QDB_TYPE_DECIMAL128: return VK_I128;
            case QDB_TYPE_F32: case QDB_TYPE_F64: return VK_F64;
            default: return -1;
        }
    }

    // Returns the value index, or -1 when the tree needs the generic program.
    int TrySop(int node) {
        if (plan_.nvalues >= kMaxValues) return -1;
        const qdb_expr& n = N(node);
        int kind = KindOfType(n.type);
        if (n.op == QDB_EXPR_COLUMN) kind = KindForColumn(n.type);
        if (kind < 0) return -1;
        std::vector<TBuild> terms;
        uint32_t null_cols = 0;
        if (!MatchSum(node, +1, kind, ScaleOf(n), terms, null_cols)) return -1;
        if (int(terms.size()) > kMaxTerms) return -1;
        SopValue v;
        std::memset(&v, 0, sizeof(v));
        v.kind = uint8_t(kind);
        v.nterms = uint8_t(terms.size());
        v.null_cols = uint16_t(null_cols);
        for (size_t t = 0; t < terms.size(); ++t) {
            if (int(terms[t].f.size()) > kMaxFactors) return -1;
            v.t[t].nf = uint8_t(terms[t].f.size());
            v.t[t].sign = int8_t(terms[t].sign);
            for (size_t j = 0; j < terms[t].f.size(); ++j) v.t[t].f[j] = terms[t].f[j].f;
        }
        plan_.values[plan_.nvalues] = v;
        return plan_.nvalues++;
    }

    // ---- generic program -------------------------------------------------
    int Generic(int node) {
        auto it = gmap_.find(node);
        if (it != gmap_.end()) return it->second;
        const qdb_expr& n = N(node);
        GNode g;
        std::memset(&g, 0, sizeof(g));
        int a = 0, b = 0, c = 0;
        const int ar = Arity(n.op);
        if (ar > 0) a = Generic(n.args[0]);
        if (ar > 1) b = Generic(n.args[1]);
        if (ar > 2) c = Generic(n.args[2]);
        if (plan_.prog.n >= kMaxGNodes) throw LowerError("expression too large for the device program");
        static const uint8_t opmap[] = {0, G_COL, G_CONST, G_NULL, G_ADD, G_SUB, G_MUL, G_DIV, G_NEG,
                                        G_CAST, G_EQ, G_NE, G_LT, G_LE, G_GT, G_GE, G_AND, G_OR,
                                        G_NOT, G_BETWEEN, G_IN, G_CASE, G_IS_NULL, G_IS_NOT_NULL, G_MOD};
        if (n.op < 1 || n.op > QDB_EXPR_MOD) throw LowerError("unknown expression op");
        g.op = opmap[n.op];
        const int t = n.type;
        const bool boolean = t == QDB_TYPE_BOOL || (n.op >= QDB_EXPR_EQ && n.op <= QDB_EXPR_NOT) ||
                             n.op == QDB_EXPR_BETWEEN || n.op == QDB_EXPR_IN_LIST ||
                             n.op == QDB_EXPR_IS_NULL || n.op == QDB_EXPR_IS_NOT_NULL;
        if (boolean) {
            g.dom = GD_BOOL;
            g.wrap_bits = 8;
        } else if (t == QDB_TYPE_INVALID && n.op == QDB_EXPR_NULL) {
            g.dom = GD_INT;
            g.wrap_bits = 64;
        } else {
            const TypeInfo ti = InfoOf(t);
            g.dom = ti.dom;
            g.wrap_bits = ti.wrap_bits;
            g.is_unsigned = ti.is_unsigned;
        }
        g.scale = int16_t(ScaleOf(n));
        g.a = uint8_t(a);
        g.b = uint8_t(b);
        g.c = uint8_t(c);
        if (n.op == QDB_EXPR_COLUMN) {
            g.col = uint8_t(Slot(n.column));
            // A column node carries its column's own scale and domain.
            const TypeInfo ti = InfoOf(cols_[n.column].type);
            g.dom = ti.dom;
            g.scale = int16_t(IsDecimalType(cols_[n.column].type) ? cols_[n.column].scale : 0);
        }
        if (n.op == QDB_EXPR_CONST) {
            g.imm_lo = n.imm_lo;
            g.imm_hi = n.type == QDB_TYPE_DECIMAL128 ? n.imm_hi : (n.imm_lo < 0 ? -1 : 0);
        }
        if (n.op == QDB_EXPR_IN_LIST) {
            if (list_used_ + n.list_len > kMaxList) throw LowerError("IN list too long for the device plan");
            g.list_off = uint8_t(list_used_);
            g.list_len = uint8_t(n.list_len);
            for (int j = 0; j < n.list_len; ++j) plan_.list[list_used_++] = n.list[j];
        }
        const int idx = plan_.prog.n++;
        plan_.prog.nodes[idx] = g;
        gmap_[node] = idx;
        plan_.generic_root = std::max(plan_.generic_root, idx);
        return idx;
    }

    int list_used() const { return list_used_; }

private:
    bool IsColumnLeaf(int node) const {
        const qdb_expr& n = N(node);
        return n.op == QDB_EXPR_COLUMN;
    }

    bool CollectClauses(int node, std::vector<std::vector<int>>& clauses) {
        const qdb_expr& n = N(node);
        if (n.op == QDB_EXPR_AND) {
            return CollectClauses(n.args[0], clauses) && CollectClauses(n.args[1], clauses);
        }
        std::vector<int> atoms;
        if (!CollectOr(node, atoms)) return false;
        clauses.push_back(atoms);
        return true;
    }

    bool CollectOr(int node, std::vector<int>& atoms) {
        const qdb_expr& n = N(node);
        if (n.op == QDB_EXPR_OR) return CollectOr(n.args[0], atoms) && CollectOr(n.args[1], atoms);
        atoms.push_back(node);
        return true;
    }

    static uint8_t FlipCmp(int op) {
        switch (op) {
            case QDB_EXPR_LT: return AT_GT;
            case QDB_EXPR_LE: return AT_GE;
            case QDB_EXPR_GT: return AT_LT;
            case QDB_EXPR_GE: return AT_LE;
            case QDB_EXPR_EQ: return AT_EQ;
            default: return AT_NE;
        }
    }

    static uint8_t CmpOf(int op) { return uint8_t(op - QDB_EXPR_EQ); }

    bool MakeAtom(int node, Atom& a, std::vector<int64_t>& list, int& list_used) {
        const qdb_expr& n = N(node);
        a.col2 = 0xFF;
        if (n.op == QDB_EXPR_IS_NULL || n.op == QDB_EXPR_IS_NOT_NULL) {
            if (!IsColumnLeaf(n.args[0])) return false;
            a.op = n.op == QDB_EXPR_IS_NULL ? AT_IS_NULL : AT_IS_NOT_NULL;
            a.col = uint8_t(Slot(N(n.args[0]).column));
            return true;
        }
        if (n.op >= QDB_EXPR_EQ && n.op <= QDB_EXPR_GE) {
            int cn = n.args[0], kn = n.args[1];
            uint8_t op = CmpOf(n.op);
            if (N(cn).op == QDB_EXPR_CONST && IsColumnLeaf(kn)) {
                std::swap(cn, kn);
                op = FlipCmp(n.op);
            }
            if (!IsColumnLeaf(cn)) return false;
            const qdb_expr& col = N(cn);
            const qdb_expr& k = N(kn);
            if (col.type == QDB_TYPE_BOOL || k.type == QDB_TYPE_BOOL) return false;
            a.col = uint8_t(Slot(col.column));
            if (k.op == QDB_EXPR_COLUMN) {
                if (k.type == QDB_TYPE_BOOL) return false;
                a.op = AT_COL_CMP;
                a.cmp = CmpOf(n.op);
                a.col2 = uint8_t(Slot(k.column));
                a.as_f64 = IsFloatType(col.type) || IsFloatType(k.type);
                const int s = std::max(ScaleOf(col), ScaleOf(k));
                a.mul = s - ScaleOf(col);
                a.mul2 = s - ScaleOf(k);
                return true;
            }
            if (k.op != QDB_EXPR_CONST) return false;
            a.op = op;
            a.as_f64 = IsFloatType(col.type) || IsFloatType(k.type);
            if (a.as_f64) {
                a.c0 = i128(F64Bits(ConstF64(k)));
                return true;
            }
            const int s = std::max(ScaleOf(col), ScaleOf(k));
            a.mul = s - ScaleOf(col);
            a.c0 = ConstInt(k) * P10(s - ScaleOf(k));
            return true;
        }
        if (n.op == QDB_EXPR_BETWEEN) {
            if (!IsColumnLeaf(n.args[0])) return false;
            const qdb_expr& col = N(n.args[0]);
            const qdb_expr& lo = N(n.args[1]);
            const qdb_expr& hi = N(n.args[2]);
            if (lo.op != QDB_EXPR_CONST || hi.op != QDB_EXPR_CONST || col.type == QDB_TYPE_BOOL) return false;
            a.op = AT_BETWEEN;
            a.col = uint8_t(Slot(col.column));
            a.as_f64 = IsFloatType(col.type) || IsFloatType(lo.type) || IsFloatType(hi.type);
            if (a.as_f64) {
                a.c0 = i128(F64Bits(ConstF64(lo)));
                a.c1 = i128(F64Bits(ConstF64(hi)));
                return true;
            }
            const int s = std::max({ScaleOf(col), ScaleOf(lo), ScaleOf(hi)});
            a.mul = s - ScaleOf(col);
            a.c0 = ConstInt(lo) * P10(s - ScaleOf(lo));
            a.c1 = ConstInt(hi) * P10(s - ScaleOf(hi));
            return true;
        }
        if (n.op == QDB_EXPR_IN_LIST) {
            if (!IsColumnLeaf(n.args[0])) return false;
            const qdb_expr& col = N(n.args[0]);
            if (col.type == QDB_TYPE_BOOL || col.type == QDB_TYPE_DECIMAL128) return false;
            if (list_used + n.list_len > kMaxList || n.list_len > 255) return false;
            a.op = AT_IN;
            a.col = uint8_t(Slot(col.column));
            a.as_f64 = IsFloatType(col.type);
            a.list_off = uint8_t(list_used);
            a.list_len = uint8_t(n.list_len);
            if (int(list.size()) < list_used + n.list_len) list.resize(list_used + n.list_len);
            for (int j = 0; j < n.list_len; ++j) list[list_used + j] = n.list[j];
            list_used += n.list_len;
            return true;
        }
        return false;
    }

    bool MatchSum(int node, int sign, int kind, int scale, std::vector<TBuild>& terms, uint32_t& nulls) {
        const qdb_expr& n = N(node);
        if ((n.op == QDB_EXPR_ADD || n.op == QDB_EXPR_SUB) && KindOfType(n.type) == kind &&
            ScaleOf(n) == scale) {
            if (kind == VK_F64) {
                // Left-deep only: ((p1 + p2) - p3) is summed in the tree's
                // order; a sum on the right would round differently.
                if (sign < 0) return false;
                if (!MatchSum(n.args[0], +1, kind, scale, terms, nulls)) return false;
                TBuild t;
                t.sign = n.op == QDB_EXPR_SUB ? -1 : +1;
                int ts = 0;
                if (!MatchProduct(n.args[1], kind, t, ts, nulls)) return false;
                terms.push_back(t);
                return true;
            }
            if (!MatchSum(n.args[0], sign, kind, scale, terms, nulls)) return false;
            return MatchSum(n.args[1], n.op == QDB_EXPR_SUB ? -sign : sign, kind, scale, terms, nulls);
        }
        TBuild t;
        t.sign = sign;
        int ts = 0;
        if (!MatchProduct(node, kind, t, ts, nulls)) return false;
        if (kind != VK_F64 && ts != scale) {
            if (ts > scale || scale - ts > 18) return false;
            FBuild fb;
            std::memset(&fb.f, 0, sizeof(fb.f));
            fb.f.col = 0xFF;
            fb.f.kind = uint8_t(kind);
            fb.f.c = int64_t(P10(scale - ts));
            fb.scale = 0;
            t.f.push_back(fb);
        }
        if (kind == VK_F64 && sign < 0) return false;   // -(product) first: not the tree's order
        terms.push_back(t);
        return true;
    }

    bool MatchProduct(int node, int kind, TBuild& t, int& scale, uint32_t& nulls) {
        const qdb_expr& n = N(node);
        if (n.op == QDB_EXPR_MUL && KindOfType(n.type) == kind) {
            if (kind == VK_F64) {
                int ls = 0;
                if (!MatchProduct(n.args[0], kind, t, ls, nulls)) return false;
                FBuild fb;
                if (!MatchFactor(n.args[1], kind, fb, nulls)) return false;
                t.f.push_back(fb);
                scale = 0;
                return true;
            }
            int ls = 0, rs = 0;
            if (!MatchProduct(n.args[0], kind, t, ls, nulls)) return false;
            if (!MatchProduct(n.args[1], kind, t, rs, nulls)) return false;
            if (ls + rs != ScaleOf(n)) return false;
            scale = ls + rs;
            return true;
        }
        FBuild fb;
        if (!MatchFactor(node, kind, fb, nulls)) return false;
        t.f.push_back(fb);
        scale = fb.scale;
        return true;
    }

    // Column leaf usable as x in a factor of kind `kind`; returns its scale.
    bool LeafColumn(int node, int kind, int& slot, int& scale, int64_t& mul, uint32_t& nulls) {
        const qdb_expr& n = N(node);
        mul = 1;
        if (n.op == QDB_EXPR_COLUMN) {
            if (n.type == QDB_TYPE_BOOL) return false;
            if (kind != VK_F64 && IsFloatType(n.type)) return false;
            if (kind == VK_I64 && (n.type == QDB_TYPE_DECIMAL128 || n.type == QDB_TYPE_U64)) return false;
            slot = Slot(n.column);
            scale = kind == VK_F64 ? 0 : ScaleOf(n);
            if (cols_[n.column].nullable) nulls |= 1u << slot;
            return true;
        }
        if (n.op == QDB_EXPR_CAST && N(n.args[0]).op == QDB_EXPR_COLUMN) {
            const qdb_expr& c = N(n.args[0]);
            if (c.type == QDB_TYPE_BOOL || c.type == QDB_TYPE_U64) return false;
            if (kind == VK_F64) {
                if (n.type != QDB_TYPE_F64) return false;
                slot = Slot(c.column);
                scale = 0;
                if (cols_[c.column].nullable) nulls |= 1u << slot;
                return true;
            }
            if (IsFloatType(c.type) || IsFloatType(n.type)) return false;
            if (KindOfType(n.type) != kind && !(kind == VK_I128 && KindOfType(n.type) == VK_I64)) return false;
            if (kind == VK_I64 && c.type == QDB_TYPE_DECIMAL128) return false;
            const int up = ScaleOf(n) - ScaleOf(c);
            if (up < 0 || up > 18) return false;
            slot = Slot(c.column);
            scale = ScaleOf(n);
            mul = int64_t(P10(up));
            if (cols_[c.column].nullable) nulls |= 1u << slot;
            return true;
        }
        return false;
    }

    bool MatchFactor(int node, int kind, FBuild& fb, uint32_t& nulls) {
        std::memset(&fb.f, 0, sizeof(fb.f));
        fb.f.kind = uint8_t(kind);
        const qdb_expr& n = N(node);
        int slot = 0, sc = 0;
        int64_t mul = 1;
        if (n.op == QDB_EXPR_CONST) {
            fb.f.col = 0xFF;
            if (kind == VK_F64) {
                fb.f.fc = ConstF64(n);
                fb.scale = 0;
                return true;
            }
            if (IsFloatType(n.type)) return false;
            const i128 v = ConstInt(n);
            if (!FitsI64(v)) return false;
            fb.f.c = int64_t(v);
            fb.scale = ScaleOf(n);
            return true;
        }
        if (LeafColumn(node, kind, slot, sc, mul, nulls)) {
            fb.f.col = uint8_t(slot);
            fb.f.c = 0;
            fb.f.d = mul;
            fb.f.fd = 1.0;
            fb.scale = sc;
            return true;
        }
        // NEG(x), c + x, x + c, c - x, x - c, c * x, x * c in the node's own kind.
        const int fk = KindOfType(n.type);
        if (fk < 0 || (kind != VK_F64 && fk == VK_F64) || (kind == VK_F64 && fk != VK_F64) ||
            (kind == VK_I64 && fk == VK_I128)) {
            return false;
        }
        const int ns = ScaleOf(n);
        if (n.op == QDB_EXPR_NEG) {
            if (!LeafColumn(n.args[0], fk, slot, sc, mul, nulls)) return false;
            if (fk != VK_F64 && sc != ns) return false;
            fb.f.col = uint8_t(slot);
            fb.f.kind = uint8_t(fk);
            fb.f.d = -mul;
            fb.f.fd = -1.0;
            fb.scale = ns;
            return true;
        }
        if (n.op == QDB_EXPR_ADD || n.op == QDB_EXPR_SUB || n.op == QDB_EXPR_MUL) {
            int cn = n.args[0], xn = n.args[1];
            bool const_left = true;
            if (N(cn).op != QDB_EXPR_CONST) {
                std::swap(cn, xn);
                const_left = false;
            }
            if (N(cn).op != QDB_EXPR_CONST) return false;
            if (!LeafColumn(xn, fk, slot, sc, mul, nulls)) return false;
            const qdb_expr& k = N(cn);
            fb.f.col = uint8_t(slot);
            fb.f.kind = uint8_t(fk);
            if (fk == VK_F64) {
                const double kv = ConstF64(k);
                if (n.op == QDB_EXPR_MUL) {
                    fb.f.fd = kv;   // c * x and x * c round identically
                } else {
                    fb.f.has_c = 1;
                    if (n.op == QDB_EXPR_ADD) { fb.f.fc = kv; fb.f.fd = 1.0; }
                    else if (const_left) { fb.f.fc = kv; fb.f.fd = -1.0; }
                    else { fb.f.fc = -kv; fb.f.fd = 1.0; }
                }
                fb.scale = 0;
                return true;
            }
            if (IsFloatType(k.type)) return false;
            const i128 kv = ConstInt(k);
            if (n.op == QDB_EXPR_MUL) {
                if (sc + ScaleOf(k) != ns || !FitsI64(kv * mul)) return false;
                fb.f.d = int64_t(kv * mul);
                fb.scale = ns;
                return true;
            }
            // +/-: both operands at the node's scale.
            if (ns < sc || ns < ScaleOf(k) || ns - sc > 18 || ns - ScaleOf(k) > 18) return false;
            const i128 cx = kv * P10(ns - ScaleOf(k));
            const i128 dx = i128(mul) * P10(ns - sc);
            if (!FitsI64(cx) || !FitsI64(dx)) return false;
            fb.f.has_c = 1;
            if (n.op == QDB_EXPR_ADD) { fb.f.c = int64_t(cx); fb.f.d = int64_t(dx); }
            else if (const_left) { fb.f.c = int64_t(cx); fb.f.d = -int64_t(dx); }
            else { fb.f.c = -int64_t(cx); fb.f.d = int64_t(dx); }
            fb.scale = ns;
            return true;
        }
        return false;
    }

    const qdb_column_type* cols_;
    int ncols_;
    const qdb_expr* nodes_;
    int nnodes_;
    AggPlan& plan_;
    ColumnMap& map_;
    std::map<int, int> gmap_;
    int list_used_ = 0;
};

void InitPlan(AggPlan& p) {
    std::memset(&p, 0, sizeof(p));
    p.filter_node = -1;
    p.generic_root = -1;
    p.key_null_word = -1;
    p.probe_cols = -1;
}

void LowerPredicate(Lowerer& L, AggPlan& p, int root) {
    if (root < 0) return;
    L.CheckTree(root);
    if (L.TryAtoms(root)) {
        p.filter_kind = 1;
        return;
    }
    p.natoms = 0;
    p.filter_kind = 2;
    p.filter_node = L.Generic(root);
}

// Value source of an expression: fast functor or generic node.
void LowerValue(Lowerer& L, int node, uint8_t& src, uint8_t& idx, bool& generic) {
    L.CheckTree(node);
    const int v = L.TrySop(node);
    if (v >= 0) {
        src = VS_SOP;
        idx = uint8_t(v);
        return;
    }
    src = VS_GENERIC;
    idx = uint8_t(L.Generic(node));
    generic = true;
}

bool ArgNullable(const qdb_aggregate_spec& s, int node) {
    const qdb_expr& n = s.nodes[node];
    if (n.op == QDB_EXPR_COLUMN) return s.columns[n.column].nullable != 0;
    if (n.op == QDB_EXPR_CONST) return false;
    if (n.op == QDB_EXPR_NULL) return true;
    bool any = false;
    for (int j = 0; j < Arity(n.op); ++j) any = any || ArgNullable(s, n.args[j]);
    return any;
}

}  // namespace

TypeInfo InfoOf(int type) {
    switch (type) {
        case QDB_TYPE_BOOL: return {LK_BOOLBIT, 0, GD_BOOL, 8, 1, 8};
        case QDB_TYPE_I8: return {LK_SIGNED, 1, GD_INT, 8, 0, 8};
        case QDB_TYPE_I16: return {LK_SIGNED, 2, GD_INT, 16, 0, 16};
        case QDB_TYPE_I32: return {LK_SIGNED, 4, GD_INT, 32, 0, 32};
        case QDB_TYPE_I64: return {LK_SIGNED, 8, GD_INT, 64, 0, 64};
        case QDB_TYPE_U8: return {LK_UNSIGNED, 1, GD_INT, 8, 1, 8};
        case QDB_TYPE_U16: return {LK_UNSIGNED, 2, GD_INT, 16, 1, 16};
        case QDB_TYPE_U32: return {LK_UNSIGNED, 4, GD_INT, 32, 1, 32};
        case QDB_TYPE_U64: return {LK_UNSIGNED, 8, GD_INT, 64, 1, 64};
        case QDB_TYPE_F32: return {LK_F32, 4, GD_F64, 32, 0, 64};
        case QDB_TYPE_F64: return {LK_F64, 8, GD_F64, 64, 0, 64};
        case QDB_TYPE_DATE32: return {LK_SIGNED, 4, GD_INT, 32, 0, 32};
        case QDB_TYPE_DECIMAL64: return {LK_SIGNED, 8, GD_INT, 64, 0, 64};
        case QDB_TYPE_DECIMAL128: return {LK_SIGNED, 16, GD_INT, 128, 0, 128};
        case QDB_TYPE_CHAR1: return {LK_UNSIGNED, 1, GD_INT, 8, 1, 8};
    }
    throw LowerError("unsupported column type " + std::to_string(type));
}

int StorageWidth(int type) {
    if (type == QDB_TYPE_BOOL) return 1;
    return InfoOf(type).width;
}

AggLowering LowerAggregate(const qdb_aggregate_spec& s, int probe_cols, const std::vector<int>& first_inputs) {
    AggLowering out;
    AggPlan& p = out.plan;
    InitPlan(p);
    p.probe_cols = probe_cols;
    if (s.n_columns < 0 || (s.n_columns > 0 && !s.columns)) throw LowerError("bad input schema");
    for (int c = 0; c < s.n_columns; ++c) InfoOf(s.columns[c].type);
    Lowerer L(s.columns, s.n_columns, s.nodes, s.n_nodes, p, out.cols);
    for (int c : first_inputs) L.Slot(c);

    LowerPredicate(L, p, s.filter);

    // Keys.
    if (s.n_keys > kMaxKeyParts) throw LowerError("too many group keys for the device table");
    int word = 0, shift = 0;
    std::vector<int> nullable_parts;
    for (int j = 0; j < s.n_keys; ++j) {
        L.CheckTree(s.keys[j]);
        const qdb_expr& kn = s.nodes[s.keys[j]];
        KeyPart& k = p.keys[j];
        std::memset(&k, 0, sizeof(k));
        if (kn.type == QDB_TYPE_BOOL && kn.op != QDB_EXPR_COLUMN) throw LowerError("boolean expression keys are not served");
        const TypeInfo ti = InfoOf(kn.type);
        if (kn.op == QDB_EXPR_COLUMN) {
            k.src = KS_COLUMN;
            k.idx = uint8_t(L.Slot(kn.column));
        } else {
            uint8_t src = 0, idx = 0;
            bool generic = false;
            LowerValue(L, s.keys[j], src, idx, generic);
            out.any_generic = out.any_generic || generic;
            k.src = src == VS_SOP ? KS_SOP : KS_GENERIC;
            k.idx = idx;
        }
        k.bits = ti.key_bits;
        k.is_float = ti.dom == GD_F64;
        k.is_signed = !ti.is_unsigned && ti.dom == GD_INT;
        k.out_type = uint8_t(kn.type);
        k.out_scale = int16_t(ScaleOf(kn));
        k.null_shift = 0xFF;
        if (k.bits == 128) {
            if (shift) { ++word; shift = 0; }
            k.word = uint8_t(word);
            word += 2;
        } else {
            if (shift + k.bits > 64) { ++word; shift = 0; }
            k.word = uint8_t(word);
            k.shift = uint8_t(shift);
            shift += k.bits;
            if (shift == 64) { ++word; shift = 0; }
        }
        const bool nullable = kn.op == QDB_EXPR_COLUMN ? s.columns[kn.column].nullable != 0
                                                       : ArgNullable(s, s.keys[j]);
        if (nullable) nullable_parts.push_back(j);
    }
    for (int j : nullable_parts) {
        if (shift + 1 > 64) { ++word; shift = 0; }
        p.keys[j].null_word = uint8_t(word);
        p.keys[j].null_shift = uint8_t(shift);
        p.key_null_word = word;
        ++shift;
    }
    if (shift) ++word;
    p.nkeyparts = s.n_keys;
    p.key_words = std::max(1, word);
    if (p.key_words > kMaxKeyWords) throw LowerError("group key too wide for the device table");
    int used_bits = 0;
    for (int j = 0; j < s.n_keys; ++j) used_bits += p.keys[j].bits;
    used_bits += int(nullable_parts.size());
    p.key_full64 = (p.key_words == 1 && used_bits >= 64) ? 1 : 0;

    // Aggregates and their state words.
    if (s.n_aggs > kMaxAggs) throw LowerError("too many aggregates for one device table");
    int words = 0;
    auto add_state = [&](uint8_t kind, uint8_t src, uint8_t idx) -> int {
        // A COUNT over a value that is never NULL is COUNT(*): share one word.
        if (kind == ST_COUNT && src == VS_SOP && p.values[idx].null_cols == 0) {
            src = VS_NONE;
            idx = 0;
        }
        for (int s = 0; s < p.nstates; ++s) {
            const StateDesc& o = p.states[s];
            if (o.kind == kind && o.src == src && o.idx == idx && (kind == ST_COUNT || src != VS_NONE)) return s;
        }
        if (p.nstates >= kMaxStates) throw LowerError("too many aggregate states");
        StateDesc& st = p.states[p.nstates];
        st.kind = kind;
        st.src = src;
        st.idx = idx;
        st.word = uint8_t(words);
        words += kind == ST_SUM_I128 ? 2 : 1;
        return p.nstates++;
    };
    for (int j = 0; j < s.n_aggs; ++j) {
        const qdb_agg_item& a = s.aggs[j];
        AggOut& ao = p.aggs[j];
        std::memset(&ao, 0, sizeof(ao));
        ao.func = uint8_t(a.func);
        ao.valid_state = 0xFF;
        if (a.func == QDB_AGG_COUNT_STAR) {
            ao.state = uint8_t(add_state(ST_COUNT, VS_NONE, 0));
            ao.out_type = QDB_TYPE_I64;
            out.row_types.push_back(QDB_TYPE_I64);
            out.row_scales.push_back(0);
            continue;
        }
        if (a.arg < 0 || a.arg >= s.n_nodes) throw LowerError("aggregate argument out of range");
        const qdb_expr& arg = s.nodes[a.arg];
        uint8_t src = 0, idx = 0;
        bool generic = false;
        LowerValue(L, a.arg, src, idx, generic);
        out.any_generic = out.any_generic || generic;
        const bool nullable = ArgNullable(s, a.arg);
        if (a.func == QDB_AGG_COUNT) {
            ao.state = uint8_t(add_state(ST_COUNT, src, idx));
            ao.out_type = QDB_TYPE_I64;
        } else {
            const bool fl = IsFloatType(arg.type);
            const bool dec = IsDecimalType(arg.type);
            if (arg.type == QDB_TYPE_BOOL) throw LowerError("aggregates over booleans are not served");
            if (a.func == QDB_AGG_SUM) {
                if (arg.type == QDB_TYPE_DATE32) throw LowerError("function sum(DATE) does not exist");
                if (arg.type == QDB_TYPE_U64) throw LowerError("sum over u64 is not served");
                const uint8_t kind = fl ? ST_SUM_F64 : (dec ? ST_SUM_I128 : ST_SUM_I64);
                ao.state = uint8_t(add_state(kind, src, idx));
                ao.out_type = fl ? QDB_TYPE_F64 : (dec ? QDB_TYPE_DECIMAL128 : QDB_TYPE_I64);
                ao.out_scale = int16_t(dec ? arg.scale : 0);
            } else {
                if (arg.type == QDB_TYPE_DECIMAL128 || arg.type == QDB_TYPE_U64) {
                    throw LowerError("min/max over DECIMAL128 or u64 is not served");
                }
                const bool mn = a.func == QDB_AGG_MIN;
                const uint8_t kind = fl ? (mn ? ST_MIN_F64 : ST_MAX_F64) : (mn ? ST_MIN_I64 : ST_MAX_I64);
                ao.state = uint8_t(add_state(kind, src, idx));
                ao.out_type = fl ? QDB_TYPE_F64 : (dec ? arg.type : QDB_TYPE_I64);
                ao.out_scale = int16_t(dec ? arg.scale : 0);
            }
            // A keyless aggregate over no rows still has its one group, whose
            // SUM / MIN / MAX are NULL (docs/arch/aggregation.md:144-164):
            // it keeps a count of contributions for that too.
            if (nullable || s.n_keys == 0) ao.valid_state = uint8_t(add_state(ST_COUNT, src, idx));
        }
        out.row_types.push_back(ao.out_type);
        out.row_scales.push_back(ao.out_scale);
    }
    p.naggs = s.n_aggs;
    p.state_words = words;
    for (int j = 0; j < s.n_keys; ++j) {
        out.row_types.insert(out.row_types.begin() + j, p.keys[j].out_type);
        out.row_scales.insert(out.row_scales.begin() + j, p.keys[j].out_scale);
    }
    if (int(out.row_types.size()) > kMaxCols + kMaxAggs) throw LowerError("aggregate row too wide");

    // Fused join: mark build-side slots.
    if (probe_cols >= 0) {
        for (int slot = 0; slot < p.ncols; ++slot) {
            p.cols[slot].build = out.cols.input_of[slot] >= probe_cols ? 1 : 0;
        }
    }

    // Finalize projection over (keys ++ aggregates).
    OutputPlan& o = out.out;
    std::memset(&o.prog, 0, sizeof(o.prog));
    o.row_cols = int32_t(out.row_types.size());
    for (int c = 0; c < o.row_cols; ++c) {
        const TypeInfo ti = InfoOf(out.row_types[c]);
        o.row_dom[c] = ti.dom;
        o.row_scale[c] = int16_t(IsDecimalType(out.row_types[c]) ? out.row_scales[c] : 0);
    }
    if (s.n_outputs > 0) {
        if (s.n_outputs > kMaxCols + kMaxAggs) throw LowerError("too many output columns");
        o.identity = false;
        o.n = s.n_outputs;
        std::vector<qdb_column_type> rowcols(o.row_cols);
        for (int c = 0; c < o.row_cols; ++c) {
            rowcols[c].type = out.row_types[c];
            rowcols[c].scale = out.row_scales[c];
            rowcols[c].precision = 38;
            rowcols[c].nullable = 1;
        }
        AggPlan tmp;
        InitPlan(tmp);
        ColumnMap cm;
        Lowerer OL(rowcols.data(), o.row_cols, s.output_nodes, s.n_output_nodes, tmp, cm);
        for (int k = 0; k < s.n_outputs; ++k) {
            OL.CheckTree(s.outputs[k]);
            const int g = OL.Generic(s.outputs[k]);
            o.roots[k] = uint8_t(g);
            o.root_max = std::max(o.root_max, g);
            o.out_type[k] = s.output_nodes[s.outputs[k]].type;
            o.out_scale[k] = ScaleOf(s.output_nodes[s.outputs[k]]);
        }
        // Column slots of the output program index row columns directly.
        for (int k = 0; k < tmp.prog.n; ++k) {
            GNode& g = tmp.prog.nodes[k];
            if (g.op == G_COL) g.col = uint8_t(cm.input_of[g.col]);
        }
        o.prog = tmp.prog;
        std::memcpy(o.list, tmp.list, sizeof(o.list));
    } else {
        o.identity = true;
        o.n = o.row_cols;
        for (int c = 0; c < o.n; ++c) {
            o.out_type[c] = out.row_types[c];
            o.out_scale[c] = out.row_scales[c];
        }
    }
    out.any_generic = out.any_generic || p.filter_kind == 2;
    return out;
}

ExprLowering LowerFilter(int ncols, const qdb_column_type* columns, int nnodes, const qdb_expr* nodes,
                         int predicate) {
    ExprLowering out;
    InitPlan(out.plan);
    for (int c = 0; c < ncols; ++c) InfoOf(columns[c].type);
    Lowerer L(columns, ncols, nodes, nnodes, out.plan, out.cols);
    if (predicate < 0) throw LowerError("filter needs a predicate");
    LowerPredicate(L, out.plan, predicate);
    return out;
}

ExprLowering LowerProject(int ncols, const qdb_column_type* columns, int nnodes, const qdb_expr* nodes,
                          int nexprs, const int32_t* exprs) {
    ExprLowering out;
    InitPlan(out.plan);
    for (int c = 0; c < ncols; ++c) InfoOf(columns[c].type);
    Lowerer L(columns, ncols, nodes, nnodes, out.plan, out.cols);
    for (int k = 0; k < nexprs; ++k) {
        uint8_t src = 0, idx = 0;
        bool generic = false;
        const qdb_expr& n = nodes[exprs[k]];
        if (n.type == QDB_TYPE_BOOL || n.type == QDB_TYPE_F32 || InfoOf(n.type).wrap_bits < 64) {
            // Booleans and narrow results go through the generic program,
            // which wraps to the result width.
            L.CheckTree(exprs[k]);
            src = VS_GENERIC;
            idx = uint8_t(L.Generic(exprs[k]));
        } else {
            LowerValue(L, exprs[k], src, idx, generic);
        }
        out.value_src.push_back(src);
        out.value_idx.push_back(idx);
        out.out_types.push_back(n.type);
    }
    return out;
}

}  // namespace qdb
