// fast_rt.cpp — host matchers of the typed fast-kernel shapes.
#include <cstring>

#include "fast.h"

namespace qdb {

bool MatchJoinSum(const AggPlan& p, const JoinKeyPlan& jk, int inline_slot, JoinSumShape& out) {
    std::memset(&out, 0, sizeof(out));
    if (p.nkeyparts != 0 || p.filter_kind != 0 || p.generic_root >= 0) return false;
    if (p.nstates > kJsMaxStates || p.selection != nullptr) return false;
    if (jk.n != 1 || jk.is_float[0]) return false;
    const ColDesc& kc = p.cols[jk.col[0]];
    if (kc.build || kc.width != 8 || kc.kind != LK_SIGNED || kc.mask) return false;
    out.probe_key = reinterpret_cast<const int64_t*>(kc.data);
    out.nstates = p.nstates;
    for (int s = 0; s < p.nstates; ++s) {
        const StateDesc& sd = p.states[s];
        JsState& js = out.states[s];
        js.word = sd.word;
        if (sd.kind == ST_COUNT && sd.src == VS_NONE) {
            js.nf = 0;
            continue;
        }
        if (sd.kind != ST_SUM_I64 || sd.src != VS_SOP) return false;
        const SopValue& v = p.values[sd.idx];
        if (v.kind != VK_I64 || v.nterms != 1 || v.null_cols != 0 || v.t[0].sign < 0) return false;
        const Term& t = v.t[0];
        if (t.nf < 1 || t.nf > 2) return false;
        js.nf = t.nf;
        for (int f = 0; f < t.nf; ++f) {
            const Factor& fc = t.f[f];
            if (fc.col == 0xFF || fc.kind != VK_I64) return false;
            const ColDesc& cd = p.cols[fc.col];
            if (cd.width != 8 || cd.kind != LK_SIGNED || cd.mask) return false;
            JsFactor& jf = js.f[f];
            jf.c = fc.c;
            jf.d = fc.d;
            jf.data = reinterpret_cast<const int64_t*>(cd.data);
            if (!cd.build) {
                jf.side = 0;
            } else if (fc.col == inline_slot) {
                jf.side = 1;
                out.need_pay = 1;
            } else {
                jf.side = 2;
                out.need_row = 1;
            }
        }
    }
    return true;
}

namespace {

bool IntColumn(const ColDesc& cd) {
    return !cd.build && cd.width >= 1 && cd.width <= 8 && (cd.kind == LK_SIGNED || cd.kind == LK_UNSIGNED) &&
           cd.mask == nullptr;
}

bool FitsI64(i128 v) { return v >= i128(INT64_MIN) && v <= i128(INT64_MAX); }

int FastCol(FastPlan& F, int slot) {
    for (int k = 0; k < F.ncols; ++k) {
        if (F.col_slot[k] == slot) return k;
    }
    if (F.ncols >= kFastCols) return -1;
    F.col_slot[F.ncols] = uint8_t(slot);
    return F.ncols++;
}

}  // namespace

bool MatchFast(const AggPlan& p, FastPlan& F) {
    std::memset(&F, 0, sizeof(F));
    if (p.generic_root >= 0 || p.key_words != 1 || p.nkeyparts > 2 || p.filter_kind == 2) return false;
    for (int j = 0; j < p.nkeyparts; ++j) {
        const KeyPart& k = p.keys[j];
        if (k.src != KS_COLUMN || k.is_float || k.null_shift != 0xFF || !IntColumn(p.cols[k.idx])) return false;
        const int c = FastCol(F, k.idx);
        if (c < 0) return false;
        F.key_col[j] = uint8_t(c);
        F.key_bits[j] = k.bits;
        F.key_shift[j] = k.shift;
    }
    F.nkeys = p.nkeyparts;
    if (p.filter_kind == 1) {
        if (p.natoms > kFastAtoms) return false;
        for (int j = 0; j < p.natoms; ++j) {
            const Atom& a = p.atoms[j];
            const bool cmp = a.op <= AT_GE || a.op == AT_BETWEEN || a.op == AT_IN;
            if (!cmp || a.as_f64 || a.mul != 0 || !IntColumn(p.cols[a.col])) return false;
            if (!FitsI64(a.c0) || !FitsI64(a.c1)) return false;
            const int c = FastCol(F, a.col);
            if (c < 0) return false;
            FastAtom& f = F.atoms[j];
            f.op = a.op;
            f.col = uint8_t(c);
            f.list_off = a.list_off;
            f.list_len = a.list_len;
            f.clause = a.clause;
            f.c0 = int64_t(a.c0);
            f.c1 = int64_t(a.c1);
        }
        F.natoms = p.natoms;
        F.clause_mask = p.clause_mask;
    }
    if (p.nstates > kFastStates) return false;
    for (int s = 0; s < p.nstates; ++s) {
        const StateDesc& sd = p.states[s];
        FastState& fs = F.states[s];
        fs.kind = sd.kind;
        fs.word = sd.word;
        if (sd.kind == ST_COUNT && sd.src == VS_NONE) {
            fs.nf = 0;
            continue;
        }
        if (sd.src != VS_SOP) return false;
        const SopValue& v = p.values[sd.idx];
        if (v.nterms != 1 || v.null_cols != 0 || v.t[0].sign < 0) return false;
        const Term& t = v.t[0];
        if (sd.kind == ST_SUM_F64 || sd.kind == ST_MIN_F64 || sd.kind == ST_MAX_F64) {
            // One double column, as is.
            const Factor& fc = t.f[0];
            if (v.kind != VK_F64 || t.nf != 1 || fc.col == 0xFF || fc.has_c || fc.fd != 1.0) return false;
            const ColDesc& cd = p.cols[fc.col];
            if (cd.build || cd.kind != LK_F64 || cd.width != 8 || cd.mask) return false;
            const int c = FastCol(F, fc.col);
            if (c < 0) return false;
            fs.nf = 1;
            fs.f[0].col = uint8_t(c);
            continue;
        }
        const bool ok_kind = sd.kind == ST_SUM_I64 || sd.kind == ST_SUM_I128 || sd.kind == ST_MIN_I64 ||
                             sd.kind == ST_MAX_I64;
        if (!ok_kind || v.kind == VK_F64) return false;
        if (v.kind == VK_I128 && sd.kind != ST_SUM_I128) return false;
        if (t.nf < 1 || t.nf > 3) return false;
        fs.nf = t.nf;
        fs.wide = v.kind == VK_I128 ? 1 : 0;
        for (int f = 0; f < t.nf; ++f) {
            const Factor& fc = t.f[f];
            // A 64-bit factor, or a bare 64-bit column widened into a 128-bit product.
            const bool bare = fc.col != 0xFF && fc.c == 0 && fc.d == 1;
            if (fc.kind != VK_I64 && !bare) return false;
            FastFactor& ff = fs.f[f];
            if (fc.col == 0xFF) {
                ff.col = 0;
                ff.c = fc.c;
                ff.d = 0;
                continue;
            }
            if (!IntColumn(p.cols[fc.col])) return false;
            const int c = FastCol(F, fc.col);
            if (c < 0) return false;
            ff.col = uint8_t(c);
            ff.c = fc.c;
            ff.d = fc.d;
        }
    }
    F.nstates = p.nstates;
    return true;
}

}  // namespace qdb
