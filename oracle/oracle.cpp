// oracle.cpp — CPU restatement of QumirDB's hot-path algorithms.
//
// TEST INFRASTRUCTURE ONLY: the checker of the device kernels.  Nothing in the
// product links or loads this library.  Every routine names the reference
// file:line whose behaviour it restates; the code is written from the
// behaviour, not translated from the oz sources.
#include "oracle.h"

#include <algorithm>
#include <unordered_set>
#include <random>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <functional>
#include <memory>
#include <queue>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

namespace {

using i128 = __int128;
using u128 = unsigned __int128;

struct Error : std::runtime_error {
    using std::runtime_error::runtime_error;
};

void SetErr(char* err, size_t len, const char* msg) {
    if (err && len) {
        std::snprintf(err, len, "%s", msg);
    }
}

// ---------------------------------------------------------------------------
// Values.  Integers, dates, chars and decimals live sign-extended in `i`
// (decimals unscaled); doubles in `f`; booleans as 0/1 in `i`.
// ---------------------------------------------------------------------------
struct Val {
    i128 i = 0;
    double f = 0.0;
    bool null = false;
    const uint8_t* s = nullptr;   // strings: the row's bytes
    int64_t n = 0;                // and their count
};

bool IsFloat(int t) { return t == QDB_TYPE_F32 || t == QDB_TYPE_F64; }
bool IsDecimal(int t) { return t == QDB_TYPE_DECIMAL64 || t == QDB_TYPE_DECIMAL128; }
bool IsUnsigned(int t) {
    return t == QDB_TYPE_U8 || t == QDB_TYPE_U16 || t == QDB_TYPE_U32 || t == QDB_TYPE_U64;
}

int WidthBits(int t) {
    switch (t) {
        case QDB_TYPE_BOOL: return 1;
        case QDB_TYPE_I8: case QDB_TYPE_U8: case QDB_TYPE_CHAR1: return 8;
        case QDB_TYPE_I16: case QDB_TYPE_U16: return 16;
        case QDB_TYPE_I32: case QDB_TYPE_U32: case QDB_TYPE_DATE32: case QDB_TYPE_F32: return 32;
        case QDB_TYPE_I64: case QDB_TYPE_U64: case QDB_TYPE_DECIMAL64: case QDB_TYPE_F64: return 64;
        case QDB_TYPE_DECIMAL128: return 128;
    }
    throw Error("unknown type");
}

int StorageBytes(int t) {
    if (t == QDB_TYPE_BOOL) return 1;
    return WidthBits(t) / 8;
}

// Wraps an integer result to its type's width, as the reference's fixed-width
// arithmetic does (integer ops wrap; decimals wrap at 64 or 128 bits,
// qdb/modules/qumirdb.oz:1305-1321).
i128 Wrap(i128 v, int t) {
    const int bits = WidthBits(t);
    if (bits >= 128) return v;
    const u128 mask = (u128(1) << bits) - 1;
    u128 u = u128(v) & mask;
    if (!IsUnsigned(t) && t != QDB_TYPE_CHAR1 && t != QDB_TYPE_BOOL) {
        if (u >> (bits - 1)) u |= ~mask;   // sign extend
    }
    return i128(u);
}

i128 Pow10(int k) {
    i128 r = 1;
    for (int j = 0; j < k; ++j) r *= 10;
    return r;
}

bool MaskBit(const uint8_t* mask, int64_t bit) {
    return (mask[bit >> 3] >> (bit & 7)) & 1;
}

// Reads row `row` of a column (TColumn, qdb/io/io.h:17-24): Arrow validity
// bits, bitmap-backed booleans at DataBitOffset, fixed-width values.
Val ReadCell(const qdb_column& c, const qdb_column_type& t, int64_t row) {
    Val v;
    if (c.Mask && !MaskBit(c.Mask, c.MaskBitOffset + row)) {
        v.null = true;
        return v;
    }
    const char* d = c.Data;
    switch (t.type) {
        case QDB_TYPE_BOOL: v.i = MaskBit(reinterpret_cast<const uint8_t*>(d), c.DataBitOffset + row); break;
        case QDB_TYPE_I8: v.i = reinterpret_cast<const int8_t*>(d)[row]; break;
        case QDB_TYPE_I16: v.i = reinterpret_cast<const int16_t*>(d)[row]; break;
        case QDB_TYPE_I32: case QDB_TYPE_DATE32: v.i = reinterpret_cast<const int32_t*>(d)[row]; break;
        case QDB_TYPE_I64: case QDB_TYPE_DECIMAL64: v.i = reinterpret_cast<const int64_t*>(d)[row]; break;
        case QDB_TYPE_U8: case QDB_TYPE_CHAR1: v.i = reinterpret_cast<const uint8_t*>(d)[row]; break;
        case QDB_TYPE_U16: v.i = reinterpret_cast<const uint16_t*>(d)[row]; break;
        case QDB_TYPE_U32: v.i = reinterpret_cast<const uint32_t*>(d)[row]; break;
        case QDB_TYPE_U64: v.i = reinterpret_cast<const uint64_t*>(d)[row]; break;
        case QDB_TYPE_F32: v.f = reinterpret_cast<const float*>(d)[row]; break;
        case QDB_TYPE_F64: v.f = reinterpret_cast<const double*>(d)[row]; break;
        case QDB_TYPE_DECIMAL128: {
            const uint64_t* w = reinterpret_cast<const uint64_t*>(d) + 2 * row;
            v.i = i128((u128(uint64_t(w[1])) << 64) | w[0]);
            break;
        }
        case QDB_TYPE_STRING: {   // Arrow utf8 / large_utf8: Data[Offsets[r] .. Offsets[r+1])
            int64_t b, e;
            if (c.OffsetWidth == 8) {
                b = static_cast<const int64_t*>(c.Offsets)[row];
                e = static_cast<const int64_t*>(c.Offsets)[row + 1];
            } else if (c.OffsetWidth == 4) {
                b = static_cast<const int32_t*>(c.Offsets)[row];
                e = static_cast<const int32_t*>(c.Offsets)[row + 1];
            } else {
                throw Error("string column without offsets of width 4 or 8");
            }
            v.s = reinterpret_cast<const uint8_t*>(d) + b;
            v.n = e - b;
            break;
        }
        default: throw Error("unsupported column type");
    }
    return v;
}

double ToDouble(const Val& v, int t, int scale) {
    if (IsFloat(t)) return v.f;
    if (IsDecimal(t)) return double(v.i) / std::pow(10.0, scale);
    return double(v.i);
}

// ---------------------------------------------------------------------------
// Expression evaluation under the lowering's annotated types
// (qdb/kernel/annotate_type.cpp:725-945, qdb/modules/qumirdb.oz:1290-1330,
// qdb/modules/qumirdb_runtime.cpp:680-735).
// ---------------------------------------------------------------------------
struct Expr {
    const qdb_expr* nodes;
    int32_t n;
};

int CmpAligned(const Val& a, int ta, int sa, const Val& b, int tb, int sb) {
    if (IsFloat(ta) || IsFloat(tb)) {
        const double x = ToDouble(a, ta, sa), y = ToDouble(b, tb, sb);
        return x < y ? -1 : (x > y ? 1 : 0);
    }
    const int s = std::max(IsDecimal(ta) ? sa : 0, IsDecimal(tb) ? sb : 0);
    const i128 x = a.i * Pow10(s - (IsDecimal(ta) ? sa : 0));
    const i128 y = b.i * Pow10(s - (IsDecimal(tb) ? sb : 0));
    return x < y ? -1 : (x > y ? 1 : 0);
}

// Aligns an integer/decimal operand to the result scale of +/- and CASE.
i128 AtScale(const Val& v, int t, int s, int target) {
    const int from = IsDecimal(t) ? s : 0;
    if (target >= from) return v.i * Pow10(target - from);
    return v.i / Pow10(from - target);
}

// Evaluates every node up to and including `root` for one row; `leaf(col)`
// returns input column values.  Division by zero raises (deferred row error,
// docs/arch/scheduler_runtime.md:174-186).
void EvalAll(const Expr& e, int32_t root, const std::function<Val(int32_t)>& leaf,
             std::vector<Val>& out) {
    out.resize(root + 1);
    for (int32_t k = 0; k <= root; ++k) {
        const qdb_expr& n = e.nodes[k];
        Val r;
        auto A = [&](int j) -> const Val& { return out[n.args[j]]; };
        auto T = [&](int j) { return e.nodes[n.args[j]].type; };
        auto S = [&](int j) { return e.nodes[n.args[j]].scale; };
        switch (n.op) {
            case QDB_EXPR_COLUMN: r = leaf(n.column); break;
            case QDB_EXPR_CONST:
                if (IsFloat(n.type)) {
                    std::memcpy(&r.f, &n.imm_lo, 8);
                } else if (n.type == QDB_TYPE_DECIMAL128) {
                    r.i = i128((u128(uint64_t(n.imm_hi)) << 64) | uint64_t(n.imm_lo));
                } else {
                    r.i = n.imm_lo;
                }
                break;
            case QDB_EXPR_NULL: r.null = true; break;
            case QDB_EXPR_MOD: {
                // Operands share the result scale; the remainder takes the
                // dividend's sign (qdb/modules/qumirdb.oz:1323-1328).
                const Val& a = A(0); const Val& b = A(1);
                if (a.null || b.null) { r.null = true; break; }
                const int rs = IsDecimal(n.type) ? n.scale : 0;
                const i128 x = AtScale(a, T(0), S(0), rs), y = AtScale(b, T(1), S(1), rs);
                if (y == 0) throw Error("division by zero");
                r.i = Wrap(x % y, n.type);
                break;
            }
            case QDB_EXPR_ADD: case QDB_EXPR_SUB: case QDB_EXPR_MUL: case QDB_EXPR_DIV: {
                const Val& a = A(0); const Val& b = A(1);
                if (a.null || b.null) { r.null = true; break; }
                if (IsFloat(n.type)) {
                    const double x = ToDouble(a, T(0), S(0)), y = ToDouble(b, T(1), S(1));
                    r.f = n.op == QDB_EXPR_ADD ? x + y : n.op == QDB_EXPR_SUB ? x - y
                        : n.op == QDB_EXPR_MUL ? x * y : x / y;
                    if (n.type == QDB_TYPE_F32) r.f = float(r.f);
                    break;
                }
                if (n.op == QDB_EXPR_ADD || n.op == QDB_EXPR_SUB) {
                    const i128 x = AtScale(a, T(0), S(0), IsDecimal(n.type) ? n.scale : 0);
                    const i128 y = AtScale(b, T(1), S(1), IsDecimal(n.type) ? n.scale : 0);
                    r.i = Wrap(n.op == QDB_EXPR_ADD ? i128(u128(x) + u128(y)) : i128(u128(x) - u128(y)), n.type);
                } else if (n.op == QDB_EXPR_MUL) {
                    // Unscaled operands multiply; the scales add up to the
                    // result's (DecimalProductSpec, annotate_type.cpp:746-760).
                    const int sa = IsDecimal(T(0)) ? S(0) : 0, sb = IsDecimal(T(1)) ? S(1) : 0;
                    i128 p = i128(u128(a.i) * u128(b.i));
                    const int rs = IsDecimal(n.type) ? n.scale : 0;
                    if (rs > sa + sb) p = i128(u128(p) * u128(Pow10(rs - sa - sb)));
                    r.i = Wrap(p, n.type);
                } else {
                    if (b.i == 0) throw Error("division by zero");
                    // DECIMAL / integer keeps the dividend's scale
                    // (annotate_type.cpp:908-910); DECIMAL / DECIMAL scales the
                    // dividend to the quotient's scale first.
                    const int sa = IsDecimal(T(0)) ? S(0) : 0, sb = IsDecimal(T(1)) ? S(1) : 0;
                    const int rs = IsDecimal(n.type) ? n.scale : 0;
                    const i128 x = a.i * Pow10(std::max(0, rs - sa + sb));
                    r.i = Wrap(x / b.i, n.type);
                }
                break;
            }
            case QDB_EXPR_NEG: {
                const Val& a = A(0);
                if (a.null) { r.null = true; break; }
                if (IsFloat(n.type)) r.f = -ToDouble(a, T(0), S(0));
                else r.i = Wrap(i128(u128(0) - u128(a.i)), n.type);
                break;
            }
            case QDB_EXPR_CAST: {
                const Val& a = A(0);
                if (a.null) { r.null = true; break; }
                if (IsFloat(n.type)) {
                    r.f = ToDouble(a, T(0), S(0));
                    if (n.type == QDB_TYPE_F32) r.f = float(r.f);
                } else if (IsFloat(T(0))) {
                    r.i = Wrap(i128(int64_t(a.f)), n.type);
                } else {
                    r.i = Wrap(AtScale(a, T(0), S(0), IsDecimal(n.type) ? n.scale : 0), n.type);
                }
                break;
            }
            case QDB_EXPR_EQ: case QDB_EXPR_NE: case QDB_EXPR_LT: case QDB_EXPR_LE:
            case QDB_EXPR_GT: case QDB_EXPR_GE: {
                const Val& a = A(0); const Val& b = A(1);
                if (a.null || b.null) { r.null = true; break; }
                const int c = CmpAligned(a, T(0), S(0), b, T(1), S(1));
                bool t = false;
                switch (n.op) {
                    case QDB_EXPR_EQ: t = c == 0; break;
                    case QDB_EXPR_NE: t = c != 0; break;
                    case QDB_EXPR_LT: t = c < 0; break;
                    case QDB_EXPR_LE: t = c <= 0; break;
                    case QDB_EXPR_GT: t = c > 0; break;
                    default: t = c >= 0; break;
                }
                // A NaN compares false everywhere but !=.
                if ((IsFloat(T(0)) || IsFloat(T(1))) &&
                    (std::isnan(ToDouble(a, T(0), S(0))) || std::isnan(ToDouble(b, T(1), S(1))))) {
                    t = n.op == QDB_EXPR_NE;
                }
                r.i = t;
                break;
            }
            case QDB_EXPR_AND: {
                // SQL three-valued logic (test/test_filter.cpp semantics).
                const Val& a = A(0); const Val& b = A(1);
                if ((!a.null && a.i == 0) || (!b.null && b.i == 0)) { r.i = 0; }
                else if (a.null || b.null) { r.null = true; }
                else r.i = 1;
                break;
            }
            case QDB_EXPR_OR: {
                const Val& a = A(0); const Val& b = A(1);
                if ((!a.null && a.i) || (!b.null && b.i)) { r.i = 1; }
                else if (a.null || b.null) { r.null = true; }
                else r.i = 0;
                break;
            }
            case QDB_EXPR_NOT: {
                const Val& a = A(0);
                if (a.null) r.null = true; else r.i = a.i ? 0 : 1;
                break;
            }
            case QDB_EXPR_BETWEEN: {
                const Val& a = A(0); const Val& lo = A(1); const Val& hi = A(2);
                if (a.null || lo.null || hi.null) { r.null = true; break; }
                r.i = CmpAligned(a, T(0), S(0), lo, T(1), S(1)) >= 0 &&
                      CmpAligned(a, T(0), S(0), hi, T(2), S(2)) <= 0;
                break;
            }
            case QDB_EXPR_IN_LIST: {
                const Val& a = A(0);
                if (a.null) { r.null = true; break; }
                bool found = false;
                for (int32_t j = 0; j < n.list_len && !found; ++j) {
                    if (IsFloat(T(0))) {
                        double x; std::memcpy(&x, &n.list[j], 8);
                        found = x == a.f;
                    } else {
                        found = i128(n.list[j]) == a.i;
                    }
                }
                r.i = found;
                break;
            }
            case QDB_EXPR_CASE: {
                const Val& c = A(0);
                const bool take = !c.null && c.i;
                const Val& v = take ? A(1) : A(2);
                const int vt = take ? T(1) : T(2), vs = take ? S(1) : S(2);
                r = v;
                if (!v.null) {
                    if (IsFloat(n.type)) r.f = ToDouble(v, vt, vs);
                    else r.i = Wrap(AtScale(v, vt, vs, IsDecimal(n.type) ? n.scale : 0), n.type);
                }
                break;
            }
            case QDB_EXPR_IS_NULL: r.i = A(0).null ? 1 : 0; break;
            case QDB_EXPR_IS_NOT_NULL: r.i = A(0).null ? 0 : 1; break;
            default: throw Error("unsupported expression op");
        }
        out[k] = r;
    }
}

// ---------------------------------------------------------------------------
// Key hashing: HashKeyValue (qdb/kernel/gen.cpp:233-379), rh_hash(i64)
// (qdb/kernel/aggregation/key_ops_i64.oz:4-11) and qdb_string_hash_bytes
// (qdb/modules/qumirdb_runtime.cpp:270-300).
// ---------------------------------------------------------------------------
uint64_t MixU64(uint64_t h) {
    h ^= h >> 12;
    h ^= h << 25;
    h ^= h >> 27;
    return h * 2685821657736338717ULL;
}

uint64_t ByteSwap(uint64_t x) { return __builtin_bswap64(x); }

// Strings above 16 bytes: XXH3-64 (xxHash 0.8, as vendored by Apache Arrow
// and called by qdb_string_hash_bytes) with seed 0 and the engine's own
// 136-byte secret, qdb/modules/qumirdb_runtime.cpp:253-299.  A restatement
// of the published algorithm: the 17-128, 129-240 and long (stripes of 64
// bytes, blocks of (secret - 64) / 8 stripes) paths.
const uint8_t kStringSecret[] = {
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
constexpr int64_t kStringSecretBytes = 136;
static_assert(sizeof(kStringSecret) == kStringSecretBytes, "secret size");

constexpr uint64_t kXxP32_1 = 0x9E3779B1ULL, kXxP32_2 = 0x85EBCA77ULL, kXxP32_3 = 0xC2B2AE3DULL;
constexpr uint64_t kXxP64_1 = 0x9E3779B185EBCA87ULL, kXxP64_2 = 0xC2B2AE3D27D4EB4FULL;
constexpr uint64_t kXxP64_3 = 0x165667B19E3779F9ULL, kXxP64_4 = 0x85EBCA77C2B2AE63ULL;
constexpr uint64_t kXxP64_5 = 0x27D4EB2F165667C5ULL;

uint64_t XxLe64(const uint8_t* p) {
    uint64_t v = 0;
    for (int k = 7; k >= 0; --k) v = (v << 8) | p[k];
    return v;
}

uint64_t XxFold(uint64_t a, uint64_t b) {
    const unsigned __int128 p = (unsigned __int128)a * b;
    return uint64_t(p) ^ uint64_t(p >> 64);
}

uint64_t XxAvalanche(uint64_t h) {
    h ^= h >> 37;
    h *= 0x165667919E3779F9ULL;
    return h ^ (h >> 32);
}

uint64_t XxMix16(const uint8_t* in, const uint8_t* sec) {
    return XxFold(XxLe64(in) ^ XxLe64(sec), XxLe64(in + 8) ^ XxLe64(sec + 8));
}

void XxStripe(uint64_t* acc, const uint8_t* in, const uint8_t* sec) {
    for (int i = 0; i < 8; ++i) {
        const uint64_t v = XxLe64(in + 8 * i);
        const uint64_t k = v ^ XxLe64(sec + 8 * i);
        acc[i ^ 1] += v;
        acc[i] += (k & 0xffffffffULL) * (k >> 32);
    }
}

uint64_t Xxh3WithSecret(const uint8_t* d, int64_t n, const uint8_t* sec, int64_t sec_n) {
    const uint64_t len = uint64_t(n);
    if (n <= 128) {   // 17..128
        uint64_t acc = len * kXxP64_1;
        if (n > 32) {
            if (n > 64) {
                if (n > 96) {
                    acc += XxMix16(d + 48, sec + 96);
                    acc += XxMix16(d + n - 64, sec + 112);
                }
                acc += XxMix16(d + 32, sec + 64);
                acc += XxMix16(d + n - 48, sec + 80);
            }
            acc += XxMix16(d + 16, sec + 32);
            acc += XxMix16(d + n - 32, sec + 48);
        }
        acc += XxMix16(d, sec);
        acc += XxMix16(d + n - 16, sec + 16);
        return XxAvalanche(acc);
    }
    if (n <= 240) {
        uint64_t acc = len * kXxP64_1;
        for (int i = 0; i < 8; ++i) acc += XxMix16(d + 16 * i, sec + 16 * i);
        acc = XxAvalanche(acc);
        const int rounds = int(n / 16);
        for (int i = 8; i < rounds; ++i) acc += XxMix16(d + 16 * i, sec + 16 * (i - 8) + 3);
        acc += XxMix16(d + n - 16, sec + 136 - 17);
        return XxAvalanche(acc);
    }
    uint64_t acc[8] = {kXxP32_3, kXxP64_1, kXxP64_2, kXxP64_3, kXxP64_4, kXxP32_2, kXxP64_5, kXxP32_1};
    const int64_t stripes_per_block = (sec_n - 64) / 8;
    const int64_t block = 64 * stripes_per_block;
    const int64_t blocks = (n - 1) / block;
    for (int64_t b = 0; b < blocks; ++b) {
        for (int64_t s = 0; s < stripes_per_block; ++s) XxStripe(acc, d + b * block + 64 * s, sec + 8 * s);
        for (int i = 0; i < 8; ++i) {   // scramble
            uint64_t a = acc[i];
            a ^= a >> 47;
            a ^= XxLe64(sec + sec_n - 64 + 8 * i);
            acc[i] = a * kXxP32_1;
        }
    }
    const int64_t tail_stripes = ((n - 1) - block * blocks) / 64;
    for (int64_t s = 0; s < tail_stripes; ++s) XxStripe(acc, d + blocks * block + 64 * s, sec + 8 * s);
    XxStripe(acc, d + n - 64, sec + sec_n - 64 - 7);
    uint64_t r = len * kXxP64_1;
    for (int i = 0; i < 4; ++i) r += XxFold(acc[2 * i] ^ XxLe64(sec + 11 + 16 * i), acc[2 * i + 1] ^ XxLe64(sec + 11 + 16 * i + 8));
    return XxAvalanche(r);
}

uint64_t StringHash(const uint8_t* d, int64_t n) {
    const uint64_t mul0 = 11400714785074694791ULL, mul1 = 14029467366897019727ULL;
    if (n == 0) return 1;
    if (n <= 3) {
        const uint32_t x = (uint32_t(n) << 24) ^ (uint32_t(d[0]) << 16) ^
                           (uint32_t(d[n / 2]) << 8) ^ d[n - 1];
        return ByteSwap(mul0 * x);
    }
    if (n <= 8) {
        uint32_t x, y;
        std::memcpy(&x, d + n - 4, 4);
        std::memcpy(&y, d, 4);
        return uint64_t(n) ^ ByteSwap(mul0 * x) ^ ByteSwap(mul1 * y);
    }
    if (n <= 16) {
        uint64_t x, y;
        std::memcpy(&x, d + n - 8, 8);
        std::memcpy(&y, d, 8);
        return uint64_t(n) ^ ByteSwap(mul0 * x) ^ ByteSwap(mul1 * y);
    }
    return Xxh3WithSecret(d, n, kStringSecret, kStringSecretBytes);
}

// Canonical float bits: -0 -> +0, every NaN -> one quiet NaN
// (docs/arch/aggregation.md:109-125).
uint64_t CanonicalF64Bits(double f) {
    if (f == 0.0) return 0;
    if (std::isnan(f)) return 0x7ff8000000000000ULL;
    uint64_t b; std::memcpy(&b, &f, 8);
    return b;
}

uint64_t LeafHash(const Val& v, int t) {
    switch (t) {
        case QDB_TYPE_BOOL: return uint64_t(v.i != 0) * 2685821657736338717ULL;
        case QDB_TYPE_CHAR1: { const uint8_t b = uint8_t(v.i); return StringHash(&b, 1); }
        case QDB_TYPE_STRING: return StringHash(v.s, v.n);
        case QDB_TYPE_F64: return MixU64(CanonicalF64Bits(v.f));
        case QDB_TYPE_F32: {
            float f = float(v.f);
            uint32_t b;
            if (f == 0.0f) b = 0; else if (std::isnan(f)) b = 0x7fc00000u; else std::memcpy(&b, &f, 4);
            return MixU64(b);
        }
        case QDB_TYPE_DECIMAL128: {
            uint64_t lo = uint64_t(v.i), hi = uint64_t(u128(v.i) >> 64);
            lo = MixU64(lo); hi = MixU64(hi);
            return lo ^ (hi + 0x9e3779b97f4a7c15ULL + (lo << 6) + (lo >> 2));
        }
        default: {
            const int bits = WidthBits(t);
            const uint64_t mask = bits >= 64 ? ~0ULL : ((1ULL << bits) - 1);
            return MixU64(uint64_t(v.i) & mask);
        }
    }
}

// Struct key: boost-style ordered combine over the fields of the key struct
// (gen.cpp:345-375).  A nullable key column j is two fields of that struct,
// `valid_j` (BOOL) before `key_j` (BuildAggregateKeyDescriptor,
// qdb/kernel/aggregate_key.cpp:211-260): the validity flag is hashed like a
// BOOL leaf (flag * 2685821657736338717), and a NULL key field contributes 0.
// Without `nullable` every field is taken as NOT NULL (internal placement).
uint64_t StructHash(const Val* vals, const int* types, int n, const bool* nullable = nullptr) {
    uint64_t h = 0;
    auto combine = [&h](uint64_t fh) { h ^= fh + 0x9e3779b97f4a7c15ULL + (h << 6) + (h >> 2); };
    for (int j = 0; j < n; ++j) {
        if (nullable && nullable[j]) combine(vals[j].null ? 0 : 2685821657736338717ULL);
        combine(vals[j].null ? 0 : LeafHash(vals[j], types[j]));
    }
    return h;
}

bool KeyFieldEqual(const Val& a, const Val& b, int t) {
    if (a.null || b.null) return a.null == b.null;   // NULL keys group together
    if (IsFloat(t)) return CanonicalF64Bits(a.f) == CanonicalF64Bits(b.f);
    return a.i == b.i;
}

// ---------------------------------------------------------------------------
// Aggregate state and reducers (qdb/kernel/gen.cpp:3301-3593) and result
// typing (qdb/plan/ops/aggregate.cpp:21-57).
// ---------------------------------------------------------------------------
struct AggState {
    i128 acc = 0;        // integer/decimal sum, or min/max
    double facc = 0.0;   // f64 sum/min/max
    int64_t count = 0;   // rows (COUNT) or valid contributions
};

struct ResultType {
    int type;
    int scale;
    bool nullable;
};

ResultType AggResultType(const qdb_aggregate_spec& s, const qdb_agg_item& a) {
    if (a.func == QDB_AGG_COUNT_STAR || a.func == QDB_AGG_COUNT) return {QDB_TYPE_I64, 0, false};
    const qdb_expr& arg = s.nodes[a.arg];
    bool nullable = true;   // an argument is non-null only if provably so
    if (arg.op == QDB_EXPR_COLUMN) nullable = s.columns[arg.column].nullable != 0;
    else {
        // Conservative: the tree is non-null when every COLUMN leaf is.
        nullable = false;
        std::vector<int> stack{a.arg};
        while (!stack.empty()) {
            const qdb_expr& e = s.nodes[stack.back()];
            stack.pop_back();
            if (e.op == QDB_EXPR_COLUMN && s.columns[e.column].nullable) nullable = true;
            if (e.op == QDB_EXPR_NULL || e.op == QDB_EXPR_DIV) nullable = nullable || e.op == QDB_EXPR_NULL;
            const int na = e.op == QDB_EXPR_BETWEEN || e.op == QDB_EXPR_CASE ? 3
                : (e.op == QDB_EXPR_COLUMN || e.op == QDB_EXPR_CONST || e.op == QDB_EXPR_NULL) ? 0
                : (e.op == QDB_EXPR_NEG || e.op == QDB_EXPR_CAST || e.op == QDB_EXPR_NOT ||
                   e.op == QDB_EXPR_IN_LIST || e.op == QDB_EXPR_IS_NULL || e.op == QDB_EXPR_IS_NOT_NULL) ? 1 : 2;
            for (int j = 0; j < na; ++j) stack.push_back(e.args[j]);
        }
    }
    const int t = arg.type;
    if (IsFloat(t)) return {QDB_TYPE_F64, 0, nullable};
    if (a.func == QDB_AGG_SUM) {
        if (IsDecimal(t)) return {QDB_TYPE_DECIMAL128, arg.scale, nullable};
        if (t == QDB_TYPE_DATE32) throw Error("function sum(DATE) does not exist");
        return {QDB_TYPE_I64, 0, nullable};
    }
    // MIN/MAX keep decimals; integers and dates widen to i64.
    if (IsDecimal(t)) return {t, arg.scale, nullable};
    return {QDB_TYPE_I64, 0, nullable};
}

void Reduce(const qdb_agg_item& a, const ResultType& rt, AggState& st, const Val& v) {
    switch (a.func) {
        case QDB_AGG_COUNT_STAR: ++st.count; return;
        case QDB_AGG_COUNT: if (!v.null) ++st.count; return;
        default: break;
    }
    if (v.null) return;
    const bool first = st.count == 0;
    if (rt.type == QDB_TYPE_F64) {
        const double x = v.f;
        if (a.func == QDB_AGG_SUM) st.facc = first ? x : st.facc + x;
        else if (a.func == QDB_AGG_MIN) st.facc = first ? x : (x < st.facc ? x : st.facc);
        else st.facc = first ? x : (x > st.facc ? x : st.facc);
    } else {
        const i128 x = v.i;
        if (a.func == QDB_AGG_SUM) {
            st.acc = first ? Wrap(x, rt.type) : Wrap(i128(u128(st.acc) + u128(x)), rt.type);
        } else if (a.func == QDB_AGG_MIN) {
            st.acc = first ? x : (x < st.acc ? x : st.acc);
        } else {
            st.acc = first ? x : (x > st.acc ? x : st.acc);
        }
    }
    ++st.count;
}

// Partial-state combine of the cascade (docs/arch/aggregation.md:343-348):
// counts add, sums add, min/max fold.
void Combine(const qdb_agg_item& a, const ResultType& rt, AggState& into, const AggState& from) {
    if (a.func == QDB_AGG_COUNT_STAR || a.func == QDB_AGG_COUNT) { into.count += from.count; return; }
    if (from.count == 0) return;
    if (into.count == 0) { into = from; return; }
    if (rt.type == QDB_TYPE_F64) {
        if (a.func == QDB_AGG_SUM) into.facc += from.facc;
        else if (a.func == QDB_AGG_MIN) into.facc = from.facc < into.facc ? from.facc : into.facc;
        else into.facc = from.facc > into.facc ? from.facc : into.facc;
    } else {
        if (a.func == QDB_AGG_SUM) into.acc = Wrap(i128(u128(into.acc) + u128(from.acc)), rt.type);
        else if (a.func == QDB_AGG_MIN) into.acc = from.acc < into.acc ? from.acc : into.acc;
        else into.acc = from.acc > into.acc ? from.acc : into.acc;
    }
    into.count += from.count;
}

// ---------------------------------------------------------------------------
// Swiss group table (qdb/kernel/aggregation/swiss_group.oz:5-67,
// robin_hood_dual_key.oz:14-288, aggregation_hashtable_generic.oz:88-177):
// 8-slot groups of control bytes (0x80 empty, H2 = hash & 0x7F, no
// tombstones), triangular group probing, growth before an insert would cross
// 7/8 of the capacity, groups numbered densely in first-seen order.
// ---------------------------------------------------------------------------
struct SwissTable {
    int nkeys = 0;
    const int* key_types = nullptr;
    int64_t capacity = 8;
    std::vector<uint8_t> ctrl;
    std::vector<int64_t> slot_dense;      // physical slot -> dense group id
    std::vector<Val> group_keys;          // dense id * nkeys
    std::vector<uint64_t> group_hash;

    void Init(int n, const int* types, int64_t cap) {
        nkeys = n;
        key_types = types;
        capacity = std::max<int64_t>(8, cap);
        ctrl.assign(capacity, 0x80);
        slot_dense.assign(capacity, -1);
        group_keys.clear();
        group_hash.clear();
    }
    int64_t Size() const { return int64_t(group_hash.size()); }

    bool KeysEqual(int64_t dense, const Val* key) const {
        for (int j = 0; j < nkeys; ++j) {
            if (!KeyFieldEqual(group_keys[dense * nkeys + j], key[j], key_types[j])) return false;
        }
        return true;
    }

    // rh_lookup_or_empty_physical (robin_hood_dual_key.oz:14-52).
    int64_t LookupOrEmpty(const Val* key, uint64_t hash, int64_t& empty_slot) const {
        empty_slot = -1;
        const int64_t num_groups = capacity >> 3, group_mask = num_groups - 1;
        const uint8_t h2 = uint8_t(hash & 127);
        int64_t g = int64_t(hash >> 7) & group_mask;
        for (int64_t step = 0, probes = 0; probes < num_groups; ++probes) {
            for (int s = 0; s < 8; ++s) {
                const int64_t slot = (g << 3) + s;
                if (ctrl[slot] == h2 && KeysEqual(slot_dense[slot], key)) return slot;
            }
            for (int s = 0; s < 8; ++s) {
                if (ctrl[(g << 3) + s] & 0x80) { empty_slot = (g << 3) + s; return -1; }
            }
            ++step;
            g = (g + step) & group_mask;
        }
        return -1;
    }

    // rh_find_empty_slot (robin_hood_dual_key.oz:96-124).
    int64_t FindEmpty(uint64_t hash) const {
        const int64_t num_groups = capacity >> 3, group_mask = num_groups - 1;
        int64_t g = int64_t(hash >> 7) & group_mask;
        for (int64_t step = 0, probes = 0; probes < num_groups; ++probes) {
            for (int s = 0; s < 8; ++s) {
                if (ctrl[(g << 3) + s] & 0x80) return (g << 3) + s;
            }
            ++step;
            g = (g + step) & group_mask;
        }
        return -1;
    }

    void Rehash(int64_t new_capacity) {
        capacity = new_capacity;
        ctrl.assign(capacity, 0x80);
        slot_dense.assign(capacity, -1);
        for (int64_t d = 0; d < Size(); ++d) {
            const int64_t slot = FindEmpty(group_hash[d]);
            ctrl[slot] = uint8_t(group_hash[d] & 127);
            slot_dense[slot] = d;
        }
    }

    // aht_upsert_aggregate + aht_insert_dual (robin_hood_dual_key.oz:143-224):
    // returns the dense group id and whether it is new.
    int64_t Upsert(const Val* key, uint64_t hash, bool& is_new) {
        is_new = false;
        int64_t empty = -1;
        const int64_t slot = LookupOrEmpty(key, hash, empty);
        if (slot >= 0) return slot_dense[slot];
        const int64_t dense = Size();
        if (dense + 1 > capacity - (capacity >> 3)) {   // aht_insert_grows
            Rehash(capacity * 2);
            empty = FindEmpty(hash);
        }
        ctrl[empty] = uint8_t(hash & 127);
        slot_dense[empty] = dense;
        group_keys.insert(group_keys.end(), key, key + nkeys);
        group_hash.push_back(hash);
        is_new = true;
        return dense;
    }
};

// A compiled view of an aggregate spec for the oracle.
struct AggPlan {
    const qdb_aggregate_spec* spec;
    Expr expr;
    int32_t max_root = -1;
    std::vector<int> key_types;
    std::vector<ResultType> result_types;
};

AggPlan MakePlan(const qdb_aggregate_spec& s) {
    AggPlan p;
    p.spec = &s;
    p.expr = {s.nodes, s.n_nodes};
    p.max_root = s.filter;
    for (int j = 0; j < s.n_keys; ++j) {
        p.key_types.push_back(s.nodes[s.keys[j]].type);
        p.max_root = std::max(p.max_root, s.keys[j]);
    }
    for (int j = 0; j < s.n_aggs; ++j) {
        p.result_types.push_back(AggResultType(s, s.aggs[j]));
        p.max_root = std::max(p.max_root, s.aggs[j].arg);
    }
    return p;
}

struct GroupSet {
    SwissTable table;
    std::vector<AggState> states;   // dense id * n_aggs
};

// One lane of agg_dispatch(Update) over a row range: per selected row, filter,
// key, upsert, reducers (GenGenericAggregateDispatchAst, gen.cpp:2075-2299).
void AggregateRows(const AggPlan& p, const qdb_rowset& b, int64_t begin, int64_t end, GroupSet& g) {
    const qdb_aggregate_spec& s = *p.spec;
    std::vector<Val> vals;
    std::vector<Val> key(std::max(1, s.n_keys));
    for (int64_t row = begin; row < end; ++row) {
        if (b.Selection && !b.Selection[row]) continue;
        if (p.max_root >= 0) {
            EvalAll(p.expr, p.max_root,
                    [&](int32_t c) { return ReadCell(b.Columns[c], s.columns[c], row); }, vals);
        }
        if (s.filter >= 0) {
            const Val& f = vals[s.filter];
            if (f.null || f.i == 0) continue;
        }
        for (int j = 0; j < s.n_keys; ++j) key[j] = vals[s.keys[j]];
        const uint64_t hash = StructHash(key.data(), p.key_types.data(), s.n_keys);
        bool is_new = false;
        const int64_t dense = g.table.Upsert(key.data(), hash, is_new);
        if (is_new) g.states.resize(g.states.size() + s.n_aggs);
        for (int j = 0; j < s.n_aggs; ++j) {
            Val v;
            if (s.aggs[j].arg >= 0) v = vals[s.aggs[j].arg];
            Reduce(s.aggs[j], p.result_types[j], g.states[dense * s.n_aggs + j], v);
        }
    }
}

Val StateValue(const ResultType& rt, const qdb_agg_item& a, const AggState& st) {
    Val v;
    if (a.func == QDB_AGG_COUNT_STAR || a.func == QDB_AGG_COUNT) { v.i = st.count; return v; }
    if (st.count == 0) { v.null = true; return v; }
    if (rt.type == QDB_TYPE_F64) v.f = st.facc; else v.i = st.acc;
    return v;
}

// Output projection over (keys ++ aggregates) — the finalize projection of
// the plan (AVG = sum / count, qdb/plan/sql_lowering.cpp:799-814).
void EmitTable(const AggPlan& p, const GroupSet& g, oracle_table* out) {
    const qdb_aggregate_spec& s = *p.spec;
    const int64_t rows = g.table.Size();
    std::vector<int> row_types;
    std::vector<int> row_scales;
    for (int j = 0; j < s.n_keys; ++j) {
        row_types.push_back(s.nodes[s.keys[j]].type);
        row_scales.push_back(s.nodes[s.keys[j]].scale);
    }
    for (int j = 0; j < s.n_aggs; ++j) {
        row_types.push_back(p.result_types[j].type);
        row_scales.push_back(p.result_types[j].scale);
    }
    const int ncols = s.n_outputs > 0 ? s.n_outputs : int(row_types.size());
    out->rows = rows;
    out->cols = ncols;
    out->types = static_cast<int32_t*>(std::malloc(sizeof(int32_t) * std::max(1, ncols)));
    out->scales = static_cast<int32_t*>(std::malloc(sizeof(int32_t) * std::max(1, ncols)));
    out->cells = static_cast<int64_t*>(std::calloc(std::max<int64_t>(1, rows * ncols * 2), 8));
    out->valid = static_cast<uint8_t*>(std::calloc(std::max<int64_t>(1, rows * ncols), 1));
    for (int c = 0; c < ncols; ++c) {
        if (s.n_outputs > 0) {
            out->types[c] = s.output_nodes[s.outputs[c]].type;
            out->scales[c] = s.output_nodes[s.outputs[c]].scale;
        } else {
            out->types[c] = row_types[c];
            out->scales[c] = row_scales[c];
        }
    }
    std::vector<Val> rowv(row_types.size());
    std::vector<Val> tmp;
    int32_t max_out = -1;
    for (int c = 0; c < s.n_outputs; ++c) max_out = std::max(max_out, s.outputs[c]);
    const Expr oexpr{s.output_nodes, s.n_output_nodes};
    for (int64_t r = 0; r < rows; ++r) {
        for (int j = 0; j < s.n_keys; ++j) rowv[j] = g.table.group_keys[r * s.n_keys + j];
        for (int j = 0; j < s.n_aggs; ++j) {
            rowv[s.n_keys + j] = StateValue(p.result_types[j], s.aggs[j], g.states[r * s.n_aggs + j]);
        }
        const Val* cellsrc = rowv.data();
        if (s.n_outputs > 0) {
            EvalAll(oexpr, max_out, [&](int32_t c) { return rowv[c]; }, tmp);
        }
        for (int c = 0; c < ncols; ++c) {
            const Val& v = s.n_outputs > 0 ? tmp[s.outputs[c]] : cellsrc[c];
            int64_t* cell = out->cells + (r * ncols + c) * 2;
            out->valid[r * ncols + c] = v.null ? 0 : 1;
            if (v.null) continue;
            if (IsFloat(out->types[c])) std::memcpy(cell, &v.f, 8);
            else { cell[0] = int64_t(uint64_t(v.i)); cell[1] = int64_t(uint64_t(u128(v.i) >> 64)); }
        }
    }
}

// Threaded plan shape (qdb/scheduler/lowering/plan_lowerer.cpp:1671 cascade,
// qdb/exec/aggregate_exec.cpp:158-233, runtime_adapter.cpp:1001-1003): lanes
// aggregate row ranges into partial tables, partial groups are routed by
// hash % lanes, and each final lane combines its partition.
void AggregateThreaded(const AggPlan& p, const qdb_rowset& b, int lanes, GroupSet& result) {
    const qdb_aggregate_spec& s = *p.spec;
    std::vector<GroupSet> partial(lanes);
    std::vector<std::thread> th;
    for (int l = 0; l < lanes; ++l) {
        th.emplace_back([&, l] {
            partial[l].table.Init(s.n_keys, p.key_types.data(), 8);
            const int64_t begin = b.RowCount * l / lanes, end = b.RowCount * (l + 1) / lanes;
            AggregateRows(p, b, begin, end, partial[l]);
        });
    }
    for (auto& t : th) t.join();
    th.clear();
    std::vector<GroupSet> finals(lanes);
    for (int l = 0; l < lanes; ++l) {
        th.emplace_back([&, l] {
            GroupSet& f = finals[l];
            f.table.Init(s.n_keys, p.key_types.data(), 8);
            for (int src = 0; src < lanes; ++src) {
                const GroupSet& ps = partial[src];
                for (int64_t d = 0; d < ps.table.Size(); ++d) {
                    const uint64_t h = ps.table.group_hash[d];
                    if (int(h % uint64_t(lanes)) != l) continue;
                    bool is_new = false;
                    const int64_t dense = f.table.Upsert(&ps.table.group_keys[d * s.n_keys], h, is_new);
                    if (is_new) f.states.resize(f.states.size() + s.n_aggs);
                    for (int j = 0; j < s.n_aggs; ++j) {
                        Combine(s.aggs[j], p.result_types[j], f.states[dense * s.n_aggs + j],
                                ps.states[d * s.n_aggs + j]);
                    }
                }
            }
        });
    }
    for (auto& t : th) t.join();
    result.table.Init(s.n_keys, p.key_types.data(), 8);
    for (int l = 0; l < lanes; ++l) {
        const GroupSet& f = finals[l];
        for (int64_t d = 0; d < f.table.Size(); ++d) {
            bool is_new = false;
            const int64_t dense = result.table.Upsert(&f.table.group_keys[d * s.n_keys], f.table.group_hash[d], is_new);
            if (is_new) result.states.resize(result.states.size() + s.n_aggs);
            for (int j = 0; j < s.n_aggs; ++j) {
                Combine(s.aggs[j], p.result_types[j], result.states[dense * s.n_aggs + j],
                        f.states[d * s.n_aggs + j]);
            }
        }
    }
}

// A global aggregate (no keys) over an empty input still has its one group:
// COUNT 0, SUM NULL (docs/arch/aggregation.md:144-164, EmptyInputGroups).
void EnsureGlobalGroup(const AggPlan& p, GroupSet& g) {
    if (p.spec->n_keys == 0 && g.table.Size() == 0) {
        bool is_new = false;
        g.table.Upsert(nullptr, StructHash(nullptr, nullptr, 0), is_new);
        g.states.resize(p.spec->n_aggs);
    }
}

// ---------------------------------------------------------------------------
// Row table and row join (qdb/kernel/row_table.oz:140-295,
// qdb/kernel/join/join_rows.oz:70-197).
// ---------------------------------------------------------------------------
uint64_t RtMix(uint64_t h) { return h * 0x9E3779B97F4A7C15ULL; }   // rt_mix
uint64_t RtSalt(uint64_t h) { return (h >> 16) & 0xFFFF; }          // rt_salt

struct RowTable {
    std::vector<uint64_t> entries;   // salt << 48 | (row + 1)
    uint64_t mask = 0;
    int shift = 64;

    // rt_init: load factor at most 1/2, at least 1024 entries.
    void Init(int64_t rows) {
        int64_t cap = 1024;
        while (cap < rows * 2) cap *= 2;
        entries.assign(cap, 0);
        mask = uint64_t(cap - 1);
        shift = 64 - __builtin_ctzll(uint64_t(cap));
    }
    // rt_seek: walk to the first entry that is empty or carries `salt`.
    uint64_t Seek(uint64_t off, uint64_t salt, uint64_t& out_off) const {
        uint64_t e = entries[off];
        while (e != 0 && (e >> 48) != salt) {
            off = (off + 1) & mask;
            e = entries[off];
        }
        out_off = off;
        return e;
    }
};

struct JoinSide {
    const qdb_row_join_spec* spec;
    bool build;
    int n_keys;
    std::vector<int> key_cols;
    std::vector<int> key_types;
    const qdb_column_type* columns;
};

bool ReadKey(const JoinSide& side, const qdb_rowset& b, int64_t row, Val* key) {
    for (int j = 0; j < side.n_keys; ++j) {
        key[j] = ReadCell(b.Columns[side.key_cols[j]], side.columns[side.key_cols[j]], row);
        if (key[j].null) return false;   // a NULL key matches nothing
    }
    return true;
}

struct BuildArena {
    std::vector<int32_t> batch;    // arena row -> source batch
    std::vector<int64_t> row;      // arena row -> source row
    std::vector<Val> keys;         // arena row * n_keys
    std::vector<uint64_t> hash;
    std::vector<int64_t> next;     // chain of equal keys, -1 ends
};

// GenRowJoinAppendAst (qdb/kernel/join_gen.cpp:2063-2160): append the
// selected rows with a valid key (and, fused here, that pass the build
// predicate) in input order.
void AppendBuild(const JoinSide& side, const qdb_rowset* build, int32_t n_build, BuildArena& a) {
    const qdb_row_join_spec& s = *side.spec;
    const Expr fexpr{s.build_nodes, s.n_build_nodes};
    std::vector<Val> tmp;
    std::vector<Val> key(side.n_keys);
    for (int32_t bi = 0; bi < n_build; ++bi) {
        const qdb_rowset& b = build[bi];
        for (int64_t r = 0; r < b.RowCount; ++r) {
            if (b.Selection && !b.Selection[r]) continue;
            if (s.build_filter >= 0) {
                EvalAll(fexpr, s.build_filter,
                        [&](int32_t c) { return ReadCell(b.Columns[c], s.build_columns[c], r); }, tmp);
                if (tmp[s.build_filter].null || tmp[s.build_filter].i == 0) continue;
            }
            if (!ReadKey(side, b, r, key.data())) continue;
            a.batch.push_back(bi);
            a.row.push_back(r);
            a.keys.insert(a.keys.end(), key.begin(), key.end());
            a.hash.push_back(StructHash(key.data(), side.key_types.data(), side.n_keys));
        }
    }
    a.next.assign(a.row.size(), -1);
}

bool ArenaKeyEqual(const BuildArena& a, int nk, int64_t r, const Val* key, const int* types) {
    for (int j = 0; j < nk; ++j) {
        if (!KeyFieldEqual(a.keys[r * nk + j], key[j], types[j])) return false;
    }
    return true;
}

// jr_build_rows (join_rows.oz:70-113): link rows last to first so that an
// equal-key chain lists its rows in build order.
void BuildTable(const BuildArena& a, int nk, const int* types, RowTable& t, std::vector<int64_t>& next) {
    const int64_t n = int64_t(a.row.size());
    t.Init(n);
    next.assign(n, -1);
    for (int64_t r = n - 1; r >= 0; --r) {
        const uint64_t h = RtMix(a.hash[r]);
        const uint64_t salt = RtSalt(h);
        uint64_t off = 0;
        uint64_t e = t.Seek(h >> t.shift, salt, off);
        while (true) {
            if (e == 0) {
                next[r] = -1;
                t.entries[off] = (salt << 48) | uint64_t(r + 1);
                break;
            }
            const int64_t head = int64_t(e & 0xFFFFFFFFFFFFULL) - 1;
            if (ArenaKeyEqual(a, nk, head, &a.keys[r * nk], types)) {
                next[r] = head;
                t.entries[off] = (salt << 48) | uint64_t(r + 1);
                break;
            }
            off = (off + 1) & t.mask;
            e = t.Seek(off, salt, off);
        }
    }
}

// Probe (GenRowJoinProbeAst join_gen.cpp:2161-2270, rt_seek_all
// row_table.oz:260-277, jr_probe_candidates join_rows.oz:146-197): a seek
// pass over every selected valid row, then key passes; a salt collision moves
// the row on to the next pass.  Emits (probe row, build arena row).
// With emit_unmatched (an outer join streaming its preserved side), a NULL
// key is paired with build row -1 at once in the collect pass
// (join_gen.cpp:2206-2230), and a row whose seek reaches an empty entry
// after its key passes (jr_probe_candidates' emit_unmatched).
template <class Emit>
void ProbeBatch(const JoinSide& side, const BuildArena& a, const RowTable& t,
                const std::vector<int64_t>& next, const qdb_rowset& p, Emit&& emit,
                bool emit_unmatched = false) {
    const int nk = side.n_keys;
    std::vector<int64_t> rows;
    std::vector<Val> keys;
    std::vector<uint64_t> salts, offsets, found;
    std::vector<Val> key(nk);
    for (int64_t r = 0; r < p.RowCount; ++r) {
        if (p.Selection && !p.Selection[r]) continue;
        if (!ReadKey(side, p, r, key.data())) {
            if (emit_unmatched) emit(r, int64_t(-1));
            continue;
        }
        rows.push_back(r);
        keys.insert(keys.end(), key.begin(), key.end());
    }
    const int64_t count = int64_t(rows.size());
    salts.resize(count); offsets.resize(count); found.resize(count);
    for (int64_t j = 0; j < count; ++j) {
        const uint64_t h = RtMix(StructHash(&keys[j * nk], side.key_types.data(), nk));
        salts[j] = RtSalt(h);
        found[j] = t.Seek(h >> t.shift, salts[j], offsets[j]);
    }
    std::vector<int64_t> work(count);
    int64_t k = count;
    bool first = true;
    while (k > 0) {
        int64_t m = 0;
        for (int64_t q = 0; q < k; ++q) {
            const int64_t j = first ? q : work[q];
            const uint64_t e = found[j];
            if (e == 0) {
                if (emit_unmatched) emit(rows[j], int64_t(-1));
                continue;
            }
            const int64_t head = int64_t(e & 0xFFFFFFFFFFFFULL) - 1;
            if (ArenaKeyEqual(a, nk, head, &keys[j * nk], side.key_types.data())) {
                for (int64_t cur = head; cur >= 0; cur = next[cur]) emit(rows[j], cur);
            } else {
                offsets[j] = (offsets[j] + 1) & t.mask;
                work[m++] = j;
            }
        }
        k = m;
        first = false;
        for (int64_t q = 0; q < k; ++q) {   // rt_seek_work
            const int64_t j = work[q];
            found[j] = t.Seek(offsets[j], salts[j], offsets[j]);
        }
    }
}

JoinSide MakeSide(const qdb_row_join_spec& s, bool build) {
    JoinSide side;
    side.spec = &s;
    side.build = build;
    side.n_keys = s.n_keys;
    side.columns = build ? s.build_columns : s.probe_columns;
    for (int j = 0; j < s.n_keys; ++j) {
        const int c = build ? s.build_keys[j] : s.probe_keys[j];
        side.key_cols.push_back(c);
        side.key_types.push_back(side.columns[c].type);
    }
    return side;
}

// ---------------------------------------------------------------------------
// Radix sort over packed row ids (qdb/kernel/sort/radix.oz:4-123,
// sort_rowids.oz:63-228, compiler.cpp:563-600).
// ---------------------------------------------------------------------------
// qumir_radix_key: order-preserving unsigned keys; PostgreSQL float order.
uint64_t RadixKey(const Val& v, int t) {
    switch (t) {
        case QDB_TYPE_I8: return uint64_t(uint8_t(int8_t(v.i)) ^ 0x80u);
        case QDB_TYPE_I16: return uint64_t(uint16_t(int16_t(v.i)) ^ 0x8000u);
        case QDB_TYPE_I32: case QDB_TYPE_DATE32: return uint64_t(uint32_t(int32_t(v.i)) ^ 0x80000000u);
        case QDB_TYPE_I64: case QDB_TYPE_DECIMAL64: return uint64_t(int64_t(v.i)) ^ (1ULL << 63);
        case QDB_TYPE_U8: case QDB_TYPE_U16: case QDB_TYPE_U32: case QDB_TYPE_U64: case QDB_TYPE_CHAR1:
        case QDB_TYPE_BOOL:
            return uint64_t(v.i);
        case QDB_TYPE_F64: {
            uint64_t bits; std::memcpy(&bits, &v.f, 8);
            const uint64_t mag = bits & 0x7fffffffffffffffULL;
            if (mag > 0x7ff0000000000000ULL) return ~0ULL;
            if (mag == 0) bits = 0;
            return (bits >> 63) ? ~bits : (bits ^ (1ULL << 63));
        }
        case QDB_TYPE_F32: {
            float f = float(v.f);
            uint32_t bits; std::memcpy(&bits, &f, 4);
            const uint32_t mag = bits & 0x7fffffffu;
            if (mag > 0x7f800000u) return 0xffffffffULL;
            if (mag == 0) bits = 0;
            return uint64_t((bits >> 31) ? ~bits : (bits ^ 0x80000000u));
        }
    }
    throw Error("unsupported sort key type");
}

int KeyBits(int t) {
    if (t == QDB_TYPE_BOOL) return 8;
    return WidthBits(t) <= 32 ? std::max(8, WidthBits(t)) : 64;
}

// sr_keyed_count_pass + sr_keyed_sort: stable LSD over 8-bit digits; a digit
// that is the same for every key is skipped; DESC walks buckets downwards.
void KeyedSort(std::vector<uint64_t>& keys, std::vector<int64_t>& ids, int key_bits, bool desc) {
    const int64_t n = int64_t(keys.size());
    std::vector<uint64_t> kout(n);
    std::vector<int64_t> iout(n);
    std::vector<uint64_t> counts(256);
    for (int digit = 0; digit < key_bits; digit += 8) {
        std::fill(counts.begin(), counts.end(), 0);
        for (int64_t i = 0; i < n; ++i) ++counts[(keys[i] >> digit) & 255];
        bool constant = false;
        uint64_t offset = 0;
        for (int i = 0; i < 256; ++i) {
            const int bucket = desc ? 255 - i : i;
            const uint64_t c = counts[bucket];
            if (int64_t(c) == n) { constant = true; break; }
            counts[bucket] = offset;
            offset += c;
        }
        if (constant) continue;
        for (int64_t i = 0; i < n; ++i) {
            const uint64_t b = (keys[i] >> digit) & 255;
            const uint64_t place = counts[b]++;
            kout[place] = keys[i];
            iout[place] = ids[i];
        }
        keys.swap(kout);
        ids.swap(iout);
    }
}

Val StoreCell(const qdb_sort_spec& s, const qdb_rowset* store, int64_t packed, int col) {
    const int32_t batch = int32_t(packed >> 32);
    const int32_t row = int32_t(uint32_t(packed & 0xffffffffu));
    return ReadCell(store[batch].Columns[col], s.columns[col], row);
}

// sr_sort_compare (qdb/kernel/sort/sort_rowids.oz:616-650): memcmp over the
// common length, then the shorter first.
int StringCompare(const Val& a, const Val& b) {
    const int64_t m = std::min(a.n, b.n);
    for (int64_t i = 0; i < m; ++i) {
        if (a.s[i] != b.s[i]) return a.s[i] < b.s[i] ? -1 : 1;
    }
    return a.n < b.n ? -1 : (a.n > b.n ? 1 : 0);
}

// sort_string_rowids / sort_string_rowids_nullable (sort_rowids.oz:876-1060):
// (8-byte big-endian prefix, row id) pairs through eight stable byte passes
// (DESC walks the buckets downwards; NULLs in bucket 0 or 256 by
// nulls_first), then every run of equal prefixes among the valid rows is
// ordered stably by the full comparison (sr_pair_tiebreak_runs, :818-846).
void SortStringKey(const qdb_sort_spec& s, const qdb_rowset* store, std::vector<int64_t>& ids, int col, bool desc,
                   bool nulls_first) {
    const size_t n = ids.size();
    std::vector<Val> cell(n);
    std::vector<uint64_t> prefix(n, 0);
    for (size_t i = 0; i < n; ++i) {
        cell[i] = StoreCell(s, store, ids[i], col);
        if (cell[i].null) continue;
        const int64_t lim = std::min<int64_t>(cell[i].n, 8);
        uint64_t p = 0;
        for (int64_t j = 0; j < lim; ++j) p = (p << 8) | cell[i].s[j];
        prefix[i] = p << (8 * (8 - lim));
    }
    std::vector<size_t> order(n), tmp(n);
    for (size_t i = 0; i < n; ++i) order[i] = i;
    for (int digit = 0; digit < 64; digit += 8) {
        std::vector<size_t> count(259, 0);   // buckets 0 .. 257, shifted by one
        auto bucket = [&](size_t i) -> size_t {
            if (cell[i].null) return nulls_first ? 0 : 257;
            size_t b = size_t((prefix[i] >> digit) & 255);
            if (desc) b = 255 - b;
            return b + 1;
        };
        for (size_t i : order) ++count[bucket(i) + 1];
        for (size_t b = 1; b < count.size(); ++b) count[b] += count[b - 1];
        for (size_t i : order) tmp[count[bucket(i)]++] = i;
        order.swap(tmp);
    }
    size_t lo = 0, hi = n;
    while (lo < hi && cell[order[lo]].null) ++lo;
    while (lo < hi && cell[order[hi - 1]].null) --hi;
    for (size_t a = lo; a < hi;) {
        size_t b = a + 1;
        while (b < hi && prefix[order[b]] == prefix[order[a]]) ++b;
        if (b - a > 1) {
            std::stable_sort(order.begin() + std::ptrdiff_t(a), order.begin() + std::ptrdiff_t(b),
                             [&](size_t x, size_t y) {
                                 const int c = StringCompare(cell[x], cell[y]);
                                 return desc ? c > 0 : c < 0;
                             });
        }
        a = b;
    }
    std::vector<int64_t> out(n);
    for (size_t i = 0; i < n; ++i) out[i] = ids[order[i]];
    ids.swap(out);
}

// sort_fixed_rowids(_nullable) for one key: NULL rows keep input order at
// the chosen end, valid rows are LSD-sorted (strings: SortStringKey).
void SortOneKey(const qdb_sort_spec& s, const qdb_rowset* store, std::vector<int64_t>& ids,
                int col, bool desc, bool nulls_first) {
    const int t = s.columns[col].type;
    if (t == QDB_TYPE_DECIMAL128) throw Error("DECIMAL128 sort keys are not restated");
    if (t == QDB_TYPE_STRING) {
        SortStringKey(s, store, ids, col, desc, nulls_first);
        return;
    }
    std::vector<uint64_t> keys;
    std::vector<int64_t> valid_ids, null_ids;
    for (int64_t id : ids) {
        const Val v = StoreCell(s, store, id, col);
        if (v.null) { null_ids.push_back(id); continue; }
        valid_ids.push_back(id);
        keys.push_back(RadixKey(v, t));
    }
    KeyedSort(keys, valid_ids, KeyBits(t), desc);
    ids.clear();
    if (nulls_first) { ids = null_ids; ids.insert(ids.end(), valid_ids.begin(), valid_ids.end()); }
    else { ids = valid_ids; ids.insert(ids.end(), null_ids.begin(), null_ids.end()); }
}

// Key order only (AppendSortLessBody, qdb/kernel/compiler.cpp:700-753): true
// when row a's keys come strictly before row b's.
bool KeysLess(const qdb_sort_spec& s, const qdb_rowset* store, int64_t a, int64_t b) {
    for (int k = 0; k < s.n_keys; ++k) {
        const int col = s.keys[k].column;
        const int t = s.columns[col].type;
        const Val x = StoreCell(s, store, a, col), y = StoreCell(s, store, b, col);
        const bool desc = s.keys[k].desc, nf = s.keys[k].nulls_first;
        if (x.null || y.null) {
            if (x.null && y.null) continue;
            return x.null ? nf : !nf;
        }
        const uint64_t kx = RadixKey(x, t), ky = RadixKey(y, t);
        if (kx == ky) continue;
        return desc ? kx > ky : kx < ky;
    }
    return false;
}

// SortRowsLess (qdb/exec/sort_exec.cpp:126-293) with the packed row id as the
// final tie break (qdb/kernel/compiler.h:135-148).
bool RowLess(const qdb_sort_spec& s, const qdb_rowset* store, const bool* descs,
             const bool* nulls_firsts, int64_t a, int64_t b) {
    for (int k = 0; k < s.n_keys; ++k) {
        const int col = s.keys[k].column;
        const int t = s.columns[col].type;
        const Val x = StoreCell(s, store, a, col), y = StoreCell(s, store, b, col);
        const bool desc = descs ? descs[k] : s.keys[k].desc;
        const bool nf = nulls_firsts ? nulls_firsts[k] : s.keys[k].nulls_first;
        if (x.null || y.null) {
            if (x.null && y.null) continue;
            return x.null ? nf : !nf;
        }
        const uint64_t kx = RadixKey(x, t), ky = RadixKey(y, t);
        if (kx == ky) continue;
        return desc ? kx > ky : kx < ky;
    }
    return a < b;
}

void SiftDown(std::vector<int64_t>& h, int64_t size, int64_t i,
              const std::function<bool(int64_t, int64_t)>& less) {
    // Max-heap under `less`: the root is the last kept row of the order.
    while (true) {
        const int64_t l = 2 * i + 1, r = l + 1;
        int64_t big = i;
        if (l < size && less(h[big], h[l])) big = l;
        if (r < size && less(h[big], h[r])) big = r;
        if (big == i) return;
        std::swap(h[i], h[big]);
        i = big;
    }
}

}  // namespace

// ===========================================================================
// C API
// ===========================================================================
extern "C" {

void oracle_table_free(oracle_table* t) {
    if (!t) return;
    std::free(t->types);
    std::free(t->scales);
    std::free(t->cells);
    std::free(t->valid);
    std::memset(t, 0, sizeof(*t));
}

int oracle_aggregate(const qdb_aggregate_spec* spec, const qdb_rowset* batches, int32_t n_batches,
                     int32_t lanes, oracle_table* out, char* err, size_t err_len) {
    try {
        const AggPlan p = MakePlan(*spec);
        GroupSet g;
        if (lanes <= 1 || n_batches != 1) {
            g.table.Init(spec->n_keys, p.key_types.data(), 8);
            for (int32_t b = 0; b < n_batches; ++b) AggregateRows(p, batches[b], 0, batches[b].RowCount, g);
        } else {
            AggregateThreaded(p, batches[0], lanes, g);
        }
        EnsureGlobalGroup(p, g);
        EmitTable(p, g, out);
        return 0;
    } catch (const std::exception& e) {
        SetErr(err, err_len, e.what());
        return -1;
    }
}

int oracle_filter(int32_t n_columns, const qdb_column_type* columns, int32_t n_nodes,
                  const qdb_expr* nodes, int32_t predicate, const qdb_rowset* batch,
                  uint8_t* selection, char* err, size_t err_len) {
    (void)n_columns;
    try {
        const Expr e{nodes, n_nodes};
        std::vector<Val> vals;
        for (int64_t r = 0; r < batch->RowCount; ++r) {
            if (batch->Selection && !batch->Selection[r]) { selection[r] = 0; continue; }
            EvalAll(e, predicate, [&](int32_t c) { return ReadCell(batch->Columns[c], columns[c], r); }, vals);
            selection[r] = (!vals[predicate].null && vals[predicate].i) ? 1 : 0;
        }
        return 0;
    } catch (const std::exception& ex) {
        SetErr(err, err_len, ex.what());
        return -1;
    }
}

int oracle_project(int32_t n_columns, const qdb_column_type* columns, int32_t n_nodes,
                   const qdb_expr* nodes, int32_t n_exprs, const int32_t* exprs,
                   const qdb_rowset* batch, void** out_buffers, uint8_t** out_valid,
                   char* err, size_t err_len) {
    (void)n_columns;
    try {
        const Expr e{nodes, n_nodes};
        int32_t root = -1;
        for (int k = 0; k < n_exprs; ++k) root = std::max(root, exprs[k]);
        std::vector<Val> vals;
        for (int64_t r = 0; r < batch->RowCount; ++r) {
            if (batch->Selection && !batch->Selection[r]) continue;
            EvalAll(e, root, [&](int32_t c) { return ReadCell(batch->Columns[c], columns[c], r); }, vals);
            for (int k = 0; k < n_exprs; ++k) {
                const qdb_expr& n = nodes[exprs[k]];
                const Val& v = vals[exprs[k]];
                if (out_valid && out_valid[k]) out_valid[k][r] = v.null ? 0 : 1;
                char* base = static_cast<char*>(out_buffers[k]);
                const int w = StorageBytes(n.type);
                if (v.null) { std::memset(base + r * w, 0, w); continue; }
                if (n.type == QDB_TYPE_F64) std::memcpy(base + r * 8, &v.f, 8);
                else if (n.type == QDB_TYPE_F32) { const float f = float(v.f); std::memcpy(base + r * 4, &f, 4); }
                else if (n.type == QDB_TYPE_DECIMAL128) {
                    const uint64_t w2[2] = {uint64_t(v.i), uint64_t(u128(v.i) >> 64)};
                    std::memcpy(base + r * 16, w2, 16);
                } else {
                    const uint64_t x = uint64_t(v.i);
                    std::memcpy(base + r * w, &x, w);
                }
            }
        }
        return 0;
    } catch (const std::exception& ex) {
        SetErr(err, err_len, ex.what());
        return -1;
    }
}

int oracle_hash(int32_t n_columns, const qdb_column_type* columns, int32_t n_keys,
                const int32_t* key_columns, const qdb_rowset* batch, uint64_t* hashes,
                char* err, size_t err_len) {
    (void)n_columns;
    try {
        std::vector<Val> key(n_keys);
        std::vector<int> types(n_keys);
        std::unique_ptr<bool[]> nullable(new bool[size_t(n_keys)]);
        for (int j = 0; j < n_keys; ++j) {
            types[j] = columns[key_columns[j]].type;
            nullable[j] = columns[key_columns[j]].nullable != 0;
        }
        for (int64_t r = 0; r < batch->RowCount; ++r) {
            if (batch->Selection && !batch->Selection[r]) continue;
            for (int j = 0; j < n_keys; ++j) {
                key[j] = ReadCell(batch->Columns[key_columns[j]], columns[key_columns[j]], r);
            }
            hashes[r] = StructHash(key.data(), types.data(), n_keys, nullable.get());
        }
        return 0;
    } catch (const std::exception& ex) {
        SetErr(err, err_len, ex.what());
        return -1;
    }
}

int64_t oracle_row_join(const qdb_row_join_spec* spec, const qdb_rowset* build, int32_t n_build,
                        const qdb_rowset* probe, int64_t* pairs, int64_t pair_cap,
                        char* err, size_t err_len) {
    try {
        const JoinSide bs = MakeSide(*spec, true), ps = MakeSide(*spec, false);
        BuildArena a;
        AppendBuild(bs, build, n_build, a);
        RowTable t;
        std::vector<int64_t> next;
        BuildTable(a, bs.n_keys, bs.key_types.data(), t, next);
        int64_t count = 0;
        ProbeBatch(ps, a, t, next, *probe, [&](int64_t prow, int64_t brow) {
            if (pairs && count < pair_cap) {
                pairs[2 * count] = prow;
                pairs[2 * count + 1] = brow;
            }
            ++count;
        });
        return count;
    } catch (const std::exception& e) {
        SetErr(err, err_len, e.what());
        return -1;
    }
}

int64_t oracle_row_join_typed(const qdb_row_join_spec* spec, const qdb_rowset* build, int32_t n_build,
                              const qdb_rowset* probe, int32_t n_probe, int64_t* pairs, int64_t pair_cap,
                              char* err, size_t err_len) {
    try {
        // CompileRowJoin's served shapes (qdb/kernel/compiler.cpp:3134-3148).
        const int jt = spec->join_type;
        const bool preserved = spec->build_is_left ? jt == QDB_JOIN_RIGHT : jt == QDB_JOIN_LEFT;
        const bool marks = spec->build_is_left && (jt == QDB_JOIN_LEFT_SEMI || jt == QDB_JOIN_LEFT_ANTI);
        if (jt != QDB_JOIN_INNER && !preserved && !marks) throw Error("join type not served by the row join");
        const JoinSide bs = MakeSide(*spec, true), ps = MakeSide(*spec, false);
        BuildArena a;
        AppendBuild(bs, build, n_build, a);
        RowTable t;
        std::vector<int64_t> next;
        BuildTable(a, bs.n_keys, bs.key_types.data(), t, next);
        std::vector<int64_t> first_row(size_t(n_build) + 1, 0);
        for (int32_t b = 0; b < n_build; ++b) first_row[b + 1] = first_row[b] + build[b].RowCount;
        auto source_row = [&](int64_t arena_row) { return first_row[a.batch[arena_row]] + a.row[arena_row]; };
        int64_t count = 0;
        auto push = [&](int64_t left, int64_t right) {
            if (pairs && count < pair_cap) {
                pairs[2 * count] = left;
                pairs[2 * count + 1] = right;
            }
            ++count;
        };
        std::vector<uint8_t> marked(a.row.size(), 0);
        for (int32_t pb = 0; pb < n_probe; ++pb) {
            ProbeBatch(ps, a, t, next, probe[pb], [&](int64_t prow, int64_t brow) {
                if (marks) {
                    if (brow >= 0) marked[size_t(brow)] = 1;   // jr_mark_chain: every row of the chain
                    return;
                }
                push((int64_t(pb) << 32) | prow, brow < 0 ? -1 : source_row(brow));
            }, preserved);
        }
        if (marks) {
            // jr_emit_by_mark (join_rows.oz:199-224) in build order, then the
            // NULL-key arena of an ANTI join (jr_append_null_keys), all of it.
            const bool semi = jt == QDB_JOIN_LEFT_SEMI;
            for (size_t r = 0; r < a.row.size(); ++r) {
                if ((marked[r] != 0) == semi) push(-1, source_row(int64_t(r)));
            }
            if (!semi) {
                const qdb_row_join_spec& js = *spec;
                const Expr fexpr{js.build_nodes, js.n_build_nodes};
                std::vector<Val> tmp, key(size_t(bs.n_keys));
                for (int32_t bi = 0; bi < n_build; ++bi) {
                    const qdb_rowset& b = build[bi];
                    for (int64_t r = 0; r < b.RowCount; ++r) {
                        if (b.Selection && !b.Selection[r]) continue;
                        if (js.build_filter >= 0) {
                            EvalAll(fexpr, js.build_filter,
                                    [&](int32_t c) { return ReadCell(b.Columns[c], js.build_columns[c], r); }, tmp);
                            if (tmp[js.build_filter].null || tmp[js.build_filter].i == 0) continue;
                        }
                        if (ReadKey(bs, b, r, key.data())) continue;
                        push(-1, first_row[bi] + r);
                    }
                }
            }
        }
        return count;
    } catch (const std::exception& e) {
        SetErr(err, err_len, e.what());
        return -1;
    }
}

int oracle_join_aggregate(const qdb_row_join_spec* join, const qdb_aggregate_spec* agg,
                          const qdb_rowset* build, int32_t n_build, const qdb_rowset* probe,
                          int32_t n_probe, int32_t lanes, oracle_table* out, char* err, size_t err_len) {
    (void)lanes;
    try {
        const JoinSide bs = MakeSide(*join, true), ps = MakeSide(*join, false);
        BuildArena a;
        AppendBuild(bs, build, n_build, a);
        RowTable t;
        std::vector<int64_t> next;
        BuildTable(a, bs.n_keys, bs.key_types.data(), t, next);
        const AggPlan p = MakePlan(*agg);
        GroupSet g;
        g.table.Init(agg->n_keys, p.key_types.data(), 8);
        const int np = join->n_probe_columns;
        std::vector<Val> vals;
        std::vector<Val> key(std::max(1, agg->n_keys));
        for (int32_t pb = 0; pb < n_probe; ++pb) {
            const qdb_rowset& pr = probe[pb];
            ProbeBatch(ps, a, t, next, pr, [&](int64_t prow, int64_t brow) {
                auto leaf = [&](int32_t c) -> Val {
                    if (c < np) return ReadCell(pr.Columns[c], join->probe_columns[c], prow);
                    const int bc = join->build_payload[c - np];
                    const qdb_rowset& bb = build[a.batch[brow]];
                    return ReadCell(bb.Columns[bc], join->build_columns[bc], a.row[brow]);
                };
                if (p.max_root >= 0) EvalAll(p.expr, p.max_root, leaf, vals);
                if (agg->filter >= 0 && (vals[agg->filter].null || vals[agg->filter].i == 0)) return;
                for (int j = 0; j < agg->n_keys; ++j) key[j] = vals[agg->keys[j]];
                bool is_new = false;
                const int64_t dense = g.table.Upsert(key.data(),
                    StructHash(key.data(), p.key_types.data(), agg->n_keys), is_new);
                if (is_new) g.states.resize(g.states.size() + agg->n_aggs);
                for (int j = 0; j < agg->n_aggs; ++j) {
                    Val v;
                    if (agg->aggs[j].arg >= 0) v = vals[agg->aggs[j].arg];
                    Reduce(agg->aggs[j], p.result_types[j], g.states[dense * agg->n_aggs + j], v);
                }
            });
        }
        EnsureGlobalGroup(p, g);
        EmitTable(p, g, out);
        return 0;
    } catch (const std::exception& e) {
        SetErr(err, err_len, e.what());
        return -1;
    }
}

int oracle_sort(const qdb_sort_spec* spec, const qdb_rowset* store, int64_t* row_ids, int64_t n,
                const bool* descs, const bool* nulls_firsts, char* err, size_t err_len) {
    try {
        std::vector<int64_t> ids(row_ids, row_ids + n);
        // Least significant key first (compiler.cpp:595-599).
        for (int k = spec->n_keys - 1; k >= 0; --k) {
            const bool desc = descs ? descs[k] : spec->keys[k].desc;
            const bool nf = nulls_firsts ? nulls_firsts[k] : spec->keys[k].nulls_first;
            SortOneKey(*spec, store, ids, spec->keys[k].column, desc, nf);
        }
        std::memcpy(row_ids, ids.data(), sizeof(int64_t) * n);
        return 0;
    } catch (const std::exception& e) {
        SetErr(err, err_len, e.what());
        return -1;
    }
}

int64_t oracle_top_k(const qdb_sort_spec* spec, const qdb_rowset* store, int64_t* row_ids,
                     int64_t size, int64_t limit, const bool* descs, const bool* nulls_firsts) {
    if (size <= 0 || limit <= 0) return 0;
    std::function<bool(int64_t, int64_t)> less = [&](int64_t a, int64_t b) {
        return RowLess(*spec, store, descs, nulls_firsts, a, b);
    };
    // heap_top_k (heap.oz:156-188): heapify the first K, replace the top with
    // every later row that precedes it, then pop the heap into order.
    std::vector<int64_t> h(row_ids, row_ids + size);
    const int64_t kept = std::min(limit, size);
    for (int64_t i = kept / 2 - 1; i >= 0; --i) SiftDown(h, kept, i, less);
    for (int64_t cur = kept; cur < size; ++cur) {
        if (less(h[cur], h[0])) {
            h[0] = h[cur];
            SiftDown(h, kept, 0, less);
        }
    }
    for (int64_t hs = kept; hs > 1; --hs) {
        std::swap(h[0], h[hs - 1]);
        SiftDown(h, hs - 1, 0, less);
    }
    std::memcpy(row_ids, h.data(), sizeof(int64_t) * kept);
    return kept;
}

int64_t oracle_top_sort_update(const qdb_sort_spec* spec, const qdb_rowset* state, const qdb_rowset* batch,
                               int64_t* row_ids, int64_t n, bool sort_input, uint8_t* pick_src,
                               uint32_t* pick_idx, int64_t limit, char* err, size_t err_len) {
    try {
        // qdb_top_sort_update (BuildTopSortUpdateAst, compiler.cpp:881-975):
        // sort the batch's row ids when asked (keys last to first, stable),
        // then top_sort_merge_picks (qdb/kernel/sort/top_sort.oz:15-57).
        if (sort_input && n > 0) {
            std::vector<int64_t> ids(row_ids, row_ids + n);
            for (int k = spec->n_keys - 1; k >= 0; --k) {
                SortOneKey(*spec, batch, ids, spec->keys[k].column, spec->keys[k].desc, spec->keys[k].nulls_first);
            }
            std::memcpy(row_ids, ids.data(), sizeof(int64_t) * size_t(n));
        }
        const qdb_rowset both[2] = {*state, *batch};
        const int64_t state_n = state->RowCount;
        int64_t left = 0, right = 0, out = 0;
        while (out < limit && (left < state_n || right < n)) {
            bool take_temp;
            if (right == n) take_temp = false;
            else if (left == state_n) take_temp = true;
            else {
                // qdb_top_sort_temp_before_state: the batch row strictly first.
                const int64_t temp_row = int64_t(uint32_t(row_ids[right]));
                take_temp = KeysLess(*spec, both, (int64_t(1) << 32) | temp_row, left);
            }
            if (take_temp) {
                pick_src[out] = 1;
                pick_idx[out] = uint32_t(row_ids[right]);
                ++right;
            } else {
                pick_src[out] = 0;
                pick_idx[out] = uint32_t(left);
                ++left;
            }
            ++out;
        }
        return out;
    } catch (const std::exception& e) {
        SetErr(err, err_len, e.what());
        return -1;
    }
}

double oracle_bench_aggregate(const qdb_aggregate_spec* spec, const qdb_rowset* batch, int32_t threads,
                              int64_t* groups_out) {
    try {
        const AggPlan p = MakePlan(*spec);
        const auto t0 = std::chrono::steady_clock::now();
        GroupSet g;
        AggregateThreaded(p, *batch, std::max(1, threads), g);
        const auto t1 = std::chrono::steady_clock::now();
        if (groups_out) *groups_out = g.table.Size();
        return std::chrono::duration<double>(t1 - t0).count();
    } catch (...) {
        return -1.0;
    }
}

// Threaded join plan shape (docs/arch/scheduler_runtime.md:270-289): build
// rows partitioned by hash % P, one row table per partition, probe lanes route
// each probe row to its partition's table.  Fused SUM(payload * value), COUNT.
double oracle_bench_join_sum(const int64_t* b_key, const int64_t* b_payload, const int32_t* b_attr,
                             int64_t build_rows, int32_t attr_lt, const int64_t* p_fk,
                             const int64_t* p_value, int64_t probe_rows, int32_t threads,
                             int64_t* sum_out, int64_t* count_out) {
    const int P = std::max(1, threads);
    const auto t0 = std::chrono::steady_clock::now();
    struct Part {
        std::vector<int64_t> key, payload;
        std::vector<int64_t> next;
        RowTable t;
    };
    std::vector<Part> parts(P);
    std::vector<std::thread> th;
    for (int l = 0; l < P; ++l) {
        th.emplace_back([&, l] {
            Part& pt = parts[l];
            for (int64_t r = 0; r < build_rows; ++r) {
                if (b_attr[r] >= attr_lt) continue;
                Val v; v.i = b_key[r];
                const int ty = QDB_TYPE_I64;
                const uint64_t kh = StructHash(&v, &ty, 1);
                if (int(kh % uint64_t(P)) != l) continue;
                pt.key.push_back(b_key[r]);
                pt.payload.push_back(b_payload[r]);
            }
            const int64_t n = int64_t(pt.key.size());
            pt.t.Init(n);
            pt.next.assign(n, -1);
            for (int64_t r = n - 1; r >= 0; --r) {
                Val v; v.i = pt.key[r];
                const int ty = QDB_TYPE_I64;
                const uint64_t h = RtMix(StructHash(&v, &ty, 1));
                const uint64_t salt = RtSalt(h);
                uint64_t off = 0;
                uint64_t e = pt.t.Seek(h >> pt.t.shift, salt, off);
                while (true) {
                    if (e == 0) { pt.t.entries[off] = (salt << 48) | uint64_t(r + 1); break; }
                    const int64_t head = int64_t(e & 0xFFFFFFFFFFFFULL) - 1;
                    if (pt.key[head] == pt.key[r]) {
                        pt.next[r] = head;
                        pt.t.entries[off] = (salt << 48) | uint64_t(r + 1);
                        break;
                    }
                    off = (off + 1) & pt.t.mask;
                    e = pt.t.Seek(off, salt, off);
                }
            }
        });
    }
    for (auto& t : th) t.join();
    th.clear();
    std::vector<int64_t> sums(P, 0), counts(P, 0);
    for (int l = 0; l < P; ++l) {
        th.emplace_back([&, l] {
            int64_t sum = 0, cnt = 0;
            const int64_t begin = probe_rows * l / P, end = probe_rows * (l + 1) / P;
            const int ty = QDB_TYPE_I64;
            for (int64_t r = begin; r < end; ++r) {
                Val v; v.i = p_fk[r];
                const uint64_t kh = StructHash(&v, &ty, 1);
                const Part& pt = parts[kh % uint64_t(P)];
                const uint64_t h = RtMix(kh);
                const uint64_t salt = RtSalt(h);
                uint64_t off = 0;
                uint64_t e = pt.t.Seek(h >> pt.t.shift, salt, off);
                while (e != 0) {
                    const int64_t head = int64_t(e & 0xFFFFFFFFFFFFULL) - 1;
                    if (pt.key[head] == p_fk[r]) {
                        for (int64_t cur = head; cur >= 0; cur = pt.next[cur]) {
                            sum += pt.payload[cur] * p_value[r];
                            ++cnt;
                        }
                        break;
                    }
                    off = (off + 1) & pt.t.mask;
                    e = pt.t.Seek(off, salt, off);
                }
            }
            sums[l] = sum;
            counts[l] = cnt;
        });
    }
    for (auto& t : th) t.join();
    const auto t1 = std::chrono::steady_clock::now();
    int64_t sum = 0, cnt = 0;
    for (int l = 0; l < P; ++l) { sum += sums[l]; cnt += counts[l]; }
    if (sum_out) *sum_out = sum;
    if (count_out) *count_out = cnt;
    return std::chrono::duration<double>(t1 - t0).count();
}

// Threaded sort plan shape (BuildSortMerge plan_lowerer.cpp:2133-2211): each
// lane LSD-sorts its range by k2 ASC then k1 DESC (pass skipping as in
// sr_keyed_count_pass), then a heap k-way merge (TMergeProcessor::Finish,
// sort_exec.cpp:521+) with the row id as the tie break.
double oracle_bench_sort(const int64_t* k1, const int32_t* k2, int64_t rows, int32_t threads,
                         int64_t* rowids_out) {
    const int L = std::max(1, threads);
    const auto t0 = std::chrono::steady_clock::now();
    std::vector<std::vector<int64_t>> runs(L);
    std::vector<std::thread> th;
    for (int l = 0; l < L; ++l) {
        th.emplace_back([&, l] {
            const int64_t begin = rows * l / L, end = rows * (l + 1) / L;
            std::vector<int64_t> ids(end - begin);
            std::vector<uint64_t> keys(end - begin);
            for (int64_t i = begin; i < end; ++i) {
                ids[i - begin] = i;
                keys[i - begin] = uint64_t(uint32_t(k2[i]) ^ 0x80000000u);
            }
            KeyedSort(keys, ids, 32, false);
            for (int64_t i = 0; i < end - begin; ++i) keys[i] = uint64_t(k1[ids[i]]) ^ (1ULL << 63);
            KeyedSort(keys, ids, 64, true);
            runs[l].swap(ids);
        });
    }
    for (auto& t : th) t.join();
    auto before = [&](int64_t a, int64_t b) {
        if (k1[a] != k1[b]) return k1[a] > k1[b];
        if (k2[a] != k2[b]) return k2[a] < k2[b];
        return a < b;
    };
    using Item = std::pair<int64_t, int>;   // (row, run)
    auto cmp = [&](const Item& x, const Item& y) { return before(y.first, x.first); };
    std::priority_queue<Item, std::vector<Item>, decltype(cmp)> pq(cmp);
    std::vector<size_t> pos(L, 0);
    for (int l = 0; l < L; ++l) if (!runs[l].empty()) pq.push({runs[l][0], l});
    int64_t o = 0;
    while (!pq.empty()) {
        const Item it = pq.top();
        pq.pop();
        if (rowids_out) rowids_out[o] = it.first;
        ++o;
        if (++pos[it.second] < runs[it.second].size()) pq.push({runs[it.second][pos[it.second]], it.second});
    }
    const auto t1 = std::chrono::steady_clock::now();
    return std::chrono::duration<double>(t1 - t0).count();
}


// ---------------------------------------------------------------------------
// Runtime join filter (qdb/kernel/join/runtime_filter.oz), on host memory.
// ---------------------------------------------------------------------------
static uint64_t RfMixHost(uint64_t v) {   // rf_mix (:78-84)
    v ^= v >> 30;
    v *= 0xbf58476d1ce4e5b9ULL;
    v ^= v >> 27;
    v *= 0x94d049bb133111ebULL;
    return v ^ (v >> 31);
}

static bool RfSelected(const uint8_t* sel, int64_t r) { return sel == nullptr || sel[r] != 0; }

// rf_bloom_base / rf_bloom_bits / rf_bloom_bit (:88-106) and rf_bloom_add (:126-147).
static void RfBloomAdd(uint64_t* words, int64_t nwords, const uint64_t* hashes, const uint8_t* sel, int64_t n) {
    const uint64_t block_mask = uint64_t(nwords / 8 - 1);
    for (int64_t r = 0; r < n; ++r) {
        if (!RfSelected(sel, r)) continue;
        const uint64_t h = hashes[r];
        const uint64_t base = (RfMixHost(h) & block_mask) * 8;
        const uint64_t bits = RfMixHost(h ^ 0x9e3779b97f4a7c15ULL);
        for (int w = 0; w < 8; ++w) words[base + w] |= 1ULL << ((bits >> (8 * w)) & 63);
    }
}

static bool RfBloomContains(const uint64_t* words, int64_t nwords, uint64_t h) {   // :114-124
    const uint64_t block_mask = uint64_t(nwords / 8 - 1);
    const uint64_t base = (RfMixHost(h) & block_mask) * 8;
    const uint64_t bits = RfMixHost(h ^ 0x9e3779b97f4a7c15ULL);
    for (int w = 0; w < 8; ++w) {
        if ((words[base + w] & (1ULL << ((bits >> (8 * w)) & 63))) == 0) return false;
    }
    return true;
}

// rf_exact_stored / rf_exact_slot (:257-279).
static uint64_t RfStored(uint64_t h) { return h == 0 ? 1 : h; }
static int64_t RfExactSlot(const uint64_t* table, uint64_t mask, uint64_t h) {
    const uint64_t stored = RfStored(h);
    uint64_t slot = h & mask;
    while (table[slot] != 0 && table[slot] != stored) slot = (slot + 1) & mask;
    return int64_t(slot);
}

// The dedup set (:336-396): ctrl 0x80 marks an empty slot; a probe walks
// from mix(h) & (capacity - 1).  Only membership is observable.
static bool RfSetInsert(uint8_t* ctrl, uint64_t* slots, int64_t capacity, uint64_t h) {
    const uint64_t mask = uint64_t(capacity - 1);
    uint64_t slot = RfMixHost(h) & mask;
    for (int64_t p = 0; p < capacity; ++p) {
        if (ctrl[slot] == 0x80) {
            ctrl[slot] = uint8_t(RfMixHost(h) & 127);
            slots[slot] = h;
            return true;
        }
        if (slots[slot] == h) return false;
        slot = (slot + 1) & mask;
    }
    return false;
}

static void RfSetFill(uint8_t* ctrl, uint64_t* slots, int64_t capacity, const uint64_t* keys, int64_t n) {
    std::fill(ctrl, ctrl + capacity, uint8_t(0x80));
    for (int64_t i = 0; i < n; ++i) RfSetInsert(ctrl, slots, capacity, keys[i]);
}

int64_t oracle_rf_build(qdb_rf_build_state* st, const uint64_t* hashes, const uint8_t* sel, int64_t count) {
    // rf_build (:419-499).
    const int64_t max_keys = st->MaxKeys;
    uint64_t* keys = st->Keys;
    int64_t row = 0;
    st->Want = 0;
    if (st->Mode == 0) {
        const int64_t limit = max_keys * 2;
        int64_t used = st->KeyCount;
        while (row < count && used < limit) {
            if (RfSelected(sel, row)) keys[used++] = hashes[row];
            ++row;
        }
        st->KeyCount = used;
        if (used < limit) return row;
        if (st->SetCapacity == 0) {
            st->Want = 1;
            return row;
        }
        // rf_keys_sort_unique (:307-333).
        std::sort(keys, keys + used);
        used = int64_t(std::unique(keys, keys + used) - keys);
        st->KeyCount = used;
        if (used > max_keys) {
            st->Mode = 2;
        } else {
            RfSetFill(st->SetCtrl, st->SetSlots, st->SetCapacity, keys, used);
            st->Mode = 1;
        }
    }
    if (st->Mode == 1) {
        int64_t used = st->KeyCount;
        while (row < count && used <= max_keys) {
            if (RfSelected(sel, row) && RfSetInsert(st->SetCtrl, st->SetSlots, st->SetCapacity, hashes[row])) {
                keys[used++] = hashes[row];
            }
            ++row;
        }
        st->KeyCount = used;
        if (used <= max_keys) return row;
        st->Mode = 2;
    }
    if (st->Mode == 2) {
        if (st->BloomWords < 0) {
            st->Want = 2;
            return row;
        }
        if (st->BloomWords > 0) RfBloomAdd(st->Bloom, st->BloomWords, keys, nullptr, st->KeyCount);
        st->KeyCount = 0;
        st->Mode = 3;
    }
    if (st->BloomWords > 0) RfBloomAdd(st->Bloom, st->BloomWords, hashes, sel, count);
    return count;
}

int64_t oracle_rf_publish(qdb_rf_publish_state* st, const qdb_rf_partial* partials, int64_t n) {
    // rf_publish (:502-556).
    st->Kind = 0;
    if (st->BloomSeeded == 0) {
        std::vector<uint64_t> distinct;
        std::unordered_set<uint64_t> seen;
        for (int64_t i = 0; i < n && int64_t(distinct.size()) <= st->MaxKeys; ++i) {
            for (int64_t k = 0; k < partials[i].KeyCount && int64_t(distinct.size()) <= st->MaxKeys; ++k) {
                const uint64_t h = partials[i].Keys[k];
                if (seen.insert(h).second) distinct.push_back(h);
            }
        }
        if (int64_t(distinct.size()) <= st->MaxKeys) {
            int64_t size = 8;
            while (size < int64_t(distinct.size()) * 2) size *= 2;
            for (uint64_t h : distinct) st->Table[RfExactSlot(st->Table, uint64_t(size - 1), h)] = RfStored(h);
            st->TableSize = size;
            st->ExactKeys = int64_t(distinct.size());
            st->Kind = 1;
            return 0;
        }
        if (st->BloomWords == 0) return 0;
    }
    for (int64_t p = 0; p < n; ++p) {
        for (int64_t w = 0; w < partials[p].BloomWords; ++w) st->Bloom[w] |= partials[p].Bloom[w];
        RfBloomAdd(st->Bloom, st->BloomWords, partials[p].Keys, nullptr, partials[p].KeyCount);
    }
    st->Kind = 2;
    int64_t bits = 0;
    for (int64_t w = 0; w < st->BloomWords; ++w) bits += __builtin_popcountll(st->Bloom[w]);
    st->BloomSetBits = bits;
    return 0;
}

int64_t oracle_rf_probe(const qdb_rf_data* data, const uint64_t* hashes, const uint8_t* sel, uint8_t* out,
                        int64_t count) {
    // rf_probe (:561-577), scalar paths (:149-170, :292-305).
    int64_t kept = 0;
    for (int64_t r = 0; r < count; ++r) {
        bool keep = false;
        if (RfSelected(sel, r)) {
            const uint64_t h = hashes[r];
            if (data->Kind == 1) {
                const uint64_t mask = uint64_t(data->WordCount - 1);
                keep = data->Words[RfExactSlot(data->Words, mask, h)] == RfStored(h);
            } else {
                keep = RfBloomContains(data->Words, data->WordCount, h);
            }
        }
        out[r] = keep ? 1 : 0;
        kept += keep;
    }
    return kept;
}

void oracle_rf_merge(uint64_t* target, const uint64_t* source, int64_t count) {   // rf_merge (:580-584)
    for (int64_t i = 0; i < count; ++i) target[i] |= source[i];
}

// std::mt19937_64 output (the generator the reference's runtime-filter
// tests draw their hashes from, test/test_runtime_filter.cpp:31-39).
uint64_t oracle_string_hash(const uint8_t* data, int64_t size) { return StringHash(data, size); }

const uint8_t* oracle_string_secret(void) { return kStringSecret; }

void oracle_mt19937_64(uint64_t seed, int64_t n, uint64_t* out) {
    std::mt19937_64 rng(seed);
    for (int64_t i = 0; i < n; ++i) out[i] = rng();
}


// THashShuffleTask::OutputOf (qdb/scheduler/tasks/runtime_adapter.cpp:998-1011)
// over a batch: dest[r] = the output of selected row r, -1 for an unselected
// row.  Returns -1 when a row's partition is routed nowhere, else 0.
int64_t oracle_route(const uint64_t* hashes, const uint8_t* sel, int64_t n, const int64_t* routes,
                     int64_t n_routes, int64_t n_outputs, int64_t* dest) {
    for (int64_t r = 0; r < n; ++r) {
        if (sel && !sel[r]) {
            dest[r] = -1;
            continue;
        }
        if (n_routes == 0) {
            dest[r] = int64_t(hashes[r] % uint64_t(n_outputs));
            continue;
        }
        const int64_t out = routes[hashes[r] % uint64_t(n_routes)];
        if (out < 0 || out >= n_outputs) return -1;
        dest[r] = out;
    }
    return 0;
}

}  // extern "C"
