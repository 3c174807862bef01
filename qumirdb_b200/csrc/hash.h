// hash.h — the engine's shuffle hash of key columns, so that device-computed
// hashes route rows exactly as the host's hash % P does
// (qdb/scheduler/tasks/runtime_adapter.cpp:1001-1003).
//
//   integer leaf: xorshift-multiply mix of the value's unsigned bits
//                 (qdb/kernel/aggregation/key_ops_i64.oz:4-11, gen.cpp:268-277)
//   one-byte string leaf: short-string hash (qdb/modules/qumirdb_runtime.cpp:270)
//   double leaf: mix of canonical bits (-0 -> +0, NaN -> one NaN)
//   struct key: ordered boost-style combine of the field hashes (gen.cpp:345-375)
#pragma once

#include "eval.h"
#include "plan.h"

namespace qdb {

QDB_HD inline uint64_t RhMix(uint64_t h) {
    h ^= h >> 12;
    h ^= h << 25;
    h ^= h >> 27;
    return h * 2685821657736338717ull;
}

QDB_HD inline uint64_t ByteSwap64(uint64_t x) {
    x = ((x & 0x00000000ffffffffull) << 32) | (x >> 32);
    x = ((x & 0x0000ffff0000ffffull) << 16) | ((x >> 16) & 0x0000ffff0000ffffull);
    x = ((x & 0x00ff00ff00ff00ffull) << 8) | ((x >> 8) & 0x00ff00ff00ff00ffull);
    return x;
}

// Hash of a one-byte string (n = 1 branch of the short-string hash).
QDB_HD inline uint64_t Char1Hash(uint8_t b) {
    const uint32_t x = (1u << 24) ^ (uint32_t(b) << 16) ^ (uint32_t(b) << 8) ^ uint32_t(b);
    return ByteSwap64(11400714785074694791ull * uint64_t(x));
}

QDB_HD inline uint64_t Combine(uint64_t h, uint64_t field) {
    return h ^ (field + 0x9e3779b97f4a7c15ull + (h << 6) + (h >> 2));
}

// Leaf hash by qdb_type code (values as loaded by an accessor).
QDB_HD inline uint64_t LeafHashOf(int type, i128 iv, double fv) {
    switch (type) {
        case 1: /* BOOL */ return uint64_t(iv != 0) * 2685821657736338717ull;
        case 15: /* CHAR1 */ return Char1Hash(uint8_t(iv));
        case 10: /* F32 */ {
            const float f = float(fv);
            uint32_t b;
            if (f == 0.0f) b = 0;
            else if (f != f) b = 0x7fc00000u;
            else __builtin_memcpy(&b, &f, 4);
            return RhMix(b);
        }
        case 11: /* F64 */ return RhMix(CanonF64(fv));
        case 14: /* DECIMAL128 */ {
            const uint64_t lo = RhMix(uint64_t(u128(iv)));
            const uint64_t hi = RhMix(uint64_t(u128(iv) >> 64));
            return lo ^ (hi + 0x9e3779b97f4a7c15ull + (lo << 6) + (lo >> 2));
        }
        case 2: case 6: return RhMix(uint64_t(u128(iv)) & 0xffull);
        case 3: case 7: return RhMix(uint64_t(u128(iv)) & 0xffffull);
        case 4: case 8: case 12: return RhMix(uint64_t(u128(iv)) & 0xffffffffull);
        default: return RhMix(uint64_t(u128(iv)));
    }
}

}  // namespace qdb
