// rfilter.cuh — device membership tests of a published runtime join filter
// (formats of qdb/kernel/join/runtime_filter.oz:78-113, :257-300), shared by
// the filter's own kernels and the hash kernel that fuses the probe.
#pragma once

#include <cstdint>

namespace qdb {

constexpr uint64_t kBloomSalt = 0x9e3779b97f4a7c15ull;

// splitmix64's finalizer (rf_mix, runtime_filter.oz:78-84).
__host__ __device__ __forceinline__ uint64_t RfMix(uint64_t v) {
    v ^= v >> 30;
    v *= 0xbf58476d1ce4e5b9ull;
    v ^= v >> 27;
    v *= 0x94d049bb133111ebull;
    return v ^ (v >> 31);
}

// A hash picks block mix(h) & block_mask and, in word j of it, bit
// (mix(h ^ salt) >> 8j) & 63 (rf_bloom_base / rf_bloom_bits / rf_bloom_bit).
__device__ __forceinline__ bool BloomContains(const uint64_t* words, uint64_t block_mask, uint64_t h) {
    const uint64_t base = (RfMix(h) & block_mask) * 8;
    const uint64_t bits = RfMix(h ^ kBloomSalt);
    // One 64-byte block: two 32-byte sector loads.
    const ulonglong4 a = *reinterpret_cast<const ulonglong4*>(words + base);
    const ulonglong4 b = *reinterpret_cast<const ulonglong4*>(words + base + 4);
    const uint64_t w[8] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w};
    bool in = true;
#pragma unroll
    for (int j = 0; j < 8; ++j) in &= ((w[j] >> ((bits >> (8 * j)) & 63)) & 1) != 0;
    return in;
}

// rf_exact_slot / rf_exact_probe (runtime_filter.oz:268-300): linear
// probing from h & mask; 0 is empty and hash 0 is stored as 1.
__device__ __forceinline__ bool ExactContains(const uint64_t* table, uint64_t mask, uint64_t h) {
    const uint64_t stored = h == 0 ? 1 : h;
    uint64_t slot = h & mask;
    for (uint64_t p = 0; p <= mask; ++p) {
        const uint64_t f = table[slot];
        if (f == stored) return true;
        if (f == 0) return false;
        slot = (slot + 1) & mask;
    }
    return false;
}

// Kind 1 (exact table of nwords slots) or 2 (Bloom of nwords words).
__device__ __forceinline__ bool FilterContains(int64_t kind, const uint64_t* words, int64_t nwords, uint64_t h) {
    return kind == 1 ? ExactContains(words, uint64_t(nwords - 1), h)
                     : BloomContains(words, uint64_t(nwords / 8 - 1), h);
}

}  // namespace qdb
