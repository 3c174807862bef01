// jtable.cuh — device reads of the built join table (two-slot buckets, one
// 32-byte sector each; layout in kernels.h JTableDev).
#pragma once

#include "kernels.h"

namespace qdb {

__device__ __forceinline__ ulonglong2 BucketKeys(const JTableDev& t, uint64_t b) {
    return __ldg(reinterpret_cast<const ulonglong2*>(t.buckets + 4 * b));
}
__device__ __forceinline__ ulonglong2 BucketPays(const JTableDev& t, uint64_t b) {
    return __ldg(reinterpret_cast<const ulonglong2*>(t.buckets + 4 * b + 2));
}

// Calls f(slot, bucket, j) for every slot holding `key`, starting at bucket b
// whose keys `k` are already loaded; returns the number of matches.
template <class F>
__device__ __forceinline__ unsigned VisitMatches(const JTableDev& t, uint64_t key, uint64_t b, ulonglong2 k, F&& f) {
    unsigned n = 0;
    for (uint64_t p = 0; p <= t.bmask; ++p) {
        if (k.x == kEmptyKey) break;
        if (k.x == key) {
            f(2 * b, b, 0);
            ++n;
        }
        if (k.y == kEmptyKey) break;
        if (k.y == key) {
            f(2 * b + 1, b, 1);
            ++n;
        }
        b = (b + 1) & t.bmask;
        k = BucketKeys(t, b);
    }
    return n;
}

}  // namespace qdb
