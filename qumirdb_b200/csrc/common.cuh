// common.cuh — device helpers shared by the kernels: bulk-copy staging through
// mbarriers (with bounded waits), warp reductions, device error codes.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>

#include "plan.h"

namespace qdb {

constexpr unsigned kFull = 0xffffffffu;

// Device error codes (a kernel records the first one it meets and returns).
enum DeviceError : int {
    DE_OK = 0,
    DE_WAIT_TIMEOUT = 1,      // an mbarrier or flag wait ran out of iterations
    DE_DIV_ZERO = 2,          // row error: division by zero
    DE_SPILL_FULL = 3,        // spill buffer capacity exceeded
    DE_DEFER_FULL = 4,        // deferred-row buffer capacity exceeded
    DE_LOOKBACK_TIMEOUT = 5,  // a scan's decoupled look-back ran out of iterations
    DE_PROBE_LIMIT = 6,       // a table probe exceeded its bound
    DE_BAD_ROW_ID = 7,        // a packed row id names a batch outside the store
};

// Upper bound of any spin in device code, in SM clock cycles (~1 s).
constexpr long long kSpinCycles = 2000000000ll;

__device__ __forceinline__ void SetError(int* err, int code) {
    if (err) atomicCAS(err, 0, code);
}

__device__ __forceinline__ uint32_t SmemAddr(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void MbarInit(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(SmemAddr(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void FenceBarrierInit() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void FenceProxyAsync() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void MbarArriveExpectTx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(SmemAddr(bar)), "r"(bytes)
                 : "memory");
}

// 1-D bulk copy global -> shared, completing `bytes` of transaction count on
// `bar`.  Both addresses 16-byte aligned, `bytes` a multiple of 16.
__device__ __forceinline__ void BulkG2S(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            SmemAddr(dst)),
        "l"(src), "r"(bytes), "r"(SmemAddr(bar))
        : "memory");
}

// L2 policy that evicts first: streamed input then does not displace the
// tables a kernel keeps resident in L2.
__device__ __forceinline__ uint64_t EvictFirstPolicy() {
    uint64_t p;
    asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
    return p;
}

// BulkG2S with an L2 cache policy (EvictFirstPolicy).
__device__ __forceinline__ void BulkG2SHint(void* dst, const void* src, uint32_t bytes, uint64_t* bar,
                                            uint64_t policy) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint [%0], [%1], %2, [%3], %4;" ::
            "r"(SmemAddr(dst)),
        "l"(src), "r"(bytes), "r"(SmemAddr(bar)), "l"(policy)
        : "memory");
}

__device__ __forceinline__ bool MbarTryWait(uint64_t* bar, uint32_t phase) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(SmemAddr(bar)), "r"(phase)
        : "memory");
    return ok != 0;
}

// Waits for phase `phase` of `bar` for at most kSpinCycles; false on timeout.
__device__ __forceinline__ bool MbarWaitBounded(uint64_t* bar, uint32_t phase) {
    if (MbarTryWait(bar, phase)) return true;
    const long long start = clock64();
    while (!MbarTryWait(bar, phase)) {
        if (clock64() - start > kSpinCycles) return false;
    }
    return true;
}

// ---- warp reductions (all 32 lanes participate) ---------------------------
__device__ __forceinline__ uint64_t WarpSumU64(uint64_t v) {
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) v += __shfl_xor_sync(kFull, v, d);
    return v;
}

__device__ __forceinline__ void WarpSumU128(uint64_t& lo, uint64_t& hi) {
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) {
        const uint64_t olo = __shfl_xor_sync(kFull, lo, d);
        const uint64_t ohi = __shfl_xor_sync(kFull, hi, d);
        const uint64_t nlo = lo + olo;
        hi = hi + ohi + (nlo < lo ? 1ull : 0ull);
        lo = nlo;
    }
}

__device__ __forceinline__ double WarpSumF64(double v) {
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) v += __shfl_xor_sync(kFull, v, d);
    return v;
}

__device__ __forceinline__ long long WarpMinI64(long long v) {
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) {
        const long long o = __shfl_xor_sync(kFull, v, d);
        v = o < v ? o : v;
    }
    return v;
}

__device__ __forceinline__ long long WarpMaxI64(long long v) {
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) {
        const long long o = __shfl_xor_sync(kFull, v, d);
        v = o > v ? o : v;
    }
    return v;
}

__device__ __forceinline__ unsigned long long WarpMinU64(unsigned long long v) {
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) {
        const unsigned long long o = __shfl_xor_sync(kFull, v, d);
        v = o < v ? o : v;
    }
    return v;
}

__device__ __forceinline__ unsigned long long WarpMaxU64(unsigned long long v) {
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) {
        const unsigned long long o = __shfl_xor_sync(kFull, v, d);
        v = o > v ? o : v;
    }
    return v;
}

__device__ __forceinline__ int LaneId() { return threadIdx.x & 31; }

}  // namespace qdb
