// rfilter.cu — the runtime join filter on the device (sm_100a): the four
// entries of the reference's runtime-filter kernel (rf_build, rf_publish,
// rf_probe, rf_merge; qdb/kernel/join/runtime_filter.oz) over device storage,
// and a probe fused with the probe side's key hash.
//
// Formats are the reference's, since producers, the publisher and consumers
// exchange them: a Bloom filter is a power-of-two number of 64-byte blocks;
// a hash picks block (mix(h) & (blocks - 1)) and in each of its eight words
// bit (mix(h ^ 0x9e3779b97f4a7c15) >> 8w) & 63 (runtime_filter.oz:88-113);
// the published exact set is a linear-probing table of raw hashes, slot
// h & (size - 1), zero empty and hash 0 stored as 1 (:257-300).
//
// rf_build's contribution state machine (collect, then one sort + dedup
// compaction at 2 * MaxKeys keys, then dedup, then Bloom) runs on the host,
// every data-parallel step on the device: compaction of selected hashes,
// the sort (the onesweep passes of sort.cu), set membership, first
// occurrences in row order, Bloom adds (atomic ORs), table inserts (CAS).
// The dedup set lives in SetSlots as an open-addressing table of raw hashes
// (all-ones marks an empty slot; the all-ones hash itself is a flag in
// SetCtrl[0]), so it can be built and read by many threads at once.
#include <algorithm>
#include <cstring>
#include <vector>

#include "common.cuh"
#include "kernels.h"
#include "rfilter.cuh"
#include "runtime.h"
#include "sort.h"

namespace qdb {

namespace {

constexpr uint64_t kSetEmpty = ~0ull;

__device__ __forceinline__ bool Selected(const uint8_t* sel, int64_t r) { return sel == nullptr || sel[r] != 0; }

__device__ __forceinline__ void BloomAdd(uint64_t* words, uint64_t block_mask, uint64_t h) {
    const uint64_t base = (RfMix(h) & block_mask) * 8;
    const uint64_t bits = RfMix(h ^ kBloomSalt);
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        const unsigned long long bit = 1ull << ((bits >> (8 * j)) & 63);
        unsigned long long* w = reinterpret_cast<unsigned long long*>(words + base + j);
        if ((*w & bit) == 0) atomicOr(w, bit);
    }
}

__global__ void __launch_bounds__(256) RfProbeKernel(int64_t kind, const uint64_t* words, int64_t nwords,
                                                     const uint64_t* hashes, const uint8_t* sel, uint8_t* out,
                                                     int64_t n, unsigned long long* kept) {
    unsigned long long local = 0;
    for (int64_t r = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; r < n; r += int64_t(gridDim.x) * blockDim.x) {
        const bool keep = Selected(sel, r) && FilterContains(kind, words, nwords, hashes[r]);
        out[r] = keep ? 1 : 0;
        local += keep;
    }
    local = WarpSumU64(local);
    if (LaneId() == 0 && local) atomicAdd(kept, local);
}

__global__ void __launch_bounds__(256) RfBloomAddKernel(uint64_t* words, uint64_t block_mask, const uint64_t* hashes,
                                                        const uint8_t* sel, int64_t n) {
    for (int64_t r = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; r < n; r += int64_t(gridDim.x) * blockDim.x) {
        if (Selected(sel, r)) BloomAdd(words, block_mask, hashes[r]);
    }
}

__global__ void __launch_bounds__(256) RfOrKernel(uint64_t* target, const uint64_t* source, int64_t n) {
    for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
        target[i] |= source[i];
    }
}

__global__ void __launch_bounds__(256) RfPopcountKernel(const uint64_t* words, int64_t n, unsigned long long* bits) {
    unsigned long long local = 0;
    for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
        local += __popcll(words[i]);
    }
    local = WarpSumU64(local);
    if (LaneId() == 0 && local) atomicAdd(bits, local);
}

// rf_exact_build (runtime_filter.oz:281-290) with concurrent inserts: every
// key claims the first slot of its sequence holding zero or itself, so the
// table holds exactly the keys whatever the insertion order.
__global__ void __launch_bounds__(256) RfExactInsertKernel(uint64_t* table, uint64_t mask, const uint64_t* keys,
                                                           int64_t n) {
    for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
        const uint64_t h = keys[i];
        const unsigned long long stored = h == 0 ? 1 : h;
        uint64_t slot = h & mask;
        for (uint64_t p = 0; p <= mask; ++p) {
            const unsigned long long cur = atomicCAS(reinterpret_cast<unsigned long long*>(table + slot), 0ull, stored);
            if (cur == 0 || cur == stored) break;
            slot = (slot + 1) & mask;
        }
    }
}

// Dedup set of raw hashes: open addressing over a power-of-two `slots`
// array (kSetEmpty = empty); the all-ones hash is the flag *ones.
__device__ __forceinline__ bool SetInsert(uint64_t* slots, uint64_t mask, uint8_t* ones, uint64_t h) {
    if (h == kSetEmpty) {
        // A byte flag set once: the first thread to see it clear wins.
        unsigned* word = reinterpret_cast<unsigned*>(reinterpret_cast<uintptr_t>(ones) & ~uintptr_t(3));
        const unsigned bit = 1u << (8 * (reinterpret_cast<uintptr_t>(ones) & 3));
        return (atomicOr(word, bit) & bit) == 0;
    }
    uint64_t slot = RfMix(h) & mask;
    for (uint64_t p = 0; p <= mask; ++p) {
        const unsigned long long cur =
            atomicCAS(reinterpret_cast<unsigned long long*>(slots + slot), kSetEmpty, h);
        if (cur == kSetEmpty) return true;
        if (cur == h) return false;
        slot = (slot + 1) & mask;
    }
    return false;
}

__device__ __forceinline__ bool SetContains(const uint64_t* slots, uint64_t mask, const uint8_t* ones, uint64_t h) {
    if (h == kSetEmpty) return *ones != 0;
    uint64_t slot = RfMix(h) & mask;
    for (uint64_t p = 0; p <= mask; ++p) {
        const uint64_t cur = slots[slot];
        if (cur == h) return true;
        if (cur == kSetEmpty) return false;
        slot = (slot + 1) & mask;
    }
    return false;
}

__global__ void __launch_bounds__(256) RfSetInsertKernel(uint64_t* slots, uint64_t mask, uint8_t* ones,
                                                         const uint64_t* keys, int64_t n,
                                                         unsigned long long* inserted) {
    unsigned long long local = 0;
    for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
        local += SetInsert(slots, mask, ones, keys[i]);
    }
    local = WarpSumU64(local);
    if (inserted && LaneId() == 0 && local) atomicAdd(inserted, local);
}

// Rows [0, n) of a batch whose hash is selected and not yet in the set.
__global__ void __launch_bounds__(256) RfNewFlagsKernel(const uint64_t* slots, uint64_t mask, const uint8_t* ones,
                                                        const uint64_t* hashes, const uint8_t* sel, int64_t n,
                                                        uint8_t* flags) {
    for (int64_t r = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; r < n; r += int64_t(gridDim.x) * blockDim.x) {
        flags[r] = Selected(sel, r) && !SetContains(slots, mask, ones, hashes[r]) ? 1 : 0;
    }
}

// First occurrence per hash among the candidate rows cand[0, m): a table of
// (hash, smallest position) with atomicMin; the all-ones hash keeps its
// smallest position in *ones_pos.
__global__ void __launch_bounds__(256) RfFirstPosKernel(uint64_t* keys, unsigned long long* pos, uint64_t mask,
                                                        unsigned long long* ones_pos, const uint64_t* hashes,
                                                        const int64_t* cand, int64_t m) {
    for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < m; i += int64_t(gridDim.x) * blockDim.x) {
        const uint64_t h = hashes[cand[i]];
        if (h == kSetEmpty) {
            atomicMin(ones_pos, (unsigned long long)i);
            continue;
        }
        uint64_t slot = RfMix(h) & mask;
        for (uint64_t p = 0; p <= mask; ++p) {
            const unsigned long long cur = atomicCAS(reinterpret_cast<unsigned long long*>(keys + slot), kSetEmpty, h);
            if (cur == kSetEmpty || cur == h) {
                atomicMin(pos + slot, (unsigned long long)i);
                break;
            }
            slot = (slot + 1) & mask;
        }
    }
}

__global__ void __launch_bounds__(256) RfFirstFlagsKernel(const uint64_t* keys, const unsigned long long* pos,
                                                          uint64_t mask, const unsigned long long* ones_pos,
                                                          const uint64_t* hashes, const int64_t* cand, int64_t m,
                                                          uint8_t* flags) {
    for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < m; i += int64_t(gridDim.x) * blockDim.x) {
        const uint64_t h = hashes[cand[i]];
        bool first = false;
        if (h == kSetEmpty) {
            first = *ones_pos == (unsigned long long)i;
        } else {
            uint64_t slot = RfMix(h) & mask;
            for (uint64_t p = 0; p <= mask; ++p) {
                if (keys[slot] == h) {
                    first = pos[slot] == (unsigned long long)i;
                    break;
                }
                slot = (slot + 1) & mask;
            }
        }
        flags[i] = first ? 1 : 0;
    }
}

// out[i] = src[idx[i]] (u64), or src[idx2[idx[i]]] when idx2 is set.
__global__ void __launch_bounds__(256) RfGatherKernel(const uint64_t* src, const int64_t* idx, const int64_t* idx2,
                                                      int64_t n, uint64_t* out) {
    for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
        const int64_t j = idx2 ? idx2[idx[i]] : idx[i];
        out[i] = src[j];
    }
}

// The eight 8-bit digit histograms of raw u64 keys.
__global__ void __launch_bounds__(256) RfDigitHistKernel(const uint64_t* keys, int64_t n, unsigned long long* hist) {
    __shared__ unsigned h[8 * 256];
    for (int i = threadIdx.x; i < 8 * 256; i += blockDim.x) h[i] = 0;
    __syncthreads();
    for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
        const uint64_t k = keys[i];
#pragma unroll
        for (int d = 0; d < 8; ++d) atomicAdd(&h[d * 256 + ((k >> (8 * d)) & 255)], 1u);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < 8 * 256; i += blockDim.x) {
        if (h[i]) atomicAdd(&hist[i], (unsigned long long)h[i]);
    }
}

// flags[i] = 1 at the first of each run of equal sorted keys.
__global__ void __launch_bounds__(256) RfRunHeadKernel(const uint64_t* sorted, int64_t n, uint8_t* flags) {
    for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
        flags[i] = (i == 0 || sorted[i] != sorted[i - 1]) ? 1 : 0;
    }
}

__global__ void RfFillKernel(uint64_t* p, int64_t n, uint64_t v) {
    for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) p[i] = v;
}

int Grid(int64_t n) {
    return int(std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, int64_t(DeviceSMs()) * 16)));
}

// Device scratch freed when the call ends (in stream order).
struct CallScratch {
    cudaStream_t s;
    std::vector<void*> held;
    explicit CallScratch(cudaStream_t st) : s(st) {}
    ~CallScratch() {
        for (void* p : held) DevFree(p, s);
    }
    template <class T>
    T* Get(int64_t count) {
        void* p = DevAlloc(size_t(std::max<int64_t>(count, 1)) * sizeof(T), s);
        if (p) held.push_back(p);
        return static_cast<T*>(p);
    }
};

bool ReadU64(const unsigned long long* d, unsigned long long& out, cudaStream_t s, const char* what) {
    cudaMemcpyAsync(&out, d, 8, cudaMemcpyDeviceToHost, s);
    return CudaOk(cudaStreamSynchronize(s), what);
}

// Ascending indices of the nonzero flags; the count, or -1.
int64_t Compact(const uint8_t* flags, int64_t n, int64_t* idx, CallScratch& sc) {
    if (n == 0) return 0;
    auto* cnt = sc.Get<unsigned long long>(1);
    auto* scratch = static_cast<char*>(sc.Get<char>(int64_t(CompactScratch(n))));
    if (!cnt || !scratch) return -1;
    CompactFlags(flags, n, idx, cnt, scratch, sc.s);
    unsigned long long k = 0;
    if (!ReadU64(cnt, k, sc.s, "runtime filter compaction")) return -1;
    return int64_t(k);
}

// Sorts keys[0, n) ascending in place with the onesweep passes (constant
// digits skipped).
bool SortKeys(uint64_t* keys, int64_t n, CallScratch& sc) {
    if (n <= 1) return true;
    cudaStream_t s = sc.s;
    auto* hist = sc.Get<unsigned long long>(8 * 256);
    if (!hist) return false;
    cudaMemsetAsync(hist, 0, 8 * 256 * 8, s);
    RfDigitHistKernel<<<Grid(n), 256, 0, s>>>(keys, n, hist);
    CountLaunch();
    std::vector<unsigned long long> h(8 * 256);
    cudaMemcpyAsync(h.data(), hist, h.size() * 8, cudaMemcpyDeviceToHost, s);
    if (!CudaOk(cudaStreamSynchronize(s), "runtime filter sort histogram")) return false;
    std::vector<int> digits;
    std::vector<unsigned long long> bases;
    for (int d = 0; d < 8; ++d) {
        bool constant = false;
        unsigned long long run = 0;
        for (int x = 0; x < 256; ++x) {
            constant |= int64_t(h[d * 256 + x]) == n;
            bases.push_back(run);
            run += h[d * 256 + x];
        }
        if (constant) {
            bases.resize(bases.size() - 256);
        } else {
            digits.push_back(d);
        }
    }
    if (digits.empty()) return true;
    const int64_t tiles = (n + kSortTile - 1) / kSortTile;
    auto* dbases = sc.Get<unsigned long long>(int64_t(bases.size()));
    auto* status = sc.Get<unsigned long long>(tiles * 256);
    auto* counter = sc.Get<unsigned int>(1);
    auto* derr = sc.Get<int>(1);
    uint64_t* kbuf[2] = {sc.Get<uint64_t>(n), sc.Get<uint64_t>(n)};
    uint32_t* ibuf[2] = {sc.Get<uint32_t>(n), sc.Get<uint32_t>(n)};
    if (!dbases || !status || !counter || !derr || !kbuf[0] || !kbuf[1] || !ibuf[0] || !ibuf[1]) return false;
    cudaMemcpyAsync(dbases, bases.data(), bases.size() * 8, cudaMemcpyHostToDevice, s);
    cudaMemsetAsync(status, 0, size_t(tiles) * 256 * 8, s);
    cudaMemsetAsync(derr, 0, sizeof(int), s);
    const void* kin = keys;
    const uint32_t* idx = nullptr;
    int cur = 0;
    for (size_t p = 0; p < digits.size(); ++p) {
        SortPass(true, kin, idx, false, kbuf[cur], ibuf[cur], n, 8 * digits[p], dbases + p * 256, status,
                 uint32_t(p + 1), counter, derr, s);
        kin = kbuf[cur];
        idx = ibuf[cur];
        cur ^= 1;
    }
    cudaMemcpyAsync(keys, kin, size_t(n) * 8, cudaMemcpyDeviceToDevice, s);
    int herr = 0;
    cudaMemcpyAsync(&herr, derr, sizeof(int), cudaMemcpyDeviceToHost, s);
    if (!CudaOk(cudaStreamSynchronize(s), "runtime filter sort")) return false;
    if (herr) {
        SetErr("runtime filter sort: device error %d", herr);
        return false;
    }
    return true;
}

// rf_keys_sort_unique (runtime_filter.oz:307-333): sorts keys[0, n) and
// drops repeats in place; the distinct count, or -1.
int64_t SortUnique(uint64_t* keys, int64_t n, CallScratch& sc) {
    if (n <= 1) return n;
    if (!SortKeys(keys, n, sc)) return -1;
    auto* flags = sc.Get<uint8_t>(n);
    auto* idx = sc.Get<int64_t>(n);
    auto* tmp = sc.Get<uint64_t>(n);
    if (!flags || !idx || !tmp) return -1;
    RfRunHeadKernel<<<Grid(n), 256, 0, sc.s>>>(keys, n, flags);
    CountLaunch();
    const int64_t k = Compact(flags, n, idx, sc);
    if (k < 0) return -1;
    RfGatherKernel<<<Grid(k), 256, 0, sc.s>>>(keys, idx, nullptr, k, tmp);
    cudaMemcpyAsync(keys, tmp, size_t(k) * 8, cudaMemcpyDeviceToDevice, sc.s);
    CountLaunch();
    return k;
}

uint64_t SetMask(const qdb_rf_build_state* st) { return uint64_t(st->SetCapacity - 1); }

// rf_set_fill (runtime_filter.oz:383-396): the set holds exactly keys[0, n).
void SetFill(qdb_rf_build_state* st, const uint64_t* keys, int64_t n, cudaStream_t s) {
    RfFillKernel<<<Grid(st->SetCapacity), 256, 0, s>>>(st->SetSlots, st->SetCapacity, kSetEmpty);
    cudaMemsetAsync(st->SetCtrl, 0, 1, s);
    if (n > 0) RfSetInsertKernel<<<Grid(n), 256, 0, s>>>(st->SetSlots, SetMask(st), st->SetCtrl, keys, n, nullptr);
    CountLaunch(n > 0 ? 2 : 1);
}

void BloomAddKeys(uint64_t* words, int64_t nwords, const uint64_t* hashes, const uint8_t* sel, int64_t n,
                  cudaStream_t s) {
    if (n <= 0 || nwords <= 0) return;
    RfBloomAddKernel<<<Grid(n), 256, 0, s>>>(words, uint64_t(nwords / 8 - 1), hashes, sel, n);
    CountLaunch();
}

// Collect mode: appends the selected hashes from row 0 until `limit` keys;
// returns the rows consumed, -1 on failure.
int64_t Collect(qdb_rf_build_state* st, const uint64_t* hashes, const uint8_t* sel, int64_t count, int64_t limit,
                CallScratch& sc) {
    const int64_t room = limit - st->KeyCount;
    if (room <= 0) return 0;
    cudaStream_t s = sc.s;
    int64_t nsel = count;
    const int64_t* idx = nullptr;
    if (sel) {
        auto* ix = sc.Get<int64_t>(count);
        if (!ix) return -1;
        nsel = Compact(sel, count, ix, sc);
        if (nsel < 0) return -1;
        idx = ix;
    }
    const int64_t k = std::min(nsel, room);
    if (k > 0) {
        if (idx) {
            RfGatherKernel<<<Grid(k), 256, 0, s>>>(hashes, idx, nullptr, k, st->Keys + st->KeyCount);
            CountLaunch();
        } else {
            cudaMemcpyAsync(st->Keys + st->KeyCount, hashes, size_t(k) * 8, cudaMemcpyDeviceToDevice, s);
        }
    }
    st->KeyCount += k;
    if (nsel < room) return count;
    // The loop stops right after the row that filled the keys.
    int64_t last = k - 1;
    if (idx) {
        cudaMemcpyAsync(&last, idx + (k - 1), 8, cudaMemcpyDeviceToHost, s);
        if (!CudaOk(cudaStreamSynchronize(s), "runtime filter collect")) return -1;
    }
    return last + 1;
}

// Dedup mode from row `row`: appends the hashes not yet in the set, in the
// order of their first selected row, until the keys exceed MaxKeys; returns
// the rows consumed (rf_build's mode-1 loop, runtime_filter.oz:453-470).
int64_t Dedup(qdb_rf_build_state* st, const uint64_t* hashes, const uint8_t* sel, int64_t row, int64_t count,
              CallScratch& sc) {
    const int64_t n = count - row;
    if (n <= 0) return count;
    cudaStream_t s = sc.s;
    const uint64_t* h = hashes + row;
    const uint8_t* sl = sel ? sel + row : nullptr;
    auto* flags = sc.Get<uint8_t>(n);
    auto* cand = sc.Get<int64_t>(n);
    if (!flags || !cand) return -1;
    RfNewFlagsKernel<<<Grid(n), 256, 0, s>>>(st->SetSlots, SetMask(st), st->SetCtrl, h, sl, n, flags);
    CountLaunch();
    const int64_t m = Compact(flags, n, cand, sc);
    if (m < 0) return -1;
    if (m == 0) return count;
    int64_t cap = 16;
    while (cap < 2 * m) cap *= 2;
    auto* tkeys = sc.Get<uint64_t>(cap);
    auto* tpos = sc.Get<unsigned long long>(cap + 1);
    auto* first = sc.Get<uint8_t>(m);
    auto* order = sc.Get<int64_t>(m);
    if (!tkeys || !tpos || !first || !order) return -1;
    RfFillKernel<<<Grid(cap), 256, 0, s>>>(tkeys, cap, kSetEmpty);
    RfFillKernel<<<Grid(cap + 1), 256, 0, s>>>(reinterpret_cast<uint64_t*>(tpos), cap + 1, ~0ull);
    RfFirstPosKernel<<<Grid(m), 256, 0, s>>>(tkeys, tpos, uint64_t(cap - 1), tpos + cap, h, cand, m);
    RfFirstFlagsKernel<<<Grid(m), 256, 0, s>>>(tkeys, tpos, uint64_t(cap - 1), tpos + cap, h, cand, m, first);
    CountLaunch(4);
    const int64_t k = Compact(first, m, order, sc);
    if (k < 0) return -1;
    const int64_t take = std::min(k, st->MaxKeys + 1 - st->KeyCount);
    if (take > 0) {
        uint64_t* dst = st->Keys + st->KeyCount;
        RfGatherKernel<<<Grid(take), 256, 0, s>>>(h, order, cand, take, dst);
        RfSetInsertKernel<<<Grid(take), 256, 0, s>>>(st->SetSlots, SetMask(st), st->SetCtrl, dst, take, nullptr);
        CountLaunch(2);
    }
    st->KeyCount += take;
    if (take == k) return count;
    // The row of the key that went over MaxKeys is the last one consumed.
    int64_t ci = 0, r = 0;
    cudaMemcpyAsync(&ci, order + (take - 1), 8, cudaMemcpyDeviceToHost, s);
    if (!CudaOk(cudaStreamSynchronize(s), "runtime filter dedup")) return -1;
    cudaMemcpyAsync(&r, cand + ci, 8, cudaMemcpyDeviceToHost, s);
    if (!CudaOk(cudaStreamSynchronize(s), "runtime filter dedup")) return -1;
    return row + r + 1;
}

bool DeviceArgs(std::initializer_list<const void*> ptrs, const char* what) {
    for (const void* p : ptrs) {
        if (p && !IsDevicePtr(p)) {
            SetErr("%s: every array must be in device memory", what);
            return false;
        }
    }
    return true;
}

}  // namespace

}  // namespace qdb

using namespace qdb;

extern "C" {

int64_t qdb_gpu_rf_build(qdb_rf_build_state* st, const uint64_t* hashes, const uint8_t* selection, int64_t count) {
    t_error.clear();
    if (!st || count < 0 || (count > 0 && !hashes)) {
        SetErr("rf_build: bad arguments");
        return -1;
    }
    // A batch of no rows may point one past its array (the caller's next row).
    if (count > 0 && !DeviceArgs({hashes, selection}, "rf_build")) return -1;
    if (!DeviceArgs({st->Keys, st->SetSlots, st->Bloom}, "rf_build")) return -1;
    cudaStream_t s = CurStream();
    CallScratch sc(s);
    const int64_t max_keys = st->MaxKeys;
    int64_t row = 0;
    st->Want = 0;
    if (st->Mode == 0) {
        row = Collect(st, hashes, selection, count, max_keys * 2, sc);
        if (row < 0) return -1;
        if (st->KeyCount < max_keys * 2) return row;
        if (st->SetCapacity == 0) {
            st->Want = 1;
            return row;
        }
        const int64_t used = SortUnique(st->Keys, st->KeyCount, sc);
        if (used < 0) return -1;
        st->KeyCount = used;
        if (used > max_keys) {
            st->Mode = 2;
        } else {
            SetFill(st, st->Keys, used, s);
            st->Mode = 1;
        }
    }
    if (st->Mode == 1) {
        if (st->KeyCount <= max_keys) {
            row = Dedup(st, hashes, selection, row, count, sc);
            if (row < 0) return -1;
        }
        if (st->KeyCount <= max_keys) return CudaOk(cudaStreamSynchronize(s), "rf_build") ? row : -1;
        st->Mode = 2;
    }
    if (st->Mode == 2) {
        if (st->BloomWords < 0) {
            st->Want = 2;
            return CudaOk(cudaStreamSynchronize(s), "rf_build") ? row : -1;
        }
        BloomAddKeys(st->Bloom, st->BloomWords, st->Keys, nullptr, st->KeyCount, s);
        st->KeyCount = 0;
        st->Mode = 3;
    }
    // Bloom storage arrives between calls, so no row of this batch has been
    // consumed yet: the whole batch goes in.
    BloomAddKeys(st->Bloom, st->BloomWords, hashes, selection, count, s);
    return CudaOk(cudaStreamSynchronize(s), "rf_build") ? count : -1;
}

int64_t qdb_gpu_rf_publish(qdb_rf_publish_state* st, const qdb_rf_partial* partials, int64_t n) {
    t_error.clear();
    if (!st || n < 0 || (n > 0 && !partials)) {
        SetErr("rf_publish: bad arguments");
        return -1;
    }
    if (!DeviceArgs({st->Table, st->Bloom}, "rf_publish")) return -1;
    for (int64_t i = 0; i < n; ++i) {
        if (partials[i].KeyCount > 0 && !DeviceArgs({partials[i].Keys}, "rf_publish")) return -1;
        if (partials[i].BloomWords > 0 && !DeviceArgs({partials[i].Bloom}, "rf_publish")) return -1;
    }
    cudaStream_t s = CurStream();
    CallScratch sc(s);
    st->Kind = 0;
    int64_t total = 0;
    for (int64_t i = 0; i < n; ++i) total += partials[i].KeyCount;
    if (st->BloomSeeded == 0) {
        // Distinct keys over every partial; more than MaxKeys makes it Bloom.
        int64_t cap = 16;
        while (cap < 2 * total) cap *= 2;
        auto* slots = sc.Get<uint64_t>(cap);
        auto* ones = sc.Get<uint8_t>(4);
        auto* cnt = sc.Get<unsigned long long>(1);
        if (!slots || !ones || !cnt) return -1;
        RfFillKernel<<<Grid(cap), 256, 0, s>>>(slots, cap, kSetEmpty);
        cudaMemsetAsync(ones, 0, 4, s);
        cudaMemsetAsync(cnt, 0, 8, s);
        CountLaunch();
        for (int64_t i = 0; i < n; ++i) {
            if (partials[i].KeyCount <= 0) continue;
            RfSetInsertKernel<<<Grid(partials[i].KeyCount), 256, 0, s>>>(slots, uint64_t(cap - 1), ones,
                                                                         partials[i].Keys, partials[i].KeyCount, cnt);
            CountLaunch();
        }
        unsigned long long distinct = 0;
        if (!ReadU64(cnt, distinct, s, "rf_publish")) return -1;
        if (int64_t(distinct) <= st->MaxKeys) {
            int64_t size = 8;
            while (size < int64_t(distinct) * 2) size *= 2;
            for (int64_t i = 0; i < n; ++i) {
                if (partials[i].KeyCount <= 0) continue;
                RfExactInsertKernel<<<Grid(partials[i].KeyCount), 256, 0, s>>>(st->Table, uint64_t(size - 1),
                                                                               partials[i].Keys,
                                                                               partials[i].KeyCount);
                CountLaunch();
            }
            st->TableSize = size;
            st->ExactKeys = int64_t(distinct);
            st->Kind = 1;
            return CudaOk(cudaStreamSynchronize(s), "rf_publish") ? 0 : -1;
        }
        if (st->BloomWords == 0) return 0;
    }
    for (int64_t i = 0; i < n; ++i) {
        const int64_t w = std::min(partials[i].BloomWords, st->BloomWords);
        if (w > 0) {
            RfOrKernel<<<Grid(w), 256, 0, s>>>(st->Bloom, partials[i].Bloom, w);
            CountLaunch();
        }
        BloomAddKeys(st->Bloom, st->BloomWords, partials[i].Keys, nullptr, partials[i].KeyCount, s);
    }
    st->Kind = 2;
    auto* bits = sc.Get<unsigned long long>(1);
    if (!bits) return -1;
    cudaMemsetAsync(bits, 0, 8, s);
    RfPopcountKernel<<<Grid(st->BloomWords), 256, 0, s>>>(st->Bloom, st->BloomWords, bits);
    CountLaunch();
    unsigned long long b = 0;
    if (!ReadU64(bits, b, s, "rf_publish")) return -1;
    st->BloomSetBits = int64_t(b);
    return 0;
}

int64_t qdb_gpu_rf_probe(const qdb_rf_data* data, const uint64_t* hashes, const uint8_t* selection, uint8_t* output,
                         int64_t count, int64_t vectorized, uint64_t* selected_hashes, uint8_t* selected_output) {
    (void)vectorized;
    (void)selected_hashes;
    (void)selected_output;
    t_error.clear();
    if (!data || count < 0 || (count > 0 && (!hashes || !output)) || (data->Kind != 1 && data->Kind != 2)) {
        SetErr("rf_probe: bad arguments (Kind must be 1 exact or 2 Bloom)");
        return -1;
    }
    if (count == 0) return 0;
    if (!DeviceArgs({hashes, selection, output, data->Words}, "rf_probe")) return -1;
    cudaStream_t s = CurStream();
    CallScratch sc(s);
    auto* kept = sc.Get<unsigned long long>(1);
    if (!kept) return -1;
    cudaMemsetAsync(kept, 0, 8, s);
    ProfileBegin(s, "rf_probe", count);
    RfProbeKernel<<<Grid(count), 256, 0, s>>>(data->Kind, data->Words, data->WordCount, hashes, selection, output,
                                              count, kept);
    ProfileEnd(s);
    CountLaunch();
    unsigned long long k = 0;
    if (!ReadU64(kept, k, s, "rf_probe")) return -1;
    return int64_t(k);
}

int64_t qdb_gpu_rf_merge(uint64_t* target, const uint64_t* source, int64_t count) {
    t_error.clear();
    if (count < 0 || (count > 0 && (!target || !source))) {
        SetErr("rf_merge: bad arguments");
        return -1;
    }
    if (count == 0) return 0;
    if (!DeviceArgs({target, source}, "rf_merge")) return -1;
    cudaStream_t s = CurStream();
    RfOrKernel<<<Grid(count), 256, 0, s>>>(target, source, count);
    CountLaunch();
    return CudaOk(cudaStreamSynchronize(s), "rf_merge") ? 0 : -1;
}

}  // extern "C"
