// sort.h — device sort of packed row ids (ORDER BY) and top-K selection:
// launchers implemented in sort.cu, driven by sort_rt.cpp.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace qdb {

// Per-batch column pointers of a row-set store (device arrays, batch-major:
// entry b * ncols + c is column slot c of batch b).  A packed row id is
// (batch << 32) | row (qdb/exec/join_exec.h:25-36).
struct StoreTable {
    const char* const* data = nullptr;      // string columns: the bytes
    const char* const* offsets = nullptr;   // string columns: Arrow offsets (4 or 8 bytes each)
    const uint8_t* const* mask = nullptr;   // validity bitmaps (nullptr entries: all valid)
    const int64_t* data_bit = nullptr;      // DataBitOffset (bit-packed BOOL)
    const int64_t* mask_bit = nullptr;      // MaskBitOffset
    int32_t ncols = 0;
    int32_t nbatches = 0;
};

// One LSD stage (least significant first): the order-preserving radix key
// of a column (DESC inverted, NULL rank packed above keys of <= 32 bits), the
// NULL rank of a 64-bit key (a separate, more significant stage), or the
// packed row id itself (top-K tie break).
// A string key is ordered by the bytes, shorter first on a common prefix
// (sr_sort_compare): stages of its 8-byte big-endian chunks, zero-padded
// (chunk 0 most significant), and below them its length, which breaks the
// ties that the padding leaves; its NULL rank is a stage above them all.
enum SortStageSrc : int32_t { SS_KEY = 0, SS_NULL_RANK = 1, SS_ROW_ID = 2, SS_STR_CHUNK = 3, SS_STR_LEN = 4 };

struct SortStage {
    int32_t src = SS_KEY;
    int32_t tcol = 0;          // StoreTable column slot
    int32_t type = 0;          // qdb_type
    int32_t desc = 0;
    int32_t nulls_first = 0;
    int32_t nullable = 0;
    int32_t wide = 0;          // u64 stage keys (else u32)
    int32_t chunk = 0;         // SS_STR_CHUNK: bytes [8 * chunk, 8 * chunk + 8)
    int32_t owidth = 0;        // string stages: offset bytes (4 or 8)
    int32_t pad = 0;
};

constexpr int kMaxSortStages = 16;                 // stages one extraction launch writes
constexpr int kMaxSortStagesTotal = 48;            // stages of one sort (string keys add a stage per 8 bytes)
constexpr int kSortDigits = 8;                     // 8-bit digits of a u64 key
constexpr int kSortTile = 4096;                    // keys per onesweep tile

// Radix key bits of a column type: 8 / 16 / 32 / 64; 0: not a served key type.
__host__ __device__ inline int SortKeyBits(int type) {
    switch (type) {
        case 1: case 2: case 6: case 15: return 8;     // BOOL, I8, U8, CHAR1
        case 3: case 7: return 16;                     // I16, U16
        case 4: case 8: case 10: case 12: return 32;   // I32, U32, F32, DATE32
        case 5: case 9: case 11: case 13: return 64;   // I64, U64, F64, DECIMAL64
        default: return 0;
    }
}

// Longest string (bytes) of column slot `tcol` (offsets of `owidth` bytes)
// among the rows ids[0, n), into *out (device, pre-zeroed).
void SortStringMaxLen(const int64_t* ids, int64_t n, const StoreTable& st, int tcol, int owidth,
                      unsigned long long* out, int* err, cudaStream_t s);

// Writes every stage's keys (input order, u32 or u64 by stage.wide) and
// adds their digit histograms (stage-major, kSortDigits x 256 counters) to
// `hist` (pre-zeroed).  `err` gets a nonzero code on a row id outside the store.
void SortExtract(const int64_t* ids, int64_t n, const StoreTable& st, const SortStage* stages, int nstages,
                 void* const* keys, unsigned long long* hist, int* err, cudaStream_t s);

// One stable counting pass on digit `shift` (onesweep with decoupled
// look-back): keys_in/idx_in -> keys_out/idx_out.  idx_in == nullptr means the
// identity; with `gather`, key i is keys_in[idx_in[i]] (a stage's first pass).
// `status` holds ceil(n / kSortTile) * 256 words zeroed before the sort;
// `epoch` is distinct (1, 2, ...) for every pass over the same status array.
void SortPass(bool wide, const void* keys_in, const uint32_t* idx_in, bool gather, void* keys_out, uint32_t* idx_out,
              int64_t n, int shift, const unsigned long long* bucket_base, unsigned long long* status, uint32_t epoch,
              unsigned int* tile_counter, int* err, cudaStream_t s);

// out[i] = ids[idx[i]].  With `tiles` (SortMaxBatch's dense-run marks of
// ids), ids in dense tiles are computed from the marks; ids may then be null
// when every tile is dense.
void SortGatherIds(const int64_t* ids, const uint32_t* idx, int64_t n, const int64_t* tiles, int64_t* out,
                   cudaStream_t s);

// Row ids per tile of `SortMaxBatch`'s dense-run marks.
constexpr int kSortIdTile = 256;

// Largest batch index among n row ids (written to out[0], device).  With
// `tiles` (ceil(n / kSortIdTile) words), also marks each full tile of
// kSortIdTile ids that are consecutive rows of one batch: tiles[t] = the
// tile's first id, -1 for every other tile, and counts the other tiles in
// out[1].
void SortMaxBatch(const int64_t* ids, int64_t n, unsigned long long* out, int64_t* tiles, cudaStream_t s);

// Materializes column slot `tcol` of the rows `ids[0, n)` into `out` (width
// bytes per row; BOOL as one byte 0/1) and sets validity bits in `valid`
// (pre-zeroed words).
void SortMaterialize(const StoreTable& st, int tcol, int type, const int64_t* ids, int64_t n, char* out,
                     uint32_t* valid, int* err, cudaStream_t s);

// Bytes one cell of a sort key type occupies in its batch column (0: one bit,
// BOOL; -1: not a sort key type).
__host__ __device__ inline int SortKeyWidth(int type) {
    switch (type) {
        case 1: return 0;                              // BOOL
        case 2: case 6: case 15: return 1;             // I8, U8, CHAR1
        case 3: case 7: return 2;                      // I16, U16
        case 4: case 8: case 10: case 12: return 4;    // I32, U32, F32, DATE32
        case 5: case 9: case 11: case 13: return 8;    // I64, U64, F64, DECIMAL64
        default: return -1;
    }
}

// Primary keys of `n_samples` rows spread evenly over `ids` (the row id at
// position j * n / n_samples) written to `keys`, and the r-th smallest of
// them (1-based) to *out (device).
void TopKThreshold(const int64_t* ids, int64_t n, const StoreTable& st, const SortStage& stage, uint64_t* keys,
                   int64_t n_samples, int64_t r, uint64_t* out, int* err, cudaStream_t s);

// Top-K radix select on the primary key of `stage`: counts (4096 bins) of
// digit (p >> shift) & (2^dbits - 1) among rows whose top prefix_bits of p
// equal `prefix` (all rows when prefix_bits == 0).
void TopKHistogram(const int64_t* ids, int64_t n, const StoreTable& st, const SortStage& stage, int shift,
                   int dbits, uint64_t prefix, int prefix_bits, unsigned long long* counts, int* err, cudaStream_t s);
// Appends every row id whose primary key p satisfies p >> (64 - prefix_bits)
// <= prefix (p <= *limit_dev when limit_dev is set) to `out` (at most out_cap
// rows written; the full count in *count).  `tiles`: SortMaxBatch's
// dense-run marks of the same ids.
void TopKCollect(const int64_t* ids, int64_t n, const StoreTable& st, const SortStage& stage, uint64_t prefix,
                 int prefix_bits, const uint64_t* limit_dev, int64_t* out, int64_t out_cap,
                 unsigned long long* count, const int64_t* tiles, int* err, cudaStream_t s);

}  // namespace qdb
