// plan.h — device-side operator plans, filled on the host by lower.cpp and
// passed to kernels by value (__grid_constant__).  Shared by host and device.
#pragma once

#include <cstdint>

#if defined(__CUDACC__)
#define QDB_HD __host__ __device__
#define QDB_NOINLINE __noinline__
#else
#define QDB_HD
#define QDB_NOINLINE
#endif

namespace qdb {

using i128 = __int128;
using u128 = unsigned __int128;

constexpr int kMaxCols = 16;      // input columns one plan reads
constexpr int kMaxAtoms = 16;     // predicate atoms (fast path)
constexpr int kMaxClauses = 16;   // predicate = AND of clauses, clause = OR of atoms
constexpr int kMaxTerms = 4;      // sum-of-products value: terms
constexpr int kMaxFactors = 3;    //   factors per term
constexpr int kMaxValues = 12;    // fast-path values
constexpr int kMaxStates = 24;    // aggregate state words
constexpr int kMaxAggs = 16;
constexpr int kMaxKeyParts = 6;
constexpr int kMaxKeyWords = 8;
constexpr int kMaxGNodes = 40;    // generic expression program
constexpr int kMaxList = 64;      // IN-list constants per plan

// How a column's bytes are interpreted when loaded.
enum LoadKind : uint8_t {
    LK_SIGNED = 0,    // sign-extended integer of `width` bytes (ints, dates, decimals)
    LK_UNSIGNED = 1,  // zero-extended integer (unsigned, char codes)
    LK_F32 = 2,
    LK_F64 = 3,
    LK_BOOLBIT = 4,   // one bit per row at bit_off
};

struct ColDesc {
    const char* data;        // device pointer (row 0 of the launch's range)
    const uint8_t* mask;     // device validity bitmap or nullptr
    int64_t mask_off;        // bit offset of row 0 in `mask`
    int64_t bit_off;         // LK_BOOLBIT: bit offset of row 0 in `data`
    uint8_t width;           // bytes per value: 1, 2, 4, 8, 16
    uint8_t kind;            // LoadKind
    uint8_t nullable;        // mask may be non-null
    uint8_t stage;           // staged through shared memory by bulk copies
    int32_t smem_off;        // byte offset of its tile inside a stage
    int32_t scale;           // decimal scale (F64() divides by 10^scale)
    int32_t build;           // fused join: value comes from the matched build row
    const char* offsets;     // QDB_TYPE_STRING: device offsets (row 0 of the range), `data` the bytes
    int32_t offset_width;    // 4 or 8 (0: not a string column)
};

// Value kinds of the fast path and of state words.
enum ValueKind : uint8_t {
    VK_I64 = 0,   // 64-bit two's complement, wrapping
    VK_I128 = 1,  // 128-bit two's complement, wrapping (DECIMAL128)
    VK_F64 = 2,
};

// Predicate atom: compares a column (times 10^exp, integer domain) with
// constants or a second column.  A NULL operand makes the atom false; the
// fast path only takes predicates whose NULL handling that reproduces.
enum AtomOp : uint8_t {
    AT_EQ = 0, AT_NE, AT_LT, AT_LE, AT_GT, AT_GE,
    AT_BETWEEN,     // c0 <= x <= c1
    AT_IN,          // x in list[list_off, list_off + list_len)
    AT_IS_NULL, AT_IS_NOT_NULL,
    AT_COL_CMP,     // x `cmp` y (second column), cmp in `cmp`
};

struct Atom {
    uint8_t op;
    uint8_t cmp;        // AT_COL_CMP: AT_EQ..AT_GE
    uint8_t clause;
    uint8_t col;
    uint8_t col2;
    uint8_t as_f64;     // compare in double
    uint8_t list_len;
    uint8_t list_off;
    int32_t mul;        // x multiplied by 10^mul before comparing (integer domain)
    int32_t mul2;       // y multiplied by 10^mul2
    i128 c0, c1;        // integer constants (aligned), or f64 bits in the low word
};

// Factor of a product: c + d * x, x = column `col` as a number of kind
// `kind` (0xFF: the factor is the constant c).  Computed in its own kind
// (wrapping), then widened to the value's kind.
struct Factor {
    uint8_t col;
    uint8_t kind;
    uint8_t has_c;      // the tree adds a constant (f64: c + d*x, not d*x)
    uint8_t pad[5];
    int64_t c;
    int64_t d;
    double fc;
    double fd;
};

struct Term {
    uint8_t nf;
    int8_t sign;        // +1 or -1
    uint8_t pad[6];
    Factor f[kMaxFactors];
};

// Sum of products: sum_t sign_t * prod_f factor_tf, evaluated left to right
// in `kind`.  NULL when any column in `null_cols` is NULL at the row.
struct SopValue {
    uint8_t kind;
    uint8_t nterms;
    uint16_t null_cols;
    uint8_t pad[4];
    Term t[kMaxTerms];
};

// Generic expression program (any expression tree the fast path does not
// take): nodes in operand-before-user order, evaluated per row.
enum GOp : uint8_t {
    G_COL = 0, G_CONST, G_NULL,
    G_ADD, G_SUB, G_MUL, G_DIV, G_NEG, G_CAST,
    G_EQ, G_NE, G_LT, G_LE, G_GT, G_GE,
    G_AND, G_OR, G_NOT, G_BETWEEN, G_IN, G_CASE, G_IS_NULL, G_IS_NOT_NULL, G_MOD,
};

// Numeric domain of a generic value.
enum GDomain : uint8_t {
    GD_INT = 0,   // integer or decimal (unscaled) held as i128
    GD_F64 = 1,
    GD_BOOL = 2,
};

struct GNode {
    uint8_t op;
    uint8_t dom;        // GDomain of the result
    uint8_t wrap_bits;  // integer results wrap to this many bits (8..128)
    uint8_t is_unsigned;
    uint8_t a, b, c;    // operand nodes
    uint8_t col;
    int16_t scale;      // decimal scale of the result (0 for plain ints)
    uint8_t list_off;
    uint8_t list_len;
    int32_t pad;
    int64_t imm_lo;
    int64_t imm_hi;
};

struct GProg {
    int32_t n;
    int32_t pad;
    GNode nodes[kMaxGNodes];
};

// Aggregate state word kinds.
enum StateKind : uint8_t {
    ST_COUNT = 0,      // += 1 per row (COUNT(*)) or per non-NULL value
    ST_SUM_I64,        // wrapping i64 sum
    ST_SUM_I128,       // two words: low, high
    ST_SUM_F64,
    ST_MIN_I64,
    ST_MAX_I64,
    ST_MIN_F64,        // order-preserving u64 image of the double
    ST_MAX_F64,
};

// Where a state's input value comes from.
enum ValueSrc : uint8_t {
    VS_NONE = 0,       // COUNT(*)
    VS_SOP = 1,        // fast-path value `idx`
    VS_GENERIC = 2,    // generic node `idx`
};

struct StateDesc {
    uint8_t kind;
    uint8_t src;
    uint8_t idx;
    uint8_t word;       // first state word
};

// One aggregate's output: which state words make it.
struct AggOut {
    uint8_t func;       // qdb_agg_func
    uint8_t state;      // main state index
    uint8_t valid_state;// state counting non-NULL inputs (0xFF: none)
    uint8_t out_type;   // qdb_type of the result
    int16_t out_scale;
    int16_t pad;
};

// Group key packing: each part contributes whole words; NULL flags go to
// the last word when any part is nullable.
enum KeySrc : uint8_t {
    KS_COLUMN = 0,     // raw column bits
    KS_SOP = 1,        // fast-path value
    KS_GENERIC = 2,    // generic node
};

struct KeyPart {
    uint8_t src;
    uint8_t idx;        // column, value or node
    uint8_t bits;       // value bits: 8, 16, 32, 64 or 128
    uint8_t word;       // word holding the value's low bits
    uint8_t shift;      // bit offset inside that word (bits < 64)
    uint8_t null_word;
    uint8_t null_shift; // 0xFF: not nullable
    uint8_t is_float;   // canonical double bits
    uint8_t is_signed;  // sign-extend when unpacking
    uint8_t out_type;   // qdb_type of the output column
    int16_t out_scale;
};

struct AggPlan {
    // Inputs.
    int32_t ncols;
    int32_t has_selection;
    ColDesc cols[kMaxCols];
    const uint8_t* selection;     // device pointer or nullptr (row 0 of range)

    // Filter.
    int32_t filter_kind;          // 0 none, 1 atoms, 2 generic node
    int32_t filter_node;
    int32_t natoms;
    uint32_t clause_mask;         // one bit per clause that must hold
    Atom atoms[kMaxAtoms];
    int64_t list[kMaxList];       // IN-list constants (aligned to the column)

    // Fast-path values and generic program.
    int32_t nvalues;
    int32_t generic_root;         // highest generic node needed, -1 none
    SopValue values[kMaxValues];
    GProg prog;

    // Keys.
    int32_t nkeyparts;
    int32_t key_words;            // packed key words (1 = single-word path)
    int32_t key_null_word;        // word holding NULL flags, -1 none
    int32_t key_full64;           // a one-word key may take any 64-bit value
    KeyPart keys[kMaxKeyParts];

    // States.
    int32_t nstates;
    int32_t state_words;
    StateDesc states[kMaxStates];
    int32_t naggs;
    AggOut aggs[kMaxAggs];

    // Join (fused probe): columns >= probe_cols come from the build side.
    int32_t probe_cols;
};

// Typed row shape (filled by the host when a plan qualifies): every column
// the row reads is an integer of at most 8 bytes without NULLs; predicates
// compare one column with 64-bit constants; states fold products of up to
// three 64-bit affine factors.  Rows then load each column once as int64.
constexpr int kFastCols = 8;
constexpr int kFastAtoms = 4;
constexpr int kFastStates = 8;

struct FastAtom {
    uint8_t op;         // AT_EQ..AT_GE, AT_BETWEEN, AT_IN
    uint8_t col;        // index into the fast column list
    uint8_t list_off;
    uint8_t list_len;
    uint8_t clause;
    uint8_t pad[3];
    int64_t c0, c1;
};

struct FastFactor {
    uint8_t col;
    uint8_t pad[7];
    int64_t c;
    int64_t d;
};

struct FastState {
    uint8_t kind;       // ST_COUNT (no factors), ST_SUM_I64, ST_SUM_I128, ST_MIN_I64, ST_MAX_I64
    uint8_t nf;         // 0..3
    uint8_t wide;       // product kept in 128 bits (decimal)
    uint8_t word;
    uint8_t pad[4];
    FastFactor f[3];
};

struct FastPlan {
    int32_t ncols;
    int32_t natoms;
    uint32_t clause_mask;
    int32_t nkeys;
    int32_t nstates;
    int32_t pad;
    uint8_t col_slot[kFastCols];     // plan column slot of each fast column
    uint8_t key_col[2];
    uint8_t key_bits[2];
    uint8_t key_shift[2];
    uint8_t pad2[2];
    FastAtom atoms[kFastAtoms];
    FastState states[kFastStates];
};

// Order-preserving map of doubles onto u64 (min/max state images).
QDB_HD inline uint64_t F64Ordered(double f) {
    uint64_t b;
    __builtin_memcpy(&b, &f, 8);
    return (b >> 63) ? ~b : (b | (1ull << 63));
}
QDB_HD inline double F64FromOrdered(uint64_t u) {
    const uint64_t b = (u >> 63) ? (u & ~(1ull << 63)) : ~u;
    double f;
    __builtin_memcpy(&f, &b, 8);
    return f;
}

// 64-bit finalizer (MurmurHash3 fmix64) for internal table placement; no
// result depends on it.
QDB_HD inline uint64_t Fmix64(uint64_t k) {
    k ^= k >> 33;
    k *= 0xff51afd7ed558ccdull;
    k ^= k >> 33;
    k *= 0xc4ceb9fe1a85ec53ull;
    k ^= k >> 33;
    return k;
}

}  // namespace qdb
