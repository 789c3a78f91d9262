// Internal definitions shared by the host runtime (C++) and the sm_100a
// kernels (CUDA) of the MiniLake B200 execution core.
#pragma once

#include <stdint.h>

#include "../../include/minilake_gpu.h"

#if defined(__CUDACC__)
#define ML_HD __host__ __device__
#else
#define ML_HD
#endif

namespace mlg {

// ---- limits --------------------------------------------------------------------
constexpr int kMaxCols = 24;       // column slots one pipeline may reference
constexpr int kMaxProbes = 4;      // HashJoinProbe operators fused in front of a sink
constexpr int kMaxLuts = 16;       // dictionary predicates (per-entry boolean tables)
constexpr int kMaxKeys = 4;        // GROUP BY / join key expressions
constexpr int kMaxAggs = 8;        // aggregate expressions
constexpr int kMaxFilters = 4;     // filter predicates (one per Filter operator)
constexpr int kStack = 6;          // depth of the expression evaluation stack
constexpr int kKeyWords = 2;       // normalized key: up to 128 bits
constexpr uint32_t kNone = 0xFFFFFFFFu;
constexpr int kTopNChunk = 4096;   // rows one CTA sorts in shared memory
constexpr int kMaxTopN = 2048;

// ---- device column -----------------------------------------------------------------
enum ColKind : int32_t {
    CK_FIXED = 0,     // fixed-width values
    CK_UTF8 = 1,      // plain strings: offsets + bytes
    CK_DICT = 2,      // u32 codes; `gid` maps code -> pipeline-global string id
    CK_STRID = 3,     // u32 canonical string ids stored alongside a plain UTF8 column
};

struct DCol {
    int32_t dt;             // ML_TYPE_*
    int32_t kind;           // ColKind
    int32_t src;            // 0 = pipeline source row, p+1 = build row of probe p
    uint32_t dict_len;      // CK_DICT: dictionary entries (codes are clamped to this)
    const void* data;       // values / dict codes / utf8 bytes
    const uint32_t* off;    // utf8 offsets (n+1); CK_DICT: dictionary offsets (dict_len+1)
    const uint64_t* valid;  // validity words or nullptr
    const uint32_t* gid;    // CK_DICT: code -> global id ; CK_UTF8 of a build side: canonical id
    const uint8_t* dbytes;  // CK_DICT: dictionary bytes
    int64_t n;
};

// ---- expression stack machine -------------------------------------------------------
// Programs are postfix; every instruction pushes one value (or rewrites the top).
enum Op : uint8_t {
    I_COL = 0,       // push column a (typed load)
    I_LIT,           // push literal
    I_BIN,           // pop r, pop l, push l <sub> r computed in type t
    I_NOT,           // boolean NOT (validity kept)
    I_NEG,           // negate type t
    I_ISNULL,        // push(valid == flag)  (flag = negated)
    I_CAST,          // cast top from type t to type sub
    I_STRPRED,       // push string predicate spec (arena c) on column a; dictionary columns read
                     // the per-entry table luts[b] by code (cmp.rs:47-61, string.rs:11-30)
    I_STRCMP_COL,    // push  str(col a) <sub> str(col b)
    I_INLIST,        // top := top IN literals (arena b, count c), type t, flag = negated
    I_SELECT,        // pop val, pop cond, pop rest: push cond TRUE ? val : rest
};

enum LikeShape : uint8_t { LK_EXACT = 0, LK_PREFIX, LK_SUFFIX, LK_CONTAINS, LK_GENERAL };

// A predicate over one string value: compare with a literal, LIKE, or IN (list).
enum StrWhat : uint8_t { SW_CMP = 0, SW_LIKE = 1, SW_IN = 2 };
struct StrSpec {
    uint8_t what, op, negated, pad;  // op: comparison op (SW_CMP) or LIKE shape
    uint32_t lit_off, lit_len;       // literal / pattern bytes in the arena
    uint32_t count;                  // SW_IN: `count` (offset, length) u32 pairs at lit_off
};

struct Instr {
    uint8_t op, sub, t, flag;
    int32_t a, b, c;
    uint64_t bits;  // literal value bits
    uint32_t lit_valid;
    uint32_t pad;
};
static_assert(sizeof(Instr) == 32, "Instr layout");

// Common program shapes get a direct evaluation path (no interpreter loop).
enum FastPath : int32_t {
    FP_NONE = 0,
    FP_COL = 1,           // [COL a]
    FP_COL_LIT_BIN = 2,   // [COL a, LIT, BIN]              a <op> lit
    FP_COL_LCB_BIN = 3,   // [COL a, LIT, COL b, BIN, BIN]   a <op2> (lit <op1> b)
};

struct Prog {
    int32_t start, len;  // range in the pipeline's instruction array
    int32_t type;        // result type
    int32_t maybe_null;  // host analysis: result can be NULL
    int32_t fast;        // FastPath
};

// ---- normalized keys -----------------------------------------------------------------
// A key tuple is packed into up to kKeyWords u64 words: key k occupies `width`
// bits at (word, shift).  NULL keys are flagged in a separate null mask (bit k),
// which the hash table keeps in the upper bits of the slot's state word.
struct KeyField {
    int8_t word, shift, width, type;
    int8_t strid, pad0, pad1, pad2;  // strid: key is a string id (dict global / build canonical)
};
struct KeyLayout {
    int32_t nkeys, nwords;
    KeyField f[kMaxKeys];
    Prog prog[kMaxKeys];
};

// ---- hash tables ---------------------------------------------------------------------
// Open addressing, power-of-two capacity, linear probing, array-of-structs slots:
//   u64 word 0 = state (low 32 bits) | payload (high 32 bits), words 1.. = key words
// (16-byte slots for one key word, 32-byte slots for two), so one probe reads one
// 32-byte sector.  State: 0 empty, 1 claimed (being written), 2 | nullmask << 8 full.
// Insertion claims a slot with a CAS on the state, writes key and payload, then
// publishes the full state; a thread that meets a claimed slot waits for it with a
// bounded spin.
struct TableView {
    uint64_t* slots;
    uint64_t mask;       // capacity - 1
    int32_t nwords;      // key words (1 or 2)
    int32_t stride;      // u64 words per slot (2 or 4)
};

// ---- device error word bits -------------------------------------------------------------
enum DevErr : uint32_t { DE_TIMEOUT = 1u, DE_OVERFLOW_LOST = 2u, DE_BAD_INDEX = 4u };

// ---- aggregate accumulators ---------------------------------------------------------------
// Every group owns a block of `stride` u64 words: word 0 counts its rows (COUNT(*) and
// the seen-flags), each aggregate has its value word at `off` (AVG: sum at off, count
// at off+1).  A group's accumulators thus share one or two 32-byte sectors.
enum AccKind : int32_t {
    A_COUNT = 0,   // u64 count of valid inputs (COUNT(x)); COUNT(*) reads word 0
    A_SUM_I64,     // i64 wrapping sum
    A_SUM_F64,
    A_AVG,         // f64 sum + u64 count of valid inputs
    A_MIN_I64, A_MAX_I64,
    A_MIN_F64, A_MAX_F64,
    // MIN/MAX of a string: (rank + 1) << 32 | string id, the rank being the string's place in
    // byte order among the context's interned strings (AggArgs::str_rank); ranks are renumbered
    // in the group blocks when new strings are interned, so u64 min/max compare strings.
    A_MIN_STR, A_MAX_STR,
};

struct AggDev {
    int32_t kind;
    int32_t func;         // ML_AGG_*
    int32_t has_arg;
    int32_t off;          // word offset inside the group block
    int32_t count_valid;  // maintain vcnt (valid-input counter) in this launch
    int32_t pad;
    Prog arg;
    uint64_t* vcnt;       // valid-input counts by group (seen-tracking for SUM/MIN/MAX)
};

}  // namespace mlg
