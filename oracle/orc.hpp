// TEST INFRASTRUCTURE — the CPU oracle.
//
// A C++17 restatement of MiniLake's CPU hot path (the reference is Rust and
// cannot be built in this environment: no cargo/rustc, crates not vendored).
// Only the tests, the smoke check and bench.py's CPU-baseline / reference arm
// load this library; the product path never calls it.
//
// Each function cites the reference file:line (paths inside the MiniLake
// project) whose algorithm it restates.
#pragma once

#include <atomic>
#include <cstdint>
#include <cstring>
#include <functional>
#include <memory>
#include <mutex>
#include <optional>
#include <stdexcept>
#include <string>
#include <string_view>
#include <vector>

#include "../include/minilake_gpu.h"

namespace orc {

// ---- errors: crates/minilake-core/src/error.rs:8-48 -----------------------------
struct Error : std::runtime_error {
    int code;
    std::string op;
    uint64_t requested = 0, used = 0, limit = 0;
    Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};
[[noreturn]] inline void fail(int code, const std::string& m) { throw Error(code, m); }

enum DT : int32_t { BOOL = 0, I32 = 1, I64 = 2, F64 = 3, DATE = 4, UTF8 = 5 };
const char* dt_name(int dt);
bool is_numeric(int dt);  // types.rs:31-34
int numeric_supertype(int a, int b);  // types.rs:54-62, -1 = none

// ---- hash.rs:11-54 -------------------------------------------------------------
constexpr uint64_t SEED = 0x243F6A8885A308D3ull;
constexpr uint64_t MUL = 0x9E3779B97F4A7C15ull;
constexpr uint64_t MUL2 = 0xBF58476D1CE4E5B9ull;
constexpr uint64_t NULL_HASH = 0x7C159E3779B97F4Aull;
inline uint64_t fold_mul(uint64_t a, uint64_t b) {
    unsigned __int128 r = (unsigned __int128)a * b;
    return (uint64_t)r ^ (uint64_t)(r >> 64);
}
inline uint64_t hash_u64(uint64_t x) { return fold_mul(x ^ SEED, MUL); }
inline uint64_t combine(uint64_t h, uint64_t v) { return fold_mul(h ^ v, MUL2); }
uint64_t hash_bytes(const uint8_t* b, size_t n);

// ---- bitmap.rs:9-179 ------------------------------------------------------------
struct Bitmap {
    std::vector<uint64_t> words;
    size_t len = 0;
    static Bitmap set_all(size_t n);
    static Bitmap unset_all(size_t n);
    static Bitmap from_bools(const std::vector<uint8_t>& b);
    bool get(size_t i) const { return (words[i >> 6] >> (i & 63)) & 1; }
    void set(size_t i, bool v) {
        uint64_t m = 1ull << (i & 63);
        if (v) words[i >> 6] |= m; else words[i >> 6] &= ~m;
    }
    size_t count_set() const;
};

// ---- column.rs:14-150 -----------------------------------------------------------
struct Strings {  // StringVec: offsets (n+1) + bytes
    std::vector<uint32_t> off{0};
    std::vector<uint8_t> bytes;
    size_t len() const { return off.size() - 1; }
    std::string_view get(size_t i) const {
        return std::string_view((const char*)bytes.data() + off[i], off[i + 1] - off[i]);
    }
    void push(std::string_view s) {
        bytes.insert(bytes.end(), s.begin(), s.end());
        off.push_back((uint32_t)bytes.size());
    }
};

// A column: typed values (owned or borrowed) + optional validity.
struct Column {
    int dt = I64;
    bool dict = false;         // ColumnData::Dict
    size_t n = 0;
    const void* vals = nullptr;      // fixed-width values / dict codes
    const uint32_t* off = nullptr;   // utf8 plain offsets (n+1), absolute into `bytes`
    const uint8_t* bytes = nullptr;  // utf8 plain bytes
    std::shared_ptr<const Strings> dictv;  // dictionary
    const uint64_t* vw = nullptr;    // validity words (nullptr = all valid)
    size_t voff = 0;                 // bit offset of row 0 in vw
    std::shared_ptr<const void> own; // keeps owned buffers alive

    bool has_validity() const { return vw != nullptr; }
    bool valid(size_t i) const {
        if (!vw) return true;
        size_t k = voff + i;
        return (vw[k >> 6] >> (k & 63)) & 1;
    }
    template <class T> const T* as() const { return (const T*)vals; }
    const uint32_t* codes() const { return (const uint32_t*)vals; }
    std::string_view str(size_t i) const {  // Column::str_bytes (column.rs:259-266)
        if (dict) return dictv->get(codes()[i]);
        return std::string_view((const char*)bytes + off[i], off[i + 1] - off[i]);
    }
    size_t null_count() const;
    int data_type() const { return dt; }
};
using ColPtr = std::shared_ptr<const Column>;

// Builders for owned columns.
ColPtr make_bool(std::vector<uint8_t>&& v, std::optional<Bitmap>&& valid);
ColPtr make_i32(std::vector<int32_t>&& v, std::optional<Bitmap>&& valid, int dt = I32);
ColPtr make_i64(std::vector<int64_t>&& v, std::optional<Bitmap>&& valid);
ColPtr make_f64(std::vector<double>&& v, std::optional<Bitmap>&& valid);
ColPtr make_utf8(Strings&& s, std::optional<Bitmap>&& valid);
ColPtr make_dict(std::shared_ptr<const Strings> dict, std::vector<uint32_t>&& codes,
                 std::optional<Bitmap>&& valid);
ColPtr with_validity(const ColPtr& c, std::optional<Bitmap>&& valid);
std::optional<Bitmap> validity_of(const Column& c);  // materialized copy
ColPtr gather(const Column& c, const uint32_t* idx, size_t k);  // column.rs:380-398
ColPtr nulls_column(int dt, size_t n);                           // column.rs:313-336
ColPtr column_from_view(const ml_column& c, int64_t row0, int64_t nrows);

// ---- batch.rs:20-134 ------------------------------------------------------------
struct Batch {
    std::vector<ColPtr> cols;
    size_t n = 0;
    std::shared_ptr<const std::vector<uint32_t>> sel;  // SelectionVector
    size_t active_rows() const { return sel ? sel->size() : n; }
    Batch compact() const;
};
Batch concat(const std::vector<Batch>& bs, size_t ncols);

// ---- scalar.rs:9-150 ------------------------------------------------------------
struct Scalar {
    enum Kind { NUL, BOOLV, I32V, I64V, F64V, DATEV, UTF8V } kind = NUL;
    int64_t i = 0;
    double f = 0;
    std::string s;
    bool is_null() const { return kind == NUL; }
    int data_type() const;  // -1 for NULL
    std::optional<double> as_f64() const;
    std::optional<int64_t> as_i64() const;
    std::optional<bool> as_bool() const;
    Scalar cast_to(int dt) const;              // scalar.rs:82-113
    std::optional<int> compare(const Scalar& o) const;  // scalar.rs:117-133
    std::string to_string() const;
    static Scalar b(bool v) { Scalar x; x.kind = BOOLV; x.i = v; return x; }
    static Scalar null() { return Scalar(); }
};
Scalar scalar_at(const Column& c, size_t i);  // column.rs:269-282

// ---- dates: crates/minilake-core/src/date.rs -------------------------------------
int32_t days_from_civil(int32_t y, uint32_t m, uint32_t d);
std::string format_date(int32_t days);
std::optional<int32_t> parse_date(std::string_view s);

// ---- expr/like.rs:9-115 ----------------------------------------------------------
struct LikePattern {
    enum Shape { EXACT, PREFIX, SUFFIX, CONTAINS, GENERAL } shape = EXACT;
    std::string p;
    static LikePattern compile(std::string_view pattern);
    bool matches(std::string_view s) const;
};
bool like_contains(std::string_view hay, std::string_view needle);
bool like_general(std::string_view s, std::string_view p);

// ---- expr/mod.rs:109-173 ---------------------------------------------------------
struct Expr {
    int kind = ML_EXPR_COLUMN;
    int op = 0, dtype = 0, flag = 0;
    int64_t index = 0;
    Scalar lit;
    LikePattern like;
    std::vector<Expr> kids;
    int data_type(const std::vector<int>& schema) const;  // expr/mod.rs:199-234
};
Expr parse_expr(const ml_expr& e);
Expr parse_nodes(const ml_expr_node* nodes, int32_t nnodes);

struct Datum {
    bool scalar = false;
    Scalar s;
    ColPtr col;
};
Datum evaluate(const Expr& e, const Batch& b);                         // eval.rs:61-151
ColPtr evaluate_to_column(const Expr& e, const Batch& b, int dt);      // eval.rs:154-160
std::vector<uint32_t> select(const Expr& e, const Batch& b, const std::vector<uint32_t>* input);
ColPtr cast_column(const ColPtr& c, int to);                           // cast.rs:6-73
Scalar scalar_binary(int op, const Scalar& l, const Scalar& r);        // scalar_ops.rs:12-105
std::vector<uint32_t> mask_to_selection(const uint8_t* mask, size_t n, const Column* validity,
                                        const std::vector<uint32_t>* input);  // cmp.rs:85-118

// ---- kernels/hash.rs:16-101 ------------------------------------------------------
// rows: nullptr = All(n) else Sel(rows[0..k])
void hash_columns(const std::vector<ColPtr>& cols, size_t n, const uint32_t* rows, size_t k,
                  std::vector<uint64_t>& out);
bool values_equal(const Column& x, size_t a, const Column& y, size_t b);

// ---- swiss.rs:50-302 -------------------------------------------------------------
struct SwissTable {
    std::vector<uint8_t> ctrl;
    std::vector<uint64_t> hashes;
    std::vector<uint32_t> payloads;
    size_t len = 0, group_mask = 0;
    explicit SwissTable(size_t n = 0);
    size_t capacity() const { return ctrl.size(); }
    size_t memory_size() const { return capacity() * 13; }
    uint64_t load_group(size_t g) const;
    template <class Eq> std::optional<uint32_t> find(uint64_t h, Eq eq) const;
    // Probe: found = true -> payload, else vacant slot
    template <class Eq> std::pair<bool, size_t> find_or_vacant(uint64_t h, Eq eq);
    void insert_at(size_t slot, uint64_t h, uint32_t payload);
    size_t first_empty(uint64_t h) const;
    void reserve(size_t extra);
    // KeyStore: equals(payload, k), insert(k) -> payload
    template <class KS>
    size_t find_or_insert_batch(const std::vector<uint64_t>& hashes, KS& keys,
                                std::vector<uint32_t>& out);
};
uint64_t swar_match_tag(uint64_t group, uint8_t tag);
uint64_t swar_match_empty(uint64_t group);

// ---- memory.rs:22-157 ------------------------------------------------------------
struct MemoryPool {
    uint64_t limit;
    std::atomic<uint64_t> used{0}, peak{0};
    explicit MemoryPool(uint64_t lim) : limit(lim ? lim : UINT64_MAX) {}
    bool try_grow(uint64_t bytes, uint64_t* observed);
    void shrink(uint64_t bytes) { used.fetch_sub(bytes); }
};
struct MemoryReservation {
    std::shared_ptr<MemoryPool> pool;
    std::string name;
    uint64_t size = 0, peak = 0;
    MemoryReservation(std::shared_ptr<MemoryPool> p, std::string n) : pool(std::move(p)), name(std::move(n)) {}
    MemoryReservation(MemoryReservation&& o) noexcept;
    MemoryReservation(const MemoryReservation&) = delete;
    ~MemoryReservation() { free(); }
    void try_grow(uint64_t bytes);
    void try_resize(uint64_t sz) { if (sz > size) try_grow(sz - size); else shrink(size - sz); }
    void shrink(uint64_t bytes);
    void free() { shrink(size); }
};

// ---- aggregate: accumulator.rs, group_keys.rs, aggregate/hash.rs ------------------
struct AggSpec {
    int func;
    int arg_type;  // -1 for COUNT(*)
    std::optional<Expr> arg;
};

struct Accumulator {  // accumulator.rs:97-594
    int func, output_type, input_type;  // input_type -1 = None
    int kind;  // state kind
    std::vector<int64_t> i;   // Count / SumI64 sum / Avg count / MinMaxI64 v
    std::vector<double> f;    // SumF64 sum / Avg sum / MinMaxF64 v
    std::vector<uint8_t> seen;
    std::vector<std::optional<std::string>> str;  // MinMaxStr
    Accumulator(int func, int arg_type);
    size_t num_groups() const;
    void resize(size_t n);
    ColPtr prepare_input(const ColPtr& c) const;
    void update(const Column* input, size_t nrows, const uint32_t* rows, size_t k,
                const uint32_t* gids);
    std::vector<ColPtr> state() const;
    std::vector<int> state_types() const;
    void merge(const std::vector<ColPtr>& st, const uint32_t* gids, size_t k);
    ColPtr finish() const;
    size_t memory_size() const;
};
double sum_f64(const double* v, size_t n);                       // accumulator.rs:562-576
double sum_f64_sel(const double* v, const uint32_t* s, size_t n);  // accumulator.rs:580-594

struct GroupKeys {  // group_keys.rs:27-150
    struct KeyCol {
        int dt;
        std::vector<int32_t> i32;
        std::vector<int64_t> i64;
        std::vector<double> f64;
        std::vector<uint8_t> b;
        Strings s;
        std::vector<uint8_t> valid;
    };
    std::vector<KeyCol> cols;
    size_t len = 0, bytes = 0;
    explicit GroupKeys(const std::vector<int>& types);
    uint32_t push(const std::vector<ColPtr>& in, size_t row);
    bool equals(uint32_t g, const std::vector<ColPtr>& in, size_t row) const;
    std::vector<ColPtr> to_columns() const;
};

struct HashAggState {  // aggregate/hash.rs:204-322
    std::vector<int> key_types;
    GroupKeys keys;
    SwissTable table;
    std::vector<Accumulator> accs;
    std::vector<uint64_t> hashes;
    std::vector<uint32_t> gids;
    HashAggState(const std::vector<int>& key_types, const std::vector<AggSpec>& aggs);
    size_t num_groups() const { return keys.len; }
    void assign_groups(const std::vector<ColPtr>& key_cols, size_t n, const uint32_t* rows, size_t k);
    void update(const Batch& b, const std::vector<Expr>& group_exprs, const std::vector<AggSpec>& aggs);
    void merge_partial(const Batch& b);
    void merge_state(const HashAggState& o);
    Batch partial_batch() const;
    Batch final_batch() const;
    size_t memory_size() const;
};

// ---- join.rs:33-337 ---------------------------------------------------------------
struct JoinTable {
    Batch batch;
    std::vector<ColPtr> keys;
    SwissTable table;
    std::vector<uint32_t> next;
};
std::unique_ptr<JoinTable> build_table(const std::vector<Batch>& batches,
                                       const std::vector<Expr>& key_exprs,
                                       const std::vector<int>& key_types, size_t ncols);
// HashJoinProbe::execute without the batch-size split: all pairs of one batch.
void probe_pairs(const JoinTable& jt, const std::vector<Expr>& key_exprs,
                 const std::vector<int>& key_types, const Batch& b, std::vector<uint32_t>& pi,
                 std::vector<uint32_t>& bi);

// ---- sort.rs:23-132 ---------------------------------------------------------------
struct SortKey {
    Expr expr;
    bool asc, nulls_first;
};
std::optional<Batch> sort_batches(const std::vector<Batch>& batches, const std::vector<SortKey>& keys,
                                  std::optional<size_t> limit, size_t ncols);

// ---- pipelines: pipeline.rs, executor.rs, scheduler.rs ----------------------------
struct PipeOp {
    int kind;  // ML_PIPE_*
    std::vector<Expr> exprs;
    std::vector<int> types;  // PROJECT output types / PROBE key types
    const JoinTable* join = nullptr;
    bool build_is_left = false;
};

// An in-memory source: morsel i = row group i (scan.rs:13-56) cut into batches.
struct MorselSource {
    const ml_column* cols;  // nmorsels * ncols views
    int nmorsels, ncols;
    const int64_t* rows;
    size_t batch_size;
};

// A result: dense columns.
struct Result {
    std::vector<ColPtr> cols;
    size_t n = 0;
};

void run_operators(const std::vector<PipeOp>& ops, size_t idx, Batch b,
                   const std::function<void(Batch)>& sink);  // Pipeline::push (pipeline.rs:139-161)

}  // namespace orc

// ---- SwissTable templates (swiss.rs:205-350) ------------------------------------
namespace orc {
template <class Eq> std::optional<uint32_t> SwissTable::find(uint64_t h, Eq eq) const {
    uint8_t tag = (uint8_t)(h >> 57);
    size_t g = (size_t)h & group_mask, stride = 0;
    for (;;) {
        uint64_t group = load_group(g);
        uint64_t m = swar_match_tag(group, tag);
        while (m) {
            size_t i = g * 8 + __builtin_ctzll(m) / 8;
            if (ctrl[i] == tag && hashes[i] == h && eq(payloads[i])) return payloads[i];
            m &= m - 1;
        }
        if (swar_match_empty(group)) return std::nullopt;
        stride++;
        g = (g + stride) & group_mask;
    }
}
template <class Eq> std::pair<bool, size_t> SwissTable::find_or_vacant(uint64_t h, Eq eq) {
    reserve(1);
    uint8_t tag = (uint8_t)(h >> 57);
    size_t g = (size_t)h & group_mask, stride = 0;
    for (;;) {
        uint64_t group = load_group(g);
        uint64_t m = swar_match_tag(group, tag);
        while (m) {
            size_t i = g * 8 + __builtin_ctzll(m) / 8;
            if (ctrl[i] == tag && hashes[i] == h && eq(payloads[i])) return {true, payloads[i]};
            m &= m - 1;
        }
        uint64_t e = swar_match_empty(group);
        if (e) return {false, g * 8 + __builtin_ctzll(e) / 8};
        stride++;
        g = (g + stride) & group_mask;
    }
}
template <class KS>
size_t SwissTable::find_or_insert_batch(const std::vector<uint64_t>& hs, KS& keys,
                                        std::vector<uint32_t>& out) {
    reserve(hs.size());
    out.clear();
    out.reserve(hs.size());
    size_t inserted = 0;
    for (size_t k = 0; k < hs.size(); k++) {
        uint64_t h = hs[k];
        uint8_t tag = (uint8_t)(h >> 57);
        size_t g = (size_t)h & group_mask, stride = 0;
        uint32_t payload;
        for (;;) {
            uint64_t group = load_group(g);
            uint64_t m = swar_match_tag(group, tag);
            bool found = false;
            while (m) {
                size_t i = g * 8 + __builtin_ctzll(m) / 8;
                if (ctrl[i] == tag && hashes[i] == h && keys.equals(payloads[i], k)) {
                    payload = payloads[i];
                    found = true;
                    break;
                }
                m &= m - 1;
            }
            if (found) break;
            uint64_t e = swar_match_empty(group);
            if (e) {
                size_t slot = g * 8 + __builtin_ctzll(e) / 8;
                payload = keys.insert(k);
                insert_at(slot, h, payload);
                inserted++;
                break;
            }
            stride++;
            g = (g + stride) & group_mask;
        }
        out.push_back(payload);
    }
    return inserted;
}
}  // namespace orc
