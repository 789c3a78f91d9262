// Host runtime of the MiniLake B200 execution core: context, HBM budget pool,
// caching device allocator, device batches and the expression compiler.
#pragma once

#include <cuda_runtime.h>

#include <atomic>
#include <map>
#include <memory>
#include <mutex>
#include <optional>
#include <shared_mutex>
#include <stdexcept>
#include <string>
#include <unordered_map>
#include <vector>

#include "ml_internal.hpp"
#include "ml_kernels.cuh"

namespace mlg {

// ---- errors (crates/minilake-core/src/error.rs) -----------------------------------------
struct MlError : std::runtime_error {
    int code;
    MlError(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};
[[noreturn]] void raise(int code, const std::string& msg);
void check_cuda(cudaError_t e, const char* what);
#define CK(x) ::mlg::check_cuda((x), #x)

struct BudgetInfo {
    std::string op;
    uint64_t requested = 0, used = 0, limit = 0;
};
void set_last_error(const std::string& m);
void set_budget_error(const BudgetInfo& b);
const char* last_error();
const BudgetInfo& last_budget();

// ---- memory pool: crates/minilake-exec/src/memory.rs:22-157 ---------------------------------
struct MemoryPool {
    uint64_t limit;
    std::atomic<uint64_t> used{0}, peak{0};
    explicit MemoryPool(uint64_t lim) : limit(lim ? lim : UINT64_MAX) {}
    // CAS loop: check + add is one atomic step (memory.rs:58-77)
    bool try_grow(uint64_t bytes, uint64_t* observed);
    void shrink(uint64_t bytes) { used.fetch_sub(bytes); }
};

class Ctx;

// RAII reservation (MemoryReservation, memory.rs:84-158).
class Reservation {
   public:
    Reservation(Ctx* ctx, std::string name) : ctx_(ctx), name_(std::move(name)) {}
    ~Reservation() { free(); }
    Reservation(const Reservation&) = delete;
    void try_grow(uint64_t bytes);
    void try_resize(uint64_t sz) {
        if (sz > size_) try_grow(sz - size_);
        else shrink(size_ - sz);
    }
    void shrink(uint64_t bytes);
    void free() { shrink(size_); }
    uint64_t size() const { return size_; }
    const std::string& name() const { return name_; }

   private:
    Ctx* ctx_;
    std::string name_;
    uint64_t size_ = 0;
};

// A device allocation from the context's caching allocator, charged to a reservation.
class DevBuf {
   public:
    DevBuf() = default;
    DevBuf(Ctx* ctx, size_t bytes, Reservation* res);
    ~DevBuf() { release(); }
    DevBuf(DevBuf&& o) noexcept { *this = std::move(o); }
    DevBuf& operator=(DevBuf&& o) noexcept;
    DevBuf(const DevBuf&) = delete;
    void release();
    template <class T = void> T* get() const { return (T*)ptr_; }
    size_t bytes() const { return bytes_; }
    explicit operator bool() const { return ptr_ != nullptr; }

   private:
    Ctx* ctx_ = nullptr;
    void* ptr_ = nullptr;
    size_t bytes_ = 0, cap_ = 0;
    Reservation* res_ = nullptr;
};

// Global string ids: every string a key reads (a dictionary entry, a plain string of a key
// column) gets one id per context, so group keys, join build sides and probe sides that hold
// equal strings hold equal ids whatever their encoding (the dictionaries differ per row group).
struct StringIntern {
    std::mutex mu;
    std::unordered_map<std::string, uint32_t> ids;
    std::vector<std::string> strs;
    uint32_t id(const std::string& s);  // mu held
};

// ---- context ------------------------------------------------------------------------------
class Ctx {
   public:
    Ctx(int device, uint64_t budget, uint32_t flags);
    ~Ctx();
    int device;
    uint32_t flags;
    MemoryPool pool;
    cudaStream_t stream = nullptr;  // default stream of the context
    std::atomic<uint64_t> launches{0};
    StringIntern strings;

    void* dalloc(size_t bytes, size_t* cap);
    void dfree(void* p, size_t cap);
    void* halloc(size_t bytes);  // pinned
    void hfree(void* p);
    // 64-byte pinned slots for small device->host readbacks (error words, counters),
    // carved from slabs that live as long as the context.
    void* pinned_slot();
    void release_slot(void* p);
    void set_current() const;
    cudaStream_t new_stream();
    void free_stream(cudaStream_t s);
    void sync_all();
    void count_launch(uint64_t n = 1) { launches.fetch_add(n); }
    bool profiling() const { return (flags & ML_CTX_PROFILE) != 0; }
    void add_profile(const std::string& k, double ms);
    void read_profile(const std::string& k, uint64_t* n, double* ms, bool reset);
    // Kernel timings are collected lazily: a launch's event pair waits here until the profile
    // is read (or the list is long), so timing a kernel adds no host synchronization.
    void add_timing(const char* name, cudaEvent_t a, cudaEvent_t b);
    cudaEvent_t get_event();

   private:
    std::mutex mu_, prof_mu_;
    std::map<std::string, std::pair<uint64_t, double>> prof_;
    struct Timing {
        const char* name;
        cudaEvent_t a, b;
    };
    std::vector<Timing> timings_;   // under prof_mu_
    std::vector<cudaEvent_t> events_;  // idle events, under prof_mu_
    void drain_timings(size_t keep);  // prof_mu_ held
    std::multimap<size_t, void*> free_;  // cached device blocks by capacity
    std::vector<cudaStream_t> streams_, idle_streams_;
    std::vector<void*> slabs_, free_slots_;
    size_t cached_bytes_ = 0;
};

// Times one kernel launch on `s` with CUDA events when the context profiles.
class KernelTimer {
   public:
    KernelTimer(Ctx* ctx, cudaStream_t s, const char* name);
    ~KernelTimer();
    void stop();  // records the end event; the time is collected when the profile is read

   private:
    Ctx* ctx_;
    cudaStream_t s_;
    const char* name_;
    cudaEvent_t a_ = nullptr, b_ = nullptr;
};

// Pinned staging buffer owned by one stream user.
class Staging {
   public:
    explicit Staging(Ctx* ctx) : ctx_(ctx) {}
    ~Staging();
    void* get(size_t bytes);

   private:
    Ctx* ctx_;
    void* p_ = nullptr;
    size_t cap_ = 0;
};

// ---- device batch ---------------------------------------------------------------------------
struct HostDict {  // dictionary of a dict-encoded string column (host copy)
    std::vector<uint32_t> off{0};
    std::vector<uint8_t> bytes;
    size_t len() const { return off.size() - 1; }
    std::string get(size_t i) const {
        return std::string((const char*)bytes.data() + off[i], off[i + 1] - off[i]);
    }
};

struct DevColumn {
    int dtype = ML_TYPE_INT64;
    int kind = CK_FIXED;  // CK_FIXED / CK_UTF8 / CK_DICT
    int64_t n = 0;
    DevBuf data, offsets, validity;
    std::shared_ptr<HostDict> dict;  // CK_DICT
    DevBuf strid;                    // canonical ids of a plain UTF8 column (build sides)
    // borrowed views (when the column was not copied)
    const void* data_p = nullptr;
    const uint32_t* off_p = nullptr;
    const uint64_t* valid_p = nullptr;
    const void* dptr() const { return data ? data.get() : data_p; }
    const uint32_t* optr() const { return offsets ? offsets.get<uint32_t>() : off_p; }
    const uint64_t* vptr() const { return validity ? validity.get<uint64_t>() : valid_p; }
    int64_t str_bytes_host() const;  // UTF8: total bytes (reads the last offset)
};

}  // namespace mlg

// Members are destroyed in reverse order: every reservation is declared before the
// device buffers charged to it, so the buffers are released while it is alive.
struct ml_batch {
    mlg::Ctx* ctx = nullptr;
    std::unique_ptr<mlg::Reservation> res;
    int64_t nrows = 0;
    std::vector<std::unique_ptr<mlg::DevColumn>> cols;
};

namespace mlg {

// Stage host or device ml_column views into device columns (host data is copied with
// cudaMemcpyAsync on `s`; device data is borrowed).
std::unique_ptr<DevColumn> stage_column(Ctx* ctx, const ml_column& c, int64_t nrows, cudaStream_t s, Staging& st,
                                        Reservation* res);
int width_of(int dtype);
// Host -> device copy that has landed when it returns (a pageable cudaMemcpy may return before
// its DMA ends, and kernels on non-blocking streams do not wait for the legacy stream).
void h2d_now(void* dst, const void* src, size_t bytes);

// ---- host scalar semantics (crates/minilake-core/src/scalar.rs, kernels/scalar_ops.rs) -------
struct HScalar {
    enum Kind { NUL = -1 } ;
    int kind = -1;  // -1 NULL, else ML_TYPE_*
    int64_t i = 0;
    double f = 0;
    std::string s;
    bool is_null() const { return kind < 0; }
    static HScalar b(bool v) { HScalar x; x.kind = ML_TYPE_BOOL; x.i = v; return x; }
};
HScalar scalar_cast(const HScalar& s, int to);
HScalar scalar_binary(int op, const HScalar& l, const HScalar& r);
std::optional<int> scalar_compare(const HScalar& a, const HScalar& b);
uint64_t scalar_bits(const HScalar& s);  // stack-machine representation
std::optional<int32_t> parse_date(const std::string& s);

// ---- expressions -------------------------------------------------------------------------------
struct ExprNode {
    int kind = 0, op = 0, dtype = 0, flag = 0;
    int64_t index = 0;
    HScalar lit;
    std::string str;
    std::vector<ExprNode> kids;
};
ExprNode parse_expr(const ml_expr& e);

// Where a column of an operator's output comes from.
struct ColRef {
    int kind = 0;  // 0 = source column, 1 = build column, 2 = computed expression
    int src = 0;   // 0 = pipeline source, p+1 = build side of probe p
    int index = 0;
    int dtype = 0;
    std::shared_ptr<ExprNode> expr;            // kind 2
    std::shared_ptr<std::vector<ColRef>> env;  // schema the expression reads
};
using Schema = std::vector<ColRef>;

// Per-column description of a pipeline's inputs, fixed when the pipeline is built.
struct SlotInfo {
    int src = 0, index = 0;
    int dtype = 0;
    int kind = CK_FIXED;
};

// A dictionary predicate evaluated once per dictionary entry (cmp.rs:47-61, string.rs:11-30).
struct LutSpec {
    int slot;         // column slot of the dict column
    int what;         // 0 = compare with literal, 1 = LIKE, 2 = IN list
    int op;           // comparison op
    int shape;        // LIKE shape
    bool negated;
    std::string lit;  // literal / pattern
    std::vector<std::string> list;
};

// Compiled program set of one pipeline.
class Compiler {
   public:
    std::vector<Instr> code;
    std::vector<uint8_t> arena;
    std::vector<SlotInfo> slots;
    std::vector<LutSpec> luts;
    std::vector<int> string_key_slots;  // slots read as string keys (global string ids)

    // Compile `e` (reading `schema`) as a value of type `out_type`.
    Prog compile_value(const ExprNode& e, const Schema& schema, int out_type);
    // Compile a string-valued key (dict global id / build canonical id).
    Prog compile_string_key(const ExprNode& e, const Schema& schema, int* slot_out);
    int slot_for(int src, int index, int dtype, int kind);
    // The source/build origin of a plain column reference (after inlining projections), or
    // nullopt if `e` is not a column reference.
    std::optional<SlotInfo> column_origin(const ExprNode& e, const Schema& schema);

    struct CV;
    CV compile(const ExprNode& e, const Schema& schema);

   private:
    int add_arena(const void* p, size_t n, size_t align = 8);
};

int like_shape(const std::string& pattern, std::string* inner);
void classify(Prog& p, const std::vector<Instr>& code);  // sets Prog::fast
bool like_match_host(const std::string& s, const std::string& p, int shape);

}  // namespace mlg
