// Pipelines: the streaming operators fused in front of a sink, compiled once and
// launched per pushed batch (morsel).
#pragma once

#include "ml_runtime.hpp"

struct ml_join_table;

namespace mlg {

// How a key field is decoded back into a column.
struct KeyDecode {
    int type = 0;
    int str_kind = 0;  // 0 = not a string, 1 = dictionary global id, 2 = build-side canonical row
    int build = -1;    // str_kind 2: probe index whose build batch holds the strings
    int build_col = -1;
    int slot = -1;     // column slot the key reads
};

struct ProbeInfo {
    ml_join_table* jt = nullptr;
    KeyLayout keys{};
};

class Pipeline {
   public:
    Pipeline(Ctx* ctx) : ctx(ctx), intern(ctx ? ctx->strings : own_strings_) {}
    Ctx* ctx;
    Compiler C;
    std::vector<int> input_types;
    Schema out;  // schema after the prologue (what the sink reads)
    int nstages = 0;
    Stage stages[kMaxFilters + kMaxProbes]{};
    std::vector<Prog> filters;
    std::vector<ProbeInfo> probes;
   private:
    StringIntern own_strings_;  // only for a pipeline without a context (source generation)

   public:
    // The context's string ids: dictionary entries and plain strings that a key reads
    StringIntern& intern;
    // The program and its arena in one device buffer (one copy per upload).
    DevBuf d_code;
    Instr* d_prog = nullptr;
    uint8_t* d_arena = nullptr;
    // Runtime-specialized kernels already looked up for this pipeline, by the launch's
    // structural signature (the fields the source generator reads), so repeated launches skip
    // generating the source again.
    mutable std::mutex jit_mu;
    mutable std::vector<std::pair<std::string, void*>> jit_memo;

    void build(const ml_pipe_op* ops, int nops, const int32_t* types, int ntypes);
    KeyLayout key_layout(const ml_expr* exprs, int n, const Schema& schema, bool group, std::vector<KeyDecode>* dec);
    void upload();

    // Per-launch state: staged source columns, gid maps and predicate tables.
    struct Launch {
        std::vector<std::unique_ptr<DevColumn>> src;
        DevBuf scratch;
        PipeArgs P{};
        std::vector<int> col_valid;  // slot has a validity bitmap in this launch
        // dictionary-coded source slots: the least and greatest string id of this batch's
        // dictionary (clamp entry included); first > second for every other slot
        std::vector<std::pair<uint32_t, uint32_t>> gid_range;
        std::vector<DevBuf> strids;  // global string ids of plain string key columns, per row
    };
    // With `tables_dst`, the per-batch tables are copied there (at most `tables_cap` bytes,
    // from pageable memory) instead of into a new device buffer.
    void prepare(Launch& L, const ml_column* cols, int ncols, int64_t nrows, const uint32_t* sel, int64_t nsel,
                 cudaStream_t s, Staging& st, Reservation* res, uint8_t* tables_dst = nullptr, size_t tables_cap = 0);
    // Global string ids (the context's intern table) of every row of a plain UTF8 column.
    DevBuf intern_plain_strings(const DevColumn& col, cudaStream_t s);
    // Slot mask check: does program `p` read a column with a validity bitmap?
    bool reads_nullable(const Prog& p, const Launch& L) const;
};

// Ordered selection of the rows where all of the pipeline's stages pass (no probes).
// Returns the number of selected rows; `out` holds them (device).  Its device buffers are
// charged to `res` when given.
int64_t run_select(Ctx* ctx, const Pipeline& pipe, const PipeArgs& P, DevBuf& out, cudaStream_t s,
                   Reservation* res = nullptr);

// Exclusive scan helper (device u32 counts -> u64 offsets incl. total); returns the total.
uint64_t scan_counts(Ctx* ctx, const uint32_t* counts, int64_t n, DevBuf& offsets, cudaStream_t s,
                     Reservation* res = nullptr);

// Gather a plain UTF8 column: strings at `idx` (or all rows) into a new column.
void gather_utf8(Ctx* ctx, const uint32_t* off, const uint8_t* bytes, const uint32_t* idx, int64_t k, DevColumn& out,
                 cudaStream_t s, Reservation* res);

}  // namespace mlg

struct ml_join_table {
    mlg::Ctx* ctx = nullptr;
    std::unique_ptr<mlg::Reservation> res;  // declared first: released last
    ml_batch batch;  // the concatenated build side
    std::vector<int> key_types;
    std::vector<int> key_cols;  // build key k is build column key_cols[k] (-1: a computed key)
    int nwords = 1;
    mlg::DevBuf slots, next, dup;
    uint64_t cap = 0;
    bool has_dups = false;
    // Dense integer key: a direct-mapped index replaces the hash table (see ProbeDev).
    mlg::DevBuf dense;
    uint64_t dmin = 0, drange = 0;
    // One bit per dense index position (a build row has that key): the semi-join form of the
    // index (ProbeDev::member), built by the first launch that probes the table as a semi-join
    // (member_bits); `member_ready` marks its completion for launches on other streams.
    mlg::DevBuf member;
    cudaEvent_t member_ready = nullptr;
    std::mutex member_mu;
    ~ml_join_table() {
        if (member_ready) cudaEventDestroy(member_ready);
    }
    mlg::TableView view() const {
        mlg::TableView t{};
        t.slots = slots.get<uint64_t>();
        t.mask = cap - 1;
        t.nwords = nwords;
        t.stride = nwords == 1 ? 2 : 4;
        return t;
    }
};
