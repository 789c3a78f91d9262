// TEST INFRASTRUCTURE — CPU oracle, part 3: C entry points used by the tests
// and by bench.py's CPU baseline.  Pipelines run morsel-driven on std::threads
// exactly like MiniLake's executor: an atomic morsel counter
// (scheduler.rs:44-68), one thread-local sink per worker (pipeline.rs:109-136),
// `combine` under a mutex once per worker, then `finalize` on one thread.
#include <algorithm>
#include <thread>

#include "orc.hpp"

using namespace orc;

namespace {
thread_local std::string g_err;
thread_local Error g_budget(0, "");

int handle_exc(const std::exception& e) {
    g_err = e.what();
    if (auto* x = dynamic_cast<const Error*>(&e)) {
        if (x->code == ML_ERR_BUDGET) g_budget = *x;
        return x->code;
    }
    return ML_ERR_INTERNAL;
}
#define ORC_TRY try {
#define ORC_CATCH                                   \
    }                                               \
    catch (const std::exception& e) { return handle_exc(e); }

struct OBatch {
    std::vector<ColPtr> cols;
    size_t n = 0;
    // host views handed out by orc_batch_columns
    std::vector<std::vector<uint32_t>> dict_off;
};

ColPtr slice_view(const ColPtr& base, size_t off, size_t len) {
    auto c = std::make_shared<Column>(*base);
    c->n = len;
    if (base->dt == UTF8 && !base->dict) {
        c->off = base->off + off;
    } else {
        size_t w = base->dict ? 4 : (base->dt == BOOL ? 1 : (base->dt == I32 || base->dt == DATE) ? 4 : 8);
        c->vals = (const uint8_t*)base->vals + off * w;
    }
    if (base->vw) {
        c->voff = base->voff + off;
        bool any_null = false;  // Column::new drops a bitmap without nulls
        for (size_t i = 0; i < len && !any_null; i++) any_null = !c->valid(i);
        if (!any_null) c->vw = nullptr;
    }
    c->own = base;
    return c;
}

std::vector<Expr> parse_list(const ml_expr* e, int n) {
    std::vector<Expr> v;
    for (int i = 0; i < n; i++) v.push_back(parse_expr(e[i]));
    return v;
}

std::vector<PipeOp> parse_prologue(const ml_pipe_op* ops, int n) {
    std::vector<PipeOp> out;
    for (int i = 0; i < n; i++) {
        PipeOp p;
        p.kind = ops[i].kind;
        p.exprs = parse_list(ops[i].exprs, ops[i].nexprs);
        for (int k = 0; k < ops[i].nexprs; k++) p.types.push_back(ops[i].exprs[k].dtype);
        p.join = (const JoinTable*)ops[i].join;
        p.build_is_left = ops[i].build_is_left != 0;
        if (p.kind == ML_PIPE_PROBE && !p.join) fail(ML_ERR_INVALID, "probe without a join table");
        out.push_back(std::move(p));
    }
    return out;
}

size_t batch_memory(const Batch& b) {  // Batch::memory_size approximation
    size_t s = 0;
    for (auto& c : b.cols) {
        size_t w = c->dt == BOOL ? 1 : (c->dt == I32 || c->dt == DATE || c->dict) ? 4 : 8;
        if (c->dt == UTF8 && !c->dict) s += (c->n + 1) * 4 + (c->off[c->n] - c->off[0]);
        else s += c->n * w;
        if (c->vw) s += (c->n + 63) / 64 * 8;
    }
    return s;
}

// Run `work(worker)` on `threads` workers (scheduler.rs:102-144).
void run_parallel(int threads, const std::function<void(int)>& work, std::atomic<bool>& cancel) {
    if (threads <= 1) {
        work(0);
        return;
    }
    std::vector<std::exception_ptr> errs(threads);
    std::vector<std::thread> ts;
    for (int w = 0; w < threads; w++)
        ts.emplace_back([&, w]() {
            try {
                work(w);
            } catch (...) {
                errs[w] = std::current_exception();
                cancel.store(true);
            }
        });
    for (auto& t : ts) t.join();
    for (auto& e : errs)
        if (e) std::rethrow_exception(e);
}

// Drive a pipeline: morsels -> batches -> operators -> local sink.
template <class Local>
void drive(const ml_column* cols, int nmorsels, int ncols, const int64_t* rows, const std::vector<PipeOp>& ops,
           int threads, size_t batch_size, const std::function<std::unique_ptr<Local>()>& make_local,
           const std::function<void(std::unique_ptr<Local>)>& combine) {
    std::atomic<int> next{0};
    std::atomic<bool> cancel{false};
    if (threads < 1) threads = 1;
    batch_size = std::max<size_t>(batch_size, 1);
    run_parallel(
        threads,
        [&](int) {
            auto local = make_local();
            for (;;) {
                int m = next.fetch_add(1);
                if (m >= nmorsels || cancel.load()) break;
                size_t n = (size_t)rows[m];
                std::vector<ColPtr> base;
                for (int c = 0; c < ncols; c++) base.push_back(column_from_view(cols[(size_t)m * ncols + c], 0, (int64_t)n));
                for (size_t off = 0; off < n; off += batch_size) {
                    size_t len = std::min(batch_size, n - off);
                    Batch b;
                    b.n = len;
                    for (auto& bc : base) b.cols.push_back(slice_view(bc, off, len));
                    run_operators(ops, 0, std::move(b), [&](Batch x) { local->sink(std::move(x)); });
                }
            }
            combine(std::move(local));
        },
        cancel);
}

// ---- HashAggregate sink (aggregate/hash.rs:285-484, ungrouped.rs) --------------------
struct AggShared {
    std::vector<Expr> group;
    std::vector<int> key_types;
    std::vector<AggSpec> aggs;
    std::shared_ptr<MemoryPool> pool;
    std::mutex mu;
    std::unique_ptr<HashAggState> global;
    std::optional<MemoryReservation> global_res;
    std::vector<Accumulator> ungrouped;  // no GROUP BY: one slot
    bool have_ungrouped = false;
};
struct AggLocal {
    AggShared* sh;
    HashAggState state;
    MemoryReservation res;
    std::vector<Accumulator> accs;
    AggLocal(AggShared* s) : sh(s), state(s->key_types, s->aggs), res(s->pool, "HashAggregate") {
        for (auto& a : s->aggs) {
            accs.emplace_back(a.func, a.arg_type);
            accs.back().resize(1);
        }
    }
    void sink(Batch b) {
        if (sh->group.empty()) {  // UngroupedLocal::sink (ungrouped.rs:113-131)
            const uint32_t* rows = b.sel ? b.sel->data() : nullptr;
            size_t k = b.sel ? b.sel->size() : b.n;
            for (size_t a = 0; a < sh->aggs.size(); a++) {
                ColPtr arg;
                if (sh->aggs[a].arg) arg = accs[a].prepare_input(evaluate_to_column(*sh->aggs[a].arg, b, sh->aggs[a].arg_type));
                accs[a].update(arg.get(), b.n, rows, k, nullptr);
            }
            return;
        }
        state.update(b, sh->group, sh->aggs);
        res.try_resize(state.memory_size());  // HashAggLocal::account without a spill dir
    }
};

}  // namespace

extern "C" {

const char* orc_last_error(void) { return g_err.c_str(); }
int orc_last_budget_error(char* op, size_t cap, uint64_t* requested, uint64_t* used, uint64_t* limit) {
    if (op && cap) {
        strncpy(op, g_budget.op.c_str(), cap - 1);
        op[cap - 1] = 0;
    }
    if (requested) *requested = g_budget.requested;
    if (used) *used = g_budget.used;
    if (limit) *limit = g_budget.limit;
    return ML_OK;
}

uint64_t orc_hash_u64(uint64_t x) { return hash_u64(x); }
uint64_t orc_combine(uint64_t h, uint64_t v) { return combine(h, v); }
uint64_t orc_hash_bytes(const uint8_t* b, size_t n) { return hash_bytes(b, n); }
uint64_t orc_fold_mul(uint64_t a, uint64_t b) { return fold_mul(a, b); }
uint64_t orc_swar_match_tag(uint64_t g, uint8_t tag) { return swar_match_tag(g, tag); }
uint64_t orc_swar_match_empty(uint64_t g) { return swar_match_empty(g); }

// Property-test driver for SwissTable::find_or_insert_batch (proptest_tables.rs:14-41):
// `keys` holds nbatch batches (sizes in `sizes`); hash_mode 0 = hash_u64, 1 = x % 4,
// 2 = constant 42.  Writes the payload of every key into `out`; returns len via *len and
// verifies every stored key with find() (status ML_ERR_INTERNAL on mismatch).
int orc_swiss_batches(const uint64_t* keys, const int64_t* sizes, int nbatch, int hash_mode, uint32_t* out,
                      int64_t* len, int64_t* capacity) {
    ORC_TRY
    SwissTable t(0);
    std::vector<uint64_t> stored;
    auto hf = [&](uint64_t k) { return hash_mode == 0 ? hash_u64(k) : hash_mode == 1 ? k % 4 : 42ull; };
    size_t pos = 0;
    std::vector<uint32_t> o;
    for (int b = 0; b < nbatch; b++) {
        std::vector<uint64_t> hs;
        const uint64_t* in = keys + pos;
        for (int64_t i = 0; i < sizes[b]; i++) hs.push_back(hf(in[i]));
        struct KS {
            const uint64_t* in;
            std::vector<uint64_t>& st;
            bool equals(uint32_t p, size_t k) const { return st[p] == in[k]; }
            uint32_t insert(size_t k) {
                st.push_back(in[k]);
                return (uint32_t)(st.size() - 1);
            }
        } ks{in, stored};
        t.find_or_insert_batch(hs, ks, o);
        for (int64_t i = 0; i < sizes[b]; i++) out[pos + i] = o[i];
        pos += sizes[b];
    }
    for (size_t g = 0; g < stored.size(); g++) {
        auto f = t.find(hf(stored[g]), [&](uint32_t p) { return stored[p] == stored[g]; });
        if (!f || *f != g) fail(ML_ERR_INTERNAL, "find after insert disagrees");
    }
    *len = (int64_t)t.len;
    *capacity = (int64_t)t.capacity();
    return ML_OK;
    ORC_CATCH
}

// MemoryPool known-answer driver (memory.rs:160-201): ops[i] = (reservation id, kind, bytes)
// kind 0 = try_grow, 1 = try_resize, 2 = drop.  results[i] = status; used/peak after each op.
int orc_pool_script(uint64_t limit, const int64_t* ops, int nops, int* results, uint64_t* used, uint64_t* peak) {
    ORC_TRY
    auto pool = std::make_shared<MemoryPool>(limit);
    std::vector<std::unique_ptr<MemoryReservation>> res(16);
    for (int i = 0; i < nops; i++) {
        int id = (int)ops[3 * i], kind = (int)ops[3 * i + 1];
        uint64_t bytes = (uint64_t)ops[3 * i + 2];
        if (!res[id]) res[id] = std::make_unique<MemoryReservation>(pool, "r" + std::to_string(id));
        results[i] = ML_OK;
        try {
            if (kind == 0) res[id]->try_grow(bytes);
            else if (kind == 1) res[id]->try_resize(bytes);
            else res[id].reset();
        } catch (const Error& e) {
            results[i] = e.code;
            if (e.code == ML_ERR_BUDGET) g_budget = e;
        }
        used[i] = pool->used.load();
        peak[i] = pool->peak.load();
    }
    return ML_OK;
    ORC_CATCH
}

// ---- single-batch operators -------------------------------------------------------------
int orc_filter(const ml_expr* pred, const ml_column* cols, int ncols, int64_t nrows, const uint32_t* sel_in,
               int64_t nsel_in, uint32_t* sel_out, int64_t* nout) {
    ORC_TRY
    Batch b;
    b.n = (size_t)nrows;
    for (int c = 0; c < ncols; c++) b.cols.push_back(column_from_view(cols[c], 0, nrows));
    std::vector<uint32_t> in;
    if (sel_in) in.assign(sel_in, sel_in + nsel_in);
    auto s = select(parse_expr(*pred), b, sel_in ? &in : nullptr);
    std::copy(s.begin(), s.end(), sel_out);
    *nout = (int64_t)s.size();
    return ML_OK;
    ORC_CATCH
}

int orc_project(const ml_expr* e, const ml_column* cols, int ncols, int64_t nrows, void** out) {
    ORC_TRY
    Batch b;
    b.n = (size_t)nrows;
    for (int c = 0; c < ncols; c++) b.cols.push_back(column_from_view(cols[c], 0, nrows));
    auto ob = new OBatch();
    ob->cols.push_back(evaluate_to_column(parse_expr(*e), b, e->dtype));
    ob->n = (size_t)nrows;
    *out = ob;
    return ML_OK;
    ORC_CATCH
}

int orc_hash_columns(const ml_column* cols, int ncols, int64_t nrows, const uint32_t* sel, int64_t nsel,
                     uint64_t* out) {
    ORC_TRY
    std::vector<ColPtr> cs;
    for (int c = 0; c < ncols; c++) cs.push_back(column_from_view(cols[c], 0, nrows));
    std::vector<uint64_t> h;
    hash_columns(cs, (size_t)nrows, sel, (size_t)(sel ? nsel : nrows), h);
    std::copy(h.begin(), h.end(), out);
    return ML_OK;
    ORC_CATCH
}

// ---- sinks over morsels -------------------------------------------------------------------
int orc_hashagg_run(const ml_column* cols, int nmorsels, int ncols, const int64_t* rows, const ml_pipe_op* pro,
                    int npro, const ml_expr* group, int ngroup, const ml_agg_spec* aggs, int nagg, int threads,
                    int64_t batch_size, uint64_t pool_limit, void** out) {
    ORC_TRY
    AggShared sh;
    sh.group = parse_list(group, ngroup);
    for (int g = 0; g < ngroup; g++) sh.key_types.push_back(group[g].dtype);
    for (int a = 0; a < nagg; a++) {
        AggSpec s;
        s.func = aggs[a].func;
        s.arg_type = aggs[a].func == ML_AGG_COUNT_STAR ? -1 : aggs[a].arg_type;
        if (aggs[a].arg.nnodes > 0) s.arg = parse_expr(aggs[a].arg);
        sh.aggs.push_back(std::move(s));
    }
    sh.pool = std::make_shared<MemoryPool>(pool_limit);
    auto ops = parse_prologue(pro, npro);
    drive<AggLocal>(
        cols, nmorsels, ncols, rows, ops, threads, (size_t)batch_size,
        [&]() { return std::make_unique<AggLocal>(&sh); },
        [&](std::unique_ptr<AggLocal> l) {  // HashAggLocal::combine (aggregate/hash.rs:439-484)
            std::lock_guard<std::mutex> g(sh.mu);
            if (sh.group.empty()) {
                if (!sh.have_ungrouped) {
                    sh.ungrouped = std::move(l->accs);
                    sh.have_ungrouped = true;
                } else {
                    uint32_t z = 0;
                    for (size_t a = 0; a < sh.ungrouped.size(); a++) sh.ungrouped[a].merge(l->accs[a].state(), &z, 1);
                }
                return;
            }
            if (!sh.global) {
                sh.global = std::make_unique<HashAggState>(std::move(l->state));
            } else {
                sh.global->merge_state(l->state);
            }
            l->res.free();
            if (!sh.global_res) sh.global_res.emplace(sh.pool, "HashAggregate(global)");
            sh.global_res->try_resize(sh.global->memory_size());
        });
    auto ob = new OBatch();
    if (sh.group.empty()) {  // UngroupedAggregateSink::finalize
        if (!sh.have_ungrouped)
            for (auto& a : sh.aggs) {
                sh.ungrouped.emplace_back(a.func, a.arg_type);
                sh.ungrouped.back().resize(1);
            }
        for (auto& a : sh.ungrouped) ob->cols.push_back(a.finish());
        ob->n = 1;
    } else if (sh.global) {
        Batch fb = sh.global->final_batch();
        ob->cols = fb.cols;
        ob->n = fb.n;
    } else {
        HashAggState empty(sh.key_types, sh.aggs);
        Batch fb = empty.final_batch();
        ob->cols = fb.cols;
        ob->n = 0;
    }
    *out = ob;
    return ML_OK;
    ORC_CATCH
}

int orc_join_build_run(const ml_column* cols, int nmorsels, int ncols, const int64_t* rows, const ml_pipe_op* pro,
                       int npro, const ml_expr* keys, int nkeys, int threads, int64_t batch_size,
                       uint64_t pool_limit, void** out) {
    ORC_TRY
    auto ops = parse_prologue(pro, npro);
    std::vector<Expr> kx = parse_list(keys, nkeys);
    std::vector<int> kt;
    for (int k = 0; k < nkeys; k++) kt.push_back(keys[k].dtype);
    auto pool = std::make_shared<MemoryPool>(pool_limit);
    struct BLocal {
        std::vector<Batch> batches;
        MemoryReservation res;
        BLocal(std::shared_ptr<MemoryPool> p) : res(std::move(p), "HashJoinBuild") {}
        void sink(Batch b) {  // BuildLocal::sink (join.rs:217-222)
            Batch c = b.compact();
            res.try_grow(batch_memory(c));
            batches.push_back(std::move(c));
        }
    };
    std::mutex mu;
    std::vector<Batch> all;
    std::vector<MemoryReservation> reservations;
    size_t out_cols = (size_t)ncols;
    drive<BLocal>(
        cols, nmorsels, ncols, rows, ops, threads, (size_t)batch_size, [&]() { return std::make_unique<BLocal>(pool); },
        [&](std::unique_ptr<BLocal> l) {
            std::lock_guard<std::mutex> g(mu);
            for (auto& b : l->batches) all.push_back(std::move(b));
            reservations.push_back(std::move(l->res));
        });
    if (!all.empty()) out_cols = all[0].cols.size();
    else {
        // column count after the prologue: a projection changes it, a probe adds the build side
        for (auto& op : ops) {
            if (op.kind == ML_PIPE_PROJECT) out_cols = op.exprs.size();
            if (op.kind == ML_PIPE_PROBE) out_cols += op.join->batch.cols.size();
        }
    }
    auto jt = build_table(all, kx, kt, out_cols);
    *out = jt.release();
    return ML_OK;
    ORC_CATCH
}
int orc_join_destroy(void* j) {
    delete (JoinTable*)j;
    return ML_OK;
}
int orc_join_stats(void* j, int64_t* build_rows, int64_t* distinct, int64_t* capacity) {
    auto* jt = (JoinTable*)j;
    *build_rows = (int64_t)jt->batch.n;
    *distinct = (int64_t)jt->table.len;
    *capacity = (int64_t)jt->table.capacity();
    return ML_OK;
}

int orc_join_probe(void* j, const ml_expr* keys, int nkeys, const ml_column* cols, int ncols, int64_t nrows,
                   const uint32_t* sel, int64_t nsel, uint32_t* pi, uint32_t* bi, int64_t cap, int64_t* npairs) {
    ORC_TRY
    Batch b;
    b.n = (size_t)nrows;
    for (int c = 0; c < ncols; c++) b.cols.push_back(column_from_view(cols[c], 0, nrows));
    if (sel) b.sel = std::make_shared<const std::vector<uint32_t>>(sel, sel + nsel);
    std::vector<int> kt;
    for (int k = 0; k < nkeys; k++) kt.push_back(keys[k].dtype);
    std::vector<uint32_t> p, q;
    probe_pairs(*(JoinTable*)j, parse_list(keys, nkeys), kt, b, p, q);
    *npairs = (int64_t)p.size();
    if ((int64_t)p.size() > cap) fail(ML_ERR_INVALID, "pair buffer too small");
    std::copy(p.begin(), p.end(), pi);
    std::copy(q.begin(), q.end(), bi);
    return ML_OK;
    ORC_CATCH
}

int orc_topn_run(const ml_column* cols, int nmorsels, int ncols, const int64_t* rows, const ml_pipe_op* pro, int npro,
                 const ml_sort_key* keys, int nkeys, int64_t limit, int threads, int64_t batch_size, void** out) {
    ORC_TRY
    auto ops = parse_prologue(pro, npro);
    std::vector<SortKey> sk;
    for (int k = 0; k < nkeys; k++) sk.push_back({parse_expr(keys[k].expr), keys[k].asc != 0, keys[k].nulls_first != 0});
    // limit < 0: ORDER BY without a limit (sort.rs:85-132, `limit: None`)
    const std::optional<size_t> l = limit < 0 ? std::nullopt : std::optional<size_t>((size_t)limit);
    size_t out_cols = (size_t)ncols;
    for (auto& op : ops) {
        if (op.kind == ML_PIPE_PROJECT) out_cols = op.exprs.size();
        if (op.kind == ML_PIPE_PROBE) out_cols += op.join->batch.cols.size();
    }
    struct TLocal {  // SortLocal (sort.rs:178-267)
        const std::vector<SortKey>* keys;
        std::optional<size_t> limit;
        size_t ncols, rows = 0;
        std::vector<Batch> batches;
        void truncate() {
            auto b = sort_batches(batches, *keys, limit, ncols);
            if (b) {
                rows = b->n;
                batches = {std::move(*b)};
            }
        }
        void sink(Batch b) {
            rows += b.active_rows();
            batches.push_back(b.compact());
            if (limit && rows > std::max<size_t>(4 * *limit, 16384)) truncate();
        }
    };
    std::mutex mu;
    std::vector<Batch> all;
    drive<TLocal>(
        cols, nmorsels, ncols, rows, ops, threads, (size_t)batch_size,
        [&]() {
            auto t = std::make_unique<TLocal>();
            t->keys = &sk;
            t->limit = l;
            t->ncols = out_cols;
            return t;
        },
        [&](std::unique_ptr<TLocal> t) {
            t->truncate();
            std::lock_guard<std::mutex> g(mu);
            for (auto& b : t->batches) all.push_back(std::move(b));
        });
    auto ob = new OBatch();
    auto r = sort_batches(all, sk, l, out_cols);
    if (r) {
        ob->cols = r->cols;
        ob->n = r->n;
    }
    *out = ob;
    return ML_OK;
    ORC_CATCH
}

// ---- results -------------------------------------------------------------------------------
int orc_batch_num_rows(void* b, int64_t* n) {
    *n = (int64_t)((OBatch*)b)->n;
    return ML_OK;
}
int orc_batch_num_columns(void* b, int32_t* n) {
    *n = (int32_t)((OBatch*)b)->cols.size();
    return ML_OK;
}
int orc_batch_column_info(void* bp, int32_t col, int32_t* dtype, int64_t* str_bytes, int32_t* has_validity) {
    auto* b = (OBatch*)bp;
    if (col < 0 || (size_t)col >= b->cols.size()) {
        g_err = "column out of range";
        return ML_ERR_INVALID;
    }
    const Column& c = *b->cols[col];
    *dtype = c.dt;
    int64_t sb = 0;
    if (c.dt == UTF8)
        for (size_t i = 0; i < c.n; i++) sb += (int64_t)c.str(i).size();
    *str_bytes = sb;
    *has_validity = c.vw != nullptr;
    return ML_OK;
}
// Copies a column: fixed width values; UTF8 as offsets (n+1) + bytes (dictionary decoded).
int orc_batch_fetch(void* bp, int32_t col, void* values, uint32_t* offsets, uint64_t* validity) {
    auto* b = (OBatch*)bp;
    if (col < 0 || (size_t)col >= b->cols.size()) {
        g_err = "column out of range";
        return ML_ERR_INVALID;
    }
    const Column& c = *b->cols[col];
    size_t n = c.n;
    if (c.dt == UTF8) {
        uint32_t pos = 0;
        uint8_t* out = (uint8_t*)values;
        for (size_t i = 0; i < n; i++) {
            offsets[i] = pos;
            auto s = c.str(i);
            memcpy(out + pos, s.data(), s.size());
            pos += (uint32_t)s.size();
        }
        offsets[n] = pos;
    } else {
        size_t w = c.dt == BOOL ? 1 : (c.dt == I32 || c.dt == DATE) ? 4 : 8;
        memcpy(values, c.vals, n * w);
    }
    if (validity) {
        size_t nw = (n + 63) / 64;
        for (size_t k = 0; k < nw; k++) validity[k] = 0;
        for (size_t i = 0; i < n; i++)
            if (c.valid(i)) validity[i / 64] |= 1ull << (i % 64);
    }
    return ML_OK;
}
// Host views of the batch's columns (dictionary columns are exposed as plain UTF8 copies are
// not needed: a dict column keeps its dictionary), for feeding another oracle pipeline.
int orc_batch_columns(void* bp, ml_column* out, int32_t ncols) {
    auto* b = (OBatch*)bp;
    if ((size_t)ncols != b->cols.size()) {
        g_err = "column count mismatch";
        return ML_ERR_INVALID;
    }
    b->dict_off.assign(b->cols.size(), {});
    for (size_t i = 0; i < b->cols.size(); i++) {
        const Column& c = *b->cols[i];
        ml_column m{};
        m.dtype = c.dt;
        m.len = (int64_t)c.n;
        m.location = ML_LOC_HOST;
        if (c.vw && c.voff != 0) {
            g_err = "unaligned validity";
            return ML_ERR_INTERNAL;
        }
        m.validity = c.vw;
        if (c.dt == UTF8 && c.dict) {
            m.encoding = ML_ENC_DICT;
            m.data = c.vals;
            m.dict_len = (int64_t)c.dictv->len();
            m.dict_offsets = c.dictv->off.data();
            m.dict_data = c.dictv->bytes.data();
        } else if (c.dt == UTF8) {
            m.encoding = ML_ENC_PLAIN;
            m.offsets = c.off;
            m.data = c.bytes;
        } else {
            m.data = c.vals;
        }
        out[i] = m;
    }
    return ML_OK;
}
int orc_batch_destroy(void* b) {
    delete (OBatch*)b;
    return ML_OK;
}

}  // extern "C"
