// C ABI of the MiniLake B200 execution core (include/minilake_gpu.h).
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <shared_mutex>

#include "ml_api_common.hpp"
#include "ml_jit.hpp"
#include "ml_pipeline.hpp"

using namespace mlg;



namespace {

uint64_t pow2_at_least(uint64_t x) {
    uint64_t p = 1;
    while (p < x) p <<= 1;
    return p;
}

bool is_device_ptr(const void* p) {
    if (!p) return false;
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

// Selection vector on the device (copied when it is host memory).
const uint32_t* device_sel(Ctx* ctx, const uint32_t* sel, int64_t nsel, DevBuf& hold, cudaStream_t s,
                           Reservation* res = nullptr) {
    if (!sel) return nullptr;
    if (nsel < 0) raise(ML_ERR_INVALID, "negative selection length");
    if (is_device_ptr(sel)) return sel;
    hold = DevBuf(ctx, std::max<size_t>((size_t)nsel * 4, 4), res);
    if (nsel) CK(cudaMemcpyAsync(hold.get(), sel, (size_t)nsel * 4, cudaMemcpyHostToDevice, s));
    return hold.get<uint32_t>();
}

void check_sel_bounds(const uint32_t* sel, int64_t nsel, int64_t nrows) {
    if (!sel || is_device_ptr(sel)) return;  // device selections are trusted like device columns
    for (int64_t i = 0; i < nsel; i++)
        if (sel[i] >= (uint64_t)nrows) raise(ML_ERR_INVALID, "selection index out of range");
}

// Deep copy of expressions (the caller's nodes are borrowed only for the call).
struct OwnedExprs {
    std::vector<std::vector<ml_expr_node>> nodes;
    std::vector<std::string> strs;
    std::vector<ml_expr> exprs;
    void add(const ml_expr& e) {
        if (!e.nodes || e.nnodes <= 0) raise(ML_ERR_INVALID, "empty expression");
        nodes.emplace_back(e.nodes, e.nodes + e.nnodes);
        exprs.push_back(e);
    }
    void finish() {
        strs.reserve(4096);
        for (size_t i = 0; i < nodes.size(); i++) {
            for (auto& n : nodes[i])
                if (n.str) {
                    strs.emplace_back(n.str, (size_t)n.str_len);
                    n.str = strs.back().data();
                }
            exprs[i].nodes = nodes[i].data();
        }
    }
};

std::unique_ptr<DevColumn> copy_column(Ctx* ctx, const DevColumn& s, cudaStream_t st, Reservation* res) {
    auto d = std::make_unique<DevColumn>();
    d->dtype = s.dtype;
    d->kind = s.kind;
    d->n = s.n;
    d->dict = s.dict;
    if (s.kind == CK_UTF8) {
        uint32_t first = 0, last = 0;
        if (s.n) {
            CK(cudaMemcpyAsync(&first, s.optr(), 4, cudaMemcpyDeviceToHost, st));
            CK(cudaMemcpyAsync(&last, s.optr() + s.n, 4, cudaMemcpyDeviceToHost, st));
            CK(cudaStreamSynchronize(st));
        }
        d->offsets = DevBuf(ctx, (size_t)(s.n + 1) * 4, res);
        launch_offsets_rebase(s.optr(), s.n, 0, d->offsets.get<uint32_t>(), st);
        ctx->count_launch();
        d->data = DevBuf(ctx, std::max<size_t>(last - first, 1), res);
        if (last > first)
            CK(cudaMemcpyAsync(d->data.get(), (const uint8_t*)s.dptr() + first, last - first, cudaMemcpyDeviceToDevice, st));
    } else {
        size_t w = s.kind == CK_DICT ? 4 : (size_t)width_of(s.dtype);
        d->data = DevBuf(ctx, std::max<size_t>(s.n * w, 1), res);
        if (s.n) CK(cudaMemcpyAsync(d->data.get(), s.dptr(), s.n * w, cudaMemcpyDeviceToDevice, st));
    }
    if (s.vptr()) {
        size_t vb = (size_t)(s.n + 63) / 64 * 8;
        d->validity = DevBuf(ctx, std::max<size_t>(vb, 8), res);
        if (vb) CK(cudaMemcpyAsync(d->validity.get(), s.vptr(), vb, cudaMemcpyDeviceToDevice, st));
    }
    return d;
}

// Rows `idx` (device, k entries; nullptr = all rows) of a column into a new owned column.
// Dictionary strings are decoded into plain UTF8.
std::unique_ptr<DevColumn> gather_column(Ctx* ctx, const DevColumn& s, const uint32_t* idx, int64_t k, cudaStream_t st,
                                         Reservation* res) {
    if (!idx && s.kind != CK_DICT) return copy_column(ctx, s, st, res);
    auto d = std::make_unique<DevColumn>();
    d->dtype = s.dtype;
    d->n = k;
    if (s.kind == CK_FIXED) {
        d->kind = CK_FIXED;
        int w = width_of(s.dtype);
        d->data = DevBuf(ctx, std::max<size_t>((size_t)k * w, 1), res);
        launch_gather_fixed(s.dptr(), w, idx, k, d->data.get(), st);
        ctx->count_launch();
    } else if (s.kind == CK_UTF8) {
        gather_utf8(ctx, s.optr(), (const uint8_t*)s.dptr(), idx, k, *d, st, res);
    } else {  // dictionary: codes -> dictionary strings
        DevBuf codes;
        const uint32_t* cidx = (const uint32_t*)s.dptr();
        if (idx) {
            codes = DevBuf(ctx, std::max<size_t>((size_t)k * 4, 4), nullptr);
            launch_gather_fixed(s.dptr(), 4, idx, k, codes.get(), st);
            ctx->count_launch();
            cidx = codes.get<uint32_t>();
        }
        const HostDict& hd = *s.dict;
        DevBuf doff(ctx, hd.off.size() * 4, nullptr), dbytes(ctx, std::max<size_t>(hd.bytes.size(), 1), nullptr);
        CK(cudaMemcpyAsync(doff.get(), hd.off.data(), hd.off.size() * 4, cudaMemcpyHostToDevice, st));
        if (!hd.bytes.empty()) CK(cudaMemcpyAsync(dbytes.get(), hd.bytes.data(), hd.bytes.size(), cudaMemcpyHostToDevice, st));
        gather_utf8(ctx, doff.get<uint32_t>(), dbytes.get<uint8_t>(), cidx, k, *d, st, res);
        CK(cudaStreamSynchronize(st));
    }
    if (s.vptr()) {
        size_t words = (size_t)(k + 63) / 64;
        d->validity = DevBuf(ctx, std::max<size_t>(words * 8, 8), res);
        CK(cudaMemsetAsync(d->validity.get(), 0, std::max<size_t>(words * 8, 8), st));
        if (idx) {
            launch_gather_valid(s.vptr(), idx, k, d->validity.get<uint32_t>(), st);
        } else {
            launch_copy_bits(s.vptr(), k, d->validity.get<uint64_t>(), 0, st);
        }
        ctx->count_launch();
    }
    return d;
}

// Evaluate program `p` for the rows of launch `P` into a new fixed-width column.
std::unique_ptr<DevColumn> project_column(Ctx* ctx, const PipeArgs& P, Prog p, int type, cudaStream_t st, Reservation* res) {
    auto d = std::make_unique<DevColumn>();
    d->dtype = type;
    d->kind = CK_FIXED;
    d->n = P.n;
    d->data = DevBuf(ctx, std::max<size_t>((size_t)P.n * width_of(type), 1), res);
    size_t words = (size_t)(P.n + 63) / 64;
    d->validity = DevBuf(ctx, std::max<size_t>(words * 8, 8), res);
    CK(cudaMemsetAsync(d->validity.get(), 0, std::max<size_t>(words * 8, 8), st));
    launch_project(P, p, type, d->data.get(), d->validity.get<uint32_t>(), st);
    ctx->count_launch();
    return d;
}

void check_device_error(Ctx* ctx, uint32_t err);

// hash_columns (kernels/hash.rs:16-23) of the active rows of `cols` into `o` (one u64 per row)
// on stream s: dictionary columns hash each entry once on the host (kernels/hash.rs:66-77).
void hash_rows(Ctx* ctx, const ml_column* cols, int ncols, int64_t nrows, const uint32_t* dsel, int64_t nsel,
               cudaStream_t s, Staging& st, DevBuf& o) {
    std::vector<std::unique_ptr<DevColumn>> staged;
    PipeArgs P{};
    P.sel = dsel;
    P.n = dsel ? nsel : nrows;
    P.nsrc = nrows;
    DevBuf err(ctx, 8, nullptr);
    CK(cudaMemsetAsync(err.get(), 0, 4, s));
    P.err = err.get<uint32_t>();
    std::vector<DevBuf> dh;
    std::vector<const uint64_t*> dh_ptr(ncols, nullptr);
    for (int c = 0; c < ncols; c++) {
        staged.push_back(stage_column(ctx, cols[c], nrows, s, st, nullptr));
        const DevColumn& col = *staged.back();
        DCol& d = P.cols[c];
        d.dt = col.dtype;
        d.kind = col.kind;
        d.data = col.dptr();
        d.off = col.optr();
        d.valid = col.vptr();
        d.n = col.n;
        if (col.kind == CK_DICT) {
            d.dict_len = (uint32_t)col.dict->len();
            std::vector<uint64_t> hv(col.dict->len() + 1);
            for (size_t e = 0; e < col.dict->len(); e++) {
                uint64_t x = 0x243F6A8885A308D3ull ^ ((uint64_t)(col.dict->off[e + 1] - col.dict->off[e]) * 0x9E3779B97F4A7C15ull);
                const uint8_t* bytes = col.dict->bytes.data() + col.dict->off[e];
                size_t nbytes = col.dict->off[e + 1] - col.dict->off[e];
                auto fm = [](uint64_t a, uint64_t m) {
                    unsigned __int128 r = (unsigned __int128)a * m;
                    return (uint64_t)r ^ (uint64_t)(r >> 64);
                };
                size_t full = nbytes / 8;
                for (size_t q = 0; q < full; q++) {
                    uint64_t w;
                    memcpy(&w, bytes + q * 8, 8);
                    x = fm(x ^ w, 0x9E3779B97F4A7C15ull);
                }
                if (nbytes % 8) {
                    uint64_t w = 0;
                    memcpy(&w, bytes + full * 8, nbytes % 8);
                    x = fm(x ^ w, 0xBF58476D1CE4E5B9ull);
                }
                hv[e] = x;
            }
            dh.emplace_back(ctx, hv.size() * 8, nullptr);
            CK(cudaMemcpyAsync(dh.back().get(), hv.data(), hv.size() * 8, cudaMemcpyHostToDevice, s));
            dh_ptr[c] = dh.back().get<uint64_t>();
        }
    }
    DevBuf ptrs(ctx, std::max<size_t>(ncols * 8, 8), nullptr);
    if (ncols) CK(cudaMemcpyAsync(ptrs.get(), dh_ptr.data(), ncols * 8, cudaMemcpyHostToDevice, s));
    o = DevBuf(ctx, std::max<size_t>((size_t)P.n * 8, 8), nullptr);
    launch_hash_columns(P, ncols, ptrs.get<const uint64_t*>(), o.get<uint64_t>(), s);
    ctx->count_launch();
    uint32_t e = 0;
    CK(cudaMemcpyAsync(&e, err.get(), 4, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));  // the staged columns and tables go out of scope here
    check_device_error(ctx, e);
}

void check_device_error(Ctx* ctx, uint32_t err) {
    (void)ctx;
    if (err & DE_BAD_INDEX) raise(ML_ERR_INVALID, "a selection vector holds a row id past the batch's rows");
    if (err & DE_TIMEOUT) raise(ML_ERR_TIMEOUT, "a bounded device-side wait ran out");
    if (err & DE_OVERFLOW_LOST) raise(ML_ERR_INTERNAL, "hash-table overflow buffer exhausted");
    if (err) raise(ML_ERR_INTERNAL, "device error word " + std::to_string(err));
}

struct ErrWord {  // a device error word plus a pinned readback slot
    DevBuf d;
    uint32_t* h = nullptr;
    Ctx* ctx;
    explicit ErrWord(Ctx* c) : d(c, 64, nullptr), ctx(c) { h = (uint32_t*)c->pinned_slot(); }
    ~ErrWord() { ctx->release_slot(h); }
};

// The streams a sink's work runs on: its live local sinks' streams and one stream of its
// own (finalize, reset).  Waiting for a sink waits for these only, never for the device work
// of other sinks (other queries in flight).
class SinkStreams {
   public:
    explicit SinkStreams(Ctx* c) : ctx_(c) {}
    ~SinkStreams() {
        if (own_) {
            cudaStreamSynchronize(own_);
            ctx_->free_stream(own_);
        }
    }
    cudaStream_t own() {
        std::lock_guard<std::mutex> g(mu_);
        if (!own_) own_ = ctx_->new_stream();
        return own_;
    }
    void add(cudaStream_t s) {
        std::lock_guard<std::mutex> g(mu_);
        live_.push_back(s);
    }
    void remove(cudaStream_t s) {
        std::lock_guard<std::mutex> g(mu_);
        live_.erase(std::find(live_.begin(), live_.end(), s));
    }
    void sync() {
        std::vector<cudaStream_t> ss;
        {
            std::lock_guard<std::mutex> g(mu_);
            ss = live_;
            if (own_) ss.push_back(own_);
        }
        for (auto s : ss) CK(cudaStreamSynchronize(s));
    }

   private:
    Ctx* ctx_;
    std::mutex mu_;
    std::vector<cudaStream_t> live_;
    cudaStream_t own_ = nullptr;
};

// The prologue's output for one batch, materialized as owned device columns.
// With `borrow`, a pipeline that keeps every row and only passes source columns through returns
// views of the launch's source columns (no copy); the caller must be done with them before L goes.
std::unique_ptr<ml_batch> materialize(Ctx* ctx, Pipeline& pipe, const std::vector<Prog>& out_progs, Pipeline::Launch& L,
                                      cudaStream_t st, Reservation* res, ErrWord& ew, bool borrow = false) {
    DevBuf idx;
    const uint32_t* rows = L.P.sel;
    int64_t k = L.P.n;
    if (pipe.nstages > 0) {
        CK(cudaMemsetAsync(ew.d.get(), 0, 4, st));
        L.P.err = ew.d.get<uint32_t>();
        k = run_select(ctx, pipe, L.P, idx, st);
        rows = idx.get<uint32_t>();
    }
    auto b = std::make_unique<ml_batch>();
    b->ctx = ctx;
    b->nrows = k;
    bool plain = borrow && rows == nullptr;  // every row, every output a source column: no copy
    for (const ColRef& r : pipe.out) plain = plain && r.kind == 0;
    if (plain) {
        for (const ColRef& r : pipe.out) {
            const DevColumn& src = *L.src[r.index];
            auto d = std::make_unique<DevColumn>();
            d->dtype = src.dtype;
            d->kind = src.kind;
            d->n = src.n;
            d->dict = src.dict;
            d->data_p = src.dptr();
            d->off_p = src.optr();
            d->valid_p = src.vptr();
            b->cols.push_back(std::move(d));
        }
        return b;
    }
    PipeArgs Q = L.P;
    Q.sel = rows;
    Q.n = k;
    Q.nstages = 0;
    for (size_t c = 0; c < pipe.out.size(); c++) {
        const ColRef& r = pipe.out[c];
        if (r.kind == 0) {
            b->cols.push_back(gather_column(ctx, *L.src[r.index], rows, k, st, res));
        } else if (r.kind == 2) {
            if (r.dtype == ML_TYPE_UTF8) raise(ML_ERR_UNSUPPORTED, "computed string column on the GPU");
            b->cols.push_back(project_column(ctx, Q, out_progs[c], r.dtype, st, res));
        } else {
            raise(ML_ERR_UNSUPPORTED, "a probe in front of this sink");
        }
    }
    CK(cudaStreamSynchronize(st));
    return b;
}

std::vector<Prog> compile_outputs(Pipeline& pipe) {
    std::vector<Prog> progs(pipe.out.size());
    for (size_t c = 0; c < pipe.out.size(); c++) {
        const ColRef& r = pipe.out[c];
        if (r.kind == 2 && r.dtype != ML_TYPE_UTF8) progs[c] = pipe.C.compile_value(*r.expr, *r.env, r.dtype);
    }
    return progs;
}

std::vector<ml_column> device_views(const ml_batch& b) {
    std::vector<ml_column> v;
    for (auto& c : b.cols) {
        ml_column m{};
        m.dtype = c->dtype;
        m.encoding = c->kind == CK_DICT ? ML_ENC_DICT : ML_ENC_PLAIN;
        m.location = ML_LOC_DEVICE;
        m.len = c->n;
        m.data = c->dptr();
        m.offsets = c->optr();
        m.validity = c->vptr();
        if (c->dict) {
            m.dict_len = (int64_t)c->dict->len();
            m.dict_offsets = c->dict->off.data();
            m.dict_data = c->dict->bytes.data();
        }
        v.push_back(m);
    }
    return v;
}

// Concatenate batches column by column into one owned batch.
std::unique_ptr<ml_batch> concat_batches(Ctx* ctx, std::vector<std::unique_ptr<ml_batch>>& parts, const std::vector<int>& types,
                                         cudaStream_t st, Reservation* res) {
    auto out = std::make_unique<ml_batch>();
    out->ctx = ctx;
    int64_t n = 0;
    for (auto& p : parts) n += p->nrows;
    out->nrows = n;
    if (parts.size() == 1) {
        out->cols = std::move(parts[0]->cols);
        return out;
    }
    for (size_t c = 0; c < types.size(); c++) {
        auto d = std::make_unique<DevColumn>();
        d->dtype = types[c];
        d->n = n;
        bool utf8 = types[c] == ML_TYPE_UTF8;
        d->kind = utf8 ? CK_UTF8 : CK_FIXED;
        bool any_valid = false;
        for (auto& p : parts) any_valid |= p->cols[c]->vptr() != nullptr;
        if (utf8) {
            std::vector<uint32_t> sizes;
            uint64_t total = 0;
            for (auto& p : parts) {
                uint32_t first = 0, last = 0;
                const DevColumn& s = *p->cols[c];
                if (s.n) {
                    CK(cudaMemcpy(&first, s.optr(), 4, cudaMemcpyDeviceToHost));
                    CK(cudaMemcpy(&last, s.optr() + s.n, 4, cudaMemcpyDeviceToHost));
                }
                sizes.push_back(last - first);
                total += last - first;
            }
            if (total > 0xFFFFFFFFull) raise(ML_ERR_UNSUPPORTED, "string column larger than 4 GiB");
            d->offsets = DevBuf(ctx, (size_t)(n + 1) * 4, res);
            d->data = DevBuf(ctx, std::max<size_t>(total, 1), res);
            uint64_t row = 0, byte = 0;
            for (size_t i = 0; i < parts.size(); i++) {
                const DevColumn& s = *parts[i]->cols[c];
                launch_offsets_rebase(s.optr(), s.n, (uint32_t)byte, d->offsets.get<uint32_t>() + row, st);
                uint32_t first = 0;
                if (s.n) CK(cudaMemcpy(&first, s.optr(), 4, cudaMemcpyDeviceToHost));
                if (sizes[i])
                    CK(cudaMemcpyAsync(d->data.get<uint8_t>() + byte, (const uint8_t*)s.dptr() + first, sizes[i],
                                       cudaMemcpyDeviceToDevice, st));
                row += s.n;
                byte += sizes[i];
                ctx->count_launch();
            }
        } else {
            int w = width_of(types[c]);
            d->data = DevBuf(ctx, std::max<size_t>((size_t)n * w, 1), res);
            uint64_t row = 0;
            for (auto& p : parts) {
                const DevColumn& s = *p->cols[c];
                if (s.n) CK(cudaMemcpyAsync(d->data.get<uint8_t>() + row * w, s.dptr(), (size_t)s.n * w, cudaMemcpyDeviceToDevice, st));
                row += s.n;
            }
        }
        if (any_valid) {
            size_t vb = std::max<size_t>((size_t)(n + 63) / 64 * 8, 8);
            d->validity = DevBuf(ctx, vb, res);
            CK(cudaMemsetAsync(d->validity.get(), 0, vb, st));
            uint64_t row = 0;
            for (auto& p : parts) {
                const DevColumn& s = *p->cols[c];
                launch_copy_bits(s.vptr(), s.n, d->validity.get<uint64_t>(), (int64_t)row, st);
                ctx->count_launch();
                row += s.n;
            }
        }
        out->cols.push_back(std::move(d));
    }
    CK(cudaStreamSynchronize(st));
    return out;
}

// A finished batch in host memory (fixed-width or plain UTF8 columns): the spilled aggregation
// parks each partition's output here, so HBM holds the final output only once.
struct HostCol {
    int dtype = 0;
    bool utf8 = false, has_valid = false;
    std::vector<uint8_t> data;
    std::vector<uint32_t> offs;   // UTF8: n + 1, rebased to 0
    std::vector<uint64_t> valid;  // bit r of word r / 64
};
struct HostBatch {
    int64_t n = 0;
    std::vector<HostCol> cols;
};

HostBatch batch_to_host(const ml_batch& b, cudaStream_t st) {
    HostBatch h;
    h.n = b.nrows;
    for (const auto& cp : b.cols) {
        const DevColumn& c = *cp;
        HostCol o;
        o.dtype = c.dtype;
        o.utf8 = c.kind == CK_UTF8;
        if (c.kind == CK_DICT) raise(ML_ERR_UNSUPPORTED, "dictionary column in a spilled output");
        if (o.utf8) {
            o.offs.resize(c.n + 1);
            CK(cudaMemcpyAsync(o.offs.data(), c.optr(), (size_t)(c.n + 1) * 4, cudaMemcpyDeviceToHost, st));
            CK(cudaStreamSynchronize(st));
            const uint32_t first = o.offs[0];
            o.data.resize(o.offs[c.n] - first);
            if (!o.data.empty())
                CK(cudaMemcpyAsync(o.data.data(), (const uint8_t*)c.dptr() + first, o.data.size(), cudaMemcpyDeviceToHost, st));
            for (auto& x : o.offs) x -= first;
        } else {
            o.data.resize((size_t)c.n * width_of(c.dtype));
            if (!o.data.empty()) CK(cudaMemcpyAsync(o.data.data(), c.dptr(), o.data.size(), cudaMemcpyDeviceToHost, st));
        }
        if (c.vptr()) {
            o.has_valid = true;
            o.valid.resize((size_t)(c.n + 63) / 64);
            if (!o.valid.empty()) CK(cudaMemcpyAsync(o.valid.data(), c.vptr(), o.valid.size() * 8, cudaMemcpyDeviceToHost, st));
        }
        h.cols.push_back(std::move(o));
    }
    CK(cudaStreamSynchronize(st));
    return h;
}

// Concatenate host batches into one device batch, one column at a time.
std::unique_ptr<ml_batch> host_batches_to_device(Ctx* ctx, const std::vector<HostBatch>& parts, const std::vector<int>& types,
                                                 Reservation* res) {
    auto out = std::make_unique<ml_batch>();
    out->ctx = ctx;
    int64_t n = 0;
    for (const auto& p : parts) n += p.n;
    out->nrows = n;
    for (size_t c = 0; c < types.size(); c++) {
        auto d = std::make_unique<DevColumn>();
        d->dtype = types[c];
        d->n = n;
        const bool utf8 = types[c] == ML_TYPE_UTF8;
        d->kind = utf8 ? CK_UTF8 : CK_FIXED;
        std::vector<uint8_t> data;
        std::vector<uint32_t> offs(utf8 ? 1 : 0, 0);
        bool any_valid = false;
        for (const auto& p : parts) {
            const HostCol& s = p.cols[c];
            any_valid |= s.has_valid;
            if (utf8) {
                const uint64_t base = data.size();
                if (base + s.data.size() > 0xFFFFFFFFull) raise(ML_ERR_UNSUPPORTED, "string column larger than 4 GiB");
                for (int64_t r = 1; r <= p.n; r++) offs.push_back((uint32_t)(base + s.offs[r]));
            }
            data.insert(data.end(), s.data.begin(), s.data.end());
        }
        d->data = DevBuf(ctx, std::max<size_t>(data.size(), 8), res);
        h2d_now(d->data.get(), data.data(), data.size());
        if (utf8) {
            d->offsets = DevBuf(ctx, offs.size() * 4, res);
            h2d_now(d->offsets.get(), offs.data(), offs.size() * 4);
        }
        if (any_valid) {
            std::vector<uint64_t> bits((size_t)(n + 63) / 64 + 1, 0);
            int64_t row = 0;
            for (const auto& p : parts) {
                const HostCol& s = p.cols[c];
                for (int64_t r = 0; r < p.n; r++, row++)
                    if (!s.has_valid || ((s.valid[r / 64] >> (r % 64)) & 1)) bits[row / 64] |= 1ull << (row % 64);
            }
            d->validity = DevBuf(ctx, bits.size() * 8, res);
            h2d_now(d->validity.get(), bits.data(), bits.size() * 8);
        }
        out->cols.push_back(std::move(d));
    }
    return out;
}

// ---- top-N over a device batch (sort.rs:85-132) ------------------------------------------
struct SortKeySpec {
    ExprNode expr;
    int type;
    bool asc, nulls_first;
};

std::unique_ptr<ml_batch> sort_batch(Ctx* ctx, ml_batch& b, const std::vector<SortKeySpec>& keys, int64_t limit,
                                     cudaStream_t st, Reservation* res);

std::unique_ptr<ml_batch> topn_batch(Ctx* ctx, ml_batch& b, const std::vector<SortKeySpec>& keys, int64_t limit,
                                     cudaStream_t st, Reservation* res) {
    for (auto& key : keys)  // dictionary sort keys take the radix sort (ranks of the entries)
        if (key.expr.kind == ML_EXPR_COLUMN && key.expr.index >= 0 && (size_t)key.expr.index < b.cols.size() &&
            b.cols[key.expr.index]->kind == CK_DICT)
            return sort_batch(ctx, b, keys, limit, st, res);
    int64_t n = b.nrows;
    int64_t k = std::min<int64_t>(limit, n);
    auto out = std::make_unique<ml_batch>();
    out->ctx = ctx;
    out->nrows = k;
    std::vector<int> types;
    for (auto& c : b.cols) types.push_back(c->dtype);
    if (k <= 0) {
        for (auto& c : b.cols) {
            auto d = std::make_unique<DevColumn>();
            d->dtype = c->dtype;
            d->kind = c->dtype == ML_TYPE_UTF8 ? CK_UTF8 : CK_FIXED;
            d->n = 0;
            if (d->kind == CK_UTF8) {
                d->offsets = DevBuf(ctx, 4, res);
                CK(cudaMemsetAsync(d->offsets.get(), 0, 4, st));
                d->data = DevBuf(ctx, 1, res);
            } else {
                d->data = DevBuf(ctx, 8, res);
            }
            out->cols.push_back(std::move(d));
        }
        out->nrows = 0;
        return out;
    }
    // key columns: plain column references read the batch; other expressions are evaluated
    Pipeline kp(ctx);
    kp.build(nullptr, 0, types.data(), (int)types.size());
    std::vector<std::unique_ptr<DevColumn>> temps;
    SortDev S{};
    S.nkeys = (int)keys.size();
    std::vector<Prog> progs;
    std::vector<int> direct;
    for (auto& key : keys) {
        if (key.expr.kind == ML_EXPR_COLUMN && key.expr.index >= 0 && (size_t)key.expr.index < types.size() &&
            types[key.expr.index] == key.type) {
            direct.push_back((int)key.expr.index);
            progs.push_back(Prog{});
        } else {
            direct.push_back(-1);
            progs.push_back(kp.C.compile_value(key.expr, kp.out, key.type));
        }
    }
    kp.upload();
    Staging stg(ctx);
    Pipeline::Launch L;
    auto views = device_views(b);
    kp.prepare(L, views.data(), (int)views.size(), n, nullptr, 0, st, stg, nullptr);
    for (size_t i = 0; i < keys.size(); i++) {
        const DevColumn* c;
        if (direct[i] >= 0) {
            c = b.cols[direct[i]].get();
        } else {
            temps.push_back(project_column(ctx, L.P, progs[i], keys[i].type, st, nullptr));
            c = temps.back().get();
        }
        if (c->kind == CK_DICT) raise(ML_ERR_UNSUPPORTED, "sorting a dictionary column on the GPU");
        DCol& d = S.cols[i];
        d.dt = c->dtype;
        d.kind = c->kind;
        d.data = c->dptr();
        d.off = c->optr();
        d.valid = c->vptr();
        d.n = c->n;
        S.asc[i] = keys[i].asc;
        S.nulls_first[i] = keys[i].nulls_first;
    }
    DevBuf a, bb;
    const uint32_t* in = nullptr;
    if (k <= kTopNWarpMax) {  // small limits: one sorted list per warp, one launch
        const int nb = topn_warp_blocks(n);
        const size_t rows_b = ((size_t)nb * k * 4 + 15) & ~(size_t)15, cand_b = (size_t)nb * k * topn_entry_bytes();
        a = DevBuf(ctx, rows_b + (nb > 1 ? cand_b + 16 + (size_t)k * 4 : 0), nullptr);
        void* cand = nullptr;
        unsigned int* done = nullptr;
        uint32_t* final_out = nullptr;
        if (nb > 1) {
            cand = a.get<uint8_t>() + rows_b;
            done = (unsigned int*)(a.get<uint8_t>() + rows_b + cand_b);
            final_out = (uint32_t*)(done + 4);
            CK(cudaMemsetAsync(done, 0, 16, st));  // finished-CTA counter and the shared top-k threshold
        }
        KernelTimer kt(ctx, st, "topn");
        const int launched = launch_topn_warp(S, n, (int)k, nb, a.get<uint32_t>(), cand, done, final_out, st);
        kt.stop();
        ctx->count_launch(launched);
        in = nb > 1 ? final_out : a.get<uint32_t>();
    } else {  // rounds of chunk sorts until one chunk remains
        int64_t m = n;
        for (;;) {
            int64_t nb = (m + kTopNChunk - 1) / kTopNChunk;
            DevBuf& dst = (in == a.get<uint32_t>() && in) ? bb : a;
            dst = DevBuf(ctx, (size_t)nb * k * 4, nullptr);
            {
                KernelTimer kt(ctx, st, "topn");
                launch_topn_chunk(S, in, m, (int)k, dst.get<uint32_t>(), st);
                kt.stop();
            }
            ctx->count_launch();
            in = dst.get<uint32_t>();
            if (nb == 1) break;
            m = nb * k;
        }
    }
    for (auto& c : b.cols) out->cols.push_back(gather_column(ctx, *c, in, k, st, res));
    CK(cudaStreamSynchronize(st));
    return out;
}

// ---- full ORDER BY (sort.rs:85-132 without a limit): stable LSD radix sort of row ids --------
// The key words of each sort key, least significant first: value words (a fixed-width value; a
// plain string's length, then its 8-byte chunks from the last; a dictionary entry's rank), then
// the NULL flag.  Keys are taken last first, so the first key decides first.
std::vector<SortWord> sort_words(Ctx* ctx, const std::vector<const DevColumn*>& cols, const std::vector<SortKeySpec>& keys,
                                 std::vector<DevBuf>& hold, cudaStream_t st) {
    std::vector<SortWord> words;
    for (int k = (int)keys.size() - 1; k >= 0; k--) {
        const DevColumn& c = *cols[k];
        SortWord w{};
        w.col.dt = c.dtype;
        w.col.kind = c.kind;
        w.col.data = c.dptr();
        w.col.off = c.optr();
        w.col.valid = c.vptr();
        w.col.n = c.n;
        w.desc = keys[k].asc ? 0 : 1;
        w.nulls_first = keys[k].nulls_first ? 1 : 0;
        if (c.kind == CK_DICT) {  // rank of each entry among the dictionary's strings (byte order)
            const HostDict& hd = *c.dict;
            std::vector<uint32_t> order(hd.len());
            for (size_t e = 0; e < order.size(); e++) order[e] = (uint32_t)e;
            std::stable_sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) { return hd.get(a) < hd.get(b); });
            std::vector<uint32_t> rank(hd.len() + 1, 0);
            uint32_t rk = 0;
            for (size_t i = 0; i < order.size(); i++) {
                if (i && hd.get(order[i]) != hd.get(order[i - 1])) rk++;
                rank[order[i]] = rk;
            }
            rank[hd.len()] = rk + 1;  // the clamp entry of an out-of-range code
            hold.emplace_back(ctx, rank.size() * 4, nullptr);
            h2d_now(hold.back().get(), rank.data(), rank.size() * 4);
            w.col.dict_len = (uint32_t)hd.len();
            w.what = SW_RANK;
            w.rank = hold.back().get<uint32_t>();
            words.push_back(w);
        } else if (c.kind == CK_UTF8) {
            DevBuf mx(ctx, 8, nullptr);
            CK(cudaMemsetAsync(mx.get(), 0, 8, st));
            launch_max_strlen(c.optr(), c.n, mx.get<unsigned int>(), st);
            ctx->count_launch();
            unsigned int maxlen = 0;
            CK(cudaMemcpyAsync(&maxlen, mx.get(), 4, cudaMemcpyDeviceToHost, st));
            CK(cudaStreamSynchronize(st));
            w.what = SW_LENGTH;
            words.push_back(w);
            for (int ch = (int)((maxlen + 7) / 8) - 1; ch >= 0; ch--) {
                w.what = SW_CHUNK;
                w.chunk = ch;
                words.push_back(w);
            }
        } else {
            w.what = SW_VALUE;
            words.push_back(w);
        }
        if (c.vptr()) {  // NULLs present: the flag ranks them first or last, before the value
            w.what = SW_NULL_FLAG;
            w.desc = 0;
            words.push_back(w);
        }
    }
    return words;
}

// The sorted order of n rows (perm[i] = row at position i) by `words`; nullptr-free result.
DevBuf radix_sort_rows(Ctx* ctx, const std::vector<SortWord>& words, int64_t n, cudaStream_t st, Reservation* res) {
    DevBuf ka(ctx, std::max<size_t>((size_t)n * 8, 8), res), kb(ctx, std::max<size_t>((size_t)n * 8, 8), res);
    DevBuf pa(ctx, std::max<size_t>((size_t)n * 4, 4), res), pb(ctx, std::max<size_t>((size_t)n * 4, 4), res);
    DevBuf hist(ctx, 8 * 256 * 8, nullptr);
    const int nb = radix_blocks(n);
    DevBuf counts(ctx, std::max<size_t>((size_t)nb * 256 * 4, 4), nullptr);
    bool have_perm = false;  // pa holds the current order (else: rows in input order)
    std::vector<unsigned long long> h(8 * 256);
    for (const SortWord& w : words) {
        launch_sort_words(w, have_perm ? pa.get<uint32_t>() : nullptr, n, ka.get<uint64_t>(), st);
        CK(cudaMemsetAsync(hist.get(), 0, 8 * 256 * 8, st));
        launch_radix_hist8(ka.get<uint64_t>(), n, hist.get<unsigned long long>(), st);
        ctx->count_launch(2);
        CK(cudaMemcpyAsync(h.data(), hist.get(), 8 * 256 * 8, cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        for (int b = 0; b < 8; b++) {
            bool trivial = false;  // one digit for every row: the pass would not move anything
            for (int d = 0; d < 256 && !trivial; d++) trivial = h[b * 256 + d] == (unsigned long long)n;
            if (trivial) continue;
            launch_radix_count(ka.get<uint64_t>(), n, 8 * b, counts.get<uint32_t>(), st);
            DevBuf offs;
            scan_counts(ctx, counts.get<uint32_t>(), (int64_t)nb * 256, offs, st);
            launch_radix_scatter(ka.get<uint64_t>(), have_perm ? pa.get<uint32_t>() : nullptr, n, 8 * b,
                                 offs.get<uint64_t>(), kb.get<uint64_t>(), pb.get<uint32_t>(), st);
            ctx->count_launch(2);
            std::swap(ka, kb);
            std::swap(pa, pb);
            have_perm = true;
        }
    }
    if (!have_perm) launch_iota_u32(pa.get<uint32_t>(), n, st);
    return pa;
}

// ORDER BY keys [LIMIT limit] over a device batch: the first min(limit, n) rows in sorted order
// (a stable sort: equal keys keep their input order).  limit < 0: every row.
std::unique_ptr<ml_batch> sort_batch(Ctx* ctx, ml_batch& b, const std::vector<SortKeySpec>& keys, int64_t limit,
                                     cudaStream_t st, Reservation* res) {
    const int64_t n = b.nrows;
    const int64_t k = limit < 0 ? n : std::min<int64_t>(limit, n);
    std::vector<int> types;
    for (auto& c : b.cols) types.push_back(c->dtype);
    Pipeline kp(ctx);
    kp.build(nullptr, 0, types.data(), (int)types.size());
    // key columns: plain column references read the batch; other expressions are evaluated
    std::vector<Prog> progs(keys.size());
    std::vector<int> direct(keys.size(), -1);
    bool computed = false;
    for (size_t i = 0; i < keys.size(); i++) {
        const auto& key = keys[i];
        if (key.expr.kind == ML_EXPR_COLUMN && key.expr.index >= 0 && (size_t)key.expr.index < types.size() &&
            types[key.expr.index] == key.type) {
            direct[i] = (int)key.expr.index;
            continue;
        }
        if (key.type == ML_TYPE_UTF8) raise(ML_ERR_UNSUPPORTED, "sorting by a computed string expression on the GPU");
        progs[i] = kp.C.compile_value(key.expr, kp.out, key.type);
        computed = true;
    }
    std::vector<std::unique_ptr<DevColumn>> temps;
    std::vector<const DevColumn*> kcols;
    Staging stg(ctx);
    Pipeline::Launch L;
    if (computed) {
        kp.upload();
        auto views = device_views(b);
        kp.prepare(L, views.data(), (int)views.size(), n, nullptr, 0, st, stg, nullptr);
    }
    for (size_t i = 0; i < keys.size(); i++) {
        if (direct[i] >= 0) {
            kcols.push_back(b.cols[direct[i]].get());
        } else {
            temps.push_back(project_column(ctx, L.P, progs[i], keys[i].type, st, nullptr));
            kcols.push_back(temps.back().get());
        }
    }
    std::vector<DevBuf> hold;
    auto words = sort_words(ctx, kcols, keys, hold, st);
    DevBuf perm = radix_sort_rows(ctx, words, n, st, nullptr);
    auto out = std::make_unique<ml_batch>();
    out->ctx = ctx;
    out->nrows = k;
    for (auto& c : b.cols) out->cols.push_back(gather_column(ctx, *c, perm.get<uint32_t>(), k, st, res));
    CK(cudaStreamSynchronize(st));
    return out;
}

}  // namespace

// =====================================================================================================
// context
// =====================================================================================================
extern "C" {

const char* ml_gpu_last_error(void) { return last_error(); }

int ml_gpu_last_budget_error(char* op, size_t op_cap, uint64_t* requested, uint64_t* used, uint64_t* limit) {
    const BudgetInfo& b = last_budget();
    if (op && op_cap) {
        strncpy(op, b.op.c_str(), op_cap - 1);
        op[op_cap - 1] = 0;
    }
    if (requested) *requested = b.requested;
    if (used) *used = b.used;
    if (limit) *limit = b.limit;
    return ML_OK;
}

int ml_gpu_ctx_create(int device, uint64_t hbm_budget_bytes, uint32_t flags, ml_ctx** out) {
    API_BEGIN
    REQUIRE(out, "null output");
    REQUIRE((flags & ~(uint32_t)(ML_CTX_PROFILE | ML_CTX_INTERPRET | ML_CTX_SPILL)) == 0, "unknown context flags");
    *out = new ml_ctx(device, hbm_budget_bytes, flags);
    API_END
}

int ml_gpu_ctx_destroy(ml_ctx* ctx) {
    API_BEGIN
    delete ctx;
    API_END
}

int ml_gpu_pool_stats(ml_ctx* ctx, uint64_t* used, uint64_t* peak, uint64_t* limit) {
    API_BEGIN
    REQUIRE(ctx, "null context");
    if (used) *used = ctx->pool.used.load();
    if (peak) *peak = ctx->pool.peak.load();
    if (limit) *limit = ctx->pool.limit;
    API_END
}

int ml_gpu_ctx_synchronize(ml_ctx* ctx) {
    API_BEGIN
    REQUIRE(ctx, "null context");
    ctx->sync_all();
    API_END
}

int ml_gpu_kernel_launches(ml_ctx* ctx, uint64_t* count) {
    API_BEGIN
    REQUIRE(ctx && count, "null argument");
    *count = ctx->launches.load();
    API_END
}

int ml_gpu_profile_read(ml_ctx* ctx, const char* kernel, uint64_t* launches, double* total_ms, int32_t reset) {
    API_BEGIN
    REQUIRE(ctx && kernel, "null argument");
    ctx->read_profile(kernel, launches, total_ms, reset != 0);
    API_END
}

// =====================================================================================================
// batches
// =====================================================================================================
int ml_gpu_batch_upload(ml_ctx* ctx, const ml_column* cols, int32_t ncols, int64_t nrows, ml_batch** out) {
    API_BEGIN
    REQUIRE(ctx && out && (cols || ncols == 0) && ncols >= 0 && nrows >= 0, "bad arguments");
    ctx->set_current();
    OpStream op_stream(ctx);
    const cudaStream_t s = op_stream.s;
    auto b = std::make_unique<ml_batch>();
    b->ctx = ctx;
    b->nrows = nrows;
    b->res = std::make_unique<Reservation>(ctx, "Batch");
    Staging st(ctx);
    for (int c = 0; c < ncols; c++) {
        auto col = stage_column(ctx, cols[c], nrows, s, st, b->res.get());
        if (cols[c].location == ML_LOC_DEVICE) col = copy_column(ctx, *col, s, b->res.get());
        b->cols.push_back(std::move(col));
    }
    CK(cudaStreamSynchronize(s));
    *out = b.release();
    API_END
}

int ml_gpu_batch_num_rows(const ml_batch* b, int64_t* nrows) {
    API_BEGIN
    REQUIRE(b && nrows, "null argument");
    *nrows = b->nrows;
    API_END
}

int ml_gpu_batch_num_columns(const ml_batch* b, int32_t* ncols) {
    API_BEGIN
    REQUIRE(b && ncols, "null argument");
    *ncols = (int32_t)b->cols.size();
    API_END
}

int ml_gpu_batch_columns(const ml_batch* b, ml_column* out, int32_t ncols) {
    API_BEGIN
    REQUIRE(b && out, "null argument");
    REQUIRE(ncols == (int32_t)b->cols.size(), "column count mismatch");
    auto v = device_views(*b);
    for (int i = 0; i < ncols; i++) out[i] = v[i];
    API_END
}

int ml_gpu_batch_column_info(const ml_batch* b, int32_t col, int32_t* dtype, int64_t* str_bytes, int32_t* has_validity) {
    API_BEGIN
    REQUIRE(b, "null batch");
    REQUIRE(col >= 0 && col < (int32_t)b->cols.size(), "column out of range");
    b->ctx->set_current();
    const DevColumn& c = *b->cols[col];
    if (dtype) *dtype = c.dtype;
    if (has_validity) *has_validity = c.vptr() != nullptr;
    if (str_bytes) {
        if (c.kind == CK_UTF8) *str_bytes = c.str_bytes_host();
        else if (c.kind == CK_DICT) {
            std::vector<uint32_t> codes(c.n);
            if (c.n) CK(cudaMemcpy(codes.data(), c.dptr(), c.n * 4, cudaMemcpyDeviceToHost));
            int64_t s = 0;
            for (uint32_t k : codes) s += c.dict->off[k + 1] - c.dict->off[k];
            *str_bytes = s;
        } else *str_bytes = 0;
    }
    API_END
}

int ml_gpu_batch_fetch(const ml_batch* b, int32_t col, void* values, uint32_t* offsets, uint64_t* validity) {
    API_BEGIN
    HostTimer host_timer_(b ? b->ctx : nullptr, "host:batch_fetch");
    REQUIRE(b, "null batch");
    REQUIRE(col >= 0 && col < (int32_t)b->cols.size(), "column out of range");
    b->ctx->set_current();
    const DevColumn& c = *b->cols[col];
    int64_t n = c.n;
    if (c.kind == CK_UTF8) {
        REQUIRE(offsets, "UTF8 fetch needs an offsets buffer");
        std::vector<uint32_t> off(n + 1);
        CK(cudaMemcpy(off.data(), c.optr(), (n + 1) * 4, cudaMemcpyDeviceToHost));
        uint32_t first = off[0];
        for (auto& o : off) o -= first;
        memcpy(offsets, off.data(), (n + 1) * 4);
        if (off[n]) {
            REQUIRE(values, "null values buffer");
            CK(cudaMemcpy(values, (const uint8_t*)c.dptr() + first, off[n], cudaMemcpyDeviceToHost));
        }
    } else if (c.kind == CK_DICT) {
        REQUIRE(offsets, "UTF8 fetch needs an offsets buffer");
        std::vector<uint32_t> codes(n);
        if (n) CK(cudaMemcpy(codes.data(), c.dptr(), n * 4, cudaMemcpyDeviceToHost));
        uint32_t pos = 0;
        for (int64_t i = 0; i < n; i++) {
            offsets[i] = pos;
            uint32_t a = c.dict->off[codes[i]], e = c.dict->off[codes[i] + 1];
            if (e > a) memcpy((uint8_t*)values + pos, c.dict->bytes.data() + a, e - a);
            pos += e - a;
        }
        offsets[n] = pos;
    } else if (n) {
        REQUIRE(values, "null values buffer");
        CK(cudaMemcpy(values, c.dptr(), (size_t)n * width_of(c.dtype), cudaMemcpyDeviceToHost));
    }
    if (validity) {
        size_t words = (size_t)(n + 63) / 64;
        if (c.vptr()) {
            if (words) CK(cudaMemcpy(validity, c.vptr(), words * 8, cudaMemcpyDeviceToHost));
            if (n % 64) validity[words - 1] &= (1ull << (n % 64)) - 1;
        } else {
            for (size_t w = 0; w < words; w++) validity[w] = ~0ull;
            if (n % 64) validity[words - 1] = (1ull << (n % 64)) - 1;
        }
    }
    API_END
}

int ml_gpu_batch_destroy(ml_batch* b) {
    API_BEGIN
    if (b) {
        b->ctx->set_current();
        b->cols.clear();
        delete b;
    }
    API_END
}

// =====================================================================================================
// operators
// =====================================================================================================
int ml_gpu_filter(ml_ctx* ctx, const ml_expr* pred, const ml_column* cols, int32_t ncols, int64_t nrows,
                  const uint32_t* sel_in, int64_t nsel_in, int32_t location, uint32_t* sel_out, int64_t* nsel_out) {
    API_BEGIN
    REQUIRE(ctx && pred && sel_out && nsel_out, "null argument");
    ctx->set_current();
    OpStream op_stream(ctx);
    cudaStream_t s = op_stream.s;
    if (location == ML_LOC_HOST) check_sel_bounds(sel_in, nsel_in, nrows);
    std::vector<int32_t> types;
    for (int c = 0; c < ncols; c++) types.push_back(cols[c].dtype);
    Pipeline p(ctx);
    ml_pipe_op op{};
    op.kind = ML_PIPE_FILTER;
    op.nexprs = 1;
    op.exprs = pred;
    p.build(&op, 1, types.data(), ncols);
    p.upload();
    Staging st(ctx);
    // the call's device temporaries count against the query's HBM budget (ResourcesExhausted
    // when it is spent); ml_gpu_filter_static allocates none
    Reservation res(ctx, "Filter");
    DevBuf sel_hold;
    const uint32_t* dsel = device_sel(ctx, sel_in, nsel_in, sel_hold, s, &res);
    Pipeline::Launch L;
    p.prepare(L, cols, ncols, nrows, dsel, nsel_in, s, st, nullptr);
    ErrWord ew(ctx);
    CK(cudaMemsetAsync(ew.d.get(), 0, 4, s));
    L.P.err = ew.d.get<uint32_t>();
    DevBuf out;
    int64_t k = run_select(ctx, p, L.P, out, s, &res);
    CK(cudaMemcpyAsync(ew.h, ew.d.get(), 4, cudaMemcpyDeviceToHost, s));
    if (k) CK(cudaMemcpyAsync(sel_out, out.get(), (size_t)k * 4,
                              location == ML_LOC_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    check_device_error(ctx, *ew.h);
    *nsel_out = k;
    API_END
}

// ml_gpu_filter with every temporary in the device's static scratch array (no allocation).
namespace {
constexpr int kStaticMaxDevices = 64;
std::mutex g_static_mu[kStaticMaxDevices];  // one call at a time per device: they share the array
uint8_t* g_static_base[kStaticMaxDevices];
}  // namespace

int ml_gpu_filter_static(ml_ctx* ctx, const ml_expr* pred, const ml_column* cols, int32_t ncols, int64_t nrows,
                         const uint32_t* sel_in, int64_t nsel_in, uint32_t* sel_out, int64_t* nsel_out) {
    API_BEGIN
    REQUIRE(ctx && pred && sel_out && nsel_out && (cols || ncols == 0) && ncols >= 0 && nrows >= 0, "bad arguments");
    REQUIRE(ctx->device >= 0 && ctx->device < kStaticMaxDevices, "device index out of range");
    for (int c = 0; c < ncols; c++)
        REQUIRE(cols[c].location == ML_LOC_DEVICE, "ml_gpu_filter_static reads device-resident columns only");
    if (sel_in) REQUIRE(nsel_in >= 0, "bad selection length");  // nsel_in is ignored without a selection
    if (nrows > 0xFFFFFFFFll)
        raise(ML_ERR_INVALID, "ml_gpu_filter_static: a batch of " + std::to_string(nrows) +
                                  " rows; row ids are 32-bit, so a batch holds at most 4294967295 rows");
    const int64_t n = sel_in ? nsel_in : nrows;
    if (n > kStaticFilterMaxRows)
        raise(ML_ERR_INVALID, "ml_gpu_filter_static: " + std::to_string(n) + (sel_in ? " selected rows" : " rows") +
                                  " exceed the static scratch limit of " + std::to_string(kStaticFilterMaxRows) +
                                  " rows per call");
    ctx->set_current();
    // everything that is checked on the host comes before the first copy into the shared array
    std::vector<int32_t> types;
    for (int c = 0; c < ncols; c++) types.push_back(cols[c].dtype);
    Pipeline p(ctx);
    ml_pipe_op op{};
    op.kind = ML_PIPE_FILTER;
    op.nexprs = 1;
    op.exprs = pred;
    p.build(&op, 1, types.data(), ncols);
    const size_t pbytes = p.C.code.size() * sizeof(Instr), abytes = p.C.arena.size();
    if (pbytes > kStaticProgBytes || abytes > kStaticArenaBytes)
        raise(ML_ERR_INVALID, "ml_gpu_filter_static: the predicate compiles to " + std::to_string(pbytes) +
                                  " bytes of program and " + std::to_string(abytes) + " bytes of literals; the limits are " +
                                  std::to_string(kStaticProgBytes) + " and " + std::to_string(kStaticArenaBytes));
    std::lock_guard<std::mutex> dev_lock(g_static_mu[ctx->device]);
    if (!g_static_base[ctx->device]) {  // first call on this device: look the array up (device is current)
        g_static_base[ctx->device] = (uint8_t*)static_filter_scratch();
        REQUIRE(g_static_base[ctx->device], "cudaGetSymbolAddress failed for the static filter scratch");
    }
    uint8_t* base = g_static_base[ctx->device];
    OpStream op_stream(ctx);
    cudaStream_t s = op_stream.s;
    // Declared after the locks, so destroyed before them: whichever way the call ends (an error
    // raised after some copies or kernels were queued included), the stream has drained before
    // another call may touch the array.
    struct Drain {
        cudaStream_t s;
        ~Drain() { cudaStreamSynchronize(s); }
    } drain{s};
    Staging st(ctx);  // unused: device-resident columns are read in place
    Pipeline::Launch L;
    p.prepare(L, cols, ncols, nrows, sel_in, nsel_in, s, st, nullptr, base + kStaticTablesOff, kStaticTablesBytes);
    if (pbytes) CK(cudaMemcpyAsync(base + kStaticProgOff, p.C.code.data(), pbytes, cudaMemcpyHostToDevice, s));
    if (abytes) CK(cudaMemcpyAsync(base + kStaticArenaOff, p.C.arena.data(), abytes, cudaMemcpyHostToDevice, s));
    L.P.prog = (const Instr*)(base + kStaticProgOff);
    L.P.arena = base + kStaticArenaOff;
    uint32_t* err = (uint32_t*)(base + kStaticErrOff);
    CK(cudaMemsetAsync(err, 0, 4, s));
    L.P.err = err;
    uint32_t* bits = (uint32_t*)(base + kStaticBitsOff);
    uint32_t* counts = (uint32_t*)(base + kStaticCountsOff);
    uint64_t* offs = (uint64_t*)(base + kStaticOffsetsOff);
    const int nb = select_blocks(n);
    launch_select_flags(L.P, bits, counts, s);
    launch_scan_u32(counts, offs, nb, (uint64_t*)(base + kStaticScanOff), s);
    launch_select_write(L.P, bits, offs, sel_out, s);
    ctx->count_launch(5);
    uint64_t total = 0;
    uint32_t errw = 0;
    CK(cudaMemcpyAsync(&total, offs + nb, 8, cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(&errw, err, 4, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    check_device_error(ctx, errw);
    *nsel_out = (int64_t)total;
    API_END
}

int ml_gpu_project(ml_ctx* ctx, const ml_expr* expr, const ml_column* cols, int32_t ncols, int64_t nrows, ml_batch** out) {
    API_BEGIN
    REQUIRE(ctx && expr && out, "null argument");
    ctx->set_current();
    OpStream op_stream(ctx);
    cudaStream_t s = op_stream.s;
    std::vector<int32_t> types;
    for (int c = 0; c < ncols; c++) types.push_back(cols[c].dtype);
    Pipeline p(ctx);
    p.build(nullptr, 0, types.data(), ncols);
    ExprNode e = parse_expr(*expr);
    Staging st(ctx);
    auto b = std::make_unique<ml_batch>();
    b->ctx = ctx;
    b->nrows = nrows;
    b->res = std::make_unique<Reservation>(ctx, "Projection");
    auto origin = p.C.column_origin(e, p.out);
    if (origin && types[origin->index] == expr->dtype) {  // pass-through column (an Arc clone in the reference)
        Pipeline::Launch L;
        p.upload();
        p.prepare(L, cols, ncols, nrows, nullptr, 0, s, st, nullptr);
        b->cols.push_back(gather_column(ctx, *L.src[origin->index], nullptr, nrows, s, b->res.get()));
    } else {
        Prog pr = p.C.compile_value(e, p.out, expr->dtype);
        p.upload();
        Pipeline::Launch L;
        p.prepare(L, cols, ncols, nrows, nullptr, 0, s, st, nullptr);
        b->cols.push_back(project_column(ctx, L.P, pr, expr->dtype, s, b->res.get()));
    }
    CK(cudaStreamSynchronize(s));
    *out = b.release();
    API_END
}

int ml_gpu_hash_columns(ml_ctx* ctx, const ml_column* cols, int32_t ncols, int64_t nrows, const uint32_t* sel, int64_t nsel,
                        int32_t location, uint64_t* out) {
    API_BEGIN
    REQUIRE(ctx && out && (cols || ncols == 0), "null argument");
    REQUIRE(ncols <= kMaxCols, "too many columns");
    ctx->set_current();
    OpStream op_stream(ctx);
    cudaStream_t s = op_stream.s;
    if (location == ML_LOC_HOST) check_sel_bounds(sel, nsel, nrows);
    Staging st(ctx);
    DevBuf sel_hold;
    const uint32_t* dsel = device_sel(ctx, sel, nsel, sel_hold, s);
    DevBuf o;
    hash_rows(ctx, cols, ncols, nrows, dsel, nsel, s, st, o);
    const int64_t n = sel ? nsel : nrows;
    if (n) CK(cudaMemcpyAsync(out, o.get(), (size_t)n * 8,
                              location == ML_LOC_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    API_END
}

int ml_gpu_partition(ml_ctx* ctx, const ml_column* cols, int32_t ncols, int64_t nrows, const int32_t* key_cols,
                     int32_t nkeys, int32_t nparts, ml_batch** out, int64_t* counts) {
    API_BEGIN
    REQUIRE(ctx && out && counts && (cols || ncols == 0) && key_cols && nkeys > 0, "null argument");
    REQUIRE(ncols <= kMaxCols && nkeys <= ncols, "too many columns");
    REQUIRE(nparts >= 1 && nparts <= kMaxExchangeParts, "partitions out of range (1..64)");
    REQUIRE(nrows >= 0 && nrows < 0xFFFFFFFFll, "row count out of range");
    std::vector<ml_column> keys;
    for (int k = 0; k < nkeys; k++) {
        REQUIRE(key_cols[k] >= 0 && key_cols[k] < ncols, "key column out of range");
        keys.push_back(cols[key_cols[k]]);
    }
    ctx->set_current();
    OpStream op_stream(ctx);
    cudaStream_t s = op_stream.s;
    Staging st(ctx);
    auto b = std::make_unique<ml_batch>();
    b->ctx = ctx;
    b->nrows = nrows;
    b->res = std::make_unique<Reservation>(ctx, "Exchange");
    std::vector<std::unique_ptr<DevColumn>> src;
    for (int c = 0; c < ncols; c++) src.push_back(stage_column(ctx, cols[c], nrows, s, st, b->res.get()));
    DevBuf h;
    hash_rows(ctx, keys.data(), nkeys, nrows, nullptr, 0, s, st, h);
    const int nb = xpart_blocks(nrows);
    DevBuf bc(ctx, std::max<size_t>((size_t)nb * nparts * 4, 4), nullptr), offs;
    launch_xpart_count(h.get<uint64_t>(), nrows, nparts, bc.get<uint32_t>(), s);
    scan_counts(ctx, bc.get<uint32_t>(), (int64_t)nb * nparts, offs, s);
    DevBuf perm(ctx, std::max<size_t>((size_t)nrows * 4, 4), nullptr);
    launch_xpart_scatter(h.get<uint64_t>(), nrows, nparts, offs.get<uint64_t>(), perm.get<uint32_t>(), s);
    ctx->count_launch(2);
    for (auto& c : src) b->cols.push_back(gather_column(ctx, *c, perm.get<uint32_t>(), nrows, s, b->res.get()));
    // partition p's rows start at offs[p * nb]; offs[nparts * nb] is the total
    std::vector<uint64_t> starts(nparts + 1, 0);
    if (nb) CK(cudaMemcpy2DAsync(starts.data(), 8, offs.get(), (size_t)nb * 8, 8, nparts + 1, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    for (int p = 0; p < nparts; p++) counts[p] = (int64_t)(starts[p + 1] - starts[p]);
    *out = b.release();
    API_END
}

}  // extern "C"

// =====================================================================================================
// JoinBuildSink (join.rs:72-242)
// =====================================================================================================
struct ml_join_build {
    Ctx* ctx;
    std::unique_ptr<Reservation> res;  // declared before everything charged to it
    Pipeline pipe;
    std::vector<Prog> out_progs;
    OwnedExprs keys;
    std::vector<int> out_types;
    std::mutex mu;
    std::vector<std::unique_ptr<ml_batch>> parts;
    std::unique_ptr<ml_join_table> table;
    SinkStreams streams;
    ml_join_build(Ctx* c) : ctx(c), pipe(c), streams(c) {}
};
struct ml_join_build_local {
    ml_join_build* sink;
    cudaStream_t s;
    Staging st;
    std::unique_ptr<ErrWord> ew;
    ml_join_build_local(ml_join_build* k) : sink(k), s(k->ctx->new_stream()), st(k->ctx), ew(new ErrWord(k->ctx)) {
        sink->streams.add(s);
    }
    ~ml_join_build_local() {
        sink->streams.remove(s);
        sink->ctx->free_stream(s);
    }
};

extern "C" {

int ml_gpu_join_build_create(ml_ctx* ctx, const ml_pipe_op* prologue, int32_t nprologue, const int32_t* input_types,
                             int32_t ninput, const ml_expr* key_exprs, int32_t nkeys, ml_join_build** out) {
    API_BEGIN
    HostTimer host_timer_(ctx, "host:join_build_create");
    REQUIRE(ctx && out && key_exprs && nkeys > 0, "bad arguments");
    REQUIRE(nkeys <= kMaxKeys, "too many join keys");
    ctx->set_current();
    auto j = std::make_unique<ml_join_build>(ctx);
    j->pipe.build(prologue, nprologue, input_types, ninput);
    for (auto& r : j->pipe.out) j->out_types.push_back(r.dtype);
    j->out_progs = compile_outputs(j->pipe);
    j->pipe.upload();
    for (int k = 0; k < nkeys; k++) j->keys.add(key_exprs[k]);
    j->keys.finish();
    j->res = std::make_unique<Reservation>(ctx, "HashJoinBuild");
    *out = j.release();
    API_END
}

int ml_gpu_join_build_local_create(ml_join_build* sink, ml_join_build_local** out) {
    API_BEGIN
    REQUIRE(sink && out, "null argument");
    sink->ctx->set_current();
    *out = new ml_join_build_local(sink);
    API_END
}

// BuildLocal::sink: compact the batch and keep it (join.rs:217-222)
int ml_gpu_join_build_sink(ml_join_build_local* local, const ml_column* cols, int32_t ncols, int64_t nrows, const uint32_t* sel,
                           int64_t nsel) {
    API_BEGIN
    HostTimer host_timer_(local ? local->sink->ctx : nullptr, "host:join_build_sink");
    REQUIRE(local, "null local sink");
    ml_join_build* j = local->sink;
    REQUIRE(!j->table, "join build sink already finalized");
    Ctx* ctx = j->ctx;
    ctx->set_current();
    check_sel_bounds(sel, nsel, nrows);
    DevBuf sel_hold;
    const uint32_t* dsel = device_sel(ctx, sel, nsel, sel_hold, local->s);
    Pipeline::Launch L;
    j->pipe.prepare(L, cols, ncols, nrows, dsel, nsel, local->s, local->st, nullptr);
    auto part = materialize(ctx, j->pipe, j->out_progs, L, local->s, j->res.get(), *local->ew);
    CK(cudaMemcpyAsync(local->ew->h, local->ew->d.get(), 4, cudaMemcpyDeviceToHost, local->s));
    CK(cudaStreamSynchronize(local->s));
    check_device_error(ctx, j->pipe.nstages > 0 ? *local->ew->h : 0);
    std::lock_guard<std::mutex> g(j->mu);
    j->parts.push_back(std::move(part));
    API_END
}

int ml_gpu_join_build_combine(ml_join_build_local* local) {
    API_BEGIN
    if (local) {
        local->sink->ctx->set_current();
        CK(cudaStreamSynchronize(local->s));
        delete local;
    }
    API_END
}

// build_table (join.rs:160-203)
int ml_gpu_join_build_finalize(ml_join_build* j, ml_join_table** table) {
    API_BEGIN
    HostTimer host_timer_(j ? j->ctx : nullptr, "host:join_build_finalize");
    REQUIRE(j && table, "null argument");
    Ctx* ctx = j->ctx;
    ctx->set_current();
    if (j->table) {
        *table = j->table.get();
        return ML_OK;
    }
    j->streams.sync();
    cudaStream_t s = j->streams.own();
    auto jt = std::make_unique<ml_join_table>();
    jt->ctx = ctx;
    jt->res = std::make_unique<Reservation>(ctx, "HashJoinBuild(table)");
    std::vector<std::unique_ptr<ml_batch>> parts;
    {
        std::lock_guard<std::mutex> g(j->mu);
        parts = std::move(j->parts);
    }
    if (parts.empty()) {
        auto e = std::make_unique<ml_batch>();
        e->ctx = ctx;
        for (int t : j->out_types) {
            auto d = std::make_unique<DevColumn>();
            d->dtype = t;
            d->kind = t == ML_TYPE_UTF8 ? CK_UTF8 : CK_FIXED;
            if (d->kind == CK_UTF8) {
                d->offsets = DevBuf(ctx, 4, j->res.get());
                CK(cudaMemsetAsync(d->offsets.get(), 0, 4, s));
            }
            d->data = DevBuf(ctx, 8, j->res.get());
            e->cols.push_back(std::move(d));
        }
        parts.push_back(std::move(e));
    }
    auto merged = concat_batches(ctx, parts, j->out_types, s, j->res.get());
    jt->batch.ctx = ctx;
    jt->batch.nrows = merged->nrows;
    jt->batch.cols = std::move(merged->cols);
    int64_t n = jt->batch.nrows;
    REQUIRE(n < 0xFFFFFFFFll, "build side larger than 2^32 rows");
    for (int k = 0; k < (int)j->keys.exprs.size(); k++) jt->key_types.push_back(j->keys.exprs[k].dtype);
    // key programs over the build batch
    Pipeline kp(ctx);
    kp.build(nullptr, 0, j->out_types.data(), (int)j->out_types.size());
    KeyLayout L = kp.key_layout(j->keys.exprs.data(), (int)j->keys.exprs.size(), kp.out, false, nullptr);
    jt->nwords = L.nwords;
    for (auto& k : j->keys.exprs) {  // which build column each key reads (for GROUP BY the join key)
        ExprNode e = parse_expr(k);
        auto o = kp.C.column_origin(e, kp.out);
        jt->key_cols.push_back(o && e.kind == ML_EXPR_COLUMN ? o->index : -1);
    }
    jt->next = DevBuf(ctx, std::max<size_t>((size_t)n * 4, 4), jt->res.get());
    jt->dup = DevBuf(ctx, 8, nullptr);
    CK(cudaMemsetAsync(jt->next.get(), 0xFF, std::max<size_t>((size_t)n * 4, 4), s));
    CK(cudaMemsetAsync(jt->dup.get(), 0, 8, s));
    // A single integer key that is a build column, with a value range of at most 4 entries
    // per build row or at most 2^20 entries (a 4 MB index, which L2 holds), is indexed directly
    // (no hashing, one 4-byte load per probe).
    const DevColumn* kc = nullptr;
    if (n > 0 && jt->key_types.size() == 1 && jt->key_cols[0] >= 0) {
        const DevColumn* c = jt->batch.cols[jt->key_cols[0]].get();
        int t = jt->key_types[0];
        if (c->kind == CK_FIXED && c->dtype == t && (t == ML_TYPE_INT32 || t == ML_TYPE_DATE || t == ML_TYPE_INT64)) kc = c;
    }
    if (kc) {
        DevBuf mm(ctx, 16, nullptr);
        uint64_t init[2] = {~0ull, 0ull}, got[2];
        CK(cudaMemcpyAsync(mm.get(), init, 16, cudaMemcpyHostToDevice, s));
        launch_key_range(kc->dptr(), kc->dtype, kc->vptr(), n, mm.get<unsigned long long>(), s);
        ctx->count_launch();
        CK(cudaMemcpyAsync(got, mm.get(), 16, cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
        const uint64_t limit = std::max<uint64_t>(4 * (uint64_t)n + 1024, 1ull << 20);
        if (got[0] <= got[1] && got[1] - got[0] < std::min<uint64_t>(limit, 0xFFFFFFFFull)) {
            jt->dmin = got[0];
            jt->drange = got[1] - got[0] + 1;
        } else {
            kc = nullptr;  // no valid key, or too sparse: hash table
        }
    }
    if (kc) {
        jt->dense = DevBuf(ctx, jt->drange * 4, jt->res.get());
        CK(cudaMemsetAsync(jt->dense.get(), 0xFF, jt->drange * 4, s));
        KernelTimer kt(ctx, s, "join_insert");
        launch_dense_insert(kc->dptr(), kc->dtype, kc->vptr(), n, jt->dmin, jt->drange, jt->dense.get<uint32_t>(),
                            jt->next.get<uint32_t>(), jt->dup.get<uint32_t>(), nullptr, s);
        kt.stop();
        ctx->count_launch();
    }
    const int64_t nh = kc ? 0 : n;  // rows the hash table takes
    jt->cap = pow2_at_least(std::max<uint64_t>(16, ((uint64_t)nh * 4 + 2) / 3));  // load factor <= 3/4
    size_t slot_bytes = jt->cap * 8 * (L.nwords == 1 ? 2 : 4);
    jt->slots = DevBuf(ctx, slot_bytes, jt->res.get());
    CK(cudaMemsetAsync(jt->slots.get(), 0, slot_bytes, s));
    ErrWord ew(ctx);
    CK(cudaMemsetAsync(ew.d.get(), 0, 4, s));
    if (nh) {  // the key programs run only here (a dense index reads the key column directly)
        kp.upload();
        Staging st(ctx);
        Pipeline::Launch LA;
        auto views = device_views(jt->batch);
        kp.prepare(LA, views.data(), (int)views.size(), nh, nullptr, 0, s, st, nullptr);
        LA.P.err = ew.d.get<uint32_t>();
        void* jit = jit_join_insert_kernel(ctx, kp, LA.P, L);
        KernelTimer kt(ctx, s, "join_insert");
        if (jit) {
            TableView tv = jt->view();
            uint32_t* next = jt->next.get<uint32_t>();
            uint32_t* dup = jt->dup.get<uint32_t>();
            int64_t nn = nh;
            void* args[] = {&LA.P, &L, &tv, &next, &dup, &nn};
            jit_launch(jit, pipeline_grid(nh), kPipelineThreads, 0, s, args);
            ctx->add_profile("jit_launch", 0);
        } else {
            launch_join_insert(LA.P, L, jt->view(), jt->next.get<uint32_t>(), jt->dup.get<uint32_t>(), nh, s);
        }
        kt.stop();
        ctx->count_launch();
    }
    // canonical ids of the build side's strings (GROUP BY on a build-side string column)
    for (auto& c : jt->batch.cols) {
        if (c->kind != CK_UTF8 || n == 0) continue;
        uint64_t cap = pow2_at_least(std::max<uint64_t>(16, (uint64_t)n * 2));
        DevBuf tslots(ctx, cap * 16, nullptr);
        CK(cudaMemsetAsync(tslots.get(), 0, cap * 16, s));
        TableView tv{tslots.get<uint64_t>(), cap - 1, 1, 2};
        c->strid = DevBuf(ctx, (size_t)n * 4, jt->res.get());
        launch_strid(c->optr(), (const uint8_t*)c->dptr(), c->vptr(), n, tv, c->strid.get<uint32_t>(), ew.d.get<uint32_t>(), s);
        ctx->count_launch();
        CK(cudaStreamSynchronize(s));
    }
    uint32_t dup = 0;
    CK(cudaMemcpyAsync(&dup, jt->dup.get(), 4, cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(ew.h, ew.d.get(), 4, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    check_device_error(ctx, *ew.h);
    jt->has_dups = dup != 0;
    j->table = std::move(jt);
    *table = j->table.get();
    API_END
}

int ml_gpu_join_table_stats(const ml_join_table* t, int64_t* build_rows, int64_t* distinct_keys, int64_t* capacity) {
    API_BEGIN
    REQUIRE(t, "null table");
    t->ctx->set_current();
    if (build_rows) *build_rows = t->batch.nrows;
    if (capacity) *capacity = (int64_t)(t->dense ? t->drange : t->cap);
    if (distinct_keys) {
        DevBuf c(t->ctx, 8, nullptr);
        CK(cudaMemsetAsync(c.get(), 0, 8, t->ctx->stream));
        if (t->dense) launch_count_dense(t->dense.get<uint32_t>(), t->drange, c.get<unsigned long long>(), t->ctx->stream);
        else launch_count_slots(t->view(), c.get<unsigned long long>(), t->ctx->stream);
        t->ctx->count_launch();
        unsigned long long d = 0;
        CK(cudaMemcpyAsync(&d, c.get(), 8, cudaMemcpyDeviceToHost, t->ctx->stream));
        CK(cudaStreamSynchronize(t->ctx->stream));
        *distinct_keys = (int64_t)d;
    }
    API_END
}

int ml_gpu_join_build_destroy(ml_join_build* j) {
    API_BEGIN
    if (j) {
        j->ctx->set_current();
        j->streams.sync();
        delete j;
    }
    API_END
}

// HashJoinProbe::execute (join.rs:263-315): all (probe_row, build_row) pairs, by probe row.
int ml_gpu_join_probe(ml_ctx* ctx, ml_join_table* table, const ml_expr* key_exprs, int32_t nkeys, const ml_column* cols,
                      int32_t ncols, int64_t nrows, const uint32_t* sel, int64_t nsel, int32_t location, uint32_t* probe_idx,
                      uint32_t* build_idx, int64_t cap, int64_t* npairs) {
    API_BEGIN
    REQUIRE(ctx && table && key_exprs && npairs, "null argument");
    ctx->set_current();
    OpStream op_stream(ctx);
    cudaStream_t s = op_stream.s;
    if (location == ML_LOC_HOST) check_sel_bounds(sel, nsel, nrows);
    std::vector<int32_t> types;
    for (int c = 0; c < ncols; c++) types.push_back(cols[c].dtype);
    Pipeline p(ctx);
    ml_pipe_op op{};
    op.kind = ML_PIPE_PROBE;
    op.nexprs = nkeys;
    op.exprs = key_exprs;
    op.join = table;
    p.build(&op, 1, types.data(), ncols);
    p.upload();
    Staging st(ctx);
    DevBuf sel_hold;
    const uint32_t* dsel = device_sel(ctx, sel, nsel, sel_hold, s);
    Pipeline::Launch L;
    p.prepare(L, cols, ncols, nrows, dsel, nsel, s, st, nullptr);
    ErrWord ew(ctx);
    CK(cudaMemsetAsync(ew.d.get(), 0, 4, s));
    L.P.err = ew.d.get<uint32_t>();
    DevBuf counts(ctx, std::max<size_t>((size_t)L.P.n * 4, 4), nullptr);
    launch_probe_count(L.P, counts.get<uint32_t>(), s);
    ctx->count_launch();
    DevBuf offs;
    uint64_t total = scan_counts(ctx, counts.get<uint32_t>(), L.P.n, offs, s);
    *npairs = (int64_t)total;
    if ((int64_t)total > cap) raise(ML_ERR_INVALID, "pair buffer too small: " + std::to_string(total) + " pairs");
    DevBuf pi(ctx, std::max<size_t>(total * 4, 4), nullptr), bi(ctx, std::max<size_t>(total * 4, 4), nullptr);
    launch_probe_write(L.P, offs.get<uint64_t>(), pi.get<uint32_t>(), bi.get<uint32_t>(), s);
    ctx->count_launch();
    auto kind = location == ML_LOC_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
    if (total) {
        REQUIRE(probe_idx && build_idx, "null pair buffers");
        CK(cudaMemcpyAsync(probe_idx, pi.get(), total * 4, kind, s));
        CK(cudaMemcpyAsync(build_idx, bi.get(), total * 4, kind, s));
    }
    CK(cudaMemcpyAsync(ew.h, ew.d.get(), 4, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    check_device_error(ctx, *ew.h);
    API_END
}

}  // extern "C"

// =====================================================================================================
// HashAggregateSink (aggregate/hash.rs:285-484)
// =====================================================================================================
namespace {
struct AggState {
    int func, kind, arg_type, in_type, out_type;
    bool has_arg;
    int off = 0;           // word offset in the group block
    Prog arg{};
    bool vcnt_on = false;  // valid-input counts maintained
    DevBuf vcnt;
};

// Probes whose build rows nothing downstream reads (no column slot of that build side, not the
// GROUP BY probe) test membership in the bitmap of a dense, duplicate-free index: a semi-join
// that reads 1/32 of the index's bytes per probe row.
// The membership bitmap of a dense join index (ml_join_table::member), built on stream `s` by
// the first caller; later callers' streams wait for it.
const uint32_t* member_bits(Ctx* ctx, ml_join_table* jt, cudaStream_t s) {
    std::lock_guard<std::mutex> g(jt->member_mu);
    if (!jt->member) {
        jt->member = DevBuf(ctx, std::max<size_t>((jt->drange + 31) / 32 * 4, 4), jt->res.get());
        launch_dense_bits(jt->dense.get<uint32_t>(), jt->drange, jt->member.get<uint32_t>(), s);
        ctx->count_launch();
        CK(cudaEventCreateWithFlags(&jt->member_ready, cudaEventDisableTiming));
        CK(cudaEventRecord(jt->member_ready, s));
    } else {
        CK(cudaStreamWaitEvent(s, jt->member_ready, 0));
    }
    return jt->member.get<uint32_t>();
}

void semi_probes(Ctx* ctx, PipeArgs& P, const Pipeline& pipe, int head_probe, cudaStream_t s) {
    for (size_t p = 0; p < pipe.probes.size(); p++) {
        ml_join_table* jt = pipe.probes[p].jt;
        if (!jt->dense || jt->has_dups || (int)p == head_probe || P.probes[p].late) continue;
        bool read = false;
        for (const SlotInfo& si : pipe.C.slots) read = read || si.src == (int)p + 1;
        if (!read) P.probes[p].member = member_bits(ctx, jt, s);
    }
}

// Grid of a runtime-specialized aggregate launch: the CTAs the rows need, at most one wave of
// resident CTAs (each CTA sets up and flushes its shared-memory groups once).
int agg_grid(void* jit, const PipeArgs& P, int smem) {
    const int64_t k = jit_rows_per_thread(P);
    return std::min<int64_t>(pipeline_grid((P.n + k - 1) / k),
                             (int64_t)jit_resident_blocks(jit, kPipelineThreads, smem) * num_sms());
}
}  // namespace

constexpr uint32_t kSmemPreaggMaxGroups = 65536;

struct ml_hashagg {
    Ctx* ctx;
    std::unique_ptr<Reservation> res;  // declared before everything charged to it
    Pipeline pipe;
    KeyLayout keys{};
    std::vector<KeyDecode> dec;
    std::vector<AggState> aggs;
    bool ungrouped = false;
    int group_probe = -1;
    bool dense_groups = false;  // group id = the join key's dense-index position (ProbeDev::late)  // GROUP BY the join key of this probe: group id = matched build row
    std::vector<int> group_build_cols;
    double max_load = 0.5;
    int stride = 1;        // u64 words per group block
    std::shared_mutex rw;  // shared: a launch in flight; exclusive: table growth
    uint64_t cap = 0;
    uint32_t gid_cap = 0;
    DevBuf slots, gkeys, gnull, acc, ngroups;
    int64_t resizes = 0;
    int64_t final_groups = -1;  // set by finalize
    int smem_groups = 256;
    // ml_gpu_hashagg_run_resident: persistent launch state and the captured launch graphs
    struct Resident {
        DevBuf tables, ovf, count;  // per-batch dictionary tables, overflow rows, overflow count
        std::unique_ptr<ErrWord> ew;
        uint64_t* host_count = nullptr;  // pinned
        cudaStream_t s = nullptr;
        std::vector<std::pair<std::string, cudaGraphExec_t>> graphs;  // launch parameters -> graph
        std::vector<std::string> seen;  // launch parameters run once without a graph (recent 64)
        uint64_t hits = 0, builds = 0;
    } run;
    SinkStreams streams;
    ml_hashagg(Ctx* c) : ctx(c), pipe(c), streams(c) {}
    void resume_overflow(Pipeline::Launch& L, uint64_t count, DevBuf& ovf, int w, cudaStream_t s,
                         unsigned long long* d_count, uint64_t* h_count, ErrWord& ew);
    // Out-of-HBM aggregation (ML_CTX_SPILL): when the HBM budget refuses a table resize, every
    // group's partial state moves to host memory, split by spill partition (key hash bits
    // 32..35), and the table starts empty again (aggregate/hash.rs:189-281, 330-351).
    struct SpillChunk {
        uint32_t n = 0;
        std::vector<uint64_t> keys;    // key words: nwords planes of n
        std::vector<uint32_t> nulls;   // null masks
        std::vector<uint64_t> acc;     // group blocks: n x stride words
        std::vector<uint64_t> vcnt;    // valid-input counts: one plane of n per aggregate in vaggs
        std::vector<int> vaggs;        // aggregates that kept valid-input counts when it spilled
    };
    std::vector<SpillChunk> spills[kSpillParts];
    uint64_t spill_events = 0, spilled_groups = 0;
    // MIN/MAX over strings (accumulator.rs:156-160): the context's interned strings ranked in
    // byte order, rebuilt when strings were interned since (rank_strings = how many it ranks)
    bool str_minmax = false;
    DevBuf str_rank;
    size_t rank_strings = 0;
    void refresh_ranks(cudaStream_t s);
    void spill_state(cudaStream_t s, ErrWord& ew);
    bool can_spill() const { return (ctx->flags & ML_CTX_SPILL) && !ungrouped && group_probe < 0 && !str_minmax; }
    void spill_and_regrow(uint64_t want, cudaStream_t s, ErrWord& ew);
    void regrow(uint64_t want, cudaStream_t s, ErrWord& ew);
    void merge_spilled(const SpillChunk& c, cudaStream_t s, ErrWord& ew);
    void reset_groups(cudaStream_t s);
    // Free the table and its group arrays (it holds no groups); grow() allocates a new one.
    void release_table() {
        slots.release(), gkeys.release(), gnull.release(), acc.release();
        for (auto& a : aggs) a.vcnt.release();
        cap = 0;
        gid_cap = 0;
    }
    ~ml_hashagg() {
        for (auto& g : run.graphs) cudaGraphExecDestroy(g.second);
        if (run.host_count) ctx->release_slot(run.host_count);
        if (run.s) ctx->free_stream(run.s);
    }

    TableView table() const {
        return TableView{slots.get<uint64_t>(), cap ? cap - 1 : 0, keys.nwords, keys.nwords == 1 ? 2 : 4};
    }

    // Direct group slots of this launch (AggArgs::dslots), for the runtime-specialized kernel:
    // every key a dictionary-coded string column of the scanned batch or a BOOL value, and the
    // product of the keys' value counts (NULL included) at most kDirectSlots.
    void direct_slots(AggArgs& A, const Pipeline::Launch& L) const {
        A.dslots = 0;
        if (!agg_direct_on(A)) return;
        uint64_t total = 1;
        uint32_t mul[kMaxKeys], base[kMaxKeys];
        for (int k = 0; k < A.keys.nkeys; k++) {
            const Prog& p = A.keys.prog[k];
            uint64_t range;
            if (A.keys.f[k].type == ML_TYPE_BOOL) {
                base[k] = 0;
                range = 3;
            } else {
                if (p.len != 1 || p.start < 0 || p.start >= (int)pipe.C.code.size()) return;
                const Instr& in = pipe.C.code[p.start];
                if (in.op != I_COL || in.a < 0 || in.a >= (int)L.gid_range.size()) return;
                const auto r = L.gid_range[in.a];
                if (r.first > r.second) return;  // not a dictionary-coded source column
                base[k] = r.first;
                range = (uint64_t)(r.second - r.first) + 2;
            }
            mul[k] = (uint32_t)total;
            total *= range;
            if (total > (uint64_t)kDirectSlots) return;
        }
        A.dslots = (uint32_t)total;
        for (int k = 0; k < A.keys.nkeys; k++) A.dmul[k] = mul[k], A.dbase[k] = base[k];
    }

    AggArgs args(unsigned long long* ovf_count, uint32_t* ovf, uint64_t ovf_cap) {
        AggArgs A{};
        A.keys = keys;
        A.t = table();
        A.gkeys = gkeys.get<uint64_t>();
        A.gnull = gnull.get<uint32_t>();
        A.ngroups = ngroups.get<uint32_t>();
        A.gid_cap = gid_cap;
        A.nagg = (int)aggs.size();
        A.ungrouped = ungrouped;
        A.group_probe = group_probe;
        A.stride = stride;
        A.acc = acc.get<uint64_t>();
        // shared-memory pre-aggregation pays off when the group space is small enough that
        // the first groups take a large share of the rows
        A.smem_groups = (ungrouped || gid_cap <= kSmemPreaggMaxGroups) ? std::min<int>(smem_groups, (int)gid_cap) : 0;
        // the first groups get per-thread accumulators (no atomics) in what the shared-memory
        // budget leaves (three CTAs per SM)
        bool vcnt = false;
        for (const AggState& a : aggs) vcnt = vcnt || (a.vcnt_on && a.kind != A_AVG);
        const int fixed = (int)((size_t)A.smem_groups * stride * 8 + agg_direct_bytes(A));
        A.priv_groups = vcnt || !A.smem_groups
                            ? 0
                            : std::max(0, std::min({A.smem_groups, 8, (kAggSmemBudget - fixed) / (stride * 256 * 8)}));
        A.ovf = ovf;
        A.ovf_count = ovf_count;
        A.ovf_cap = ovf_cap;
        A.str_rank = str_rank.get<uint32_t>();
        for (size_t k = 0; k < aggs.size(); k++) {
            AggDev& d = A.aggs[k];
            const AggState& a = aggs[k];
            d.kind = a.kind;
            d.func = a.func;
            d.has_arg = a.has_arg;
            d.off = a.off;
            d.count_valid = a.vcnt_on && a.kind != A_AVG;
            d.arg = a.arg;
            d.vcnt = a.vcnt_on && a.kind != A_AVG ? a.vcnt.get<uint64_t>() : nullptr;
        }
        return A;
    }

    // Allocate (or grow to) `want` group ids; existing groups are rehashed into the new
    // table (the doubling of SwissTable::reserve, swiss.rs:287-301).
    void grow(uint64_t want, cudaStream_t s, ErrWord& ew) {
        uint32_t old_cap = gid_cap;
        bool hashed = !ungrouped && group_probe < 0;
        uint64_t ncap = hashed ? pow2_at_least((uint64_t)std::ceil(std::max<uint64_t>(want, 8) / max_load)) : 0;
        uint32_t ngid = hashed ? (uint32_t)std::min<uint64_t>((uint64_t)(ncap * max_load), 0xFFFFFFF0ull)
                               : (uint32_t)std::max<uint64_t>(want, 1);
        uint32_t ng = 0;
        if (old_cap && hashed) {
            CK(cudaMemcpyAsync(ew.h, ngroups.get(), 4, cudaMemcpyDeviceToHost, s));
            CK(cudaStreamSynchronize(s));
            ng = std::min(*ew.h, old_cap);
        }
        int nw = keys.nwords ? keys.nwords : 1;
        int sw = nw == 1 ? 2 : 4;
        DevBuf nslots, ngk, ngn;
        if (hashed) {
            nslots = DevBuf(ctx, ncap * 8 * sw, res.get());
            CK(cudaMemsetAsync(nslots.get(), 0, ncap * 8 * sw, s));
            ngk = DevBuf(ctx, (size_t)ngid * 8 * nw, res.get());
            ngn = DevBuf(ctx, (size_t)ngid * 4, res.get());
        }
        DevBuf nacc(ctx, (size_t)ngid * 8 * stride, res.get());
        std::vector<DevBuf> nvc(aggs.size());
        for (size_t k = 0; k < aggs.size(); k++)
            if (aggs[k].vcnt_on && aggs[k].kind != A_AVG) nvc[k] = DevBuf(ctx, (size_t)ngid * 8, res.get());
        if (old_cap) {  // keep the existing groups
            if (hashed) {
                for (int w = 0; w < nw; w++)
                    if (ng) CK(cudaMemcpyAsync(ngk.get<uint64_t>() + (size_t)w * ngid, gkeys.get<uint64_t>() + (size_t)w * old_cap,
                                               (size_t)ng * 8, cudaMemcpyDeviceToDevice, s));
                if (ng) CK(cudaMemcpyAsync(ngn.get(), gnull.get(), (size_t)ng * 4, cudaMemcpyDeviceToDevice, s));
            }
            CK(cudaMemcpyAsync(nacc.get(), acc.get(), (size_t)old_cap * 8 * stride, cudaMemcpyDeviceToDevice, s));
            for (size_t k = 0; k < aggs.size(); k++)
                if (nvc[k]) CK(cudaMemcpyAsync(nvc[k].get(), aggs[k].vcnt.get(), (size_t)old_cap * 8, cudaMemcpyDeviceToDevice, s));
        }
        slots = std::move(nslots);
        gkeys = std::move(ngk);
        gnull = std::move(ngn);
        acc = std::move(nacc);
        for (size_t k = 0; k < aggs.size(); k++) aggs[k].vcnt = std::move(nvc[k]);
        cap = ncap;
        gid_cap = ngid;
        AggArgs A = args(nullptr, nullptr, 0);
        for (size_t k = 0; k < aggs.size(); k++) A.aggs[k].vcnt = aggs[k].vcnt.get<uint64_t>();
        launch_acc_init(A, old_cap, ngid, s);
        ctx->count_launch();
        if (hashed && ng) {
            CK(cudaMemsetAsync(ew.d.get(), 0, 4, s));
            launch_agg_rehash(A.t, gkeys.get<uint64_t>(), gnull.get<uint32_t>(), gid_cap, ng, nw, ew.d.get<uint32_t>(), s);
            ctx->count_launch();
            CK(cudaMemcpyAsync(ew.h, ew.d.get(), 4, cudaMemcpyDeviceToHost, s));
        }
        CK(cudaMemcpyAsync(ngroups.get(), &ng, 4, cudaMemcpyHostToDevice, s));
        CK(cudaStreamSynchronize(s));
        if (hashed && ng) check_device_error(ctx, *ew.h);
    }

    // The join key of probe p is the GROUP BY key when every group key reads the same
    // column as the probe key (or the build key it matched) with the same type: then the
    // matched build row identifies the group and no aggregate hash table is needed.
    void detect_group_probe(const ml_expr* group, int ngroup) {
        for (int p = (int)pipe.probes.size() - 1; p >= 0 && ngroup > 0; p--) {
            ml_join_table* jt = pipe.probes[p].jt;
            if ((int)jt->key_types.size() != ngroup) continue;
            const KeyLayout& pk = pipe.probes[p].keys;
            bool ok = true;
            std::vector<int> cols;
            for (int k = 0; k < ngroup && ok; k++) {
                ExprNode ge = parse_expr(group[k]);
                auto go = pipe.C.column_origin(ge, pipe.out);
                int bc = jt->key_cols[k];
                ok = go && group[k].dtype == jt->key_types[k] && group[k].dtype != ML_TYPE_UTF8 && bc >= 0;
                if (!ok) break;
                // the probe key program is a single column load (a column reference)
                const Prog& pr = pk.prog[k];
                bool probe_col = pr.len == 1 && pipe.C.code[pr.start].op == I_COL;
                const SlotInfo* ps = probe_col ? &pipe.C.slots[pipe.C.code[pr.start].a] : nullptr;
                bool same_probe = ps && ps->src == go->src && ps->index == go->index;
                bool same_build = go->src == p + 1 && go->index == bc;
                ok = same_probe || same_build;
                cols.push_back(bc);
            }
            if (ok) {
                group_probe = p;
                group_build_cols = cols;
                return;
            }
        }
    }
};

// resize-on-overflow (swiss.rs:219-232 grows by doubling; here the table grows to hold
// the groups so far plus the rows that did not fit), then aggregate those rows again
void ml_hashagg::resume_overflow(Pipeline::Launch& L, uint64_t count, DevBuf& ovf, int w, cudaStream_t s,
                                 unsigned long long* d_count, uint64_t* h_count, ErrWord& ew) {
    while (count) {
        std::unique_lock<std::shared_mutex> lk(rw);
        streams.sync();
        if (run.s) CK(cudaStreamSynchronize(run.s));
        CK(cudaMemcpyAsync(ew.h, ngroups.get(), 4, cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
        uint32_t ng = std::min(*ew.h, gid_cap);
        uint64_t want = std::max<uint64_t>((uint64_t)gid_cap * 2, (uint64_t)ng + std::min<uint64_t>(count, 1ull << 30));
        try {
            grow(std::min<uint64_t>(want, 0x7FFFFFFFull), s, ew);
            resizes++;
        } catch (const MlError& e) {
            // HashAggLocal::account (aggregate/hash.rs:330-351): with spilling on, a refused
            // resize moves the groups to host memory and the rows that did not fit go into the
            // emptied table; without it the refusal is the query's error
            if (e.code != ML_ERR_BUDGET || !can_spill()) throw;
            spill_and_regrow(std::min<uint64_t>(want, 0x7FFFFFFFull), s, ew);
        }
        DevBuf ovf2(ctx, count * w * 4, nullptr);
        CK(cudaMemsetAsync(d_count, 0, 8, s));
        CK(cudaMemsetAsync(ew.d.get(), 0, 4, s));
        L.P.err = ew.d.get<uint32_t>();
        AggArgs A = args(d_count, ovf2.get<uint32_t>(), count);
        A.priv_groups = 0;  // the few rows that overflowed: shared-memory atomics suffice
        void* jit = jit_agg_resume_kernel(ctx, pipe, L.P, A);
        if (jit) {
            const uint32_t* rows = ovf.get<uint32_t>();
            uint64_t cnt = count;
            int ww = w;
            void* args[] = {&L.P, &A, &rows, &cnt, &ww};
            jit_launch(jit, pipeline_grid((int64_t)count), kPipelineThreads, agg_smem_bytes(A), s, args);
            ctx->add_profile("jit_launch", 0);
        } else {
            launch_agg_resume(L.P, A, ovf.get<uint32_t>(), count, w, agg_smem_bytes(A), s);
        }
        ctx->count_launch();
        CK(cudaMemcpyAsync(h_count, d_count, 8, cudaMemcpyDeviceToHost, s));
        CK(cudaMemcpyAsync(ew.h, ew.d.get(), 4, cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
        check_device_error(ctx, *ew.h);
        count = *h_count;
        ovf = std::move(ovf2);
    }
}

// Called with the sink's lock held exclusively and its launches drained.
void ml_hashagg::refresh_ranks(cudaStream_t s) {
    std::vector<uint32_t> rank;
    {
        std::lock_guard<std::mutex> g(pipe.intern.mu);
        const auto& strs = pipe.intern.strs;
        if (str_rank && strs.size() == rank_strings) return;
        std::vector<uint32_t> order(strs.size());
        for (size_t i = 0; i < order.size(); i++) order[i] = (uint32_t)i;
        std::sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) { return strs[a] < strs[b]; });
        rank.assign(std::max<size_t>(strs.size(), 1), 0);
        for (size_t i = 0; i < order.size(); i++) rank[order[i]] = (uint32_t)i;
        rank_strings = strs.size();
    }
    DevBuf nr(ctx, rank.size() * 4, res.get());
    CK(cudaMemcpyAsync(nr.get(), rank.data(), rank.size() * 4, cudaMemcpyHostToDevice, s));
    RerankOffs R{};
    for (const AggState& a : aggs)
        if (a.kind == A_MIN_STR || a.kind == A_MAX_STR) R.off[R.n++] = a.off;
    if (gid_cap) launch_str_rerank(acc.get<uint64_t>(), stride, gid_cap, R, nr.get<uint32_t>(), s);
    ctx->count_launch();
    CK(cudaStreamSynchronize(s));  // `rank` is read by the copy; the states use the new ranks
    str_rank = std::move(nr);
}

void ml_hashagg::reset_groups(cudaStream_t s) {
    CK(cudaMemsetAsync(ngroups.get(), 0, 16, s));
    if (cap) CK(cudaMemsetAsync(slots.get(), 0, cap * 8 * (keys.nwords == 1 ? 2 : 4), s));
    AggArgs A = args(nullptr, nullptr, 0);
    for (size_t k = 0; k < aggs.size(); k++) A.aggs[k].vcnt = aggs[k].vcnt.get<uint64_t>();
    launch_acc_init(A, 0, gid_cap, s);
    ctx->count_launch();
}

void ml_hashagg::spill_and_regrow(uint64_t want, cudaStream_t s, ErrWord& ew) {
    spill_state(s, ew);
    regrow(want, s, ew);
}

void ml_hashagg::regrow(uint64_t want, cudaStream_t s, ErrWord& ew) {
    // the emptied table is freed, then the largest table the budget admits replaces it (no old
    // groups to copy now); below 1024 groups the refusal stands
    release_table();
    for (uint64_t w = want;; w /= 2) {
        try {
            grow(std::max<uint64_t>(w, 1024), s, ew);
            return;
        } catch (const MlError& e) {
            if (e.code != ML_ERR_BUDGET || w <= 1024) throw;
        }
    }
}

void ml_hashagg::spill_state(cudaStream_t s, ErrWord& ew) {
    uint32_t ng = 0;
    CK(cudaMemcpyAsync(ew.h, ngroups.get(), 4, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    ng = std::min(*ew.h, gid_cap);
    spill_events++;
    if (!ng) return;
    const int nw = keys.nwords ? keys.nwords : 1;
    std::vector<int> vc;  // aggregates keeping valid-input counts
    for (size_t k = 0; k < aggs.size(); k++)
        if (aggs[k].vcnt_on && aggs[k].kind != A_AVG) vc.push_back((int)k);
    // group ids grouped by spill partition (a stable counting sort on the device)
    DevBuf part(ctx, (size_t)ng * 8, nullptr), perm(ctx, (size_t)ng * 4, nullptr), offs;
    launch_spill_part(gkeys.get<uint64_t>(), gnull.get<uint32_t>(), gid_cap, ng, nw, part.get<uint64_t>(), s);
    const int nb = xpart_blocks(ng);
    DevBuf bc(ctx, (size_t)nb * kSpillParts * 4, nullptr);
    launch_xpart_count(part.get<uint64_t>(), ng, kSpillParts, bc.get<uint32_t>(), s);
    scan_counts(ctx, bc.get<uint32_t>(), (int64_t)nb * kSpillParts, offs, s);
    launch_xpart_scatter(part.get<uint64_t>(), ng, kSpillParts, offs.get<uint64_t>(), perm.get<uint32_t>(), s);
    std::vector<uint64_t> starts(kSpillParts + 1);
    CK(cudaMemcpy2DAsync(starts.data(), 8, offs.get(), (size_t)nb * 8, 8, kSpillParts + 1, cudaMemcpyDeviceToHost, s));
    // the partial states in partition order, then to host memory
    const uint32_t* pm = perm.get<uint32_t>();
    DevBuf gk(ctx, (size_t)ng * 8 * nw, nullptr), gn(ctx, (size_t)ng * 4, nullptr);
    DevBuf ga(ctx, (size_t)ng * 8 * stride, nullptr), gv(ctx, std::max<size_t>((size_t)ng * 8 * vc.size(), 8), nullptr);
    for (int w = 0; w < nw; w++)
        launch_gather_fixed(gkeys.get<uint64_t>() + (size_t)w * gid_cap, 8, pm, ng, gk.get<uint64_t>() + (size_t)w * ng, s);
    launch_gather_fixed(gnull.get(), 4, pm, ng, gn.get(), s);
    launch_gather_fixed(acc.get(), 8 * stride, pm, ng, ga.get(), s);
    for (size_t v = 0; v < vc.size(); v++)
        launch_gather_fixed(aggs[vc[v]].vcnt.get(), 8, pm, ng, gv.get<uint64_t>() + v * ng, s);
    ctx->count_launch(4 + nw + vc.size());
    std::vector<uint64_t> hk((size_t)ng * nw), ha((size_t)ng * stride), hv((size_t)ng * vc.size());
    std::vector<uint32_t> hn(ng);
    CK(cudaMemcpyAsync(hk.data(), gk.get(), hk.size() * 8, cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(hn.data(), gn.get(), hn.size() * 4, cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(ha.data(), ga.get(), ha.size() * 8, cudaMemcpyDeviceToHost, s));
    if (!hv.empty()) CK(cudaMemcpyAsync(hv.data(), gv.get(), hv.size() * 8, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    for (int p = 0; p < kSpillParts; p++) {
        const uint64_t a = starts[p], b = starts[p + 1];
        if (a == b) continue;
        SpillChunk c;
        c.n = (uint32_t)(b - a);
        for (int w = 0; w < nw; w++) c.keys.insert(c.keys.end(), hk.begin() + (size_t)w * ng + a, hk.begin() + (size_t)w * ng + b);
        c.nulls.assign(hn.begin() + a, hn.begin() + b);
        c.acc.assign(ha.begin() + a * stride, ha.begin() + b * stride);
        for (size_t v = 0; v < vc.size(); v++)
            c.vcnt.insert(c.vcnt.end(), hv.begin() + v * ng + a, hv.begin() + v * ng + b);
        c.vaggs = vc;
        spills[p].push_back(std::move(c));
    }
    spilled_groups += ng;
    reset_groups(s);
    CK(cudaStreamSynchronize(s));
}

void ml_hashagg::merge_spilled(const SpillChunk& c, cudaStream_t s, ErrWord& ew) {
    AggArgs A = args(nullptr, nullptr, 0);
    for (size_t k = 0; k < aggs.size(); k++) A.aggs[k].vcnt = aggs[k].vcnt.get<uint64_t>();
    CK(cudaMemsetAsync(ew.d.get(), 0, 4, s));
    std::vector<int> vc;  // aggregates keeping valid-input counts now
    for (size_t k = 0; k < aggs.size(); k++)
        if (aggs[k].vcnt_on && aggs[k].kind != A_AVG) vc.push_back((int)k);
    {
        // valid-input counts in the order the merge reads them; an aggregate that started counting
        // after this chunk spilled had only valid inputs before: its count is the group's rows
        std::vector<uint64_t> planes((size_t)c.n * vc.size());
        for (size_t v = 0; v < vc.size(); v++) {
            const auto it = std::find(c.vaggs.begin(), c.vaggs.end(), vc[v]);
            for (uint32_t r = 0; r < c.n; r++)
                planes[v * c.n + r] = it != c.vaggs.end() ? c.vcnt[(size_t)(it - c.vaggs.begin()) * c.n + r]
                                                          : c.acc[(size_t)r * stride];
        }
        DevBuf k(ctx, c.keys.size() * 8, nullptr), nl(ctx, c.nulls.size() * 4, nullptr), a(ctx, c.acc.size() * 8, nullptr);
        DevBuf v(ctx, std::max<size_t>(planes.size() * 8, 8), nullptr);
        CK(cudaMemcpyAsync(k.get(), c.keys.data(), c.keys.size() * 8, cudaMemcpyHostToDevice, s));
        CK(cudaMemcpyAsync(nl.get(), c.nulls.data(), c.nulls.size() * 4, cudaMemcpyHostToDevice, s));
        CK(cudaMemcpyAsync(a.get(), c.acc.data(), c.acc.size() * 8, cudaMemcpyHostToDevice, s));
        if (!planes.empty()) CK(cudaMemcpyAsync(v.get(), planes.data(), planes.size() * 8, cudaMemcpyHostToDevice, s));
        launch_agg_merge_spill(A, k.get<uint64_t>(), nl.get<uint32_t>(), a.get<uint64_t>(), v.get<uint64_t>(), c.n,
                               ew.d.get<uint32_t>(), s);
        ctx->count_launch();
        CK(cudaStreamSynchronize(s));  // the chunk's device copies go out of scope
    }
    CK(cudaMemcpyAsync(ew.h, ew.d.get(), 4, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    check_device_error(ctx, *ew.h);
}

// The host side of HashAggregateSink::new: compile the prologue, the GROUP BY keys and the
// aggregate arguments into the sink's pipeline, and lay out the group blocks.
void compile_hashagg(ml_hashagg* h, const ml_pipe_op* prologue, int32_t nprologue, const int32_t* input_types,
                     int32_t ninput, const ml_expr* group_exprs, int32_t ngroup, const ml_agg_spec* aggs, int32_t nagg) {
    h->pipe.build(prologue, nprologue, input_types, ninput);
    h->ungrouped = ngroup == 0;
    if (!h->ungrouped) {
        h->detect_group_probe(group_exprs, ngroup);
        if (h->group_probe < 0) h->keys = h->pipe.key_layout(group_exprs, ngroup, h->pipe.out, true, &h->dec);
    }
    int words = 1;  // word 0: rows of the group
    for (int k = 0; k < nagg; k++) {  // Accumulator::new (accumulator.rs:110-169)
        AggState a{};
        a.func = aggs[k].func;
        a.arg_type = aggs[k].arg_type;
        int t = a.arg_type;
        auto bad = [&]() { raise(ML_ERR_UNSUPPORTED, "aggregate function " + std::to_string(a.func) + " over type " + std::to_string(t)); };
        switch (a.func) {
            case ML_AGG_COUNT_STAR: a.kind = A_COUNT; a.in_type = -1; a.out_type = ML_TYPE_INT64; break;
            case ML_AGG_COUNT: a.kind = A_COUNT; a.in_type = t; a.out_type = ML_TYPE_INT64; break;
            case ML_AGG_SUM:
                if (t == ML_TYPE_INT32 || t == ML_TYPE_INT64 || t == ML_TYPE_BOOL) { a.kind = A_SUM_I64; a.in_type = ML_TYPE_INT64; a.out_type = ML_TYPE_INT64; }
                else if (t == ML_TYPE_FLOAT64) { a.kind = A_SUM_F64; a.in_type = t; a.out_type = t; }
                else bad();
                break;
            case ML_AGG_AVG:
                if (t == ML_TYPE_INT32 || t == ML_TYPE_INT64 || t == ML_TYPE_FLOAT64) { a.kind = A_AVG; a.in_type = ML_TYPE_FLOAT64; a.out_type = ML_TYPE_FLOAT64; a.vcnt_on = true; }
                else bad();
                break;
            case ML_AGG_MIN:
            case ML_AGG_MAX: {
                bool mn = a.func == ML_AGG_MIN;
                if (t == ML_TYPE_INT32 || t == ML_TYPE_INT64 || t == ML_TYPE_DATE) { a.kind = mn ? A_MIN_I64 : A_MAX_I64; a.in_type = ML_TYPE_INT64; a.out_type = t; }
                else if (t == ML_TYPE_FLOAT64) { a.kind = mn ? A_MIN_F64 : A_MAX_F64; a.in_type = t; a.out_type = t; }
                else if (t == ML_TYPE_UTF8) {  // the argument is the string's id (compile_string_key)
                    a.kind = mn ? A_MIN_STR : A_MAX_STR;
                    a.in_type = ML_TYPE_UTF8;
                    a.out_type = ML_TYPE_UTF8;
                    h->str_minmax = true;
                }
                else bad();
                break;
            }
            default: bad();
        }
        if (a.func != ML_AGG_COUNT_STAR) {
            a.off = words;
            words += a.kind == A_AVG ? 2 : 1;
        }
        a.has_arg = a.func != ML_AGG_COUNT_STAR;
        if (a.has_arg) {
            REQUIRE(aggs[k].arg.nnodes > 0, "aggregate without an argument");
            ExprNode e = parse_expr(aggs[k].arg);
            if (t == ML_TYPE_UTF8) {  // COUNT(string): only validity matters
                int slot;
                a.arg = h->pipe.C.compile_string_key(e, h->pipe.out, &slot);
            } else {
                a.arg = h->pipe.C.compile_value(e, h->pipe.out, t);
                if (a.in_type >= 0 && a.in_type != t) {  // Accumulator::prepare_input cast
                    Instr c{};
                    c.op = I_CAST;
                    c.sub = (uint8_t)a.in_type;
                    c.t = (uint8_t)t;
                    h->pipe.C.code.push_back(c);
                    a.arg.len++;
                    a.arg.type = a.in_type;
                    classify(a.arg, h->pipe.C.code);
                }
            }
        }
        h->aggs.push_back(std::move(a));
    }
    h->stride = words;
    // GROUP BY a dense, distinct join key whose probe ends the pipeline, with nothing reading
    // that probe's build row: group by the index position and check membership at finalize
    if (h->group_probe >= 0) {
        const int p = h->group_probe;
        const ml_join_table* jt = h->pipe.probes[p].jt;
        bool ok = jt->dense && !jt->has_dups && h->pipe.nstages > 0 && h->pipe.stages[h->pipe.nstages - 1].kind == 1 &&
                  h->pipe.stages[h->pipe.nstages - 1].idx == p;
        for (const SlotInfo& si : h->pipe.C.slots) ok = ok && si.src != p + 1;
        h->dense_groups = ok;
    }
}

struct ml_hashagg_local {
    ml_hashagg* sink;
    cudaStream_t s;
    Staging st;
    ErrWord ew;
    DevBuf ovf_count;  // u64
    uint64_t* h_count;
    ml_hashagg_local(ml_hashagg* k)
        : sink(k), s(k->ctx->new_stream()), st(k->ctx), ew(k->ctx), ovf_count(k->ctx, 16, nullptr) {
        h_count = (uint64_t*)k->ctx->pinned_slot();
        sink->streams.add(s);
    }
    ~ml_hashagg_local() {
        sink->streams.remove(s);
        sink->ctx->release_slot(h_count);
        sink->ctx->free_stream(s);
    }
};

extern "C" {

int ml_gpu_hashagg_create(ml_ctx* ctx, const ml_pipe_op* prologue, int32_t nprologue, const int32_t* input_types, int32_t ninput,
                          const ml_expr* group_exprs, int32_t ngroup, const ml_agg_spec* aggs, int32_t nagg, int64_t size_hint,
                          ml_hashagg** out) {
    API_BEGIN
    HostTimer host_timer_(ctx, "host:hashagg_create");
    REQUIRE(ctx && out, "null argument");
    REQUIRE(ngroup >= 0 && nagg >= 0 && (ngroup == 0 || group_exprs) && (nagg == 0 || aggs), "bad arguments");
    REQUIRE(nagg <= kMaxAggs, "too many aggregates");
    ctx->set_current();
    auto h = std::make_unique<ml_hashagg>(ctx);
    compile_hashagg(h.get(), prologue, nprologue, input_types, ninput, group_exprs, ngroup, aggs, nagg);
    h->pipe.upload();
    h->res = std::make_unique<Reservation>(ctx, "HashAggregate");
    h->ngroups = DevBuf(ctx, 16, nullptr);
    CK(cudaMemsetAsync(h->ngroups.get(), 0, 16, ctx->stream));  // grow() below runs on ctx->stream
    ErrWord ew(ctx);
    uint64_t want;
    if (h->ungrouped) want = 1;
    else if (h->dense_groups) want = h->pipe.probes[h->group_probe].jt->drange;
    else if (h->group_probe >= 0) want = (uint64_t)std::max<int64_t>(h->pipe.probes[h->group_probe].jt->batch.nrows, 1);
    else want = (uint64_t)std::min<int64_t>(std::max<int64_t>(size_hint > 0 ? size_hint : 1024, 16), 0x7FFFFFFF);
    h->grow(want, ctx->stream, ew);
    *out = h.release();
    API_END
}

int ml_gpu_hashagg_local_create(ml_hashagg* sink, ml_hashagg_local** out) {
    API_BEGIN
    REQUIRE(sink && out, "null argument");
    sink->ctx->set_current();
    *out = new ml_hashagg_local(sink);
    API_END
}

int ml_gpu_hashagg_sink(ml_hashagg_local* local, const ml_column* cols, int32_t ncols, int64_t nrows, const uint32_t* sel,
                        int64_t nsel) {
    API_BEGIN
    HostTimer host_timer_(local ? local->sink->ctx : nullptr, "host:hashagg_sink");
    REQUIRE(local, "null local sink");
    ml_hashagg* h = local->sink;
    Ctx* ctx = h->ctx;
    ctx->set_current();
    cudaStream_t s = local->s;
    check_sel_bounds(sel, nsel, nrows);
    DevBuf sel_hold;
    const uint32_t* dsel = device_sel(ctx, sel, nsel, sel_hold, s);
    Pipeline::Launch L;
    h->pipe.prepare(L, cols, ncols, nrows, dsel, nsel, s, local->st, nullptr);
    if (h->str_minmax) {  // this batch's strings are interned now: rank them with the rest
        std::unique_lock<std::shared_mutex> lk(h->rw);
        h->streams.sync();
        if (h->run.s) CK(cudaStreamSynchronize(h->run.s));
        h->refresh_ranks(s);
    }
    // seen-tracking: once an argument can be NULL, count valid inputs per group
    for (auto& a : h->aggs) {
        if (!a.has_arg || a.vcnt_on || a.kind == A_COUNT) continue;
        if (a.arg.maybe_null || h->pipe.reads_nullable(a.arg, L)) {
            std::unique_lock<std::shared_mutex> lk(h->rw);
            if (!a.vcnt_on) {
                h->streams.sync();
                try {
                    a.vcnt = DevBuf(ctx, (size_t)h->gid_cap * 8, h->res.get());
                    // every contribution so far was valid: start from the groups' row counts
                    CK(cudaMemcpy2DAsync(a.vcnt.get(), 8, h->acc.get(), (size_t)h->stride * 8, 8, h->gid_cap,
                                         cudaMemcpyDeviceToDevice, s));
                    CK(cudaStreamSynchronize(s));
                    a.vcnt_on = true;
                } catch (const MlError& e) {
                    // no room for the counts: the groups spill (their counts are their rows) and
                    // a table with the counts, as large as the budget admits, replaces this one
                    if (e.code != ML_ERR_BUDGET || !h->can_spill()) throw;
                    ErrWord ew(ctx);
                    const uint64_t want = h->gid_cap;
                    h->spill_state(s, ew);
                    a.vcnt_on = true;  // after the spill: the spilled chunk holds no counts for it
                    h->regrow(want, s, ew);
                }
            }
        }
    }
    int w = 1 + (int)h->pipe.probes.size();
    bool can_overflow = !h->ungrouped && h->group_probe < 0;
    uint64_t ovf_cap = can_overflow ? std::max<uint64_t>((uint64_t)L.P.n, 1024) : 0;
    DevBuf ovf(ctx, std::max<uint64_t>(ovf_cap * w * 4, 16), nullptr);
    uint64_t count;
    {
        std::shared_lock<std::shared_mutex> lk(h->rw);
        CK(cudaMemsetAsync(local->ovf_count.get(), 0, 8, s));
        CK(cudaMemsetAsync(local->ew.d.get(), 0, 4, s));
        L.P.err = local->ew.d.get<uint32_t>();
        L.P.head_probe = h->group_probe;
        if (h->dense_groups) L.P.probes[h->group_probe].late = 1;
        semi_probes(ctx, L.P, h->pipe, h->group_probe, s);
        AggArgs A = h->args(local->ovf_count.get<unsigned long long>(), ovf.get<uint32_t>(), ovf_cap);
        h->direct_slots(A, L);
        void* jit = jit_agg_kernel(ctx, h->pipe, L.P, A);
        if (!jit) A.priv_groups = 0, A.dslots = 0;  // both exist in specialized kernels only
        KernelTimer kt(ctx, s, "pipeline_aggregate");
        if (jit) {
            if (L.P.n) {
                void* args[] = {&L.P, &A};
                const int smem = agg_smem_bytes(A);
                jit_launch(jit, agg_grid(jit, L.P, smem), kPipelineThreads, smem, s, args);
            }
            ctx->add_profile("jit_launch", 0);
        } else {
            launch_agg(L.P, A, agg_smem_bytes(A), s);
        }
        kt.stop();
        ctx->count_launch();
        CK(cudaMemcpyAsync(local->h_count, local->ovf_count.get(), 8, cudaMemcpyDeviceToHost, s));
        CK(cudaMemcpyAsync(local->ew.h, local->ew.d.get(), 4, cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
        check_device_error(ctx, *local->ew.h);
        count = *local->h_count;
    }
    // resize-on-overflow: grow the table, then aggregate the rows that did not fit
    h->resume_overflow(L, count, ovf, w, s, local->ovf_count.get<unsigned long long>(), local->h_count, local->ew);
    API_END
}

int ml_gpu_hashagg_rebind(ml_hashagg* h, const ml_pipe_op* prologue, int32_t nprologue, const int32_t* input_types,
                          int32_t ninput, const ml_expr* group_exprs, int32_t ngroup, const ml_agg_spec* aggs,
                          int32_t nagg) {
    API_BEGIN
    REQUIRE(h, "null sink");
    REQUIRE(nagg <= kMaxAggs && nagg == (int32_t)h->aggs.size(), "rebind: the aggregates differ from the sink's");
    Ctx* ctx = h->ctx;
    ctx->set_current();
    ml_hashagg fresh(ctx);
    compile_hashagg(&fresh, prologue, nprologue, input_types, ninput, group_exprs, ngroup, aggs, nagg);
    const Compiler &a = h->pipe.C, &b = fresh.pipe.C;
    bool same = a.code.size() == b.code.size() && a.arena.size() == b.arena.size() && a.slots.size() == b.slots.size() &&
                a.luts.size() == b.luts.size() && fresh.stride == h->stride && fresh.group_probe == h->group_probe &&
                fresh.ungrouped == h->ungrouped && fresh.dense_groups == h->dense_groups &&
                fresh.pipe.nstages == h->pipe.nstages &&
                fresh.pipe.probes.size() == h->pipe.probes.size() && memcmp(&fresh.keys, &h->keys, sizeof(KeyLayout)) == 0;
    for (size_t i = 0; same && i < a.code.size(); i++) {
        const Instr &x = a.code[i], &y = b.code[i];
        same = x.op == y.op && x.sub == y.sub && x.t == y.t && x.flag == y.flag && x.a == y.a && x.b == y.b && x.c == y.c &&
               x.lit_valid == y.lit_valid;
    }
    for (size_t i = 0; same && i < a.slots.size(); i++)
        same = a.slots[i].src == b.slots[i].src && a.slots[i].index == b.slots[i].index && a.slots[i].dtype == b.slots[i].dtype;
    for (size_t i = 0; same && i < a.luts.size(); i++)
        same = a.luts[i].slot == b.luts[i].slot && a.luts[i].what == b.luts[i].what && a.luts[i].op == b.luts[i].op;
    // the group state is sized for the grouping join table: it cannot change
    if (same && h->group_probe >= 0)
        same = fresh.pipe.probes[h->group_probe].jt == h->pipe.probes[h->group_probe].jt;
    if (!same) raise(ML_ERR_INVALID, "rebind: the pipeline's shape differs from the sink's (only constants may change)");
    std::unique_lock<std::shared_mutex> lk(h->rw);
    h->streams.sync();
    if (h->run.s) CK(cudaStreamSynchronize(h->run.s));
    h->pipe.C.code = b.code;
    h->pipe.C.arena = b.arena;
    h->pipe.C.luts = b.luts;
    for (size_t p = 0; p < h->pipe.probes.size(); p++) h->pipe.probes[p].jt = fresh.pipe.probes[p].jt;
    for (size_t k = 0; k < h->aggs.size(); k++) h->aggs[k].arg = fresh.aggs[k].arg;
    cudaStream_t s = h->streams.own();
    if (!b.code.empty())
        CK(cudaMemcpyAsync(h->pipe.d_prog, b.code.data(), b.code.size() * sizeof(Instr), cudaMemcpyHostToDevice, s));
    if (!b.arena.empty()) CK(cudaMemcpyAsync(h->pipe.d_arena, b.arena.data(), b.arena.size(), cudaMemcpyHostToDevice, s));
    CK(cudaStreamSynchronize(s));
    API_END
}

int ml_gpu_hashagg_reset(ml_hashagg* h) {
    API_BEGIN
    REQUIRE(h, "null sink");
    Ctx* ctx = h->ctx;
    ctx->set_current();
    std::unique_lock<std::shared_mutex> lk(h->rw);
    h->streams.sync();
    if (h->run.s) CK(cudaStreamSynchronize(h->run.s));
    cudaStream_t s = h->streams.own();
    CK(cudaMemsetAsync(h->ngroups.get(), 0, 16, s));
    if (h->cap) CK(cudaMemsetAsync(h->slots.get(), 0, h->cap * 8 * (h->keys.nwords == 1 ? 2 : 4), s));
    launch_acc_init(h->args(nullptr, nullptr, 0), 0, h->gid_cap, s);
    ctx->count_launch();
    CK(cudaStreamSynchronize(s));
    h->final_groups = -1;
    API_END
}

// One device-resident batch through the sink, launched as a CUDA graph: the graph (reset of
// the group state when asked, overflow counter and error word, the fused pipeline kernel,
// read-back of both words) is captured once per set of launch parameters and replayed.
int ml_gpu_hashagg_run_resident(ml_hashagg* h, const ml_column* cols, int32_t ncols, int64_t nrows, int32_t reset) {
    API_BEGIN
    REQUIRE(h && (cols || ncols == 0) && nrows >= 0, "bad arguments");
    for (int c = 0; c < ncols; c++)
        REQUIRE(cols[c].location == ML_LOC_DEVICE, "ml_gpu_hashagg_run_resident reads device-resident columns only");
    Ctx* ctx = h->ctx;
    ctx->set_current();
    std::unique_lock<std::shared_mutex> lk(h->rw);  // one resident run at a time per sink
    ml_hashagg::Resident& R = h->run;
    if (!R.s) {
        R.s = ctx->new_stream();
        R.ew = std::make_unique<ErrWord>(ctx);
        R.host_count = (uint64_t*)ctx->pinned_slot();
        R.count = DevBuf(ctx, 16, nullptr);
        R.tables = DevBuf(ctx, 64 << 10, nullptr);
    }
    cudaStream_t s = R.s;
    Staging st(ctx);
    Pipeline::Launch L;
    h->pipe.prepare(L, cols, ncols, nrows, nullptr, 0, s, st, nullptr, R.tables.get<uint8_t>(), R.tables.bytes());
    if (h->str_minmax) {
        h->streams.sync();
        h->refresh_ranks(s);
    }
    for (auto& a : h->aggs)
        if (a.has_arg && !a.vcnt_on && a.kind != A_COUNT && (a.arg.maybe_null || h->pipe.reads_nullable(a.arg, L)))
            raise(ML_ERR_UNSUPPORTED, "ml_gpu_hashagg_run_resident: an aggregate input can be NULL; use a local sink");
    const int w = 1 + (int)h->pipe.probes.size();
    const bool can_overflow = !h->ungrouped && h->group_probe < 0;
    const uint64_t ovf_cap = can_overflow ? std::max<uint64_t>((uint64_t)L.P.n, 1024) : 0;
    if (R.ovf.bytes() < std::max<uint64_t>(ovf_cap * w * 4, 16)) R.ovf = DevBuf(ctx, std::max<uint64_t>(ovf_cap * w * 4, 16), nullptr);
    L.P.err = R.ew->d.get<uint32_t>();
    L.P.head_probe = h->group_probe;
        if (h->dense_groups) L.P.probes[h->group_probe].late = 1;
    semi_probes(ctx, L.P, h->pipe, h->group_probe, s);
    AggArgs A = h->args(R.count.get<unsigned long long>(), R.ovf.get<uint32_t>(), ovf_cap);
    h->direct_slots(A, L);
    void* jit = jit_agg_kernel(ctx, h->pipe, L.P, A);
    if (!jit) A.priv_groups = 0, A.dslots = 0;  // both exist in specialized kernels only
    const int smem = agg_smem_bytes(A);
    const int grid = jit ? agg_grid(jit, L.P, smem) : pipeline_grid(L.P.n);
    // the graph is keyed by everything its nodes capture
    std::string key((const char*)&L.P, sizeof(PipeArgs));
    key.append((const char*)&A, sizeof(AggArgs));
    key.append((const char*)&jit, sizeof(jit));
    key.append(1, (char)(reset != 0));
    // the whole run: reset, clear the read-back words, the fused kernel, read back
    auto enqueue = [&]() {
        if (reset) {
            CK(cudaMemsetAsync(h->ngroups.get(), 0, 16, s));
            if (h->cap) CK(cudaMemsetAsync(h->slots.get(), 0, h->cap * 8 * (h->keys.nwords == 1 ? 2 : 4), s));
            launch_acc_init(A, 0, h->gid_cap, s);
        }
        CK(cudaMemsetAsync(R.count.get(), 0, 8, s));
        CK(cudaMemsetAsync(R.ew->d.get(), 0, 4, s));
        if (L.P.n) {
            if (jit) {
                void* args[] = {&L.P, &A};
                jit_launch(jit, grid, kPipelineThreads, smem, s, args);
            } else {
                launch_agg(L.P, A, smem, s);
            }
        }
        CK(cudaMemcpyAsync(R.host_count, R.count.get(), 8, cudaMemcpyDeviceToHost, s));
        CK(cudaMemcpyAsync(R.ew->h, R.ew->d.get(), 4, cudaMemcpyDeviceToHost, s));
    };
    cudaGraphExec_t exec = nullptr;
    for (auto& g : R.graphs)
        if (g.first == key) exec = g.second;
    // a launch shape is captured the second time it is seen: one-off shapes (a join table built
    // for one query) run directly instead of paying for a capture and evicting graphs that recur
    bool seen = exec != nullptr;
    if (!exec) {
        for (auto& k : R.seen) seen = seen || k == key;
        if (!seen) {
            if (R.seen.size() >= 64) R.seen.erase(R.seen.begin());
            R.seen.push_back(key);
        }
    }
    if (exec) {
        R.hits++;
    } else if (seen) {
        const auto t_cap = std::chrono::steady_clock::now();
        cudaGraph_t graph;
        CK(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
        enqueue();
        CK(cudaStreamEndCapture(s, &graph));
        cudaError_t e = cudaGraphInstantiate(&exec, graph, 0);
        cudaGraphDestroy(graph);
        CK(e);
        if (R.graphs.size() >= 32) {  // keep the most recent shapes
            cudaGraphExecDestroy(R.graphs.front().second);
            R.graphs.erase(R.graphs.begin());
        }
        R.graphs.emplace_back(key, exec);
        R.builds++;
        ctx->add_profile("graph_capture",
                         std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_cap).count());
    }
    {
        KernelTimer kt(ctx, s, "pipeline_aggregate");
        if (exec) CK(cudaGraphLaunch(exec, s));
        else enqueue();
        kt.stop();
    }
    ctx->count_launch(reset ? 2 : 1);
    if (jit) ctx->add_profile("jit_launch", 0);
    CK(cudaStreamSynchronize(s));
    check_device_error(ctx, *R.ew->h);
    if (reset) h->final_groups = -1;
    uint64_t count = *R.host_count;
    lk.unlock();
    if (count) {
        DevBuf ovf(ctx, count * w * 4, nullptr);
        CK(cudaMemcpyAsync(ovf.get(), R.ovf.get(), count * w * 4, cudaMemcpyDeviceToDevice, s));
        h->resume_overflow(L, count, ovf, w, s, R.count.get<unsigned long long>(), R.host_count, *R.ew);
    }
    API_END
}

int ml_gpu_hashagg_graph_stats(ml_hashagg* h, uint64_t* built, uint64_t* replayed) {
    API_BEGIN
    REQUIRE(h, "null sink");
    if (built) *built = h->run.builds;
    if (replayed) *replayed = h->run.hits;
    API_END
}

int ml_gpu_hashagg_combine(ml_hashagg_local* local) {
    API_BEGIN
    if (local) {  // every local sink updates the one device state: combine only waits
        local->sink->ctx->set_current();
        CK(cudaStreamSynchronize(local->s));
        delete local;
    }
    API_END
}

// Sink::finalize -> final_batches (aggregate/hash.rs:307-314)
}  // extern "C"

// The output batch of the sink's current groups (Sink::finalize's final values,
// accumulator.rs:500-594): one row per group, key columns then one column per aggregate.
std::unique_ptr<ml_batch> hashagg_emit(ml_hashagg* h, cudaStream_t s) {
    Ctx* ctx = h->ctx;
    uint32_t ng = 1;
    DevBuf gids;  // output row -> group id (GROUP BY the join key: the non-empty build rows)
    if (h->group_probe >= 0) {
        int64_t n = h->gid_cap;
        int nb = select_blocks(n);
        DevBuf bits(ctx, std::max<size_t>((size_t)(n + 31) / 32 * 4, 4), nullptr);
        DevBuf counts(ctx, std::max<size_t>((size_t)nb * 4, 4), nullptr);
        const uint32_t* member = h->dense_groups ? h->pipe.probes[h->group_probe].jt->dense.get<uint32_t>() : nullptr;
        launch_group_flags(h->acc.get<uint64_t>(), h->stride, n, member, bits.get<uint32_t>(), counts.get<uint32_t>(), s);
        DevBuf offs;
        uint64_t total = scan_counts(ctx, counts.get<uint32_t>(), nb, offs, s);
        gids = DevBuf(ctx, std::max<size_t>(total * 4, 4), nullptr);
        launch_index_write(n, bits.get<uint32_t>(), offs.get<uint64_t>(), gids.get<uint32_t>(), s);
        ctx->count_launch(2);
        ng = (uint32_t)total;
    } else if (!h->ungrouped) {
        CK(cudaMemcpy(&ng, h->ngroups.get(), 4, cudaMemcpyDeviceToHost));
        ng = std::min(ng, h->gid_cap);
    }
    h->final_groups = ng;
    auto b = std::make_unique<ml_batch>();
    b->ctx = ctx;
    b->nrows = ng;
    b->res = std::make_unique<Reservation>(ctx, "HashAggregate(output)");
    FinalArgs F{};
    F.ngroups = ng;
    F.gid_cap = h->gid_cap;
    F.nkeys = h->ungrouped || h->group_probe >= 0 ? 0 : h->keys.nkeys;
    F.nagg = (int)h->aggs.size();
    F.ungrouped = h->ungrouped;
    F.stride = h->stride;
    F.gkeys = h->gkeys.get<uint64_t>();
    F.gnull = h->gnull.get<uint32_t>();
    F.acc = h->acc.get<uint64_t>();
    F.gids = gids.get<uint32_t>();
    size_t vbytes = std::max<size_t>((size_t)(ng + 63) / 64 * 8, 8);
    std::vector<std::unique_ptr<DevColumn>> keycols, aggcols;
    std::vector<DevBuf> id_bufs(std::max(F.nkeys, 0));
    for (int k = 0; k < F.nkeys; k++) {
        F.f[k] = h->keys.f[k];
        auto d = std::make_unique<DevColumn>();
        d->dtype = h->dec[k].type;
        d->kind = CK_FIXED;
        d->n = ng;
        d->validity = DevBuf(ctx, vbytes, b->res.get());
        CK(cudaMemsetAsync(d->validity.get(), 0, vbytes, s));
        if (h->dec[k].str_kind) {
            id_bufs[k] = DevBuf(ctx, std::max<size_t>((size_t)ng * 4, 4), nullptr);
            F.key_out[k] = id_bufs[k].get();
        } else {
            d->data = DevBuf(ctx, std::max<size_t>((size_t)ng * width_of(d->dtype), 8), b->res.get());
            F.key_out[k] = d->data.get();
        }
        F.key_valid[k] = d->validity.get<uint32_t>();
        keycols.push_back(std::move(d));
    }
    if (h->dense_groups) {  // the key is the index position plus the index's smallest key
        const ml_join_table* jt = h->pipe.probes[h->group_probe].jt;
        auto d = std::make_unique<DevColumn>();
        d->dtype = jt->key_types[0];
        d->kind = CK_FIXED;
        d->n = ng;
        d->data = DevBuf(ctx, std::max<size_t>((size_t)ng * width_of(d->dtype), 8), b->res.get());
        launch_dense_keys(gids.get<uint32_t>(), ng, jt->dmin, d->dtype, d->data.get(), s);
        ctx->count_launch();
        keycols.push_back(std::move(d));
    } else if (h->group_probe >= 0) {  // the keys are the build keys of the matched rows
        const ml_batch& bb = h->pipe.probes[h->group_probe].jt->batch;
        for (int c : h->group_build_cols) keycols.push_back(gather_column(ctx, *bb.cols[c], gids.get<uint32_t>(), ng, s, b->res.get()));
    }
    for (int k = 0; k < F.nagg; k++) {
        const AggState& a = h->aggs[k];
        AggDev& ad = F.aggs[k];
        ad.kind = a.kind;
        ad.func = a.func;
        ad.off = a.off;
        ad.vcnt = a.vcnt_on && a.kind != A_AVG ? a.vcnt.get<uint64_t>() : nullptr;
        F.out_type[k] = a.out_type;
        auto d = std::make_unique<DevColumn>();
        d->dtype = a.out_type;
        d->kind = CK_FIXED;
        d->n = ng;
        d->data = DevBuf(ctx, std::max<size_t>((size_t)ng * width_of(a.out_type), 8), b->res.get());
        d->validity = DevBuf(ctx, vbytes, b->res.get());
        CK(cudaMemsetAsync(d->validity.get(), 0, vbytes, s));
        F.agg_out[k] = d->data.get();
        F.agg_valid[k] = d->validity.get<uint32_t>();
        aggcols.push_back(std::move(d));
    }
    launch_agg_final(F, s);
    ctx->count_launch();
    CK(cudaStreamSynchronize(s));
    // global string ids (dictionary keys, string MIN/MAX) become the strings on the host
    auto strings_of_ids = [&](DevColumn& c, const void* id_dev) {
        std::vector<uint32_t> ids(ng);
        if (ng) CK(cudaMemcpy(ids.data(), id_dev, (size_t)ng * 4, cudaMemcpyDeviceToHost));
        std::vector<uint64_t> valid((ng + 63) / 64 + 1, 0);
        if (ng) CK(cudaMemcpy(valid.data(), c.validity.get(), (size_t)(ng + 63) / 64 * 8, cudaMemcpyDeviceToHost));
        std::vector<uint32_t> off(ng + 1, 0);
        std::string bytes;
        {
            std::lock_guard<std::mutex> g(h->pipe.intern.mu);
            for (uint32_t g2 = 0; g2 < ng; g2++) {
                bool v = (valid[g2 / 64] >> (g2 % 64)) & 1;
                if (v) bytes += h->pipe.intern.strs.at(ids[g2]);
                off[g2 + 1] = (uint32_t)bytes.size();
            }
        }
        c.kind = CK_UTF8;
        c.offsets = DevBuf(ctx, (size_t)(ng + 1) * 4, b->res.get());
        c.data = DevBuf(ctx, std::max<size_t>(bytes.size(), 1), b->res.get());
        h2d_now(c.offsets.get(), off.data(), (size_t)(ng + 1) * 4);
        h2d_now(c.data.get(), bytes.data(), bytes.size());
    };
    for (int k = 0; k < F.nagg; k++)
        if (h->aggs[k].out_type == ML_TYPE_UTF8) {
            DevBuf ids = std::move(aggcols[k]->data);
            strings_of_ids(*aggcols[k], ids.get());
        }
    // string keys: dictionary ids decode on the host, build-side ids gather on the device
    for (int k = 0; k < F.nkeys; k++) {
        const KeyDecode& d = h->dec[k];
        if (!d.str_kind) continue;
        auto& kc = keycols[k];
        kc->kind = CK_UTF8;
        if (d.str_kind == 1) {
            strings_of_ids(*kc, id_bufs[k].get());
        } else {
            const DevColumn& src = *h->pipe.probes[d.build].jt->batch.cols[d.build_col];
            DevColumn tmp;
            gather_utf8(ctx, src.optr(), (const uint8_t*)src.dptr(), id_bufs[k].get<uint32_t>(), ng, tmp, s, b->res.get());
            kc->offsets = std::move(tmp.offsets);
            kc->data = std::move(tmp.data);
            CK(cudaStreamSynchronize(s));
        }
    }
    for (auto& c : keycols) b->cols.push_back(std::move(c));
    for (auto& c : aggcols) b->cols.push_back(std::move(c));
    CK(cudaStreamSynchronize(s));
    return b;
}

extern "C" {

int ml_gpu_hashagg_finalize(ml_hashagg* h, ml_batch** out) {
    API_BEGIN
    HostTimer host_timer_(h ? h->ctx : nullptr, "host:hashagg_finalize");
    REQUIRE(h && out, "null argument");
    Ctx* ctx = h->ctx;
    ctx->set_current();
    std::unique_lock<std::shared_mutex> lk(h->rw);
    h->streams.sync();
    if (h->run.s) CK(cudaStreamSynchronize(h->run.s));
    cudaStream_t s = h->streams.own();
    if (!h->spill_events) {
        *out = hashagg_emit(h, s).release();
        return ML_OK;
    }
    // Spilled: the groups in HBM go to host memory too, then one spill partition at a time is
    // merged back into the (empty) table and emitted (aggregate/hash.rs:369-425), so the table
    // holds about 1/16 of the groups at once.
    ErrWord ew(ctx);
    h->spill_state(s, ew);
    // finished partitions wait in host memory: HBM holds one partition's table, then the output
    std::vector<HostBatch> parts;
    std::vector<int> types;
    uint64_t total_groups = 0;
    h->release_table();  // the table the spills emptied: the partitions start small
    for (int p = 0; p < kSpillParts; p++) {
        if (h->spills[p].empty()) continue;
        h->grow(1024, s, ew);
        for (const auto& c : h->spills[p]) {
            CK(cudaMemcpyAsync(ew.h, h->ngroups.get(), 4, cudaMemcpyDeviceToHost, s));
            CK(cudaStreamSynchronize(s));
            const uint64_t need = (uint64_t)std::min(*ew.h, h->gid_cap) + c.n;  // every row may be new
            if (need > h->gid_cap) h->grow(need, s, ew);
            h->merge_spilled(c, s, ew);
        }
        std::vector<ml_hashagg::SpillChunk>().swap(h->spills[p]);
        auto part = hashagg_emit(h, s);
        total_groups += part->nrows;
        if (types.empty())
            for (auto& c : part->cols) types.push_back(c->dtype);
        parts.push_back(batch_to_host(*part, s));
        part.reset();
        h->release_table();
    }
    h->final_groups = (int64_t)total_groups;
    if (parts.empty()) {
        *out = hashagg_emit(h, s).release();
        return ML_OK;
    }
    auto res = std::make_unique<Reservation>(ctx, "HashAggregate(output)");
    auto all = host_batches_to_device(ctx, parts, types, res.get());
    all->res = std::move(res);
    *out = all.release();
    API_END
}

int ml_gpu_hashagg_stats(ml_hashagg* h, int64_t* groups, int64_t* capacity, int64_t* resizes) {
    API_BEGIN
    REQUIRE(h, "null sink");
    h->ctx->set_current();
    if (groups) {
        uint32_t ng = 1;
        if (h->group_probe >= 0 || h->spill_events) {
            REQUIRE(h->final_groups >= 0, "the number of groups is known after finalize");
            ng = (uint32_t)h->final_groups;
        } else if (!h->ungrouped) {
            CK(cudaMemcpy(&ng, h->ngroups.get(), 4, cudaMemcpyDeviceToHost));
            ng = std::min(ng, h->gid_cap);
        }
        *groups = ng;
    }
    if (capacity) *capacity = (int64_t)h->cap;
    if (resizes) *resizes = h->resizes;
    API_END
}

int ml_gpu_hashagg_spill_stats(ml_hashagg* h, int64_t* spills, int64_t* spilled_groups) {
    API_BEGIN
    REQUIRE(h, "null sink");
    if (spills) *spills = (int64_t)h->spill_events;
    if (spilled_groups) *spilled_groups = (int64_t)h->spilled_groups;
    API_END
}

int ml_gpu_hashagg_destroy(ml_hashagg* h) {
    API_BEGIN
    if (h) {
        h->ctx->set_current();
        h->streams.sync();
        if (h->run.s) CK(cudaStreamSynchronize(h->run.s));
        delete h;
    }
    API_END
}

}  // extern "C"

// =====================================================================================================
// SortSink with a limit (sort.rs:145-267)
// =====================================================================================================
struct ml_topn {
    Ctx* ctx;
    std::unique_ptr<Reservation> res;  // declared before everything charged to it
    Pipeline pipe;
    std::vector<Prog> out_progs;
    std::vector<SortKeySpec> keys;
    std::vector<int> out_types;
    int64_t limit;  // < 0: ORDER BY without a limit
    std::mutex mu;
    std::vector<std::unique_ptr<ml_batch>> cands;
    SinkStreams streams;
    ml_topn(Ctx* c) : ctx(c), pipe(c), streams(c) {}
    // No limit, or more rows than the per-warp top-N keeps: the morsels are kept as they come
    // and sorted once at finalize (the radix sort), as SortLocal keeps its batches (sort.rs:239-249).
    bool full_sort() const { return limit < 0 || limit > kMaxTopN; }
};
struct ml_topn_local {
    ml_topn* sink;
    cudaStream_t s;
    Staging st;
    std::unique_ptr<ErrWord> ew;
    ml_topn_local(ml_topn* k) : sink(k), s(k->ctx->new_stream()), st(k->ctx), ew(new ErrWord(k->ctx)) {
        sink->streams.add(s);
    }
    ~ml_topn_local() {
        sink->streams.remove(s);
        sink->ctx->free_stream(s);
    }
};

extern "C" {

int ml_gpu_topn_create(ml_ctx* ctx, const ml_pipe_op* prologue, int32_t nprologue, const int32_t* input_types, int32_t ninput,
                       const ml_sort_key* keys, int32_t nkeys, int64_t limit, ml_topn** out) {
    API_BEGIN
    HostTimer host_timer_(ctx, "host:topn_create");
    REQUIRE(ctx && out && keys && nkeys > 0, "bad arguments");
    REQUIRE(nkeys <= kMaxKeys, "too many sort keys");

    ctx->set_current();
    auto t = std::make_unique<ml_topn>(ctx);
    t->pipe.build(prologue, nprologue, input_types, ninput);
    for (auto& r : t->pipe.out) t->out_types.push_back(r.dtype);
    t->out_progs = compile_outputs(t->pipe);
    t->pipe.upload();
    for (int k = 0; k < nkeys; k++)
        t->keys.push_back(SortKeySpec{parse_expr(keys[k].expr), keys[k].expr.dtype, keys[k].asc != 0, keys[k].nulls_first != 0});
    t->limit = limit;
    t->res = std::make_unique<Reservation>(ctx, "Sort");
    *out = t.release();
    API_END
}

int ml_gpu_topn_local_create(ml_topn* sink, ml_topn_local** out) {
    API_BEGIN
    REQUIRE(sink && out, "null argument");
    sink->ctx->set_current();
    *out = new ml_topn_local(sink);
    API_END
}

// SortLocal::sink + truncate: keep only this batch's best `limit` rows
int ml_gpu_topn_sink(ml_topn_local* local, const ml_column* cols, int32_t ncols, int64_t nrows, const uint32_t* sel, int64_t nsel) {
    API_BEGIN
    HostTimer host_timer_(local ? local->sink->ctx : nullptr, "host:topn_sink");
    REQUIRE(local, "null local sink");
    ml_topn* t = local->sink;
    Ctx* ctx = t->ctx;
    ctx->set_current();
    check_sel_bounds(sel, nsel, nrows);
    DevBuf sel_hold;
    const uint32_t* dsel = device_sel(ctx, sel, nsel, sel_hold, local->s);
    Pipeline::Launch L;
    t->pipe.prepare(L, cols, ncols, nrows, dsel, nsel, local->s, local->st, nullptr);
    if (t->full_sort()) {  // keep the morsel (an owned copy, charged to the sort)
        auto r = std::make_unique<Reservation>(ctx, "Sort");
        auto part = materialize(ctx, t->pipe, t->out_progs, L, local->s, r.get(), *local->ew, false);
        part->res = std::move(r);
        CK(cudaStreamSynchronize(local->s));
        std::lock_guard<std::mutex> g(t->mu);
        t->cands.push_back(std::move(part));
        return ML_OK;
    }
    auto part = materialize(ctx, t->pipe, t->out_progs, L, local->s, nullptr, *local->ew, true);
    auto r = std::make_unique<Reservation>(ctx, "Sort(candidates)");
    auto best = topn_batch(ctx, *part, t->keys, t->limit, local->s, r.get());
    best->res = std::move(r);  // the candidates own their memory: one of them may be the output
    std::lock_guard<std::mutex> g(t->mu);
    t->cands.push_back(std::move(best));
    API_END
}

int ml_gpu_topn_combine(ml_topn_local* local) {
    API_BEGIN
    if (local) {
        local->sink->ctx->set_current();
        CK(cudaStreamSynchronize(local->s));
        delete local;
    }
    API_END
}

int ml_gpu_topn_finalize(ml_topn* t, ml_batch** out) {
    API_BEGIN
    HostTimer host_timer_(t ? t->ctx : nullptr, "host:topn_finalize");
    REQUIRE(t && out, "null argument");
    Ctx* ctx = t->ctx;
    ctx->set_current();
    t->streams.sync();
    std::vector<std::unique_ptr<ml_batch>> cands;
    {
        std::lock_guard<std::mutex> g(t->mu);
        cands = std::move(t->cands);
    }
    cudaStream_t s = t->streams.own();
    if (cands.size() == 1 && !t->full_sort()) {  // one local sink: its candidates are the sorted top N already
        *out = cands[0].release();
        return ML_OK;
    }
    std::unique_ptr<ml_batch> all;
    if (cands.empty()) {
        all = std::make_unique<ml_batch>();
        all->ctx = ctx;
        for (int ty : t->out_types) {
            auto d = std::make_unique<DevColumn>();
            d->dtype = ty;
            d->kind = ty == ML_TYPE_UTF8 ? CK_UTF8 : CK_FIXED;
            d->n = 0;
            if (d->kind == CK_UTF8) {
                d->offsets = DevBuf(ctx, 4, nullptr);
                CK(cudaMemsetAsync(d->offsets.get(), 0, 4, s));
            }
            d->data = DevBuf(ctx, 8, nullptr);
            all->cols.push_back(std::move(d));
        }
    } else {
        all = concat_batches(ctx, cands, t->out_types, s, nullptr);
    }
    auto res = std::make_unique<Reservation>(ctx, "Sort(output)");
    auto best = t->full_sort() ? sort_batch(ctx, *all, t->keys, t->limit, s, res.get())
                               : topn_batch(ctx, *all, t->keys, t->limit, s, res.get());
    best->res = std::move(res);
    *out = best.release();
    API_END
}

int ml_gpu_topn_destroy(ml_topn* t) {
    API_BEGIN
    if (t) {
        t->ctx->set_current();
        t->streams.sync();
        delete t;
    }
    API_END
}

}  // extern "C"

// =====================================================================================================
// Prepared query (executor.rs:270-288 runs a physical plan's pipelines in dependency order)
// =====================================================================================================
// One plan over device-resident tables: join builds, then one hash aggregate whose prologue
// probes them, then optionally a top-N of the aggregate's output.  The first run goes through
// the sink calls and records what depends on the data (the dense-index range or hash capacity,
// the group table, the result's row count); later runs replay every pipeline as one CUDA graph
// over the same buffers: the build columns are copied in and the join index rebuilt, the group
// table reset and the fused kernel run, the groups emitted, the top-N taken and read back.
// Kernels check each recorded choice against the run's data (guard bits below); a failed check
// makes the run return ML_ERR_STALE_PLAN.
namespace {
constexpr uint32_t kGuardRange = 1;      // a build key outside the dense index
constexpr uint32_t kGuardDups = 2;       // duplicate build keys appeared or went away
constexpr uint32_t kGuardOverflow = 4;   // the group table overflowed
constexpr uint32_t kGuardRows = 8;       // the group count no longer gives the planned result rows
constexpr uint32_t kGuardTopRows = 16;   // a top-k list came back short
}  // namespace

struct ml_query {
    Ctx* ctx;
    std::unique_ptr<Reservation> res;  // declared before everything charged to it
    struct Build {
        ml_join_build* sink = nullptr;
        std::vector<ml_column> cols;
        int64_t nrows = 0;
        ml_join_table* jt = nullptr;
        std::unique_ptr<Pipeline> kp;  // hash-table form: the key programs over the build batch
        Pipeline::Launch LA;
        KeyLayout L{};
        void* jit = nullptr;
    };
    std::vector<std::unique_ptr<Build>> builds;
    ml_hashagg* agg = nullptr;
    std::vector<ml_column> agg_cols;
    int64_t agg_rows = 0;
    std::vector<SortKeySpec> keys;
    int64_t limit = 0;
    bool topn = false;
    // ---- the replay ----
    cudaStream_t s = nullptr;
    std::unique_ptr<Staging> st;
    std::unique_ptr<ErrWord> ew;
    cudaGraphExec_t exec = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;  // around the fused aggregate kernel
    std::string why_not;                     // why runs take the sink calls ("" while replaying)
    int64_t runs = 0, replays = 0;
    int nkernels = 0;   // kernels one replay launches
    int64_t cap = 0;    // output rows the aggregate can emit (its group ids)
    int64_t k = 0;      // result rows of the top-N
    Pipeline::Launch AL;
    AggArgs A{};
    void* jit = nullptr;
    int grid = 0, smem = 0;
    DevBuf tables, ovf, count, guard, ng, gids, bits, counts, offs, scratch, tbuf;
    std::vector<std::unique_ptr<DevColumn>> outcols, rescols;
    FinalArgs F{};
    uint32_t* hguard = nullptr;  // pinned readbacks
    uint64_t* hng = nullptr;
    std::vector<void*> hres;     // pinned copies of the top-N result: per column values, validity
    explicit ml_query(Ctx* c) : ctx(c) {}
    ~ml_query() {
        if (exec) cudaGraphExecDestroy(exec);
        for (void* p : hres)
            if (p) cudaFreeHost(p);
        if (e0) cudaEventDestroy(e0);
        if (e1) cudaEventDestroy(e1);
        if (hguard) ctx->release_slot(hguard);
        if (hng) ctx->release_slot(hng);
        if (s) {
            cudaStreamSynchronize(s);
            ctx->free_stream(s);
        }
    }
};

namespace {
void check_status(int st) {
    if (st != ML_OK) raise(st, last_error());
}

// Why a plan cannot be replayed as recorded ("" when it can).
std::string query_replay_blocker(ml_query* q) {
    for (auto& b : q->builds) {
        const ml_join_build* j = b->sink;
        if (j->pipe.nstages > 0) return "a join build pipeline filters its rows";
        for (const ColRef& r : j->pipe.out)
            if (r.kind != 0) return "a join build pipeline computes a column";
        for (auto& c : b->jt->batch.cols)
            if (c->kind != CK_FIXED) return "a join build side holds strings";
        for (auto& c : b->cols)
            if (c.location != ML_LOC_DEVICE) return "a join build source is not device-resident";
    }
    ml_hashagg* h = q->agg;
    if (!h) return "no aggregate";
    for (auto& c : q->agg_cols)
        if (c.location != ML_LOC_DEVICE) return "the aggregate's source is not device-resident";
    if (h->spill_events) return "the aggregate spilled";
    for (auto& d : h->dec)
        if (d.str_kind) return "a string group key";
    if (h->str_minmax) return "a string MIN or MAX";
    for (auto& kk : q->keys)
        if (kk.expr.kind != ML_EXPR_COLUMN) return "a computed sort key";
    if (q->topn && h->keys.nkeys + (int)h->aggs.size() + (int)h->group_build_cols.size() + 1 > kMaxResultCols)
        return "more than 16 output columns";
    if (q->topn && (q->limit <= 0 || q->limit > kTopNWarpMax)) return "a limit above 32";
    return "";
}
}  // namespace

namespace {
// Every launch of one run of the plan, on q->s; captured once into the query's graph.
void query_enqueue(ml_query* q) {
    cudaStream_t s = q->s;
    int nk = 0;
    uint32_t* guard = q->guard.get<uint32_t>();
    CK(cudaMemsetAsync(guard, 0, 4, s));
    CK(cudaMemsetAsync(q->ew->d.get(), 0, 4, s));
    // 1. join builds (build_table, join.rs:160-203): the build columns, then the index
    for (auto& bp : q->builds) {
        ml_query::Build& b = *bp;
        ml_join_table* jt = b.jt;
        const int64_t n = jt->batch.nrows;
        const ml_join_build* j = b.sink;
        for (size_t c = 0; c < j->pipe.out.size(); c++) {
            const ml_column& src = b.cols[j->pipe.out[c].index];
            DevColumn& dst = *jt->batch.cols[c];
            const size_t bytes = (size_t)n * width_of(dst.dtype);
            if (bytes) CK(cudaMemcpyAsync(dst.data.get(), src.data, bytes, cudaMemcpyDeviceToDevice, s));
            if (dst.validity && src.validity && n)
                CK(cudaMemcpyAsync(dst.validity.get(), src.validity, (size_t)(n + 63) / 64 * 8, cudaMemcpyDeviceToDevice, s));
        }
        CK(cudaMemsetAsync(jt->next.get(), 0xFF, std::max<size_t>((size_t)n * 4, 4), s));
        CK(cudaMemsetAsync(jt->dup.get(), 0, 8, s));
        if (jt->dense) {
            const DevColumn& kc = *jt->batch.cols[jt->key_cols[0]];
            CK(cudaMemsetAsync(jt->dense.get(), 0xFF, jt->drange * 4, s));
            launch_dense_insert(kc.dptr(), kc.dtype, kc.vptr(), n, jt->dmin, jt->drange, jt->dense.get<uint32_t>(),
                                jt->next.get<uint32_t>(), jt->dup.get<uint32_t>(), guard, s);
            nk++;
            if (jt->member) {
                launch_dense_bits(jt->dense.get<uint32_t>(), jt->drange, jt->member.get<uint32_t>(), s);
                nk++;
            }
        } else {
            CK(cudaMemsetAsync(jt->slots.get(), 0, jt->cap * 8 * (jt->nwords == 1 ? 2 : 4), s));
            if (n) {
                TableView tv = jt->view();
                uint32_t* next = jt->next.get<uint32_t>();
                uint32_t* dup = jt->dup.get<uint32_t>();
                int64_t nn = n;
                if (b.jit) {
                    void* args[] = {&b.LA.P, &b.L, &tv, &next, &dup, &nn};
                    jit_launch(b.jit, pipeline_grid(n), kPipelineThreads, 0, s, args);
                } else {
                    launch_join_insert(b.LA.P, b.L, tv, next, dup, n, s);
                }
                nk++;
            }
        }
        // the probes were specialized on whether build keys repeat
        launch_plan_check(jt->dup.get(), 4, 0, jt->has_dups ? 1 : 0, kGuardDups, guard, s);
        nk++;
    }
    // 2. the aggregate (HashAggLocal::sink): reset the groups, the fused kernel
    ml_hashagg* h = q->agg;
    CK(cudaMemsetAsync(h->ngroups.get(), 0, 16, s));
    if (h->cap) CK(cudaMemsetAsync(h->slots.get(), 0, h->cap * 8 * (h->keys.nwords == 1 ? 2 : 4), s));
    launch_acc_init(q->A, 0, h->gid_cap, s);
    nk++;
    CK(cudaMemsetAsync(q->count.get(), 0, 8, s));
    CK(cudaEventRecordWithFlags(q->e0, s, cudaEventRecordExternal));
    if (q->AL.P.n) {
        if (q->jit) {
            void* args[] = {&q->AL.P, &q->A};
            jit_launch(q->jit, q->grid, kPipelineThreads, q->smem, s, args);
        } else {
            launch_agg(q->AL.P, q->A, q->smem, s);
        }
        nk++;
    }
    CK(cudaEventRecordWithFlags(q->e1, s, cudaEventRecordExternal));
    launch_plan_check(q->count.get(), 8, 0, 0, kGuardOverflow, guard, s);
    nk++;
    // 3. the groups' final values (accumulator.rs:500-594) at the table's capacity; the number
    //    of groups stays on the device (q->F.ng64)
    const uint64_t* ngd = q->F.ng64;
    for (auto& c : q->outcols)
        if (c->validity) CK(cudaMemsetAsync(c->validity.get(), 0, c->validity.bytes(), s));
    if (h->group_probe >= 0) {  // GROUP BY the join key: the groups are matched build rows
        const ml_join_table* jt = h->pipe.probes[h->group_probe].jt;
        const int nb = select_blocks(q->cap);
        launch_group_flags(h->acc.get<uint64_t>(), h->stride, q->cap, h->dense_groups ? jt->dense.get<uint32_t>() : nullptr,
                           q->bits.get<uint32_t>(), q->counts.get<uint32_t>(), s);
        launch_scan_u32(q->counts.get<uint32_t>(), q->offs.get<uint64_t>(), nb, q->scratch.get<uint64_t>(), s);
        nk += 4;
        if (!h->dense_groups)  // the key gathers read every position: past the groups, build row 0
            CK(cudaMemsetAsync(q->gids.get(), 0, (size_t)q->cap * 4, s));
        launch_index_write(q->cap, q->bits.get<uint32_t>(), q->offs.get<uint64_t>(), q->gids.get<uint32_t>(), s);
        nk++;
        if (h->dense_groups) {
            DevColumn& kc = *q->outcols[0];
            launch_dense_keys(q->gids.get<uint32_t>(), q->cap, jt->dmin, kc.dtype, kc.data.get(), s, ngd);
            nk++;
        } else {
            for (size_t i = 0; i < h->group_build_cols.size(); i++) {
                const DevColumn& src = *jt->batch.cols[h->group_build_cols[i]];
                DevColumn& dst = *q->outcols[i];
                launch_gather_fixed(src.dptr(), width_of(src.dtype), q->gids.get<uint32_t>(), q->cap, dst.data.get(), s);
                nk++;
                if (src.vptr()) {
                    launch_gather_valid(src.vptr(), q->gids.get<uint32_t>(), q->cap, dst.validity.get<uint32_t>(), s);
                    nk++;
                }
            }
        }
    } else if (!h->ungrouped) {
        launch_plan_count(h->ngroups.get<uint32_t>(), h->gid_cap, q->ng.get<uint64_t>(), s);
        nk++;
    }
    launch_agg_final(q->F, s);
    nk++;
    // 4. the top-N (sort.rs:117-122) and the result's read-back
    if (q->topn) {
        const int nb = topn_warp_blocks(q->cap);
        const size_t rows_b = ((size_t)nb * q->k * 4 + 15) & ~(size_t)15, cand_b = (size_t)nb * q->k * topn_entry_bytes();
        uint8_t* base = q->tbuf.get<uint8_t>();
        uint32_t* rows = nullptr;
        SortDev S{};
        S.nkeys = (int)q->keys.size();
        for (size_t i = 0; i < q->keys.size(); i++) {
            const DevColumn& c = *q->outcols[q->keys[i].expr.index];
            DCol& d = S.cols[i];
            d.dt = c.dtype;
            d.kind = CK_FIXED;
            d.data = c.dptr();
            d.valid = c.vptr();
            d.n = q->cap;
            S.asc[i] = q->keys[i].asc;
            S.nulls_first[i] = q->keys[i].nulls_first;
        }
        if (nb > 1) {
            unsigned int* done = (unsigned int*)(base + rows_b + cand_b);
            rows = (uint32_t*)(done + 4);
            CK(cudaMemsetAsync(done, 0, 16, s));
            nk += launch_topn_warp(S, q->cap, (int)q->k, nb, (uint32_t*)base, base + rows_b, done, rows, s, ngd);
        } else {
            rows = (uint32_t*)base;
            nk += launch_topn_warp(S, q->cap, (int)q->k, nb, rows, nullptr, nullptr, nullptr, s, ngd);
        }
        // as many groups as the planned result needs (at least `limit`, or exactly the planned
        // rows), the row ids in range, then the result's columns
        ResultCols G{};
        G.ncols = (int)q->outcols.size();
        for (size_t c = 0; c < q->outcols.size(); c++) {
            const DevColumn& src = *q->outcols[c];
            DevColumn& dst = *q->rescols[c];
            G.width[c] = width_of(src.dtype);
            G.src[c] = src.dptr();
            G.sval[c] = src.vptr();
            G.dst[c] = dst.data.get();
            G.dval[c] = src.vptr() ? dst.validity.get<uint32_t>() : nullptr;
            if (dst.validity) CK(cudaMemsetAsync(dst.validity.get(), 0, dst.validity.bytes(), s));
        }
        launch_plan_result(rows, (int)q->k, ngd, q->cap, q->k < q->limit, kGuardTopRows, kGuardRows, guard, G, s);
        nk += 1;
        for (size_t c = 0; c < q->outcols.size(); c++) {
            DevColumn& dst = *q->rescols[c];
            // the rows to host memory too (ml_gpu_query_run_host)
            CK(cudaMemcpyAsync(q->hres[2 * c], dst.data.get(), (size_t)q->k * width_of(dst.dtype), cudaMemcpyDeviceToHost, s));
            if (dst.validity)
                CK(cudaMemcpyAsync(q->hres[2 * c + 1], dst.validity.get(), (size_t)(q->k + 63) / 64 * 8,
                                   cudaMemcpyDeviceToHost, s));
        }
    } else {
        CK(cudaMemcpyAsync(q->hng, ngd, 8, cudaMemcpyDeviceToHost, s));
    }
    CK(cudaMemcpyAsync(q->hguard, guard, 4, cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(q->ew->h, q->ew->d.get(), 4, cudaMemcpyDeviceToHost, s));
    q->nkernels = nk;
}
}  // namespace

namespace {
// Set up the replay of a planned query (buffers at the recorded sizes, the aggregate's launch
// as ml_gpu_hashagg_run_resident sets it up) and capture it into one CUDA graph.
void query_capture(ml_query* q) {
    Ctx* ctx = q->ctx;
    ml_hashagg* h = q->agg;
    cudaStream_t s = q->s;
    // hash-table builds: the key programs over the build batch (as ml_gpu_join_build_finalize)
    for (auto& bp : q->builds) {
        ml_query::Build& b = *bp;
        ml_join_table* jt = b.jt;
        if (jt->dense || jt->batch.nrows == 0) continue;
        const ml_join_build* j = b.sink;
        b.kp = std::make_unique<Pipeline>(ctx);
        b.kp->build(nullptr, 0, j->out_types.data(), (int)j->out_types.size());
        b.L = b.kp->key_layout(j->keys.exprs.data(), (int)j->keys.exprs.size(), b.kp->out, false, nullptr);
        b.kp->upload();
        auto views = device_views(jt->batch);
        b.kp->prepare(b.LA, views.data(), (int)views.size(), jt->batch.nrows, nullptr, 0, s, *q->st, nullptr);
        b.LA.P.err = q->ew->d.get<uint32_t>();
        b.jit = jit_join_insert_kernel(ctx, *b.kp, b.LA.P, b.L);
    }
    // the aggregate's launch
    q->tables = DevBuf(ctx, 64 << 10, nullptr);
    h->pipe.prepare(q->AL, q->agg_cols.data(), (int)q->agg_cols.size(), q->agg_rows, nullptr, 0, s, *q->st, nullptr,
                    q->tables.get<uint8_t>(), q->tables.bytes());
    const int w = 1 + (int)h->pipe.probes.size();
    const bool can_overflow = !h->ungrouped && h->group_probe < 0;
    const uint64_t ovf_cap = can_overflow ? std::max<uint64_t>((uint64_t)q->AL.P.n, 1024) : 0;
    q->ovf = DevBuf(ctx, std::max<uint64_t>(ovf_cap * w * 4, 16), nullptr);
    q->count = DevBuf(ctx, 16, nullptr);
    q->AL.P.err = q->ew->d.get<uint32_t>();
    q->AL.P.head_probe = h->group_probe;
    if (h->dense_groups) q->AL.P.probes[h->group_probe].late = 1;
    semi_probes(ctx, q->AL.P, h->pipe, h->group_probe, s);
    q->A = h->args(q->count.get<unsigned long long>(), q->ovf.get<uint32_t>(), ovf_cap);
    h->direct_slots(q->A, q->AL);
    q->jit = jit_agg_kernel(ctx, h->pipe, q->AL.P, q->A);
    if (!q->jit) q->A.priv_groups = 0, q->A.dslots = 0;
    q->smem = agg_smem_bytes(q->A);
    q->grid = q->jit ? agg_grid(q->jit, q->AL.P, q->smem) : pipeline_grid(q->AL.P.n);
    // the groups' output at the table's capacity
    q->cap = h->ungrouped ? 1 : (int64_t)h->gid_cap;
    const size_t vbytes = std::max<size_t>((size_t)(q->cap + 63) / 64 * 8, 8);
    q->ng = DevBuf(ctx, 8, nullptr);
    FinalArgs& F = q->F;
    F = FinalArgs{};
    F.ngroups = (uint32_t)q->cap;
    F.gid_cap = h->gid_cap;
    F.nkeys = h->ungrouped || h->group_probe >= 0 ? 0 : h->keys.nkeys;
    F.nagg = (int)h->aggs.size();
    F.ungrouped = h->ungrouped;
    F.stride = h->stride;
    F.gkeys = h->gkeys.get<uint64_t>();
    F.gnull = h->gnull.get<uint32_t>();
    F.acc = h->acc.get<uint64_t>();
    F.ng64 = q->ng.get<uint64_t>();
    if (h->ungrouped) {
        const uint64_t one = 1;
        h2d_now(q->ng.get(), &one, 8);
    }
    auto column = [&](int dtype, bool valid) {
        auto d = std::make_unique<DevColumn>();
        d->dtype = dtype;
        d->kind = CK_FIXED;
        d->n = q->cap;
        d->data = DevBuf(ctx, std::max<size_t>((size_t)q->cap * width_of(dtype), 8), q->res.get());
        if (valid) d->validity = DevBuf(ctx, vbytes, q->res.get());
        return d;
    };
    q->outcols.clear();
    for (int k = 0; k < F.nkeys; k++) {
        F.f[k] = h->keys.f[k];
        q->outcols.push_back(column(h->dec[k].type, true));
        F.key_out[k] = q->outcols.back()->data.get();
        F.key_valid[k] = q->outcols.back()->validity.get<uint32_t>();
    }
    if (h->group_probe >= 0) {
        const ml_join_table* jt = h->pipe.probes[h->group_probe].jt;
        const int nb = select_blocks(q->cap);
        q->bits = DevBuf(ctx, std::max<size_t>((size_t)(q->cap + 31) / 32 * 4, 4), nullptr);
        q->counts = DevBuf(ctx, std::max<size_t>((size_t)nb * 4, 4), nullptr);
        q->offs = DevBuf(ctx, (size_t)(nb + 1) * 8, nullptr);
        q->scratch = DevBuf(ctx, std::max<size_t>(scan_scratch_words(nb) * 8, 8), nullptr);
        q->gids = DevBuf(ctx, std::max<size_t>((size_t)q->cap * 4, 4), q->res.get());
        F.gids = q->gids.get<uint32_t>();
        F.ng64 = q->offs.get<uint64_t>() + nb;  // the scan's total: the groups with rows
        if (h->dense_groups) {  // the key is the index position plus the index's smallest key
            q->outcols.push_back(column(jt->key_types[0], false));
        } else {  // the build keys of the matched rows
            for (int c : h->group_build_cols) {
                const DevColumn& src = *jt->batch.cols[c];
                q->outcols.push_back(column(src.dtype, src.vptr() != nullptr));
            }
        }
    }
    for (int k = 0; k < F.nagg; k++) {
        const AggState& a = h->aggs[k];
        AggDev& ad = F.aggs[k];
        ad.kind = a.kind;
        ad.func = a.func;
        ad.off = a.off;
        ad.vcnt = a.vcnt_on && a.kind != A_AVG ? a.vcnt.get<uint64_t>() : nullptr;
        F.out_type[k] = a.out_type;
        q->outcols.push_back(column(a.out_type, true));
        F.agg_out[k] = q->outcols.back()->data.get();
        F.agg_valid[k] = q->outcols.back()->validity.get<uint32_t>();
    }
    // the top-N's scratch and result
    q->rescols.clear();
    if (q->topn) {
        for (auto& kk : q->keys) {
            const int c = (int)kk.expr.index;
            if (c < 0 || c >= (int)q->outcols.size() || q->outcols[c]->dtype != kk.type)
                raise(ML_ERR_INVALID, "a sort key does not name an output column of its type");
        }
        const int nb = topn_warp_blocks(q->cap);
        const size_t rows_b = ((size_t)nb * q->k * 4 + 15) & ~(size_t)15, cand_b = (size_t)nb * q->k * topn_entry_bytes();
        q->tbuf = DevBuf(ctx, rows_b + cand_b + 16 + (size_t)q->k * 4, nullptr);
        for (auto& c : q->outcols) {
            auto d = std::make_unique<DevColumn>();
            d->dtype = c->dtype;
            d->kind = CK_FIXED;
            d->n = q->k;
            d->data = DevBuf(ctx, std::max<size_t>((size_t)q->k * width_of(c->dtype), 8), q->res.get());
            if (c->validity) d->validity = DevBuf(ctx, std::max<size_t>((size_t)(q->k + 63) / 64 * 8, 8), q->res.get());
            void* hv = nullptr;
            void* hb = nullptr;
            CK(cudaMallocHost(&hv, std::max<size_t>((size_t)q->k * width_of(c->dtype), 8)));
            q->hres.push_back(hv);
            if (c->validity) CK(cudaMallocHost(&hb, std::max<size_t>((size_t)(q->k + 63) / 64 * 8, 8)));
            q->hres.push_back(hb);
            q->rescols.push_back(std::move(d));
        }
    }
    q->guard = DevBuf(ctx, 8, nullptr);
    CK(cudaEventCreate(&q->e0));
    CK(cudaEventCreate(&q->e1));
    CK(cudaStreamSynchronize(s));  // the launch's tables and programs are on the device
    cudaGraph_t g = nullptr;
    CK(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    try {
        query_enqueue(q);
    } catch (...) {
        cudaStreamEndCapture(s, &g);
        if (g) cudaGraphDestroy(g);
        throw;
    }
    CK(cudaStreamEndCapture(s, &g));
    cudaError_t e = cudaGraphInstantiate(&q->exec, g, 0);
    cudaGraphDestroy(g);
    CK(e);
}

// The first run: every pipeline through the sink calls; records the result's row count.
std::unique_ptr<ml_batch> query_plan_run(ml_query* q) {
    Ctx* ctx = q->ctx;
    ml_hashagg* h = q->agg;
    ml_hashagg_local* local = nullptr;
    check_status(ml_gpu_hashagg_local_create(h, &local));
    int st = ml_gpu_hashagg_sink(local, q->agg_cols.data(), (int32_t)q->agg_cols.size(), q->agg_rows, nullptr, 0);
    const int st2 = ml_gpu_hashagg_combine(local);
    check_status(st);
    check_status(st2);
    ml_batch* raw = nullptr;
    check_status(ml_gpu_hashagg_finalize(h, &raw));
    std::unique_ptr<ml_batch> groups(raw);
    if (!q->topn) return groups;
    auto res = std::make_unique<Reservation>(ctx, "Query(output)");
    auto best = topn_batch(ctx, *groups, q->keys, q->limit, q->s, res.get());
    best->res = std::move(res);
    q->k = best->nrows;
    return best;
}

void query_launch(ml_query* q) {
    CK(cudaGraphLaunch(q->exec, q->s));
    q->ctx->count_launch(q->nkernels);
    if (q->jit) q->ctx->add_profile("jit_launch", 0);
}

// After a replay's stream work: the checks' verdict, device errors, the kernel's time.
void query_finish(ml_query* q) {
    Ctx* ctx = q->ctx;
    if (const uint32_t g = *q->hguard) {
        cudaGraphExecDestroy(q->exec);
        q->exec = nullptr;
        q->why_not = "stale";
        raise(ML_ERR_STALE_PLAN, std::string("the data no longer fits the prepared plan:") +
                                     (g & kGuardRange ? " a build key outside the dense index" : "") +
                                     (g & kGuardDups ? " build-key duplicates changed" : "") +
                                     (g & kGuardOverflow ? " the group table overflowed" : "") +
                                     (g & (kGuardRows | kGuardTopRows) ? " the group count changed the result rows" : ""));
    }
    check_device_error(ctx, *q->ew->h);
    if (ctx->profiling()) {
        float ms = 0;
        if (cudaEventElapsedTime(&ms, q->e0, q->e1) == cudaSuccess) ctx->add_profile("pipeline_aggregate", ms);
        else (void)cudaGetLastError();
    }
    q->replays++;
}

// A replay: one graph launch, then the result out of the graph's buffers.
std::unique_ptr<ml_batch> query_replay(ml_query* q) {
    Ctx* ctx = q->ctx;
    cudaStream_t s = q->s;
    query_launch(q);
    auto out = std::make_unique<ml_batch>();
    out->ctx = ctx;
    out->res = std::make_unique<Reservation>(ctx, "Query(output)");
    if (q->topn) {
        out->nrows = q->k;
        for (auto& c : q->rescols) out->cols.push_back(copy_column(ctx, *c, s, out->res.get()));
        CK(cudaStreamSynchronize(s));
    } else {
        CK(cudaStreamSynchronize(s));
        const int64_t n = *q->hguard ? 0 : (int64_t)*q->hng;
        out->nrows = n;
        for (auto& c : q->outcols) {
            DevColumn v;
            v.dtype = c->dtype;
            v.kind = CK_FIXED;
            v.n = n;
            v.data_p = c->dptr();
            v.valid_p = c->vptr();
            out->cols.push_back(copy_column(ctx, v, s, out->res.get()));
        }
        CK(cudaStreamSynchronize(s));
    }
    query_finish(q);
    return out;
}
}  // namespace

extern "C" {

int ml_gpu_query_create(ml_ctx* ctx, ml_query** out) {
    API_BEGIN
    REQUIRE(ctx && out, "null argument");
    ctx->set_current();
    auto q = std::make_unique<ml_query>(ctx);
    q->res = std::make_unique<Reservation>(ctx, "Query");
    q->s = ctx->new_stream();
    q->st = std::make_unique<Staging>(ctx);
    q->ew = std::make_unique<ErrWord>(ctx);
    q->hguard = (uint32_t*)ctx->pinned_slot();
    q->hng = (uint64_t*)ctx->pinned_slot();
    *out = q.release();
    API_END
}

// The build pipeline runs now, through the sink calls (JoinBuildSink, join.rs:72-242).
int ml_gpu_query_add_build(ml_query* q, ml_join_build* sink, const ml_column* cols, int32_t ncols, int64_t nrows,
                           ml_join_table** table) {
    API_BEGIN
    REQUIRE(q && sink && table && (cols || ncols == 0) && nrows >= 0, "bad arguments");
    REQUIRE(!q->agg, "join builds come before the aggregate");
    REQUIRE(!sink->table, "the join build sink is already finalized");
    q->ctx->set_current();
    auto b = std::make_unique<ml_query::Build>();
    b->sink = sink;
    b->cols.assign(cols, cols + ncols);
    b->nrows = nrows;
    ml_join_build_local* local = nullptr;
    check_status(ml_gpu_join_build_local_create(sink, &local));
    const int st = ml_gpu_join_build_sink(local, cols, ncols, nrows, nullptr, 0);
    const int st2 = ml_gpu_join_build_combine(local);
    check_status(st);
    check_status(st2);
    check_status(ml_gpu_join_build_finalize(sink, &b->jt));
    *table = b->jt;
    q->builds.push_back(std::move(b));
    API_END
}

int ml_gpu_query_set_aggregate(ml_query* q, ml_hashagg* sink, const ml_column* cols, int32_t ncols, int64_t nrows) {
    API_BEGIN
    REQUIRE(q && sink && (cols || ncols == 0) && nrows >= 0, "bad arguments");
    REQUIRE(!q->agg, "the query has its aggregate");
    q->agg = sink;
    q->agg_cols.assign(cols, cols + ncols);
    q->agg_rows = nrows;
    API_END
}

int ml_gpu_query_set_topn(ml_query* q, const ml_sort_key* keys, int32_t nkeys, int64_t limit) {
    API_BEGIN
    REQUIRE(q && keys && nkeys > 0 && nkeys <= kMaxKeys, "bad arguments");
    REQUIRE(limit > 0, "the top-N of a query needs a limit");
    REQUIRE(!q->runs, "the query has run");
    q->keys.clear();
    for (int k = 0; k < nkeys; k++)
        q->keys.push_back(SortKeySpec{parse_expr(keys[k].expr), keys[k].expr.dtype, keys[k].asc != 0, keys[k].nulls_first != 0});
    q->limit = limit;
    q->topn = true;
    API_END
}

int ml_gpu_query_run(ml_query* q, ml_batch** out) {
    API_BEGIN
    HostTimer host_timer_(q ? q->ctx : nullptr, "host:query_run");
    REQUIRE(q && out, "null argument");
    REQUIRE(q->agg, "the query has no aggregate");
    q->ctx->set_current();
    if (q->runs == 0) {
        q->runs++;
        auto r = query_plan_run(q);
        q->why_not = query_replay_blocker(q);
        if (q->why_not.empty() && q->topn && q->k == 0) q->why_not = "an empty result";
        if (q->why_not.empty()) query_capture(q);
        *out = r.release();
        return ML_OK;
    }
    if (!q->exec) {
        if (q->why_not == "stale") raise(ML_ERR_STALE_PLAN, "the data no longer fits the prepared plan");
        raise(ML_ERR_UNSUPPORTED, "this plan runs once (" + q->why_not + "); create it again to run it again");
    }
    q->runs++;
    *out = query_replay(q).release();
    API_END
}

int ml_gpu_query_run_host(ml_query* q, int64_t* nrows) {
    API_BEGIN
    HostTimer host_timer_(q ? q->ctx : nullptr, "host:query_run");
    REQUIRE(q && nrows, "null argument");
    if (!q->exec || !q->topn) {
        if (q->why_not == "stale") raise(ML_ERR_STALE_PLAN, "the data no longer fits the prepared plan");
        raise(ML_ERR_UNSUPPORTED, "ml_gpu_query_run_host replays a planned top-N query (plan it with ml_gpu_query_run)");
    }
    q->ctx->set_current();
    q->runs++;
    query_launch(q);
    CK(cudaStreamSynchronize(q->s));
    query_finish(q);
    *nrows = q->k;
    API_END
}

int ml_gpu_query_result(const ml_query* q, int32_t col, void* values, uint64_t* validity, int32_t* has_validity) {
    API_BEGIN
    REQUIRE(q && values, "null argument");
    REQUIRE(q->topn && !q->hres.empty(), "no host result: the query has no replayed top-N");
    REQUIRE(col >= 0 && (size_t)col < q->rescols.size(), "column out of range");
    const DevColumn& c = *q->rescols[col];
    memcpy(values, q->hres[2 * col], (size_t)q->k * width_of(c.dtype));
    const void* hv = q->hres[2 * col + 1];
    if (has_validity) *has_validity = hv != nullptr;
    if (hv && validity) memcpy(validity, hv, (size_t)(q->k + 63) / 64 * 8);
    API_END
}

int ml_gpu_query_stats(const ml_query* q, int64_t* runs, int64_t* replays, int32_t* kernels, char* why, int32_t why_cap) {
    API_BEGIN
    REQUIRE(q, "null query");
    if (runs) *runs = q->runs;
    if (replays) *replays = q->replays;
    if (kernels) *kernels = q->nkernels;
    if (why && why_cap > 0) {
        const std::string& w = q->why_not;
        const size_t n = std::min<size_t>(w.size(), (size_t)why_cap - 1);
        memcpy(why, w.data(), n);
        why[n] = 0;
    }
    API_END
}

int ml_gpu_query_destroy(ml_query* q) {
    API_BEGIN
    if (q) {
        q->ctx->set_current();
        delete q;
    }
    API_END
}

}  // extern "C"
