// Host runtime: errors, HBM budget pool, caching allocator, staging, device
// columns, scalar semantics and the expression compiler.
#include "ml_runtime.hpp"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>

namespace mlg {

// ---- errors ----------------------------------------------------------------------------------
namespace {
thread_local std::string t_err;
thread_local BudgetInfo t_budget;
}  // namespace
void set_last_error(const std::string& m) { t_err = m; }
void set_budget_error(const BudgetInfo& b) { t_budget = b; }
const char* last_error() { return t_err.c_str(); }
const BudgetInfo& last_budget() { return t_budget; }
[[noreturn]] void raise(int code, const std::string& msg) { throw MlError(code, msg); }
void check_cuda(cudaError_t e, const char* what) {
    if (e != cudaSuccess) raise(ML_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

// ---- memory pool (memory.rs:58-77) ------------------------------------------------------------
bool MemoryPool::try_grow(uint64_t bytes, uint64_t* observed) {
    uint64_t cur = used.load(std::memory_order_relaxed);
    for (;;) {
        uint64_t nw = cur + bytes;
        if (nw < cur || nw > limit) {
            *observed = cur;
            return false;
        }
        if (used.compare_exchange_weak(cur, nw, std::memory_order_relaxed)) {
            uint64_t p = peak.load(std::memory_order_relaxed);
            while (nw > p && !peak.compare_exchange_weak(p, nw)) {
            }
            return true;
        }
    }
}

void Reservation::try_grow(uint64_t bytes) {
    uint64_t observed = 0;
    if (!ctx_->pool.try_grow(bytes, &observed)) {
        BudgetInfo b{name_, bytes, observed, ctx_->pool.limit};
        set_budget_error(b);
        raise(ML_ERR_BUDGET, "Resources exhausted: " + name_ + " requested " + std::to_string(bytes) + " bytes, " +
                                 std::to_string(observed) + " of " + std::to_string(ctx_->pool.limit) + " used");
    }
    size_ += bytes;
}
void Reservation::shrink(uint64_t bytes) {
    uint64_t b = std::min(bytes, size_);
    ctx_->pool.shrink(b);
    size_ -= b;
}

// ---- device buffers --------------------------------------------------------------------------------
DevBuf::DevBuf(Ctx* ctx, size_t bytes, Reservation* res) : ctx_(ctx), bytes_(bytes), res_(res) {
    if (res_) res_->try_grow(bytes);
    try {
        ptr_ = ctx->dalloc(bytes, &cap_);
    } catch (...) {
        if (res_) res_->shrink(bytes);
        throw;
    }
}
DevBuf& DevBuf::operator=(DevBuf&& o) noexcept {
    if (this != &o) {
        release();
        ctx_ = o.ctx_;
        ptr_ = o.ptr_;
        bytes_ = o.bytes_;
        cap_ = o.cap_;
        res_ = o.res_;
        o.ptr_ = nullptr;
        o.res_ = nullptr;
        o.bytes_ = o.cap_ = 0;
    }
    return *this;
}
void DevBuf::release() {
    if (ptr_) {
        ctx_->dfree(ptr_, cap_);
        if (res_) res_->shrink(bytes_);
    }
    ptr_ = nullptr;
    res_ = nullptr;
    bytes_ = cap_ = 0;
}

// ---- context -----------------------------------------------------------------------------------------
Ctx::Ctx(int dev, uint64_t budget, uint32_t fl) : device(dev), flags(fl), pool(budget) {
    int n = 0;
    CK(cudaGetDeviceCount(&n));
    if (dev < 0 || dev >= n) raise(ML_ERR_INVALID, "device " + std::to_string(dev) + " out of range");
    CK(cudaSetDevice(dev));
    CK(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
}
Ctx::~Ctx() {
    cudaSetDevice(device);
    cudaDeviceSynchronize();
    for (auto& t : timings_) {
        cudaEventDestroy(t.a);
        cudaEventDestroy(t.b);
    }
    for (auto e : events_) cudaEventDestroy(e);
    for (auto s : streams_) cudaStreamDestroy(s);
    for (auto s : idle_streams_) cudaStreamDestroy(s);
    if (stream) cudaStreamDestroy(stream);
    for (auto& kv : free_) cudaFree(kv.second);
    for (void* p : slabs_) cudaFreeHost(p);
}
void* Ctx::pinned_slot() {
    std::lock_guard<std::mutex> g(mu_);
    if (free_slots_.empty()) {
        const size_t slab = 64 * 1024;
        void* p = nullptr;
        CK(cudaHostAlloc(&p, slab, cudaHostAllocDefault));
        slabs_.push_back(p);
        for (size_t o = 0; o < slab; o += 64) free_slots_.push_back((uint8_t*)p + o);
    }
    void* p = free_slots_.back();
    free_slots_.pop_back();
    return p;
}
void Ctx::release_slot(void* p) {
    std::lock_guard<std::mutex> g(mu_);
    free_slots_.push_back(p);
}
void Ctx::set_current() const { CK(cudaSetDevice(device)); }

static size_t round_cap(size_t b) {
    if (b < 256) return 256;
    if (b <= (1ull << 20)) {
        size_t p = 256;
        while (p < b) p <<= 1;
        return p;
    }
    // above 1 MiB, eight size classes per power of two (at most 12.5 % unused): buffers whose
    // sizes vary from query to query (tables presized from an estimate) still reuse cached
    // blocks, where exact sizes each needed a cudaMalloc, and cudaMalloc may stall the device
    size_t p = 1ull << 20;
    while (p * 2 <= b) p <<= 1;
    const size_t step = p / 8;
    return (b + step - 1) / step * step;
}
void* Ctx::dalloc(size_t bytes, size_t* cap) {
    size_t c = round_cap(bytes);
    {
        std::lock_guard<std::mutex> g(mu_);
        auto it = free_.lower_bound(c);
        if (it != free_.end() && it->first <= c + c / 8) {
            void* p = it->second;
            *cap = it->first;
            cached_bytes_ -= it->first;
            free_.erase(it);
            return p;
        }
    }
    void* p = nullptr;
    auto t0 = std::chrono::steady_clock::now();
    cudaError_t e = cudaMalloc(&p, c);
    add_profile("device_alloc", std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count());
    if (e != cudaSuccess) {
        cudaGetLastError();
        std::lock_guard<std::mutex> g(mu_);  // release the cache and retry once
        for (auto& kv : free_) cudaFree(kv.second);
        free_.clear();
        cached_bytes_ = 0;
        e = cudaMalloc(&p, c);
        if (e != cudaSuccess) {
            cudaGetLastError();
            raise(ML_ERR_CUDA, "cudaMalloc(" + std::to_string(c) + "): " + cudaGetErrorString(e));
        }
    }
    *cap = c;
    return p;
}
void Ctx::dfree(void* p, size_t cap) {
    std::lock_guard<std::mutex> g(mu_);
    free_.emplace(cap, p);
    cached_bytes_ += cap;
}
void* Ctx::halloc(size_t bytes) {
    void* p = nullptr;
    auto t0 = std::chrono::steady_clock::now();
    CK(cudaHostAlloc(&p, bytes, cudaHostAllocDefault));
    add_profile("pinned_alloc", std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count());
    return p;
}
void Ctx::hfree(void* p) { cudaFreeHost(p); }
cudaStream_t Ctx::new_stream() {  // streams are pooled: local sinks come and go per pipeline
    {
        std::lock_guard<std::mutex> g(mu_);
        if (!idle_streams_.empty()) {
            cudaStream_t s = idle_streams_.back();
            idle_streams_.pop_back();
            streams_.push_back(s);
            return s;
        }
    }
    cudaStream_t s;
    CK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    std::lock_guard<std::mutex> g(mu_);
    streams_.push_back(s);
    return s;
}
void Ctx::free_stream(cudaStream_t s) {
    cudaStreamSynchronize(s);
    std::lock_guard<std::mutex> g(mu_);
    auto it = std::find(streams_.begin(), streams_.end(), s);
    if (it != streams_.end()) {
        streams_.erase(it);
        idle_streams_.push_back(s);
    }
}
void Ctx::sync_all() {
    set_current();
    CK(cudaStreamSynchronize(stream));
    std::vector<cudaStream_t> ss;
    {
        std::lock_guard<std::mutex> g(mu_);
        ss = streams_;
    }
    for (auto s : ss) CK(cudaStreamSynchronize(s));
}

void Ctx::add_profile(const std::string& k, double ms) {
    std::lock_guard<std::mutex> g(prof_mu_);
    auto& e = prof_[k];
    e.first++;
    e.second += ms;
}
void Ctx::read_profile(const std::string& k, uint64_t* n, double* ms, bool reset) {
    std::lock_guard<std::mutex> g(prof_mu_);
    set_current();
    drain_timings(0);
    auto& e = prof_[k];
    if (n) *n = e.first;
    if (ms) *ms = e.second;
    if (reset) e = {0, 0.0};
}

KernelTimer::KernelTimer(Ctx* ctx, cudaStream_t s, const char* name) : ctx_(ctx), s_(s), name_(name) {
    if (!ctx_->profiling()) return;
    a_ = ctx_->get_event();
    b_ = ctx_->get_event();
    cudaEventRecord(a_, s_);
}
void KernelTimer::stop() {
    if (b_) cudaEventRecord(b_, s_);
}
KernelTimer::~KernelTimer() {
    if (a_) ctx_->add_timing(name_, a_, b_);
}

cudaEvent_t Ctx::get_event() {
    {
        std::lock_guard<std::mutex> g(prof_mu_);
        if (!events_.empty()) {
            cudaEvent_t e = events_.back();
            events_.pop_back();
            return e;
        }
    }
    cudaEvent_t e = nullptr;
    CK(cudaEventCreate(&e));
    return e;
}
void Ctx::add_timing(const char* name, cudaEvent_t a, cudaEvent_t b) {
    std::lock_guard<std::mutex> g(prof_mu_);
    timings_.push_back(Timing{name, a, b});
    if (timings_.size() > 4096) drain_timings(1024);
}
void Ctx::drain_timings(size_t keep) {  // collect all but the newest `keep` timings
    size_t n = timings_.size() > keep ? timings_.size() - keep : 0;
    for (size_t i = 0; i < n; i++) {
        Timing& t = timings_[i];
        float ms = 0;
        if (cudaEventSynchronize(t.b) == cudaSuccess && cudaEventElapsedTime(&ms, t.a, t.b) == cudaSuccess) {
            auto& e = prof_[t.name];
            e.first++;
            e.second += ms;
        }
        cudaGetLastError();
        events_.push_back(t.a);
        events_.push_back(t.b);
    }
    timings_.erase(timings_.begin(), timings_.begin() + n);
}

Staging::~Staging() {
    if (p_) ctx_->hfree(p_);
}
void* Staging::get(size_t bytes) {
    if (bytes > cap_) {
        if (p_) ctx_->hfree(p_);
        cap_ = std::max(bytes, cap_ * 2);
        p_ = ctx_->halloc(cap_);
    }
    return p_;
}

void h2d_now(void* dst, const void* src, size_t bytes) {
    if (!bytes) return;
    CK(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, cudaStreamPerThread));
    CK(cudaStreamSynchronize(cudaStreamPerThread));
}

int width_of(int dt) {
    switch (dt) {
        case ML_TYPE_BOOL: return 1;
        case ML_TYPE_INT32:
        case ML_TYPE_DATE: return 4;
        default: return 8;
    }
}

int64_t DevColumn::str_bytes_host() const {
    if (kind != CK_UTF8 || n == 0) return 0;
    uint32_t last = 0, first = 0;
    CK(cudaMemcpy(&last, optr() + n, 4, cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(&first, optr(), 4, cudaMemcpyDeviceToHost));
    return (int64_t)last - first;
}

static bool is_pinned(const void* p) {
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeHost;
}

static void h2d(void* dst, const void* src, size_t bytes, cudaStream_t s, Staging& st) {
    if (!bytes) return;
    if (is_pinned(src)) {
        CK(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s));
        return;
    }
    // pageable: copy through the pinned staging buffer in chunks (the stream is
    // synchronized before the staging buffer is refilled)
    const size_t chunk = 64ull << 20;
    for (size_t o = 0; o < bytes; o += chunk) {
        size_t k = std::min(chunk, bytes - o);
        void* p = st.get(chunk < bytes ? chunk : bytes);
        CK(cudaStreamSynchronize(s));
        memcpy(p, (const uint8_t*)src + o, k);
        CK(cudaMemcpyAsync((uint8_t*)dst + o, p, k, cudaMemcpyHostToDevice, s));
    }
}

std::unique_ptr<DevColumn> stage_column(Ctx* ctx, const ml_column& c, int64_t nrows, cudaStream_t s, Staging& st,
                                        Reservation* res) {
    auto d = std::make_unique<DevColumn>();
    d->dtype = c.dtype;
    d->n = nrows;
    if (c.dtype < 0 || c.dtype > ML_TYPE_UTF8) raise(ML_ERR_INVALID, "bad column type");
    if (c.len != nrows) raise(ML_ERR_INVALID, "column length " + std::to_string(c.len) + " != batch rows " + std::to_string(nrows));
    bool dict = c.dtype == ML_TYPE_UTF8 && c.encoding == ML_ENC_DICT;
    bool utf8 = c.dtype == ML_TYPE_UTF8 && !dict;
    d->kind = dict ? CK_DICT : (utf8 ? CK_UTF8 : CK_FIXED);
    if (nrows > 0 && !c.data) raise(ML_ERR_INVALID, "column without data");
    if (utf8 && !c.offsets) raise(ML_ERR_INVALID, "UTF8 column without offsets");
    if (dict) {
        if (c.dict_len < 0 || (c.dict_len > 0 && (!c.dict_offsets || !c.dict_data)))
            raise(ML_ERR_INVALID, "dictionary column without dictionary");
        auto hd = std::make_shared<HostDict>();
        hd->off.assign(c.dict_offsets, c.dict_offsets + c.dict_len + 1);
        if (c.dict_len >= 0 && c.dict_offsets) hd->bytes.assign(c.dict_data, c.dict_data + c.dict_offsets[c.dict_len]);
        for (size_t i = 0; i + 1 < hd->off.size(); i++)
            if (hd->off[i] > hd->off[i + 1]) raise(ML_ERR_INVALID, "corrupt dictionary offsets");
        d->dict = hd;
    }
    size_t vwords = (size_t)(nrows + 63) / 64;
    if (c.location == ML_LOC_DEVICE) {
        d->data_p = c.data;
        d->off_p = c.offsets;
        d->valid_p = c.validity;
        return d;
    }
    // host memory: copy
    if (utf8) {
        uint32_t first = c.offsets[0], last = c.offsets[nrows];
        if (last < first) raise(ML_ERR_INVALID, "corrupt string offsets");
        d->offsets = DevBuf(ctx, (size_t)(nrows + 1) * 4, res);
        h2d(d->offsets.get(), c.offsets, (size_t)(nrows + 1) * 4, s, st);
        d->data = DevBuf(ctx, std::max<size_t>(last, 1), res);
        h2d(d->data.get(), c.data, last, s, st);
    } else {
        size_t w = dict ? 4 : (size_t)width_of(c.dtype);
        d->data = DevBuf(ctx, std::max<size_t>((size_t)nrows * w, 1), res);
        h2d(d->data.get(), c.data, (size_t)nrows * w, s, st);
    }
    if (c.validity) {
        d->validity = DevBuf(ctx, std::max<size_t>(vwords * 8, 8), res);
        h2d(d->validity.get(), c.validity, vwords * 8, s, st);
    }
    return d;
}

// ---- scalars (scalar.rs:82-133, scalar_ops.rs:12-140) ---------------------------------------------
static std::string fmt_f64(double v) {
    if (std::isnan(v)) return "NaN";
    if (std::isinf(v)) return v > 0 ? "inf" : "-inf";
    char buf[64];
    snprintf(buf, sizeof buf, "%.17g", v);
    double back = strtod(buf, nullptr);
    for (int p = 1; p <= 17; p++) {  // shortest round-trip digits
        snprintf(buf, sizeof buf, "%.*g", p, v);
        if (strtod(buf, nullptr) == back) break;
    }
    return buf;
}
static std::string to_string(const HScalar& s) {
    switch (s.kind) {
        case -1: return "NULL";
        case ML_TYPE_BOOL: return s.i ? "true" : "false";
        case ML_TYPE_FLOAT64: return fmt_f64(s.f);
        case ML_TYPE_UTF8: return s.s;
        default: return std::to_string(s.i);
    }
}
static int32_t days_from_civil(int32_t y, uint32_t m, uint32_t d) {
    y = m <= 2 ? y - 1 : y;
    int32_t era = (y >= 0 ? y : y - 399) / 400;
    uint32_t yoe = (uint32_t)(y - era * 400);
    uint32_t mp = (m + 9) % 12;
    uint32_t doy = (153 * mp + 2) / 5 + d - 1;
    uint32_t doe = yoe * 365 + yoe / 4 - yoe / 100 + doy;
    return era * 146097 + (int32_t)doe - 719468;
}
std::optional<int32_t> parse_date(const std::string& in) {
    int y, m, d;
    char tail;
    if (sscanf(in.c_str(), " %d-%d-%d %c", &y, &m, &d, &tail) != 3) return std::nullopt;
    static const int dim[] = {31, 28, 31, 30, 31, 30, 31, 31, 30, 31, 30, 31};
    if (m < 1 || m > 12 || d < 1) return std::nullopt;
    bool leap = (y % 4 == 0 && y % 100 != 0) || y % 400 == 0;
    int md = dim[m - 1] + (m == 2 && leap);
    if (d > md) return std::nullopt;
    return days_from_civil(y, (uint32_t)m, (uint32_t)d);
}
static int64_t sat_i64(double f) {
    if (std::isnan(f)) return 0;
    if (f >= 9223372036854775808.0) return INT64_MAX;
    if (f <= -9223372036854775808.0) return INT64_MIN;
    return (int64_t)f;
}
static bool is_int(int k) { return k == ML_TYPE_INT32 || k == ML_TYPE_INT64 || k == ML_TYPE_DATE; }

HScalar scalar_cast(const HScalar& s, int to) {
    if (s.is_null()) return s;
    auto err = [&]() { raise(ML_ERR_INVALID, "cannot cast " + to_string(s) + " to type " + std::to_string(to)); };
    HScalar o;
    o.kind = to;
    switch (to) {
        case ML_TYPE_BOOL:
            if (s.kind != ML_TYPE_BOOL) err();
            return s;
        case ML_TYPE_INT32: {
            int64_t v;
            if (s.kind == ML_TYPE_FLOAT64) v = sat_i64(s.f);
            else if (is_int(s.kind)) v = s.i;
            else err();
            if (v < INT32_MIN || v > INT32_MAX) err();
            o.i = v;
            return o;
        }
        case ML_TYPE_INT64:
            if (s.kind == ML_TYPE_FLOAT64) o.i = sat_i64(s.f);
            else if (is_int(s.kind)) o.i = s.i;
            else err();
            return o;
        case ML_TYPE_FLOAT64:
            if (s.kind == ML_TYPE_FLOAT64) return s;
            if (!is_int(s.kind)) err();
            o.f = (double)s.i;
            return o;
        case ML_TYPE_DATE:
            if (s.kind == ML_TYPE_DATE) return s;
            if (s.kind == ML_TYPE_UTF8) {
                auto d = parse_date(s.s);
                if (!d) err();
                o.i = *d;
                return o;
            }
            err();
        case ML_TYPE_UTF8:
            o.s = to_string(s);
            return o;
    }
    raise(ML_ERR_INVALID, "cannot cast to type " + std::to_string(to));
}

std::optional<int> scalar_compare(const HScalar& a, const HScalar& b) {
    auto c3 = [](auto x, auto y) { return x < y ? -1 : (x > y ? 1 : 0); };
    if (a.is_null() || b.is_null()) return std::nullopt;
    if (a.kind == ML_TYPE_BOOL && b.kind == ML_TYPE_BOOL) return c3(a.i, b.i);
    if (a.kind == ML_TYPE_UTF8 && b.kind == ML_TYPE_UTF8) return c3(a.s.compare(b.s), 0);
    if (a.kind == ML_TYPE_DATE && b.kind == ML_TYPE_DATE) return c3(a.i, b.i);
    bool ia = a.kind == ML_TYPE_INT32 || a.kind == ML_TYPE_INT64, ib = b.kind == ML_TYPE_INT32 || b.kind == ML_TYPE_INT64;
    if (ia && ib) return c3(a.i, b.i);
    auto f = [](const HScalar& x) -> std::optional<double> {
        if (x.kind == ML_TYPE_FLOAT64) return x.f;
        if (is_int(x.kind)) return (double)x.i;
        return std::nullopt;
    };
    auto x = f(a), y = f(b);
    if (!x || !y || std::isnan(*x) || std::isnan(*y)) return std::nullopt;
    return c3(*x, *y);
}

HScalar scalar_binary(int op, const HScalar& l, const HScalar& r) {
    auto as_bool = [](const HScalar& x) -> std::optional<bool> {
        if (x.kind == ML_TYPE_BOOL) return x.i != 0;
        return std::nullopt;
    };
    if (op == ML_BIN_AND || op == ML_BIN_OR) {
        auto a = as_bool(l), b = as_bool(r);
        if (op == ML_BIN_AND) {
            if ((a && !*a) || (b && !*b)) return HScalar::b(false);
            if (a && b) return HScalar::b(true);
            return HScalar();
        }
        if ((a && *a) || (b && *b)) return HScalar::b(true);
        if (a && b) return HScalar::b(false);
        return HScalar();
    }
    if (l.is_null() || r.is_null()) return HScalar();
    if (op >= ML_BIN_EQ) {
        auto o = scalar_compare(l, r);
        if (!o) raise(ML_ERR_INVALID, "cannot compare " + to_string(l) + " with " + to_string(r));
        int c = *o;
        switch (op) {
            case ML_BIN_EQ: return HScalar::b(c == 0);
            case ML_BIN_NOTEQ: return HScalar::b(c != 0);
            case ML_BIN_LT: return HScalar::b(c < 0);
            case ML_BIN_LTEQ: return HScalar::b(c <= 0);
            case ML_BIN_GT: return HScalar::b(c > 0);
            default: return HScalar::b(c >= 0);
        }
    }
    auto overflow = [&]() { raise(ML_ERR_INVALID, "overflow in " + to_string(l) + " op " + to_string(r)); };
    HScalar o;
    if (l.kind == ML_TYPE_DATE && (r.kind == ML_TYPE_INT32 || r.kind == ML_TYPE_INT64) &&
        (op == ML_BIN_ADD || op == ML_BIN_SUB)) {
        int64_t v = op == ML_BIN_ADD ? l.i + r.i : l.i - r.i;
        if (v < INT32_MIN || v > INT32_MAX) overflow();
        o.kind = ML_TYPE_DATE;
        o.i = v;
        return o;
    }
    if (l.kind == ML_TYPE_DATE && r.kind == ML_TYPE_DATE && op == ML_BIN_SUB) {
        o.kind = ML_TYPE_INT64;
        o.i = l.i - r.i;
        return o;
    }
    auto num = [&](const HScalar& x) -> double {
        if (x.kind == ML_TYPE_FLOAT64) return x.f;
        if (is_int(x.kind)) return (double)x.i;
        raise(ML_ERR_INVALID, to_string(x) + " is not numeric");
    };
    if (op == ML_BIN_DIV) {
        double a = num(l), b = num(r);
        if (b == 0.0) return HScalar();
        o.kind = ML_TYPE_FLOAT64;
        o.f = a / b;
        return o;
    }
    bool li = l.kind == ML_TYPE_INT32 || l.kind == ML_TYPE_INT64, ri = r.kind == ML_TYPE_INT32 || r.kind == ML_TYPE_INT64;
    if (li && ri) {
        int64_t a = l.i, b = r.i, v = 0;
        bool bad = false;
        switch (op) {
            case ML_BIN_ADD: bad = __builtin_add_overflow(a, b, &v); break;
            case ML_BIN_SUB: bad = __builtin_sub_overflow(a, b, &v); break;
            case ML_BIN_MUL: bad = __builtin_mul_overflow(a, b, &v); break;
            default:
                if (b == 0) raise(ML_ERR_INVALID, "modulo by zero");
                if (a == INT64_MIN && b == -1) bad = true;
                else v = a % b;
        }
        if (bad) overflow();
        o.kind = (l.kind == ML_TYPE_INT32 && r.kind == ML_TYPE_INT32 && v >= INT32_MIN && v <= INT32_MAX) ? ML_TYPE_INT32
                                                                                                        : ML_TYPE_INT64;
        o.i = v;
        return o;
    }
    double a = num(l), b = num(r);
    o.kind = ML_TYPE_FLOAT64;
    switch (op) {
        case ML_BIN_ADD: o.f = a + b; break;
        case ML_BIN_SUB: o.f = a - b; break;
        case ML_BIN_MUL: o.f = a * b; break;
        default: o.f = std::fmod(a, b); break;
    }
    return o;
}

uint64_t scalar_bits(const HScalar& s) {
    switch (s.kind) {
        case ML_TYPE_FLOAT64: {
            uint64_t b;
            memcpy(&b, &s.f, 8);
            return b;
        }
        case ML_TYPE_INT32:
        case ML_TYPE_DATE: return (uint64_t)(int64_t)(int32_t)s.i;
        case ML_TYPE_BOOL: return s.i ? 1 : 0;
        default: return (uint64_t)s.i;
    }
}

// ---- expressions -------------------------------------------------------------------------------------
static ExprNode parse_at(const ml_expr_node* nodes, int nn, int& pos, int depth) {
    if (pos >= nn) raise(ML_ERR_INVALID, "truncated expression");
    if (depth > 64) raise(ML_ERR_INVALID, "expression too deep");
    const ml_expr_node& n = nodes[pos++];
    ExprNode e;
    e.kind = n.kind;
    e.op = n.op;
    e.dtype = n.dtype;
    e.flag = n.flag;
    e.index = n.i64;
    if (n.kind < ML_EXPR_COLUMN || n.kind > ML_EXPR_CAST) raise(ML_ERR_INVALID, "bad expression kind");
    if (n.kind == ML_EXPR_LITERAL) {
        e.lit.kind = n.dtype == ML_TYPE_NULL ? -1 : n.dtype;
        if (n.dtype == ML_TYPE_FLOAT64) e.lit.f = n.f64;
        else if (n.dtype == ML_TYPE_UTF8) e.lit.s.assign(n.str ? n.str : "", n.str ? (size_t)n.str_len : 0);
        else if (n.dtype == ML_TYPE_INT32 || n.dtype == ML_TYPE_DATE) e.lit.i = (int32_t)n.i64;
        else if (n.dtype == ML_TYPE_BOOL) e.lit.i = n.i64 != 0;
        else e.lit.i = n.i64;
    }
    if (n.kind == ML_EXPR_LIKE) e.str.assign(n.str ? n.str : "", n.str ? (size_t)n.str_len : 0);
    if (n.nchild < 0 || n.nchild > 4096) raise(ML_ERR_INVALID, "bad child count");
    for (int k = 0; k < n.nchild; k++) e.kids.push_back(parse_at(nodes, nn, pos, depth + 1));
    return e;
}
ExprNode parse_expr(const ml_expr& e) {
    if (!e.nodes || e.nnodes <= 0) raise(ML_ERR_INVALID, "empty expression");
    int pos = 0;
    ExprNode r = parse_at(e.nodes, e.nnodes, pos, 0);
    if (pos != e.nnodes) raise(ML_ERR_INVALID, "trailing expression nodes");
    return r;
}

// like.rs:26-46
int like_shape(const std::string& p, std::string* inner) {
    bool us = p.find('_') != std::string::npos;
    auto none = [](const std::string& s) { return s.find('%') == std::string::npos; };
    size_t n = p.size();
    if (!us) {
        if (none(p)) { *inner = p; return LK_EXACT; }
        if (n >= 2 && p[0] == '%' && p[n - 1] == '%' && none(p.substr(1, n - 2))) { *inner = p.substr(1, n - 2); return LK_CONTAINS; }
        if (p[n - 1] == '%' && none(p.substr(0, n - 1))) { *inner = p.substr(0, n - 1); return LK_PREFIX; }
        if (p[0] == '%' && none(p.substr(1))) { *inner = p.substr(1); return LK_SUFFIX; }
    }
    *inner = p;
    return LK_GENERAL;
}
bool like_match_host(const std::string& s, const std::string& p, int shape) {
    switch (shape) {
        case LK_EXACT: return s == p;
        case LK_PREFIX: return s.size() >= p.size() && s.compare(0, p.size(), p) == 0;
        case LK_SUFFIX: return s.size() >= p.size() && s.compare(s.size() - p.size(), p.size(), p) == 0;
        case LK_CONTAINS: return p.empty() || s.find(p) != std::string::npos;
        default: {
            size_t si = 0, pi = 0, star_s = 0;
            long star = -1;
            while (si < s.size()) {
                if (pi < p.size() && (p[pi] == '_' || p[pi] == s[si])) { si++; pi++; }
                else if (pi < p.size() && p[pi] == '%') { star = (long)pi; star_s = si; pi++; }
                else if (star >= 0) { pi = (size_t)star + 1; star_s++; si = star_s; }
                else return false;
            }
            while (pi < p.size() && p[pi] == '%') pi++;
            return pi == p.size();
        }
    }
}

// ---- the compiler ----------------------------------------------------------------------------------------
struct Compiler::CV {
    int kind = 0;  // 0 scalar, 1 code, 2 string column
    HScalar s;
    std::vector<Instr> code;
    int type = 0;
    int depth = 0;
    bool maybe_null = false;
    int slot = -1;
};

namespace {
Instr mk(uint8_t op, uint8_t sub = 0, uint8_t t = 0, uint8_t flag = 0, int a = 0, int b = 0, int c = 0) {
    Instr i{};
    i.op = op;
    i.sub = sub;
    i.t = t;
    i.flag = flag;
    i.a = a;
    i.b = b;
    i.c = c;
    return i;
}
bool castable(int from, int to) {
    if (from == to) return true;
    auto num = [](int t) { return t == ML_TYPE_INT32 || t == ML_TYPE_INT64 || t == ML_TYPE_FLOAT64 || t == ML_TYPE_DATE; };
    if (num(from) && num(to)) {
        // cast.rs has no Date->Float64 / Float64->Date / Int64->Date
        if (from == ML_TYPE_DATE && to == ML_TYPE_FLOAT64) return false;
        if (to == ML_TYPE_DATE && from != ML_TYPE_INT32) return false;
        return true;
    }
    if (from == ML_TYPE_BOOL && (to == ML_TYPE_INT32 || to == ML_TYPE_INT64 || to == ML_TYPE_FLOAT64)) return true;
    return false;
}
int common_type(int l, int r) {  // eval.rs:218-228
    if (l == r) return l;
    if ((l == ML_TYPE_DATE && r == ML_TYPE_UTF8) || (l == ML_TYPE_UTF8 && r == ML_TYPE_DATE)) return ML_TYPE_DATE;
    if ((l == ML_TYPE_DATE && (r == ML_TYPE_INT32 || r == ML_TYPE_INT64)) ||
        (r == ML_TYPE_DATE && (l == ML_TYPE_INT32 || l == ML_TYPE_INT64)))
        return ML_TYPE_INT32;
    auto num = [](int t) { return t == ML_TYPE_INT32 || t == ML_TYPE_INT64 || t == ML_TYPE_FLOAT64; };
    if (!num(l) || !num(r)) return -1;
    if (l == ML_TYPE_FLOAT64 || r == ML_TYPE_FLOAT64) return ML_TYPE_FLOAT64;
    if (l == ML_TYPE_INT64 || r == ML_TYPE_INT64) return ML_TYPE_INT64;
    return ML_TYPE_INT32;
}
}  // namespace

int Compiler::add_arena(const void* p, size_t n, size_t align) {
    size_t o = (arena.size() + align - 1) & ~(align - 1);
    arena.resize(o + n);
    if (n) memcpy(arena.data() + o, p, n);
    return (int)o;
}

int Compiler::slot_for(int src, int index, int dtype, int kind) {
    for (size_t i = 0; i < slots.size(); i++)
        if (slots[i].src == src && slots[i].index == index) return (int)i;
    if ((int)slots.size() >= kMaxCols) raise(ML_ERR_UNSUPPORTED, "pipeline references too many columns");
    slots.push_back(SlotInfo{src, index, dtype, kind});
    return (int)slots.size() - 1;
}

std::optional<SlotInfo> Compiler::column_origin(const ExprNode& e, const Schema& schema) {
    if (e.kind != ML_EXPR_COLUMN) return std::nullopt;
    if (e.index < 0 || (size_t)e.index >= schema.size()) raise(ML_ERR_INVALID, "column #" + std::to_string(e.index) + " missing");
    const ColRef& r = schema[e.index];
    if (r.kind == 2) return column_origin(*r.expr, *r.env);
    return SlotInfo{r.src, r.index, r.dtype, CK_FIXED};
}

Compiler::CV Compiler::compile(const ExprNode& e, const Schema& schema) {
    auto scalar = [](HScalar s) {
        CV v;
        v.kind = 0;
        v.s = std::move(s);
        return v;
    };
    auto type_of = [](const CV& v) { return v.kind == 0 ? v.s.kind : (v.kind == 2 ? (int)ML_TYPE_UTF8 : v.type); };
    // the value pushed by `v` as type `t` (scalars become literals)
    auto mat = [&](const CV& v, int t) -> CV {
        if (v.kind == 1) return v;
        CV o;
        o.kind = 1;
        o.type = t;
        o.depth = 1;
        if (v.kind == 0) {
            HScalar c = v.s.is_null() ? v.s : scalar_cast(v.s, t);
            Instr in = mk(I_LIT, 0, (uint8_t)t);
            in.bits = c.is_null() ? 0 : scalar_bits(c);
            in.lit_valid = !c.is_null();
            o.maybe_null = c.is_null();
            o.code.push_back(in);
            return o;
        }
        o.code.push_back(mk(I_COL, 0, ML_TYPE_UTF8, 0, v.slot));
        o.maybe_null = true;
        return o;
    };
    auto cast_cv = [&](const CV& v, int to) -> CV {
        if (v.kind == 0) return scalar(scalar_cast(v.s, to));
        int from = type_of(v);
        if (from == to) return v;
        if (v.kind == 2 || !castable(from, to))
            raise(ML_ERR_UNSUPPORTED, "cast from type " + std::to_string(from) + " to " + std::to_string(to) + " on the GPU");
        CV o = v;
        if (!((from == ML_TYPE_INT32 && to == ML_TYPE_DATE) || (from == ML_TYPE_DATE && to == ML_TYPE_INT32)))
            o.code.push_back(mk(I_CAST, (uint8_t)to, (uint8_t)from));
        o.type = to;
        return o;
    };
    auto to_bool = [&](const CV& v) -> CV {  // into_column(n, Boolean)
        if (v.kind == 0) return mat(v.s.is_null() ? v : scalar(scalar_cast(v.s, ML_TYPE_BOOL)), ML_TYPE_BOOL);
        if (type_of(v) != ML_TYPE_BOOL) raise(ML_ERR_INVALID, "AND/OR on non-boolean");
        return v;
    };
    auto join2 = [](CV a, const CV& b, Instr op, int type, bool maybe_null) {
        CV o;
        o.kind = 1;
        o.code = std::move(a.code);
        o.code.insert(o.code.end(), b.code.begin(), b.code.end());
        o.code.push_back(op);
        o.type = type;
        o.depth = std::max(a.depth, 1 + b.depth);
        o.maybe_null = maybe_null;
        return o;
    };
    auto push_pred = [&](int slot, StrSpec sp, const std::string& lit, const std::vector<std::string>* list, int what, int op,
                         bool negated) -> CV {
        sp.what = (uint8_t)what;
        sp.op = (uint8_t)op;
        sp.negated = negated;
        if (list) {
            std::vector<uint32_t> pairs;
            for (auto& s : *list) {
                int o = add_arena(s.data(), s.size(), 1);
                pairs.push_back((uint32_t)o);
                pairs.push_back((uint32_t)s.size());
            }
            sp.lit_off = (uint32_t)add_arena(pairs.data(), pairs.size() * 4, 4);
            sp.count = (uint32_t)list->size();
        } else {
            sp.lit_off = (uint32_t)add_arena(lit.data(), lit.size(), 1);
            sp.lit_len = (uint32_t)lit.size();
        }
        int spec_off = add_arena(&sp, sizeof sp, 16);
        if ((int)luts.size() >= kMaxLuts) raise(ML_ERR_UNSUPPORTED, "too many string predicates");
        LutSpec L;
        L.slot = slot;
        L.what = what;
        L.op = op;
        L.shape = op;
        L.negated = negated;
        L.lit = lit;
        if (list) L.list = *list;
        luts.push_back(L);
        CV o;
        o.kind = 1;
        o.type = ML_TYPE_BOOL;
        o.depth = 1;
        o.maybe_null = true;
        o.code.push_back(mk(I_STRPRED, 0, ML_TYPE_BOOL, 0, slot, (int)luts.size() - 1, spec_off));
        return o;
    };

    switch (e.kind) {
        case ML_EXPR_COLUMN: {
            if (e.index < 0 || (size_t)e.index >= schema.size())
                raise(ML_ERR_INVALID, "column #" + std::to_string(e.index) + " missing");
            const ColRef& r = schema[e.index];
            if (r.kind == 2) return compile(*r.expr, *r.env);
            int slot = slot_for(r.src, r.index, r.dtype, CK_FIXED);
            if (r.dtype == ML_TYPE_UTF8) {
                CV v;
                v.kind = 2;
                v.slot = slot;
                return v;
            }
            CV v;
            v.kind = 1;
            v.type = r.dtype;
            v.depth = 1;
            v.maybe_null = false;  // a column's validity is checked per launch (Pipeline::reads_nullable)
            v.code.push_back(mk(I_COL, 0, (uint8_t)r.dtype, 0, slot));
            return v;
        }
        case ML_EXPR_LITERAL: return scalar(e.lit);
        case ML_EXPR_BINARY: {
            if (e.kids.size() != 2) raise(ML_ERR_INVALID, "binary needs 2 operands");
            CV l = compile(e.kids[0], schema), r = compile(e.kids[1], schema);
            int op = e.op;
            if (op < ML_BIN_ADD || op > ML_BIN_OR) raise(ML_ERR_INVALID, "bad binary op");
            if (l.kind == 0 && r.kind == 0) return scalar(scalar_binary(op, l.s, r.s));
            if (op == ML_BIN_AND || op == ML_BIN_OR) {
                CV a = to_bool(l), b = to_bool(r);
                return join2(a, b, mk(I_BIN, (uint8_t)op, ML_TYPE_BOOL), ML_TYPE_BOOL, a.maybe_null || b.maybe_null);
            }
            if ((l.kind == 0 && l.s.is_null()) || (r.kind == 0 && r.s.is_null())) return scalar(HScalar());
            int lt = type_of(l), rt = type_of(r);
            int ct = common_type(lt, rt);
            if (ct < 0) raise(ML_ERR_INVALID, "incompatible types " + std::to_string(lt) + " " + std::to_string(rt));
            bool arith = op <= ML_BIN_MOD;
            bool date_result = arith && (lt == ML_TYPE_DATE || rt == ML_TYPE_DATE);
            bool date_diff = op == ML_BIN_SUB && lt == ML_TYPE_DATE && rt == ML_TYPE_DATE;
            l = cast_cv(l, ct);
            r = cast_cv(r, ct);
            if (op >= ML_BIN_EQ) {
                if (ct == ML_TYPE_UTF8) {
                    if (l.kind == 2 && r.kind == 0) return push_pred(l.slot, StrSpec{}, r.s.s, nullptr, SW_CMP, op, false);
                    if (l.kind == 0 && r.kind == 2) {
                        int f = op == ML_BIN_LT ? ML_BIN_GT : op == ML_BIN_LTEQ ? ML_BIN_GTEQ : op == ML_BIN_GT ? ML_BIN_LT
                                : op == ML_BIN_GTEQ ? ML_BIN_LTEQ : op;
                        return push_pred(r.slot, StrSpec{}, l.s.s, nullptr, SW_CMP, f, false);
                    }
                    if (l.kind == 2 && r.kind == 2) {
                        CV o;
                        o.kind = 1;
                        o.type = ML_TYPE_BOOL;
                        o.depth = 1;
                        o.maybe_null = true;
                        o.code.push_back(mk(I_STRCMP_COL, (uint8_t)op, ML_TYPE_BOOL, 0, l.slot, r.slot));
                        return o;
                    }
                    raise(ML_ERR_UNSUPPORTED, "string comparison of computed strings on the GPU");
                }
                CV a = mat(l, ct), b = mat(r, ct);
                return join2(a, b, mk(I_BIN, (uint8_t)op, (uint8_t)ct), ML_TYPE_BOOL, a.maybe_null || b.maybe_null);
            }
            if (op == ML_BIN_DIV) {
                CV a = mat(cast_cv(l, ML_TYPE_FLOAT64), ML_TYPE_FLOAT64), b = mat(cast_cv(r, ML_TYPE_FLOAT64), ML_TYPE_FLOAT64);
                return join2(a, b, mk(I_BIN, ML_BIN_DIV, ML_TYPE_FLOAT64), ML_TYPE_FLOAT64, true);
            }
            if (ct != ML_TYPE_INT32 && ct != ML_TYPE_DATE && ct != ML_TYPE_INT64 && ct != ML_TYPE_FLOAT64)
                raise(ML_ERR_INVALID, "arithmetic on type " + std::to_string(ct) + " is not supported");
            int arith_t = ct == ML_TYPE_DATE ? ML_TYPE_INT32 : ct;
            int out = ct;
            if (ct == ML_TYPE_INT32 || ct == ML_TYPE_DATE) out = date_diff ? ML_TYPE_INT32 : (date_result ? ML_TYPE_DATE : ML_TYPE_INT32);
            CV a = mat(l, ct), b = mat(r, ct);
            bool mn = a.maybe_null || b.maybe_null || (op == ML_BIN_MOD && ct != ML_TYPE_FLOAT64);
            return join2(a, b, mk(I_BIN, (uint8_t)op, (uint8_t)arith_t), out, mn);
        }
        case ML_EXPR_NOT: {
            CV c = compile(e.kids.at(0), schema);
            if (c.kind == 0) {
                if (c.s.kind == ML_TYPE_BOOL) return scalar(HScalar::b(!c.s.i));
                return scalar(HScalar());
            }
            if (type_of(c) != ML_TYPE_BOOL) raise(ML_ERR_INVALID, "NOT of non-boolean");
            c.code.push_back(mk(I_NOT));
            return c;
        }
        case ML_EXPR_NEGATE: {
            CV c = compile(e.kids.at(0), schema);
            if (c.kind == 0) {
                HScalar s = c.s;
                if (s.is_null()) return c;
                if (s.kind == ML_TYPE_INT32 || s.kind == ML_TYPE_INT64) s.i = -s.i;
                else if (s.kind == ML_TYPE_FLOAT64) s.f = -s.f;
                else raise(ML_ERR_INVALID, "cannot negate");
                return scalar(s);
            }
            int t = type_of(c);
            if (t != ML_TYPE_INT32 && t != ML_TYPE_INT64 && t != ML_TYPE_FLOAT64) raise(ML_ERR_INVALID, "cannot negate");
            c.code.push_back(mk(I_NEG, 0, (uint8_t)t));
            return c;
        }
        case ML_EXPR_IS_NULL: {
            CV c = compile(e.kids.at(0), schema);
            if (c.kind == 0) return scalar(HScalar::b(c.s.is_null() != (e.flag != 0)));
            CV m = mat(c, type_of(c));
            m.code.push_back(mk(I_ISNULL, 0, 0, (uint8_t)(e.flag != 0)));
            m.type = ML_TYPE_BOOL;
            m.maybe_null = false;
            return m;
        }
        case ML_EXPR_LIKE: {
            CV c = compile(e.kids.at(0), schema);
            std::string inner;
            int shape = like_shape(e.str, &inner);
            if (c.kind == 0) {
                if (c.s.kind == ML_TYPE_UTF8) return scalar(HScalar::b(like_match_host(c.s.s, inner, shape) != (e.flag != 0)));
                return scalar(HScalar());
            }
            if (c.kind != 2) raise(ML_ERR_UNSUPPORTED, "LIKE over a non-string column on the GPU");
            return push_pred(c.slot, StrSpec{}, inner, nullptr, SW_LIKE, shape, e.flag != 0);
        }
        case ML_EXPR_IN_LIST: {
            CV c = compile(e.kids.at(0), schema);
            std::vector<HScalar> list;
            for (size_t k = 1; k < e.kids.size(); k++) {
                if (e.kids[k].kind != ML_EXPR_LITERAL) raise(ML_ERR_INVALID, "IN list items must be literals");
                list.push_back(e.kids[k].lit);
            }
            bool neg = e.flag != 0;
            if (c.kind == 0) {
                if (c.s.is_null()) return scalar(HScalar());
                bool hit = false;
                for (auto& v : list) {
                    auto o = scalar_compare(c.s, v);
                    hit |= o && *o == 0;
                }
                return scalar(HScalar::b(hit != neg));
            }
            if (c.kind == 2) {
                std::vector<std::string> items;
                for (auto& v : list)
                    if (v.kind == ML_TYPE_UTF8) items.push_back(v.s);
                return push_pred(c.slot, StrSpec{}, "", &items, SW_IN, 0, neg);
            }
            int t = c.type;
            std::vector<uint64_t> items;
            for (auto& v : list) {
                if (t == ML_TYPE_BOOL) {
                    if (v.kind == ML_TYPE_BOOL) items.push_back(v.i ? 1 : 0);
                    continue;
                }
                HScalar cv = scalar_cast(v, t);  // cast_list (eval.rs:450-454)
                if (!cv.is_null()) items.push_back(scalar_bits(cv));
            }
            int off = add_arena(items.data(), items.size() * 8, 8);
            c.code.push_back(mk(I_INLIST, 0, (uint8_t)t, (uint8_t)neg, 0, off, (int)items.size()));
            c.type = ML_TYPE_BOOL;
            return c;
        }
        case ML_EXPR_CASE: {
            int dt = e.dtype;
            if (dt == ML_TYPE_UTF8) raise(ML_ERR_UNSUPPORTED, "string-valued CASE on the GPU");
            size_t k = e.kids.size() / 2;
            bool has_else = e.flag != 0;
            if (e.kids.size() != 2 * k + (has_else ? 1 : 0)) raise(ML_ERR_INVALID, "bad CASE");
            auto value = [&](const ExprNode& v) {  // evaluate_to_column(v, dt)
                CV c = compile(v, schema);
                if (c.kind == 0) return mat(c.s.is_null() ? c : scalar(scalar_cast(c.s, dt)), dt);
                return mat(cast_cv(c, dt), dt);
            };
            CV acc;
            if (has_else) acc = value(e.kids[2 * k]);
            else acc = mat(scalar(HScalar()), dt);
            for (size_t b = k; b-- > 0;) {
                CV c = to_bool(compile(e.kids[2 * b], schema));
                CV v = value(e.kids[2 * b + 1]);
                CV o;
                o.kind = 1;
                o.type = dt;
                o.code = acc.code;
                o.code.insert(o.code.end(), c.code.begin(), c.code.end());
                o.code.insert(o.code.end(), v.code.begin(), v.code.end());
                o.code.push_back(mk(I_SELECT, 0, (uint8_t)dt));
                o.depth = std::max({acc.depth, 1 + c.depth, 2 + v.depth});
                o.maybe_null = true;
                acc = std::move(o);
            }
            return acc;
        }
        case ML_EXPR_CAST: {
            CV c = compile(e.kids.at(0), schema);
            return cast_cv(c, e.dtype);
        }
    }
    raise(ML_ERR_INVALID, "bad expression");
}

// Peephole: [COL(i32) CAST(->i64) LIT(v) BIN(cmp)] compares in 32 bits when v fits (the
// planner's Int64 literals against Int32/Date columns, e.g. d <= 2467).
static void fold_casts(std::vector<Instr>& c) {
    for (size_t i = 0; i + 3 < c.size(); i++) {
        Instr &col = c[i], &cast = c[i + 1], &lit = c[i + 2], &bin = c[i + 3];
        bool narrow = col.t == ML_TYPE_INT32 || col.t == ML_TYPE_DATE;
        if (col.op == I_COL && narrow && cast.op == I_CAST && cast.t == col.t && cast.sub == ML_TYPE_INT64 &&
            lit.op == I_LIT && bin.op == I_BIN && bin.sub >= ML_BIN_EQ && bin.sub <= ML_BIN_GTEQ && bin.t == ML_TYPE_INT64) {
            int64_t v = (int64_t)lit.bits;
            if (lit.lit_valid && v >= INT32_MIN && v <= INT32_MAX) {
                lit.t = ML_TYPE_INT32;
                bin.t = ML_TYPE_INT32;
                c.erase(c.begin() + (long)i + 1);
            }
        }
    }
}

void classify(Prog& p, const std::vector<Instr>& code) {
    auto op = [&](int k) { return code[p.start + k].op; };
    p.fast = FP_NONE;
    if (p.len == 1 && op(0) == I_COL) p.fast = FP_COL;
    else if (p.len == 3 && op(0) == I_COL && op(1) == I_LIT && op(2) == I_BIN) p.fast = FP_COL_LIT_BIN;
    else if (p.len == 5 && op(0) == I_COL && op(1) == I_LIT && op(2) == I_COL && op(3) == I_BIN && op(4) == I_BIN)
        p.fast = FP_COL_LCB_BIN;
}

Prog Compiler::compile_value(const ExprNode& e, const Schema& schema, int out_type) {
    CV c = compile(e, schema);
    if (c.kind == 2) {
        if (out_type != ML_TYPE_UTF8) raise(ML_ERR_UNSUPPORTED, "string value cast on the GPU");
        raise(ML_ERR_UNSUPPORTED, "string-valued expression outside a key on the GPU");
    }
    CV v;
    if (c.kind == 0) {
        HScalar s = c.s.is_null() ? c.s : scalar_cast(c.s, out_type);
        v.kind = 1;
        v.type = out_type;
        v.depth = 1;
        Instr in = mk(I_LIT, 0, (uint8_t)out_type);
        in.bits = s.is_null() ? 0 : scalar_bits(s);
        in.lit_valid = !s.is_null();
        v.code.push_back(in);
        v.maybe_null = s.is_null();
    } else if (c.type != out_type) {
        if (!castable(c.type, out_type)) raise(ML_ERR_UNSUPPORTED, "cast on the GPU");
        v = c;
        if (!((c.type == ML_TYPE_INT32 && out_type == ML_TYPE_DATE) || (c.type == ML_TYPE_DATE && out_type == ML_TYPE_INT32)))
            v.code.push_back(mk(I_CAST, (uint8_t)out_type, (uint8_t)c.type));
        v.type = out_type;
    } else {
        v = c;
    }
    if (v.depth > kStack) raise(ML_ERR_UNSUPPORTED, "expression needs a deeper evaluation stack than the GPU kernels keep");
    fold_casts(v.code);
    Prog p{};
    p.start = (int)code.size();
    p.len = (int)v.code.size();
    p.type = out_type;
    p.maybe_null = v.maybe_null;
    code.insert(code.end(), v.code.begin(), v.code.end());
    classify(p, code);
    return p;
}

Prog Compiler::compile_string_key(const ExprNode& e, const Schema& schema, int* slot_out) {
    CV c = compile(e, schema);
    if (c.kind != 2) raise(ML_ERR_UNSUPPORTED, "string key must be a column reference on the GPU");
    *slot_out = c.slot;
    if (std::find(string_key_slots.begin(), string_key_slots.end(), c.slot) == string_key_slots.end())
        string_key_slots.push_back(c.slot);
    Prog p{};
    p.start = (int)code.size();
    p.len = 1;
    p.type = ML_TYPE_UTF8;
    p.maybe_null = 1;
    code.push_back(mk(I_COL, 0, ML_TYPE_UTF8, 0, c.slot));
    classify(p, code);
    return p;
}

}  // namespace mlg
