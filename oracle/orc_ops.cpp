// TEST INFRASTRUCTURE — CPU oracle, part 2: memory pool, accumulators, group
// keys, hash aggregation, hash join, top-N.  Restates MiniLake's Rust sources
// (paths inside the MiniLake project); used only as the parity checker and the
// timed CPU baseline.
#include <algorithm>
#include <cmath>
#include <numeric>

#include "orc.hpp"

namespace orc {

// ---- memory.rs:22-157 -------------------------------------------------------------
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
MemoryReservation::MemoryReservation(MemoryReservation&& o) noexcept
    : pool(std::move(o.pool)), name(std::move(o.name)), size(o.size), peak(o.peak) {
    o.size = 0;
}
void MemoryReservation::try_grow(uint64_t bytes) {
    uint64_t observed = 0;
    if (!pool->try_grow(bytes, &observed)) {
        Error e(ML_ERR_BUDGET, "Resources exhausted: " + name + " requested " + std::to_string(bytes) +
                                   " bytes, " + std::to_string(observed) + " of " +
                                   std::to_string(pool->limit) + " used");
        e.op = name;
        e.requested = bytes;
        e.used = observed;
        e.limit = pool->limit;
        throw e;
    }
    size += bytes;
    peak = std::max(peak, size);
}
void MemoryReservation::shrink(uint64_t bytes) {
    if (!pool) return;
    uint64_t b = std::min(bytes, size);
    pool->shrink(b);
    size -= b;
}

// ---- accumulator.rs:110-594 --------------------------------------------------------
enum { K_COUNT, K_SUMI64, K_SUMF64, K_AVG, K_MMI64, K_MMF64, K_MMSTR };

Accumulator::Accumulator(int fn, int t) : func(fn) {
    auto bad = [&]() { fail(ML_ERR_UNSUPPORTED, "aggregate not supported for this argument type"); };
    switch (fn) {
        case ML_AGG_COUNT_STAR: input_type = -1; output_type = I64; kind = K_COUNT; return;
        case ML_AGG_COUNT: input_type = t; output_type = I64; kind = K_COUNT; return;
        case ML_AGG_SUM:
            if (t == I32 || t == I64 || t == BOOL) { input_type = I64; output_type = I64; kind = K_SUMI64; return; }
            if (t == F64) { input_type = F64; output_type = F64; kind = K_SUMF64; return; }
            bad();
        case ML_AGG_AVG:
            if (is_numeric(t)) { input_type = F64; output_type = F64; kind = K_AVG; return; }
            bad();
        case ML_AGG_MIN:
        case ML_AGG_MAX:
            if (t == I32 || t == I64 || t == DATE) { input_type = I64; output_type = t; kind = K_MMI64; return; }
            if (t == F64) { input_type = F64; output_type = F64; kind = K_MMF64; return; }
            if (t == UTF8) { input_type = UTF8; output_type = UTF8; kind = K_MMSTR; return; }
            bad();
    }
    bad();
}

size_t Accumulator::num_groups() const {
    switch (kind) {
        case K_COUNT: case K_SUMI64: case K_MMI64: return i.size();
        case K_SUMF64: case K_AVG: case K_MMF64: return f.size();
        default: return str.size();
    }
}
void Accumulator::resize(size_t n) {
    switch (kind) {
        case K_COUNT: i.resize(n, 0); break;
        case K_SUMI64: case K_MMI64: i.resize(n, 0); seen.resize(n, 0); break;
        case K_SUMF64: case K_MMF64: f.resize(n, 0.0); seen.resize(n, 0); break;
        case K_AVG: f.resize(n, 0.0); i.resize(n, 0); break;
        default: str.resize(n); break;
    }
}
ColPtr Accumulator::prepare_input(const ColPtr& c) const {
    if (input_type >= 0 && func != ML_AGG_COUNT && c->dt != input_type) return cast_column(c, input_type);
    return c;
}
std::vector<int> Accumulator::state_types() const {
    switch (kind) {
        case K_COUNT: case K_SUMI64: case K_MMI64: return {I64};
        case K_SUMF64: case K_MMF64: return {F64};
        case K_AVG: return {F64, I64};
        default: return {UTF8};
    }
}

double sum_f64(const double* v, size_t n) {
    double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    size_t full = n / 8;
    for (size_t c = 0; c < full; c++)
        for (int k = 0; k < 8; k++) acc[k] += v[c * 8 + k];
    double s = 0;
    for (int k = 0; k < 8; k++) s += acc[k];
    for (size_t r = full * 8; r < n; r++) s += v[r];
    return s;
}
double sum_f64_sel(const double* v, const uint32_t* sel, size_t n) {
    double acc[4] = {0, 0, 0, 0};
    size_t full = n / 4;
    for (size_t c = 0; c < full; c++)
        for (int k = 0; k < 4; k++) acc[k] += v[sel[c * 4 + k]];
    double s = 0;
    for (int k = 0; k < 4; k++) s += acc[k];
    for (size_t r = full * 4; r < n; r++) s += v[sel[r]];
    return s;
}

void Accumulator::update(const Column* in, size_t nrows, const uint32_t* rows, size_t k,
                         const uint32_t* gids) {
    size_t m = rows ? k : nrows;
    auto row = [&](size_t j) -> size_t { return rows ? rows[j] : j; };
    auto gid = [&](size_t j) -> size_t { return gids ? gids[j] : 0; };
    bool is_min = func == ML_AGG_MIN;
    if (kind == K_COUNT) {
        bool has_valid = in && in->vw;
        if (func == ML_AGG_COUNT_STAR || !has_valid) {
            if (!gids) i[0] += (int64_t)m;
            else for (size_t j = 0; j < m; j++) i[gids[j]] += 1;
        } else {
            for (size_t j = 0; j < m; j++)
                if (in->valid(row(j))) i[gid(j)] += 1;
        }
        return;
    }
    if (!in) fail(ML_ERR_INTERNAL, "aggregate without input");
    const Column& c = *in;
    bool nv = c.vw == nullptr;
    switch (kind) {
        case K_SUMI64: {
            if (c.dt != I64) break;
            const int64_t* v = c.as<int64_t>();
            if (!gids && nv) {
                uint64_t s = 0;
                for (size_t j = 0; j < m; j++) s += (uint64_t)v[row(j)];
                i[0] = (int64_t)((uint64_t)i[0] + s);
                seen[0] |= m > 0;
            } else {
                for (size_t j = 0; j < m; j++) {
                    size_t r = row(j);
                    if (c.valid(r)) {
                        size_t g = gid(j);
                        i[g] = (int64_t)((uint64_t)i[g] + (uint64_t)v[r]);
                        seen[g] = 1;
                    }
                }
            }
            return;
        }
        case K_SUMF64: {
            if (c.dt != F64) break;
            const double* v = c.as<double>();
            if (!gids && nv) {
                f[0] += rows ? sum_f64_sel(v, rows, k) : sum_f64(v, nrows);
                seen[0] |= m > 0;
            } else {
                for (size_t j = 0; j < m; j++) {
                    size_t r = row(j);
                    if (c.valid(r)) {
                        size_t g = gid(j);
                        f[g] += v[r];
                        seen[g] = 1;
                    }
                }
            }
            return;
        }
        case K_AVG: {
            if (c.dt != F64) break;
            const double* v = c.as<double>();
            if (!gids && nv) {
                f[0] += rows ? sum_f64_sel(v, rows, k) : sum_f64(v, nrows);
                i[0] += (int64_t)m;
            } else {
                for (size_t j = 0; j < m; j++) {
                    size_t r = row(j);
                    if (c.valid(r)) {
                        size_t g = gid(j);
                        f[g] += v[r];
                        i[g] += 1;
                    }
                }
            }
            return;
        }
        case K_MMI64: {
            if (c.dt != I64) break;
            const int64_t* v = c.as<int64_t>();
            for (size_t j = 0; j < m; j++) {
                size_t r = row(j);
                if (c.valid(r)) {
                    size_t g = gid(j);
                    int64_t x = v[r];
                    if (!seen[g] || (is_min && x < i[g]) || (!is_min && x > i[g])) {
                        i[g] = x;
                        seen[g] = 1;
                    }
                }
            }
            return;
        }
        case K_MMF64: {
            if (c.dt != F64) break;
            const double* v = c.as<double>();
            for (size_t j = 0; j < m; j++) {
                size_t r = row(j);
                if (c.valid(r)) {
                    size_t g = gid(j);
                    double x = v[r];
                    if (!seen[g] || (is_min && x < f[g]) || (!is_min && x > f[g])) {
                        f[g] = x;
                        seen[g] = 1;
                    }
                }
            }
            return;
        }
        case K_MMSTR: {
            if (c.dt != UTF8) break;
            for (size_t j = 0; j < m; j++) {
                size_t r = row(j);
                if (c.valid(r)) {
                    size_t g = gid(j);
                    std::string_view x = c.str(r);
                    bool replace = !str[g] || (is_min && x < std::string_view(*str[g])) ||
                                   (!is_min && x > std::string_view(*str[g]));
                    if (replace) str[g] = std::string(x);
                }
            }
            return;
        }
    }
    fail(ML_ERR_INTERNAL, "accumulator got wrong input type");
}

std::vector<ColPtr> Accumulator::state() const {
    auto bm = [&]() { return std::optional<Bitmap>(Bitmap::from_bools(seen)); };
    switch (kind) {
        case K_COUNT: return {make_i64(std::vector<int64_t>(i), std::nullopt)};
        case K_SUMI64: case K_MMI64: return {make_i64(std::vector<int64_t>(i), bm())};
        case K_SUMF64: case K_MMF64: return {make_f64(std::vector<double>(f), bm())};
        case K_AVG: return {make_f64(std::vector<double>(f), std::nullopt), make_i64(std::vector<int64_t>(i), std::nullopt)};
        default: {
            Strings s;
            std::vector<uint8_t> v(str.size());
            for (size_t g = 0; g < str.size(); g++) {
                s.push(str[g] ? *str[g] : "");
                v[g] = str[g].has_value();
            }
            return {make_utf8(std::move(s), Bitmap::from_bools(v))};
        }
    }
}

void Accumulator::merge(const std::vector<ColPtr>& st, const uint32_t* gids, size_t k) {
    if (st.empty()) fail(ML_ERR_INTERNAL, "empty aggregate state");
    const Column& first = *st[0];
    bool is_min = func == ML_AGG_MIN;
    switch (kind) {
        case K_COUNT:
            for (size_t j = 0; j < k; j++) i[gids[j]] += first.as<int64_t>()[j];
            return;
        case K_SUMI64:
            for (size_t j = 0; j < k; j++)
                if (first.valid(j)) {
                    i[gids[j]] = (int64_t)((uint64_t)i[gids[j]] + (uint64_t)first.as<int64_t>()[j]);
                    seen[gids[j]] = 1;
                }
            return;
        case K_SUMF64:
            for (size_t j = 0; j < k; j++)
                if (first.valid(j)) {
                    f[gids[j]] += first.as<double>()[j];
                    seen[gids[j]] = 1;
                }
            return;
        case K_AVG: {
            if (st.size() < 2) fail(ML_ERR_INTERNAL, "AVG state needs 2 columns");
            for (size_t j = 0; j < k; j++) {
                f[gids[j]] += first.as<double>()[j];
                i[gids[j]] += st[1]->as<int64_t>()[j];
            }
            return;
        }
        case K_MMI64:
            for (size_t j = 0; j < k; j++) {
                size_t g = gids[j];
                int64_t x = first.as<int64_t>()[j];
                if (first.valid(j) && (!seen[g] || (is_min && x < i[g]) || (!is_min && x > i[g]))) {
                    i[g] = x;
                    seen[g] = 1;
                }
            }
            return;
        case K_MMF64:
            for (size_t j = 0; j < k; j++) {
                size_t g = gids[j];
                double x = first.as<double>()[j];
                if (first.valid(j) && (!seen[g] || (is_min && x < f[g]) || (!is_min && x > f[g]))) {
                    f[g] = x;
                    seen[g] = 1;
                }
            }
            return;
        default:
            for (size_t j = 0; j < k; j++) {
                if (!first.valid(j)) continue;
                size_t g = gids[j];
                std::string_view x = first.str(j);
                bool replace = !str[g] || (is_min && x < std::string_view(*str[g])) ||
                               (!is_min && x > std::string_view(*str[g]));
                if (replace) str[g] = std::string(x);
            }
            return;
    }
}

ColPtr Accumulator::finish() const {
    auto bm = [&]() { return std::optional<Bitmap>(Bitmap::from_bools(seen)); };
    switch (kind) {
        case K_COUNT: return make_i64(std::vector<int64_t>(i), std::nullopt);
        case K_SUMI64: return make_i64(std::vector<int64_t>(i), bm());
        case K_SUMF64: case K_MMF64: return make_f64(std::vector<double>(f), bm());
        case K_AVG: {
            std::vector<double> v(f.size());
            std::vector<uint8_t> s(f.size());
            for (size_t g = 0; g < f.size(); g++) {
                v[g] = i[g] == 0 ? 0.0 : f[g] / (double)i[g];
                s[g] = i[g] > 0;
            }
            return make_f64(std::move(v), Bitmap::from_bools(s));
        }
        case K_MMI64: {
            if (output_type == I32 || output_type == DATE) {
                std::vector<int32_t> v(i.size());
                for (size_t g = 0; g < i.size(); g++) v[g] = (int32_t)i[g];
                return make_i32(std::move(v), bm(), output_type);
            }
            return make_i64(std::vector<int64_t>(i), bm());
        }
        default: return state()[0];
    }
}

size_t Accumulator::memory_size() const {
    size_t n = num_groups();
    switch (kind) {
        case K_COUNT: return n * 8;
        case K_AVG: return n * 16;
        case K_MMSTR: {
            size_t s = 0;
            for (auto& x : str) s += 24 + (x ? x->size() : 0);
            return s;
        }
        default: return n * 9;
    }
}

// ---- group_keys.rs:27-150 -------------------------------------------------------------
GroupKeys::GroupKeys(const std::vector<int>& types) {
    for (int t : types) {
        KeyCol kc;
        kc.dt = t;
        cols.push_back(std::move(kc));
    }
}
uint32_t GroupKeys::push(const std::vector<ColPtr>& in, size_t row) {
    for (size_t c = 0; c < cols.size(); c++) {
        KeyCol& kc = cols[c];
        const Column& col = *in[c];
        kc.valid.push_back(col.valid(row));
        switch (kc.dt) {
            case I32: case DATE: kc.i32.push_back(col.dt == I32 || col.dt == DATE ? col.as<int32_t>()[row] : 0); bytes += 5; break;
            case I64: kc.i64.push_back(col.dt == I64 ? col.as<int64_t>()[row] : 0); bytes += 9; break;
            case F64: kc.f64.push_back(col.dt == F64 ? col.as<double>()[row] : 0.0); bytes += 9; break;
            case BOOL: kc.b.push_back(col.dt == BOOL ? col.as<uint8_t>()[row] : 0); bytes += 2; break;
            default: {
                std::string_view s = col.dt == UTF8 ? col.str(row) : std::string_view();
                kc.s.push(s);
                bytes += 5 + s.size();
            }
        }
    }
    len++;
    return (uint32_t)(len - 1);
}
bool GroupKeys::equals(uint32_t g, const std::vector<ColPtr>& in, size_t row) const {
    for (size_t c = 0; c < cols.size(); c++) {
        const KeyCol& kc = cols[c];
        const Column& col = *in[c];
        bool v = col.valid(row);
        if (v != (bool)kc.valid[g]) return false;
        if (!v) continue;
        switch (kc.dt) {
            case I32: case DATE: if (kc.i32[g] != col.as<int32_t>()[row]) return false; break;
            case I64: if (kc.i64[g] != col.as<int64_t>()[row]) return false; break;
            case F64: if (!(kc.f64[g] == col.as<double>()[row])) return false; break;
            case BOOL: if (kc.b[g] != col.as<uint8_t>()[row]) return false; break;
            default: if (col.str(row) != kc.s.get(g)) return false;
        }
    }
    return true;
}
std::vector<ColPtr> GroupKeys::to_columns() const {
    std::vector<ColPtr> out;
    for (auto& kc : cols) {
        auto v = std::optional<Bitmap>(Bitmap::from_bools(kc.valid));
        switch (kc.dt) {
            case I32: case DATE: out.push_back(make_i32(std::vector<int32_t>(kc.i32), std::move(v), kc.dt)); break;
            case I64: out.push_back(make_i64(std::vector<int64_t>(kc.i64), std::move(v))); break;
            case F64: out.push_back(make_f64(std::vector<double>(kc.f64), std::move(v))); break;
            case BOOL: out.push_back(make_bool(std::vector<uint8_t>(kc.b), std::move(v))); break;
            default: out.push_back(make_utf8(Strings(kc.s), std::move(v)));
        }
    }
    return out;
}

// ---- aggregate/hash.rs:204-322 ------------------------------------------------------
HashAggState::HashAggState(const std::vector<int>& kt, const std::vector<AggSpec>& aggs)
    : key_types(kt), keys(kt), table(0) {
    for (auto& a : aggs) accs.emplace_back(a.func, a.arg_type);
}

namespace {
struct Store {  // KeyStore adapter (aggregate/hash.rs:185-202)
    GroupKeys& keys;
    const std::vector<ColPtr>& cols;
    const uint32_t* rows;
    size_t row(size_t k) const { return rows ? rows[k] : k; }
    bool equals(uint32_t p, size_t k) const { return keys.equals(p, cols, row(k)); }
    uint32_t insert(size_t k) { return keys.push(cols, row(k)); }
};
}  // namespace

void HashAggState::assign_groups(const std::vector<ColPtr>& key_cols, size_t n, const uint32_t* rows, size_t k) {
    hash_columns(key_cols, n, rows, k, hashes);
    Store st{keys, key_cols, rows};
    table.find_or_insert_batch(hashes, st, gids);
    size_t ng = keys.len;
    for (auto& a : accs)
        if (a.num_groups() < ng) a.resize(ng);
}

void HashAggState::update(const Batch& b, const std::vector<Expr>& group_exprs, const std::vector<AggSpec>& aggs) {
    std::vector<ColPtr> key_cols;
    for (size_t g = 0; g < group_exprs.size(); g++)
        key_cols.push_back(evaluate_to_column(group_exprs[g], b, key_types[g]));
    const uint32_t* rows = b.sel ? b.sel->data() : nullptr;
    size_t k = b.sel ? b.sel->size() : b.n;
    assign_groups(key_cols, b.n, rows, k);
    for (size_t a = 0; a < aggs.size(); a++) {
        ColPtr arg;
        if (aggs[a].arg) arg = accs[a].prepare_input(evaluate_to_column(*aggs[a].arg, b, aggs[a].arg_type));
        accs[a].update(arg.get(), b.n, rows, k, gids.data());
    }
}

void HashAggState::merge_partial(const Batch& b0) {
    Batch b = b0.compact();
    size_t nk = key_types.size();
    std::vector<ColPtr> kc(b.cols.begin(), b.cols.begin() + nk);
    assign_groups(kc, b.n, nullptr, b.n);
    size_t c = nk;
    for (auto& a : accs) {
        size_t k = a.state_types().size();
        std::vector<ColPtr> st(b.cols.begin() + c, b.cols.begin() + c + k);
        a.merge(st, gids.data(), b.n);
        c += k;
    }
}
void HashAggState::merge_state(const HashAggState& o) {
    if (o.num_groups() == 0) return;
    merge_partial(o.partial_batch());
}
Batch HashAggState::partial_batch() const {
    Batch b;
    b.cols = keys.to_columns();
    for (auto& a : accs)
        for (auto& c : a.state()) b.cols.push_back(c);
    b.n = num_groups();
    return b;
}
Batch HashAggState::final_batch() const {
    Batch b;
    b.cols = keys.to_columns();
    for (auto& a : accs) b.cols.push_back(a.finish());
    b.n = num_groups();
    return b;
}
size_t HashAggState::memory_size() const {
    size_t s = table.memory_size() + keys.bytes;
    for (auto& a : accs) s += a.memory_size();
    return s;
}

// ---- join.rs:160-337 ------------------------------------------------------------------
static constexpr uint32_t NONE = UINT32_MAX;

std::unique_ptr<JoinTable> build_table(const std::vector<Batch>& batches, const std::vector<Expr>& key_exprs,
                                       const std::vector<int>& key_types, size_t ncols) {
    auto jt = std::make_unique<JoinTable>();
    if (batches.empty()) {
        jt->batch.n = 0;
        for (size_t c = 0; c < ncols; c++) jt->batch.cols.push_back(make_i64({}, std::nullopt));
    } else {
        jt->batch = concat(batches, ncols);
    }
    size_t n = jt->batch.n;
    for (size_t k = 0; k < key_exprs.size(); k++)
        jt->keys.push_back(evaluate_to_column(key_exprs[k], jt->batch, key_types[k]));
    std::vector<uint64_t> hashes;
    hash_columns(jt->keys, n, nullptr, n, hashes);
    jt->table = SwissTable(n);
    jt->next.assign(n, NONE);
    for (size_t r = 0; r < n; r++) {
        bool any_null = false;
        for (auto& k : jt->keys) any_null |= !k->valid(r);
        if (any_null) continue;
        auto p = jt->table.find_or_vacant(hashes[r], [&](uint32_t head) {
            for (auto& k : jt->keys)
                if (!values_equal(*k, head, *k, r)) return false;
            return true;
        });
        if (p.first) {
            uint32_t head = (uint32_t)p.second;
            jt->next[r] = jt->next[head];
            jt->next[head] = (uint32_t)r;
        } else {
            jt->table.insert_at(p.second, hashes[r], (uint32_t)r);
        }
    }
    return jt;
}

void probe_pairs(const JoinTable& jt, const std::vector<Expr>& key_exprs, const std::vector<int>& key_types,
                 const Batch& b, std::vector<uint32_t>& pi, std::vector<uint32_t>& bi) {
    pi.clear();
    bi.clear();
    if (jt.table.len == 0) return;
    std::vector<ColPtr> keys;
    for (size_t k = 0; k < key_exprs.size(); k++) keys.push_back(evaluate_to_column(key_exprs[k], b, key_types[k]));
    const uint32_t* rows = b.sel ? b.sel->data() : nullptr;
    size_t m = b.sel ? b.sel->size() : b.n;
    std::vector<uint64_t> hashes;
    hash_columns(keys, b.n, rows, m, hashes);
    for (size_t j = 0; j < m; j++) {
        size_t r = rows ? rows[j] : j;
        bool any_null = false;
        for (auto& k : keys) any_null |= !k->valid(r);
        if (any_null) continue;
        auto head = jt.table.find(hashes[j], [&](uint32_t bb) {
            for (size_t k = 0; k < keys.size(); k++)
                if (!values_equal(*jt.keys[k], bb, *keys[k], r)) return false;
            return true;
        });
        if (!head) continue;
        uint32_t x = *head;
        for (;;) {
            pi.push_back((uint32_t)r);
            bi.push_back(x);
            x = jt.next[x];
            if (x == NONE) break;
        }
    }
}

// ---- sort.rs:43-132 ---------------------------------------------------------------------
namespace {
int total_cmp(double a, double b) {  // f64::total_cmp
    int64_t x, y;
    memcpy(&x, &a, 8);
    memcpy(&y, &b, 8);
    x ^= (int64_t)(((uint64_t)(x >> 63)) >> 1);
    y ^= (int64_t)(((uint64_t)(y >> 63)) >> 1);
    return x < y ? -1 : (x > y ? 1 : 0);
}
int compare_rows(const std::vector<ColPtr>& kc, const std::vector<SortKey>& keys, size_t a, size_t b) {
    for (size_t k = 0; k < keys.size(); k++) {
        const Column& c = *kc[k];
        bool va = c.valid(a), vb = c.valid(b);
        int ord;
        if (!va && !vb) ord = 0;
        else if (!va) return keys[k].nulls_first ? -1 : 1;
        else if (!vb) return keys[k].nulls_first ? 1 : -1;
        else {
            int o;
            switch (c.dt) {
                case I32: case DATE: { auto x = c.as<int32_t>()[a], y = c.as<int32_t>()[b]; o = x < y ? -1 : x > y; break; }
                case I64: { auto x = c.as<int64_t>()[a], y = c.as<int64_t>()[b]; o = x < y ? -1 : x > y; break; }
                case F64: o = total_cmp(c.as<double>()[a], c.as<double>()[b]); break;
                case BOOL: { auto x = c.as<uint8_t>()[a], y = c.as<uint8_t>()[b]; o = x < y ? -1 : x > y; break; }
                default: { int r = c.str(a).compare(c.str(b)); o = r < 0 ? -1 : r > 0; }
            }
            ord = keys[k].asc ? o : -o;
        }
        if (ord != 0) return ord;
    }
    return 0;
}
}  // namespace

std::optional<Batch> sort_batches(const std::vector<Batch>& batches, const std::vector<SortKey>& keys,
                                  std::optional<size_t> limit, size_t ncols) {
    if (batches.empty()) return std::nullopt;
    Batch all = concat(batches, ncols);
    size_t n = all.n;
    std::vector<int> schema;
    for (auto& c : all.cols) schema.push_back(c->dt);
    std::vector<ColPtr> kc;
    for (auto& k : keys) kc.push_back(evaluate_to_column(k.expr, all, k.expr.data_type(schema)));
    std::vector<uint32_t> idx(n);
    std::iota(idx.begin(), idx.end(), 0);
    auto less = [&](uint32_t a, uint32_t b) { return compare_rows(kc, keys, a, b) < 0; };
    if (limit && *limit < n) {
        std::nth_element(idx.begin(), idx.begin() + *limit, idx.end(), less);
        idx.resize(*limit);
        std::stable_sort(idx.begin(), idx.end(), less);
    } else {
        std::stable_sort(idx.begin(), idx.end(), less);
    }
    Batch out;
    out.n = idx.size();
    for (auto& c : all.cols) out.cols.push_back(gather(*c, idx.data(), idx.size()));
    return out;
}

// ---- pipeline.rs:139-161: push a batch through the streaming operators ---------------
void run_operators(const std::vector<PipeOp>& ops, size_t idx, Batch b, const std::function<void(Batch)>& sink) {
    if (b.active_rows() == 0) return;
    if (idx == ops.size()) {
        sink(std::move(b));
        return;
    }
    const PipeOp& op = ops[idx];
    switch (op.kind) {
        case ML_PIPE_FILTER: {  // filter.rs:19-25
            auto sel = select(op.exprs[0], b, b.sel.get());
            if (!sel.empty()) {
                b.sel = std::make_shared<const std::vector<uint32_t>>(std::move(sel));
                run_operators(ops, idx + 1, std::move(b), sink);
            }
            return;
        }
        case ML_PIPE_PROJECT: {  // projection.rs:21-32
            Batch o;
            o.n = b.n;
            o.sel = b.sel;
            for (size_t e = 0; e < op.exprs.size(); e++) o.cols.push_back(evaluate_to_column(op.exprs[e], b, op.types[e]));
            run_operators(ops, idx + 1, std::move(o), sink);
            return;
        }
        case ML_PIPE_PROBE: {  // join.rs:263-337 (emit in batches of 2048 rows)
            std::vector<uint32_t> pi, bi;
            probe_pairs(*op.join, op.exprs, op.types, b, pi, bi);
            const size_t bs = 2048;
            for (size_t s = 0; s < pi.size(); s += bs) {
                size_t k = std::min(bs, pi.size() - s);
                Batch o;
                o.n = k;
                std::vector<ColPtr> p, q;
                for (auto& c : b.cols) p.push_back(gather(*c, pi.data() + s, k));
                for (auto& c : op.join->batch.cols) q.push_back(gather(*c, bi.data() + s, k));
                if (op.build_is_left) {
                    o.cols = q;
                    o.cols.insert(o.cols.end(), p.begin(), p.end());
                } else {
                    o.cols = p;
                    o.cols.insert(o.cols.end(), q.begin(), q.end());
                }
                run_operators(ops, idx + 1, std::move(o), sink);
            }
            return;
        }
    }
    fail(ML_ERR_INVALID, "bad pipeline operator");
}

}  // namespace orc
