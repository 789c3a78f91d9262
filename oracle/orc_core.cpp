// TEST INFRASTRUCTURE — CPU oracle, part 1: data model, hashing, SwissTable,
// expression evaluation.  Restates MiniLake's Rust sources (paths cited are
// inside the MiniLake project); used only as the parity checker and the timed
// CPU baseline.
#include <algorithm>
#include <charconv>
#include <cmath>
#include <cstdio>

#include "orc.hpp"

namespace orc {

const char* dt_name(int dt) {  // types.rs:65-76
    switch (dt) {
        case BOOL: return "BOOLEAN";
        case I32: return "INT32";
        case I64: return "INT64";
        case F64: return "DOUBLE";
        case DATE: return "DATE";
        case UTF8: return "VARCHAR";
    }
    return "?";
}
bool is_numeric(int dt) { return dt == I32 || dt == I64 || dt == F64; }
int numeric_supertype(int a, int b) {  // types.rs:54-62
    if (a == b && is_numeric(a)) return a;
    if ((a == F64 && is_numeric(b)) || (b == F64 && is_numeric(a))) return F64;
    if ((a == I64 && is_numeric(b)) || (b == I64 && is_numeric(a))) return I64;
    return -1;
}

// hash.rs:39-54
uint64_t hash_bytes(const uint8_t* b, size_t n) {
    uint64_t h = SEED ^ ((uint64_t)n * MUL);
    size_t full = n / 8;
    for (size_t c = 0; c < full; c++) {
        uint64_t w;
        memcpy(&w, b + c * 8, 8);
        h = fold_mul(h ^ w, MUL);
    }
    size_t rem = n % 8;
    if (rem) {
        uint64_t w = 0;
        memcpy(&w, b + full * 8, rem);
        h = fold_mul(h ^ w, MUL2);
    }
    return h;
}

// ---- bitmap.rs ----------------------------------------------------------------
Bitmap Bitmap::set_all(size_t n) {
    Bitmap b;
    b.len = n;
    b.words.assign((n + 63) / 64, ~0ull);
    if (n % 64) b.words.back() &= (1ull << (n % 64)) - 1;
    return b;
}
Bitmap Bitmap::unset_all(size_t n) {
    Bitmap b;
    b.len = n;
    b.words.assign((n + 63) / 64, 0);
    return b;
}
Bitmap Bitmap::from_bools(const std::vector<uint8_t>& v) {
    Bitmap b = unset_all(v.size());
    for (size_t i = 0; i < v.size(); i++)
        if (v[i]) b.words[i / 64] |= 1ull << (i % 64);
    return b;
}
size_t Bitmap::count_set() const {
    size_t c = 0;
    for (uint64_t w : words) c += __builtin_popcountll(w);
    return c;
}

// ---- columns --------------------------------------------------------------------
size_t Column::null_count() const {
    if (!vw) return 0;
    size_t c = 0;
    for (size_t i = 0; i < n; i++) c += !valid(i);
    return c;
}

namespace {
struct Owned {
    std::vector<uint8_t> b;
    std::vector<int32_t> i32;
    std::vector<int64_t> i64;
    std::vector<double> f64;
    std::vector<uint32_t> codes;
    Strings s;
    std::optional<Bitmap> valid;
    std::shared_ptr<const void> parent;
};

// Column::new drops a bitmap without nulls (column.rs:204-210).
void attach_validity(Column& c, Owned& o, std::optional<Bitmap>&& v) {
    if (v && v->count_set() != v->len) {
        o.valid = std::move(v);
        c.vw = o.valid->words.data();
        c.voff = 0;
    }
}
}  // namespace

ColPtr make_bool(std::vector<uint8_t>&& v, std::optional<Bitmap>&& valid) {
    auto o = std::make_shared<Owned>();
    auto c = std::make_shared<Column>();
    o->b = std::move(v);
    c->dt = BOOL;
    c->n = o->b.size();
    c->vals = o->b.data();
    attach_validity(*c, *o, std::move(valid));
    c->own = o;
    return c;
}
ColPtr make_i32(std::vector<int32_t>&& v, std::optional<Bitmap>&& valid, int dt) {
    auto o = std::make_shared<Owned>();
    auto c = std::make_shared<Column>();
    o->i32 = std::move(v);
    c->dt = dt;
    c->n = o->i32.size();
    c->vals = o->i32.data();
    attach_validity(*c, *o, std::move(valid));
    c->own = o;
    return c;
}
ColPtr make_i64(std::vector<int64_t>&& v, std::optional<Bitmap>&& valid) {
    auto o = std::make_shared<Owned>();
    auto c = std::make_shared<Column>();
    o->i64 = std::move(v);
    c->dt = I64;
    c->n = o->i64.size();
    c->vals = o->i64.data();
    attach_validity(*c, *o, std::move(valid));
    c->own = o;
    return c;
}
ColPtr make_f64(std::vector<double>&& v, std::optional<Bitmap>&& valid) {
    auto o = std::make_shared<Owned>();
    auto c = std::make_shared<Column>();
    o->f64 = std::move(v);
    c->dt = F64;
    c->n = o->f64.size();
    c->vals = o->f64.data();
    attach_validity(*c, *o, std::move(valid));
    c->own = o;
    return c;
}
ColPtr make_utf8(Strings&& s, std::optional<Bitmap>&& valid) {
    auto o = std::make_shared<Owned>();
    auto c = std::make_shared<Column>();
    o->s = std::move(s);
    c->dt = UTF8;
    c->n = o->s.len();
    c->off = o->s.off.data();
    c->bytes = o->s.bytes.data();
    attach_validity(*c, *o, std::move(valid));
    c->own = o;
    return c;
}
ColPtr make_dict(std::shared_ptr<const Strings> dict, std::vector<uint32_t>&& codes,
                 std::optional<Bitmap>&& valid) {
    auto o = std::make_shared<Owned>();
    auto c = std::make_shared<Column>();
    o->codes = std::move(codes);
    c->dt = UTF8;
    c->dict = true;
    c->dictv = std::move(dict);
    c->n = o->codes.size();
    c->vals = o->codes.data();
    attach_validity(*c, *o, std::move(valid));
    c->own = o;
    return c;
}
ColPtr with_validity(const ColPtr& c, std::optional<Bitmap>&& valid) {
    auto o = std::make_shared<Owned>();
    auto out = std::make_shared<Column>(*c);
    o->parent = c;
    out->vw = nullptr;
    out->voff = 0;
    attach_validity(*out, *o, std::move(valid));
    out->own = o;
    return out;
}
std::optional<Bitmap> validity_of(const Column& c) {
    if (!c.vw) return std::nullopt;
    Bitmap b = Bitmap::unset_all(c.n);
    for (size_t i = 0; i < c.n; i++)
        if (c.valid(i)) b.words[i / 64] |= 1ull << (i % 64);
    return b;
}

// column.rs:380-398
ColPtr gather(const Column& c, const uint32_t* idx, size_t k) {
    std::optional<Bitmap> v;
    if (c.vw) {
        v = Bitmap::unset_all(k);
        for (size_t o = 0; o < k; o++)
            if (c.valid(idx[o])) v->words[o / 64] |= 1ull << (o % 64);
    }
    switch (c.dt) {
        case BOOL: {
            std::vector<uint8_t> out(k);
            for (size_t o = 0; o < k; o++) out[o] = c.as<uint8_t>()[idx[o]];
            return make_bool(std::move(out), std::move(v));
        }
        case I32:
        case DATE: {
            std::vector<int32_t> out(k);
            for (size_t o = 0; o < k; o++) out[o] = c.as<int32_t>()[idx[o]];
            return make_i32(std::move(out), std::move(v), c.dt);
        }
        case I64: {
            std::vector<int64_t> out(k);
            for (size_t o = 0; o < k; o++) out[o] = c.as<int64_t>()[idx[o]];
            return make_i64(std::move(out), std::move(v));
        }
        case F64: {
            std::vector<double> out(k);
            for (size_t o = 0; o < k; o++) out[o] = c.as<double>()[idx[o]];
            return make_f64(std::move(out), std::move(v));
        }
        default: break;
    }
    if (c.dict) {  // gathering dictionary codes keeps the shared dictionary
        std::vector<uint32_t> out(k);
        for (size_t o = 0; o < k; o++) out[o] = c.codes()[idx[o]];
        return make_dict(c.dictv, std::move(out), std::move(v));
    }
    Strings s;
    for (size_t o = 0; o < k; o++) s.push(c.str(idx[o]));
    return make_utf8(std::move(s), std::move(v));
}

// column.rs:313-336
ColPtr nulls_column(int dt, size_t n) {
    std::optional<Bitmap> v = Bitmap::unset_all(n);
    auto c = [&]() -> ColPtr {
        switch (dt) {
            case BOOL: return make_bool(std::vector<uint8_t>(n, 0), std::nullopt);
            case I32:
            case DATE: return make_i32(std::vector<int32_t>(n, 0), std::nullopt, dt);
            case I64: return make_i64(std::vector<int64_t>(n, 0), std::nullopt);
            case F64: return make_f64(std::vector<double>(n, 0.0), std::nullopt);
            default: {
                Strings s;
                for (size_t i = 0; i < n; i++) s.push("");
                return make_utf8(std::move(s), std::nullopt);
            }
        }
    }();
    if (n == 0) return c;
    // An all-null bitmap is always kept (count_set != len when n > 0).
    return with_validity(c, std::move(v));
}

// A borrowed view of rows [row0, row0+nrows) of an ABI column (host memory).
ColPtr column_from_view(const ml_column& m, int64_t row0, int64_t nrows) {
    auto c = std::make_shared<Column>();
    c->dt = m.dtype;
    c->n = (size_t)nrows;
    if (m.validity) {
        c->vw = m.validity;
        c->voff = (size_t)row0;
    }
    if (m.dtype == UTF8 && m.encoding == ML_ENC_DICT) {
        c->dict = true;
        c->vals = (const uint32_t*)m.data + row0;
        auto d = std::make_shared<Strings>();
        d->off.assign(m.dict_offsets, m.dict_offsets + m.dict_len + 1);
        d->bytes.assign(m.dict_data, m.dict_data + m.dict_offsets[m.dict_len]);
        c->dictv = d;
    } else if (m.dtype == UTF8) {
        c->off = m.offsets + row0;
        c->bytes = (const uint8_t*)m.data;
    } else {
        size_t w = (m.dtype == BOOL) ? 1 : (m.dtype == I32 || m.dtype == DATE) ? 4 : 8;
        c->vals = (const uint8_t*)m.data + (size_t)row0 * w;
    }
    // Column::new: a bitmap with no nulls is dropped
    if (c->vw) {
        bool any_null = false;
        for (size_t i = 0; i < c->n && !any_null; i++) any_null = !c->valid(i);
        if (!any_null) c->vw = nullptr;
    }
    return c;
}

// batch.rs:121-134
Batch Batch::compact() const {
    if (!sel) return *this;
    Batch out;
    out.n = sel->size();
    for (auto& c : cols) out.cols.push_back(gather(*c, sel->data(), sel->size()));
    return out;
}

// Batch::concat of dense batches (batch.rs), by gathering every row.
Batch concat(const std::vector<Batch>& bs, size_t ncols) {
    Batch out;
    size_t total = 0;
    for (auto& b : bs) total += b.n;
    out.n = total;
    for (size_t c = 0; c < ncols; c++) {
        int dt = bs.empty() ? I64 : bs[0].cols[c]->dt;
        bool any_valid = false, dict_all = !bs.empty();
        for (auto& b : bs) {
            any_valid |= b.cols[c]->vw != nullptr;
            dict_all &= b.cols[c]->dict && b.cols[c]->dictv == bs[0].cols[c]->dictv;
        }
        std::optional<Bitmap> v;
        if (any_valid) {
            v = Bitmap::unset_all(total);
            size_t o = 0;
            for (auto& b : bs)
                for (size_t i = 0; i < b.n; i++, o++)
                    if (b.cols[c]->valid(i)) v->words[o / 64] |= 1ull << (o % 64);
        }
        switch (dt) {
            case BOOL: {
                std::vector<uint8_t> x;
                x.reserve(total);
                for (auto& b : bs) x.insert(x.end(), b.cols[c]->as<uint8_t>(), b.cols[c]->as<uint8_t>() + b.n);
                out.cols.push_back(make_bool(std::move(x), std::move(v)));
                break;
            }
            case I32:
            case DATE: {
                std::vector<int32_t> x;
                x.reserve(total);
                for (auto& b : bs) x.insert(x.end(), b.cols[c]->as<int32_t>(), b.cols[c]->as<int32_t>() + b.n);
                out.cols.push_back(make_i32(std::move(x), std::move(v), dt));
                break;
            }
            case I64: {
                std::vector<int64_t> x;
                x.reserve(total);
                for (auto& b : bs) x.insert(x.end(), b.cols[c]->as<int64_t>(), b.cols[c]->as<int64_t>() + b.n);
                out.cols.push_back(make_i64(std::move(x), std::move(v)));
                break;
            }
            case F64: {
                std::vector<double> x;
                x.reserve(total);
                for (auto& b : bs) x.insert(x.end(), b.cols[c]->as<double>(), b.cols[c]->as<double>() + b.n);
                out.cols.push_back(make_f64(std::move(x), std::move(v)));
                break;
            }
            default: {
                if (dict_all) {
                    std::vector<uint32_t> x;
                    x.reserve(total);
                    for (auto& b : bs) x.insert(x.end(), b.cols[c]->codes(), b.cols[c]->codes() + b.n);
                    out.cols.push_back(make_dict(bs[0].cols[c]->dictv, std::move(x), std::move(v)));
                } else {
                    Strings s;
                    for (auto& b : bs)
                        for (size_t i = 0; i < b.n; i++) s.push(b.cols[c]->str(i));
                    out.cols.push_back(make_utf8(std::move(s), std::move(v)));
                }
            }
        }
    }
    return out;
}

// ---- scalars ---------------------------------------------------------------------
int Scalar::data_type() const {
    switch (kind) {
        case NUL: return -1;
        case BOOLV: return BOOL;
        case I32V: return I32;
        case I64V: return I64;
        case F64V: return F64;
        case DATEV: return DATE;
        case UTF8V: return UTF8;
    }
    return -1;
}
std::optional<double> Scalar::as_f64() const {
    switch (kind) {
        case I32V: case I64V: case DATEV: return (double)i;
        case F64V: return f;
        default: return std::nullopt;
    }
}
std::optional<int64_t> Scalar::as_i64() const {
    switch (kind) {
        case I32V: case I64V: case DATEV: return i;
        default: return std::nullopt;
    }
}
std::optional<bool> Scalar::as_bool() const {
    if (kind == BOOLV) return i != 0;
    return std::nullopt;
}

// Rust `f as i64`: saturating, NaN -> 0.
static int64_t f64_as_i64(double f) {
    if (std::isnan(f)) return 0;
    if (f >= 9223372036854775808.0) return INT64_MAX;
    if (f <= -9223372036854775808.0) return INT64_MIN;
    return (int64_t)f;
}
static int32_t f64_as_i32(double f) {
    if (std::isnan(f)) return 0;
    if (f >= 2147483648.0) return INT32_MAX;
    if (f <= -2147483649.0) return INT32_MIN;
    return (int32_t)f;
}

// Rust's `{}` for f64: shortest round-trip digits, never exponent notation.
static std::string fmt_f64(double v) {
    if (std::isnan(v)) return "NaN";
    if (std::isinf(v)) return v > 0 ? "inf" : "-inf";
    char buf[512];
    auto r = std::to_chars(buf, buf + sizeof buf, v, std::chars_format::fixed);
    return std::string(buf, r.ptr);
}

std::string Scalar::to_string() const {
    switch (kind) {
        case NUL: return "NULL";
        case BOOLV: return i ? "true" : "false";
        case I32V: case I64V: return std::to_string(i);
        case F64V: return fmt_f64(f);
        case DATEV: return format_date((int32_t)i);
        case UTF8V: return s;
    }
    return "";
}

// scalar.rs:82-113
Scalar Scalar::cast_to(int to) const {
    if (is_null()) return Scalar();
    auto err = [&]() { fail(ML_ERR_INVALID, "cannot cast " + to_string() + " to " + dt_name(to)); };
    Scalar o;
    switch (to) {
        case BOOL: {
            auto b = as_bool();
            if (!b) err();
            return Scalar::b(*b);
        }
        case I32: {
            int64_t v;
            if (kind == F64V) v = f64_as_i64(f);
            else {
                auto x = as_i64();
                if (!x) err();
                v = *x;
            }
            if (v < INT32_MIN || v > INT32_MAX) err();
            o.kind = I32V;
            o.i = v;
            return o;
        }
        case I64: {
            if (kind == F64V) { o.kind = I64V; o.i = f64_as_i64(f); return o; }
            auto x = as_i64();
            if (!x) err();
            o.kind = I64V;
            o.i = *x;
            return o;
        }
        case F64: {
            auto x = as_f64();
            if (!x) err();
            o.kind = F64V;
            o.f = *x;
            return o;
        }
        case DATE: {
            if (kind == DATEV) return *this;
            if (kind == UTF8V) {
                auto d = parse_date(s);
                if (!d) err();
                o.kind = DATEV;
                o.i = *d;
                return o;
            }
            err();
        }
        case UTF8:
            o.kind = UTF8V;
            o.s = to_string();
            return o;
    }
    err();
    return o;
}

// scalar.rs:117-133 ; returns -1/0/1 or nullopt
std::optional<int> Scalar::compare(const Scalar& o) const {
    auto cmp = [](auto a, auto b) { return a < b ? -1 : (a > b ? 1 : 0); };
    if (is_null() || o.is_null()) return std::nullopt;
    if (kind == BOOLV && o.kind == BOOLV) return cmp(i, o.i);
    if (kind == UTF8V && o.kind == UTF8V) return cmp(s.compare(o.s), 0);
    if (kind == DATEV && o.kind == DATEV) return cmp(i, o.i);
    bool ia = kind == I32V || kind == I64V, ib = o.kind == I32V || o.kind == I64V;
    if (ia && ib) return cmp(i, o.i);
    auto a = as_f64(), b = o.as_f64();
    if (!a || !b) return std::nullopt;
    if (std::isnan(*a) || std::isnan(*b)) return std::nullopt;  // partial_cmp
    return cmp(*a, *b);
}

Scalar scalar_at(const Column& c, size_t i) {
    Scalar s;
    if (!c.valid(i)) return s;
    switch (c.dt) {
        case BOOL: s.kind = Scalar::BOOLV; s.i = c.as<uint8_t>()[i]; break;
        case I32: s.kind = Scalar::I32V; s.i = c.as<int32_t>()[i]; break;
        case DATE: s.kind = Scalar::DATEV; s.i = c.as<int32_t>()[i]; break;
        case I64: s.kind = Scalar::I64V; s.i = c.as<int64_t>()[i]; break;
        case F64: s.kind = Scalar::F64V; s.f = c.as<double>()[i]; break;
        default: s.kind = Scalar::UTF8V; s.s = std::string(c.str(i)); break;
    }
    return s;
}

// ---- date.rs: Howard Hinnant's days_from_civil / civil_from_days ---------------
int32_t days_from_civil(int32_t y, uint32_t m, uint32_t d) {
    y = m <= 2 ? y - 1 : y;
    int32_t era = (y >= 0 ? y : y - 399) / 400;
    uint32_t yoe = (uint32_t)(y - era * 400);
    uint32_t mp = (m + 9) % 12;
    uint32_t doy = (153 * mp + 2) / 5 + d - 1;
    uint32_t doe = yoe * 365 + yoe / 4 - yoe / 100 + doy;
    return era * 146097 + (int32_t)doe - 719468;
}
static void civil_from_days(int32_t z, int32_t& y, uint32_t& m, uint32_t& d) {
    z += 719468;
    int32_t era = (z >= 0 ? z : z - 146096) / 146097;
    uint32_t doe = (uint32_t)(z - era * 146097);
    uint32_t yoe = (doe - doe / 1460 + doe / 36524 - doe / 146096) / 365;
    y = (int32_t)yoe + era * 400;
    uint32_t doy = doe - (365 * yoe + yoe / 4 - yoe / 100);
    uint32_t mp = (5 * doy + 2) / 153;
    d = doy - (153 * mp + 2) / 5 + 1;
    m = mp < 10 ? mp + 3 : mp - 9;
    if (m <= 2) y += 1;
}
std::string format_date(int32_t days) {
    int32_t y;
    uint32_t m, d;
    civil_from_days(days, y, m, d);
    char buf[32];
    snprintf(buf, sizeof buf, "%04d-%02u-%02u", y, m, d);
    return buf;
}
static uint32_t days_in_month(int32_t y, uint32_t m) {
    bool leap = (y % 4 == 0 && y % 100 != 0) || y % 400 == 0;
    switch (m) {
        case 1: case 3: case 5: case 7: case 8: case 10: case 12: return 31;
        case 4: case 6: case 9: case 11: return 30;
        default: return leap ? 29 : 28;
    }
}
std::optional<int32_t> parse_date(std::string_view s) {
    while (!s.empty() && isspace((unsigned char)s.front())) s.remove_prefix(1);
    while (!s.empty() && isspace((unsigned char)s.back())) s.remove_suffix(1);
    long long p[3];
    int k = 0;
    size_t pos = 0;
    while (k < 3) {
        size_t e = s.find('-', pos == 0 && !s.empty() && s[0] == '-' ? 1 : pos);
        std::string_view part = s.substr(pos, e == std::string_view::npos ? std::string_view::npos : e - pos);
        if (part.empty()) return std::nullopt;
        long long v = 0;
        auto r = std::from_chars(part.data(), part.data() + part.size(), v);
        if (r.ec != std::errc() || r.ptr != part.data() + part.size()) return std::nullopt;
        p[k++] = v;
        if (e == std::string_view::npos) { pos = std::string_view::npos; break; }
        pos = e + 1;
    }
    if (k != 3 || pos != std::string_view::npos) return std::nullopt;
    if (p[1] < 1 || p[1] > 12 || p[2] < 1 || p[2] > (long long)days_in_month((int32_t)p[0], (uint32_t)p[1]))
        return std::nullopt;
    return days_from_civil((int32_t)p[0], (uint32_t)p[1], (uint32_t)p[2]);
}

// ---- like.rs:26-115 ----------------------------------------------------------------
LikePattern LikePattern::compile(std::string_view p) {
    LikePattern lp;
    bool has_us = p.find('_') != std::string_view::npos;
    auto inner = [](std::string_view s) { return s.find('%') == std::string_view::npos; };
    size_t n = p.size();
    if (!has_us) {
        if (p.find('%') == std::string_view::npos) {
            lp.shape = EXACT;
            lp.p = std::string(p);
            return lp;
        }
        if (n >= 2 && p[0] == '%' && p[n - 1] == '%' && inner(p.substr(1, n - 2))) {
            lp.shape = CONTAINS;
            lp.p = std::string(p.substr(1, n - 2));
            return lp;
        }
        if (p[n - 1] == '%' && inner(p.substr(0, n - 1))) {
            lp.shape = PREFIX;
            lp.p = std::string(p.substr(0, n - 1));
            return lp;
        }
        if (p[0] == '%' && inner(p.substr(1))) {
            lp.shape = SUFFIX;
            lp.p = std::string(p.substr(1));
            return lp;
        }
    }
    lp.shape = GENERAL;
    lp.p = std::string(p);
    return lp;
}
bool like_contains(std::string_view h, std::string_view nd) {
    if (nd.empty()) return true;
    if (nd.size() > h.size()) return false;
    return h.find(nd) != std::string_view::npos;
}
bool like_general(std::string_view s, std::string_view p) {
    size_t si = 0, pi = 0, star_s = 0;
    long star = -1;
    while (si < s.size()) {
        if (pi < p.size() && (p[pi] == '_' || p[pi] == s[si])) {
            si++;
            pi++;
        } else if (pi < p.size() && p[pi] == '%') {
            star = (long)pi;
            star_s = si;
            pi++;
        } else if (star >= 0) {
            pi = (size_t)star + 1;
            star_s++;
            si = star_s;
        } else {
            return false;
        }
    }
    while (pi < p.size() && p[pi] == '%') pi++;
    return pi == p.size();
}
bool LikePattern::matches(std::string_view s) const {
    switch (shape) {
        case EXACT: return s == p;
        case PREFIX: return s.size() >= p.size() && s.substr(0, p.size()) == p;
        case SUFFIX: return s.size() >= p.size() && s.substr(s.size() - p.size()) == p;
        case CONTAINS: return like_contains(s, p);
        default: return like_general(s, p);
    }
}

// ---- expression parsing ------------------------------------------------------------
static Expr parse_at(const ml_expr_node* nodes, int32_t nn, int32_t& pos) {
    if (pos >= nn) fail(ML_ERR_INVALID, "truncated expression");
    const ml_expr_node& nd = nodes[pos++];
    Expr e;
    e.kind = nd.kind;
    e.op = nd.op;
    e.dtype = nd.dtype;
    e.flag = nd.flag;
    e.index = nd.i64;
    if (nd.kind == ML_EXPR_LITERAL) {
        switch (nd.dtype) {
            case BOOL: e.lit = Scalar::b(nd.i64 != 0); break;
            case I32: e.lit.kind = Scalar::I32V; e.lit.i = (int32_t)nd.i64; break;
            case I64: e.lit.kind = Scalar::I64V; e.lit.i = nd.i64; break;
            case F64: e.lit.kind = Scalar::F64V; e.lit.f = nd.f64; break;
            case DATE: e.lit.kind = Scalar::DATEV; e.lit.i = (int32_t)nd.i64; break;
            case UTF8: e.lit.kind = Scalar::UTF8V; e.lit.s.assign(nd.str, (size_t)nd.str_len); break;
            default: e.lit = Scalar(); break;
        }
    }
    if (nd.kind == ML_EXPR_LIKE) e.like = LikePattern::compile(std::string_view(nd.str, (size_t)nd.str_len));
    for (int k = 0; k < nd.nchild; k++) e.kids.push_back(parse_at(nodes, nn, pos));
    return e;
}
Expr parse_nodes(const ml_expr_node* nodes, int32_t nnodes) {
    int32_t pos = 0;
    Expr e = parse_at(nodes, nnodes, pos);
    if (pos != nnodes) fail(ML_ERR_INVALID, "trailing expression nodes");
    return e;
}
Expr parse_expr(const ml_expr& e) { return parse_nodes(e.nodes, e.nnodes); }

// expr/mod.rs:199-234
int Expr::data_type(const std::vector<int>& schema) const {
    switch (kind) {
        case ML_EXPR_COLUMN:
            if (index < 0 || (size_t)index >= schema.size()) fail(ML_ERR_INVALID, "column out of range");
            return schema[index];
        case ML_EXPR_LITERAL: {
            int t = lit.data_type();
            return t < 0 ? I64 : t;
        }
        case ML_EXPR_BINARY: {
            if ((op >= ML_BIN_EQ && op <= ML_BIN_GTEQ) || op == ML_BIN_AND || op == ML_BIN_OR) return BOOL;
            if (op == ML_BIN_DIV) return F64;
            int l = kids[0].data_type(schema), r = kids[1].data_type(schema);
            if (l == DATE || r == DATE) return DATE;
            int s = numeric_supertype(l, r);
            return s < 0 ? l : s;
        }
        case ML_EXPR_NOT: case ML_EXPR_IS_NULL: case ML_EXPR_LIKE: case ML_EXPR_IN_LIST: return BOOL;
        case ML_EXPR_NEGATE: return kids[0].data_type(schema);
        case ML_EXPR_CASE: case ML_EXPR_CAST: return dtype;
    }
    fail(ML_ERR_INVALID, "bad expression kind");
}

// ---- kernels ------------------------------------------------------------------------
static bool is_cmp(int op) { return op >= ML_BIN_EQ && op <= ML_BIN_GTEQ; }
static int flip(int op) {  // expr/mod.rs:77-85
    switch (op) {
        case ML_BIN_LT: return ML_BIN_GT;
        case ML_BIN_LTEQ: return ML_BIN_GTEQ;
        case ML_BIN_GT: return ML_BIN_LT;
        case ML_BIN_GTEQ: return ML_BIN_LTEQ;
    }
    return op;
}
template <class T> static inline bool cmp_op(int op, T a, T b) {
    switch (op) {
        case ML_BIN_EQ: return a == b;
        case ML_BIN_NOTEQ: return a != b;
        case ML_BIN_LT: return a < b;
        case ML_BIN_LTEQ: return a <= b;
        case ML_BIN_GT: return a > b;
        default: return a >= b;
    }
}
static bool compare_bytes(int op, std::string_view a, std::string_view b) {  // cmp.rs:35-45
    int c = a.compare(b);
    switch (op) {
        case ML_BIN_EQ: return c == 0;
        case ML_BIN_NOTEQ: return c != 0;
        case ML_BIN_LT: return c < 0;
        case ML_BIN_LTEQ: return c <= 0;
        case ML_BIN_GT: return c > 0;
        case ML_BIN_GTEQ: return c >= 0;
    }
    return false;
}

// An operand: slice or scalar (kernels/mod.rs:26-37)
template <class T> struct Operand {
    const T* p = nullptr;
    T s{};
    T at(size_t i) const { return p ? p[i] : s; }
};

// cmp.rs:85-118
std::vector<uint32_t> mask_to_selection(const uint8_t* mask, size_t n, const Column* validity,
                                        const std::vector<uint32_t>* input) {
    std::vector<uint32_t> out;
    if (!input) {
        out.resize(n);
        size_t k = 0;
        if (!validity || !validity->vw) {
            for (size_t i = 0; i < n; i++) {
                out[k] = (uint32_t)i;
                k += mask[i] & 1;
            }
        } else {
            for (size_t i = 0; i < n; i++) {
                out[k] = (uint32_t)i;
                k += (mask[i] & validity->valid(i)) & 1;
            }
        }
        out.resize(k);
        return out;
    }
    out.reserve(input->size());
    for (uint32_t i : *input)
        if (mask[i] && (!validity || validity->valid(i))) out.push_back(i);
    return out;
}

static std::optional<Bitmap> combine_validity(const Column* a, const Column* b) {  // bitmap.rs:160-167
    bool va = a && a->vw, vb = b && b->vw;
    if (!va && !vb) return std::nullopt;
    size_t n = va ? a->n : b->n;
    Bitmap out = Bitmap::unset_all(n);
    for (size_t i = 0; i < n; i++) {
        bool v = (!va || a->valid(i)) && (!vb || b->valid(i));
        if (v) out.words[i / 64] |= 1ull << (i % 64);
    }
    return out;
}

// cast.rs:6-73
ColPtr cast_column(const ColPtr& c, int to) {
    int from = c->dt;
    if (from == to) return c;
    std::optional<Bitmap> v = validity_of(*c);
    size_t n = c->n;
    auto unsupported = [&]() {
        fail(ML_ERR_UNSUPPORTED, std::string("cast from ") + dt_name(from) + " to " + dt_name(to));
    };
    if (to == UTF8) {
        Strings s;
        for (size_t i = 0; i < n; i++) s.push(scalar_at(*c, i).to_string());
        return make_utf8(std::move(s), std::move(v));
    }
    switch (from) {
        case I32:
        case DATE: {
            const int32_t* x = c->as<int32_t>();
            if (to == I64 || (from == DATE && to == I64)) {
                std::vector<int64_t> o(x, x + n);
                return make_i64(std::move(o), std::move(v));
            }
            if (to == F64 && from == I32) {
                std::vector<double> o(n);
                for (size_t i = 0; i < n; i++) o[i] = (double)x[i];
                return make_f64(std::move(o), std::move(v));
            }
            if ((from == I32 && to == DATE) || (from == DATE && to == I32))
                return make_i32(std::vector<int32_t>(x, x + n), std::move(v), to);
            unsupported();
        }
        case I64: {
            const int64_t* x = c->as<int64_t>();
            if (to == I32) {
                std::vector<int32_t> o(n);
                for (size_t i = 0; i < n; i++) o[i] = (int32_t)(uint32_t)(uint64_t)x[i];
                return make_i32(std::move(o), std::move(v));
            }
            if (to == F64) {
                std::vector<double> o(n);
                for (size_t i = 0; i < n; i++) o[i] = (double)x[i];
                return make_f64(std::move(o), std::move(v));
            }
            unsupported();
        }
        case F64: {
            const double* x = c->as<double>();
            if (to == I64) {
                std::vector<int64_t> o(n);
                for (size_t i = 0; i < n; i++) o[i] = f64_as_i64(x[i]);
                return make_i64(std::move(o), std::move(v));
            }
            if (to == I32) {
                std::vector<int32_t> o(n);
                for (size_t i = 0; i < n; i++) o[i] = f64_as_i32(x[i]);
                return make_i32(std::move(o), std::move(v));
            }
            unsupported();
        }
        case BOOL: {
            const uint8_t* x = c->as<uint8_t>();
            if (to == I32) return make_i32(std::vector<int32_t>(x, x + n), std::move(v));
            if (to == I64) return make_i64(std::vector<int64_t>(x, x + n), std::move(v));
            if (to == F64) {
                std::vector<double> o(n);
                for (size_t i = 0; i < n; i++) o[i] = (double)x[i];
                return make_f64(std::move(o), std::move(v));
            }
            unsupported();
        }
        case UTF8: {
            if (to == DATE) {
                std::vector<int32_t> o(n);
                for (size_t i = 0; i < n; i++) {
                    if (c->valid(i)) {
                        auto d = parse_date(c->str(i));
                        if (!d) fail(ML_ERR_INVALID, "cannot cast '" + std::string(c->str(i)) + "' to DATE");
                        o[i] = *d;
                    }
                }
                return make_i32(std::move(o), std::move(v), DATE);
            }
            unsupported();
        }
    }
    unsupported();
    return c;
}

// Column::from_scalar (column.rs:286-310)
static ColPtr column_from_scalar(const Scalar& s0, size_t n, int dt) {
    if (s0.is_null()) return nulls_column(dt, n);
    Scalar s = s0.cast_to(dt);
    switch (dt) {
        case BOOL: return make_bool(std::vector<uint8_t>(n, (uint8_t)s.i), std::nullopt);
        case I32: case DATE: return make_i32(std::vector<int32_t>(n, (int32_t)s.i), std::nullopt, dt);
        case I64: return make_i64(std::vector<int64_t>(n, s.i), std::nullopt);
        case F64: return make_f64(std::vector<double>(n, s.f), std::nullopt);
        default: {
            auto d = std::make_shared<Strings>();
            d->push(s.s);
            return make_dict(d, std::vector<uint32_t>(n, 0), std::nullopt);
        }
    }
}

static Datum arr(ColPtr c) { Datum d; d.col = std::move(c); return d; }
static Datum sca(Scalar s) { Datum d; d.scalar = true; d.s = std::move(s); return d; }
static int datum_type(const Datum& d) { return d.scalar ? d.s.data_type() : d.col->dt; }

static Datum cast_datum(const Datum& d, int to) {  // eval.rs:202-208
    if (d.scalar) return sca(d.s.cast_to(to));
    if (d.col->dt == to) return d;
    return arr(cast_column(d.col, to));
}
static ColPtr into_column(const Datum& d, size_t n, int dt) {  // eval.rs:44-49
    if (!d.scalar) return d.col;
    return column_from_scalar(d.s, n, dt);
}

// scalar_ops.rs:12-128
static std::optional<int64_t> int_op(int op, int64_t a, int64_t b) {
    int64_t r;
    switch (op) {
        case ML_BIN_ADD: if (__builtin_add_overflow(a, b, &r)) return std::nullopt; return r;
        case ML_BIN_SUB: if (__builtin_sub_overflow(a, b, &r)) return std::nullopt; return r;
        case ML_BIN_MUL: if (__builtin_mul_overflow(a, b, &r)) return std::nullopt; return r;
        case ML_BIN_MOD:
            if (b == 0) fail(ML_ERR_INVALID, "modulo by zero");
            if (a == INT64_MIN && b == -1) return std::nullopt;
            return a % b;
    }
    return std::nullopt;
}
Scalar scalar_binary(int op, const Scalar& l, const Scalar& r) {
    if (op == ML_BIN_AND) {
        auto a = l.as_bool(), b = r.as_bool();
        if ((a && !*a) || (b && !*b)) return Scalar::b(false);
        if (a && b && *a && *b) return Scalar::b(true);
        return Scalar();
    }
    if (op == ML_BIN_OR) {
        auto a = l.as_bool(), b = r.as_bool();
        if ((a && *a) || (b && *b)) return Scalar::b(true);
        if (a && b && !*a && !*b) return Scalar::b(false);
        return Scalar();
    }
    if (l.is_null() || r.is_null()) return Scalar();
    if (is_cmp(op)) {
        auto o = l.compare(r);
        if (!o) fail(ML_ERR_INVALID, "cannot compare " + l.to_string() + " with " + r.to_string());
        return Scalar::b(cmp_op(op, *o, 0));
    }
    auto overflow = [&]() { fail(ML_ERR_INVALID, "overflow in " + l.to_string() + " op " + r.to_string()); };
    if (l.kind == Scalar::DATEV && (r.kind == Scalar::I32V || r.kind == Scalar::I64V) &&
        (op == ML_BIN_ADD || op == ML_BIN_SUB)) {
        int64_t v = op == ML_BIN_ADD ? l.i + r.i : l.i - r.i;
        if (v < INT32_MIN || v > INT32_MAX) overflow();
        Scalar o;
        o.kind = Scalar::DATEV;
        o.i = v;
        return o;
    }
    if (l.kind == Scalar::DATEV && r.kind == Scalar::DATEV && op == ML_BIN_SUB) {
        Scalar o;
        o.kind = Scalar::I64V;
        o.i = l.i - r.i;
        return o;
    }
    if (op == ML_BIN_DIV) {
        auto a = l.as_f64(), b = r.as_f64();
        if (!a || !b) fail(ML_ERR_INVALID, "not numeric");
        if (*b == 0.0) return Scalar();
        Scalar o;
        o.kind = Scalar::F64V;
        o.f = *a / *b;
        return o;
    }
    if (l.kind == Scalar::I32V && r.kind == Scalar::I32V) {
        auto v = int_op(op, l.i, r.i);
        if (!v) overflow();
        Scalar o;
        o.kind = (*v >= INT32_MIN && *v <= INT32_MAX) ? Scalar::I32V : Scalar::I64V;
        o.i = *v;
        return o;
    }
    bool li = l.kind == Scalar::I32V || l.kind == Scalar::I64V;
    bool ri = r.kind == Scalar::I32V || r.kind == Scalar::I64V;
    if (li && ri) {
        auto v = int_op(op, l.i, r.i);
        if (!v) overflow();
        Scalar o;
        o.kind = Scalar::I64V;
        o.i = *v;
        return o;
    }
    auto a = l.as_f64(), b = r.as_f64();
    if (!a || !b) fail(ML_ERR_INVALID, "not numeric");
    Scalar o;
    o.kind = Scalar::F64V;
    switch (op) {
        case ML_BIN_ADD: o.f = *a + *b; break;
        case ML_BIN_SUB: o.f = *a - *b; break;
        case ML_BIN_MUL: o.f = *a * *b; break;
        case ML_BIN_MOD: o.f = std::fmod(*a, *b); break;
        default: fail(ML_ERR_INTERNAL, "scalar op");
    }
    return o;
}
static Scalar scalar_negate(const Scalar& v) {  // scalar_ops.rs:131-140
    Scalar o = v;
    switch (v.kind) {
        case Scalar::NUL: return v;
        case Scalar::I32V: o.i = (int32_t)(-(int64_t)v.i); return o;
        case Scalar::I64V: o.i = (int64_t)(0 - (uint64_t)v.i); return o;
        case Scalar::F64V: o.f = -v.f; return o;
        default: fail(ML_ERR_INVALID, "cannot negate " + v.to_string());
    }
}

// eval.rs:218-228
static int common_type(int l, int r) {
    if (l == r) return l;
    if ((l == DATE && r == UTF8) || (l == UTF8 && r == DATE)) return DATE;
    if ((l == DATE && (r == I32 || r == I64)) || (r == DATE && (l == I32 || l == I64))) return I32;
    return numeric_supertype(l, r);
}

template <class T> static Operand<T> operand(const Datum& d) {
    Operand<T> o;
    if (d.scalar) {
        if constexpr (std::is_same_v<T, double>) {
            auto v = d.s.as_f64();
            if (!v) fail(ML_ERR_INVALID, "expected f64 constant");
            o.s = *v;
        } else if constexpr (std::is_same_v<T, uint8_t>) {
            auto v = d.s.as_bool();
            if (!v) fail(ML_ERR_INVALID, "expected bool constant");
            o.s = *v;
        } else {
            auto v = d.s.as_i64();
            if (!v) fail(ML_ERR_INVALID, "expected integer constant");
            o.s = (T)*v;
        }
    } else {
        o.p = d.col->as<T>();
    }
    return o;
}

// mask_zero_divisors (eval.rs:303-324)
template <class T>
static std::optional<Bitmap> mask_zero(std::optional<Bitmap> validity, const Operand<T>& d, size_t n) {
    if (!d.p) {
        if (d.s == T(0)) return Bitmap::unset_all(n);
        return validity;
    }
    bool any = false;
    for (size_t i = 0; i < n && !any; i++) any = d.p[i] == T(0);
    if (!any) return validity;
    Bitmap bm = validity ? *validity : Bitmap::set_all(n);
    for (size_t i = 0; i < n; i++)
        if (d.p[i] == T(0)) bm.set(i, false);
    return bm;
}

template <class T> static T arith1(int op, T a, T b) {  // arith.rs:14-92
    if constexpr (std::is_same_v<T, double>) {
        switch (op) {
            case ML_BIN_ADD: return a + b;
            case ML_BIN_SUB: return a - b;
            case ML_BIN_MUL: return a * b;
            default: return std::fmod(a, b);
        }
    } else {
        using U = std::make_unsigned_t<T>;
        switch (op) {
            case ML_BIN_ADD: return (T)((U)a + (U)b);
            case ML_BIN_SUB: return (T)((U)a - (U)b);
            case ML_BIN_MUL: return (T)((U)a * (U)b);
            default:
                if (b == 0) return 0;
                if (b == -1) return 0;  // wrapping_rem(MIN, -1) == 0 ; x % -1 == 0
                return a % b;
        }
    }
}

static Datum bool_array(std::vector<uint8_t>&& m, std::optional<Bitmap>&& v) {
    return arr(make_bool(std::move(m), std::move(v)));
}

static Datum logical(int op, const Datum& l, const Datum& r, size_t n) {  // eval.rs:348-360
    ColPtr a = into_column(l, n, BOOL), b = into_column(r, n, BOOL);
    if (a->dt != BOOL || b->dt != BOOL) fail(ML_ERR_INVALID, "AND/OR on non-boolean");
    const uint8_t *av = a->as<uint8_t>(), *bv = b->as<uint8_t>();
    std::vector<uint8_t> vals(n);
    for (size_t i = 0; i < n; i++) vals[i] = op == ML_BIN_AND ? (av[i] & bv[i]) : (av[i] | bv[i]);
    if (!a->vw && !b->vw) return bool_array(std::move(vals), std::nullopt);
    std::vector<uint8_t> bits(n);  // boolean.rs:18-58
    for (size_t i = 0; i < n; i++) {
        bool va = a->valid(i), vb = b->valid(i);
        if (op == ML_BIN_AND)
            bits[i] = (va && vb) || (va && !av[i]) || (vb && !bv[i]);
        else
            bits[i] = (va && vb) || (va && av[i]) || (vb && bv[i]);
    }
    return bool_array(std::move(vals), Bitmap::from_bools(bits));
}

static std::vector<uint8_t> compare_string_scalar(int op, const Column& c, std::string_view s) {
    std::vector<uint8_t> m(c.n);  // cmp.rs:52-61
    if (c.dict) {
        std::vector<uint8_t> per(c.dictv->len());
        for (size_t e = 0; e < per.size(); e++) per[e] = compare_bytes(op, c.dictv->get(e), s);
        for (size_t i = 0; i < c.n; i++) m[i] = per[c.codes()[i]];
    } else {
        for (size_t i = 0; i < c.n; i++) m[i] = compare_bytes(op, c.str(i), s);
    }
    return m;
}

static std::vector<uint8_t> comparison(int op, const Datum& l, const Datum& r, size_t n, int ct) {
    std::vector<uint8_t> m(n);  // eval.rs:326-346
    auto run = [&](auto a, auto b) {
        for (size_t i = 0; i < n; i++) m[i] = cmp_op(op, a.at(i), b.at(i));
    };
    switch (ct) {
        case I32: case DATE: run(operand<int32_t>(l), operand<int32_t>(r)); return m;
        case I64: run(operand<int64_t>(l), operand<int64_t>(r)); return m;
        case F64: run(operand<double>(l), operand<double>(r)); return m;
        case BOOL: run(operand<uint8_t>(l), operand<uint8_t>(r)); return m;
    }
    if (!l.scalar && r.scalar && r.s.kind == Scalar::UTF8V) return compare_string_scalar(op, *l.col, r.s.s);
    if (l.scalar && !r.scalar && l.s.kind == Scalar::UTF8V) return compare_string_scalar(flip(op), *r.col, l.s.s);
    if (!l.scalar && !r.scalar) {
        for (size_t i = 0; i < n; i++) m[i] = compare_bytes(op, l.col->str(i), r.col->str(i));
        return m;
    }
    if (l.scalar && r.scalar) {
        bool v = compare_bytes(op, l.s.to_string(), r.s.to_string());
        std::fill(m.begin(), m.end(), v);
        return m;
    }
    fail(ML_ERR_INTERNAL, "string comparison operands");
}

static Datum binary(int op, Datum l, Datum r, size_t n) {  // eval.rs:230-301
    if (l.scalar && r.scalar) return sca(scalar_binary(op, l.s, r.s));
    if (op == ML_BIN_AND || op == ML_BIN_OR) return logical(op, l, r, n);
    if ((l.scalar && l.s.is_null()) || (r.scalar && r.s.is_null())) return sca(Scalar());
    int lt = datum_type(l), rt = datum_type(r);
    if (lt < 0) lt = I64;
    if (rt < 0) rt = I64;
    int ct = common_type(lt, rt);
    if (ct < 0) fail(ML_ERR_INVALID, std::string("incompatible types ") + dt_name(lt) + " " + dt_name(rt));
    bool arith_op = op <= ML_BIN_MOD;
    bool date_result = arith_op && (lt == DATE || rt == DATE);
    bool date_diff = op == ML_BIN_SUB && lt == DATE && rt == DATE;
    l = cast_datum(l, ct);
    r = cast_datum(r, ct);
    std::optional<Bitmap> validity = combine_validity(l.scalar ? nullptr : l.col.get(), r.scalar ? nullptr : r.col.get());
    if (is_cmp(op)) return bool_array(comparison(op, l, r, n, ct), std::move(validity));
    if (op == ML_BIN_DIV) {
        l = cast_datum(l, F64);
        r = cast_datum(r, F64);
        auto a = operand<double>(l), b = operand<double>(r);
        std::vector<double> v(n);
        for (size_t i = 0; i < n; i++) v[i] = a.at(i) / b.at(i);
        return arr(make_f64(std::move(v), mask_zero(std::move(validity), b, n)));
    }
    switch (ct) {
        case I32:
        case DATE: {
            auto a = operand<int32_t>(l), b = operand<int32_t>(r);
            std::vector<int32_t> v(n);
            for (size_t i = 0; i < n; i++) v[i] = arith1<int32_t>(op, a.at(i), b.at(i));
            if (op == ML_BIN_MOD) validity = mask_zero(std::move(validity), b, n);
            int dt = date_diff ? I32 : (date_result ? DATE : I32);
            return arr(make_i32(std::move(v), std::move(validity), dt));
        }
        case I64: {
            auto a = operand<int64_t>(l), b = operand<int64_t>(r);
            std::vector<int64_t> v(n);
            for (size_t i = 0; i < n; i++) v[i] = arith1<int64_t>(op, a.at(i), b.at(i));
            if (op == ML_BIN_MOD) validity = mask_zero(std::move(validity), b, n);
            return arr(make_i64(std::move(v), std::move(validity)));
        }
        case F64: {
            auto a = operand<double>(l), b = operand<double>(r);
            std::vector<double> v(n);
            for (size_t i = 0; i < n; i++) v[i] = arith1<double>(op, a.at(i), b.at(i));
            return arr(make_f64(std::move(v), std::move(validity)));
        }
    }
    fail(ML_ERR_INVALID, std::string("arithmetic on ") + dt_name(ct) + " is not supported");
}

static Datum in_list(const Datum& d, const std::vector<Scalar>& list, bool negated) {  // eval.rs:393-448
    if (d.scalar) {
        if (d.s.is_null()) return sca(Scalar());
        bool hit = false;
        for (auto& v : list) {
            auto o = d.s.compare(v);
            hit |= o && *o == 0;
        }
        return sca(Scalar::b(hit != negated));
    }
    const Column& c = *d.col;
    size_t n = c.n;
    std::vector<uint8_t> mask(n);
    int dt = c.dt;
    auto cast_list = [&]() {
        std::vector<Scalar> out;
        for (auto& v : list) out.push_back(v.cast_to(dt));
        return out;
    };
    if (dt == UTF8) {
        std::vector<std::string> items;
        for (auto& v : list)
            if (v.kind == Scalar::UTF8V) items.push_back(v.s);
        auto hit = [&](std::string_view s) {
            for (auto& x : items) if (x == s) return true;
            return false;
        };
        if (c.dict) {
            std::vector<uint8_t> per(c.dictv->len());
            for (size_t e = 0; e < per.size(); e++) per[e] = hit(c.dictv->get(e));
            for (size_t i = 0; i < n; i++) mask[i] = per[c.codes()[i]];
        } else {
            for (size_t i = 0; i < n; i++) mask[i] = hit(c.str(i));
        }
    } else if (dt == I32 || dt == DATE) {
        std::vector<int32_t> items;
        for (auto& s : cast_list()) if (auto x = s.as_i64()) items.push_back((int32_t)*x);
        for (size_t i = 0; i < n; i++)
            mask[i] = std::find(items.begin(), items.end(), c.as<int32_t>()[i]) != items.end();
    } else if (dt == I64) {
        std::vector<int64_t> items;
        for (auto& s : cast_list()) if (auto x = s.as_i64()) items.push_back(*x);
        for (size_t i = 0; i < n; i++)
            mask[i] = std::find(items.begin(), items.end(), c.as<int64_t>()[i]) != items.end();
    } else if (dt == F64) {
        std::vector<double> items;
        for (auto& s : cast_list()) if (auto x = s.as_f64()) items.push_back(*x);
        for (size_t i = 0; i < n; i++)
            mask[i] = std::find(items.begin(), items.end(), c.as<double>()[i]) != items.end();
    } else {
        std::vector<uint8_t> items;
        for (auto& s : list) if (auto x = s.as_bool()) items.push_back(*x);
        for (size_t i = 0; i < n; i++)
            mask[i] = std::find(items.begin(), items.end(), c.as<uint8_t>()[i]) != items.end();
    }
    if (negated)
        for (auto& m : mask) m = !m;
    return bool_array(std::move(mask), validity_of(c));
}

static Datum case_expr(const Expr& e, const Batch& b) {  // eval.rs:466-532
    size_t n = b.n;
    size_t k = e.kids.size() / 2;
    bool has_else = e.flag != 0;
    int dt = e.dtype;
    std::vector<uint32_t> choice(n, (uint32_t)k);
    std::vector<uint8_t> decided(n, 0);
    for (size_t bi = 0; bi < k; bi++) {
        ColPtr c = into_column(evaluate(e.kids[2 * bi], b), n, BOOL);
        if (c->dt != BOOL) fail(ML_ERR_INVALID, "CASE condition is not boolean");
        for (size_t i = 0; i < n; i++) {
            bool take = !decided[i] && c->as<uint8_t>()[i] && c->valid(i);
            if (take) {
                choice[i] = (uint32_t)bi;
                decided[i] = 1;
            }
        }
    }
    std::vector<ColPtr> values;
    for (size_t bi = 0; bi < k; bi++) values.push_back(evaluate_to_column(e.kids[2 * bi + 1], b, dt));
    values.push_back(has_else ? evaluate_to_column(e.kids[2 * k], b, dt) : nulls_column(dt, n));
    std::vector<uint8_t> valid(n);
    for (size_t i = 0; i < n; i++) valid[i] = values[choice[i]]->valid(i);
    switch (dt) {
        case BOOL: {
            std::vector<uint8_t> o(n);
            for (size_t i = 0; i < n; i++) o[i] = values[choice[i]]->as<uint8_t>()[i];
            return arr(make_bool(std::move(o), Bitmap::from_bools(valid)));
        }
        case I32: case DATE: {
            std::vector<int32_t> o(n);
            for (size_t i = 0; i < n; i++) o[i] = values[choice[i]]->as<int32_t>()[i];
            return arr(make_i32(std::move(o), Bitmap::from_bools(valid), dt));
        }
        case I64: {
            std::vector<int64_t> o(n);
            for (size_t i = 0; i < n; i++) o[i] = values[choice[i]]->as<int64_t>()[i];
            return arr(make_i64(std::move(o), Bitmap::from_bools(valid)));
        }
        case F64: {
            std::vector<double> o(n);
            for (size_t i = 0; i < n; i++) o[i] = values[choice[i]]->as<double>()[i];
            return arr(make_f64(std::move(o), Bitmap::from_bools(valid)));
        }
        default: {
            Strings s;
            for (size_t i = 0; i < n; i++) s.push(values[choice[i]]->str(i));
            return arr(make_utf8(std::move(s), Bitmap::from_bools(valid)));
        }
    }
}

// eval.rs:61-151
Datum evaluate(const Expr& e, const Batch& b) {
    size_t n = b.n;
    switch (e.kind) {
        case ML_EXPR_COLUMN:
            if (e.index < 0 || (size_t)e.index >= b.cols.size())
                fail(ML_ERR_INTERNAL, "column #" + std::to_string(e.index) + " missing");
            return arr(b.cols[e.index]);
        case ML_EXPR_LITERAL: return sca(e.lit);
        case ML_EXPR_BINARY: return binary(e.op, evaluate(e.kids[0], b), evaluate(e.kids[1], b), n);
        case ML_EXPR_NOT: {
            Datum d = evaluate(e.kids[0], b);
            if (d.scalar) {
                auto v = d.s.as_bool();
                return sca(v ? Scalar::b(!*v) : Scalar());
            }
            if (d.col->dt != BOOL) fail(ML_ERR_INVALID, "NOT of non-boolean");
            std::vector<uint8_t> o(n);
            for (size_t i = 0; i < n; i++) o[i] = !d.col->as<uint8_t>()[i];
            return bool_array(std::move(o), validity_of(*d.col));
        }
        case ML_EXPR_NEGATE: {
            Datum d = evaluate(e.kids[0], b);
            if (d.scalar) return sca(scalar_negate(d.s));
            const Column& c = *d.col;
            switch (c.dt) {
                case I32: {
                    std::vector<int32_t> o(n);
                    for (size_t i = 0; i < n; i++) o[i] = (int32_t)(0u - (uint32_t)c.as<int32_t>()[i]);
                    return arr(make_i32(std::move(o), validity_of(c)));
                }
                case I64: {
                    std::vector<int64_t> o(n);
                    for (size_t i = 0; i < n; i++) o[i] = (int64_t)(0ull - (uint64_t)c.as<int64_t>()[i]);
                    return arr(make_i64(std::move(o), validity_of(c)));
                }
                case F64: {
                    std::vector<double> o(n);
                    for (size_t i = 0; i < n; i++) o[i] = -c.as<double>()[i];
                    return arr(make_f64(std::move(o), validity_of(c)));
                }
            }
            fail(ML_ERR_INVALID, "cannot negate");
        }
        case ML_EXPR_IS_NULL: {
            Datum d = evaluate(e.kids[0], b);
            bool negated = e.flag != 0;
            if (d.scalar) return sca(Scalar::b(d.s.is_null() != negated));
            std::vector<uint8_t> o(d.col->n);
            for (size_t i = 0; i < d.col->n; i++) o[i] = d.col->valid(i) == negated;
            return bool_array(std::move(o), std::nullopt);
        }
        case ML_EXPR_LIKE: {
            Datum d = evaluate(e.kids[0], b);
            bool negated = e.flag != 0;
            if (d.scalar) {
                if (d.s.kind == Scalar::UTF8V) return sca(Scalar::b(e.like.matches(d.s.s) != negated));
                return sca(Scalar());
            }
            const Column& c = *d.col;
            std::vector<uint8_t> m(c.n, 0);  // string.rs:11-20
            if (c.dt == UTF8 && c.dict) {
                std::vector<uint8_t> per(c.dictv->len());
                for (size_t k = 0; k < per.size(); k++) per[k] = e.like.matches(c.dictv->get(k));
                for (size_t i = 0; i < c.n; i++) m[i] = per[c.codes()[i]];
            } else if (c.dt == UTF8) {
                for (size_t i = 0; i < c.n; i++) m[i] = e.like.matches(c.str(i));
            }
            if (negated)
                for (auto& x : m) x = !x;
            return bool_array(std::move(m), validity_of(c));
        }
        case ML_EXPR_IN_LIST: {
            std::vector<Scalar> list;
            for (size_t k = 1; k < e.kids.size(); k++) list.push_back(e.kids[k].lit);
            return in_list(evaluate(e.kids[0], b), list, e.flag != 0);
        }
        case ML_EXPR_CASE: return case_expr(e, b);
        case ML_EXPR_CAST: return cast_datum(evaluate(e.kids[0], b), e.dtype);
    }
    fail(ML_ERR_INVALID, "bad expression");
}

ColPtr evaluate_to_column(const Expr& e, const Batch& b, int dt) {
    ColPtr c = into_column(evaluate(e, b), b.n, dt);
    if (c->dt != dt) return cast_column(c, dt);
    return c;
}

// eval.rs:167-196
std::vector<uint32_t> select(const Expr& e, const Batch& b, const std::vector<uint32_t>* input) {
    if (e.kind == ML_EXPR_BINARY && e.op == ML_BIN_AND) {
        std::vector<uint32_t> sel = select(e.kids[0], b, input);
        if (sel.empty()) return sel;
        return select(e.kids[1], b, &sel);
    }
    auto all = [&]() {
        if (input) return *input;
        std::vector<uint32_t> v(b.n);
        for (size_t i = 0; i < b.n; i++) v[i] = (uint32_t)i;
        return v;
    };
    Datum d = evaluate(e, b);
    if (d.scalar) {
        if (d.s.kind == Scalar::BOOLV && d.s.i) return all();
        return {};
    }
    if (d.col->dt != BOOL) fail(ML_ERR_INVALID, "filter predicate is not boolean");
    return mask_to_selection(d.col->as<uint8_t>(), d.col->n, d.col.get(), input);
}

// ---- kernels/hash.rs:16-101 ---------------------------------------------------------
void hash_columns(const std::vector<ColPtr>& cols, size_t n, const uint32_t* rows, size_t k,
                  std::vector<uint64_t>& out) {
    size_t m = rows ? k : n;
    out.assign(m, SEED);
    for (auto& cp : cols) {
        const Column& c = *cp;
        auto row = [&](size_t j) -> size_t { return rows ? rows[j] : j; };
        auto mix = [&](auto to_u64) {
            if (!rows && !c.vw) {
                for (size_t j = 0; j < m; j++) out[j] = combine(out[j], hash_u64(to_u64(j)));
            } else {
                for (size_t j = 0; j < m; j++) {
                    size_t r = row(j);
                    uint64_t x = c.valid(r) ? hash_u64(to_u64(r)) : NULL_HASH;
                    out[j] = combine(out[j], x);
                }
            }
        };
        switch (c.dt) {
            case I32: case DATE: {
                const int32_t* v = c.as<int32_t>();
                mix([&](size_t r) { return (uint64_t)(int64_t)v[r]; });
                break;
            }
            case I64: {
                const int64_t* v = c.as<int64_t>();
                mix([&](size_t r) { return (uint64_t)v[r]; });
                break;
            }
            case F64: {
                const double* v = c.as<double>();
                mix([&](size_t r) {
                    double x = v[r];
                    uint64_t bits;
                    memcpy(&bits, &x, 8);
                    return x == 0.0 ? 0ull : bits;
                });
                break;
            }
            case BOOL: {
                const uint8_t* v = c.as<uint8_t>();
                mix([&](size_t r) { return (uint64_t)v[r]; });
                break;
            }
            default: {
                if (c.dict) {
                    std::vector<uint64_t> dh(c.dictv->len());
                    for (size_t e = 0; e < dh.size(); e++) {
                        auto s = c.dictv->get(e);
                        dh[e] = hash_bytes((const uint8_t*)s.data(), s.size());
                    }
                    for (size_t j = 0; j < m; j++) {
                        size_t r = row(j);
                        out[j] = combine(out[j], c.valid(r) ? dh[c.codes()[r]] : NULL_HASH);
                    }
                } else {
                    for (size_t j = 0; j < m; j++) {
                        size_t r = row(j);
                        uint64_t x = NULL_HASH;
                        if (c.valid(r)) {
                            auto s = c.str(r);
                            x = hash_bytes((const uint8_t*)s.data(), s.size());
                        }
                        out[j] = combine(out[j], x);
                    }
                }
            }
        }
    }
}

bool values_equal(const Column& x, size_t a, const Column& y, size_t b) {
    bool va = x.valid(a), vb = y.valid(b);
    if (!va && !vb) return true;
    if (va != vb) return false;
    if ((x.dt == I32 && y.dt == I32) || (x.dt == DATE && y.dt == DATE)) return x.as<int32_t>()[a] == y.as<int32_t>()[b];
    if (x.dt == I64 && y.dt == I64) return x.as<int64_t>()[a] == y.as<int64_t>()[b];
    if (x.dt == F64 && y.dt == F64) return x.as<double>()[a] == y.as<double>()[b];
    if (x.dt == BOOL && y.dt == BOOL) return x.as<uint8_t>()[a] == y.as<uint8_t>()[b];
    if (x.dt == UTF8 && y.dt == UTF8) return x.str(a) == y.str(b);
    return false;
}

// ---- swiss.rs -------------------------------------------------------------------------
static constexpr size_t GROUP = 8;
static constexpr uint8_t EMPTY = 0x80;
static constexpr uint64_t LSB = 0x0101010101010101ull, MSB = 0x8080808080808080ull;
static inline uint8_t h2(uint64_t h) { return (uint8_t)(h >> 57); }
uint64_t swar_match_tag(uint64_t group, uint8_t tag) {
    uint64_t x = group ^ (LSB * tag);
    return (x - LSB) & ~x & MSB;
}
uint64_t swar_match_empty(uint64_t group) { return group & MSB; }

static size_t next_pow2(size_t x) {
    size_t p = 1;
    while (p < x) p <<= 1;
    return p;
}
SwissTable::SwissTable(size_t n) {
    size_t slots = std::max(next_pow2(n * 8 / 7 + 1), GROUP * 2);
    ctrl.assign(slots, EMPTY);
    hashes.assign(slots, 0);
    payloads.assign(slots, 0);
    len = 0;
    group_mask = slots / GROUP - 1;
}
uint64_t SwissTable::load_group(size_t g) const {
    uint64_t w;
    memcpy(&w, ctrl.data() + g * GROUP, 8);
    return w;
}
void SwissTable::insert_at(size_t slot, uint64_t h, uint32_t p) {
    ctrl[slot] = h2(h);
    hashes[slot] = h;
    payloads[slot] = p;
    len++;
}
size_t SwissTable::first_empty(uint64_t h) const {
    size_t g = (size_t)h & group_mask, stride = 0;
    for (;;) {
        uint64_t e = swar_match_empty(load_group(g));
        if (e) return g * GROUP + __builtin_ctzll(e) / 8;
        stride++;
        g = (g + stride) & group_mask;
    }
}
void SwissTable::reserve(size_t extra) {
    size_t needed = len + extra;
    if (needed * 8 <= capacity() * 7) return;
    SwissTable bigger(std::max(needed, len * 2));
    for (size_t i = 0; i < capacity(); i++) {
        if (ctrl[i] != EMPTY) bigger.insert_at(bigger.first_empty(hashes[i]), hashes[i], payloads[i]);
    }
    *this = std::move(bigger);
}

}  // namespace orc
