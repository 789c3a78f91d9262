// Device helpers for the MiniLake B200 kernels: the reference hash, typed
// column loads, the expression stack machine, string predicates, normalized
// keys and the open-addressing hash table.
#pragma once

#ifndef __CUDACC_RTC__
#include <stdint.h>
#endif

#include "ml_internal.hpp"

namespace mlg {

// ---- hash: minilake-hashtable/src/hash.rs:11-54 -------------------------------------------
constexpr uint64_t kSeed = 0x243F6A8885A308D3ull;
constexpr uint64_t kMul = 0x9E3779B97F4A7C15ull;
constexpr uint64_t kMul2 = 0xBF58476D1CE4E5B9ull;
constexpr uint64_t kNullHash = 0x7C159E3779B97F4Aull;

__device__ __forceinline__ uint64_t fold_mul(uint64_t a, uint64_t b) {
    return (a * b) ^ __umul64hi(a, b);
}
__device__ __forceinline__ uint64_t hash_u64(uint64_t x) { return fold_mul(x ^ kSeed, kMul); }
__device__ __forceinline__ uint64_t hash_combine(uint64_t h, uint64_t v) { return fold_mul(h ^ v, kMul2); }
__device__ inline uint64_t hash_bytes(const uint8_t* b, uint32_t n) {
    uint64_t h = kSeed ^ ((uint64_t)n * kMul);
    uint32_t full = n / 8;
    for (uint32_t c = 0; c < full; c++) {
        uint64_t w = 0;
#pragma unroll
        for (int k = 0; k < 8; k++) w |= (uint64_t)b[c * 8 + k] << (8 * k);
        h = fold_mul(h ^ w, kMul);
    }
    uint32_t rem = n % 8;
    if (rem) {
        uint64_t w = 0;
        for (uint32_t k = 0; k < rem; k++) w |= (uint64_t)b[full * 8 + k] << (8 * k);
        h = fold_mul(h ^ w, kMul2);
    }
    return h;
}

// ---- row context: the source row and the matched build row of every probe --------------
struct RowCtx {
    uint32_t r;
    uint32_t b0, b1, b2, b3;
    uint32_t head;  // first match (chain head) of the probe whose join key is the GROUP BY key
    __device__ __forceinline__ uint32_t row_of(int src) const {
        switch (src) {
            case 0: return r;
            case 1: return b0;
            case 2: return b1;
            case 3: return b2;
            default: return b3;
        }
    }
    __device__ __forceinline__ void set_build(int p, uint32_t v) {
        switch (p) {
            case 0: b0 = v; break;
            case 1: b1 = v; break;
            case 2: b2 = v; break;
            default: b3 = v; break;
        }
    }
};

__device__ __forceinline__ bool valid_bit(const uint64_t* w, uint32_t row) {
    return w == nullptr || ((__ldg(w + (row >> 6)) >> (row & 63)) & 1ull);
}

// Dictionary code of a row, clamped to the table size so a corrupt code reads the
// spare last entry instead of memory past the table.
__device__ __forceinline__ uint32_t dict_code(const DCol& c, uint32_t row) {
    uint32_t code = __ldg((const uint32_t*)c.data + row);
    return code < c.dict_len ? code : c.dict_len;
}

// Streaming column reads are read once: load them with an L2 evict-first policy so they
// do not push the hash tables and accumulators (re-read at random) out of L2.
__device__ __forceinline__ uint64_t l2_evict_first() {
    uint64_t p;
    asm("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
    return p;
}
__device__ __forceinline__ uint64_t l2_evict_last() {
    uint64_t p;
    asm("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
    return p;
}
__device__ __forceinline__ uint32_t ld_stream_u32(const void* a) {
    uint32_t v;
    asm("ld.global.nc.L2::cache_hint.u32 %0, [%1], %2;" : "=r"(v) : "l"(a), "l"(l2_evict_first()));
    return v;
}
__device__ __forceinline__ uint64_t ld_stream_u64(const void* a) {
    uint64_t v;
    asm("ld.global.nc.L2::cache_hint.u64 %0, [%1], %2;" : "=l"(v) : "l"(a), "l"(l2_evict_first()));
    return v;
}
// Consecutive values of a streamed column in one 16-byte load (16-byte aligned address).
__device__ __forceinline__ void ld_stream_v4_u32(const void* a, uint32_t* v) {
    asm("ld.global.nc.L2::cache_hint.v4.u32 {%0, %1, %2, %3}, [%4], %5;"
        : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3])
        : "l"(a), "l"(l2_evict_first()));
}
__device__ __forceinline__ void ld_stream_v2_u64(const void* a, uint64_t* v) {
    asm("ld.global.nc.L2::cache_hint.v2.u64 {%0, %1}, [%2], %3;" : "=l"(v[0]), "=l"(v[1]) : "l"(a), "l"(l2_evict_first()));
}
__device__ __forceinline__ uint32_t ld_stream_u8(const void* a) {
    uint16_t v;
    asm("ld.global.nc.L2::cache_hint.u8 %0, [%1], %2;" : "=h"(v) : "l"(a), "l"(l2_evict_first()));
    return v;
}

// Typed load: BOOL 0/1, I32/DATE sign-extended, I64/F64 raw bits, strings as ids.
// Source columns (src 0) stream; build-side columns are read at random and stay in L2.
__device__ __forceinline__ uint64_t load_value(const DCol& c, uint32_t row) {
    if (c.kind == CK_DICT) return (uint64_t)__ldg(c.gid + dict_code(c, row));
    if (c.kind == CK_UTF8 || c.kind == CK_STRID) return c.gid ? (uint64_t)__ldg(c.gid + row) : (uint64_t)row;
    if (c.src == 0) {
        switch (c.dt) {
            case ML_TYPE_BOOL: return (uint64_t)ld_stream_u8((const uint8_t*)c.data + row);
            case ML_TYPE_INT32:
            case ML_TYPE_DATE: return (uint64_t)(int64_t)(int32_t)ld_stream_u32((const int32_t*)c.data + row);
            default: return ld_stream_u64((const unsigned long long*)c.data + row);
        }
    }
    switch (c.dt) {
        case ML_TYPE_BOOL: return (uint64_t)__ldg((const uint8_t*)c.data + row);
        case ML_TYPE_INT32:
        case ML_TYPE_DATE: return (uint64_t)(int64_t)__ldg((const int32_t*)c.data + row);
        default: return (uint64_t)__ldg((const unsigned long long*)c.data + row);
    }
}

__device__ __forceinline__ double as_f64(uint64_t b) { return __longlong_as_double((long long)b); }
__device__ __forceinline__ uint64_t f64_bits(double d) { return (uint64_t)__double_as_longlong(d); }

// ---- strings ----------------------------------------------------------------------------
struct Str {
    const uint8_t* p;
    uint32_t n;
};
__device__ __forceinline__ Str col_str(const DCol& c, uint32_t row) {
    if (c.kind == CK_DICT) {
        uint32_t code = dict_code(c, row);
        uint32_t a = __ldg(c.off + code), b = __ldg(c.off + code + 1);
        return Str{c.dbytes + a, b - a};
    }
    uint32_t a = __ldg(c.off + row), b = __ldg(c.off + row + 1);
    return Str{(const uint8_t*)c.data + a, b - a};
}
// Lexicographic byte order, then length (Rust slice Ord).
__device__ inline int str_cmp(Str x, Str y) {
    uint32_t m = x.n < y.n ? x.n : y.n;
    for (uint32_t i = 0; i < m; i++) {
        uint8_t a = x.p[i], b = y.p[i];
        if (a != b) return a < b ? -1 : 1;
    }
    return x.n < y.n ? -1 : (x.n > y.n ? 1 : 0);
}
__device__ __forceinline__ bool cmp_result(int op, int c) {
    switch (op) {
        case ML_BIN_EQ: return c == 0;
        case ML_BIN_NOTEQ: return c != 0;
        case ML_BIN_LT: return c < 0;
        case ML_BIN_LTEQ: return c <= 0;
        case ML_BIN_GT: return c > 0;
        default: return c >= 0;
    }
}
__device__ inline bool bytes_eq(const uint8_t* a, const uint8_t* b, uint32_t n) {
    for (uint32_t i = 0; i < n; i++)
        if (a[i] != b[i]) return false;
    return true;
}
// LIKE by shape (expr/like.rs:48-115)
__device__ inline bool like_match(Str s, const uint8_t* p, uint32_t pn, int shape) {
    switch (shape) {
        case LK_EXACT: return s.n == pn && bytes_eq(s.p, p, pn);
        case LK_PREFIX: return s.n >= pn && bytes_eq(s.p, p, pn);
        case LK_SUFFIX: return s.n >= pn && bytes_eq(s.p + (s.n - pn), p, pn);
        case LK_CONTAINS: {
            if (pn == 0) return true;
            if (pn > s.n) return false;
            for (uint32_t i = 0; i + pn <= s.n; i++)
                if (s.p[i] == p[0] && bytes_eq(s.p + i, p, pn)) return true;
            return false;
        }
        default: {  // two pointers with one backtrack point
            uint32_t si = 0, pi = 0, star_s = 0;
            int64_t star = -1;
            while (si < s.n) {
                if (pi < pn && (p[pi] == '_' || p[pi] == s.p[si])) {
                    si++;
                    pi++;
                } else if (pi < pn && p[pi] == '%') {
                    star = pi;
                    star_s = si;
                    pi++;
                } else if (star >= 0) {
                    pi = (uint32_t)star + 1;
                    star_s++;
                    si = star_s;
                } else {
                    return false;
                }
            }
            while (pi < pn && p[pi] == '%') pi++;
            return pi == pn;
        }
    }
}

__device__ inline bool str_pred(const StrSpec& sp, const uint8_t* arena, Str v) {
    bool r;
    if (sp.what == SW_CMP) {
        r = cmp_result(sp.op, str_cmp(v, Str{arena + sp.lit_off, sp.lit_len}));
    } else if (sp.what == SW_LIKE) {
        r = like_match(v, arena + sp.lit_off, sp.lit_len, sp.op);
    } else {
        const uint32_t* items = (const uint32_t*)(arena + sp.lit_off);
        r = false;
        for (uint32_t k = 0; k < sp.count && !r; k++) {
            uint32_t o = items[2 * k], n = items[2 * k + 1];
            r = n == v.n && bytes_eq(v.p, arena + o, n);
        }
    }
    return r != (sp.negated != 0);
}

// ---- expression stack machine --------------------------------------------------------------
// The stack lives in six named registers; push/pop shift them, so no register is
// ever indexed dynamically (no local-memory traffic).  Every instruction of a
// program is the same for all threads of a warp, so the dispatch is uniform.
struct Stack {
    uint64_t v0, v1, v2, v3, v4, v5;
    uint32_t ok;  // bit i = validity of slot i (0 = top)
    __device__ __forceinline__ void push(uint64_t v, bool valid) {
        v5 = v4; v4 = v3; v3 = v2; v2 = v1; v1 = v0; v0 = v;
        ok = (ok << 1) | (valid ? 1u : 0u);
    }
    __device__ __forceinline__ void pop() {
        v0 = v1; v1 = v2; v2 = v3; v3 = v4; v4 = v5;
        ok >>= 1;
    }
};

template <class T> __device__ __forceinline__ bool cmp_typed(int op, T a, T b) {
    switch (op) {
        case ML_BIN_EQ: return a == b;
        case ML_BIN_NOTEQ: return a != b;
        case ML_BIN_LT: return a < b;
        case ML_BIN_LTEQ: return a <= b;
        case ML_BIN_GT: return a > b;
        default: return a >= b;
    }
}

// l <op> r in type t; returns value bits, updates `valid`.
__device__ __forceinline__ uint64_t binop(int op, int t, uint64_t l, uint64_t r, bool& valid, bool lv, bool rv) {
    if (op == ML_BIN_AND || op == ML_BIN_OR) {  // Kleene (boolean.rs:18-58)
        bool a = l & 1, b = r & 1;
        if (op == ML_BIN_AND) {
            valid = (lv && rv) || (lv && !a) || (rv && !b);
            return (uint64_t)(a & b);
        }
        valid = (lv && rv) || (lv && a) || (rv && b);
        return (uint64_t)(a | b);
    }
    valid = lv && rv;
    if (op >= ML_BIN_EQ) {
        switch (t) {
            case ML_TYPE_FLOAT64: return cmp_typed(op, as_f64(l), as_f64(r));
            case ML_TYPE_INT64: return cmp_typed(op, (int64_t)l, (int64_t)r);
            case ML_TYPE_BOOL: return cmp_typed(op, (uint32_t)(l & 1), (uint32_t)(r & 1));
            case ML_TYPE_UTF8: return cmp_typed(op, (uint32_t)l, (uint32_t)r);  // ids: EQ/NOTEQ only
            default: return cmp_typed(op, (int32_t)l, (int32_t)r);
        }
    }
    if (t == ML_TYPE_FLOAT64) {
        double a = as_f64(l), b = as_f64(r);
        switch (op) {  // explicit round-to-nearest ops: no FMA contraction
            case ML_BIN_ADD: return f64_bits(__dadd_rn(a, b));
            case ML_BIN_SUB: return f64_bits(__dsub_rn(a, b));
            case ML_BIN_MUL: return f64_bits(__dmul_rn(a, b));
            case ML_BIN_DIV:
                if (b == 0.0) valid = false;  // x / 0 is NULL (eval.rs:260-271)
                return f64_bits(__ddiv_rn(a, b));
            default: return f64_bits(fmod(a, b));
        }
    }
    if (t == ML_TYPE_INT64) {
        uint64_t a = l, b = r;
        switch (op) {  // wrapping (arith.rs:52-73)
            case ML_BIN_ADD: return a + b;
            case ML_BIN_SUB: return a - b;
            case ML_BIN_MUL: return a * b;
            default:
                if (b == 0) { valid = false; return 0; }
                if ((int64_t)b == -1) return 0;
                return (uint64_t)((int64_t)a % (int64_t)b);
        }
    }
    // INT32 / DATE
    uint32_t a = (uint32_t)l, b = (uint32_t)r;
    uint32_t o;
    switch (op) {
        case ML_BIN_ADD: o = a + b; break;
        case ML_BIN_SUB: o = a - b; break;
        case ML_BIN_MUL: o = a * b; break;
        default:
            if (b == 0) { valid = false; o = 0; }
            else if ((int32_t)b == -1) o = 0;
            else o = (uint32_t)((int32_t)a % (int32_t)b);
    }
    return (uint64_t)(int64_t)(int32_t)o;
}

// Rust `as` casts (cast.rs:6-73); out-of-range float->int saturates, NaN -> 0
// (PTX cvt.rzi clamps to the destination range).
__device__ __forceinline__ uint64_t cast_value(uint64_t v, int from, int to) {
    if (from == to) return v;
    if (to == ML_TYPE_FLOAT64) {
        if (from == ML_TYPE_INT64) return f64_bits(__ll2double_rn((long long)v));
        if (from == ML_TYPE_BOOL) return f64_bits((double)(v & 1));
        return f64_bits((double)(int32_t)v);
    }
    if (to == ML_TYPE_INT64) {
        if (from == ML_TYPE_FLOAT64) return (uint64_t)__double2ll_rz(as_f64(v));
        return v;  // i32/date/bool already sign-/zero-extended
    }
    if (to == ML_TYPE_INT32 || to == ML_TYPE_DATE) {
        if (from == ML_TYPE_FLOAT64) return (uint64_t)(int64_t)__double2int_rz(as_f64(v));
        return (uint64_t)(int64_t)(int32_t)(uint32_t)v;
    }
    return v;
}

struct EvalEnv {
    const DCol* cols;
    const Instr* prog;
    const uint8_t* arena;
    const uint8_t* const* luts;
};

__device__ __forceinline__ void load_col(const EvalEnv& env, int a, const RowCtx& x, uint64_t& v, bool& ok) {
    const DCol& c = env.cols[a];
    uint32_t row = x.row_of(c.src);
    v = load_value(c, row);
    ok = valid_bit(c.valid, row);
}

__device__ inline void eval_prog(const EvalEnv& env, Prog p, const RowCtx& x, uint64_t& out, bool& out_ok) {
    switch (p.fast) {  // the shape is the same for every thread: a uniform branch
        case FP_COL: {
            load_col(env, env.prog[p.start].a, x, out, out_ok);
            return;
        }
        case FP_COL_LIT_BIN: {
            const Instr& lit = env.prog[p.start + 1];
            const Instr& bin = env.prog[p.start + 2];
            uint64_t a;
            bool av;
            load_col(env, env.prog[p.start].a, x, a, av);
            out = binop(bin.sub, bin.t, a, lit.bits, out_ok, av, lit.lit_valid != 0);
            return;
        }
        case FP_COL_LCB_BIN: {
            const Instr& lit = env.prog[p.start + 1];
            const Instr& b1 = env.prog[p.start + 3];
            const Instr& b2 = env.prog[p.start + 4];
            uint64_t a, b;
            bool av, bv, tv;
            load_col(env, env.prog[p.start].a, x, a, av);
            load_col(env, env.prog[p.start + 2].a, x, b, bv);
            uint64_t t = binop(b1.sub, b1.t, lit.bits, b, tv, lit.lit_valid != 0, bv);
            out = binop(b2.sub, b2.t, a, t, out_ok, av, tv);
            return;
        }
        default: break;
    }
    Stack s;
    s.ok = 0;
    s.v0 = s.v1 = s.v2 = s.v3 = s.v4 = s.v5 = 0;
    for (int i = 0; i < p.len; i++) {
        const Instr in = env.prog[p.start + i];
        switch (in.op) {
            case I_COL: {
                const DCol& c = env.cols[in.a];
                uint32_t row = x.row_of(c.src);
                s.push(load_value(c, row), valid_bit(c.valid, row));
                break;
            }
            case I_LIT: s.push(in.bits, in.lit_valid != 0); break;
            case I_BIN: {
                bool lv = (s.ok >> 1) & 1, rv = s.ok & 1, v;
                uint64_t r = binop(in.sub, in.t, s.v1, s.v0, v, lv, rv);
                s.pop();
                s.v0 = r;
                s.ok = (s.ok & ~1u) | (v ? 1u : 0u);
                break;
            }
            case I_NOT: s.v0 = (~s.v0) & 1ull; break;
            case I_NEG:
                if (in.t == ML_TYPE_FLOAT64) s.v0 ^= 0x8000000000000000ull;
                else if (in.t == ML_TYPE_INT64) s.v0 = 0ull - s.v0;
                else s.v0 = (uint64_t)(int64_t)(int32_t)(0u - (uint32_t)s.v0);
                break;
            case I_ISNULL: {
                bool v = s.ok & 1;
                s.v0 = (v == (in.flag != 0)) ? 1 : 0;
                s.ok |= 1u;
                break;
            }
            case I_CAST: s.v0 = cast_value(s.v0, in.t, in.sub); break;
            case I_STRPRED: {
                const DCol& c = env.cols[in.a];
                uint32_t row = x.row_of(c.src);
                bool v;
                if (c.kind == CK_DICT) {
                    v = __ldg(env.luts[in.b] + dict_code(c, row)) != 0;
                } else {
                    v = str_pred(*(const StrSpec*)(env.arena + in.c), env.arena, col_str(c, row));
                }
                s.push(v, valid_bit(c.valid, row));
                break;
            }
            case I_STRCMP_COL: {
                const DCol& c = env.cols[in.a];
                const DCol& d = env.cols[in.b];
                uint32_t ra = x.row_of(c.src), rb = x.row_of(d.src);
                int r = str_cmp(col_str(c, ra), col_str(d, rb));
                s.push(cmp_result(in.sub, r), valid_bit(c.valid, ra) && valid_bit(d.valid, rb));
                break;
            }
            case I_INLIST: {
                const uint64_t* items = (const uint64_t*)(env.arena + in.b);
                bool hit = false;
                for (int k = 0; k < in.c; k++) {
                    uint64_t it = items[k];
                    if (in.t == ML_TYPE_FLOAT64) hit |= as_f64(it) == as_f64(s.v0);
                    else hit |= it == s.v0;
                }
                s.v0 = hit != (in.flag != 0);
                break;
            }
            case I_SELECT: {  // stack: rest (2), cond (1), val (0)
                bool take = ((s.ok >> 1) & 1) && (s.v1 & 1);
                uint64_t v = take ? s.v0 : s.v2;
                bool ok = take ? (s.ok & 1) : ((s.ok >> 2) & 1);
                s.pop();
                s.pop();
                s.v0 = v;
                s.ok = (s.ok & ~1u) | (ok ? 1u : 0u);
                break;
            }
        }
    }
    out = s.v0;
    out_ok = s.ok & 1;
}

// ---- normalized keys -----------------------------------------------------------------------
// Returns false when a key is NULL and `null_kills` (join keys: NULL never matches).
__device__ inline bool make_key(const EvalEnv& env, const KeyLayout& L, const RowCtx& x, uint64_t* w, uint32_t* nm,
                                bool null_kills) {
    uint64_t w0 = 0, w1 = 0;
    w[0] = 0;
    w[1] = 0;
    *nm = 0;
    for (int k = 0; k < L.nkeys; k++) {
        uint64_t v;
        bool ok;
        eval_prog(env, L.prog[k], x, v, ok);
        const KeyField f = L.f[k];
        if (!ok) {
            if (null_kills) return false;
            *nm |= 1u << k;
            continue;
        }
        if (f.type == ML_TYPE_FLOAT64 && as_f64(v) == 0.0) v = 0;  // +0.0 == -0.0 (kernels/hash.rs:52-53)
        uint64_t m = f.width >= 64 ? ~0ull : ((1ull << f.width) - 1);
        uint64_t bits = (v & m) << f.shift;
        if (f.word == 0) w0 |= bits;  // named registers: no dynamic indexing of w[]
        else w1 |= bits;
    }
    w[0] = w0;
    w[1] = w1;
    return true;
}
__device__ __forceinline__ uint64_t key_hash(const uint64_t* w, int nwords, uint32_t nm = 0) {
    uint64_t h = hash_u64(w[0] ^ ((uint64_t)nm << 56));
    if (nwords > 1) h = hash_combine(h, hash_u64(w[1]));
    return h;
}

// ---- hash table ------------------------------------------------------------------------------
constexpr uint32_t kSpinLimit = 1u << 22;

__device__ __forceinline__ uint32_t load_state(uint32_t* p) {
    uint32_t v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void publish_state(uint32_t* p, uint32_t v) {
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ uint64_t* slot_at(const TableView& t, uint64_t i) { return t.slots + i * t.stride; }

// Read-only lookup in a finished table (join probe): one 128-bit load per slot.  The
// first slot's load is separate so a caller can issue it for several rows before
// resolving any of them.
__device__ __forceinline__ ulonglong2 slot_load(const TableView& t, uint64_t i) {
    ulonglong2 v;
    asm("ld.global.nc.L2::cache_hint.v2.u64 {%0, %1}, [%2], %3;"
        : "=l"(v.x), "=l"(v.y)
        : "l"(slot_at(t, i)), "l"(l2_evict_last()));
    return v;
}
__device__ __forceinline__ uint32_t table_find_from(const TableView& t, const uint64_t* w, uint64_t h, ulonglong2 v) {
    uint64_t i = h & t.mask;
    for (uint64_t n = 0; n <= t.mask; n++) {
        if ((uint32_t)v.x == 0) return kNone;
        if (v.y == w[0] && (t.nwords == 1 || __ldg((const unsigned long long*)slot_at(t, i) + 2) == w[1]))
            return (uint32_t)(v.x >> 32);
        i = (i + 1) & t.mask;
        v = slot_load(t, i);
    }
    return kNone;
}
__device__ __forceinline__ uint32_t table_find(const TableView& t, const uint64_t* w, uint64_t h) {
    return table_find_from(t, w, h, slot_load(t, h & t.mask));
}

// Chain head of a dense join index entry (kept in L2 like the hash tables).
__device__ __forceinline__ uint32_t dense_load(const uint32_t* p) {
    uint32_t v;
    asm("ld.global.nc.L2::cache_hint.u32 %0, [%1], %2;" : "=r"(v) : "l"(p), "l"(l2_evict_last()));
    return v;
}
__device__ __forceinline__ uint32_t dense_find(const uint32_t* dense, uint64_t dmin, uint64_t drange, uint64_t key) {
    const uint64_t off = key - dmin;
    return off < drange ? dense_load(dense + off) : kNone;
}
// Membership of a key in a dense index's bitmap (ProbeDev::member): 0 when present, else kNone.
__device__ __forceinline__ uint32_t dense_member(const uint32_t* bits, uint64_t dmin, uint64_t drange, uint64_t key) {
    const uint64_t off = key - dmin;
    return off < drange && ((__ldg(bits + (off >> 5)) >> (off & 31)) & 1u) ? 0u : kNone;
}

// Index position of a key in a dense index's range (kNone outside it), without reading it.
__device__ __forceinline__ uint32_t dense_slot(uint64_t dmin, uint64_t drange, uint64_t key) {
    const uint64_t off = key - dmin;
    return off < drange ? (uint32_t)off : kNone;
}

// 128-bit compare-and-swap (sm_90+): returns the slot's previous contents.
__device__ __forceinline__ ulonglong2 cas128(uint64_t* p, ulonglong2 expect, ulonglong2 desired) {
    ulonglong2 old;
    asm volatile(
        "{\n\t.reg .b128 c, d, o;\n\t"
        "mov.b128 c, {%2, %3};\n\t"
        "mov.b128 d, {%4, %5};\n\t"
        "atom.relaxed.gpu.global.cas.b128 o, [%6], c, d;\n\t"
        "mov.b128 {%0, %1}, o;\n\t}"
        : "=l"(old.x), "=l"(old.y)
        : "l"(expect.x), "l"(expect.y), "l"(desired.x), "l"(desired.y), "l"(p)
        : "memory");
    return old;
}

// Insert one build row under a one-word key (join build, 16-byte slots): the slot's
// state, payload and key are written by one 128-bit CAS, so there is no claimed state
// and no waiting.  Returns the payload stored for the key: `row` when this thread
// inserted it (*inserted = true), else the current chain head.
__device__ inline uint32_t table_insert_row1(const TableView& t, uint64_t key, uint64_t h, uint32_t row, bool* inserted,
                                             uint64_t* slot_out) {
    const ulonglong2 want = make_ulonglong2(2ull | ((uint64_t)row << 32), key);
    uint64_t i = h & t.mask;
    *inserted = false;
    for (uint64_t n = 0; n <= t.mask; n++, i = (i + 1) & t.mask) {
        ulonglong2 old = cas128(slot_at(t, i), make_ulonglong2(0ull, 0ull), want);
        if (old.x == 0 && old.y == 0) {
            *inserted = true;
            *slot_out = i;
            return row;
        }
        if (old.y == key) {
            *slot_out = i;
            return (uint32_t)(old.x >> 32);
        }
    }
    return kNone;
}

// Find or insert under concurrent insertion.  On insert, `assign` produces the payload
// (kNone = refuse: the slot is released and kNone returned).  *inserted tells the caller
// whether this thread created the entry.
// With `count` set, a new key is refused without touching the slot once *count has reached
// `limit` (a full aggregation table: the row goes to the overflow list at once).
template <class Assign>
__device__ inline uint32_t table_upsert(const TableView& t, const uint64_t* w, uint32_t nm, uint64_t h, uint32_t* err,
                                        Assign assign, bool* inserted, uint64_t* slot_out,
                                        const uint32_t* count = nullptr, uint32_t limit = 0) {
    uint64_t i = h & t.mask;
    const uint32_t full = 2u | (nm << 8);
    *inserted = false;
    for (uint64_t n = 0; n <= t.mask;) {
        uint64_t* s = slot_at(t, i);
        uint32_t* st_p = (uint32_t*)s;
        uint32_t st = load_state(st_p);
        if (st == 0) {
            if (count && *(const volatile uint32_t*)count >= limit) return kNone;
            uint32_t old = atomicCAS(st_p, 0u, 1u);
            if (old == 0) {
                uint32_t p = assign();
                if (p == kNone) {
                    publish_state(st_p, 0);
                    return kNone;
                }
                s[1] = w[0];
                if (t.nwords > 1) s[2] = w[1];
                st_p[1] = p;
                publish_state(st_p, full);
                *inserted = true;
                *slot_out = i;
                return p;
            }
            st = old;
        }
        if (st == 1) {
            uint32_t spins = 0;
            do {
                __nanosleep(20);
                st = load_state(st_p);
            } while (st == 1 && ++spins < kSpinLimit);
            if (st == 1) {
                atomicOr(err, (uint32_t)DE_TIMEOUT);
                return kNone;
            }
            if (st == 0) continue;  // the claimer released the slot: retry it
        }
        if (st == full && s[1] == w[0] && (t.nwords == 1 || s[2] == w[1])) {
            *slot_out = i;
            return st_p[1];
        }
        i = (i + 1) & t.mask;
        n++;
    }
    return kNone;
}

// Order-preserving map of f64 onto u64 (for atomic MIN/MAX).
__device__ __forceinline__ uint64_t f64_order(double d) {
    uint64_t b = f64_bits(d);
    return (b & 0x8000000000000000ull) ? ~b : (b | 0x8000000000000000ull);
}
__device__ __forceinline__ double f64_unorder(uint64_t u) {
    uint64_t b = (u & 0x8000000000000000ull) ? (u & ~0x8000000000000000ull) : ~u;
    return as_f64(b);
}

}  // namespace mlg
