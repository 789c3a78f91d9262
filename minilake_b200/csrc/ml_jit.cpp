// Runtime-specialized pipeline kernels: source generation, NVRTC compilation for
// sm_100a and a process-wide kernel cache.
#include "ml_jit.hpp"

#include <cuda.h>
#include <dlfcn.h>
#include <nvrtc.h>

#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <map>
#include <set>
#include <type_traits>
#include <sstream>

namespace mlg {

// Device headers, embedded at build time (generated from ml_internal.hpp, ml_args.hpp,
// ml_device.cuh, ml_agg.cuh and include/minilake_gpu.h).
#include "jit_headers.inc"

namespace {

// ---- NVRTC (loaded at first use) and the driver's module API (through the runtime) -----------
struct Nvrtc {
    bool ok = false;
    std::string why;
    nvrtcResult (*create)(nvrtcProgram*, const char*, const char*, int, const char* const*, const char* const*);
    nvrtcResult (*compile)(nvrtcProgram, int, const char* const*);
    nvrtcResult (*log_size)(nvrtcProgram, size_t*);
    nvrtcResult (*log)(nvrtcProgram, char*);
    nvrtcResult (*cubin_size)(nvrtcProgram, size_t*);
    nvrtcResult (*cubin)(nvrtcProgram, char*);
    nvrtcResult (*destroy)(nvrtcProgram*);
    CUresult (*load)(CUmodule*, const void*);
    CUresult (*get_fn)(CUfunction*, CUmodule, const char*);
    CUresult (*launch)(CUfunction, unsigned, unsigned, unsigned, unsigned, unsigned, unsigned, unsigned, CUstream,
                       void**, void**);
    CUresult (*set_attr)(CUfunction, CUfunction_attribute, int);
    CUresult (*occupancy)(int*, CUfunction, int, size_t);

    Nvrtc() {
        const char* names[] = {"libnvrtc.so.12", "libnvrtc.so", "/usr/local/cuda/lib64/libnvrtc.so.12"};
        void* h = nullptr;
        for (const char* n : names)
            if ((h = dlopen(n, RTLD_NOW | RTLD_LOCAL))) break;
        if (!h) {
            why = "libnvrtc.so.12 not found";
            return;
        }
        bool got = true;
        auto sym = [&](auto& fp, const char* n) {
            fp = (std::remove_reference_t<decltype(fp)>)dlsym(h, n);
            got = got && fp != nullptr;
        };
        sym(create, "nvrtcCreateProgram");
        sym(compile, "nvrtcCompileProgram");
        sym(log_size, "nvrtcGetProgramLogSize");
        sym(log, "nvrtcGetProgramLog");
        sym(cubin_size, "nvrtcGetCUBINSize");
        sym(cubin, "nvrtcGetCUBIN");
        sym(destroy, "nvrtcDestroyProgram");
        auto drv = [&](auto& fp, const char* n) {
            void* p = nullptr;
            cudaDriverEntryPointQueryResult q;
            if (cudaGetDriverEntryPointByVersion(n, &p, 12000, cudaEnableDefault, &q) != cudaSuccess ||
                q != cudaDriverEntryPointSuccess)
                p = nullptr;
            fp = (std::remove_reference_t<decltype(fp)>)p;
            got = got && p != nullptr;
        };
        drv(load, "cuModuleLoadData");
        drv(get_fn, "cuModuleGetFunction");
        drv(launch, "cuLaunchKernel");
        drv(set_attr, "cuFuncSetAttribute");
        drv(occupancy, "cuOccupancyMaxActiveBlocksPerMultiprocessor");
        ok = got;
        if (!ok) why = "NVRTC or driver module entry points missing";
    }
};

Nvrtc& nvrtc() {
    static Nvrtc n;
    return n;
}

bool jit_enabled(Ctx* ctx) {
    if (ctx->flags & ML_CTX_INTERPRET) return false;
    static const bool env_off = [] {
        const char* e = getenv("MINILAKE_GPU_JIT");
        return e && e[0] == '0';
    }();
    return !env_off && nvrtc().ok;
}

const char kStdint[] =
    "#pragma once\n"
    "typedef signed char int8_t; typedef short int16_t; typedef int int32_t; typedef long int64_t;\n"
    "typedef unsigned char uint8_t; typedef unsigned short uint16_t; typedef unsigned int uint32_t;\n"
    "typedef unsigned long uint64_t;\n";
const char kStddef[] = "#pragma once\ntypedef unsigned long size_t;\n";

// One entry per (device, source): the first thread to ask compiles it while later askers for
// the same source wait on the entry; other sources are looked up and compiled meanwhile.
struct CacheEntry {
    std::mutex mu;
    bool done = false;
    CUfunction fn = nullptr;
};
struct Cache {
    std::mutex mu;
    std::map<std::pair<int, std::string>, std::shared_ptr<CacheEntry>> fns;
};
Cache& cache() {
    static Cache c;
    return c;
}

CUfunction compile_kernel(Ctx* ctx, const std::string& src, const char* name);

// Compile `src` (defining extern "C" kernel `name`) for this device, or return the cached kernel.
CUfunction get_kernel(Ctx* ctx, const std::string& src, const char* name) {
    Cache& C = cache();
    std::shared_ptr<CacheEntry> e;
    {
        std::lock_guard<std::mutex> g(C.mu);
        auto& slot = C.fns[std::make_pair(ctx->device, src)];
        if (!slot) slot = std::make_shared<CacheEntry>();
        e = slot;
    }
    std::lock_guard<std::mutex> g(e->mu);
    if (!e->done) {
        e->fn = compile_kernel(ctx, src, name);  // throws on failure: the next asker tries again
        e->done = true;
    }
    return e->fn;
}

CUfunction compile_kernel(Ctx* ctx, const std::string& src, const char* name) {
    Nvrtc& N = nvrtc();
    // MINILAKE_GPU_JIT_DUMP=<dir>: keep each generated source there (<kernel>_<hash>.cu) to read
    // or compile offline
    if (const char* dir = getenv("MINILAKE_GPU_JIT_DUMP")) {
        const std::string path = std::string(dir) + "/" + name + "_" + std::to_string(std::hash<std::string>{}(src)) + ".cu";
        if (FILE* f = fopen(path.c_str(), "w")) {
            fwrite(src.data(), 1, src.size(), f);
            fclose(f);
        }
    }
    auto t0 = std::chrono::steady_clock::now();
    std::vector<const char*> texts, names;
    for (int i = 0; i < kJitHeaderCount; i++) {
        texts.push_back(kJitHeaderText[i]);
        names.push_back(kJitHeaderName[i]);
    }
    texts.push_back(kStdint);
    names.push_back("stdint.h");
    texts.push_back(kStddef);
    names.push_back("stddef.h");
    nvrtcProgram prog;
    if (N.create(&prog, src.c_str(), "ml_pipeline_kernel.cu", (int)texts.size(), texts.data(), names.data()) !=
        NVRTC_SUCCESS)
        raise(ML_ERR_INTERNAL, "nvrtcCreateProgram failed");
    const char* opts[] = {"--gpu-architecture=sm_100a", "-std=c++17", "--fmad=false", "-lineinfo"};
    nvrtcResult r = N.compile(prog, 4, opts);
    if (r != NVRTC_SUCCESS) {
        size_t n = 0;
        N.log_size(prog, &n);
        std::string log(n, '\0');
        if (n) N.log(prog, &log[0]);
        N.destroy(&prog);
        raise(ML_ERR_INTERNAL, "runtime kernel compilation failed:\n" + log + "\n--- source ---\n" + src);
    }
    size_t n = 0;
    N.cubin_size(prog, &n);
    std::vector<char> bin(n);
    N.cubin(prog, bin.data());
    N.destroy(&prog);
    ctx->set_current();
    CK(cudaFree(nullptr));  // the runtime's primary context is current for the driver calls
    CUmodule mod;
    CUfunction fn;
    if (N.load(&mod, bin.data()) != CUDA_SUCCESS) raise(ML_ERR_CUDA, "cuModuleLoadData failed for a pipeline kernel");
    if (N.get_fn(&fn, mod, name) != CUDA_SUCCESS) raise(ML_ERR_CUDA, "cuModuleGetFunction failed");
    double ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    ctx->add_profile("jit_compile", ms);
    return fn;
}

// ---- source generation --------------------------------------------------------------------------
std::string num(int64_t v) { return std::to_string(v); }
std::string hex(uint64_t v) {
    char b[32];
    snprintf(b, sizeof b, "0x%llxull", (unsigned long long)v);
    return b;
}

// Rows a thread carries through the stages together in the batched form: the loads of
// each stage are issued for all of them before any is used, so every thread keeps
// several HBM / L2 requests in flight instead of one dependent chain per row.
constexpr int kRowsPerThread = 4;

class Gen {
   public:
    Gen(const std::vector<Instr>& code, const PipeArgs& P) : code_(code), P_(P) {}

    struct V {
        std::string v, k;  // value bits and validity expressions
    };

    std::string pre() const { return pre_.str(); }
    std::string body() const { return o_.str(); }
    void line(const std::string& s) { o_ << std::string(4 * ind_, ' ') << s << '\n'; }
    void open(const std::string& s) {
        line(s);
        ind_++;
    }
    void close(const std::string& s = "}") {
        ind_--;
        line(s);
    }
    int fresh() { return nv_++; }

    // Rows per thread of the batched form, and whether a thread's rows are consecutive
    // (x<j>.r = r0 + j, `full` when all are in range): then the source columns of the rows are
    // read with vector loads, one validity word per thread.
    int rows_per_thread = kRowsPerThread;
    bool contig = false;
    // Statement that leaves the current tile (empty: tiles are never cut short).
    std::string tile_skip;
    // The row context the generated statements read (x, or x<j> in the batched form), the
    // statement that abandons the current row combination, and preloaded columns.
    std::string x = "x";
    std::string fail = "continue;";
    std::map<int, V> cols;

    std::string row(int src) const { return src == 0 ? x + ".r" : x + ".b" + num(src - 1); }

    // Typed load of column slot `a` (load_value, specialized on the column's kind and type).
    std::string col_value(int a) const {
        const DCol& c = P_.cols[a];
        std::string C = "P.cols[" + num(a) + "]", R = row(c.src);
        if (c.kind == CK_DICT) return "(uint64_t)__ldg(" + C + ".gid + dict_code(" + C + ", " + R + "))";
        if (c.kind == CK_UTF8 || c.kind == CK_STRID)
            return c.gid ? "(uint64_t)__ldg(" + C + ".gid + " + R + ")" : "(uint64_t)" + R;
        bool stream = c.src == 0;
        switch (c.dt) {
            case ML_TYPE_BOOL:
                return stream ? "(uint64_t)ld_stream_u8((const uint8_t*)" + C + ".data + " + R + ")"
                              : "(uint64_t)__ldg((const uint8_t*)" + C + ".data + " + R + ")";
            case ML_TYPE_INT32:
            case ML_TYPE_DATE:
                return stream ? "(uint64_t)(int64_t)(int32_t)ld_stream_u32((const int32_t*)" + C + ".data + " + R + ")"
                              : "(uint64_t)(int64_t)__ldg((const int32_t*)" + C + ".data + " + R + ")";
            default:
                return stream ? "(uint64_t)ld_stream_u64((const unsigned long long*)" + C + ".data + " + R + ")"
                              : "(uint64_t)__ldg((const unsigned long long*)" + C + ".data + " + R + ")";
        }
    }
    std::string col_valid(int a) const {
        const DCol& c = P_.cols[a];
        return c.valid ? "valid_bit(P.cols[" + num(a) + "].valid, " + row(c.src) + ")" : "true";
    }

    // Column slots a program reads through I_COL.
    void slots_of(const Prog& p, std::set<int>& out) const {
        for (int i = 0; i < p.len; i++)
            if (code_[p.start + i].op == I_COL) out.insert(code_[p.start + i].a);
    }
    // Load `slots` of the current row into registers, only when `alive` holds.
    void preload(const std::set<int>& slots, const std::string& alive) {
        for (int a : slots) {
            std::string n = num(fresh()), v = "c" + n, k = "n" + n;
            line("uint64_t " + v + " = 0;");
            line("bool " + k + " = false;");
            open("if (" + alive + ") {");
            line(v + " = " + col_value(a) + ";");
            line(k + " = " + col_valid(a) + ";");
            close();
            cols[a] = V{v, k};
        }
    }

    // Load `slots` for the batched rows x0.. (alive a0..) into pre[j].  With consecutive rows a
    // fixed-width or dictionary-coded source column is read with one vector load per thread when
    // all its rows are in range, its validity with one word.
    // Width in bytes of a column's per-row value as the vector loads read it (0: not loaded so).
    int vec_width(int a) const {
        const DCol& c = P_.cols[a];
        if (c.src != 0 || (c.kind != CK_FIXED && c.kind != CK_DICT)) return 0;
        if (c.kind == CK_DICT) return 4;
        if (c.dt == ML_TYPE_BOOL) return 1;
        return (c.dt == ML_TYPE_INT32 || c.dt == ML_TYPE_DATE) ? 4 : 8;
    }
    void vec_decl(int W, const std::string& t) {
        const int K = rows_per_thread;
        if (W == 4) line("uint32_t " + t + "[" + num(K) + "];");
        else if (W == 8) line("uint64_t " + t + "[" + num(K) + "];");
        else line("uint64_t " + t + ";");
    }
    // The K consecutive values of slot `a` from x0.r on into `t` (16-byte loads: the widest this
    // toolchain's runtime compiler accepts).
    void vec_load(int a, int W, const std::string& t) {
        const int K = rows_per_thread;
        const std::string C = "P.cols[" + num(a) + "]";
        if (W == 4) {
            for (int q = 0; q < K; q += 4)
                line("ld_stream_v4_u32((const uint32_t*)" + C + ".data + x0.r + " + num(q) + ", " + t + " + " + num(q) + ");");
        } else if (W == 8) {
            for (int q = 0; q < K; q += 2)
                line("ld_stream_v2_u64((const unsigned long long*)" + C + ".data + x0.r + " + num(q) + ", " + t + " + " +
                     num(q) + ");");
        } else {
            line(t + " = " +
                 (K == 8 ? "ld_stream_u64((const unsigned long long*)(" : "(uint64_t)ld_stream_u32((const uint32_t*)(") +
                 "(const uint8_t*)" + C + ".data + x0.r));");
        }
    }

    // Load `slots` for the batched rows x0.. (alive a0..) into pre[j].  With consecutive rows a
    // fixed-width or dictionary-coded source column is read with one vector load per thread when
    // all its rows are in range, its validity with one word; a column loaded ahead of the tile's
    // first stage (`spec_vals`) is reused when that speculative load ran.
    void preload_rows(const std::set<int>& slots, std::vector<std::map<int, V>>& pre) {
        const int K = rows_per_thread;
        pre.assign(K, {});
        auto per_row = [&](const std::set<int>& sl) {
            for (int j = 0; j < K; j++) {
                x = "x" + num(j);
                cols.clear();
                preload(sl, "a" + num(j));
                for (auto& e : cols) pre[j][e.first] = e.second;
            }
            x = "x";
            cols.clear();
        };
        if (!contig) {
            per_row(slots);
            return;
        }
        std::string any = "(";
        for (int j = 0; j < K; j++) any += (j ? " || a" : "a") + num(j);
        any += ")";
        for (int a : slots) {
            const DCol& c = P_.cols[a];
            const int W = vec_width(a);
            if (!W) {
                per_row({a});
                continue;
            }
            const std::string n = num(fresh()), C = "P.cols[" + num(a) + "]";
            for (int j = 0; j < K; j++) {
                line("uint64_t c" + n + "_" + num(j) + " = 0;");
                line("bool n" + n + "_" + num(j) + " = false;");
            }
            auto ahead = spec_vals.find(a);
            std::string t;
            if (ahead != spec_vals.end()) {
                t = ahead->second;
                open("if (specd || (full && " + any + ")) {");
                open("if (!specd) {");
                vec_load(a, W, t);
                close();
            } else {
                t = "t" + n;
                open("if (full && " + any + ") {");
                vec_decl(W, t);
                vec_load(a, W, t);
            }
            for (int j = 0; j < K; j++) {
                const std::string J = num(j), v = "c" + n + "_" + J;
                if (c.kind == CK_DICT)
                    line(v + " = (uint64_t)__ldg(" + C + ".gid + (" + t + "[" + J + "] < " + C + ".dict_len ? " + t + "[" + J +
                         "] : " + C + ".dict_len));");
                else if (W == 4)
                    line(v + " = (uint64_t)(int64_t)(int32_t)" + t + "[" + J + "];");
                else if (W == 8)
                    line(v + " = " + t + "[" + J + "];");
                else
                    line(v + " = (" + t + " >> " + num(8 * j) + ") & 0xFFull;");
            }
            close("} else {");
            ind_++;
            for (int j = 0; j < K; j++) {
                x = "x" + num(j);
                line("if (a" + num(j) + ") c" + n + "_" + num(j) + " = " + col_value(a) + ";");
            }
            x = "x";
            close();
            if (c.valid) {
                line("const uint64_t w" + n + " = " + any + " ? __ldg(" + C + ".valid + (x0.r >> 6)) : 0ull;");
                for (int j = 0; j < K; j++)
                    line("n" + n + "_" + num(j) + " = a" + num(j) + " && ((w" + n + " >> ((x0.r & 63u) + " + num(j) +
                         "u)) & 1ull);");
            } else {
                for (int j = 0; j < K; j++) line("n" + n + "_" + num(j) + " = a" + num(j) + ";");
            }
            for (int j = 0; j < K; j++) pre[j][a] = V{"c" + n + "_" + num(j), "n" + n + "_" + num(j)};
        }
    }

    // Speculative loads: with consecutive rows, the source columns that only later stages (and
    // the sink: `sink_slots`) read are loaded at the start of the tile, together with the first
    // stage's columns, when `spec` holds, so the tile waits for memory once instead of once per
    // stage.  `spec` is each thread's own guess: at least half of its rows passed the first stage
    // in its previous tile (rows that then fail only waste bytes that are read anyway when most
    // rows pass).
    // Only where the extra registers are free and the first stage is a filter: kernels whose
    // residency shared memory already limits (per-thread accumulators); a selective first join
    // probe or a register-limited kernel loses more than it gains (measured).
    bool speculate = false;
    std::set<int> sink_slots;
    std::map<int, std::string> spec_vals;

    // Hoisted per-thread load of an instruction field (literal bits, arena offsets, counts).
    std::string field(int idx, const char* f, const char* type) {
        std::string name = std::string("f_") + f + num(idx);
        if (hoisted_.insert(name).second)
            pre_ << "    const " << type << " " << name << " = P.prog[" << idx << "]." << f << ";\n";
        return name;
    }

    // Straight-line evaluation of a postfix program (eval_prog, one statement per instruction).
    V expr(const Prog& p) {
        std::vector<V> st;
        auto pop = [&]() {
            V v = st.back();
            st.pop_back();
            return v;
        };
        for (int i = 0; i < p.len; i++) {
            const int idx = p.start + i;
            const Instr& in = code_[idx];
            const std::string n = num(fresh()), v = "v" + n, k = "k" + n;
            switch (in.op) {
                case I_COL: {
                    auto it = cols.find(in.a);
                    if (it != cols.end()) {
                        st.push_back(it->second);
                        break;
                    }
                    line("const uint64_t " + v + " = " + col_value(in.a) + ";");
                    line("const bool " + k + " = " + col_valid(in.a) + ";");
                    st.push_back({v, k});
                    break;
                }
                case I_LIT: st.push_back({field(idx, "bits", "uint64_t"), in.lit_valid ? "true" : "false"}); break;
                case I_BIN: {
                    V r = pop(), l = pop();
                    line("bool " + k + ";");
                    line("const uint64_t " + v + " = binop(" + num(in.sub) + ", " + num(in.t) + ", " + l.v + ", " + r.v +
                         ", " + k + ", " + l.k + ", " + r.k + ");");
                    st.push_back({v, k});
                    break;
                }
                case I_NOT: {
                    V a = pop();
                    line("const uint64_t " + v + " = (~" + a.v + ") & 1ull;");
                    st.push_back({v, a.k});
                    break;
                }
                case I_NEG: {
                    V a = pop();
                    if (in.t == ML_TYPE_FLOAT64) line("const uint64_t " + v + " = " + a.v + " ^ 0x8000000000000000ull;");
                    else if (in.t == ML_TYPE_INT64) line("const uint64_t " + v + " = 0ull - " + a.v + ";");
                    else line("const uint64_t " + v + " = (uint64_t)(int64_t)(int32_t)(0u - (uint32_t)" + a.v + ");");
                    st.push_back({v, a.k});
                    break;
                }
                case I_ISNULL: {
                    V a = pop();
                    line("const uint64_t " + v + " = ((" + a.k + ") == " + (in.flag ? "true" : "false") +
                         ") ? 1ull : 0ull;");
                    st.push_back({v, "true"});
                    break;
                }
                case I_CAST: {
                    V a = pop();
                    line("const uint64_t " + v + " = cast_value(" + a.v + ", " + num(in.t) + ", " + num(in.sub) + ");");
                    st.push_back({v, a.k});
                    break;
                }
                case I_STRPRED: {
                    const DCol& c = P_.cols[in.a];
                    std::string C = "P.cols[" + num(in.a) + "]", R = row(c.src);
                    if (c.kind == CK_DICT) {
                        line("const uint64_t " + v + " = __ldg(P.luts[" + num(in.b) + "] + dict_code(" + C + ", " + R +
                             ")) != 0;");
                    } else {
                        std::string off = field(idx, "c", "int32_t");
                        line("const uint64_t " + v + " = str_pred(*(const StrSpec*)(P.arena + " + off +
                             "), P.arena, col_str(" + C + ", " + R + "));");
                    }
                    line("const bool " + k + " = " + col_valid(in.a) + ";");
                    st.push_back({v, k});
                    break;
                }
                case I_STRCMP_COL: {
                    const DCol& c = P_.cols[in.a];
                    const DCol& d = P_.cols[in.b];
                    line("const uint64_t " + v + " = cmp_result(" + num(in.sub) + ", str_cmp(col_str(P.cols[" + num(in.a) +
                         "], " + row(c.src) + "), col_str(P.cols[" + num(in.b) + "], " + row(d.src) + ")));");
                    line("const bool " + k + " = " + col_valid(in.a) + " && " + col_valid(in.b) + ";");
                    st.push_back({v, k});
                    break;
                }
                case I_INLIST: {
                    V a = pop();
                    std::string items = field(idx, "b", "int32_t"), cnt = field(idx, "c", "int32_t");
                    line("bool h" + n + " = false;");
                    open("for (int q = 0; q < " + cnt + "; q++) {");
                    line("const uint64_t it = ((const uint64_t*)(P.arena + " + items + "))[q];");
                    if (in.t == ML_TYPE_FLOAT64) line("h" + n + " |= as_f64(it) == as_f64(" + a.v + ");");
                    else line("h" + n + " |= it == " + a.v + ";");
                    close();
                    line("const uint64_t " + v + " = h" + n + " != " + (in.flag ? "true" : "false") + ";");
                    st.push_back({v, a.k});
                    break;
                }
                case I_SELECT: {  // stack: rest (2), cond (1), val (0)
                    V val = pop(), cond = pop(), rest = pop();
                    line("const bool t" + n + " = (" + cond.k + ") && ((" + cond.v + ") & 1);");
                    line("const uint64_t " + v + " = t" + n + " ? " + val.v + " : " + rest.v + ";");
                    line("const bool " + k + " = t" + n + " ? (" + val.k + ") : (" + rest.k + ");");
                    st.push_back({v, k});
                    break;
                }
                default: raise(ML_ERR_INTERNAL, "unknown instruction in pipeline program");
            }
        }
        if (st.size() != 1) raise(ML_ERR_INTERNAL, "malformed pipeline program");
        return st.back();
    }

    // Normalized key words of layout L (make_key) into `wk` (a declared uint64_t[2], zeroed).
    // A NULL key runs `on_null` (join keys) or sets its bit in `nm` (GROUP BY keys).
    // `ds` (optional): also sum the key's direct slot (AggArgs::dslots) into that variable.
    void key(const KeyLayout& L, const std::string& wk, const std::string& on_null, const std::string& nm,
             const std::string& ds = "") {
        for (int k = 0; k < L.nkeys; k++) {
            V e = expr(L.prog[k]);
            const KeyField& f = L.f[k];
            uint64_t mask = f.width >= 64 ? ~0ull : ((1ull << f.width) - 1);
            std::string val = e.v;
            if (f.type == ML_TYPE_FLOAT64) val = "(as_f64(" + e.v + ") == 0.0 ? 0ull : " + e.v + ")";
            std::string pack = wk + "[" + num(f.word) + "] |= ((" + val + ") & " + hex(mask) + ") << " + num(f.shift) + ";";
            if (nm.empty()) {
                line("if (!(" + e.k + ")) { " + on_null + " }");
                line(pack);
            } else {
                open("if (!(" + e.k + ")) {");
                line(nm + " |= " + num(1u << k) + "u;");
                close("} else {");
                ind_++;
                line(pack);
                if (!ds.empty()) {
                    const std::string v = f.type == ML_TYPE_BOOL ? "((uint32_t)(" + e.v + ") & 1u)" : "(uint32_t)(" + e.v + ")";
                    line(ds + " += (" + v + " - A.dbase[" + num(k) + "] + 1u) * A.dmul[" + num(k) + "];");
                }
                close();
            }
        }
    }

    // Streaming stages from `s` on for one row (run_stages): filters and probes `continue`
    // on failure; duplicate-key chains are walked as nested loops.
    template <class Sink> void stages(int s, Sink&& sink) {
        if (s == P_.nstages) {
            sink();
            return;
        }
        const Stage st = P_.stages[s];
        if (st.kind == 0) {
            open("{  // filter " + num(st.idx));
            V e = expr(P_.filters[st.idx]);
            line("if (!((" + e.k + ") && ((" + e.v + ") & 1))) continue;");
            stages(s + 1, sink);
            close();
            return;
        }
        const ProbeDev& pd = P_.probes[st.idx];
        std::string tag = "p" + num(s), p = num(st.idx);
        open("{  // probe " + p);
        line("uint64_t wk" + tag + "[2] = {0ull, 0ull};");
        key(pd.keys, "wk" + tag, "continue;", "");
        if (pd.dense && pd.late)
            line("const uint32_t hb" + tag + " = dense_slot(P.probes[" + p + "].dmin, P.probes[" + p + "].drange, wk" +
                 tag + "[0]);");
        else if (pd.dense && pd.member)
            line("const uint32_t hb" + tag + " = dense_member(P.probes[" + p + "].member, P.probes[" + p +
                 "].dmin, P.probes[" + p + "].drange, wk" + tag + "[0]);");
        else if (pd.dense)
            line("const uint32_t hb" + tag + " = dense_find(P.probes[" + p + "].dense, P.probes[" + p + "].dmin, P.probes[" +
                 p + "].drange, wk" + tag + "[0]);");
        else
            line("const uint32_t hb" + tag + " = table_find(P.probes[" + p + "].t, wk" + tag + ", key_hash(wk" + tag +
                 ", " + num(pd.keys.nwords) + "));");
        line("if (hb" + tag + " == kNone) continue;");
        if (st.idx == P_.head_probe) line("x.head = hb" + tag + ";");
        if (P_.has_chains && pd.next) {
            open("for (uint32_t b = hb" + tag + "; b != kNone; b = __ldg(P.probes[" + p + "].next + b)) {");
            line("x.b" + p + " = b;");
            stages(s + 1, sink);
            close();
        } else {
            line("x.b" + p + " = hb" + tag + ";");
            stages(s + 1, sink);
        }
        close();
    }

    // The same stages for kRowsPerThread rows x0.. with liveness flags a0..: each stage first
    // loads its columns for every live row, then evaluates (no chains: one match per probe).
    template <class Sink> void batched_stages(Sink&& sink) {
        const int K = rows_per_thread;
        auto rows = [&](auto&& f) {
            for (int j = 0; j < K; j++) {
                x = "x" + num(j);
                f(j, "a" + num(j));
            }
            x = "x";
        };
        // after a join probe (joins are where most rows of a star query drop out), a tile where no
        // lane of the warp has a live row skips the rest; the decision is warp-uniform, so the
        // warp stays converged.  Not after filters: the vote costs more than it saves when most
        // rows pass.
        auto skip_dead_tile = [&](int after) {
            if (tile_skip.empty() || P_.stages[after].kind != 1) return;
            std::string any;
            for (int j = 0; j < K; j++) any += (j ? " || a" : "a") + num(j);
            line("if (!__any_sync(0xFFFFFFFFu, " + any + ")) " + tile_skip);
        };
        spec_vals.clear();
        if (contig && speculate && P_.nstages > 0 && P_.stages[0].kind == 0) {
            std::set<int> first, later = sink_slots;
            const Stage s0 = P_.stages[0];
            if (s0.kind == 0) slots_of(P_.filters[s0.idx], first);
            else for (int k = 0; k < P_.probes[s0.idx].keys.nkeys; k++) slots_of(P_.probes[s0.idx].keys.prog[k], first);
            for (int s = 1; s < P_.nstages; s++) {
                const Stage st = P_.stages[s];
                if (st.kind == 0) slots_of(P_.filters[st.idx], later);
                else for (int k = 0; k < P_.probes[st.idx].keys.nkeys; k++) slots_of(P_.probes[st.idx].keys.prog[k], later);
            }
            for (int a : later) {
                const int W = vec_width(a);
                if (!W || first.count(a)) continue;
                const std::string t = "sp" + num(fresh());
                vec_decl(W, t);
                spec_vals[a] = t;
            }
            if (!spec_vals.empty()) {
                if (hoisted_.insert("spec").second) pre_ << "    bool spec = true;  // speculative loads (see Gen::spec_vals)\n";
                // this tile's decision (spec itself is updated for the next tile after stage 0)
                line("const bool specd = full && spec;");
                open("if (specd) {");
                for (auto& e : spec_vals) vec_load(e.first, vec_width(e.first), e.second);
                close();
            }
        }
        for (int s = 0; s < P_.nstages; s++) {
            if (s == 1 && !spec_vals.empty()) {  // this tile's first-stage pass rate decides the next tile
                std::string alive;
                for (int j = 0; j < K; j++) alive += (j ? " + (a" : "(a") + num(j) + " ? 1 : 0)";
                line("spec = 2 * (" + alive + ") >= " + num(K) + ";");
            }
            if (s > 0) skip_dead_tile(s - 1);
            const Stage st = P_.stages[s];
            std::set<int> slots;
            if (st.kind == 0) {
                slots_of(P_.filters[st.idx], slots);
                std::vector<std::map<int, V>> pre;
                preload_rows(slots, pre);
                rows([&](int j, const std::string& a) {
                    cols = pre[j];
                    open("if (" + a + ") {  // filter " + num(st.idx));
                    V e = expr(P_.filters[st.idx]);
                    line(a + " = (" + e.k + ") && ((" + e.v + ") & 1);");
                    close();
                });
                cols.clear();
                continue;
            }
            const ProbeDev& pd = P_.probes[st.idx];
            const std::string p = num(st.idx);
            for (int k = 0; k < pd.keys.nkeys; k++) slots_of(pd.keys.prog[k], slots);
            std::vector<std::map<int, V>> pre;
            preload_rows(slots, pre);
            if (pd.dense) {  // direct index: one 4-byte load per row, issued for every row first
                rows([&](int j, const std::string& a) {
                    cols = pre[j];
                    std::string tag = "p" + num(s) + "_" + num(j);
                    line("uint64_t wk" + tag + "[2] = {0ull, 0ull};");
                    line("uint32_t d" + tag + " = kNone;");
                    open("if (" + a + ") {  // probe " + p + " (dense index)");
                    key(pd.keys, "wk" + tag, a + " = false;", "");
                    if (pd.late)  // membership is checked per group at finalize: no index read per row
                        line("d" + tag + " = dense_slot(P.probes[" + p + "].dmin, P.probes[" + p + "].drange, wk" + tag +
                             "[0]);");
                    else if (pd.member)  // semi-join: one bit per key
                        line("d" + tag + " = dense_member(P.probes[" + p + "].member, P.probes[" + p + "].dmin, P.probes[" +
                             p + "].drange, wk" + tag + "[0]);");
                    else
                        line("d" + tag + " = dense_find(P.probes[" + p + "].dense, P.probes[" + p + "].dmin, P.probes[" +
                             p + "].drange, wk" + tag + "[0]);");
                    close();
                });
                cols.clear();
                rows([&](int j, const std::string& a) {
                    std::string tag = "p" + num(s) + "_" + num(j);
                    open("if (" + a + ") {");
                    line(a + " = d" + tag + " != kNone;");
                    line(x + ".b" + p + " = d" + tag + ";");
                    if (st.idx == P_.head_probe) line(x + ".head = d" + tag + ";");
                    close();
                });
                continue;
            }
            rows([&](int j, const std::string& a) {
                cols = pre[j];
                std::string tag = "p" + num(s) + "_" + num(j);
                line("uint64_t wk" + tag + "[2] = {0ull, 0ull};");
                line("uint64_t h" + tag + " = 0;");
                open("if (" + a + ") {  // probe " + p + " key");
                key(pd.keys, "wk" + tag, a + " = false;", "");
                line("h" + tag + " = key_hash(wk" + tag + ", " + num(pd.keys.nwords) + ");");
                close();
            });
            cols.clear();
            rows([&](int j, const std::string& a) {
                std::string tag = "p" + num(s) + "_" + num(j);
                line("ulonglong2 s" + tag + " = make_ulonglong2(0ull, 0ull);");
                line("if (" + a + ") s" + tag + " = slot_load(P.probes[" + p + "].t, h" + tag + " & P.probes[" + p +
                     "].t.mask);");
            });
            rows([&](int j, const std::string& a) {
                std::string tag = "p" + num(s) + "_" + num(j);
                open("if (" + a + ") {  // probe " + p);
                line("const uint32_t b = table_find_from(P.probes[" + p + "].t, wk" + tag + ", h" + tag + ", s" + tag + ");");
                line(a + " = b != kNone;");
                line(x + ".b" + p + " = b;");
                if (st.idx == P_.head_probe) line(x + ".head = b;");
                close();
            });
        }
        if (P_.nstages == 1 && !spec_vals.empty()) {  // a single stage: decide before the sink
            std::string alive;
            for (int j = 0; j < K; j++) alive += (j ? " + (a" : "(a") + num(j) + " ? 1 : 0)";
            line("spec = 2 * (" + alive + ") >= " + num(K) + ";");
        }
        if (P_.nstages > 0) skip_dead_tile(P_.nstages - 1);
        sink(rows);
    }

   private:
    const std::vector<Instr>& code_;
    const PipeArgs& P_;
    std::ostringstream pre_, o_;
    std::set<std::string> hoisted_;
    int nv_ = 0, ind_ = 2;
};

// Batched form applies when no probe walks chains (at most one match per probe row).
bool batchable(const PipeArgs& P) { return !P.has_chains; }

// Declarations of the batched rows x0.. / a0.. of the tile at `base`: strided (x<j>.r = base +
// j * 256 + thread) or, with `contig`, consecutive (x<j>.r = r0 + j, r0 = base + K * thread, and
// `full` when all K are rows).
std::string tile_rows(const PipeArgs& P, int K, bool contig, const std::string& ind) {
    std::string s;
    if (contig) {  // 32-bit row arithmetic (contig_ok bounds the row count below 2^32 - 2^16)
        s += ind + "const uint32_t r0 = (uint32_t)base + threadIdx.x * " + num(K) + "u;\n";
        s += ind + "const uint32_t n32 = (uint32_t)P.n;\n";
        s += ind + "const bool full = r0 + " + num(K) + "u <= n32;\n";
    }
    for (int j = 0; j < K; j++) {
        std::string J = num(j), x = "x" + J, a = "a" + J;
        s += ind + "RowCtx " + x + ";\n";
        if (contig) {
            s += ind + "bool " + a + " = r0 + " + J + "u < n32;\n";
            s += ind + x + ".r = r0 + " + J + "u;\n";
        } else {
            s += ind + "const int64_t i" + J + " = base + " + J + " * (int64_t)blockDim.x + threadIdx.x;\n";
            s += ind + "bool " + a + " = i" + J + " < P.n;\n";
            if (P.sel)  // a selected row id past the batch is skipped and reported (sel_row)
                s += ind + x + ".r = " + a + " ? sel_row(P, i" + J + ", " + a + ") : 0u;\n";
            else
                s += ind + x + ".r = " + a + " ? (uint32_t)i" + J + " : 0u;\n";
        }
        s += ind + x + ".b0 = " + x + ".b1 = " + x + ".b2 = " + x + ".b3 = 0;\n";
        s += ind + x + ".head = 0;\n";
    }
    return s;
}

// Consecutive rows per thread need no selection vector and every fixed-width or dictionary
// source column aligned to 16 bytes (the vector loads' width).
bool contig_ok(const PipeArgs& P) {
    if (P.sel || P.n > 0xFFFF0000ll) return false;
    for (const DCol& c : P.cols)
        if (c.src == 0 && (c.kind == CK_FIXED || c.kind == CK_DICT) && ((uintptr_t)c.data & 15)) return false;
    return true;
}

std::string row_loop(const PipeArgs& P, bool batched, const std::string& body, int K = kRowsPerThread,
                     bool contig = false) {
    std::string s;
    if (!batched) {
        s += "    const int64_t stride = (int64_t)gridDim.x * blockDim.x;\n";
        s += "    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < P.n; i += stride) {\n";
        s += "        RowCtx x;\n";
        s += P.sel ? "        bool sel_ok = true;\n        x.r = sel_row(P, i, sel_ok);\n        if (!sel_ok) continue;\n"
                   : "        x.r = (uint32_t)i;\n";
        s += "        x.b0 = x.b1 = x.b2 = x.b3 = 0;\n        x.head = 0;\n";
    } else {
        s += "    const int64_t tile = (int64_t)" + num(K) + " * blockDim.x;\n";
        s += "    for (int64_t base = (int64_t)blockIdx.x * tile; base < P.n; base += (int64_t)gridDim.x * tile) {\n";
        s += tile_rows(P, K, contig, "        ");
    }
    s += body;
    // Batched tiles have the same trip count in every lane: reconverge the warp once per tile,
    // so lanes split by a data-dependent branch (a group's first lookup, a claimed slot) do
    // not go on issuing the next tile's loads separately.
    if (batched) s += "        __syncwarp();\n";
    s += "    }\n";
    return s;
}

// The aggregate update of one row combination (agg_update + agg_fold), in `g`'s current
// row context; `g.fail` abandons the combination.
void emit_aggregate(Gen& g, const AggArgs& A) {
    const bool smem = A.smem_groups > 0;
    const std::string S = num(A.stride);
    if (A.group_probe >= 0) {
        g.line("const uint32_t g = " + g.x + ".head;");
    } else if (A.ungrouped) {
        g.line("const uint32_t g = 0;");
    } else {
        const bool direct = A.dslots > 0;  // implies agg_direct_on(A)
        g.line("uint64_t wkg[2] = {0ull, 0ull};");
        g.line("uint32_t nmg = 0;");
        if (direct) g.line("uint32_t dsg = 0;");
        g.key(A.keys, "wkg", "", "nmg", direct ? "dsg" : "");
        g.line("bool ins = false;");
        // with direct slots, the CTA's index first: the global table only on the slot's first use
        g.line(direct ? "uint32_t g = dsg < A.dslots ? dsl[dsg] - 1u : kNone;" : "uint32_t g = kNone;");
        g.open("if (g == kNone) {");
        g.line("uint64_t slot;");
        g.line("g = table_upsert(A.t, wkg, nmg, key_hash(wkg, " + num(A.keys.nwords) +
               ", nmg), P.err, [&]() -> uint32_t { const uint32_t id = atomicAdd(A.ngroups, 1u); "
               "return id < A.gid_cap ? id : kNone; }, &ins, &slot, A.ngroups, A.gid_cap);");
        if (direct) g.line("if (g != kNone && dsg < A.dslots) dsl[dsg] = g + 1u;");
        g.close();
        g.open("if (g == kNone) {");
        g.line("record_overflow(P, A, " + g.x + ");");
        g.line(g.fail);
        g.close();
        g.open("if (ins) {");
        g.line("A.gkeys[g] = wkg[0];");
        if (A.keys.nwords > 1) g.line("A.gkeys[(uint64_t)A.gid_cap + g] = wkg[1];");
        g.line("A.gnull[g] = nmg;");
        g.close();
    }
    // every aggregate's argument, evaluated once for whichever accumulators the group uses
    std::vector<Gen::V> args(A.nagg);
    for (int k = 0; k < A.nagg; k++) {
        const AggDev& a = A.aggs[k];
        if (a.func != ML_AGG_COUNT_STAR && a.has_arg) args[k] = g.expr(a.arg);
    }
    const int priv = A.priv_groups;
    if (priv > 0) {  // per-thread accumulators: plain updates, no atomics
        g.open("if (g < " + num(priv) + "u) {");
        g.line("uint64_t* pv = smem + (uint64_t)A.smem_groups * " + S + " + (uint64_t)g * " + num(A.stride * 256) +
               " + threadIdx.x;");
        g.line("pv[0] += 1ull;");
        for (int k = 0; k < A.nagg; k++) {
            const AggDev& a = A.aggs[k];
            if (a.func == ML_AGG_COUNT_STAR) continue;
            const std::string w = "pv[" + num(a.off * 256) + "]", v = a.has_arg ? args[k].v : "0ull";
            if (a.has_arg) g.open("if (" + args[k].k + ") {");
            switch (a.kind) {
                case A_SUM_I64: g.line(w + " += " + v + ";"); break;
                case A_SUM_F64: g.line(w + " = f64_bits(__dadd_rn(as_f64(" + w + "), as_f64(" + v + ")));"); break;
                case A_AVG:
                    g.line(w + " = f64_bits(__dadd_rn(as_f64(" + w + "), as_f64(" + v + ")));");
                    g.line("pv[" + num((a.off + 1) * 256) + "] += 1ull;");
                    break;
                case A_MIN_I64: g.line(w + " = (uint64_t)min((long long)" + w + ", (long long)" + v + ");"); break;
                case A_MAX_I64: g.line(w + " = (uint64_t)max((long long)" + w + ", (long long)" + v + ");"); break;
                case A_MIN_F64:
                    g.line(w + " = (uint64_t)min((unsigned long long)" + w + ", (unsigned long long)f64_order(as_f64(" + v +
                           ")));");
                    break;
                case A_MAX_F64:
                    g.line(w + " = (uint64_t)max((unsigned long long)" + w + ", (unsigned long long)f64_order(as_f64(" + v +
                           ")));");
                    break;
                default: g.line(w + " += 1ull;"); break;  // COUNT(x)
            }
            if (a.has_arg) g.close();
        }
        g.close("} else {");
        g.open("");
    }
    if (smem) {
        g.line("uint64_t* blk = (int)g < A.smem_groups ? smem + (uint64_t)g * " + S + " : A.acc + (uint64_t)g * " + S + ";");
        g.line("atomicAdd((unsigned long long*)blk, 1ull);");
    } else {
        g.line("uint64_t* blk = A.acc + (uint64_t)g * " + S + ";");
        g.line("count_global(blk);");
    }
    for (int k = 0; k < A.nagg; k++) {
        const AggDev& a = A.aggs[k];
        if (a.func == ML_AGG_COUNT_STAR) continue;  // the group's row counter (word 0)
        g.open("{  // aggregate " + num(k));
        std::string v = "0ull";
        if (a.has_arg) {
            g.open("if (" + args[k].k + ") {");
            v = args[k].v;
        }
        g.line(std::string(smem ? "acc_apply(" : "acc_apply_global(") + num(a.kind) + ", blk + " + num(a.off) + ", " + v +
               ");");
        if (a.count_valid) {
            if (smem) g.line("atomicAdd((unsigned long long*)A.aggs[" + num(k) + "].vcnt + g, 1ull);");
            else g.line("count_global(A.aggs[" + num(k) + "].vcnt + g);");
        }
        if (a.has_arg) g.close();
        g.close();
    }
    if (priv > 0) g.close();
}

// What each word of a group block holds: 0 = integer count or sum, 1 = f64 sum, 2/3 = signed
// min/max, 4/5 = order-mapped f64 min/max (unsigned compare).
std::vector<int> word_ops(const AggArgs& A) {
    std::vector<int> ops(A.stride, 0);
    for (int k = 0; k < A.nagg; k++) {
        const AggDev& a = A.aggs[k];
        if (a.func == ML_AGG_COUNT_STAR) continue;
        switch (a.kind) {
            case A_SUM_F64:
            case A_AVG: ops[a.off] = 1; break;
            case A_MIN_I64: ops[a.off] = 2; break;
            case A_MAX_I64: ops[a.off] = 3; break;
            case A_MIN_F64: ops[a.off] = 4; break;
            case A_MAX_F64: ops[a.off] = 5; break;
            default: break;
        }
    }
    return ops;
}

// Start values of the per-thread accumulators, then (after the rows) their reduction over the
// CTA's threads and one global update per group and word (skipped for groups with no rows).
std::string priv_init(const AggArgs& A) {
    const int S = A.stride, P = A.priv_groups;
    std::string id = "{";
    for (int w = 0; w < S; w++) id += (w ? ", " : "") + std::string("0ull");
    id += "}";
    std::string src;
    src += "    {\n        uint64_t idw[" + num(S) + "] = " + id + ";\n";
    for (int k = 0; k < A.nagg; k++)
        if (A.aggs[k].func != ML_AGG_COUNT_STAR)
            src += "        idw[" + num(A.aggs[k].off) + "] = agg_identity(" + num(A.aggs[k].kind) + ");\n";
    src += "        uint64_t* pv = smem + (uint64_t)A.smem_groups * " + num(S) + ";\n";
    src += "        for (int i = threadIdx.x; i < " + num(P * S * 256) + "; i += blockDim.x) pv[i] = idw[(i >> 8) % " +
           num(S) + "];\n";
    src += "    }\n    __syncthreads();\n";
    return src;
}

std::string priv_flush(const AggArgs& A) {
    const int S = A.stride, P = A.priv_groups;
    const std::vector<int> ops = word_ops(A);
    std::string src;
    src += "    {\n";
    src += "        const uint64_t* pv = smem + (uint64_t)A.smem_groups * " + num(S) + ";\n";
    src += "        const int lane = threadIdx.x & 31;\n";
    src += "        for (int pair = threadIdx.x >> 5; pair < " + num(P * S) + "; pair += blockDim.x >> 5) {\n";
    src += "            const int gg = pair / " + num(S) + ", w = pair % " + num(S) + ";\n";
    src += "            const uint64_t* c = pv + (uint64_t)gg * " + num(S * 256) + ";\n";
    src += "            unsigned long long rows = 0;\n";
    src += "            for (int t = lane; t < 256; t += 32) rows += c[t];\n";
    src += "            for (int o = 16; o; o >>= 1) rows += __shfl_xor_sync(0xFFFFFFFFu, rows, o);\n";
    src += "            if (rows == 0) continue;  // no row of this group in this CTA\n";
    src += "            const uint64_t* x = c + w * 256;\n";
    src += "            uint64_t* dst = A.acc + (uint64_t)gg * " + num(S) + " + w;\n";
    src += "            switch (w) {\n";
    for (int w = 0; w < S; w++) {
        src += "                case " + num(w) + ": {\n";
        switch (ops[w]) {
            case 1:
                src += "                    double v = 0.0;\n";
                src += "                    for (int t = lane; t < 256; t += 32) v = __dadd_rn(v, as_f64(x[t]));\n";
                src += "                    for (int o = 16; o; o >>= 1) v = __dadd_rn(v, __shfl_xor_sync(0xFFFFFFFFu, v, o));\n";
                src += "                    if (lane == 0) atomicAdd((double*)dst, v);\n";
                break;
            case 2:
            case 3: {
                const char* f = ops[w] == 2 ? "min" : "max";
                src += "                    long long v = (long long)x[lane];\n";
                src += std::string("                    for (int t = lane + 32; t < 256; t += 32) v = ") + f +
                       "(v, (long long)x[t]);\n";
                src += std::string("                    for (int o = 16; o; o >>= 1) v = ") + f +
                       "(v, (long long)__shfl_xor_sync(0xFFFFFFFFu, (unsigned long long)v, o));\n";
                src += std::string("                    if (lane == 0) atomic") + (ops[w] == 2 ? "Min" : "Max") +
                       "((long long*)dst, v);\n";
                break;
            }
            case 4:
            case 5: {
                const char* f = ops[w] == 4 ? "min" : "max";
                src += "                    unsigned long long v = x[lane];\n";
                src += std::string("                    for (int t = lane + 32; t < 256; t += 32) v = ") + f +
                       "(v, (unsigned long long)x[t]);\n";
                src += std::string("                    for (int o = 16; o; o >>= 1) v = ") + f +
                       "(v, __shfl_xor_sync(0xFFFFFFFFu, v, o));\n";
                src += std::string("                    if (lane == 0) atomic") + (ops[w] == 4 ? "Min" : "Max") +
                       "((unsigned long long*)dst, v);\n";
                break;
            }
            default:
                src += "                    unsigned long long v = 0;\n";
                src += "                    for (int t = lane; t < 256; t += 32) v += x[t];\n";
                src += "                    for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xFFFFFFFFu, v, o);\n";
                src += "                    if (lane == 0 && v) atomicAdd((unsigned long long*)dst, v);\n";
                break;
        }
        src += "                    break;\n                }\n";
    }
    src += "            }\n        }\n    }\n";
    return src;
}

const char* kPrelude = "#include \"ml_agg.cuh\"\nusing namespace mlg;\n";

}  // namespace

std::string jit_agg_source(const Pipeline& pipe, const PipeArgs& P, const AggArgs& A, bool contig) {
    Gen g(pipe.C.code, P);
    const bool smem = A.smem_groups > 0;
    const bool batched = batchable(P);
    g.contig = contig && batched;
    g.tile_skip = "continue;";  // the tile loop of row_loop
    g.speculate = A.priv_groups > 0;
    if (A.group_probe < 0 && !A.ungrouped)
        for (int k = 0; k < A.keys.nkeys; k++) g.slots_of(A.keys.prog[k], g.sink_slots);
    for (int k = 0; k < A.nagg; k++)
        if (A.aggs[k].has_arg && A.aggs[k].func != ML_AGG_COUNT_STAR) g.slots_of(A.aggs[k].arg, g.sink_slots);
    if (batched) {
        g.fail = "break;";
        g.batched_stages([&](auto&& rows) {
            std::set<int> slots;
            if (A.group_probe < 0 && !A.ungrouped)
                for (int k = 0; k < A.keys.nkeys; k++) g.slots_of(A.keys.prog[k], slots);
            for (int k = 0; k < A.nagg; k++)
                if (A.aggs[k].has_arg && A.aggs[k].func != ML_AGG_COUNT_STAR) g.slots_of(A.aggs[k].arg, slots);
            std::vector<std::map<int, Gen::V>> pre;
            g.preload_rows(slots, pre);
            rows([&](int j, const std::string& a) {
                g.cols = pre[j];
                g.open("if (" + a + ") do {  // aggregate");
                emit_aggregate(g, A);
                g.close("} while (0);");
            });
            g.cols.clear();
        });
    } else {
        g.stages(0, [&]() {
            g.open("{  // aggregate");
            emit_aggregate(g, A);
            g.close();
        });
    }
    std::string src = kPrelude;
    src += "extern \"C\" __global__ void __launch_bounds__(256) ml_pipeline_aggregate(const __grid_constant__ PipeArgs P, "
           "const __grid_constant__ AggArgs A) {\n";
    src += "    extern __shared__ __align__(16) uint64_t smem[];\n";
    if (smem) src += "    smem_setup(A, smem);\n    __syncthreads();\n";
    if (A.dslots > 0) src += "    uint32_t* const dsl = direct_slots(A, smem);\n";
    if (A.priv_groups > 0) src += priv_init(A);
    src += g.pre();
    src += row_loop(P, batched, g.body(), kRowsPerThread, g.contig);
    if (smem) src += "    __syncthreads();\n    smem_flush(A, smem);\n";
    if (A.priv_groups > 0) src += priv_flush(A);
    src += "}\n";
    return src;
}

int jit_rows_per_thread(const PipeArgs& P) { return batchable(P) ? kRowsPerThread : 1; }

namespace {

// The launch arguments with every runtime-only value cleared (pointers reduced to presence,
// sizes and constants to zero): equal signatures give equal generated sources.
std::string signature(char kind, const PipeArgs& P, const AggArgs* A, const KeyLayout* L) {
    PipeArgs p = P;
    p.n = 0;
    p.sel = P.sel ? (const uint32_t*)1 : nullptr;
    p.prog = nullptr;
    p.arena = nullptr;
    p.err = nullptr;
    for (auto& l : p.luts) l = nullptr;
    for (auto& c : p.cols) {
        c.data = nullptr;
        c.off = nullptr;
        c.valid = c.valid ? (const uint64_t*)1 : nullptr;
        c.gid = c.gid ? (const uint32_t*)1 : nullptr;
        c.dbytes = nullptr;
        c.n = 0;
        c.dict_len = 0;
    }
    for (auto& pd : p.probes) {
        pd.t = TableView{};
        pd.next = pd.next ? (const uint32_t*)1 : nullptr;
        pd.dense = pd.dense ? (const uint32_t*)1 : nullptr;
        pd.member = pd.member ? (const uint32_t*)1 : nullptr;
        pd.dmin = pd.drange = 0;
    }
    std::string key(1, kind);
    key.append((const char*)&p, sizeof p);
    if (A) {
        AggArgs a = *A;
        a.t = TableView{};
        a.gkeys = nullptr;
        a.gnull = nullptr;
        a.ngroups = nullptr;
        a.acc = nullptr;
        a.ovf = nullptr;
        a.ovf_count = nullptr;
        a.gid_cap = 0;
        a.ovf_cap = 0;
        a.smem_groups = a.smem_groups > 0;
        a.dslots = a.dslots > 0;
        for (int k = 0; k < kMaxKeys; k++) a.dmul[k] = a.dbase[k] = 0;
        for (auto& g : a.aggs) g.vcnt = g.vcnt ? (uint64_t*)1 : nullptr;
        key.append((const char*)&a, sizeof a);
    }
    if (L) key.append((const char*)L, sizeof *L);
    return key;
}

template <class Make>
void* memoized(const Pipeline& pipe, std::string key, Make make) {
    {
        std::lock_guard<std::mutex> g(pipe.jit_mu);
        for (auto& e : pipe.jit_memo)
            if (e.first == key) return e.second;
    }
    void* fn = make();
    std::lock_guard<std::mutex> g(pipe.jit_mu);
    if (pipe.jit_memo.size() >= 16) pipe.jit_memo.erase(pipe.jit_memo.begin());
    pipe.jit_memo.emplace_back(std::move(key), fn);
    return fn;
}

}  // namespace

// String MIN/MAX look their strings' ranks up (AggArgs::str_rank): the interpreter kernels do.
bool has_string_minmax(const AggArgs& A) {
    for (int k = 0; k < A.nagg; k++)
        if (A.aggs[k].kind == A_MIN_STR || A.aggs[k].kind == A_MAX_STR) return true;
    return false;
}

void* jit_agg_kernel(Ctx* ctx, const Pipeline& pipe, const PipeArgs& P, const AggArgs& A) {
    if (!jit_enabled(ctx) || has_string_minmax(A)) return nullptr;
    const bool contig = batchable(P) && contig_ok(P);
    return memoized(pipe, signature('a', P, &A, nullptr) + std::string((const char*)&ctx->device, sizeof(int)) +
                              (contig ? "c" : "s"),
                    [&] { return (void*)get_kernel(ctx, jit_agg_source(pipe, P, A, contig), "ml_pipeline_aggregate"); });
}

void* jit_agg_resume_kernel(Ctx* ctx, const Pipeline& pipe, const PipeArgs& P, const AggArgs& A) {
    if (!jit_enabled(ctx) || has_string_minmax(A)) return nullptr;
    // the rows a full table sent to the overflow list, aggregated again after the table grew
    Gen g(pipe.C.code, P);
    g.fail = "break;";
    g.open("do {  // aggregate");
    emit_aggregate(g, A);
    g.close("} while (0);");
    const bool smem = A.smem_groups > 0;
    std::string src = kPrelude;
    src += "extern \"C\" __global__ void __launch_bounds__(256) ml_pipeline_aggregate_resume(const __grid_constant__ "
           "PipeArgs P, const __grid_constant__ AggArgs A, const uint32_t* rows, uint64_t count, int w) {\n";
    src += "    extern __shared__ __align__(16) uint64_t smem[];\n";
    if (smem) src += "    smem_setup(A, smem);\n    __syncthreads();\n";
    if (A.dslots > 0) src += "    uint32_t* const dsl = direct_slots(A, smem);\n";
    src += g.pre();
    src += "    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;\n";
    src += "    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += stride) {\n";
    src += "        const uint32_t* c = rows + i * (uint64_t)w;\n";
    src += "        RowCtx x;\n        x.r = c[0];\n        x.b0 = w > 1 ? c[1] : 0;\n        x.b1 = w > 2 ? c[2] : 0;\n";
    src += "        x.b2 = w > 3 ? c[3] : 0;\n        x.b3 = w > 4 ? c[4] : 0;\n        x.head = 0;\n";
    src += g.body();
    src += "    }\n";
    if (smem) src += "    __syncthreads();\n    smem_flush(A, smem);\n";
    src += "}\n";
    return (void*)get_kernel(ctx, src, "ml_pipeline_aggregate_resume");
}

void* jit_join_insert_kernel(Ctx* ctx, const Pipeline& pipe, const PipeArgs& P, const KeyLayout& L) {
    if (!jit_enabled(ctx)) return nullptr;
    // build_table (join.rs:160-203): distinct keys in the table, duplicates chained in `next`.
    // One-word keys insert with a single 128-bit CAS; wider keys use the claim protocol.
    Gen g(pipe.C.code, P);
    g.open("{  // insert");
    g.line("uint64_t wkk[2] = {0ull, 0ull};");
    g.key(L, "wkk", "continue;", "");
    g.line("bool ins;");
    g.line("uint64_t slot;");
    g.line("const uint32_t r = x.r;");
    if (L.nwords == 1)
        g.line("const uint32_t p = table_insert_row1(t, wkk[0], key_hash(wkk, 1), r, &ins, &slot);");
    else
        g.line("const uint32_t p = table_upsert(t, wkk, 0u, key_hash(wkk, " + num(L.nwords) +
               "), P.err, [&]() { return r; }, &ins, &slot);");
    g.line("if (p == kNone) continue;");
    g.open("if (!ins) {");
    g.line("const uint32_t old = atomicExch((uint32_t*)slot_at(t, slot) + 1, r);");
    g.line("next[r] = old;");
    g.line("if (*dup_flag == 0) atomicExch(dup_flag, 1u);");
    g.close();
    g.close();
    std::string src = kPrelude;
    src += "extern \"C\" __global__ void __launch_bounds__(256) ml_join_insert(const __grid_constant__ PipeArgs P, "
           "const __grid_constant__ KeyLayout L, TableView t, uint32_t* next, uint32_t* dup_flag, int64_t n) {\n";
    src += g.pre();
    src += "    const int64_t stride = (int64_t)gridDim.x * blockDim.x;\n";
    src += "    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {\n";
    src += "        RowCtx x;\n        x.r = (uint32_t)i;\n        x.b0 = x.b1 = x.b2 = x.b3 = 0;\n        x.head = 0;\n";
    src += g.body();
    src += "    }\n}\n";
    return (void*)get_kernel(ctx, src, "ml_join_insert");
}

void* jit_select_kernel(Ctx* ctx, const Pipeline& pipe, const PipeArgs& P) {
    if (!jit_enabled(ctx) || !batchable(P)) return nullptr;
    const bool contig = contig_ok(P);
    return memoized(pipe, signature('s', P, nullptr, nullptr) + std::string((const char*)&ctx->device, sizeof(int)) +
                              (contig ? "c" : "s"),
                    [&] { return (void*)get_kernel(ctx, jit_select_source(pipe, P, contig), "ml_select_flags"); });
}

std::string jit_select_source(const Pipeline& pipe, const PipeArgs& P, bool contig) {
    {
        // Pass bits and per-chunk pass counts of 2048-row chunks (the layout of the ahead-of-time
        // k_select_flags), 8 rows per thread with every chunk's loads issued together.  CTAs stride
        // over the chunks; each warp adds its count to the chunk's (zeroed) counter.
        Gen g(pipe.C.code, P);
        g.rows_per_thread = 8;
        g.contig = contig;
        g.fail = "break;";
        g.batched_stages([&](auto&&) {});
        const int K = g.rows_per_thread;
        std::string src = kPrelude;
        src += "extern \"C\" __global__ void __launch_bounds__(256) ml_select_flags(const __grid_constant__ PipeArgs P, "
               "uint32_t* bits, uint32_t* chunk_counts) {\n";
        src += g.pre();
        src += "    const int lane = threadIdx.x & 31;\n";
        src += "    const int64_t chunks = (P.n + 2047) / 2048;\n";
        src += "    for (int64_t c = blockIdx.x; c < chunks; c += gridDim.x) {\n";
        src += "        const int64_t base = c * 2048;\n";
        if (contig) {
            // thread t's rows are base + 8t .. +7 (the per-CTA tile of the strided form, 8 x 256)
            src += tile_rows(P, K, true, "        ");
            src += g.body();
            src += "        uint32_t byte = 0;\n";
            for (int j = 0; j < K; j++) src += "        byte |= (a" + num(j) + " ? 1u : 0u) << " + num(j) + ";\n";
            // a 32-row word is the bytes of 4 consecutive lanes
            src += "        uint32_t word = byte << (8 * (lane & 3));\n";
            src += "        word |= __shfl_xor_sync(0xFFFFFFFFu, word, 1);\n";
            src += "        word |= __shfl_xor_sync(0xFFFFFFFFu, word, 2);\n";
            src += "        if ((lane & 3) == 0 && r0 < P.n) bits[r0 >> 5] = word;\n";
            src += "        const uint32_t cnt = __reduce_add_sync(0xFFFFFFFFu, (uint32_t)__popc(byte));\n";
        } else {
            src += tile_rows(P, K, false, "        ");
            src += g.body();
            src += "        uint32_t cnt = 0;\n";
            for (int j = 0; j < K; j++) {
                std::string J = num(j);
                src += "        {\n            const uint32_t b = __ballot_sync(0xFFFFFFFFu, a" + J + ");\n";
                src += "            const int64_t w0 = base + " + J + " * 256 + (threadIdx.x & ~31);\n";
                src += "            if (lane == 0 && w0 < P.n) bits[w0 >> 5] = b;\n";
                src += "            cnt += __popc(b);\n        }\n";
            }
        }
        src += "        if (lane == 0 && cnt) atomicAdd(chunk_counts + c, cnt);\n";
        src += "        __syncwarp();\n";
        src += "    }\n}\n";
        return src;
    }
}

void* jit_hll_kernel(Ctx* ctx, const Pipeline& pipe, const PipeArgs& P, const KeyLayout& L) {
    if (!jit_enabled(ctx) || !batchable(P)) return nullptr;
    const bool contig = contig_ok(P);
    std::string key = signature('h', P, nullptr, &L) + std::string((const char*)&ctx->device, sizeof(int)) +
                      (contig ? "c" : "s");
    return memoized(pipe, key, [&] { return (void*)get_kernel(ctx, jit_hll_source(pipe, P, L, contig), "ml_card_hll"); });
}

std::string jit_hll_source(const Pipeline& pipe, const PipeArgs& P, const KeyLayout& L, bool contig) {
    {
        // The cardinality features scan: every row's key hashed into 2^14 HyperLogLog registers
        // privatized in shared memory, NULL count and the first key word's range; each CTA
        // leaves its registers as bytes in cta_regs[blockIdx.x][4096 words] for the merge kernel.
        Gen g(pipe.C.code, P);
        g.rows_per_thread = 8;
        g.contig = contig;
        g.fail = "break;";
        g.batched_stages([&](auto&& rows) {
            std::set<int> slots;
            for (int k = 0; k < L.nkeys; k++) g.slots_of(L.prog[k], slots);
            std::vector<std::map<int, Gen::V>> pre;
            g.preload_rows(slots, pre);
            rows([&](int j, const std::string& a) {
                g.cols = pre[j];
                g.open("if (" + a + ") {  // key " + num(j));
                g.line("uint64_t wk[2] = {0ull, 0ull};");
                g.line("uint32_t nmk = 0;");
                g.key(L, "wk", "", "nmk");
                g.open("if (nmk) {");
                g.line("nulls++;");
                g.close("} else {");
                g.open("");
                g.line("lo = wk[0] < lo ? wk[0] : lo;");
                g.line("hi = wk[0] > hi ? wk[0] : hi;");
                g.close();
                g.line("const uint64_t h = hll_mix(key_hash(wk, " + num(L.nwords) + ", nmk));");
                g.line("const uint64_t rest = (h << 14) | (1ull << 13);  // guard bit: rank <= 51");
                g.line("atomicMax(&regs[(uint32_t)(h >> 50)], (uint32_t)__clzll((long long)rest) + 1u);");
                g.close();
            });
            g.cols.clear();
        });
        std::string src = kPrelude;
        src += "// MurmurHash3's 64-bit finalizer (fmix64) over the engine's key hash.\n";
        src += "__device__ __forceinline__ uint64_t hll_mix(uint64_t k) {\n"
               "    k ^= k >> 33;\n    k *= 0xff51afd7ed558ccdull;\n    k ^= k >> 33;\n"
               "    k *= 0xc4ceb9fe1a85ec53ull;\n    k ^= k >> 33;\n    return k;\n}\n";
        src += "extern \"C\" __global__ void __launch_bounds__(256) ml_card_hll(const __grid_constant__ PipeArgs P, "
               "const __grid_constant__ KeyLayout L, uint32_t* cta_regs, unsigned long long* nulls_out, "
               "unsigned long long* minmax) {\n";
        src += "    extern __shared__ uint32_t regs[];\n";
        src += "    for (int i = threadIdx.x; i < 16384; i += blockDim.x) regs[i] = 0;\n    __syncthreads();\n";
        src += "    unsigned long long nulls = 0, lo = ~0ull, hi = 0;\n";
        src += g.pre();
        src += row_loop(P, true, g.body(), g.rows_per_thread, contig);
        src += "    for (int o = 16; o; o >>= 1) {\n"
               "        nulls += __shfl_xor_sync(0xFFFFFFFFu, nulls, o);\n"
               "        const unsigned long long l2 = __shfl_xor_sync(0xFFFFFFFFu, lo, o), h2 = __shfl_xor_sync(0xFFFFFFFFu, hi, o);\n"
               "        lo = l2 < lo ? l2 : lo;\n        hi = h2 > hi ? h2 : hi;\n    }\n";
        src += "    if ((threadIdx.x & 31) == 0) {\n        if (nulls) atomicAdd(nulls_out, nulls);\n"
               "        if (lo != ~0ull) atomicMin(minmax, lo);\n        if (hi) atomicMax(minmax + 1, hi);\n    }\n";
        src += "    __syncthreads();\n    uint32_t* dst = cta_regs + (uint64_t)blockIdx.x * 4096;\n";
        src += "    for (int w = threadIdx.x; w < 4096; w += blockDim.x)\n"
               "        dst[w] = regs[4 * w] | (regs[4 * w + 1] << 8) | (regs[4 * w + 2] << 16) | (regs[4 * w + 3] << 24);\n}\n";
        return src;
    }
}

int jit_resident_blocks(void* fn, unsigned block, size_t smem) {
    static std::mutex mu;
    static std::vector<std::pair<std::pair<void*, size_t>, int>> memo;
    std::lock_guard<std::mutex> g(mu);
    for (auto& e : memo)
        if (e.first.first == fn && e.first.second == smem) return e.second;
    Nvrtc& N = nvrtc();
    if (smem > 48 * 1024 &&
        N.set_attr((CUfunction)fn, CU_FUNC_ATTRIBUTE_MAX_DYNAMIC_SHARED_SIZE_BYTES, (int)smem) != CUDA_SUCCESS)
        raise(ML_ERR_CUDA, "cuFuncSetAttribute failed for a pipeline kernel");
    int n = 0;
    if (N.occupancy(&n, (CUfunction)fn, (int)block, smem) != CUDA_SUCCESS || n < 1) n = 1;
    if (memo.size() >= 256) memo.erase(memo.begin());
    memo.push_back({{fn, smem}, n});
    return n;
}

void jit_launch(void* fn, unsigned grid, unsigned block, size_t smem, cudaStream_t s, void** args) {
    Nvrtc& N = nvrtc();
    if (smem > 48 * 1024 &&
        N.set_attr((CUfunction)fn, CU_FUNC_ATTRIBUTE_MAX_DYNAMIC_SHARED_SIZE_BYTES, (int)smem) != CUDA_SUCCESS)
        raise(ML_ERR_CUDA, "cuFuncSetAttribute failed for a pipeline kernel");
    CUresult r = N.launch((CUfunction)fn, grid, 1, 1, block, 1, 1, (unsigned)smem, (CUstream)s, args, nullptr);
    if (r != CUDA_SUCCESS)
        raise(ML_ERR_CUDA, "launch of a runtime-specialized pipeline kernel failed (CUresult " + std::to_string((int)r) +
                               ")");
}

}  // namespace mlg
