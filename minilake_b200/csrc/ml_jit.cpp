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

struct Cache {
    std::mutex mu;
    std::map<std::pair<int, std::string>, CUfunction> fns;
};
Cache& cache() {
    static Cache c;
    return c;
}

// Compile `src` (defining extern "C" kernel `name`) for this device, or return the cached kernel.
CUfunction get_kernel(Ctx* ctx, const std::string& src, const char* name) {
    Nvrtc& N = nvrtc();
    Cache& C = cache();
    std::lock_guard<std::mutex> g(C.mu);
    auto key = std::make_pair(ctx->device, src);
    auto it = C.fns.find(key);
    if (it != C.fns.end()) return it->second;
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
    C.fns.emplace(key, fn);
    double ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    ctx->add_profile("jit_compile", ms);
    return fn;
}

// ---- source generation --------------------------------------------------------------------------
std::string num(int64_t v) { return std::to_string(v); }

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

    static std::string row(int src) { return src == 0 ? "x.r" : "x.b" + num(src - 1); }

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
                case I_COL:
                    line("const uint64_t " + v + " = " + col_value(in.a) + ";");
                    line("const bool " + k + " = " + col_valid(in.a) + ";");
                    st.push_back({v, k});
                    break;
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

    // Normalized key words of layout L into w<tag>0/1 (and null mask nm<tag> when NULLs
    // group): make_key.  With null_kills a NULL key skips the row combination (`continue`).
    void key(const KeyLayout& L, bool null_kills, const std::string& tag) {
        line("uint64_t w" + tag + "0 = 0, w" + tag + "1 = 0;");
        if (!null_kills) line("uint32_t nm" + tag + " = 0;");
        for (int k = 0; k < L.nkeys; k++) {
            V e = expr(L.prog[k]);
            const KeyField& f = L.f[k];
            uint64_t mask = f.width >= 64 ? ~0ull : ((1ull << f.width) - 1);
            std::string bits = "(uint64_t)";
            std::string word = "w" + tag + num(f.word);
            std::string val = e.v;
            if (f.type == ML_TYPE_FLOAT64) val = "(as_f64(" + e.v + ") == 0.0 ? 0ull : " + e.v + ")";
            char hex[32];
            snprintf(hex, sizeof hex, "0x%llxull", (unsigned long long)mask);
            std::string pack = word + " |= ((" + val + ") & " + hex + ") << " + num(f.shift) + ";";
            if (null_kills) {
                line("if (!(" + e.k + ")) continue;");
                line(pack);
            } else {
                open("if (!(" + e.k + ")) {");
                line("nm" + tag + " |= " + num(1u << k) + "u;");
                close("} else {");
                ind_++;
                line(pack);
                close();
            }
        }
        line("const uint64_t wk" + tag + "[2] = {w" + tag + "0, w" + tag + "1};");
    }

    // Streaming stages from `s` on (run_stages): filters `continue` on failure; probes
    // look up the build table and walk duplicate-key chains as nested loops.
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
        key(pd.keys, true, tag);
        line("const uint32_t hb" + tag + " = table_find(P.probes[" + p + "].t, wk" + tag + ", key_hash(wk" + tag + ", " +
             num(pd.keys.nwords) + "));");
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

   private:
    const std::vector<Instr>& code_;
    const PipeArgs& P_;
    std::ostringstream pre_, o_;
    std::set<std::string> hoisted_;
    int nv_ = 0, ind_ = 2;
};

std::string row_loop_head(const PipeArgs& P) {
    std::string s;
    s += "    const int64_t stride = (int64_t)gridDim.x * blockDim.x;\n";
    s += "    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < P.n; i += stride) {\n";
    s += "        RowCtx x;\n";
    s += P.sel ? "        x.r = __ldg(P.sel + i);\n" : "        x.r = (uint32_t)i;\n";
    s += "        x.b0 = x.b1 = x.b2 = x.b3 = 0;\n        x.head = 0;\n";
    return s;
}

}  // namespace

std::string jit_agg_source(const Pipeline& pipe, const PipeArgs& P, const AggArgs& A) {
    Gen g(pipe.C.code, P);
    const bool smem = A.smem_groups > 0;
    const std::string S = num(A.stride);
    g.stages(0, [&]() {
        g.open("{  // aggregate");
        if (A.group_probe >= 0) {
            g.line("const uint32_t g = x.head;");
        } else if (A.ungrouped) {
            g.line("const uint32_t g = 0;");
        } else {
            g.key(A.keys, false, "g");
            g.line("bool ins;");
            g.line("uint64_t slot;");
            g.line("const uint32_t g = table_upsert(A.t, wkg, nmg, key_hash(wkg, " + num(A.keys.nwords) +
                   ", nmg), P.err, [&]() -> uint32_t { const uint32_t id = atomicAdd(A.ngroups, 1u); "
                   "return id < A.gid_cap ? id : kNone; }, &ins, &slot);");
            g.open("if (g == kNone) {");
            g.line("record_overflow(P, A, x);");
            g.line("continue;");
            g.close();
            g.open("if (ins) {");
            g.line("A.gkeys[g] = wg0;");
            if (A.keys.nwords > 1) g.line("A.gkeys[(uint64_t)A.gid_cap + g] = wg1;");
            g.line("A.gnull[g] = nmg;");
            g.close();
        }
        if (smem)
            g.line("uint64_t* blk = (int)g < A.smem_groups ? smem + (uint64_t)g * " + S + " : A.acc + (uint64_t)g * " + S +
                   ";");
        else
            g.line("uint64_t* blk = A.acc + (uint64_t)g * " + S + ";");
        g.line("atomicAdd((unsigned long long*)blk, 1ull);");
        for (int k = 0; k < A.nagg; k++) {
            const AggDev& a = A.aggs[k];
            if (a.func == ML_AGG_COUNT_STAR) continue;  // the group's row counter (word 0)
            g.open("{  // aggregate " + num(k));
            std::string v = "0ull";
            if (a.has_arg) {
                Gen::V e = g.expr(a.arg);
                g.open("if (" + e.k + ") {");
                v = e.v;
            }
            g.line("acc_apply(" + num(a.kind) + ", blk + " + num(a.off) + ", " + v + ");");
            if (a.count_valid) g.line("atomicAdd((unsigned long long*)A.aggs[" + num(k) + "].vcnt + g, 1ull);");
            if (a.has_arg) g.close();
            g.close();
        }
        g.close();
    });
    std::string src;
    src += "#include \"ml_agg.cuh\"\nusing namespace mlg;\n";
    src += "extern \"C\" __global__ void __launch_bounds__(256) ml_pipeline_aggregate(const __grid_constant__ PipeArgs P, "
           "const __grid_constant__ AggArgs A) {\n";
    src += "    extern __shared__ __align__(16) uint64_t smem[];\n";
    if (smem) src += "    smem_setup(A, smem);\n    __syncthreads();\n";
    src += g.pre();
    src += row_loop_head(P);
    src += g.body();
    src += "    }\n";
    if (smem) src += "    __syncthreads();\n    smem_flush(A, smem);\n";
    src += "}\n";
    return src;
}

void* jit_agg_kernel(Ctx* ctx, const Pipeline& pipe, const PipeArgs& P, const AggArgs& A) {
    if (!jit_enabled(ctx)) return nullptr;
    return (void*)get_kernel(ctx, jit_agg_source(pipe, P, A), "ml_pipeline_aggregate");
}

void* jit_join_insert_kernel(Ctx* ctx, const Pipeline& pipe, const PipeArgs& P, const KeyLayout& L) {
    if (!jit_enabled(ctx)) return nullptr;
    // build_table (join.rs:160-203): distinct keys in the table, duplicates chained in `next`
    Gen g(pipe.C.code, P);
    g.open("{  // insert");
    g.key(L, true, "k");
    g.line("bool ins;");
    g.line("uint64_t slot;");
    g.line("const uint32_t r = x.r;");
    g.line("const uint32_t p = table_upsert(t, wkk, 0u, key_hash(wkk, " + num(L.nwords) +
           "), P.err, [&]() { return r; }, &ins, &slot);");
    g.line("if (p == kNone) continue;");
    g.open("if (!ins) {");
    g.line("const uint32_t old = atomicExch((uint32_t*)slot_at(t, slot) + 1, r);");
    g.line("next[r] = old;");
    g.line("if (*dup_flag == 0) atomicExch(dup_flag, 1u);");
    g.close();
    g.close();
    std::string src;
    src += "#include \"ml_agg.cuh\"\nusing namespace mlg;\n";
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

void jit_launch(void* fn, unsigned grid, unsigned block, size_t smem, cudaStream_t s, void** args) {
    Nvrtc& N = nvrtc();
    if (smem > 48 * 1024 &&
        N.set_attr((CUfunction)fn, CU_FUNC_ATTRIBUTE_MAX_DYNAMIC_SHARED_SIZE_BYTES, (int)smem) != CUDA_SUCCESS)
        raise(ML_ERR_CUDA, "cuFuncSetAttribute failed for a pipeline kernel");
    CUresult r = N.launch((CUfunction)fn, grid, 1, 1, block, 1, 1, (unsigned)smem, (CUstream)s, args, nullptr);
    if (r != CUDA_SUCCESS) raise(ML_ERR_CUDA, "launch of a runtime-specialized pipeline kernel failed (CUresult " +
                                                  std::to_string((int)r) + ")");
}

}  // namespace mlg
