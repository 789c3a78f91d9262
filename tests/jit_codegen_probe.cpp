// Prints the runtime-specialized kernel sources the library generates for a set of pipeline
// shapes (no GPU needed), separated by lines "//@@ <name>", for tests/test_jit_codegen.py to
// compile with NVRTC.  Built by that test against libminilake_gpu.so.
#include <cstdio>
#include <string>

#include "ml_jit.hpp"

using namespace mlg;

namespace {

Instr ins(uint8_t op, uint8_t sub, uint8_t t, int a, uint64_t bits) {
    Instr in{};
    in.op = op;
    in.sub = sub;
    in.t = t;
    in.a = a;
    in.bits = bits;
    in.lit_valid = 1;
    return in;
}

void emit(const char* name, const std::string& src) { printf("//@@ %s\n%s\n", name, src.c_str()); }

}  // namespace

int main() {
    // slot 0: d (int32), slot 1: v (int64, nullable), slot 2: dictionary-coded string, slot 3: f64
    Pipeline pipe(nullptr);
    pipe.C.code = {ins(I_COL, 0, ML_TYPE_INT32, 0, 0), ins(I_LIT, 0, ML_TYPE_INT32, 0, 2467),
                   ins(I_BIN, ML_BIN_LTEQ, ML_TYPE_INT32, 0, 0),  // 0..2: d <= 2467
                   ins(I_COL, 0, ML_TYPE_INT64, 1, 0),            // 3: v
                   ins(I_COL, 0, ML_TYPE_UTF8, 2, 0),             // 4: dictionary string
                   ins(I_COL, 0, ML_TYPE_FLOAT64, 3, 0)};         // 5: f64
    PipeArgs P{};
    P.n = 1000;
    P.head_probe = -1;
    P.nstages = 1;
    P.stages[0] = {0, 0};
    P.filters[0] = Prog{0, 3, ML_TYPE_BOOL, 0, 0};
    P.cols[0] = DCol{ML_TYPE_INT32, CK_FIXED, 0};
    P.cols[1] = DCol{ML_TYPE_INT64, CK_FIXED, 0};
    P.cols[1].valid = (const uint64_t*)8;
    P.cols[2] = DCol{ML_TYPE_UTF8, CK_DICT, 0};
    P.cols[2].gid = (const uint32_t*)8;
    P.cols[3] = DCol{ML_TYPE_FLOAT64, CK_FIXED, 0};

    for (int contig = 0; contig < 2; contig++) {
        const std::string c = contig ? "_contig" : "_strided";
        emit(("select" + c).c_str(), jit_select_source(pipe, P, contig));

        PipeArgs H = P;  // cardinality scan of v
        H.nstages = 0;
        KeyLayout L{};
        L.nkeys = 1;
        L.nwords = 1;
        L.f[0] = KeyField{0, 0, 64, ML_TYPE_INT64, 0};
        L.prog[0] = Prog{3, 1, ML_TYPE_INT64, 1, 1};
        emit(("hll" + c).c_str(), jit_hll_source(pipe, H, L, contig));

        // GROUP BY the dictionary string: per-thread accumulators and direct group slots
        AggArgs A{};
        A.group_probe = -1;
        A.stride = 4;
        A.smem_groups = 256;
        A.priv_groups = 4;
        A.dslots = 8;
        A.dmul[0] = 1;
        A.keys.nkeys = 1;
        A.keys.nwords = 1;
        A.keys.f[0] = KeyField{0, 0, 32, ML_TYPE_UTF8, 1};
        A.keys.prog[0] = Prog{4, 1, ML_TYPE_UTF8, 0, 1};
        A.nagg = 3;
        A.aggs[0] = AggDev{A_SUM_F64, ML_AGG_SUM, 1, 1, 0};
        A.aggs[0].arg = Prog{5, 1, ML_TYPE_FLOAT64, 0, 1};
        A.aggs[1] = AggDev{A_MAX_I64, ML_AGG_MAX, 1, 2, 0};
        A.aggs[1].arg = Prog{3, 1, ML_TYPE_INT64, 1, 1};
        A.aggs[2] = AggDev{A_AVG, ML_AGG_AVG, 1, 3, 0};  // words 3..: sum and count (stride 5)
        A.aggs[2].arg = Prog{5, 1, ML_TYPE_FLOAT64, 0, 1};
        A.stride = 5;
        emit(("aggregate_groups" + c).c_str(), jit_agg_source(pipe, P, A, contig));

        // filter -> dense join probe (semi-join bitmap) -> GROUP BY d, COUNT(*)
        PipeArgs J = P;
        J.nstages = 2;
        J.nprobes = 1;
        J.stages[1] = {1, 0};
        J.probes[0].dense = (const uint32_t*)8;
        J.probes[0].member = (const uint32_t*)8;
        J.probes[0].keys.nkeys = 1;
        J.probes[0].keys.nwords = 1;
        J.probes[0].keys.f[0] = KeyField{0, 0, 64, ML_TYPE_INT64, 0};
        J.probes[0].keys.prog[0] = Prog{3, 1, ML_TYPE_INT64, 1, 1};
        AggArgs B{};
        B.group_probe = -1;
        B.stride = 1;
        B.smem_groups = 256;
        B.priv_groups = 8;
        B.keys.nkeys = 1;
        B.keys.nwords = 1;
        B.keys.f[0] = KeyField{0, 0, 32, ML_TYPE_INT32, 0};
        B.keys.prog[0] = Prog{0, 1, ML_TYPE_INT32, 0, 1};
        B.nagg = 1;
        B.aggs[0] = AggDev{A_COUNT, ML_AGG_COUNT_STAR, 0, 0, 0};
        emit(("aggregate_semi_join" + c).c_str(), jit_agg_source(pipe, J, B, contig));

        // GROUP BY the dense join key (late membership): no shared-memory groups
        PipeArgs G = J;
        G.probes[0].member = nullptr;
        G.probes[0].late = 1;
        G.head_probe = 0;
        AggArgs D{};
        D.group_probe = 0;
        D.stride = 2;
        D.nagg = 2;
        D.aggs[0] = AggDev{A_COUNT, ML_AGG_COUNT_STAR, 0, 0, 0};
        D.aggs[1] = AggDev{A_SUM_F64, ML_AGG_SUM, 1, 1, 0};
        D.aggs[1].arg = Prog{5, 1, ML_TYPE_FLOAT64, 0, 1};
        emit(("aggregate_dense_groups" + c).c_str(), jit_agg_source(pipe, G, D, contig));
    }
    return 0;
}
