// Kernel argument blocks of the fused pipeline kernels.  Shared by the host runtime,
// the ahead-of-time kernels and the runtime-specialized (NVRTC) kernels, so the
// layout is one definition.
#pragma once

#include "ml_internal.hpp"

namespace mlg {

struct Stage {
    int8_t kind;  // 0 = filter, 1 = probe
    int8_t idx;
};

struct ProbeDev {
    TableView t;
    const uint32_t* next;  // chain links, nullptr when every build key is distinct
    KeyLayout keys;
    // Direct-mapped index for a dense integer key: dense[key - dmin] is the chain head of
    // the build rows with that key (kNone = no row), for key - dmin < drange.  nullptr
    // when the build side uses the hash table `t`.
    const uint32_t* dense;
    uint64_t dmin, drange;
    // With a dense index whose keys are distinct, when nothing after this probe reads the build
    // row (a GROUP BY of the join key that is the pipeline's last stage): the probe yields the
    // key's index position (key - dmin) without reading the index, and membership in the build
    // side is checked once per group when the aggregate is finalized.
    int32_t late, pad;
    // With a dense index whose keys are distinct, when nothing after this probe reads the build
    // row (a semi-join): one bit per index position (bit set = a build row has that key), so the
    // probe reads 1/32 of the index's bytes; a match yields build row 0, which nothing reads.
    const uint32_t* member;
};

// The streaming part of a pipeline (Filter / Projection folded into expressions /
// HashJoinProbe) for one launch.
struct PipeArgs {
    int64_t n;               // rows to visit (selection length when `sel` is set)
    const uint32_t* sel;     // optional input selection vector
    int64_t nsrc;            // rows of the source batch: every selected row id is below it
    const Instr* prog;
    const uint8_t* arena;
    uint32_t* err;
    int32_t nstages, nprobes;
    int32_t head_probe;      // record the chain head of this probe in RowCtx::head (-1: none)
    int32_t has_chains;      // some probed build side has duplicate keys
    Stage stages[kMaxFilters + kMaxProbes];
    Prog filters[kMaxFilters];
    ProbeDev probes[kMaxProbes];
    const uint8_t* luts[kMaxLuts];
    DCol cols[kMaxCols];
};

struct AggArgs {
    KeyLayout keys;
    TableView t;
    uint64_t* gkeys;          // normalized key words by group id (nwords x gid_cap)
    uint32_t* gnull;          // null mask by group id
    uint32_t* ngroups;
    uint32_t gid_cap;
    int32_t nagg;
    int32_t ungrouped;        // no GROUP BY: every row goes to group 0
    int32_t group_probe;      // >= 0: GROUP BY the join key of this probe; group id = matched build row
    int32_t smem_groups;      // group ids below this are pre-aggregated in shared memory
    int32_t priv_groups;      // group ids below this have per-thread accumulators in shared memory
                              // (runtime-specialized kernels only; 0 for the interpreter)
    int32_t stride;           // u64 words per group block
    uint64_t* acc;            // group blocks (gid_cap x stride)
    uint32_t* ovf;            // overflow row contexts
    unsigned long long* ovf_count;
    uint64_t ovf_cap;
    // Direct group slots (runtime-specialized kernels only; 0 = off): when every GROUP BY key
    // takes few values in this launch (a dictionary-coded string: its string ids lie in
    // [dbase, dbase + range - 2]; a BOOL), the key's slot is sum_k term_k * dmul[k] with
    // term_k = 0 for NULL, else value - dbase[k] + 1, and dslots (<= kDirectSlots) bounds it.
    uint32_t dslots;
    uint32_t dmul[kMaxKeys];
    uint32_t dbase[kMaxKeys];
    const uint32_t* str_rank;  // string id -> rank in byte order (A_MIN_STR / A_MAX_STR)
    AggDev aggs[kMaxAggs];
};

// Shared memory of an aggregate launch (256 threads), in this order: the pre-aggregated group
// blocks (smem_groups x stride words), the per-thread accumulators (priv_groups x stride x 256
// words), then, for a keyed GROUP BY with shared-memory groups, kDirectSlots u32 entries of the
// CTA's direct group index (group id + 1 by direct slot, 0 = not yet looked up).
constexpr int kDirectSlots = 1024;
// Per-CTA budget that keeps three 256-thread CTAs resident on an SM (228 KB of shared memory).
constexpr int kAggSmemBudget = 74 << 10;

ML_HD inline bool agg_direct_on(const AggArgs& A) { return A.smem_groups > 0 && !A.ungrouped && A.group_probe < 0; }
ML_HD inline uint64_t agg_direct_bytes(const AggArgs& A) { return agg_direct_on(A) ? 4 * kDirectSlots : 0; }

struct SortDev {
    int32_t nkeys, pad;
    DCol cols[kMaxKeys];
    int32_t asc[kMaxKeys], nulls_first[kMaxKeys];
};

#ifdef __CUDACC__
// Row `i` of a launch: the selection's row id, checked against the batch (a device-resident
// selection is not checked on the host).  An id past the batch's rows is skipped (ok = false)
// and reported through the launch's error word.
__device__ __forceinline__ uint32_t sel_row(const PipeArgs& P, int64_t i, bool& ok) {
    if (!P.sel) return (uint32_t)i;
    const uint32_t r = __ldg(P.sel + i);
    if ((int64_t)r >= P.nsrc) {
        if (P.err) atomicOr(P.err, (uint32_t)DE_BAD_INDEX);
        ok = false;
        return 0;
    }
    return r;
}
#endif

}  // namespace mlg
