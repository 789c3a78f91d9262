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
};

// The streaming part of a pipeline (Filter / Projection folded into expressions /
// HashJoinProbe) for one launch.
struct PipeArgs {
    int64_t n;               // rows to visit (selection length when `sel` is set)
    const uint32_t* sel;     // optional input selection vector
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
    int32_t stride;           // u64 words per group block
    uint64_t* acc;            // group blocks (gid_cap x stride)
    uint32_t* ovf;            // overflow row contexts
    unsigned long long* ovf_count;
    uint64_t ovf_cap;
    AggDev aggs[kMaxAggs];
};

struct SortDev {
    int32_t nkeys, pad;
    DCol cols[kMaxKeys];
    int32_t asc[kMaxKeys], nulls_first[kMaxKeys];
};

}  // namespace mlg
