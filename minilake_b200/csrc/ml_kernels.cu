// sm_100a kernels of the MiniLake execution core.
//
// All of MiniLake's hot-path operators are HBM-bandwidth or L2-latency bound
// integer/byte/FP64 work: nothing here is a dense contraction, so there is no
// tensor-core code.  The design rules are the ones that matter for HBM-bound
// kernels on B200: one pass over each column with coalesced loads, grids sized
// as a multiple of the 148 SMs, state that fits in L2 (126 MB) kept there, and
// shared-memory privatization wherever many rows hit few addresses.
#include <algorithm>

#include "ml_agg.cuh"
#include "ml_kernels.cuh"

namespace mlg {

int num_sms() {
    static const int sms = [] {
        int dev = 0, n = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
        return n > 0 ? n : 148;
    }();
    return sms;
}

namespace {
constexpr int kThreads = 256;
int grid_for(int64_t n, int per_sm = 8) {
    int64_t want = (n + kThreads - 1) / kThreads;
    int64_t cap = (int64_t)num_sms() * per_sm;
    if (want < 1) want = 1;
    return (int)(want < cap ? want : cap);
}

__device__ __forceinline__ EvalEnv env_of(const PipeArgs& P) {
    return EvalEnv{P.cols, P.prog, P.arena, P.luts};
}

// Chain cursors of up to four probes, in named registers (no local-memory array).
struct Cursors {
    uint32_t c0 = kNone, c1 = kNone, c2 = kNone, c3 = kNone;
    __device__ __forceinline__ uint32_t get(int p) const {
        switch (p) {
            case 0: return c0;
            case 1: return c1;
            case 2: return c2;
            default: return c3;
        }
    }
    __device__ __forceinline__ void set(int p, uint32_t v) {
        switch (p) {
            case 0: c0 = v; break;
            case 1: c1 = v; break;
            case 2: c2 = v; break;
            default: c3 = v; break;
        }
    }
};

// Build row matching the normalized key `w` through probe `pd` (dense index or hash table).
__device__ __forceinline__ uint32_t probe_find(const ProbeDev& pd, const uint64_t* w) {
    if (pd.dense && pd.late) return dense_slot(pd.dmin, pd.drange, w[0]);
    if (pd.dense && pd.member) return dense_member(pd.member, pd.dmin, pd.drange, w[0]);
    if (pd.dense) return dense_find(pd.dense, pd.dmin, pd.drange, w[0]);
    return table_find(pd.t, w, key_hash(w, pd.t.nwords));
}

// Run the streaming stages for one source row; call sink(ctx) for every surviving
// (row, build matches...) combination.  Duplicate build keys are walked through their
// chains with backtracking, like HashJoinProbe's chain walk (join.rs:297-309).
template <class Sink>
__device__ __forceinline__ void run_stages(const PipeArgs& P, const EvalEnv& env, RowCtx& x, Sink&& sink) {
    if (!P.has_chains) {  // every build key is distinct: at most one match per probe, no backtracking
        for (int s = 0; s < P.nstages; s++) {
            const Stage st = P.stages[s];
            if (st.kind == 0) {
                uint64_t v;
                bool ok;
                eval_prog(env, P.filters[st.idx], x, v, ok);
                if (!(ok && (v & 1))) return;
            } else {
                const ProbeDev& pd = P.probes[st.idx];
                uint64_t w[2];
                uint32_t nm;
                if (!make_key(env, pd.keys, x, w, &nm, true)) return;
                uint32_t b = probe_find(pd, w);
                if (b == kNone) return;
                x.set_build(st.idx, b);
                if (st.idx == P.head_probe) x.head = b;
            }
        }
        sink(x);
        return;
    }
    Cursors cur;
    int s = 0;
    for (;;) {
        bool advance = false;
        if (s == P.nstages) {
            sink(x);
        } else {
            const Stage st = P.stages[s];
            if (st.kind == 0) {
                uint64_t v;
                bool ok;
                eval_prog(env, P.filters[st.idx], x, v, ok);
                advance = ok && (v & 1);
            } else {
                const ProbeDev& pd = P.probes[st.idx];
                uint64_t w[2];
                uint32_t nm;
                if (make_key(env, pd.keys, x, w, &nm, true)) {
                    uint32_t b = probe_find(pd, w);
                    if (b != kNone) {
                        x.set_build(st.idx, b);
                        if (st.idx == P.head_probe) x.head = b;
                        cur.set(st.idx, pd.next ? __ldg(pd.next + b) : kNone);
                        advance = true;
                    }
                }
            }
        }
        if (advance) {
            s++;
            continue;
        }
        int q = s - 1;
        for (; q >= 0; q--) {
            const Stage st = P.stages[q];
            if (st.kind != 1) continue;
            uint32_t c = cur.get(st.idx);
            if (c != kNone) {
                x.set_build(st.idx, c);
                cur.set(st.idx, __ldg(P.probes[st.idx].next + c));
                break;
            }
        }
        if (q < 0) return;
        s = q + 1;
    }
}

__device__ __forceinline__ void agg_fold(const PipeArgs& P, const AggArgs& A, const EvalEnv& env, const RowCtx& x,
                                         uint64_t* blk, uint32_t g) {
    atomicAdd((unsigned long long*)blk, 1ull);
    for (int k = 0; k < A.nagg; k++) {
        const AggDev& a = A.aggs[k];
        if (a.func == ML_AGG_COUNT_STAR) continue;  // COUNT(*) is the row counter (word 0)
        uint64_t v = 0;
        bool ok = true;
        if (a.has_arg) eval_prog(env, a.arg, x, v, ok);
        if (!ok) continue;
        if (a.kind == A_MIN_STR || a.kind == A_MAX_STR) v = str_pack(A.str_rank, (uint32_t)v);
        acc_apply(a.kind, blk + a.off, v);
        if (a.count_valid) atomicAdd((unsigned long long*)a.vcnt + g, 1ull);
    }
}

__device__ __forceinline__ void agg_update(const PipeArgs& P, const AggArgs& A, const EvalEnv& env, const RowCtx& x,
                                           uint64_t* smem) {
    uint32_t g;
    if (A.group_probe >= 0) {
        g = x.head;  // every row of a key's chain aggregates into the chain head's group
    } else if (A.ungrouped) {
        g = 0;
    } else {
        uint64_t w[2];
        uint32_t nm;
        make_key(env, A.keys, x, w, &nm, false);
        uint64_t h = key_hash(w, A.keys.nwords, nm);
        bool inserted;
        uint64_t slot;
        g = table_upsert(
            A.t, w, nm, h, P.err,
            [&]() -> uint32_t {
                uint32_t id = atomicAdd(A.ngroups, 1u);
                return id < A.gid_cap ? id : kNone;
            },
            &inserted, &slot, A.ngroups, A.gid_cap);
        if (g == kNone) {
            record_overflow(P, A, x);
            return;
        }
        if (inserted) {
            A.gkeys[g] = w[0];
            if (A.keys.nwords > 1) A.gkeys[(uint64_t)A.gid_cap + g] = w[1];
            A.gnull[g] = nm;
        }
    }
    if ((int)g < A.smem_groups) agg_fold(P, A, env, x, smem + (uint64_t)g * A.stride, g);
    else agg_fold(P, A, env, x, A.acc + (uint64_t)g * A.stride, g);
}

__global__ void __launch_bounds__(kThreads) k_agg(const __grid_constant__ PipeArgs P, const __grid_constant__ AggArgs A) {
    extern __shared__ __align__(16) uint64_t smem[];
    smem_setup(A, smem);
    __syncthreads();
    const EvalEnv env = env_of(P);
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < P.n; i += stride) {
        RowCtx x;
        bool ok = true;
        x.r = sel_row(P, i, ok);
        if (!ok) continue;
        x.b0 = x.b1 = x.b2 = x.b3 = 0;
        x.head = 0;
        run_stages(P, env, x, [&](const RowCtx& c) { agg_update(P, A, env, c, smem); });
    }
    __syncthreads();
    smem_flush(A, smem);
}

__global__ void __launch_bounds__(kThreads) k_agg_resume(const __grid_constant__ PipeArgs P, const __grid_constant__ AggArgs A,
                                                         const uint32_t* ctx, uint64_t count, int w) {
    extern __shared__ __align__(16) uint64_t smem[];
    smem_setup(A, smem);
    __syncthreads();
    const EvalEnv env = env_of(P);
    uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += stride) {
        const uint32_t* c = ctx + i * (uint64_t)w;
        RowCtx x;
        x.r = c[0];
        x.b0 = w > 1 ? c[1] : 0;
        x.b1 = w > 2 ? c[2] : 0;
        x.b2 = w > 3 ? c[3] : 0;
        x.b3 = w > 4 ? c[4] : 0;
        x.head = 0;
        agg_update(P, A, env, x, smem);
    }
    __syncthreads();
    smem_flush(A, smem);
}

// ---- exchange partitioning: rows grouped by key hash % nparts, input order kept ----------------
// Per 1024-row block: counts[p * blocks + b] = rows of block b in partition p.
__global__ void __launch_bounds__(kXPartRows) k_xpart_count(const uint64_t* h, int64_t n, int nparts, uint32_t* counts) {
    __shared__ uint32_t hist[kMaxExchangeParts];
    for (int i = threadIdx.x; i < nparts; i += blockDim.x) hist[i] = 0;
    __syncthreads();
    const int64_t r = (int64_t)blockIdx.x * kXPartRows + threadIdx.x;
    if (r < n) atomicAdd(&hist[h[r] % (uint64_t)nparts], 1u);
    __syncthreads();
    for (int i = threadIdx.x; i < nparts; i += blockDim.x) counts[(int64_t)i * gridDim.x + blockIdx.x] = hist[i];
}
// perm[pos] = row: pos = the (partition, block) offset + the row's rank among the block's rows of
// its partition (warps in order, lanes in order within a warp: a stable counting sort).
__global__ void __launch_bounds__(kXPartRows) k_xpart_scatter(const uint64_t* h, int64_t n, int nparts,
                                                             const uint64_t* offs, uint32_t* perm) {
    __shared__ uint32_t wcnt[kXPartRows / 32][kMaxExchangeParts];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int i = threadIdx.x; i < (kXPartRows / 32) * kMaxExchangeParts; i += blockDim.x)
        wcnt[i / kMaxExchangeParts][i % kMaxExchangeParts] = 0;
    __syncthreads();
    const int64_t r = (int64_t)blockIdx.x * kXPartRows + threadIdx.x;
    const bool in = r < n;
    const uint32_t p = in ? (uint32_t)(h[r] % (uint64_t)nparts) : 0xFFFFFFFFu;
    const unsigned same = __match_any_sync(0xFFFFFFFFu, p);
    const uint32_t rank = __popc(same & ((1u << lane) - 1u));
    if (in && rank == 0) wcnt[w][p] = __popc(same);  // the group's lowest lane
    __syncthreads();
    for (int q = threadIdx.x; q < nparts; q += blockDim.x) {  // exclusive prefix over the warps
        uint32_t run = 0;
        for (int ww = 0; ww < kXPartRows / 32; ww++) {
            const uint32_t c = wcnt[ww][q];
            wcnt[ww][q] = run;
            run += c;
        }
    }
    __syncthreads();
    if (in) perm[offs[(int64_t)p * gridDim.x + blockIdx.x] + wcnt[w][p] + rank] = (uint32_t)r;
}

// ---- out-of-HBM aggregation (aggregate/hash.rs:189-281, 369-425) ------------------------------
// Spill partition of each group: bits 32..35 of its key hash, which the table's slot choice (the
// low bits) does not use, so every partition's groups still hash well into a table of their own.
__global__ void k_spill_part(const uint64_t* gkeys, const uint32_t* gnull, uint32_t gid_cap, uint32_t ng, int nwords,
                             uint64_t* part) {
    const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= ng) return;
    const uint64_t w[2] = {gkeys[g], nwords > 1 ? gkeys[(uint64_t)gid_cap + g] : 0ull};
    part[g] = (key_hash(w, nwords, gnull[g]) >> 32) & (kSpillParts - 1);
}
// Merge spilled partial states (n groups: key words as nwords planes of n, null masks, group
// blocks of A.stride words, valid-input counts as planes of n for the aggregates that keep them)
// into the table: a group's block adds up (counts, sums, AVG's sum and count) or folds (MIN/MAX),
// as HashAggState::merge_partial merges partial batches (aggregate/hash.rs:125-139).
__global__ void k_agg_merge_spill(const __grid_constant__ AggArgs A, const uint64_t* keys, const uint32_t* nulls,
                                  const uint64_t* acc, const uint64_t* vcnt, uint32_t n, uint32_t* err) {
    const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n) return;
    const uint64_t w[2] = {keys[r], A.keys.nwords > 1 ? keys[(uint64_t)n + r] : 0ull};
    const uint32_t nm = nulls[r];
    bool ins;
    uint64_t slot;
    const uint32_t g = table_upsert(A.t, w, nm, key_hash(w, A.keys.nwords, nm), err, [&]() -> uint32_t {
        const uint32_t id = atomicAdd(A.ngroups, 1u);
        return id < A.gid_cap ? id : kNone;
    }, &ins, &slot, A.ngroups, A.gid_cap);
    if (g == kNone) {  // the table is sized for every spilled row of the partition: not reached
        atomicOr(err, (uint32_t)DE_OVERFLOW_LOST);
        return;
    }
    if (ins) {
        A.gkeys[g] = w[0];
        if (A.keys.nwords > 1) A.gkeys[(uint64_t)A.gid_cap + g] = w[1];
        A.gnull[g] = nm;
    }
    uint64_t* blk = A.acc + (uint64_t)g * A.stride;
    const uint64_t* src = acc + (uint64_t)r * A.stride;
    if (src[0]) atomicAdd((unsigned long long*)blk, (unsigned long long)src[0]);
    int v = 0;
    for (int k = 0; k < A.nagg; k++) {
        const AggDev& a = A.aggs[k];
        if (a.func == ML_AGG_COUNT_STAR) continue;
        acc_merge(a.kind, blk + a.off, src + a.off);
        if (a.vcnt) {
            const uint64_t c = vcnt[(uint64_t)v * n + r];
            if (c) atomicAdd((unsigned long long*)a.vcnt + g, (unsigned long long)c);
            v++;
        }
    }
}

__global__ void k_agg_rehash(TableView t, const uint64_t* gkeys, const uint32_t* gnull, uint32_t gid_cap, uint32_t ngroups,
                             int nwords, uint32_t* err) {
    uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= ngroups) return;
    uint64_t w[2] = {gkeys[g], nwords > 1 ? gkeys[(uint64_t)gid_cap + g] : 0ull};
    uint32_t nm = gnull[g];
    bool inserted;
    uint64_t slot;
    table_upsert(t, w, nm, key_hash(w, nwords, nm), err, [&]() { return g; }, &inserted, &slot);
}

__global__ void k_acc_init(AggArgs A, uint32_t from, uint32_t to) {
    uint32_t g = from + blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= to) return;
    uint64_t* b = A.acc + (uint64_t)g * A.stride;
    for (int w = 0; w < A.stride; w++) b[w] = 0;
    for (int k = 0; k < A.nagg; k++) {
        const AggDev& a = A.aggs[k];
        if (a.func != ML_AGG_COUNT_STAR) b[a.off] = agg_identity(a.kind);
        if (a.vcnt) a.vcnt[g] = 0;
    }
}

// Final values (accumulator.rs:500-526): AVG = sum / count, empty -> NULL.
__global__ void k_agg_final(const __grid_constant__ FinalArgs F) {
    uint32_t o = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t ng = F.ngroups;
    if (F.ng64) ng = (uint32_t)min((uint64_t)ng, __ldg(F.ng64));
    if (F.ng32) ng = min(ng, __ldg(F.ng32));
    bool in = o < ng;
    uint32_t g = in ? (F.gids ? F.gids[o] : o) : 0;
    uint32_t lane = threadIdx.x & 31;
    for (int k = 0; k < F.nkeys; k++) {
        const KeyField f = F.f[k];
        bool valid = true;
        if (in) {
            uint64_t w = F.gkeys[(uint64_t)f.word * F.gid_cap + g];
            valid = !((F.gnull[g] >> k) & 1u);
            uint64_t m = f.width >= 64 ? ~0ull : ((1ull << f.width) - 1);
            uint64_t v = (w >> f.shift) & m;
            if (f.strid) ((uint32_t*)F.key_out[k])[o] = (uint32_t)v;
            else if (f.type == ML_TYPE_BOOL) ((uint8_t*)F.key_out[k])[o] = (uint8_t)v;
            else if (f.type == ML_TYPE_INT32 || f.type == ML_TYPE_DATE) ((int32_t*)F.key_out[k])[o] = (int32_t)(uint32_t)v;
            else ((uint64_t*)F.key_out[k])[o] = v;
        }
        uint32_t bits = __ballot_sync(0xFFFFFFFFu, in && valid);
        if (lane == 0 && (o >> 5) < (ng + 31) / 32) F.key_valid[k][o >> 5] = bits;
    }
    const uint64_t* blk = F.acc + (uint64_t)g * F.stride;
    for (int k = 0; k < F.nagg; k++) {
        const AggDev& a = F.aggs[k];
        bool valid = false;
        if (in) {
            uint64_t rows = blk[0];
            uint64_t vc = a.vcnt ? a.vcnt[g] : rows;
            if (a.func == ML_AGG_COUNT_STAR) {
                ((int64_t*)F.agg_out[k])[o] = (int64_t)rows;
                valid = true;
            } else if (a.func == ML_AGG_COUNT) {
                ((int64_t*)F.agg_out[k])[o] = (int64_t)blk[a.off];
                valid = true;
            } else {
                uint64_t v = blk[a.off];
                valid = vc > 0;
                switch (a.kind) {
                    case A_AVG: {
                        uint64_t c = blk[a.off + 1];
                        valid = c > 0;
                        double r = c == 0 ? 0.0 : __ddiv_rn(as_f64(v), __ll2double_rn((long long)c));
                        ((double*)F.agg_out[k])[o] = r;
                        break;
                    }
                    case A_MIN_F64:
                    case A_MAX_F64: ((double*)F.agg_out[k])[o] = valid ? f64_unorder(v) : 0.0; break;
                    case A_MIN_STR:
                    case A_MAX_STR: ((uint32_t*)F.agg_out[k])[o] = valid ? (uint32_t)v : 0u; break;  // the id
                    case A_MIN_I64:
                    case A_MAX_I64:
                        if (F.out_type[k] == ML_TYPE_INT32 || F.out_type[k] == ML_TYPE_DATE)
                            ((int32_t*)F.agg_out[k])[o] = valid ? (int32_t)(int64_t)v : 0;
                        else
                            ((int64_t*)F.agg_out[k])[o] = valid ? (int64_t)v : 0;
                        break;
                    default: ((uint64_t*)F.agg_out[k])[o] = v; break;
                }
            }
        }
        uint32_t bits = __ballot_sync(0xFFFFFFFFu, in && valid);
        if (lane == 0 && (o >> 5) < (ng + 31) / 32) F.agg_valid[k][o >> 5] = bits;
    }
}

// ---- filter: pass bits + per-block counts, then ordered compaction ---------------------------
constexpr int kSelRowsPerBlock = kThreads * 8;

__global__ void __launch_bounds__(kThreads) k_select_flags(const __grid_constant__ PipeArgs P, uint32_t* bits,
                                                           uint32_t* block_counts) {
    const EvalEnv env = env_of(P);
    int64_t base = (int64_t)blockIdx.x * kSelRowsPerBlock;
    uint32_t cnt = 0;
    for (int it = 0; it < 8; it++) {
        int64_t i = base + it * kThreads + threadIdx.x;
        bool pass = false;
        bool ok = i < P.n;
        RowCtx x;
        if (ok) x.r = sel_row(P, i, ok);
        if (ok) {
            x.b0 = x.b1 = x.b2 = x.b3 = 0;
            x.head = 0;
            run_stages(P, env, x, [&](const RowCtx&) { pass = true; });
        }
        uint32_t b = __ballot_sync(0xFFFFFFFFu, pass);
        if ((threadIdx.x & 31) == 0 && base + it * kThreads + (threadIdx.x & ~31) < P.n)
            bits[(base + it * kThreads + threadIdx.x) >> 5] = b;
        cnt += pass;
    }
    // block reduce
    __shared__ uint32_t red[kThreads / 32];
    for (int o = 16; o; o >>= 1) cnt += __shfl_xor_sync(0xFFFFFFFFu, cnt, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = cnt;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t t = 0;
        for (int w = 0; w < kThreads / 32; w++) t += red[w];
        block_counts[blockIdx.x] = t;
    }
}

// Bits of a pass mask (u32 words) -> the ordered positions (sel[i] when a selection is given).
__global__ void __launch_bounds__(kThreads) k_index_write(int64_t n, const uint32_t* sel, const uint32_t* bits,
                                                          const uint64_t* block_offsets, uint32_t* out) {
    __shared__ uint32_t warp_tot[kThreads / 32 * 8];
    int64_t base = (int64_t)blockIdx.x * kSelRowsPerBlock;
    int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    uint32_t w[8];
    for (int it = 0; it < 8; it++) {
        int64_t wi = (base >> 5) + it * (kThreads / 32) + warp;
        w[it] = wi * 32 < n ? bits[wi] : 0u;
        if (lane == 0) warp_tot[it * (kThreads / 32) + warp] = __popc(w[it]);
    }
    __syncthreads();
    static_assert(8 * (kThreads / 32) == 64, "two words per lane in the scan below");
    if (warp == 0) {  // exclusive scan over the 64 words in row order, two per lane
        const uint32_t a = warp_tot[2 * lane], b = warp_tot[2 * lane + 1];
        uint32_t x = a + b;
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, x, o);
            if (lane >= o) x += y;
        }
        warp_tot[2 * lane] = x - a - b;
        warp_tot[2 * lane + 1] = x - b;
    }
    __syncthreads();
    uint64_t off = block_offsets[blockIdx.x];
    for (int it = 0; it < 8; it++) {
        int64_t wi = (base >> 5) + it * (kThreads / 32) + warp;
        uint32_t m = w[it];
        if ((m >> lane) & 1u) {
            uint32_t pos = warp_tot[it * (kThreads / 32) + warp] + __popc(m & ((1u << lane) - 1u));
            int64_t i = wi * 32 + lane;
            out[off + pos] = sel ? __ldg(sel + i) : (uint32_t)i;
        }
    }
}

__global__ void __launch_bounds__(kThreads) k_group_flags(const uint64_t* acc, int stride, int64_t n,
                                                          const uint32_t* member, uint32_t* bits,
                                                          uint32_t* block_counts) {
    int64_t base = (int64_t)blockIdx.x * kSelRowsPerBlock;
    uint32_t cnt = 0;
    for (int it = 0; it < 8; it++) {
        int64_t i = base + it * kThreads + threadIdx.x;
        bool pass = i < n && acc[i * stride] != 0 && (member == nullptr || member[i] != kNone);
        uint32_t b = __ballot_sync(0xFFFFFFFFu, pass);
        if ((threadIdx.x & 31) == 0 && base + it * kThreads + (threadIdx.x & ~31) < n) bits[(base + it * kThreads + threadIdx.x) >> 5] = b;
        cnt += pass;
    }
    __shared__ uint32_t red[kThreads / 32];
    for (int o = 16; o; o >>= 1) cnt += __shfl_xor_sync(0xFFFFFFFFu, cnt, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = cnt;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t t = 0;
        for (int w = 0; w < kThreads / 32; w++) t += red[w];
        block_counts[blockIdx.x] = t;
    }
}

// ---- scan (exclusive, u32 -> u64) ------------------------------------------------------------
constexpr int kScanItems = 4;
constexpr int kScanBlock = 1024 * kScanItems;

__device__ uint64_t block_exclusive_scan(uint64_t v, uint64_t* tmp, uint64_t* total) {
    int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint64_t x = v;
    for (int o = 1; o < 32; o <<= 1) {
        uint64_t y = __shfl_up_sync(0xFFFFFFFFu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) tmp[warp] = x;
    __syncthreads();
    if (warp == 0) {
        int nw = blockDim.x >> 5;
        uint64_t t = lane < nw ? tmp[lane] : 0;
        for (int o = 1; o < 32; o <<= 1) {
            uint64_t y = __shfl_up_sync(0xFFFFFFFFu, t, o);
            if (lane >= o) t += y;
        }
        if (lane < nw) tmp[lane] = t;
    }
    __syncthreads();
    uint64_t before = warp ? tmp[warp - 1] : 0;
    if (total) *total = tmp[(blockDim.x >> 5) - 1];
    __syncthreads();
    return before + x - v;
}

__global__ void k_scan_reduce(const uint32_t* in, int64_t n, uint64_t* sums) {
    __shared__ uint64_t tmp[32];
    int64_t base = (int64_t)blockIdx.x * kScanBlock;
    uint64_t s = 0;
    for (int k = 0; k < kScanItems; k++) {
        int64_t i = base + (int64_t)threadIdx.x * kScanItems + k;
        if (i < n) s += in[i];
    }
    uint64_t total;
    block_exclusive_scan(s, tmp, &total);
    if (threadIdx.x == 0) sums[blockIdx.x] = total;
}
__global__ void k_scan_sums(uint64_t* sums, int64_t nb) {  // single block, in place, exclusive
    __shared__ uint64_t tmp[32];
    __shared__ uint64_t carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (int64_t base = 0; base < nb; base += blockDim.x) {
        int64_t i = base + threadIdx.x;
        uint64_t v = i < nb ? sums[i] : 0;
        uint64_t total;
        uint64_t ex = block_exclusive_scan(v, tmp, &total);
        if (i < nb) sums[i] = carry + ex;
        __syncthreads();
        if (threadIdx.x == 0) carry += total;
        __syncthreads();
    }
    if (threadIdx.x == 0) sums[nb] = carry;
}
__global__ void k_scan_apply(const uint32_t* in, int64_t n, const uint64_t* sums, uint64_t* out) {
    __shared__ uint64_t tmp[32];
    int64_t base = (int64_t)blockIdx.x * kScanBlock;
    uint64_t vals[kScanItems];
    uint64_t s = 0;
    for (int k = 0; k < kScanItems; k++) {
        int64_t i = base + (int64_t)threadIdx.x * kScanItems + k;
        vals[k] = i < n ? in[i] : 0;
        s += vals[k];
    }
    uint64_t ex = block_exclusive_scan(s, tmp, nullptr) + sums[blockIdx.x];
    for (int k = 0; k < kScanItems; k++) {
        int64_t i = base + (int64_t)threadIdx.x * kScanItems + k;
        if (i < n) out[i] = ex;
        ex += vals[k];
    }
    if (blockIdx.x == gridDim.x - 1 && threadIdx.x == blockDim.x - 1) out[n] = ex;
}

// ---- projection / hashing ---------------------------------------------------------------------
__global__ void __launch_bounds__(kThreads) k_project(const __grid_constant__ PipeArgs P, Prog prog, int out_type,
                                                      void* out, uint32_t* valid) {
    const EvalEnv env = env_of(P);
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    // the loop trip count is uniform per warp (stride is a multiple of 32)
    for (int64_t i0 = (int64_t)blockIdx.x * blockDim.x; i0 < P.n; i0 += stride) {
        int64_t i = i0 + threadIdx.x;
        bool in = i < P.n, ok = false;
        RowCtx x;
        if (in) x.r = sel_row(P, i, in);
        if (in) {
            x.b0 = x.b1 = x.b2 = x.b3 = 0;
            x.head = 0;
            uint64_t v;
            eval_prog(env, prog, x, v, ok);
            switch (out_type) {
                case ML_TYPE_BOOL: ((uint8_t*)out)[i] = (uint8_t)(v & 1); break;
                case ML_TYPE_INT32:
                case ML_TYPE_DATE: ((int32_t*)out)[i] = (int32_t)(uint32_t)v; break;
                case ML_TYPE_UTF8: ((uint32_t*)out)[i] = (uint32_t)v; break;
                default: ((uint64_t*)out)[i] = v; break;
            }
        }
        uint32_t b = __ballot_sync(0xFFFFFFFFu, in && ok);
        if ((threadIdx.x & 31) == 0 && i < P.n) valid[i >> 5] = b;
    }
}

// kernels/hash.rs:16-79: h = SEED; for col: h = combine(h, valid ? hash(col[r]) : NULL_HASH)
__global__ void k_hash_columns(const __grid_constant__ PipeArgs P, int ncols, const uint64_t* const* dict_hash,
                               uint64_t* out) {
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < P.n; i += stride) {
        bool ok = true;
        const uint32_t r = sel_row(P, i, ok);
        if (!ok) {
            out[i] = 0;
            continue;
        }
        uint64_t h = kSeed;
        for (int c = 0; c < ncols; c++) {
            const DCol& col = P.cols[c];
            uint64_t x = kNullHash;
            if (valid_bit(col.valid, r)) {
                if (col.kind == CK_DICT) {
                    x = dict_hash[c][dict_code(col, r)];
                } else if (col.kind == CK_UTF8) {
                    Str s = col_str(col, r);
                    x = hash_bytes(s.p, s.n);
                } else {
                    uint64_t v = load_value(col, r);
                    if (col.dt == ML_TYPE_FLOAT64 && as_f64(v) == 0.0) v = 0;
                    x = hash_u64(v);
                }
            }
            h = hash_combine(h, x);
        }
        out[i] = h;
    }
}

// ---- join build / probe --------------------------------------------------------------------------
// build_table (join.rs:160-203): one table entry per distinct key; rows with the same
// key are chained through `next`.  NULL keys are not inserted.
__global__ void k_join_insert(const __grid_constant__ PipeArgs P, const __grid_constant__ KeyLayout L, TableView t,
                              uint32_t* next, uint32_t* dup_flag, int64_t n) {
    const EvalEnv env = env_of(P);
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        RowCtx x;
        x.r = (uint32_t)i;
        x.b0 = x.b1 = x.b2 = x.b3 = 0;
        x.head = 0;
        uint64_t w[2];
        uint32_t nm;
        if (!make_key(env, L, x, w, &nm, true)) continue;
        bool inserted;
        uint64_t slot;
        uint32_t r = (uint32_t)i;
        uint32_t p = table_upsert(t, w, 0u, key_hash(w, t.nwords), P.err, [&]() { return r; }, &inserted, &slot);
        if (p == kNone) continue;  // error already flagged (timeout) or table full (never: presized)
        if (!inserted) {
            uint32_t old = atomicExch((uint32_t*)slot_at(t, slot) + 1, r);
            next[r] = old;
            if (*dup_flag == 0) atomicExch(dup_flag, 1u);
        }
    }
}

__global__ void k_probe_count(const __grid_constant__ PipeArgs P, uint32_t* counts) {
    const EvalEnv env = env_of(P);
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < P.n; i += stride) {
        RowCtx x;
        bool ok = true;
        x.r = sel_row(P, i, ok);
        x.b0 = x.b1 = x.b2 = x.b3 = 0;
        x.head = 0;
        uint32_t c = 0;
        if (ok) run_stages(P, env, x, [&](const RowCtx&) { c++; });
        counts[i] = c;
    }
}
__global__ void k_probe_write(const __grid_constant__ PipeArgs P, const uint64_t* offsets, uint32_t* pi, uint32_t* bi) {
    const EvalEnv env = env_of(P);
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < P.n; i += stride) {
        RowCtx x;
        bool ok = true;
        x.r = sel_row(P, i, ok);
        if (!ok) continue;  // counted no pairs
        x.b0 = x.b1 = x.b2 = x.b3 = 0;
        x.head = 0;
        uint64_t o = offsets[i];
        run_stages(P, env, x, [&](const RowCtx& c) {
            pi[o] = c.r;
            bi[o] = c.b0;
            o++;
        });
    }
}

// Range of a one-column integer join key over the valid build rows, as normalized key
// words (int32/date keys zero-extended from 32 bits, int64 keys as is).
__device__ __forceinline__ uint64_t norm_int_key(const void* data, int dt, uint32_t r) {
    if (dt == ML_TYPE_INT64) return (uint64_t)__ldg((const unsigned long long*)data + r);
    return (uint64_t)(uint32_t)__ldg((const int32_t*)data + r);
}
__global__ void k_key_range(const void* data, int dt, const uint64_t* valid, int64_t n, unsigned long long* mm) {
    unsigned long long lo = ~0ull, hi = 0;
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        if (!valid_bit(valid, (uint32_t)i)) continue;
        unsigned long long k = norm_int_key(data, dt, (uint32_t)i);
        lo = k < lo ? k : lo;
        hi = k > hi ? k : hi;
    }
    for (int o = 16; o; o >>= 1) {
        unsigned long long l2 = __shfl_xor_sync(0xFFFFFFFFu, lo, o), h2 = __shfl_xor_sync(0xFFFFFFFFu, hi, o);
        lo = l2 < lo ? l2 : lo;
        hi = h2 > hi ? h2 : hi;
    }
    if ((threadIdx.x & 31) == 0) {
        atomicMin(mm, lo);
        atomicMax(mm + 1, hi);
    }
}
// build_table (join.rs:160-203) over a dense key: the index entry holds the chain head,
// later rows with the same key push the previous head into `next`.
// Membership bitmap of a dense index: bit i of the words = (dense[i] != kNone); one warp per word.
__global__ void k_dense_bits(const uint32_t* dense, uint64_t n, uint32_t* bits) {
    const uint64_t words = (n + 31) / 32;
    const int lane = threadIdx.x & 31;
    const uint64_t warps = (uint64_t)gridDim.x * (blockDim.x >> 5);
    for (uint64_t w = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; w < words; w += warps) {
        const uint64_t i = w * 32 + lane;
        const unsigned b = __ballot_sync(0xFFFFFFFFu, i < n && dense[i] != kNone);
        if (lane == 0) bits[w] = b;
    }
}

__global__ void k_dense_insert(const void* data, int dt, const uint64_t* valid, int64_t n, uint64_t dmin, uint64_t drange,
                               uint32_t* dense, uint32_t* next, uint32_t* dup_flag, uint32_t* range_err) {
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        uint32_t r = (uint32_t)i;
        if (!valid_bit(valid, r)) continue;  // NULL keys never match
        const uint64_t pos = norm_int_key(data, dt, r) - dmin;
        if (pos >= drange) {  // outside the index (a replayed plan's data changed): skipped, reported
            if (range_err) atomicOr(range_err, 1u);
            continue;
        }
        uint32_t old = atomicExch(dense + pos, r);
        if (old != kNone) {
            next[r] = old;
            if (*dup_flag == 0) atomicExch(dup_flag, 1u);
        }
    }
}
__global__ void k_count_dense(const uint32_t* dense, uint64_t n, unsigned long long* out) {
    unsigned long long c = 0;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        c += dense[i] != kNone;
    for (int o = 16; o; o >>= 1) c += __shfl_xor_sync(0xFFFFFFFFu, c, o);
    if ((threadIdx.x & 31) == 0 && c) atomicAdd(out, c);
}

__global__ void k_count_slots(TableView t, unsigned long long* out) {
    uint64_t n = t.mask + 1;
    unsigned long long c = 0;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        c += (uint32_t)slot_at(t, i)[0] != 0;
    for (int o = 16; o; o >>= 1) c += __shfl_xor_sync(0xFFFFFFFFu, c, o);
    if ((threadIdx.x & 31) == 0 && c) atomicAdd(out, c);
}

// ---- canonical string ids (equal strings -> the smallest-claimed row) ---------------------------
__global__ void k_strid(const uint32_t* off, const uint8_t* bytes, const uint64_t* valid, int64_t n, TableView t,
                        uint32_t* canon, uint32_t* err) {
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        uint32_t r = (uint32_t)i;
        if (!valid_bit(valid, r)) {
            canon[r] = r;
            continue;
        }
        uint32_t a = off[r], b = off[r + 1];
        uint64_t h = hash_bytes(bytes + a, b - a);
        uint64_t s = h & t.mask;
        uint32_t result = kNone;
        for (uint64_t k = 0; k <= t.mask && result == kNone;) {
            uint64_t* sl = slot_at(t, s);
            uint32_t* st_p = (uint32_t*)sl;
            uint32_t st = load_state(st_p);
            if (st == 0) {
                uint32_t old = atomicCAS(st_p, 0u, 1u);
                if (old == 0) {
                    sl[1] = h;
                    st_p[1] = r;
                    publish_state(st_p, 2);
                    result = r;
                    break;
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
                    result = r;
                    break;
                }
            }
            if (sl[1] == h) {
                uint32_t c = st_p[1];
                uint32_t ca = off[c], cb = off[c + 1];
                if (cb - ca == b - a && bytes_eq(bytes + a, bytes + ca, b - a)) {
                    result = c;
                    break;
                }
            }
            s = (s + 1) & t.mask;
            k++;
        }
        canon[r] = result == kNone ? r : result;
    }
}

// ---- gathers ------------------------------------------------------------------------------------
__global__ void k_gather_fixed(const uint8_t* src, int width, const uint32_t* idx, int64_t k, uint8_t* dst) {
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < k; i += stride) {
        uint64_t r = idx[i];
        switch (width) {
            case 1: dst[i] = src[r]; break;
            case 4: ((uint32_t*)dst)[i] = ((const uint32_t*)src)[r]; break;
            case 8: ((uint64_t*)dst)[i] = ((const uint64_t*)src)[r]; break;
            default: {  // rows of width / 8 words (a group's accumulator block)
                const int w = width / 8;
                const uint64_t* s8 = (const uint64_t*)src + r * w;
                uint64_t* d8 = (uint64_t*)dst + i * w;
                for (int j = 0; j < w; j++) d8[j] = s8[j];
                break;
            }
        }
    }
}
__global__ void k_gather_valid(const uint64_t* src, const uint32_t* idx, int64_t k, uint32_t* dst) {
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i0 = (int64_t)blockIdx.x * blockDim.x; i0 < k; i0 += stride) {
        int64_t i = i0 + threadIdx.x;
        bool v = false;
        if (i < k) v = valid_bit(src, idx[i]);
        uint32_t b = __ballot_sync(0xFFFFFFFFu, v);
        if ((threadIdx.x & 31) == 0 && i < k) dst[i >> 5] = b;
    }
}
__global__ void k_utf8_lengths(const uint32_t* off, const uint32_t* idx, int64_t k, uint32_t* len) {
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < k; i += stride) {
        uint32_t r = idx ? idx[i] : (uint32_t)i;
        len[i] = off[r + 1] - off[r];
    }
}
__global__ void k_utf8_copy(const uint32_t* off, const uint8_t* bytes, const uint32_t* idx, int64_t k,
                            const uint64_t* dst_off, uint8_t* dst) {
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < k; i += stride) {
        uint32_t r = idx ? idx[i] : (uint32_t)i;
        uint32_t a = off[r], b = off[r + 1];
        uint8_t* d = dst + dst_off[i];
        for (uint32_t j = a; j < b; j++) d[j - a] = bytes[j];
    }
}
__global__ void k_u64_to_u32(const uint64_t* in, uint32_t* out, int64_t n) {
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) out[i] = (uint32_t)in[i];
}

__global__ void k_offsets_rebase(const uint32_t* src, int64_t n, uint32_t base, uint32_t* dst) {
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    uint32_t first = src[0];
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i <= n; i += stride) dst[i] = src[i] - first + base;
}
__global__ void k_copy_bits(const uint64_t* src, int64_t n, uint64_t* dst, int64_t dst_off) {
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        bool v = src == nullptr || ((src[i >> 6] >> (i & 63)) & 1ull);
        if (v) {
            int64_t o = dst_off + i;
            atomicOr((unsigned long long*)dst + (o >> 6), 1ull << (o & 63));
        }
    }
}

// ---- top-N -------------------------------------------------------------------------------------------
// compare_rows (sort.rs:43-82): per key, NULLs first/last, f64 by total order, asc/desc.
__device__ __forceinline__ int64_t total_key(double d) {
    int64_t x = __double_as_longlong(d);
    return x ^ (int64_t)(((uint64_t)(x >> 63)) >> 1);
}
// Not inlined: the sorting networks call it only when two prefixes tie, and inlining it into
// every compare-exchange multiplies their code size.
__device__ __noinline__ int cmp_rows(const SortDev& S, uint32_t a, uint32_t b) {
    if (a == kNone || b == kNone) return (a == kNone) - (b == kNone);  // padding sorts last
    for (int k = 0; k < S.nkeys; k++) {
        const DCol& c = S.cols[k];
        bool va = valid_bit(c.valid, a), vb = valid_bit(c.valid, b);
        int o = 0;
        if (!va && !vb) o = 0;
        else if (!va) return S.nulls_first[k] ? -1 : 1;
        else if (!vb) return S.nulls_first[k] ? 1 : -1;
        else {
            if (c.kind == CK_UTF8) {
                o = str_cmp(col_str(c, a), col_str(c, b));
            } else {
                uint64_t x = load_value(c, a), y = load_value(c, b);
                switch (c.dt) {
                    case ML_TYPE_FLOAT64: {
                        int64_t p = total_key(as_f64(x)), q = total_key(as_f64(y));
                        o = p < q ? -1 : (p > q);
                        break;
                    }
                    case ML_TYPE_BOOL: o = (x < y) ? -1 : (x > y); break;
                    default: o = ((int64_t)x < (int64_t)y) ? -1 : ((int64_t)x > (int64_t)y); break;
                }
            }
            if (!S.asc[k]) o = -o;
        }
        if (o) return o;
    }
    return 0;
}

// Order-preserving 64-bit prefix of the first sort key: prefix(a) < prefix(b) implies
// cmp_rows(a, b) < 0, so rows are compared through shared memory and cmp_rows runs
// only on equal prefixes (ties, NULLs and padding).
__device__ __forceinline__ uint64_t sort_prefix(const SortDev& S, uint32_t r) {
    if (r == kNone) return ~0ull;
    const DCol& c = S.cols[0];
    if (!valid_bit(c.valid, r)) return S.nulls_first[0] ? 0ull : ~0ull;
    uint64_t p;
    if (c.kind == CK_UTF8) {
        Str s = col_str(c, r);
        p = 0;
        uint32_t m = s.n < 8 ? s.n : 8;
        for (uint32_t j = 0; j < m; j++) p |= (uint64_t)__ldg(s.p + j) << (56 - 8 * j);
    } else {
        uint64_t x = load_value(c, r);
        if (c.dt == ML_TYPE_FLOAT64) p = (uint64_t)total_key(as_f64(x)) ^ 0x8000000000000000ull;
        else if (c.dt == ML_TYPE_BOOL) p = x;
        else p = x ^ 0x8000000000000000ull;
    }
    return S.asc[0] ? p : ~p;
}

// One block sorts kTopNChunk rows (bitonic, ascending by compare_rows) and writes the
// first k.  Keys are compared by their shared-memory prefix first.
__global__ void __launch_bounds__(1024) k_topn_chunk(const __grid_constant__ SortDev S, const uint32_t* in, int64_t n,
                                                    int k, uint32_t* out) {
    __shared__ uint64_t pre[kTopNChunk];
    __shared__ uint32_t idx[kTopNChunk];
    int64_t base = (int64_t)blockIdx.x * kTopNChunk;
    for (int j = threadIdx.x; j < kTopNChunk; j += blockDim.x) {
        int64_t i = base + j;
        uint32_t r = i < n ? (in ? in[i] : (uint32_t)i) : kNone;
        idx[j] = r;
        pre[j] = sort_prefix(S, r);
    }
    __syncthreads();
    for (int size = 2; size <= kTopNChunk; size <<= 1) {
        for (int stride = size >> 1; stride > 0; stride >>= 1) {
            for (int t = threadIdx.x; t < kTopNChunk / 2; t += blockDim.x) {
                int lo = 2 * t - (t & (stride - 1));
                int hi = lo + stride;
                bool up = (lo & size) == 0;
                uint64_t pa = pre[lo], pb = pre[hi];
                int c = pa < pb ? -1 : (pa > pb ? 1 : cmp_rows(S, idx[lo], idx[hi]));
                if (c == 0) c = idx[lo] < idx[hi] ? -1 : (idx[lo] > idx[hi]);  // equal keys: input order
                if ((c > 0) == up && c != 0) {
                    uint32_t a = idx[lo];
                    idx[lo] = idx[hi];
                    idx[hi] = a;
                    pre[lo] = pb;
                    pre[hi] = pa;
                }
            }
            __syncthreads();
        }
    }
    for (int j = threadIdx.x; j < k; j += blockDim.x) out[(int64_t)blockIdx.x * k + j] = idx[j];
}

// ---- top-N for small limits (k <= 32): one sorted list per warp ------------------------------
// Each lane holds one entry of the warp's current best 32 (ascending); a batch of 32 new
// rows is skipped unless one of them beats the k-th entry, else it is sorted with a
// shuffle bitonic network and merged in.  The CTA then merges its warps' lists.
struct TopEntry {
    uint64_t p;  // sort_prefix
    uint32_t r;  // row (kNone = padding)
};
// Rows with equal keys keep their input order (the row id breaks the tie), as in a stable sort.
__device__ __forceinline__ bool entry_less(const SortDev& S, TopEntry a, TopEntry b) {
    if (a.p != b.p) return a.p < b.p;
    const int c = cmp_rows(S, a.r, b.r);
    return c ? c < 0 : a.r < b.r;
}
__device__ __forceinline__ TopEntry shfl_entry(TopEntry e, int src) {
    return TopEntry{__shfl_sync(0xFFFFFFFFu, e.p, src), __shfl_sync(0xFFFFFFFFu, e.r, src)};
}
// Compare-exchange with the lane `lane ^ j`; the lower lane keeps the smaller entry when
// `ascending`.  Both lanes evaluate entry_less(upper, lower), so ties resolve consistently.
__device__ __forceinline__ TopEntry cmp_exchange(const SortDev& S, TopEntry e, int lane, int j, bool ascending) {
    TopEntry o = shfl_entry(e, lane ^ j);
    bool lower = (lane & j) == 0;
    TopEntry lo = lower ? e : o, hi = lower ? o : e;
    bool swap = entry_less(S, hi, lo);
    bool keep_min = lower == ascending;
    if (keep_min) return swap ? hi : lo;
    return swap ? lo : hi;
}
// The networks' loops stay rolled: these kernels run them a few times per warp from a cold
// instruction cache, where fetching unrolled copies costs more than the loop overhead.
__device__ __forceinline__ TopEntry warp_sort32(const SortDev& S, TopEntry e, int lane) {
#pragma unroll 1
    for (int k = 2; k <= 32; k <<= 1)
#pragma unroll 1
        for (int j = k >> 1; j > 0; j >>= 1) e = cmp_exchange(S, e, lane, j, (lane & k) == 0);
    return e;
}
// Merge sorted `n` into sorted `l`: keep the 32 smallest of both, sorted ascending.
__device__ __forceinline__ TopEntry warp_merge32(const SortDev& S, TopEntry l, TopEntry n, int lane) {
    TopEntry rev = shfl_entry(n, 31 - lane);
    TopEntry e = entry_less(S, rev, l) ? rev : l;  // bitonic: the 32 smallest of the union
#pragma unroll 1
    for (int j = 16; j > 0; j >>= 1) e = cmp_exchange(S, e, lane, j, true);
    return e;
}

// The qn queued entries into the warp's sorted list: a few are inserted one at a time (a ballot
// for the position, a shuffle to move the larger entries up one lane), more are sorted in groups
// of 32 and merged.  Queued rows are never in the list already.  One out-of-line copy serves
// every call site (the whole warp calls it).
__device__ __noinline__ TopEntry warp_absorb(const SortDev& S, TopEntry best, const TopEntry* queue, int qn, int lane) {
    if (qn <= 8) {
#pragma unroll 1
        for (int i = 0; i < qn; i++) {
            const TopEntry c = queue[i];
            const int pos = __popc(__ballot_sync(0xFFFFFFFFu, entry_less(S, best, c)));
            const TopEntry up{__shfl_up_sync(0xFFFFFFFFu, best.p, 1), __shfl_up_sync(0xFFFFFFFFu, best.r, 1)};
            if (lane >= pos) best = lane == pos ? c : up;
        }
    } else {
#pragma unroll 1
        for (int i = 0; i < qn; i += 32) {
            const TopEntry e = i + lane < qn ? queue[i + lane] : TopEntry{~0ull, kNone};
            best = warp_merge32(S, best, warp_sort32(S, e, lane), lane);
        }
    }
    return best;
}

// Rows that beat the warp's current k-th entry are queued in shared memory; a full queue
// (32 entries) is sorted and merged into the list, so the sort runs once per 32
// candidates, not once per 32 rows (about k * ln(rows / k) candidates reach a warp).
// One warp's best k of n entries (batches of 32 from batch index `batch` on, every `batches`
// batches), as a sorted list across the lanes; get(i) yields entry i.
template <class Get>
__device__ TopEntry warp_topk(const SortDev& S, int64_t n, int k, int64_t batch, int64_t batches, TopEntry* queue,
                              int lane, Get get) {
    TopEntry best{~0ull, kNone};
    TopEntry kth = best;
    int qn = 0;  // entries in the warp's queue (warp-uniform)
    auto flush = [&]() {
        __syncwarp();
        best = warp_absorb(S, best, queue, qn, lane);
        __syncwarp();
        kth = shfl_entry(best, k - 1);
        qn = 0;
    };
    for (int64_t base = batch * 32; base < n; base += batches * 32) {
        int64_t i = base + lane;
        TopEntry e = i < n ? get(i) : TopEntry{~0ull, kNone};
        bool take = e.r != kNone && entry_less(S, e, kth);
        unsigned m = __ballot_sync(0xFFFFFFFFu, take);
        if (!m) continue;
        if (qn + __popc(m) > 32) {
            flush();
            take = take && entry_less(S, e, kth);
            m = __ballot_sync(0xFFFFFFFFu, take);
        }
        if (take) queue[qn + __popc(m & ((1u << lane) - 1))] = e;
        qn += __popc(m);
        __syncwarp();
    }
    if (qn) flush();
    return best;
}

// sort_prefix of a fixed-width first key of type DT from its loaded value (load_value's form):
// `flip` is 0 for ascending keys and ~0 for descending ones, `nullp` the prefix of a NULL.
template <int DT>
__device__ __forceinline__ uint64_t fixed_prefix(uint64_t x, bool valid, uint64_t flip, uint64_t nullp) {
    uint64_t p;
    if (DT == ML_TYPE_FLOAT64) p = (uint64_t)total_key(as_f64(x)) ^ 0x8000000000000000ull;
    else if (DT == ML_TYPE_BOOL) p = x;
    else p = x ^ 0x8000000000000000ull;
    return valid ? p ^ flip : nullp;
}

// Four consecutive values of the key column (registers, not an array: no stack traffic).
struct Quad {
    uint64_t v0, v1, v2, v3;
};

// Four consecutive rows of the key column from r0 (one or two 16-byte loads when the column is
// aligned and the four rows exist; rows past n read as 0 and are never queued).
template <int DT>
__device__ __forceinline__ Quad load_quad(const DCol& c, bool vec, uint32_t n32, uint32_t r0) {
    Quad q{0ull, 0ull, 0ull, 0ull};
    if (vec && (uint64_t)r0 + 4u <= (uint64_t)n32) {
        if (DT == ML_TYPE_FLOAT64 || DT == ML_TYPE_INT64) {
            uint64_t t[2], u[2];
            ld_stream_v2_u64((const unsigned long long*)c.data + r0, t);
            ld_stream_v2_u64((const unsigned long long*)c.data + r0 + 2, u);
            q = Quad{t[0], t[1], u[0], u[1]};
        } else if (DT == ML_TYPE_BOOL) {
            const uint32_t w = ld_stream_u32((const uint8_t*)c.data + r0);
            q = Quad{w & 0xFFu, (w >> 8) & 0xFFu, (w >> 16) & 0xFFu, w >> 24};
        } else {
            uint32_t w[4];
            ld_stream_v4_u32((const uint32_t*)c.data + r0, w);
            q = Quad{(uint64_t)(int64_t)(int32_t)w[0], (uint64_t)(int64_t)(int32_t)w[1],
                     (uint64_t)(int64_t)(int32_t)w[2], (uint64_t)(int64_t)(int32_t)w[3]};
        }
    } else {
        const uint64_t r = r0;
        if (r < n32) q.v0 = load_value(c, r0);
        if (r + 1u < n32) q.v1 = load_value(c, r0 + 1u);
        if (r + 2u < n32) q.v2 = load_value(c, r0 + 2u);
        if (r + 3u < n32) q.v3 = load_value(c, r0 + 3u);
    }
    return q;
}

// Queues the lane's four rows from r0 that can still be in the top k: prefix at or below
// `bound` (the warp's k-th entry and the launch-wide threshold) and ahead of the k-th entry.
// The queue holds (at most) 31 entries carried over plus the 128 of a half-step.
template <int DT>
__device__ __forceinline__ void queue_quad(const SortDev& S, const DCol& c, const Quad& q, uint32_t r0, uint32_t n32,
                                           uint64_t flip, uint64_t nullp, uint64_t bound, TopEntry kth,
                                           TopEntry* queue, int lane, int& qn) {
    const uint32_t rem = r0 < n32 ? n32 - r0 : 0u;  // rows of the four that exist
    uint32_t vb = 0xFu;
    if (c.valid && rem) vb = (uint32_t)(__ldg(c.valid + (r0 >> 6)) >> (r0 & 63u));
    const uint64_t p0 = fixed_prefix<DT>(q.v0, vb & 1u, flip, nullp);
    const uint64_t p1 = fixed_prefix<DT>(q.v1, vb & 2u, flip, nullp);
    const uint64_t p2 = fixed_prefix<DT>(q.v2, vb & 4u, flip, nullp);
    const uint64_t p3 = fixed_prefix<DT>(q.v3, vb & 8u, flip, nullp);
    const bool any = (rem > 0 && p0 <= bound) || (rem > 1 && p1 <= bound) || (rem > 2 && p2 <= bound) ||
                     (rem > 3 && p3 <= bound);
    if (!__any_sync(0xFFFFFFFFu, any)) return;
    const unsigned lt = (1u << lane) - 1u;
#pragma unroll
    for (uint32_t j = 0; j < 4; j++) {
        const uint64_t p = j == 0 ? p0 : j == 1 ? p1 : j == 2 ? p2 : p3;
        const TopEntry e{p, r0 + j};
        const bool take = rem > j && p <= bound && entry_less(S, e, kth);
        const unsigned m = __ballot_sync(0xFFFFFFFFu, take);
        if (take) queue[qn + __popc(m & lt)] = e;
        qn += __popc(m);
    }
}

// warp_topk over the source rows when the first sort key is a fixed-width column of type DT:
// 256-row steps, each lane reading 4 consecutive rows of each 128-row half (one or two 16-byte
// loads when the column is aligned); the next step's values and the shared threshold are loaded
// before the current step is compared, so a warp keeps 4 KB in flight.  Each half queues the
// rows that beat the k-th entry (usually none: it costs its loads and compares), and a queue of
// 32 or more goes into the list (warp_absorb, one out-of-line copy; the warp's state stays in
// registers).
// `shared_thr` (optional, starts at 0) holds ~T for the smallest full-list k-th prefix T any warp
// of the launch has published: k rows have prefixes <= T, so a
// row with a larger prefix cannot be in the top k and no warp queues it.
constexpr int kTopNQueue = 160;  // 31 carried over + the 128 rows of a half-step, rounded up
template <int DT>
__device__ TopEntry warp_topk_fixed(const SortDev& S, int64_t n, int k, int64_t chunk, int64_t chunks, TopEntry* queue,
                                    int lane, unsigned long long* shared_thr) {
    const DCol& c = S.cols[0];
    const bool vec = ((uintptr_t)c.data & 15) == 0;
    const uint64_t flip = S.asc[0] ? 0ull : ~0ull, nullp = S.nulls_first[0] ? 0ull : ~0ull;
    const uint32_t n32 = (uint32_t)n;  // row ids are 32-bit
    TopEntry best{~0ull, kNone};
    TopEntry kth = best;
    int qn = 0;  // entries in the warp's queue (warp-uniform)
    uint64_t thr = ~0ull;
    const Quad zero{0ull, 0ull, 0ull, 0ull};
    int64_t base = chunk * 256;
    Quad qa = zero, qb = zero;
    uint64_t pc = 0;
    auto absorb = [&]() {  // the queue into the list; publish a tighter k-th
        __syncwarp();
        best = warp_absorb(S, best, queue, qn, lane);
        __syncwarp();
        kth = shfl_entry(best, k - 1);
        qn = 0;
        if (shared_thr && kth.r != kNone && kth.p < thr) {
            thr = kth.p;
            if (lane == 0) atomicMax(shared_thr, ~kth.p);
        }
    };
    if (base < n) {
        qa = load_quad<DT>(c, vec, n32, (uint32_t)base + (uint32_t)lane * 4u);
        qb = load_quad<DT>(c, vec, n32, (uint32_t)base + 128u + (uint32_t)lane * 4u);
    }
    for (;;) {
        const bool more = base < n;
        if (more) {
            const int64_t next = base + chunks * 256;
            Quad na = zero, nb = zero;
            uint64_t pn = pc;
            if (next < n) {
                na = load_quad<DT>(c, vec, n32, (uint32_t)next + (uint32_t)lane * 4u);
                nb = load_quad<DT>(c, vec, n32, (uint32_t)next + 128u + (uint32_t)lane * 4u);
                if (shared_thr) pn = __ldcg(shared_thr);
            }
            thr = ~pc < thr ? ~pc : thr;
            queue_quad<DT>(S, c, qa, (uint32_t)base + (uint32_t)lane * 4u, n32, flip, nullp,
                           kth.p < thr ? kth.p : thr, kth, queue, lane, qn);
            if (qn >= 32) absorb();
            queue_quad<DT>(S, c, qb, (uint32_t)base + 128u + (uint32_t)lane * 4u, n32, flip, nullp,
                           kth.p < thr ? kth.p : thr, kth, queue, lane, qn);
            qa = na;
            qb = nb;
            pc = pn;
            base = next;
        }
        if (qn >= 32 || (!more && qn)) absorb();
        if (!more) break;
    }
    return best;
}

// Each CTA writes its best k rows to out[block * k ..].  With `final_out`, CTAs also write
// their (prefix, row) entries to `cand`, and the last CTA to finish (the counter `done` starts
// at zero) merges all CTAs' entries into final_out[0 .. k): the whole top-k in one launch.
// DT: the first sort key's type when it is a fixed-width column (warp_topk_fixed), -1 otherwise.
template <int DT>
__global__ void __launch_bounds__(256, 2) k_topn_warp(const __grid_constant__ SortDev S, int64_t n, int k, uint32_t* out,
                                                   TopEntry* cand, unsigned int* done, uint32_t* final_out,
                                                   const uint64_t* n_dev) {
    if (n_dev) n = min(n, (int64_t)__ldcg(n_dev));  // a replayed plan's row count
    __shared__ TopEntry lists[8][32];
    __shared__ TopEntry queue[8][kTopNQueue];
    __shared__ bool last;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    TopEntry best;
    // `done` points at 16 zeroed bytes: the finished-CTA counter, then the shared threshold
    unsigned long long* thr = done ? reinterpret_cast<unsigned long long*>(done + 2) : nullptr;
    if (DT >= 0)
        best = warp_topk_fixed<DT < 0 ? 0 : DT>(S, n, k, (int64_t)blockIdx.x * 8 + warp, (int64_t)gridDim.x * 8,
                                                  queue[warp], lane, thr);
    else
        best = warp_topk(S, n, k, (int64_t)blockIdx.x * 8 + warp, (int64_t)gridDim.x * 8, queue[warp], lane,
                         [&](int64_t i) { return TopEntry{sort_prefix(S, (uint32_t)i), (uint32_t)i}; });
    lists[warp][lane] = best;
    __syncthreads();
    if (warp == 0) {
#pragma unroll 1
        for (int w = 1; w < 8; w++) best = warp_merge32(S, best, lists[w][lane], lane);
        if (lane < k) {
            out[(int64_t)blockIdx.x * k + lane] = best.r;
            if (final_out) cand[(int64_t)blockIdx.x * k + lane] = best;
        }
    }
    if (!final_out) return;
    __threadfence();  // this CTA's entries are visible before it counts itself done
    __syncthreads();
    if (threadIdx.x == 0) last = atomicAdd(done, 1u) == gridDim.x - 1;
    __syncthreads();
    if (!last) return;
    __threadfence();
    const int64_t m = (int64_t)gridDim.x * k;
    // k rows of some warp's full list have prefixes <= the published threshold, so a candidate
    // above it cannot be in the top k: most CTAs' lists drop out here without a sort.  Each warp
    // loads four batches of 32 candidates at once, queues those that can be in the top k, and
    // takes its queue into its list from one place once it holds 32 or the candidates are done.
    const uint64_t bound = thr ? ~__ldcg(thr) : ~0ull;
    {
        TopEntry* qw = queue[warp];
        best = TopEntry{~0ull, kNone};
        TopEntry kth = best;
        int qn = 0;
        for (int64_t b0 = (int64_t)warp * 32;; b0 += 8 * 32 * 4) {
            const bool more = b0 < m;
            if (more) {
                TopEntry e[4];
#pragma unroll
                for (int j = 0; j < 4; j++) {
                    const int64_t i = b0 + j * 256 + lane;
                    e[j] = TopEntry{~0ull, kNone};
                    if (i < m) e[j] = TopEntry{__ldcg((const unsigned long long*)&cand[i].p), __ldcg(&cand[i].r)};
                }
                const unsigned lt = (1u << lane) - 1u;
#pragma unroll
                for (int j = 0; j < 4; j++) {
                    const bool take = e[j].r != kNone && e[j].p <= bound && entry_less(S, e[j], kth);
                    const unsigned mk = __ballot_sync(0xFFFFFFFFu, take);
                    if (take) qw[qn + __popc(mk & lt)] = e[j];
                    qn += __popc(mk);
                }
            }
            if (qn >= 32 || (!more && qn)) {
                __syncwarp();
                best = warp_absorb(S, best, qw, qn, lane);
                __syncwarp();
                kth = shfl_entry(best, k - 1);
                qn = 0;
            }
            if (!more) break;
        }
    }
    lists[warp][lane] = best;
    __syncthreads();
    if (warp == 0) {
#pragma unroll 1
        for (int w = 1; w < 8; w++) best = warp_merge32(S, best, lists[w][lane], lane);
        if (lane < k) final_out[lane] = best.r;
    }
}

// ---- full ORDER BY: stable LSD radix sort of row ids over 64-bit key words -------------------
// sort_batches without a limit (sort.rs:85-132) is a stable sort by compare_rows; a stable LSD
// radix sort over the key words below, least significant first, gives the same order: per key
// (last key first) its value words, then its NULL flag; byte passes whose digit is the same for
// every row are skipped.
__device__ uint64_t sort_word(const SortWord& w, uint32_t r) {
    const DCol& c = w.col;
    const bool valid = valid_bit(c.valid, r);
    if (w.what == SW_NULL_FLAG) return (valid == (w.nulls_first != 0)) ? 1ull : 0ull;
    if (!valid) return 0ull;
    uint64_t x;
    if (w.what == SW_VALUE) {
        const uint64_t v = load_value(c, r);
        if (c.dt == ML_TYPE_FLOAT64) x = (uint64_t)total_key(as_f64(v)) ^ 0x8000000000000000ull;
        else if (c.dt == ML_TYPE_BOOL) x = v;
        else x = v ^ 0x8000000000000000ull;  // sign-extended integers
    } else if (w.what == SW_CHUNK) {
        const Str s = col_str(c, r);
        x = 0;
        const uint32_t b0 = 8u * (uint32_t)w.chunk;
        for (uint32_t j = 0; j < 8; j++)
            if (b0 + j < s.n) x |= (uint64_t)__ldg(s.p + b0 + j) << (56 - 8 * j);
    } else if (w.what == SW_LENGTH) {
        x = col_str(c, r).n;
    } else {  // SW_RANK: the dictionary entry's rank among the dictionary's strings
        x = __ldg(w.rank + dict_code(c, r));
    }
    return w.desc ? ~x : x;
}
__global__ void k_sort_words(const __grid_constant__ SortWord w, const uint32_t* perm, int64_t n, uint64_t* out) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
        out[i] = sort_word(w, perm ? perm[i] : (uint32_t)i);
}
// The eight byte histograms of a word array in one pass (hist: 8 x 256 counters, zeroed).
__global__ void __launch_bounds__(256) k_radix_hist8(const uint64_t* keys, int64_t n, unsigned long long* hist) {
    __shared__ uint32_t h[8][256];
    for (int i = threadIdx.x; i < 8 * 256; i += blockDim.x) h[i >> 8][i & 255] = 0;
    __syncthreads();
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const uint64_t k = keys[i];
#pragma unroll
        for (int b = 0; b < 8; b++) atomicAdd(&h[b][(k >> (8 * b)) & 255], 1u);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < 8 * 256; i += blockDim.x)
        if (h[i >> 8][i & 255]) atomicAdd(hist + i, (unsigned long long)h[i >> 8][i & 255]);
}
// Per 1024-row block: counts[digit * blocks + b] of the byte at `shift`.
__global__ void __launch_bounds__(kRadixRows) k_radix_count(const uint64_t* keys, int64_t n, int shift, uint32_t* counts) {
    __shared__ uint32_t h[256];
    for (int i = threadIdx.x; i < 256; i += blockDim.x) h[i] = 0;
    __syncthreads();
    const int64_t r = (int64_t)blockIdx.x * kRadixRows + threadIdx.x;
    if (r < n) atomicAdd(&h[(keys[r] >> shift) & 255], 1u);
    __syncthreads();
    for (int i = threadIdx.x; i < 256; i += blockDim.x) counts[(int64_t)i * gridDim.x + blockIdx.x] = h[i];
}
// Stable scatter of (key, row) pairs by the byte at `shift`: a row's position is its digit's
// offset for the block plus its rank among the block's rows with that digit (warps in order,
// lanes in order within a warp).  perm_in nullptr = rows in input order.
__global__ void __launch_bounds__(kRadixRows) k_radix_scatter(const uint64_t* keys_in, const uint32_t* perm_in, int64_t n,
                                                              int shift, const uint64_t* offs, uint64_t* keys_out,
                                                              uint32_t* perm_out) {
    __shared__ uint32_t wcnt[kRadixRows / 32][256];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int i = threadIdx.x; i < (kRadixRows / 32) * 256; i += blockDim.x) wcnt[i >> 8][i & 255] = 0;
    __syncthreads();
    const int64_t r = (int64_t)blockIdx.x * kRadixRows + threadIdx.x;
    const bool in = r < n;
    const uint64_t k = in ? keys_in[r] : 0ull;
    const uint32_t d = in ? (uint32_t)((k >> shift) & 255) : 256u;
    const unsigned same = __match_any_sync(0xFFFFFFFFu, d);
    const uint32_t rank = __popc(same & ((1u << lane) - 1u));
    if (in && rank == 0) wcnt[w][d] = __popc(same);
    __syncthreads();
    for (int q = threadIdx.x; q < 256; q += blockDim.x) {
        uint32_t run = 0;
        for (int ww = 0; ww < kRadixRows / 32; ww++) {
            const uint32_t c = wcnt[ww][q];
            wcnt[ww][q] = run;
            run += c;
        }
    }
    __syncthreads();
    if (in) {
        const uint64_t pos = offs[(int64_t)d * gridDim.x + blockIdx.x] + wcnt[w][d] + rank;
        keys_out[pos] = k;
        perm_out[pos] = perm_in ? perm_in[r] : (uint32_t)r;
    }
}
// Longest string of a plain UTF8 column (for the number of 8-byte chunk words).
__global__ void k_max_strlen(const uint32_t* off, int64_t n, unsigned int* out) {
    uint32_t m = 0;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) m = max(m, off[i + 1] - off[i]);
    for (int o = 16; o; o >>= 1) m = max(m, __shfl_xor_sync(0xFFFFFFFFu, m, o));
    if ((threadIdx.x & 31) == 0 && m) atomicMax(out, m);
}

}  // namespace

// Temporaries of ml_gpu_filter_static: a fixed-size device array, so that call allocates no
// device memory.  Nothing in it has to start at zero: the error word is cleared by each call
// and every other region is written before it is read.
static __device__ __align__(256) uint8_t g_static_filter_scratch[kStaticScratchBytes];
static_assert(kStaticCountsBytes >= 4 * (kStaticFilterMaxRows / kSelRowsPerBlock + 1), "block counts");
static_assert(kStaticOffsetsBytes >= 8 * (kStaticFilterMaxRows / kSelRowsPerBlock + 2), "block offsets");
static_assert(kStaticScanBytes >= 8 * ((kStaticFilterMaxRows / kSelRowsPerBlock + 1) / kScanBlock + 3), "scan scratch");

void* static_filter_scratch() {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_static_filter_scratch) != cudaSuccess) return nullptr;
    return p;
}

// ---- launch wrappers -------------------------------------------------------------------------------
int pipeline_grid(int64_t n) { return grid_for(n, 8); }
int agg_smem_bytes(const AggArgs& A) {
    return (int)((size_t)A.smem_groups * A.stride * 8 + (size_t)A.priv_groups * A.stride * kThreads * 8 +
                 agg_direct_bytes(A));
}
void launch_agg(const PipeArgs& P, const AggArgs& A, int smem_bytes, cudaStream_t s) {
    if (smem_bytes > (48 << 10)) cudaFuncSetAttribute(k_agg, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_bytes);
    k_agg<<<grid_for(P.n, 8), kThreads, smem_bytes, s>>>(P, A);
}
void launch_agg_resume(const PipeArgs& P, const AggArgs& A, const uint32_t* ctx, uint64_t count, int w, int smem_bytes,
                       cudaStream_t s) {
    k_agg_resume<<<grid_for((int64_t)count, 8), kThreads, smem_bytes, s>>>(P, A, ctx, count, w);
}
int xpart_blocks(int64_t n) { return (int)((n + kXPartRows - 1) / kXPartRows); }
void launch_xpart_count(const uint64_t* h, int64_t n, int nparts, uint32_t* counts, cudaStream_t s) {
    if (n > 0) k_xpart_count<<<xpart_blocks(n), kXPartRows, 0, s>>>(h, n, nparts, counts);
}
void launch_xpart_scatter(const uint64_t* h, int64_t n, int nparts, const uint64_t* offs, uint32_t* perm, cudaStream_t s) {
    if (n > 0) k_xpart_scatter<<<xpart_blocks(n), kXPartRows, 0, s>>>(h, n, nparts, offs, perm);
}
void launch_spill_part(const uint64_t* gkeys, const uint32_t* gnull, uint32_t gid_cap, uint32_t ng, int nwords,
                       uint64_t* part, cudaStream_t s) {
    if (ng) k_spill_part<<<(ng + kThreads - 1) / kThreads, kThreads, 0, s>>>(gkeys, gnull, gid_cap, ng, nwords, part);
}
void launch_agg_merge_spill(const AggArgs& A, const uint64_t* keys, const uint32_t* nulls, const uint64_t* acc,
                            const uint64_t* vcnt, uint32_t n, uint32_t* err, cudaStream_t s) {
    if (n) k_agg_merge_spill<<<(n + kThreads - 1) / kThreads, kThreads, 0, s>>>(A, keys, nulls, acc, vcnt, n, err);
}
void launch_agg_rehash(TableView t, const uint64_t* gkeys, const uint32_t* gnull, uint32_t gid_cap, uint32_t ngroups,
                       int nwords, uint32_t* err, cudaStream_t s) {
    if (!ngroups) return;
    k_agg_rehash<<<(ngroups + kThreads - 1) / kThreads, kThreads, 0, s>>>(t, gkeys, gnull, gid_cap, ngroups, nwords, err);
}
void launch_acc_init(const AggArgs& A, uint32_t from, uint32_t to, cudaStream_t s) {
    if (to <= from) return;
    k_acc_init<<<(to - from + kThreads - 1) / kThreads, kThreads, 0, s>>>(A, from, to);
}
void launch_agg_final(const FinalArgs& F, cudaStream_t s) {
    if (!F.ngroups) return;
    k_agg_final<<<(F.ngroups + kThreads - 1) / kThreads, kThreads, 0, s>>>(F);
}

int select_blocks(int64_t n) { return (int)((n + kSelRowsPerBlock - 1) / kSelRowsPerBlock); }
int select_rows_per_block() { return kSelRowsPerBlock; }
void launch_select_flags(const PipeArgs& P, uint32_t* bits, uint32_t* block_counts, cudaStream_t s) {
    int nb = select_blocks(P.n);
    if (nb) k_select_flags<<<nb, kThreads, 0, s>>>(P, bits, block_counts);
}
void launch_select_write(const PipeArgs& P, const uint32_t* bits, const uint64_t* block_offsets, uint32_t* out,
                         cudaStream_t s) {
    int nb = select_blocks(P.n);
    if (nb) k_index_write<<<nb, kThreads, 0, s>>>(P.n, P.sel, bits, block_offsets, out);
}
void launch_index_write(int64_t n, const uint32_t* bits, const uint64_t* block_offsets, uint32_t* out, cudaStream_t s) {
    int nb = select_blocks(n);
    if (nb) k_index_write<<<nb, kThreads, 0, s>>>(n, nullptr, bits, block_offsets, out);
}
__global__ void k_dense_keys(const uint32_t* gids, int64_t n, const uint64_t* n_dev, uint64_t dmin, int dt, void* out) {
    if (n_dev) n = min(n, (int64_t)__ldg(n_dev));
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const uint64_t k = dmin + gids[i];  // the normalized key word
        if (dt == ML_TYPE_INT64) ((int64_t*)out)[i] = (int64_t)k;
        else ((int32_t*)out)[i] = (int32_t)(uint32_t)k;
    }
}
void launch_dense_keys(const uint32_t* gids, int64_t n, uint64_t dmin, int dt, void* out, cudaStream_t s,
                       const uint64_t* n_dev) {
    if (n) k_dense_keys<<<grid_for(n, 8), kThreads, 0, s>>>(gids, n, n_dev, dmin, dt, out);
}
void launch_group_flags(const uint64_t* acc, int stride, int64_t n, const uint32_t* member, uint32_t* bits,
                        uint32_t* block_counts, cudaStream_t s) {
    int nb = select_blocks(n);
    if (nb) k_group_flags<<<nb, kThreads, 0, s>>>(acc, stride, n, member, bits, block_counts);
}
void launch_count_slots(TableView t, unsigned long long* out, cudaStream_t s) {
    k_count_slots<<<grid_for((int64_t)t.mask + 1, 8), kThreads, 0, s>>>(t, out);
}
size_t scan_scratch_words(int64_t n) { return (size_t)((n + kScanBlock - 1) / kScanBlock) + 2; }
void launch_scan_u32(const uint32_t* in, uint64_t* out, int64_t n, uint64_t* scratch, cudaStream_t s) {
    int64_t nb = (n + kScanBlock - 1) / kScanBlock;
    if (nb == 0) {
        cudaMemsetAsync(out, 0, sizeof(uint64_t), s);
        return;
    }
    k_scan_reduce<<<(unsigned)nb, 1024, 0, s>>>(in, n, scratch);
    k_scan_sums<<<1, 1024, 0, s>>>(scratch, nb);
    k_scan_apply<<<(unsigned)nb, 1024, 0, s>>>(in, n, scratch, out);
}

void launch_project(const PipeArgs& P, Prog prog, int out_type, void* out, uint32_t* valid, cudaStream_t s) {
    if (P.n) k_project<<<grid_for(P.n, 8), kThreads, 0, s>>>(P, prog, out_type, out, valid);
}
void launch_hash_columns(const PipeArgs& P, int ncols, const uint64_t* const* dict_hash, uint64_t* out, cudaStream_t s) {
    if (P.n) k_hash_columns<<<grid_for(P.n, 8), kThreads, 0, s>>>(P, ncols, dict_hash, out);
}
void launch_join_insert(const PipeArgs& P, const KeyLayout& L, TableView t, uint32_t* next, uint32_t* dup_flag,
                        int64_t n, cudaStream_t s) {
    if (n) k_join_insert<<<grid_for(n, 8), kThreads, 0, s>>>(P, L, t, next, dup_flag, n);
}
void launch_key_range(const void* data, int dt, const uint64_t* valid, int64_t n, unsigned long long* mm, cudaStream_t s) {
    if (n) k_key_range<<<grid_for(n, 4), kThreads, 0, s>>>(data, dt, valid, n, mm);
}
void launch_dense_insert(const void* data, int dt, const uint64_t* valid, int64_t n, uint64_t dmin, uint64_t drange,
                         uint32_t* dense, uint32_t* next, uint32_t* dup_flag, uint32_t* range_err, cudaStream_t s) {
    if (n) k_dense_insert<<<grid_for(n, 8), kThreads, 0, s>>>(data, dt, valid, n, dmin, drange, dense, next, dup_flag, range_err);
}
void launch_dense_bits(const uint32_t* dense, uint64_t n, uint32_t* bits, cudaStream_t s) {
    const uint64_t words = (n + 31) / 32;
    if (words) k_dense_bits<<<grid_for((int64_t)words * 32, 8), kThreads, 0, s>>>(dense, n, bits);
}
void launch_count_dense(const uint32_t* dense, uint64_t n, unsigned long long* out, cudaStream_t s) {
    if (n) k_count_dense<<<grid_for((int64_t)n, 8), kThreads, 0, s>>>(dense, n, out);
}
void launch_probe_count(const PipeArgs& P, uint32_t* counts, cudaStream_t s) {
    if (P.n) k_probe_count<<<grid_for(P.n, 8), kThreads, 0, s>>>(P, counts);
}
void launch_probe_write(const PipeArgs& P, const uint64_t* offsets, uint32_t* pi, uint32_t* bi, cudaStream_t s) {
    if (P.n) k_probe_write<<<grid_for(P.n, 8), kThreads, 0, s>>>(P, offsets, pi, bi);
}
void launch_strid(const uint32_t* off, const uint8_t* bytes, const uint64_t* valid, int64_t n, TableView t,
                  uint32_t* canon, uint32_t* err, cudaStream_t s) {
    if (n) k_strid<<<grid_for(n, 8), kThreads, 0, s>>>(off, bytes, valid, n, t, canon, err);
}
void launch_gather_fixed(const void* src, int width, const uint32_t* idx, int64_t k, void* dst, cudaStream_t s) {
    if (k) k_gather_fixed<<<grid_for(k, 8), kThreads, 0, s>>>((const uint8_t*)src, width, idx, k, (uint8_t*)dst);
}
void launch_gather_valid(const uint64_t* src, const uint32_t* idx, int64_t k, uint32_t* dst, cudaStream_t s) {
    if (k) k_gather_valid<<<grid_for(k, 8), kThreads, 0, s>>>(src, idx, k, dst);
}
void launch_utf8_lengths(const uint32_t* off, const uint32_t* idx, int64_t k, uint32_t* len, cudaStream_t s) {
    if (k) k_utf8_lengths<<<grid_for(k, 8), kThreads, 0, s>>>(off, idx, k, len);
}
void launch_utf8_copy(const uint32_t* off, const uint8_t* bytes, const uint32_t* idx, int64_t k, const uint64_t* dst_off,
                      uint8_t* dst, cudaStream_t s) {
    if (k) k_utf8_copy<<<grid_for(k, 8), kThreads, 0, s>>>(off, bytes, idx, k, dst_off, dst);
}
void launch_u64_to_u32(const uint64_t* in, uint32_t* out, int64_t n, cudaStream_t s) {
    if (n) k_u64_to_u32<<<grid_for(n, 8), kThreads, 0, s>>>(in, out, n);
}
int topn_warp_blocks(int64_t n) {
    if (n <= 65536) return 1;  // one CTA finishes the candidates of the previous round
    static const int resident = [] {  // CTAs per SM that every instantiation reaches: one wave
        int r = 8;
        auto at_most = [&](const void* f) {
            int b = 0;
            if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, f, 256, 0) == cudaSuccess && b > 0) r = std::min(r, b);
        };
        at_most((const void*)k_topn_warp<-1>);
        at_most((const void*)k_topn_warp<ML_TYPE_FLOAT64>);
        at_most((const void*)k_topn_warp<ML_TYPE_INT64>);
        at_most((const void*)k_topn_warp<ML_TYPE_INT32>);
        at_most((const void*)k_topn_warp<ML_TYPE_BOOL>);
        return r;
    }();
    // at least 8 chunks of 128 rows per warp: a warp's first chunk mostly enters its list, later
    // ones mostly fall below the list's k-th entry or the launch-wide threshold
    int64_t want = (n + 8191) / 8192;
    int64_t cap = (int64_t)num_sms() * resident;
    return (int)std::max<int64_t>(1, std::min(want, cap));
}
size_t topn_entry_bytes() { return sizeof(TopEntry); }
int launch_topn_warp(const SortDev& S, int64_t n, int k, int blocks, uint32_t* out, void* cand, unsigned int* done,
                     uint32_t* final_out, cudaStream_t s, const uint64_t* n_dev) {
    const DCol& c = S.cols[0];
    const int dt = S.nkeys > 0 && c.kind == CK_FIXED && c.src == 0 ? c.dt : -1;
    TopEntry* ce = (TopEntry*)cand;
    switch (dt) {
        case ML_TYPE_FLOAT64: k_topn_warp<ML_TYPE_FLOAT64><<<blocks, 256, 0, s>>>(S, n, k, out, ce, done, final_out, n_dev); break;
        case ML_TYPE_INT64: k_topn_warp<ML_TYPE_INT64><<<blocks, 256, 0, s>>>(S, n, k, out, ce, done, final_out, n_dev); break;
        case ML_TYPE_INT32:
        case ML_TYPE_DATE: k_topn_warp<ML_TYPE_INT32><<<blocks, 256, 0, s>>>(S, n, k, out, ce, done, final_out, n_dev); break;
        case ML_TYPE_BOOL: k_topn_warp<ML_TYPE_BOOL><<<blocks, 256, 0, s>>>(S, n, k, out, ce, done, final_out, n_dev); break;
        default: k_topn_warp<-1><<<blocks, 256, 0, s>>>(S, n, k, out, ce, done, final_out, n_dev); break;
    }
    return 1;
}
// The packed words of string MIN/MAX states (A_MIN_STR / A_MAX_STR) after the rank table
// changed: each holds a string id in its low half; the identities (no value yet) stay.
__global__ void k_str_rerank(uint64_t* acc, int stride, uint32_t ngroups, const __grid_constant__ RerankOffs R,
                             const uint32_t* rank) {
    const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= ngroups) return;
    uint64_t* blk = acc + (uint64_t)g * stride;
    for (int j = 0; j < R.n; j++) {
        const uint64_t w = blk[R.off[j]];
        if (w == 0ull || w == ~0ull) continue;
        blk[R.off[j]] = str_pack(rank, (uint32_t)w);
    }
}
void launch_str_rerank(uint64_t* acc, int stride, uint32_t ngroups, const RerankOffs& R, const uint32_t* rank,
                       cudaStream_t s) {
    if (ngroups && R.n) k_str_rerank<<<(ngroups + kThreads - 1) / kThreads, kThreads, 0, s>>>(acc, stride, ngroups, R, rank);
}

// ---- prepared-query checks: a replayed plan's recorded choices against this run's data ------
// *guard |= bit when the 4- or 8-byte value at p differs from v (op 0) or is below v (op 1).
__global__ void k_plan_check(const void* p, int width, int op, uint64_t v, uint32_t bit, uint32_t* guard) {
    const uint64_t x = width == 8 ? *(const uint64_t*)p : (uint64_t) * (const uint32_t*)p;
    if (op == 0 ? x != v : x < v) atomicOr(guard, bit);
}
void launch_plan_check(const void* p, int width, int op, uint64_t v, uint32_t bit, uint32_t* guard, cudaStream_t s) {
    k_plan_check<<<1, 1, 0, s>>>(p, width, op, v, bit, guard);
}
// out = min(*count, cap): a group counter as the 64-bit row count later kernels read.
__global__ void k_plan_count(const uint32_t* count, uint64_t cap, uint64_t* out) {
    const uint64_t c = *count;
    *out = c < cap ? c : cap;
}
void launch_plan_count(const uint32_t* count, uint64_t cap, uint64_t* out, cudaStream_t s) {
    k_plan_count<<<1, 1, 0, s>>>(count, cap, out);
}
// The rows of a replayed top-k (k <= 32, one warp): an id at or past the rows that exist (the
// list came back short) reads row 0 instead, so the gathers stay in bounds, and sets `bit`; the
// row count n must also give the planned result: n == k when `exact`, else n >= k (`rows_bit`).
// Then every column's k values and validity bits are gathered.
__global__ void k_plan_result(const uint32_t* rows, int k, const uint64_t* n_dev, uint64_t cap, int exact, uint32_t bit,
                              uint32_t rows_bit, uint32_t* guard, const __grid_constant__ ResultCols G) {
    const int i = threadIdx.x;
    const uint64_t n = n_dev && *n_dev < cap ? *n_dev : cap;
    if (i == 0 && (exact ? n != (uint64_t)k : n < (uint64_t)k)) atomicOr(guard, rows_bit);
    uint32_t r = 0;
    if (i < k) {
        r = rows[i];
        if (r >= n) {
            r = 0;
            atomicOr(guard, bit);
        }
    }
    for (int c = 0; c < G.ncols; c++) {
        if (i < k) {
            const int w = G.width[c];
            if (w == 8) ((uint64_t*)G.dst[c])[i] = ((const uint64_t*)G.src[c])[r];
            else if (w == 4) ((uint32_t*)G.dst[c])[i] = ((const uint32_t*)G.src[c])[r];
            else ((uint8_t*)G.dst[c])[i] = ((const uint8_t*)G.src[c])[r];
        }
        if (G.dval[c]) {
            const bool v = i < k && ((G.sval[c][r >> 6] >> (r & 63)) & 1ull);
            const unsigned b = __ballot_sync(0xFFFFFFFFu, v);
            if (i == 0) G.dval[c][0] = b;
        }
    }
}
void launch_plan_result(const uint32_t* rows, int k, const uint64_t* n_dev, uint64_t cap, int exact, uint32_t bit,
                        uint32_t rows_bit, uint32_t* guard, const ResultCols& G, cudaStream_t s) {
    k_plan_result<<<1, 32, 0, s>>>(rows, k, n_dev, cap, exact, bit, rows_bit, guard, G);
}

__global__ void k_iota_u32(uint32_t* out, int64_t n) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) out[i] = (uint32_t)i;
}
void launch_iota_u32(uint32_t* out, int64_t n, cudaStream_t s) {
    if (n > 0) k_iota_u32<<<grid_for(n, 8), kThreads, 0, s>>>(out, n);
}
int radix_blocks(int64_t n) { return (int)((n + kRadixRows - 1) / kRadixRows); }
void launch_sort_words(const SortWord& w, const uint32_t* perm, int64_t n, uint64_t* out, cudaStream_t s) {
    if (n > 0) k_sort_words<<<grid_for(n, 8), kThreads, 0, s>>>(w, perm, n, out);
}
void launch_radix_hist8(const uint64_t* keys, int64_t n, unsigned long long* hist, cudaStream_t s) {
    if (n > 0) k_radix_hist8<<<grid_for(n, 4), 256, 0, s>>>(keys, n, hist);
}
void launch_radix_count(const uint64_t* keys, int64_t n, int shift, uint32_t* counts, cudaStream_t s) {
    if (n > 0) k_radix_count<<<radix_blocks(n), kRadixRows, 0, s>>>(keys, n, shift, counts);
}
void launch_radix_scatter(const uint64_t* keys_in, const uint32_t* perm_in, int64_t n, int shift, const uint64_t* offs,
                          uint64_t* keys_out, uint32_t* perm_out, cudaStream_t s) {
    if (n > 0) k_radix_scatter<<<radix_blocks(n), kRadixRows, 0, s>>>(keys_in, perm_in, n, shift, offs, keys_out, perm_out);
}
void launch_max_strlen(const uint32_t* off, int64_t n, unsigned int* out, cudaStream_t s) {
    if (n > 0) k_max_strlen<<<grid_for(n, 4), kThreads, 0, s>>>(off, n, out);
}
void launch_topn_chunk(const SortDev& S, const uint32_t* in, int64_t n, int k, uint32_t* out, cudaStream_t s) {
    int64_t nb = (n + kTopNChunk - 1) / kTopNChunk;
    if (nb) k_topn_chunk<<<(unsigned)nb, 1024, 0, s>>>(S, in, n, k, out);
}
void launch_offsets_rebase(const uint32_t* src, int64_t n, uint32_t base, uint32_t* dst, cudaStream_t s) {
    k_offsets_rebase<<<grid_for(n + 1, 8), kThreads, 0, s>>>(src, n, base, dst);
}
void launch_copy_bits(const uint64_t* src, int64_t n, uint64_t* dst, int64_t dst_off, cudaStream_t s) {
    if (n) k_copy_bits<<<grid_for(n, 8), kThreads, 0, s>>>(src, n, dst, dst_off);
}

}  // namespace mlg
