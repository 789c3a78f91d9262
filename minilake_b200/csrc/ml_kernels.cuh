// Kernel argument blocks and launch wrappers shared by ml_kernels.cu and the host runtime.
#pragma once

#include <cuda_runtime.h>

#include "ml_args.hpp"

namespace mlg {

// ---- launch wrappers (defined in ml_kernels.cu) -----------------------------------------
void launch_agg(const PipeArgs& P, const AggArgs& A, int smem_bytes, cudaStream_t s);
void launch_agg_resume(const PipeArgs& P, const AggArgs& A, const uint32_t* ctx, uint64_t count, int ctx_words,
                       int smem_bytes, cudaStream_t s);
int agg_smem_bytes(const AggArgs& A);
// Grid of the row-parallel pipeline kernels for n rows (8 CTAs of 256 threads per SM at most).
int pipeline_grid(int64_t n);
int num_sms();  // of the current device
constexpr int kPipelineThreads = 256;
void launch_agg_rehash(TableView t, const uint64_t* gkeys, const uint32_t* gnull, uint32_t gid_cap, uint32_t ngroups,
                       int nwords, uint32_t* err, cudaStream_t s);
// Out-of-HBM aggregation: the spill partition (key hash bits 32..35) of groups [0, ng), and the
// merge of spilled partial states into a table (k_agg_merge_spill).
constexpr int kSpillParts = 16;
void launch_spill_part(const uint64_t* gkeys, const uint32_t* gnull, uint32_t gid_cap, uint32_t ng, int nwords,
                       uint64_t* part, cudaStream_t s);
void launch_agg_merge_spill(const AggArgs& A, const uint64_t* keys, const uint32_t* nulls, const uint64_t* acc,
                            const uint64_t* vcnt, uint32_t n, uint32_t* err, cudaStream_t s);
// Exchange partitioning of n rows by key hash h[r] % nparts (nparts <= kMaxExchangeParts), in
// blocks of kXPartRows rows: per-(partition, block) counts (partition-major), then, from their
// exclusive scan `offs`, the stable permutation perm[pos] = row.
constexpr int kXPartRows = 1024;
constexpr int kMaxExchangeParts = 64;
int xpart_blocks(int64_t n);
void launch_xpart_count(const uint64_t* h, int64_t n, int nparts, uint32_t* counts, cudaStream_t s);
void launch_xpart_scatter(const uint64_t* h, int64_t n, int nparts, const uint64_t* offs, uint32_t* perm, cudaStream_t s);
// Initialize group blocks [from, to) to the identities of the aggregates.
void launch_acc_init(const AggArgs& A, uint32_t from, uint32_t to, cudaStream_t s);
// Final values: keys decoded into `key_out` (fixed-width or u32 string ids), aggregates into
// `agg_out`; validity as u32 words (LSB first) in *_valid.
struct FinalArgs {
    uint32_t ngroups, gid_cap;
    int32_t nkeys, nagg, ungrouped, stride;
    KeyField f[kMaxKeys];
    const uint64_t* gkeys;
    const uint32_t* gnull;
    const uint64_t* acc;
    const uint32_t* gids;  // output row -> group id (nullptr: identity)
    void* key_out[kMaxKeys];
    uint32_t* key_valid[kMaxKeys];
    AggDev aggs[kMaxAggs];
    int32_t out_type[kMaxAggs];
    void* agg_out[kMaxAggs];
    uint32_t* agg_valid[kMaxAggs];
    // optional device-side group count (a replayed plan's): the output has min(ngroups, *ng) rows
    const uint64_t* ng64;
    const uint32_t* ng32;
};
void launch_agg_final(const FinalArgs& F, cudaStream_t s);

// Filter: pass bits (u32 words) + per-block counts, then ordered compaction.
int select_blocks(int64_t n);
int select_rows_per_block();  // rows of one select_blocks block
void launch_select_flags(const PipeArgs& P, uint32_t* bits, uint32_t* block_counts, cudaStream_t s);
void launch_select_write(const PipeArgs& P, const uint32_t* bits, const uint64_t* block_offsets, uint32_t* out,
                         cudaStream_t s);
// Groups with at least one row (group blocks' word 0 > 0) and, with `member`, whose entry
// there is not kNone: pass bits + per-block counts; then launch_index_write turns bits into
// the ordered list of group ids.
void launch_group_flags(const uint64_t* acc, int stride, int64_t n, const uint32_t* member, uint32_t* bits,
                        uint32_t* block_counts, cudaStream_t s);
// Key values of dense-index groups: out[i] = dmin + gids[i] as int64, or as int32 / date.
// n_dev (optional): the device-side count of gids (at most n)
void launch_dense_keys(const uint32_t* gids, int64_t n, uint64_t dmin, int dt, void* out, cudaStream_t s,
                       const uint64_t* n_dev = nullptr);
void launch_index_write(int64_t n, const uint32_t* bits, const uint64_t* block_offsets, uint32_t* out, cudaStream_t s);
// Exclusive scan of u32 counts into u64 offsets (offsets[n] = total).
void launch_scan_u32(const uint32_t* in, uint64_t* out, int64_t n, uint64_t* scratch, cudaStream_t s);
size_t scan_scratch_words(int64_t n);

// Projection: evaluate program `prog` for output row i = row idx[i] (or i) of the source.
void launch_project(const PipeArgs& P, Prog prog, int out_type, void* out, uint32_t* valid, cudaStream_t s);
void launch_hash_columns(const PipeArgs& P, int ncols, const uint64_t* const* dict_hash, uint64_t* out,
                         cudaStream_t s);

// Join build: insert rows 0..n of the build batch.
void launch_join_insert(const PipeArgs& P, const KeyLayout& L, TableView t, uint32_t* next, uint32_t* dup_flag,
                        int64_t n, cudaStream_t s);
// Occupied slots of a table (distinct keys).
void launch_count_slots(TableView t, unsigned long long* out, cudaStream_t s);
// Standalone probe: per-row match counts, then pair output.
void launch_probe_count(const PipeArgs& P, uint32_t* counts, cudaStream_t s);
void launch_probe_write(const PipeArgs& P, const uint64_t* offsets, uint32_t* pi, uint32_t* bi, cudaStream_t s);

// Canonical ids of a plain UTF8 column (equal strings -> the same row id).
void launch_strid(const uint32_t* off, const uint8_t* bytes, const uint64_t* valid, int64_t n, TableView t,
                  uint32_t* canon, uint32_t* err, cudaStream_t s);

// Gathers.
// dst row i = src row idx[i]; width is 1, 4 or a multiple of 8 bytes
void launch_gather_fixed(const void* src, int width, const uint32_t* idx, int64_t k, void* dst, cudaStream_t s);
void launch_gather_valid(const uint64_t* src, const uint32_t* idx, int64_t k, uint32_t* dst, cudaStream_t s);
void launch_utf8_lengths(const uint32_t* off, const uint32_t* idx, int64_t k, uint32_t* len, cudaStream_t s);
void launch_utf8_copy(const uint32_t* off, const uint8_t* bytes, const uint32_t* idx, int64_t k,
                      const uint64_t* dst_off, uint8_t* dst, cudaStream_t s);
void launch_u64_to_u32(const uint64_t* in, uint32_t* out, int64_t n, cudaStream_t s);

// Top-N: each CTA sorts a chunk of candidate rows and keeps the best k.
// Dense join index: key range of a one-column integer build key (mm[0] = min, mm[1] = max,
// initialized to ~0 / 0), the insert, and the count of distinct keys.
void launch_key_range(const void* data, int dt, const uint64_t* valid, int64_t n, unsigned long long* mm, cudaStream_t s);
// Keys outside [dmin, dmin + drange) are skipped and set bit 0 of *range_err (when given).
void launch_dense_insert(const void* data, int dt, const uint64_t* valid, int64_t n, uint64_t dmin, uint64_t drange,
                         uint32_t* dense, uint32_t* next, uint32_t* dup_flag, uint32_t* range_err, cudaStream_t s);
void launch_count_dense(const uint32_t* dense, uint64_t n, unsigned long long* out, cudaStream_t s);
// bits[i / 32] bit i % 32 = (dense[i] != kNone), for i < n.
void launch_dense_bits(const uint32_t* dense, uint64_t n, uint32_t* bits, cudaStream_t s);
void launch_topn_chunk(const SortDev& S, const uint32_t* in, int64_t n, int k, uint32_t* out, cudaStream_t s);

// Full ORDER BY: one 64-bit word of the composite sort key per row (k_sort_words), the word's
// eight byte histograms (hist8: 8 x 256 u64, zeroed), and per non-trivial byte a stable radix
// pass: per-block digit counts (digit-major), their exclusive scan `offs`, the scatter.
enum SortWordKind : int32_t { SW_VALUE = 0, SW_NULL_FLAG = 1, SW_CHUNK = 2, SW_LENGTH = 3, SW_RANK = 4 };
struct SortWord {
    DCol col;
    int32_t what;          // SortWordKind
    int32_t chunk;         // SW_CHUNK: bytes [8 * chunk, 8 * chunk + 8) of the string, big-endian
    int32_t desc;          // descending key: the word is complemented (not the NULL flag)
    int32_t nulls_first;
    const uint32_t* rank;  // SW_RANK: rank of each dictionary code (dict_len + 1 entries)
};
constexpr int kRadixRows = 1024;
int radix_blocks(int64_t n);
void launch_sort_words(const SortWord& w, const uint32_t* perm, int64_t n, uint64_t* out, cudaStream_t s);
void launch_radix_hist8(const uint64_t* keys, int64_t n, unsigned long long* hist, cudaStream_t s);
void launch_radix_count(const uint64_t* keys, int64_t n, int shift, uint32_t* counts, cudaStream_t s);
void launch_radix_scatter(const uint64_t* keys_in, const uint32_t* perm_in, int64_t n, int shift, const uint64_t* offs,
                          uint64_t* keys_out, uint32_t* perm_out, cudaStream_t s);
void launch_max_strlen(const uint32_t* off, int64_t n, unsigned int* out, cudaStream_t s);
void launch_iota_u32(uint32_t* out, int64_t n, cudaStream_t s);  // out[i] = i
// Top-k for k <= kTopNWarpMax: each CTA writes its best k rows (sorted) to out[block * k ..].
constexpr int kTopNWarpMax = 32;
int topn_warp_blocks(int64_t n);
// With final_out, `cand` (blocks * k entries of topn_entry_bytes()) and `done` (16 zeroed
// bytes: the finished-CTA counter and the launch's shared top-k threshold), the last CTA merges
// every CTA's candidates into final_out[0 .. k): one launch.
size_t topn_entry_bytes();
// n_dev (optional): a device-side row count (at most n) read by the kernel.  Returns the
// kernels launched.
int launch_topn_warp(const SortDev& S, int64_t n, int k, int blocks, uint32_t* out, void* cand, unsigned int* done,
                     uint32_t* final_out, cudaStream_t s, const uint64_t* n_dev = nullptr);

// String MIN/MAX states of groups [0, ngroups): new ranks from `rank` for the packed words at
// the listed block offsets (the rank table changed when new strings were interned).
struct RerankOffs {
    int n;
    int32_t off[kMaxAggs];
};
void launch_str_rerank(uint64_t* acc, int stride, uint32_t ngroups, const RerankOffs& R, const uint32_t* rank,
                       cudaStream_t s);

// Prepared-query checks (one thread each): *guard |= bit when the 4- or 8-byte value at p
// differs from v (op 0) or is below v (op 1); a u32 group counter as a u64 row count capped at
// cap.
void launch_plan_check(const void* p, int width, int op, uint64_t v, uint32_t bit, uint32_t* guard, cudaStream_t s);
void launch_plan_count(const uint32_t* count, uint64_t cap, uint64_t* out, cudaStream_t s);
// The result of a replayed top-k (k <= 32): its row ids checked against the device row count
// (an id past it reads row 0 and sets `bit`; n != k when `exact`, else n < k, sets `rows_bit`),
// then k values (1-, 4- or 8-byte) and the validity word of each column gathered.
constexpr int kMaxResultCols = 16;
struct ResultCols {
    int ncols;
    int width[kMaxResultCols];
    const void* src[kMaxResultCols];
    const uint64_t* sval[kMaxResultCols];  // nullptr: no validity
    void* dst[kMaxResultCols];
    uint32_t* dval[kMaxResultCols];        // nullptr: no validity; else the first u32 word
};
void launch_plan_result(const uint32_t* rows, int k, const uint64_t* n_dev, uint64_t cap, int exact, uint32_t bit,
                        uint32_t rows_bit, uint32_t* guard, const ResultCols& G, cudaStream_t s);

// ---- static scratch of ml_gpu_filter_static ----------------------------------------------
// One file-scope device array per device holds every temporary of the no-allocation filter:
// error word, program, arena, per-batch dictionary tables, flag words, block counts, scan.
constexpr int64_t kStaticFilterMaxRows = 1 << 24;  // rows (or selected input rows) per call
constexpr size_t kStaticAlign = 256;
constexpr size_t kStaticErrOff = 0;
constexpr size_t kStaticProgOff = 256;
constexpr size_t kStaticProgBytes = 64 << 10;       // 2048 instructions
constexpr size_t kStaticArenaOff = kStaticProgOff + kStaticProgBytes;
constexpr size_t kStaticArenaBytes = 64 << 10;      // literals, patterns, IN lists
constexpr size_t kStaticTablesOff = kStaticArenaOff + kStaticArenaBytes;
constexpr size_t kStaticTablesBytes = 512 << 10;    // dictionary id maps and predicate tables
constexpr size_t kStaticBitsOff = kStaticTablesOff + kStaticTablesBytes;
constexpr size_t kStaticBitsBytes = (size_t)kStaticFilterMaxRows / 8;
constexpr size_t kStaticCountsOff = kStaticBitsOff + kStaticBitsBytes;
constexpr size_t kStaticCountsBytes = 64 << 10;     // u32 per 2048-row block
constexpr size_t kStaticOffsetsOff = kStaticCountsOff + kStaticCountsBytes;
constexpr size_t kStaticOffsetsBytes = 128 << 10;   // u64 per block, + 1
constexpr size_t kStaticScanOff = kStaticOffsetsOff + kStaticOffsetsBytes;
constexpr size_t kStaticScanBytes = 4 << 10;
constexpr size_t kStaticScratchBytes = kStaticScanOff + kStaticScanBytes;  // 2,953,472 bytes
// Device address of the scratch array on the current device (cudaGetSymbolAddress).
void* static_filter_scratch();

// Concatenation helpers
// dst[i] = src[i] - src[0] + base for i in 0..=n
void launch_offsets_rebase(const uint32_t* src, int64_t n, uint32_t base, uint32_t* dst, cudaStream_t s);
// OR the first n validity bits of src (nullptr = all valid) into dst at bit dst_off
void launch_copy_bits(const uint64_t* src, int64_t n, uint64_t* dst, int64_t dst_off, cudaStream_t s);

}  // namespace mlg
