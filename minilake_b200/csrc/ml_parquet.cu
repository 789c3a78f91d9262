// Parquet column-chunk decode on the GPU: what MiniLake's read_column_chunk
// (crates/minilake-storage/src/parquet_reader.rs:215-294) gets from the parquet crate's column
// reader, then its conversions and encode_strings (:176-212).
//
// The host parses the chunk's page headers (Thrift compact protocol, parquet.thrift PageHeader)
// and copies the chunk to the device once.  Then, on the device:
//   1. Snappy pages are decompressed: a header walk per page finds where each of the
//      compressor's independent 64 KB fragments starts, then one thread per fragment decodes it
//      (a page that does not split that way is decoded by one thread);
//   2. every RLE / bit-packed hybrid stream (definition levels, dictionary indices) gets a run
//      table (one thread per stream walks the run headers, counting first, then filling);
//   3. rows are decoded in 8,192-row tiles: definition levels give the validity bits, a block
//      scan of their popcounts gives each row's position among the chunk's present values, and
//      the value comes from its page (PLAIN, or a dictionary index into the dictionary page) with
//      the column's conversion (FLOAT -> f64, DECIMAL -> f64 / 10^scale);
//   4. strings are materialized (NULL rows as "", as the reference does), canonicalized with a
//      device hash table, and dictionary-encoded in order of first occurrence when there are at
//      most clamp(rows / 8, 1, 65,536) distinct values, else kept plain (encode_strings).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

#include "ml_api_common.hpp"
#include "ml_kernels.cuh"
#include "ml_pipeline.hpp"

using namespace mlg;

namespace {

// parquet.thrift: Type, Encoding, PageType, CompressionCodec
enum PqType { PQ_BOOLEAN = 0, PQ_INT32 = 1, PQ_INT64 = 2, PQ_INT96 = 3, PQ_FLOAT = 4, PQ_DOUBLE = 5, PQ_BYTE_ARRAY = 6, PQ_FLBA = 7 };
enum PqEncoding { ENC_PLAIN = 0, ENC_PLAIN_DICTIONARY = 2, ENC_RLE = 3, ENC_BIT_PACKED = 4, ENC_RLE_DICTIONARY = 8 };
enum PqPageType { PAGE_DATA = 0, PAGE_INDEX = 1, PAGE_DICTIONARY = 2, PAGE_DATA_V2 = 3 };

// ---- Thrift compact protocol: just enough to read a PageHeader and skip the rest ------------
struct Compact {
    const uint8_t* p;
    const uint8_t* end;
    uint8_t byte() {
        if (p >= end) raise(ML_ERR_INVALID, "parquet: page header runs past the chunk");
        return *p++;
    }
    uint64_t varint() {
        uint64_t v = 0;
        for (int shift = 0; shift < 64; shift += 7) {
            const uint8_t b = byte();
            v |= (uint64_t)(b & 0x7F) << shift;
            if (!(b & 0x80)) return v;
        }
        raise(ML_ERR_INVALID, "parquet: bad varint in a page header");
    }
    int64_t zigzag() {
        const uint64_t v = varint();
        return (int64_t)(v >> 1) ^ -(int64_t)(v & 1);
    }
    void skip(int type) {
        switch (type) {
            case 1:
            case 2: return;  // bool in the field header
            case 3: byte(); return;
            case 4:
            case 5:
            case 6: varint(); return;
            case 7: need(8); p += 8; return;
            case 8: {
                const uint64_t n = varint();
                need(n);
                p += n;
                return;
            }
            case 9:
            case 10: {
                const uint8_t h = byte();
                uint64_t n = h >> 4;
                if (n == 15) n = varint();
                const int et = h & 15;
                for (uint64_t i = 0; i < n; i++) skip(et == 1 || et == 2 ? 3 : et);  // list bools are bytes
                return;
            }
            case 11: {
                const uint64_t n = varint();
                if (!n) return;
                const uint8_t kv = byte();
                for (uint64_t i = 0; i < n; i++) {
                    skip(kv >> 4 == 1 || kv >> 4 == 2 ? 3 : kv >> 4);
                    skip((kv & 15) == 1 || (kv & 15) == 2 ? 3 : kv & 15);
                }
                return;
            }
            case 12: {
                int16_t last = 0;
                for (;;) {
                    int fid, ft;
                    if (!field(last, fid, ft)) return;
                    skip(ft);
                }
            }
            default: raise(ML_ERR_INVALID, "parquet: unknown Thrift type " + std::to_string(type));
        }
    }
    void need(uint64_t n) {
        if ((uint64_t)(end - p) < n) raise(ML_ERR_INVALID, "parquet: page header runs past the chunk");
    }
    // Next field of a struct: false at its end.  `last` is the previous field id (delta encoding).
    bool field(int16_t& last, int& id, int& type) {
        const uint8_t h = byte();
        if (h == 0) return false;
        type = h & 15;
        const int delta = h >> 4;
        id = delta ? last + delta : (int16_t)zigzag();
        last = (int16_t)id;
        return true;
    }
};

struct Page {
    int type = -1;
    int64_t payload = 0;  // offset of the page's bytes in the chunk
    int32_t compressed = 0, uncompressed = 0;
    int32_t num_values = 0, encoding = 0, def_encoding = ENC_RLE;
    // DATA_PAGE_V2
    int32_t num_nulls = 0, def_bytes = 0, rep_bytes = 0;
    bool v2_compressed = true;
};

void read_data_header(Compact& c, Page& pg) {  // DataPageHeader
    int16_t last = 0;
    int id, t;
    while (c.field(last, id, t)) {
        if (id == 1 && t == 5) pg.num_values = (int32_t)c.zigzag();
        else if (id == 2 && t == 5) pg.encoding = (int32_t)c.zigzag();
        else if (id == 3 && t == 5) pg.def_encoding = (int32_t)c.zigzag();
        else c.skip(t);
    }
}
void read_dict_header(Compact& c, Page& pg) {  // DictionaryPageHeader
    int16_t last = 0;
    int id, t;
    while (c.field(last, id, t)) {
        if (id == 1 && t == 5) pg.num_values = (int32_t)c.zigzag();
        else if (id == 2 && t == 5) pg.encoding = (int32_t)c.zigzag();
        else c.skip(t);
    }
}
void read_v2_header(Compact& c, Page& pg) {  // DataPageHeaderV2
    int16_t last = 0;
    int id, t;
    while (c.field(last, id, t)) {
        if (id == 1 && t == 5) pg.num_values = (int32_t)c.zigzag();
        else if (id == 2 && t == 5) pg.num_nulls = (int32_t)c.zigzag();
        else if (id == 4 && t == 5) pg.encoding = (int32_t)c.zigzag();
        else if (id == 5 && t == 5) pg.def_bytes = (int32_t)c.zigzag();
        else if (id == 6 && t == 5) pg.rep_bytes = (int32_t)c.zigzag();
        else if (id == 7 && (t == 1 || t == 2)) pg.v2_compressed = t == 1;
        else c.skip(t);
    }
}

// Every page of a column chunk (the pages follow each other; a chunk starts with its
// dictionary page when it has one).
std::vector<Page> parse_pages(const uint8_t* chunk, int64_t n) {
    std::vector<Page> pages;
    int64_t pos = 0;
    while (pos < n) {
        Compact c{chunk + pos, chunk + n};
        Page pg;
        int16_t last = 0;
        int id, t;
        while (c.field(last, id, t)) {
            if (id == 1 && t == 5) pg.type = (int)c.zigzag();
            else if (id == 2 && t == 5) pg.uncompressed = (int32_t)c.zigzag();
            else if (id == 3 && t == 5) pg.compressed = (int32_t)c.zigzag();
            else if (id == 5 && t == 12) read_data_header(c, pg);
            else if (id == 7 && t == 12) read_dict_header(c, pg);
            else if (id == 8 && t == 12) read_v2_header(c, pg);
            else c.skip(t);
        }
        pg.payload = c.p - chunk;
        if (pg.compressed < 0 || pg.uncompressed < 0 || pg.payload + pg.compressed > n)
            raise(ML_ERR_INVALID, "parquet: a page runs past the chunk");
        pos = pg.payload + pg.compressed;
        if (pg.type == PAGE_DATA || pg.type == PAGE_DATA_V2 || pg.type == PAGE_DICTIONARY) pages.push_back(pg);
        else if (pg.type != PAGE_INDEX) raise(ML_ERR_UNSUPPORTED, "parquet: page type " + std::to_string(pg.type));
    }
    return pages;
}

}  // namespace

namespace {
constexpr uint32_t PQ_ERR_SNAPPY = 1, PQ_ERR_LAYOUT = 2, PQ_ERR_RUNS = 4, PQ_ERR_VALUES = 8;
constexpr int kPqTile = 8192;  // rows per decode tile: 256 threads x one 32-row validity word

// ---- 1. Snappy (the format's public description: a varint length, then literal and copy
// elements).  The element stream is sequential, but the compressor works on 64 KB fragments of
// its input and no match reaches back past its fragment's start, so a page of N fragments is N
// independent decodes once their starts in the stream are known.
//
// Both passes read the stream through a shared-memory window of kSnapWin bytes and first parse,
// with all 32 lanes, the element header that WOULD start at every byte of the window (its size
// with a literal's bytes, and its output length); following the real chain of elements through
// the window is then one shared-memory load per element for one lane.
//  * the walk (one 4-warp block per page) follows the chain over the whole page, one thread
//    listing each window's element starts through next-element records (two elements per
//    shared-memory round trip), then the block sums the listed elements' output lengths and
//    records where each 64 KB fragment's elements start;
//  * the decode (one warp per fragment) takes the chain 32 elements at a time, one per lane: a
//    prefix sum gives each element's output position, literals are copied in parallel (long ones
//    by the whole warp), and copies run in rounds of those whose source bytes are already written.
//    The fragment is built in shared memory and written out with 16-byte stores;
//  * a page whose elements cross a fragment boundary, or whose copies reach into an earlier
//    fragment, is decoded again by one thread from start to end (the serial pass), which is also
//    the pass that reports a malformed stream.
struct SnapJob {
    const uint8_t* src;
    uint8_t* dst;
    uint32_t src_len, dst_len;
    uint32_t plan;   // the page's plan in the plan buffer: [mode, first element, nfrag + 1 starts]
    uint32_t nfrag;  // 64 KB fragments of its output
};
constexpr uint32_t kSnapFrag = 1u << 16;  // the compressor's fragment
constexpr uint32_t kSnapWin = 2048;       // stream bytes parsed per window
constexpr uint32_t kSnapWinLoad = kSnapWin + 32;  // with room for the last headers' bytes
// plan modes: 0 the length varint is malformed, 1 the serial pass decodes the page, 2 its
// fragments decode in parallel
constexpr uint32_t kSnapSerial = 1, kSnapSplit = 2;
constexpr size_t kSnapFragSmem = kSnapFrag + kSnapWinLoad + kSnapWin * 2 + 32 * 4;

// One element header at s[0..avail): its size h (tag plus length or offset bytes), kind (0
// literal, 1 copy), output length and copy offset; false if it does not fit in `avail`.
__device__ __forceinline__ bool snap_hdr(const uint8_t* s, uint32_t avail, uint32_t& h, uint32_t& kind,
                                         uint32_t& len, uint32_t& off) {
    if (avail == 0) return false;
    const uint32_t tag = s[0], t = tag & 3;
    off = 0;
    if (t == 0) {
        kind = 0;
        len = tag >> 2;
        h = 1;
        if (len >= 60) {
            const uint32_t nb = len - 59;
            if (nb >= avail) return false;
            len = 0;
            for (uint32_t i = 0; i < nb; i++) len |= (uint32_t)s[1 + i] << (8 * i);
            h = 1 + nb;
        }
        len += 1;
        return len != 0 && len <= avail - h;  // 0: a four-byte length of 2^32
    }
    kind = 1;
    if (t == 1) {
        if (avail < 2) return false;
        h = 2;
        len = 4 + ((tag >> 2) & 7);
        off = ((tag >> 5) << 8) | s[1];
    } else {
        const uint32_t nb = t == 2 ? 2 : 4;
        if (avail < 1 + nb) return false;
        h = 1 + nb;
        len = (tag >> 2) + 1;
        for (uint32_t i = 0; i < nb; i++) off |= (uint32_t)s[1 + i] << (8 * i);
    }
    return true;
}

// The warp loads src[base, base + kSnapWinLoad) into `win`, base being the 16-byte boundary at or
// below pos (it may lie before the stream: those bytes are not used), 16 bytes per lane-load,
// stopping at the first boundary at or past `len` (the chunk buffer is padded past its end).
// Returns base (as a stream offset) and the bytes loaded.
__device__ __forceinline__ int64_t snap_load(const uint8_t* src, uint32_t len, uint32_t pos, uint8_t* win,
                                             uint32_t& loaded) {
    const uintptr_t a = (uintptr_t)(src + pos);
    const uint4* v = (const uint4*)(a & ~(uintptr_t)15);
    const int64_t base = (int64_t)pos - (int64_t)(a & 15);
    const uint64_t need = ((uint64_t)((int64_t)len - base) + 15) / 16;
    const uint32_t nvec = (uint32_t)(need < kSnapWinLoad / 16 ? need : kSnapWinLoad / 16);
    const uint32_t lane = threadIdx.x & 31;
    constexpr uint32_t kPer = (kSnapWinLoad / 16 + 31) / 32;
    uint4 r[kPer];
#pragma unroll
    for (uint32_t k = 0; k < kPer; k++)
        if (lane + 32 * k < nvec) r[k] = __ldg(v + lane + 32 * k);
#pragma unroll
    for (uint32_t k = 0; k < kPer; k++)
        if (lane + 32 * k < nvec) ((uint4*)win)[lane + 32 * k] = r[k];
    __syncwarp();
    loaded = 16 * nvec;
    return base;
}

// The record of the element that would start at window offset q (stream offset base + q):
// the step to the next element (header plus a literal's bytes) in bits 0-15 and the output
// length in bits 16-31 (the fragment decode keeps the step); 0 = the header does not parse (or q
// lies before `from`); a step of 0xFFFF = too long for the record: read the header again.
__device__ __forceinline__ uint32_t snap_record(const uint8_t* win, int64_t base, uint32_t q, uint32_t from,
                                                uint32_t end) {
    const int64_t p = base + q;
    if (p < (int64_t)from || p >= (int64_t)end) return 0;
    uint32_t h, kind, len, off;
    if (!snap_hdr(win + q, end - (uint32_t)p, h, kind, len, off)) return 0;
    const uint64_t step = (uint64_t)h + (kind == 0 ? len : 0);
    return step > 0xFFFE ? 0xFFFFu : (uint32_t)step | (len << 16);
}

// One thread's decode of the elements in [pos, end) into dst[out, out_end); copies may not reach
// below `floor`.  The serial pass: source bytes come through the thread's shared-memory window.
struct SnapSrc {
    const uint8_t* src;
    uint32_t len;
    uint8_t* win;
    int64_t wbase = 0, wend = 0;  // the window holds src[wbase, wend) (wbase may be below 0)
    __device__ uint32_t at(uint32_t p) {  // p < len
        if ((int64_t)p < wbase || (int64_t)p >= wend) {
            const uintptr_t a = (uintptr_t)(src + p);
            const uint4* v = (const uint4*)(a & ~(uintptr_t)15);
            const int64_t lead = (int64_t)(a & 15);
            const uint64_t need = ((uint64_t)(len - p) + (uint64_t)lead + 15) / 16;
            const uint32_t nvec = (uint32_t)(need < kSnapWin / 16 ? need : kSnapWin / 16);
            for (uint32_t i = 0; i < nvec; i += 4) {  // 4 loads in flight, then their stores
                uint4 r[4];
#pragma unroll
                for (uint32_t k = 0; k < 4; k++)
                    if (i + k < nvec) r[k] = __ldg(v + i + k);
#pragma unroll
                for (uint32_t k = 0; k < 4; k++)
                    if (i + k < nvec) ((uint4*)win)[i + k] = r[k];
            }
            wbase = (int64_t)p - lead;
            wend = wbase + 16 * (int64_t)nvec;
        }
        return win[(int64_t)p - wbase];
    }
};

__device__ bool snap_decode_serial(SnapSrc& S, uint32_t pos, uint32_t end, uint8_t* dst, uint32_t out_end) {
    uint32_t out = 0;
    while (out < out_end) {
        if (pos >= end) return false;
        uint8_t hb[5];
        const uint32_t avail = end - pos, nh = avail < 5 ? avail : 5;
        for (uint32_t i = 0; i < nh; i++) hb[i] = (uint8_t)S.at(pos + i);
        uint32_t h, kind, len, off;
        if (!snap_hdr(hb, avail, h, kind, len, off) || len > out_end - out) return false;
        pos += h;
        if (kind == 0) {
            for (uint32_t i = 0; i < len; i++) dst[out + i] = (uint8_t)S.at(pos + i);
            pos += len;
        } else {
            if (off == 0 || off > out) return false;
            for (uint32_t i = 0; i < len; i++) dst[out + i] = dst[out + i - off];  // may overlap itself
        }
        out += len;
    }
    return pos == end;
}

// The walk's record for window offset q (stream offset base + q): the window offset of the next
// element if an element started at q (q + its header + a literal's bytes), or kSnapNone when no
// element can start there (the header or the literal runs past `end`, or q lies before `from`).
// Branch-free: the five bytes a header can span are read at once and every form is computed.
constexpr uint32_t kSnapNone = 0xFFFFFFFFu;
__device__ __forceinline__ uint32_t snap_next(const uint8_t* win, int64_t base, uint32_t q, uint32_t from,
                                              uint32_t end) {
    const int64_t p = base + q;
    const int64_t avail = (int64_t)end - p;
    const uint32_t b0 = win[q], b1 = win[q + 1], b2 = win[q + 2], b3 = win[q + 3], b4 = win[q + 4];
    const uint32_t t = b0 & 3, l6 = b0 >> 2;
    const uint32_t nb = l6 >= 60 ? l6 - 59 : 0;  // a literal's length bytes
    const uint32_t ext = b1 | (nb >= 2 ? b2 << 8 : 0u) | (nb >= 3 ? b3 << 16 : 0u) | (nb >= 4 ? b4 << 24 : 0u);
    const uint64_t len = (uint64_t)(nb ? ext : l6) + 1;  // a literal's bytes (up to 2^32)
    const uint64_t step = t == 0 ? 1 + nb + len : t == 1 ? 2 : t == 2 ? 3 : 5;
    const bool ok = p >= (int64_t)from && avail > 0 && (int64_t)step <= avail && step < (1ull << 31);
    return ok ? q + (uint32_t)step : kSnapNone;
}

// The walk, one 4-warp block per page: the page's mode and, for a split page, where each
// fragment's elements start (plan: [mode, first element, nfrag fragment starts, stream end]).
// Per window: the block builds the next-element records and, from them, the element after next;
// one thread follows the chain two elements per shared-memory round trip, listing the element
// starts; then the block reads the listed headers' output lengths, prefix-sums them, records each
// fragment's first element and checks that no element crosses a fragment boundary.  Every loop
// and barrier is block-uniform: its conditions are read from shared memory after a barrier.
constexpr uint32_t kSnapList = kSnapWin / 2 + 1;  // elements in a window (each spans >= 2 bytes)
constexpr int kWalkThreads = 128;
__global__ void __launch_bounds__(kWalkThreads) k_pq_snappy_walk(const SnapJob* jobs, uint32_t* plan) {
    __shared__ __align__(16) uint8_t win[kSnapWinLoad];
    __shared__ uint32_t nxt[kSnapWin], nxt2[kSnapWin];
    __shared__ uint16_t list[kSnapList];
    __shared__ uint32_t olen[kSnapList];
    __shared__ uint32_t wsum[kWalkThreads / 32];
    __shared__ uint32_t sh_m, sh_qe, sh_bad;
    const SnapJob J = jobs[blockIdx.x];
    uint32_t* pl = plan + J.plan;
    const uint32_t tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    uint32_t start = 0, total = 0;
    bool ok = false;
    for (int shift = 0; shift < 35 && start < J.src_len; shift += 7) {  // the uncompressed length
        const uint32_t b = J.src[start++];
        if (shift == 28 && (b & 0x70)) break;  // past 32 bits
        total |= (b & 0x7F) << shift;
        if (!(b & 0x80)) {
            ok = true;
            break;
        }
    }
    uint32_t mode = ok && total == J.dst_len ? kSnapSerial : 0;
    if (tid == 0) pl[1] = start;
    if (mode && J.nfrag >= 1) {
        bool split = true;
        if (J.nfrag > 1) {
            uint32_t pos = start, out = 0;  // the same in every thread
            while (split && out < total) {
                if (pos >= J.src_len) {
                    split = false;
                    break;
                }
                // the window: src[base, base + kSnapWinLoad) from the 16-byte boundary at or below pos
                const uintptr_t a = (uintptr_t)(J.src + pos);
                const uint4* v = (const uint4*)(a & ~(uintptr_t)15);
                const int64_t base = (int64_t)pos - (int64_t)(a & 15);
                const uint64_t need = ((uint64_t)((int64_t)J.src_len - base) + 15) / 16;
                const uint32_t nvec = (uint32_t)(need < kSnapWinLoad / 16 ? need : kSnapWinLoad / 16);
                for (uint32_t i = tid; i < nvec; i += kWalkThreads) ((uint4*)win)[i] = __ldg(v + i);
                __syncthreads();
#pragma unroll 4
                for (uint32_t q = tid; q < kSnapWin; q += kWalkThreads) nxt[q] = snap_next(win, base, q, pos, J.src_len);
                __syncthreads();
#pragma unroll 4
                for (uint32_t q = tid; q < kSnapWin; q += kWalkThreads) {
                    const uint32_t n = nxt[q];
                    nxt2[q] = n < kSnapWin ? nxt[n] : kSnapNone;
                }
                __syncthreads();
                if (tid == 0) {  // the chain through the window, up to the stream's end
                    const int64_t rest = (int64_t)J.src_len - base;
                    const uint32_t qlim = rest < (int64_t)kSnapWin ? (uint32_t)rest : kSnapWin;
                    uint32_t q = (uint32_t)(pos - base), m = 0;
                    while (q < qlim) {
                        const uint32_t n1 = nxt[q], n2 = nxt2[q];
                        list[m++] = (uint16_t)q;
                        if (n1 >= qlim) {
                            q = n1;
                            break;
                        }
                        list[m++] = (uint16_t)n1;
                        q = n2;
                    }
                    sh_m = m;
                    sh_qe = q;
                    sh_bad = 0;
                }
                __syncthreads();
                const uint32_t m = sh_m;
                uint32_t qe = sh_qe;
                // output lengths of the listed elements (a long literal's next position, which its
                // record could not hold, from its header), each thread a consecutive run of them
                const uint32_t per = (m + kWalkThreads - 1) / kWalkThreads, i0 = tid * per, i1 = min(m, i0 + per);
                uint32_t sum = 0;
                bool bad = false;
                for (uint32_t i = i0; i < i1; i++) {
                    const uint32_t q = list[i];
                    const uint32_t p = (uint32_t)(base + q);
                    uint32_t h, kind, len, off;
                    if (!snap_hdr(win + q, J.src_len - p, h, kind, len, off)) {
                        bad = true;
                        len = 0;
                    }
                    olen[i] = len;
                    sum += len;
                    if (i == m - 1) sh_qe = qe == kSnapNone && !bad ? q + h + (kind == 0 ? len : 0) : qe;
                }
                // exclusive prefix of the threads' sums: within the warp, then over the warps
                uint32_t incl = sum;
#pragma unroll
                for (uint32_t d = 1; d < 32; d <<= 1) {
                    const uint32_t t = __shfl_up_sync(~0u, incl, d);
                    if (lane >= d) incl += t;
                }
                if (lane == 31) wsum[warp] = incl;
                __syncthreads();
                uint32_t before = 0, all = 0;
                for (uint32_t w = 0; w < kWalkThreads / 32; w++) {
                    before += w < warp ? wsum[w] : 0;
                    all += wsum[w];
                }
                uint32_t o = out + before + incl - sum;
                for (uint32_t i = i0; i < i1 && !bad; i++) {
                    const uint32_t l = olen[i];
                    if (o > total || l > total - o || (o & (kSnapFrag - 1)) + l > kSnapFrag) {
                        bad = true;  // past the end, or crossing a fragment's end
                        break;
                    }
                    if ((o & (kSnapFrag - 1)) == 0 && o < total) pl[2 + (o >> 16)] = (uint32_t)(base + list[i]);
                    o += l;
                }
                if (bad) atomicOr(&sh_bad, 1u);
                __syncthreads();
                qe = sh_qe;
                const bool stop = sh_bad || qe == kSnapNone || all > total - out;
                __syncthreads();  // sh_* and the window are rewritten by the next window
                if (stop) {
                    split = false;
                    break;
                }
                out += all;
                pos = (uint32_t)(base + qe);
            }
        }
        if (tid == 0) {
            if (J.nfrag == 1) pl[2] = start;
            pl[2 + J.nfrag] = J.src_len;
        }
        if (split) mode = kSnapSplit;
    }
    if (tid == 0) pl[0] = mode;
}

// A literal longer than a lane's share, by the whole warp: aligned 16-byte loads from the stream,
// bytes stored into the fragment (the loads may pass the literal's ends by 15 bytes, inside the
// padded chunk buffer).
__device__ __forceinline__ void snap_warp_copy(const uint8_t* src, uint32_t len, uint8_t* dst) {
    const uintptr_t a = (uintptr_t)src;
    const uint4* v = (const uint4*)(a & ~(uintptr_t)15);
    const int32_t lead = (int32_t)(a & 15);
    const uint32_t nvec = ((uint32_t)lead + len + 15) / 16;
    const uint32_t lane = threadIdx.x & 31;
    auto put = [&](const uint4& r, uint32_t i) {
        const uint32_t w[4] = {r.x, r.y, r.z, r.w};
#pragma unroll
        for (int b = 0; b < 16; b++) {
            const int32_t idx = (int32_t)(16 * i) + b - lead;
            if (idx >= 0 && (uint32_t)idx < len) dst[idx] = (uint8_t)(w[b >> 2] >> (8 * (b & 3)));
        }
    };
    for (uint32_t i = lane; i < nvec; i += 64) {
        const uint4 r0 = __ldg(v + i);
        const bool two = i + 32 < nvec;
        uint4 r1 = r0;
        if (two) r1 = __ldg(v + i + 32);
        put(r0, i);
        if (two) put(r1, i + 32);
    }
}

// One copy element by one lane: o[at, at + len) from o[at - off, ...), the source bytes read as the
// repeating pattern o[at - off, at) (what a byte-by-byte copy of an overlapping match produces), so
// the loads never depend on this copy's stores.
__device__ __forceinline__ void snap_copy(uint8_t* o, uint32_t at, uint32_t off, uint32_t len) {
    const uint8_t* s = o + at - off;
    uint32_t j = 0;
    for (uint32_t i = 0; i < len; i += 8) {
        uint8_t t[8];
#pragma unroll
        for (uint32_t k = 0; k < 8; k++) {
            t[k] = i + k < len ? s[j] : 0;
            j = j + 1 == off ? 0 : j + 1;
        }
#pragma unroll
        for (uint32_t k = 0; k < 8; k++)
            if (i + k < len) o[at + i + k] = t[k];
    }
}

// The decode, one warp per fragment of a split page (frags[i] = {page, fragment}); a fragment that
// does not decode as a unit hands its page to the serial pass.
__global__ void __launch_bounds__(32) k_pq_snappy_frag(const SnapJob* jobs, const uint2* frags, uint32_t* plan) {
    extern __shared__ __align__(16) uint8_t snap_smem[];
    uint8_t* o = snap_smem;                                    // the fragment, kSnapFrag bytes
    uint8_t* win = o + kSnapFrag;                              // the stream window
    uint16_t* rec = (uint16_t*)(win + kSnapWinLoad);           // steps to the next element
    uint32_t* list = (uint32_t*)(rec + kSnapWin);              // a batch's element starts
    const uint2 f = frags[blockIdx.x];
    const SnapJob J = jobs[f.x];
    uint32_t* pl = plan + J.plan;
    if (pl[0] != kSnapSplit) return;
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t o0 = f.y * kSnapFrag, n = min(J.dst_len - o0, kSnapFrag);
    uint32_t pos = pl[2 + f.y], out = 0;
    const uint32_t end = pl[3 + f.y];
    bool ok = true;
    while (ok && out < n) {
        if (pos >= end) {
            ok = false;
            break;
        }
        uint32_t loaded;
        const int64_t base = snap_load(J.src, end, pos, win, loaded);
        for (uint32_t q = lane; q < kSnapWin; q += 32) rec[q] = (uint16_t)(snap_record(win, base, q, pos, end) & 0xFFFF);
        __syncwarp();
        uint32_t q0 = (uint32_t)(pos - base);
        while (ok && out < n && q0 < kSnapWin && base + q0 < end) {
            uint32_t m = 0;
            if (lane == 0) {  // up to 32 elements of the chain
                uint32_t q = q0;
                while (m < 32 && q < kSnapWin && base + q < end) {
                    const uint32_t r = rec[q];
                    list[m++] = q;
                    if (r == 0 || r == 0xFFFF) break;  // its lane reads the header (or finds it malformed)
                    q += r;
                }
            }
            m = __shfl_sync(~0u, m, 0);
            __syncwarp();
            uint32_t h = 0, kind = 0, len = 0, off = 0, q = 0;
            bool good = true;
            if (lane < m) {
                q = list[lane];
                good = snap_hdr(win + q, end - (uint32_t)(base + q), h, kind, len, off);
            }
            // output positions: the exclusive prefix sum of the lengths
            const uint32_t x = lane < m && good ? len : 0;
            uint32_t incl = x;
#pragma unroll
            for (uint32_t d = 1; d < 32; d <<= 1) {
                const uint32_t t = __shfl_up_sync(~0u, incl, d);
                if (lane >= d) incl += t;
            }
            const uint32_t my = out + incl - x;
            if (lane < m && good) {
                if (my > n || len > n - my) good = false;
                else if (kind == 1 && (off == 0 || off > my)) good = false;  // before the fragment
            }
            if (__any_sync(~0u, lane < m && !good)) {
                ok = false;
                break;
            }
            // literals: short ones by their lane, long ones by the whole warp
            const uint32_t lit = (uint32_t)(base + q) + h;  // stream offset of a literal's bytes
            const bool is_lit = lane < m && kind == 0;
            if (is_lit && len <= 32) {
                if ((int64_t)lit - base + len <= (int64_t)loaded) {
                    const uint8_t* s = win + (lit - base);
                    for (uint32_t i = 0; i < len; i++) o[my + i] = s[i];
                } else {
                    for (uint32_t i = 0; i < len; i++) o[my + i] = __ldg(J.src + lit + i);
                }
            }
            uint32_t longs = __ballot_sync(~0u, is_lit && len > 32);
            while (longs) {
                const uint32_t l = __ffs(longs) - 1;
                longs &= longs - 1;
                const uint32_t ls = __shfl_sync(~0u, lit, l), ll = __shfl_sync(~0u, len, l), lo = __shfl_sync(~0u, my, l);
                snap_warp_copy(J.src + ls, ll, o + lo);
            }
            __syncwarp();
            // copies in rounds: a copy runs once every byte it reads is written, i.e. its source
            // ends at or before the output position of the earliest copy still waiting
            uint32_t pend = __ballot_sync(~0u, lane < m && kind == 1);
            const uint32_t need = kind == 1 ? (off >= len ? my - off + len : my) : 0;
            while (pend) {
                const uint32_t lim = __shfl_sync(~0u, my, __ffs(pend) - 1);
                const uint32_t ready = pend & __ballot_sync(~0u, need <= lim);
                if ((ready >> lane) & 1) snap_copy(o, my, off, len);
                __syncwarp();
                pend &= ~ready;
            }
            // the next batch starts after the last element
            const uint32_t nxt = (uint32_t)(base + q) + h + (kind == 0 ? len : 0);
            pos = __shfl_sync(~0u, nxt, m - 1);
            out += __shfl_sync(~0u, incl, 31);
            q0 = (uint32_t)(pos - base);
        }
        __syncwarp();  // the window and the records are reused
    }
    if (ok && pos != end) ok = false;
    if (!ok) {
        if (lane == 0) atomicExch(pl, kSnapSerial);
        return;
    }
    __syncwarp();
    uint8_t* d = J.dst + o0;
    if (((uintptr_t)d & 15) == 0) {
        const uint32_t nv = n / 16;
        for (uint32_t i = lane; i < nv; i += 32) ((uint4*)d)[i] = ((const uint4*)o)[i];
        for (uint32_t i = 16 * nv + lane; i < n; i += 32) d[i] = o[i];
    } else {
        for (uint32_t i = lane; i < n; i += 32) d[i] = o[i];
    }
}

// The serial pass, one thread per page not decoded by fragments: it decodes the page from start
// to end or reports it malformed.
__global__ void __launch_bounds__(32) k_pq_snappy_serial(const SnapJob* jobs, const uint32_t* plan, uint32_t* err) {
    __shared__ __align__(16) uint8_t win[kSnapWin + 16];
    if (threadIdx.x) return;
    const SnapJob J = jobs[blockIdx.x];
    const uint32_t* pl = plan + J.plan;
    const uint32_t mode = pl[0];
    if (mode == kSnapSplit) return;
    SnapSrc S{J.src, J.src_len, win};
    if (mode != kSnapSerial || !snap_decode_serial(S, pl[1], J.src_len, J.dst, J.dst_len)) atomicOr(err, PQ_ERR_SNAPPY);
}

// ---- 2. page layout and RLE / bit-packed hybrid run tables -----------------------------------
struct Run {
    uint32_t first, count;  // value index (in the stream) of the run's first value; its values
    uint32_t value;         // RLE run: the repeated value; bit-packed run: its byte offset
    uint32_t packed;
};

struct PageDev {
    const uint8_t* data;  // the page's uncompressed payload
    uint32_t len;
    int32_t v2, def_bytes, rep_bytes;  // DATA_PAGE_V2: level byte lengths
    int32_t encoding;
    int64_t row0;
    uint32_t nrows;
    // filled by k_pq_layout
    const uint8_t* levels;
    uint32_t levels_len;
    const uint8_t* values;
    uint32_t values_len;
    int32_t idx_width;  // dictionary-index (or RLE boolean) bit width; -1: PLAIN values
    // run tables (levels, then indices), filled by k_pq_runs
    uint64_t lv_run0, ix_run0;
    uint32_t lv_nruns, ix_nruns;
    uint64_t valid0;  // present values of the chunk before this page's first row
};

__device__ uint32_t le32(const uint8_t* p) { return p[0] | (p[1] << 8) | (p[2] << 16) | ((uint32_t)p[3] << 24); }

__global__ void k_pq_layout(PageDev* pages, int npages, int max_def, uint32_t* err) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= npages) return;
    PageDev& p = pages[i];
    uint32_t pos = 0;
    p.levels = nullptr;
    p.levels_len = 0;
    if (p.v2) {
        pos = (uint32_t)p.rep_bytes + (uint32_t)p.def_bytes;
        if (max_def > 0) {
            p.levels = p.data + p.rep_bytes;
            p.levels_len = (uint32_t)p.def_bytes;
        }
    } else if (max_def > 0) {
        if (p.len < 4 || le32(p.data) > p.len - 4) {
            atomicOr(err, PQ_ERR_LAYOUT);
            p.values_len = 0;
            p.idx_width = -1;
            return;
        }
        p.levels = p.data + 4;
        p.levels_len = le32(p.data);
        pos = 4 + p.levels_len;
    }
    if (pos > p.len) {
        atomicOr(err, PQ_ERR_LAYOUT);
        pos = p.len;
    }
    p.values = p.data + pos;
    p.values_len = p.len - pos;
    p.idx_width = -1;
    if (p.encoding == ENC_RLE_DICTIONARY || p.encoding == ENC_PLAIN_DICTIONARY) {
        if (p.values_len < 1 || p.values[0] > 32) {
            atomicOr(err, PQ_ERR_LAYOUT);
            return;
        }
        p.idx_width = p.values[0];
        p.values += 1;
        p.values_len -= 1;
    } else if (p.encoding == ENC_RLE) {  // RLE booleans: a 4-byte length, then the hybrid stream
        if (p.values_len < 4 || le32(p.values) > p.values_len - 4) {
            atomicOr(err, PQ_ERR_LAYOUT);
            return;
        }
        p.values_len = le32(p.values);
        p.values += 4;
        p.idx_width = 1;
    }
}

// Walk a hybrid stream of `n` values with bit width `bw`: count its runs (runs == nullptr) or
// write them.  Returns the number of runs, or -1 when the stream is malformed.
__device__ int64_t rle_walk(const uint8_t* s, uint32_t len, uint32_t n, int bw, Run* runs) {
    uint32_t pos = 0, got = 0;
    int64_t k = 0;
    const uint32_t vbytes = (bw + 7) / 8;
    while (got < n) {
        uint64_t h = 0;
        for (int shift = 0;; shift += 7) {
            if (pos >= len || shift > 35) return -1;
            const uint8_t b = s[pos++];
            h |= (uint64_t)(b & 0x7F) << shift;
            if (!(b & 0x80)) break;
        }
        Run r{got, 0, 0, 0};
        if (h & 1) {  // bit-packed: (h >> 1) groups of 8 values (none: malformed, every run holds a value)
            const uint64_t vals = (h >> 1) * 8, bytes = (h >> 1) * (uint64_t)bw;
            if (vals == 0 || pos + bytes > len) return -1;
            r.count = (uint32_t)(uint32_t)(vals < (uint64_t)(n - got) ? vals : (uint64_t)(n - got));
            r.value = pos;
            r.packed = 1;
            pos += (uint32_t)bytes;
        } else {
            r.count = (uint32_t)((h >> 1) < (uint64_t)(n - got) ? (h >> 1) : (uint64_t)(n - got));
            if (pos + vbytes > len || r.count == 0) return -1;
            for (uint32_t b = 0; b < vbytes; b++) r.value |= (uint32_t)s[pos + b] << (8 * b);
            pos += vbytes;
        }
        if (runs) runs[k] = r;
        k++;
        got += r.count;
    }
    return k;
}

// One thread per page and stream (`which` 0: definition levels, one per row; 1: dictionary
// indices or RLE booleans, one per present value, `nvalues`).  With runs == nullptr it counts
// the runs into the page; else it writes them from the page's run offset.
__global__ void k_pq_runs(PageDev* pages, int npages, int which, int level_width, const uint32_t* nvalues, Run* runs,
                          uint32_t* err) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= npages) return;
    PageDev& p = pages[i];
    const bool lv = which == 0;
    const uint8_t* s = lv ? p.levels : p.values;
    const uint32_t len = lv ? p.levels_len : p.values_len;
    const int bw = lv ? level_width : p.idx_width;
    const uint32_t n = lv ? p.nrows : nvalues[i];
    uint32_t& nruns = lv ? p.lv_nruns : p.ix_nruns;
    Run* out = runs ? runs + (lv ? p.lv_run0 : p.ix_run0) : nullptr;
    if (!s || bw < 0 || n == 0) {
        nruns = 0;
        return;
    }
    if (bw == 0) {  // every value is 0: one run, no bytes
        if (out) out[0] = Run{0, n, 0, 0};
        nruns = 1;
        return;
    }
    const int64_t k = rle_walk(s, len, n, bw, out);
    if (k < 0) {
        atomicOr(err, PQ_ERR_RUNS);
        nruns = 0;
        return;
    }
    nruns = (uint32_t)k;
}

// Value k of a stream from its run table (k < the stream's value count).
__device__ uint32_t rle_get(const Run* runs, uint32_t nruns, const uint8_t* s, int bw, uint32_t k) {
    uint32_t lo = 0, hi = nruns;
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (runs[mid].first <= k) lo = mid;
        else hi = mid;
    }
    const Run r = runs[lo];
    if (!r.packed) return r.value;
    const uint64_t bit = (uint64_t)(k - r.first) * bw;
    const uint8_t* b = s + r.value + (bit >> 3);
    uint64_t w = 0;
    const int nb = (int)(((bit & 7) + bw + 7) >> 3);
    for (int j = 0; j < nb; j++) w |= (uint64_t)b[j] << (8 * j);
    return (uint32_t)((w >> (bit & 7)) & (bw == 32 ? 0xFFFFFFFFull : ((1ull << bw) - 1)));
}

__device__ int page_of(const PageDev* pages, int npages, int64_t row) {
    int lo = 0, hi = npages;
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (pages[mid].row0 <= row) lo = mid;
        else hi = mid;
    }
    return lo;
}

// ---- 3. validity: definition level == max_def, one thread per 32-row word ----------------------
__global__ void k_pq_valid(const PageDev* pages, int npages, const Run* runs, int max_def, int level_width, int64_t nrows,
                           uint32_t* valid, uint32_t* tile_counts) {
    const int64_t w = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t bits = 0;
    if (w * 32 < nrows) {
        int p = page_of(pages, npages, w * 32);
        for (int j = 0; j < 32; j++) {
            const int64_t r = w * 32 + j;
            if (r >= nrows) break;
            while (p + 1 < npages && pages[p + 1].row0 <= r) p++;
            const PageDev& pg = pages[p];
            const uint32_t k = (uint32_t)(r - pg.row0);
            bool v = true;
            if (max_def > 0) {
                v = k < pg.nrows && pg.lv_nruns &&
                    rle_get(runs + pg.lv_run0, pg.lv_nruns, pg.levels, level_width, k) == (uint32_t)max_def;
            }
            bits |= (uint32_t)v << j;
        }
        valid[w] = bits;
    }
    // present values per 8,192-row tile
    const int c = __popc(bits);
    __shared__ uint32_t sum;
    if (threadIdx.x == 0) sum = 0;
    __syncthreads();
    if (c) atomicAdd(&sum, (uint32_t)c);
    __syncthreads();
    if (threadIdx.x == 0) tile_counts[blockIdx.x] = sum;
}

// Present values before each page's first row, and each page's present values.
__global__ void k_pq_page_valid(PageDev* pages, int npages, const uint32_t* valid, const uint64_t* tile_offs,
                                int64_t nrows, uint32_t* nvalues) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i > npages) return;
    auto rank = [&](int64_t row) -> uint64_t {  // present values in rows [0, row)
        if (row >= nrows) return tile_offs[(nrows + kPqTile - 1) / kPqTile];
        const int64_t t = row / kPqTile;
        uint64_t c = tile_offs[t];
        for (int64_t w = t * (kPqTile / 32); w < row / 32; w++) c += __popc(valid[w]);
        if (row & 31) c += __popc(valid[row / 32] & ((1u << (row & 31)) - 1u));
        return c;
    };
    if (i < npages) {
        pages[i].valid0 = rank(pages[i].row0);
        nvalues[i] = (uint32_t)(rank(pages[i].row0 + pages[i].nrows) - pages[i].valid0);
    }
}
}  // namespace

namespace {
// ---- 4. values --------------------------------------------------------------------------------
// Conversion (parquet_reader.rs:31-56), the header's ML_PQ_CONV_* values.
enum Conv { CV_BOOL = 0, CV_INT32, CV_DATE, CV_INT64, CV_FLOAT, CV_DOUBLE, CV_UTF8, CV_DEC_I32, CV_DEC_I64, CV_DEC_BYTES };

struct DecodeArgs {
    const PageDev* pages;
    int npages;
    const Run* runs;
    const uint32_t* valid;
    const uint64_t* tile_offs;
    int64_t nrows;
    int ptype, conv, type_length;
    double div;  // 10^scale for decimals
    // the dictionary page: fixed-width values, or byte-array entries (pointer + length)
    const uint8_t* dict;
    uint32_t dict_n;
    const uint8_t* const* dict_ptr;
    const uint32_t* dict_len;
    // PLAIN byte arrays of the data pages, by the value's index among the chunk's present values
    const uint8_t* const* vptr;
    const uint32_t* vlen;
    void* out;                // fixed-width output (the column's type)
    const uint8_t** str_ptr;  // strings (and byte-array decimals go through vptr)
    uint32_t* str_len;
    uint32_t* err;
};

// A big-endian two's complement integer of up to 16 bytes (be_i128, parquet_reader.rs:154-166)
// as the nearest f64 (ties to even).
__device__ double be_int_to_f64(const uint8_t* b, uint32_t n) {
    uint64_t hi = (n && (b[0] & 0x80)) ? ~0ull : 0ull, lo = hi;
    for (uint32_t i = 0; i < n && i < 16; i++) {
        hi = (hi << 8) | (lo >> 56);
        lo = (lo << 8) | b[i];
    }
    const bool neg = (int64_t)hi < 0;
    if (neg) {  // magnitude (two's complement negation)
        lo = ~lo + 1;
        hi = ~hi + (lo == 0 ? 1 : 0);
    }
    double m;
    if (hi == 0) {
        m = __ull2double_rn(lo);
    } else {
        const int lz = __clzll(hi);
        const uint64_t h = lz ? (hi << lz) | (lo >> (64 - lz)) : hi;  // top bit at 63
        const uint64_t l = lo << lz;
        uint64_t mant = h >> 11;  // 53 bits
        const bool guard = (h >> 10) & 1, sticky = (h & 0x3FF) || l;
        if (guard && (sticky || (mant & 1))) mant++;
        int e = 127 - lz - 52;
        if (mant >> 53) {
            mant >>= 1;
            e++;
        }
        m = ldexp((double)mant, e);
    }
    return neg ? -m : m;
}

__device__ uint64_t load_le(const uint8_t* p, int w) {
    uint64_t v = 0;
    for (int i = 0; i < w; i++) v |= (uint64_t)p[i] << (8 * i);
    return v;
}

__global__ void __launch_bounds__(256) k_pq_values(const __grid_constant__ DecodeArgs D) {
    __shared__ uint32_t words[256], pre[256];
    const int t = threadIdx.x;
    const int64_t w0 = (int64_t)blockIdx.x * 256;
    const uint32_t word = (w0 + t) * 32 < D.nrows ? D.valid[w0 + t] : 0u;
    words[t] = word;
    // exclusive scan of the words' popcounts
    uint32_t c = __popc(word), x = c;
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, x, o);
        if ((t & 31) >= o) x += y;
    }
    __shared__ uint32_t warp_sum[8];
    if ((t & 31) == 31) warp_sum[t >> 5] = x;
    __syncthreads();
    uint32_t wbase = 0;
    for (int i = 0; i < (t >> 5); i++) wbase += warp_sum[i];
    pre[t] = wbase + x - c;
    __syncthreads();
    const uint64_t base = D.tile_offs[blockIdx.x];
    int p = -1;
    for (int j = 0; j < 32; j++) {
        const int64_t r = (int64_t)blockIdx.x * kPqTile + j * 256 + t;
        if (r >= D.nrows) break;
        const int lw = (int)((r >> 5) - w0);
        const uint32_t bits = words[lw];
        const bool v = (bits >> (r & 31)) & 1;
        const int vw = D.conv == CV_BOOL ? 1 : (D.conv == CV_INT32 || D.conv == CV_DATE) ? 4 : 8;
        if (!v) {
            if (D.conv == CV_UTF8) {
                D.str_ptr[r] = nullptr;
                D.str_len[r] = 0;
            } else if (vw == 1) {
                ((uint8_t*)D.out)[r] = 0;
            } else if (vw == 4) {
                ((uint32_t*)D.out)[r] = 0;
            } else {
                ((uint64_t*)D.out)[r] = 0;
            }
            continue;
        }
        const uint64_t d = base + pre[lw] + __popc(bits & ((1u << (r & 31)) - 1u));  // among present values
        if (p < 0 || !(D.pages[p].row0 <= r && (p + 1 >= D.npages || D.pages[p + 1].row0 > r))) p = page_of(D.pages, D.npages, r);
        const PageDev& pg = D.pages[p];
        const uint32_t k = (uint32_t)(d - pg.valid0);
        const bool dict = pg.encoding == ENC_RLE_DICTIONARY || pg.encoding == ENC_PLAIN_DICTIONARY;
        const bool rle_bool = pg.encoding == ENC_RLE;
        uint32_t idx = 0;
        if (dict || rle_bool) {
            if (!pg.ix_nruns) {
                atomicOr(D.err, PQ_ERR_VALUES);
                continue;
            }
            idx = rle_get(D.runs + pg.ix_run0, pg.ix_nruns, pg.values, pg.idx_width, k);
            if (dict && idx >= D.dict_n) {
                atomicOr(D.err, PQ_ERR_VALUES);
                continue;
            }
        }
        // the value's bytes: a byte array (pointer, length) or a fixed-width slot
        const uint8_t* src = nullptr;
        uint32_t slen = 0;
        const int pw = D.ptype == PQ_INT32 || D.ptype == PQ_FLOAT ? 4 : D.ptype == PQ_FLBA ? D.type_length : 8;
        if (D.ptype == PQ_BYTE_ARRAY) {
            if (dict) {
                src = D.dict_ptr[idx];
                slen = D.dict_len[idx];
            } else {
                src = D.vptr[d];
                slen = D.vlen[d];
            }
        } else if (D.ptype != PQ_BOOLEAN) {
            if (dict) {
                src = D.dict + (uint64_t)idx * pw;
            } else {
                if ((uint64_t)(k + 1) * pw > pg.values_len) {
                    atomicOr(D.err, PQ_ERR_VALUES);
                    continue;
                }
                src = pg.values + (uint64_t)k * pw;
            }
            slen = pw;
        }
        switch (D.conv) {
            case CV_BOOL: {
                uint32_t b;
                if (rle_bool) {
                    b = idx;
                } else if (dict) {
                    b = D.dict[idx >> 3] >> (idx & 7);
                } else {
                    if ((k >> 3) >= pg.values_len) {
                        atomicOr(D.err, PQ_ERR_VALUES);
                        continue;
                    }
                    b = pg.values[k >> 3] >> (k & 7);
                }
                ((uint8_t*)D.out)[r] = (uint8_t)(b & 1);
                break;
            }
            case CV_INT32:
            case CV_DATE: ((uint32_t*)D.out)[r] = (uint32_t)load_le(src, 4); break;
            case CV_INT64:
            case CV_DOUBLE: ((uint64_t*)D.out)[r] = load_le(src, 8); break;
            case CV_FLOAT: ((double*)D.out)[r] = (double)__uint_as_float((uint32_t)load_le(src, 4)); break;
            case CV_DEC_I32: ((double*)D.out)[r] = __ddiv_rn((double)(int32_t)load_le(src, 4), D.div); break;
            case CV_DEC_I64: ((double*)D.out)[r] = __ddiv_rn(__ll2double_rn((long long)load_le(src, 8)), D.div); break;
            case CV_DEC_BYTES: ((double*)D.out)[r] = __ddiv_rn(be_int_to_f64(src, slen), D.div); break;
            case CV_UTF8:
                D.str_ptr[r] = src;
                D.str_len[r] = slen;
                break;
        }
    }
}

// PLAIN byte arrays (a 4-byte length, then the bytes) of the data pages, one thread per page:
// pointer and length of each value by its index among the chunk's present values.  For the
// dictionary page (dict != nullptr) the entries instead.
__global__ void k_pq_byte_arrays(const PageDev* pages, int npages, const uint32_t* nvalues, const uint8_t** ptr,
                                 uint32_t* len, const uint8_t* dict, uint32_t dict_len, uint32_t dict_n,
                                 const uint8_t** dptr, uint32_t* dlen, uint32_t* err) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const uint8_t* s;
    uint32_t n, slen;
    const uint8_t** op;
    uint32_t* ol;
    if (i < npages) {
        const PageDev& p = pages[i];
        if (p.encoding != ENC_PLAIN) return;
        s = p.values;
        slen = p.values_len;
        n = nvalues[i];
        op = ptr + p.valid0;
        ol = len + p.valid0;
    } else if (i == npages && dict) {
        s = dict;
        slen = dict_len;
        n = dict_n;
        op = dptr;
        ol = dlen;
    } else {
        return;
    }
    uint32_t pos = 0;
    for (uint32_t k = 0; k < n; k++) {
        if (pos + 4 > slen || le32(s + pos) > slen - pos - 4) {
            atomicOr(err, PQ_ERR_VALUES);
            for (; k < n; k++) op[k] = s, ol[k] = 0;
            return;
        }
        const uint32_t l = le32(s + pos);
        op[k] = s + pos + 4;
        ol[k] = l;
        pos += 4 + l;
    }
}

// ---- 5. strings: materialize, then encode_strings' dictionary decision ----------------------
__global__ void k_pq_str_copy(const uint8_t* const* ptr, const uint32_t* len, const uint64_t* offs, int64_t n,
                              uint32_t* off32, uint8_t* bytes) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < n; r += stride) {
        const uint64_t o = offs[r];
        off32[r] = (uint32_t)o;
        const uint8_t* s = ptr[r];
        for (uint32_t b = 0; b < len[r]; b++) bytes[o + b] = s[b];
        if (r == n - 1) off32[n] = (uint32_t)offs[n];
    }
}
__global__ void k_pq_first(const uint32_t* canon, int64_t n, uint32_t* first) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < n; r += stride)
        atomicMin(first + canon[r], (uint32_t)r);
}
// bits: rows that are the first occurrence of their string; block counts for the compaction
__global__ void k_pq_first_flags(const uint32_t* canon, const uint32_t* first, int64_t n, uint32_t* bits, uint32_t* counts,
                                 int rows_per_block) {
    const int64_t b0 = (int64_t)blockIdx.x * rows_per_block;
    uint32_t c = 0;
    for (int64_t w = b0 / 32 + threadIdx.x; w * 32 < (n < b0 + rows_per_block ? n : b0 + rows_per_block); w += blockDim.x) {
        uint32_t x = 0;
        for (int j = 0; j < 32; j++) {
            const int64_t r = w * 32 + j;
            if (r < n && first[canon[r]] == (uint32_t)r) x |= 1u << j;
        }
        bits[w] = x;
        c += __popc(x);
    }
    __shared__ uint32_t sum;
    if (threadIdx.x == 0) sum = 0;
    __syncthreads();
    if (c) atomicAdd(&sum, c);
    __syncthreads();
    if (threadIdx.x == 0) counts[blockIdx.x] = sum;
}
__global__ void k_pq_codes(const uint32_t* list, uint32_t ndistinct, const uint32_t* canon, uint32_t* code_of) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < ndistinct; i += stride)
        code_of[canon[list[i]]] = (uint32_t)i;
}
__global__ void k_pq_codes2(const uint32_t* canon, int64_t n, const uint32_t* code_of, uint32_t* codes) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < n; r += stride) codes[r] = code_of[canon[r]];
}
}  // namespace

namespace {
uint64_t pow2_ceil(uint64_t x) {
    uint64_t p = 1;
    while (p < x) p <<= 1;
    return p;
}
int grid_of(int64_t n, int threads = 256) { return (int)std::max<int64_t>(1, std::min<int64_t>((n + threads - 1) / threads, 148 * 16)); }

// powi as in compiler-rt's __powidf2 (binary exponentiation), which Rust's f64::powi lowers
// to for a run-time exponent: 10f64.powi(scale) (parquet_reader.rs:217).
double powi(double a, int b) {
    const bool recip = b < 0;
    double r = 1;
    for (;;) {
        if (b & 1) r *= a;
        b /= 2;
        if (b == 0) break;
        a *= a;
    }
    return recip ? 1 / r : r;
}

void check_pq(Ctx* ctx, uint32_t e) {
    (void)ctx;
    if (e & PQ_ERR_SNAPPY) raise(ML_ERR_INVALID, "parquet: a Snappy page does not decompress to its stated size");
    if (e & PQ_ERR_LAYOUT) raise(ML_ERR_INVALID, "parquet: a data page's levels or values run past the page");
    if (e & PQ_ERR_RUNS) raise(ML_ERR_INVALID, "parquet: a malformed RLE / bit-packed stream");
    if (e & PQ_ERR_VALUES) raise(ML_ERR_INVALID, "parquet: a value or dictionary index outside its page or dictionary");
    if (e) raise(ML_ERR_INVALID, "parquet: decode error " + std::to_string(e));
}
}  // namespace

extern "C" int ml_gpu_parquet_decode(ml_ctx* ctx, const uint8_t* chunk, int64_t chunk_bytes, int32_t physical_type,
                                     int32_t type_length, int32_t conversion, int32_t scale, int32_t codec,
                                     int64_t num_rows, int32_t max_def, ml_batch** out) {
    API_BEGIN
    HostTimer host_timer_(ctx, "host:parquet_decode");
    REQUIRE(ctx && out && (chunk || chunk_bytes == 0) && chunk_bytes >= 0, "null argument");
    REQUIRE(num_rows >= 0 && num_rows < 0x7FFFFFFFll, "row count out of range");
    REQUIRE(max_def >= 0 && max_def <= 255, "max definition level out of range");
    if (codec != ML_PQ_CODEC_UNCOMPRESSED && codec != ML_PQ_CODEC_SNAPPY)
        raise(ML_ERR_UNSUPPORTED, "parquet: compression codec " + std::to_string(codec));
    // Conversion::for_column (parquet_reader.rs:58-80)
    const int pt = physical_type, cv = conversion;
    const bool ok = (cv == CV_BOOL && pt == PQ_BOOLEAN) || ((cv == CV_INT32 || cv == CV_DATE || cv == CV_DEC_I32) && pt == PQ_INT32) ||
                    ((cv == CV_INT64 || cv == CV_DEC_I64) && pt == PQ_INT64) || (cv == CV_FLOAT && pt == PQ_FLOAT) ||
                    (cv == CV_DOUBLE && pt == PQ_DOUBLE) || (cv == CV_UTF8 && pt == PQ_BYTE_ARRAY) ||
                    (cv == CV_DEC_BYTES && (pt == PQ_BYTE_ARRAY || (pt == PQ_FLBA && type_length > 0)));
    if (!ok) raise(ML_ERR_UNSUPPORTED, "parquet: physical type " + std::to_string(pt) + " with conversion " + std::to_string(cv));
    const int out_type = cv == CV_BOOL ? ML_TYPE_BOOL : cv == CV_INT32 ? ML_TYPE_INT32 : cv == CV_DATE ? ML_TYPE_DATE
                         : cv == CV_INT64 ? ML_TYPE_INT64 : cv == CV_UTF8 ? ML_TYPE_UTF8 : ML_TYPE_FLOAT64;
    const int level_width = max_def ? 32 - __builtin_clz((unsigned)max_def) : 0;
    const int pw = pt == PQ_INT32 || pt == PQ_FLOAT ? 4 : pt == PQ_FLBA ? type_length : 8;
    ctx->set_current();
    OpStream op_stream(ctx);
    const cudaStream_t s = op_stream.s;
    auto b = std::make_unique<ml_batch>();
    b->ctx = ctx;
    b->nrows = num_rows;
    b->res = std::make_unique<Reservation>(ctx, "ParquetDecode");
    auto col = std::make_unique<DevColumn>();
    col->dtype = out_type;
    col->kind = CK_FIXED;
    col->n = num_rows;

    // pages and their places in the uncompressed buffer
    std::vector<Page> pages = parse_pages(chunk, chunk_bytes);
    int dict_page = -1;
    std::vector<int> data;
    int64_t rows = 0, ubytes = 0;
    std::vector<int64_t> uoff;
    for (size_t i = 0; i < pages.size(); i++) {
        const Page& pg = pages[i];
        uoff.push_back(ubytes);
        ubytes += (pg.uncompressed + 15) & ~15;
        if (pg.type == PAGE_DICTIONARY) {
            if (dict_page >= 0 || !data.empty()) raise(ML_ERR_INVALID, "parquet: a dictionary page after the first page");
            if (pg.encoding != ENC_PLAIN && pg.encoding != ENC_PLAIN_DICTIONARY)
                raise(ML_ERR_UNSUPPORTED, "parquet: dictionary page encoding " + std::to_string(pg.encoding));
            dict_page = (int)i;
            continue;
        }
        if (pg.encoding != ENC_PLAIN && pg.encoding != ENC_PLAIN_DICTIONARY && pg.encoding != ENC_RLE_DICTIONARY &&
            !(pg.encoding == ENC_RLE && pt == PQ_BOOLEAN))
            raise(ML_ERR_UNSUPPORTED, "parquet: data page encoding " + std::to_string(pg.encoding));
        if ((pg.encoding == ENC_PLAIN_DICTIONARY || pg.encoding == ENC_RLE_DICTIONARY) && dict_page < 0)
            raise(ML_ERR_INVALID, "parquet: dictionary-encoded page without a dictionary page");
        if (pg.type == PAGE_DATA && max_def > 0 && pg.def_encoding != ENC_RLE)
            raise(ML_ERR_UNSUPPORTED, "parquet: definition level encoding " + std::to_string(pg.def_encoding));
        if (pg.type == PAGE_DATA_V2 && pg.rep_bytes + pg.def_bytes > std::min(pg.compressed, pg.uncompressed))
            raise(ML_ERR_INVALID, "parquet: a v2 page's levels run past the page");
        data.push_back((int)i);
        rows += pg.num_values;
    }
    // read_all (parquet_reader.rs:104-133): the chunk must hold exactly num_rows records
    if (rows != num_rows)
        raise(ML_ERR_INVALID, "parquet: expected " + std::to_string(num_rows) + " rows, decoded " + std::to_string(rows));
    const int np = (int)data.size();
    if (num_rows == 0) {
        col->data = DevBuf(ctx, 8, b->res.get());
        if (out_type == ML_TYPE_UTF8) {
            col->kind = CK_UTF8;
            col->offsets = DevBuf(ctx, 4, b->res.get());
            CK(cudaMemsetAsync(col->offsets.get(), 0, 4, s));
        }
        CK(cudaStreamSynchronize(s));
        b->cols.push_back(std::move(col));
        *out = b.release();
        return ML_OK;
    }

    // 1. the chunk to the device, then every page uncompressed
    // 64 bytes of padding: warp_copy reads up to 8 bytes past a copy's source
    DevBuf dchunk(ctx, (size_t)chunk_bytes + 64, nullptr), upages(ctx, (size_t)ubytes + 64, nullptr);
    // from the caller's (pageable) buffer: a pinned staging buffer per call costs more than it saves
    CK(cudaMemcpyAsync(dchunk.get(), chunk, (size_t)chunk_bytes, cudaMemcpyHostToDevice, s));
    const uint8_t* dc = dchunk.get<uint8_t>();
    uint8_t* up = upages.get<uint8_t>();
    std::vector<SnapJob> jobs;
    std::vector<uint2> frags;  // {page, fragment} per 64 KB of Snappy output
    uint32_t plan_words = 0;
    for (size_t i = 0; i < pages.size(); i++) {
        const Page& pg = pages[i];
        const bool v2 = pg.type == PAGE_DATA_V2;
        const int64_t lv = v2 ? pg.rep_bytes + pg.def_bytes : 0;  // v2 levels are never compressed
        if (lv) CK(cudaMemcpyAsync(up + uoff[i], dc + pg.payload, (size_t)lv, cudaMemcpyDeviceToDevice, s));
        const bool compressed = codec == ML_PQ_CODEC_SNAPPY && (!v2 || pg.v2_compressed);
        if (compressed) {
            const uint32_t dlen = (uint32_t)(pg.uncompressed - lv);
            const uint32_t nfrag = (uint32_t)(((uint64_t)dlen + kSnapFrag - 1) / kSnapFrag);
            for (uint32_t k = 0; k < nfrag; k++) frags.push_back(uint2{(uint32_t)jobs.size(), k});
            jobs.push_back(SnapJob{dc + pg.payload + lv, up + uoff[i] + lv, (uint32_t)(pg.compressed - lv), dlen,
                                   plan_words, nfrag});
            plan_words += nfrag + 3;
        } else {
            if (pg.compressed != pg.uncompressed) raise(ML_ERR_INVALID, "parquet: an uncompressed page changes size");
            if (pg.compressed > lv)
                CK(cudaMemcpyAsync(up + uoff[i] + lv, dc + pg.payload + lv, (size_t)(pg.compressed - lv), cudaMemcpyDeviceToDevice, s));
        }
    }
    DevBuf err(ctx, 16, nullptr);
    CK(cudaMemsetAsync(err.get(), 0, 4, s));
    uint32_t* derr = err.get<uint32_t>();
    DevBuf dj, splan;  // read by the Snappy kernels: live to the end of the call
    if (!jobs.empty()) {
        // the jobs and the fragment table in one upload
        const size_t jb = jobs.size() * sizeof(SnapJob), fb = frags.size() * sizeof(uint2);
        std::vector<uint8_t> hj(jb + fb);
        std::memcpy(hj.data(), jobs.data(), jb);
        if (fb) std::memcpy(hj.data() + jb, frags.data(), fb);
        dj = DevBuf(ctx, hj.size(), nullptr);
        CK(cudaMemcpyAsync(dj.get(), hj.data(), hj.size(), cudaMemcpyHostToDevice, s));
        const SnapJob* J = dj.get<SnapJob>();
        const uint2* F = (const uint2*)(dj.get<uint8_t>() + jb);
        const int nj = (int)jobs.size(), nf = (int)frags.size();
        splan = DevBuf(ctx, (size_t)plan_words * 4, nullptr);
        // per call: the attribute belongs to the current device's copy of the kernel
        CK(cudaFuncSetAttribute(k_pq_snappy_frag, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSnapFragSmem));
        k_pq_snappy_walk<<<nj, kWalkThreads, 0, s>>>(J, splan.get<uint32_t>());
        if (nf) k_pq_snappy_frag<<<nf, 32, kSnapFragSmem, s>>>(J, F, splan.get<uint32_t>());
        k_pq_snappy_serial<<<nj, 32, 0, s>>>(J, splan.get<uint32_t>(), derr);
        ctx->count_launch(nf ? 3 : 2);
        // wait here: a long Snappy kernel with the decode queued behind it holds up other calls'
        // work that shares its hardware queue (measured: 3.6 s instead of 0.9 s for 960 chunks
        // decoded from 16 threads)
        CK(cudaStreamSynchronize(s));
    }
    auto read_err = [&]() {
        uint32_t e = 0;
        CK(cudaMemcpyAsync(&e, derr, 4, cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
        check_pq(ctx, e);
    };

    // 2. data pages (the kernels are bounds-checked, so a decode error is read once, at the end;
    //    a page's run table starts at its first row: a stream has at most one run per value): layout, level runs, validity, present values, index runs
    std::vector<PageDev> hp(np);
    int64_t row0 = 0;
    for (int j = 0; j < np; j++) {
        const Page& pg = pages[data[j]];
        PageDev& d = hp[j];
        d = PageDev{};
        d.data = up + uoff[data[j]];
        d.len = (uint32_t)pg.uncompressed;
        d.v2 = pg.type == PAGE_DATA_V2;
        d.def_bytes = pg.def_bytes;
        d.rep_bytes = pg.rep_bytes;
        d.encoding = pg.encoding == ENC_PLAIN_DICTIONARY ? ENC_RLE_DICTIONARY : pg.encoding;
        d.row0 = row0;
        d.nrows = (uint32_t)pg.num_values;
        d.lv_run0 = d.ix_run0 = (uint64_t)row0;
        row0 += pg.num_values;
    }
    DevBuf dpages(ctx, hp.size() * sizeof(PageDev), nullptr);
    PageDev* P = dpages.get<PageDev>();
    CK(cudaMemcpyAsync(P, hp.data(), hp.size() * sizeof(PageDev), cudaMemcpyHostToDevice, s));
    DevBuf lv_runs(ctx, (size_t)num_rows * sizeof(Run), nullptr), ix_runs(ctx, (size_t)num_rows * sizeof(Run), nullptr);
    k_pq_layout<<<grid_of(np), 256, 0, s>>>(P, np, max_def, derr);
    ctx->count_launch(2);
    k_pq_runs<<<grid_of(np), 256, 0, s>>>(P, np, 0, level_width, nullptr, lv_runs.get<Run>(), derr);
    const int64_t ntiles = (num_rows + kPqTile - 1) / kPqTile;
    DevBuf valid(ctx, (size_t)ntiles * kPqTile / 8, b->res.get());  // u32 words; as u64 words the validity
    DevBuf tcounts(ctx, (size_t)ntiles * 4, nullptr), toffs(ctx, (size_t)(ntiles + 1) * 8, nullptr);
    DevBuf scratch(ctx, std::max<size_t>(scan_scratch_words(ntiles) * 8, 8), nullptr);
    k_pq_valid<<<(int)ntiles, 256, 0, s>>>(P, np, lv_runs.get<Run>(), max_def, level_width, num_rows, valid.get<uint32_t>(),
                                           tcounts.get<uint32_t>());
    launch_scan_u32(tcounts.get<uint32_t>(), toffs.get<uint64_t>(), ntiles, scratch.get<uint64_t>(), s);
    DevBuf nvals(ctx, (size_t)np * 4 + 4, nullptr);
    k_pq_page_valid<<<grid_of(np + 1), 256, 0, s>>>(P, np, valid.get<uint32_t>(), toffs.get<uint64_t>(), num_rows,
                                                    nvals.get<uint32_t>());
    k_pq_runs<<<grid_of(np), 256, 0, s>>>(P, np, 1, level_width, nvals.get<uint32_t>(), ix_runs.get<Run>(), derr);
    ctx->count_launch(5);

    // 3. the dictionary page and PLAIN byte arrays
    DecodeArgs D{};
    D.pages = P;
    D.npages = np;
    D.runs = ix_runs.get<Run>();
    D.valid = valid.get<uint32_t>();
    D.tile_offs = toffs.get<uint64_t>();
    D.nrows = num_rows;
    D.ptype = pt;
    D.conv = cv;
    D.type_length = type_length;
    D.div = powi(10.0, scale);
    D.err = derr;
    DevBuf dptr, dlen, vptr, vlen;
    if (dict_page >= 0) {
        const Page& dpg = pages[dict_page];
        D.dict = up + uoff[dict_page];
        D.dict_n = (uint32_t)std::max(dpg.num_values, 0);
        if (pt != PQ_BYTE_ARRAY && (int64_t)D.dict_n * pw > dpg.uncompressed)
            raise(ML_ERR_INVALID, "parquet: the dictionary page is shorter than its entries");
    }
    if (pt == PQ_BYTE_ARRAY) {
        dptr = DevBuf(ctx, std::max<size_t>((size_t)D.dict_n * 8, 8), nullptr);
        dlen = DevBuf(ctx, std::max<size_t>((size_t)D.dict_n * 4, 4), nullptr);
        vptr = DevBuf(ctx, (size_t)num_rows * 8, nullptr);  // present values <= rows
        vlen = DevBuf(ctx, (size_t)num_rows * 4, nullptr);
        k_pq_byte_arrays<<<grid_of(np + 1), 256, 0, s>>>(
            P, np, nvals.get<uint32_t>(), vptr.get<const uint8_t*>(), vlen.get<uint32_t>(), D.dict,
            dict_page >= 0 ? (uint32_t)pages[dict_page].uncompressed : 0u, D.dict_n, dptr.get<const uint8_t*>(),
            dlen.get<uint32_t>(), derr);
        ctx->count_launch();
        D.dict_ptr = dptr.get<const uint8_t* const>();
        D.dict_len = dlen.get<uint32_t>();
        D.vptr = vptr.get<const uint8_t* const>();
        D.vlen = vlen.get<uint32_t>();
    }

    // 4. values
    DevBuf sptr, slen;
    if (cv == CV_UTF8) {
        sptr = DevBuf(ctx, (size_t)num_rows * 8, nullptr);
        slen = DevBuf(ctx, (size_t)num_rows * 4 + 4, nullptr);
        D.str_ptr = sptr.get<const uint8_t*>();
        D.str_len = slen.get<uint32_t>();
    } else {
        col->data = DevBuf(ctx, std::max<size_t>((size_t)num_rows * width_of(out_type), 8), b->res.get());
        D.out = col->data.get();
    }
    k_pq_values<<<(int)ntiles, 256, 0, s>>>(D);
    ctx->count_launch();
    uint64_t present = 0;
    CK(cudaMemcpyAsync(&present, toffs.get<uint64_t>() + ntiles, 8, cudaMemcpyDeviceToHost, s));
    read_err();  // synchronizes: `present` is on the host
    if (present != (uint64_t)num_rows) {  // validity only when a value is missing (read_all)
        col->validity = std::move(valid);
    }

    // 5. strings: encode_strings (parquet_reader.rs:176-212)
    if (cv == CV_UTF8) {
        const int64_t n = num_rows;
        DevBuf offs(ctx, (size_t)(n + 1) * 8, nullptr), sc(ctx, std::max<size_t>(scan_scratch_words(n) * 8, 8), nullptr);
        launch_scan_u32(slen.get<uint32_t>(), offs.get<uint64_t>(), n, sc.get<uint64_t>(), s);
        uint64_t total = 0;
        CK(cudaMemcpyAsync(&total, offs.get<uint64_t>() + n, 8, cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
        if (total > 0xFFFFFFFFull) raise(ML_ERR_UNSUPPORTED, "parquet: a string column larger than 4 GiB");
        DevBuf off32(ctx, (size_t)(n + 1) * 4, b->res.get()), bytes(ctx, std::max<uint64_t>(total, 1), b->res.get());
        k_pq_str_copy<<<grid_of(n), 256, 0, s>>>(sptr.get<const uint8_t* const>(), slen.get<uint32_t>(),
                                                  offs.get<uint64_t>(), n, off32.get<uint32_t>(), bytes.get<uint8_t>());
        // equal strings get one canonical row (every row: a NULL row counts as "")
        const uint64_t cap = pow2_ceil(std::max<uint64_t>(16, (uint64_t)n * 2));
        DevBuf tslots(ctx, cap * 16, nullptr), canon(ctx, (size_t)n * 4, nullptr), first(ctx, (size_t)n * 4, nullptr);
        CK(cudaMemsetAsync(tslots.get(), 0, cap * 16, s));
        TableView tv{tslots.get<uint64_t>(), cap - 1, 1, 2};
        launch_strid(off32.get<uint32_t>(), bytes.get<uint8_t>(), nullptr, n, tv, canon.get<uint32_t>(), derr, s);
        CK(cudaMemsetAsync(first.get(), 0xFF, (size_t)n * 4, s));
        k_pq_first<<<grid_of(n), 256, 0, s>>>(canon.get<uint32_t>(), n, first.get<uint32_t>());
        const int nb = select_blocks(n), rpb = select_rows_per_block();  // launch_index_write's blocks
        DevBuf bits(ctx, (size_t)nb * rpb / 8, nullptr), counts(ctx, (size_t)nb * 4, nullptr), boffs(ctx, (size_t)(nb + 1) * 8, nullptr);
        DevBuf sc2(ctx, std::max<size_t>(scan_scratch_words(nb) * 8, 8), nullptr);
        k_pq_first_flags<<<nb, 256, 0, s>>>(canon.get<uint32_t>(), first.get<uint32_t>(), n, bits.get<uint32_t>(),
                                            counts.get<uint32_t>(), rpb);
        launch_scan_u32(counts.get<uint32_t>(), boffs.get<uint64_t>(), nb, sc2.get<uint64_t>(), s);
        uint64_t distinct = 0;
        CK(cudaMemcpyAsync(&distinct, boffs.get<uint64_t>() + nb, 8, cudaMemcpyDeviceToHost, s));
        ctx->count_launch(6);
        read_err();
        const uint64_t limit = std::min<uint64_t>(std::max<uint64_t>((uint64_t)n / 8, 1), 65536);  // (n / 8).clamp(1, MAX_DICT)
        if (distinct <= limit) {
            // the first occurrences in row order are the dictionary; each row's code is its string's
            DevBuf list(ctx, (size_t)distinct * 4 + 4, nullptr), code_of(ctx, (size_t)n * 4, nullptr);
            launch_index_write(n, bits.get<uint32_t>(), boffs.get<uint64_t>(), list.get<uint32_t>(), s);
            k_pq_codes<<<grid_of((int64_t)distinct), 256, 0, s>>>(list.get<uint32_t>(), (uint32_t)distinct, canon.get<uint32_t>(),
                                                                  code_of.get<uint32_t>());
            DevBuf codes(ctx, (size_t)n * 4, b->res.get());
            k_pq_codes2<<<grid_of(n), 256, 0, s>>>(canon.get<uint32_t>(), n, code_of.get<uint32_t>(), codes.get<uint32_t>());
            ctx->count_launch(3);
            std::vector<uint32_t> hl(distinct), ho(n + 1);
            if (distinct) CK(cudaMemcpyAsync(hl.data(), list.get(), distinct * 4, cudaMemcpyDeviceToHost, s));
            CK(cudaMemcpyAsync(ho.data(), off32.get(), (size_t)(n + 1) * 4, cudaMemcpyDeviceToHost, s));
            std::vector<uint8_t> hb(total);
            if (total) CK(cudaMemcpyAsync(hb.data(), bytes.get(), total, cudaMemcpyDeviceToHost, s));
            CK(cudaStreamSynchronize(s));
            auto hd = std::make_shared<HostDict>();
            for (uint64_t i = 0; i < distinct; i++) {
                const uint32_t r = hl[i];
                hd->bytes.insert(hd->bytes.end(), hb.begin() + ho[r], hb.begin() + ho[r + 1]);
                hd->off.push_back((uint32_t)hd->bytes.size());
            }
            col->kind = CK_DICT;
            col->data = std::move(codes);
            col->dict = std::move(hd);
        } else {
            col->kind = CK_UTF8;
            col->offsets = std::move(off32);
            col->data = std::move(bytes);
        }
    }
    CK(cudaStreamSynchronize(s));
    read_err();
    b->cols.push_back(std::move(col));
    *out = b.release();
    API_END
}
