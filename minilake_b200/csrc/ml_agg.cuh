// Accumulator updates of the hash aggregate (accumulator.rs:110-594), shared by the
// ahead-of-time kernels and the runtime-specialized pipeline kernels.
#pragma once

#include "ml_args.hpp"
#include "ml_device.cuh"

namespace mlg {

// ---- hash aggregation ---------------------------------------------------------------------
__device__ __forceinline__ uint64_t agg_identity(int kind) {
    switch (kind) {
        case A_MIN_I64: return 0x7FFFFFFFFFFFFFFFull;
        case A_MAX_I64: return 0x8000000000000000ull;
        case A_MIN_F64:
        case A_MIN_STR: return ~0ull;
        case A_MAX_F64:
        case A_MAX_STR: return 0ull;
        default: return 0ull;
    }
}

// Fold value v into the accumulator word(s) at `w` (shared or global memory).
__device__ __forceinline__ void acc_apply(int kind, uint64_t* w, uint64_t v) {
    switch (kind) {
        case A_SUM_I64: atomicAdd((unsigned long long*)w, (unsigned long long)v); break;
        case A_SUM_F64: atomicAdd((double*)w, as_f64(v)); break;
        case A_AVG:
            atomicAdd((double*)w, as_f64(v));
            atomicAdd((unsigned long long*)w + 1, 1ull);
            break;
        case A_MIN_I64: atomicMin((long long*)w, (long long)v); break;
        case A_MAX_I64: atomicMax((long long*)w, (long long)v); break;
        case A_MIN_F64: atomicMin((unsigned long long*)w, (unsigned long long)f64_order(as_f64(v))); break;
        case A_MAX_F64: atomicMax((unsigned long long*)w, (unsigned long long)f64_order(as_f64(v))); break;
        case A_MIN_STR: atomicMin((unsigned long long*)w, (unsigned long long)v); break;  // v packed (str_pack)
        case A_MAX_STR: atomicMax((unsigned long long*)w, (unsigned long long)v); break;
        default: atomicAdd((unsigned long long*)w, 1ull); break;  // COUNT(x)
    }
}
// A string id as the packed word of A_MIN_STR / A_MAX_STR.
__device__ __forceinline__ uint64_t str_pack(const uint32_t* rank, uint32_t id) {
    return ((uint64_t)(__ldg(rank + id) + 1u) << 32) | id;
}
// acc_apply for accumulators known to be in global memory: fire-and-forget reductions
// (red.global), so no thread waits for the L2 to answer.
__device__ __forceinline__ void acc_apply_global(int kind, uint64_t* w, uint64_t v) {
    switch (kind) {
        case A_SUM_I64: asm volatile("red.relaxed.gpu.global.add.u64 [%0], %1;" ::"l"(w), "l"(v) : "memory"); break;
        case A_SUM_F64: asm volatile("red.relaxed.gpu.global.add.f64 [%0], %1;" ::"l"(w), "d"(as_f64(v)) : "memory"); break;
        case A_AVG:
            asm volatile("red.relaxed.gpu.global.add.f64 [%0], %1;" ::"l"(w), "d"(as_f64(v)) : "memory");
            asm volatile("red.relaxed.gpu.global.add.u64 [%0], %1;" ::"l"(w + 1), "l"(1ull) : "memory");
            break;
        case A_MIN_I64: asm volatile("red.relaxed.gpu.global.min.s64 [%0], %1;" ::"l"(w), "l"(v) : "memory"); break;
        case A_MAX_I64: asm volatile("red.relaxed.gpu.global.max.s64 [%0], %1;" ::"l"(w), "l"(v) : "memory"); break;
        case A_MIN_F64:
            asm volatile("red.relaxed.gpu.global.min.u64 [%0], %1;" ::"l"(w), "l"(f64_order(as_f64(v))) : "memory");
            break;
        case A_MAX_F64:
            asm volatile("red.relaxed.gpu.global.max.u64 [%0], %1;" ::"l"(w), "l"(f64_order(as_f64(v))) : "memory");
            break;
        default: asm volatile("red.relaxed.gpu.global.add.u64 [%0], %1;" ::"l"(w), "l"(1ull) : "memory"); break;
    }
}
__device__ __forceinline__ void count_global(uint64_t* w) {
    asm volatile("red.relaxed.gpu.global.add.u64 [%0], %1;" ::"l"(w), "l"(1ull) : "memory");
}

// Merge a shared-memory partial (word(s) at src) into the global block word(s) at dst.
__device__ __forceinline__ void acc_merge(int kind, uint64_t* dst, const uint64_t* src) {
    uint64_t v = src[0];
    switch (kind) {
        case A_SUM_I64:
        case A_COUNT: if (v) atomicAdd((unsigned long long*)dst, (unsigned long long)v); break;
        case A_SUM_F64: atomicAdd((double*)dst, as_f64(v)); break;
        case A_AVG:
            atomicAdd((double*)dst, as_f64(v));
            if (src[1]) atomicAdd((unsigned long long*)dst + 1, (unsigned long long)src[1]);
            break;
        case A_MIN_I64: atomicMin((long long*)dst, (long long)v); break;
        case A_MAX_I64: atomicMax((long long*)dst, (long long)v); break;
        case A_MIN_F64:
        case A_MIN_STR: atomicMin((unsigned long long*)dst, (unsigned long long)v); break;
        case A_MAX_F64:
        case A_MAX_STR: atomicMax((unsigned long long*)dst, (unsigned long long)v); break;
    }
}

// Append the row combination to the overflow list.  The lanes that overflow together take
// their slots with one atomic per warp (a full table sends every new key here).
__device__ inline void record_overflow(const PipeArgs& P, const AggArgs& A, const RowCtx& x) {
    const unsigned m = __activemask();
    const int lane = threadIdx.x & 31, leader = __ffs(m) - 1;
    unsigned long long base = 0;
    if (lane == leader) base = atomicAdd(A.ovf_count, (unsigned long long)__popc(m));
    base = __shfl_sync(m, base, leader);
    const unsigned long long k = base + __popc(m & ((1u << lane) - 1u));
    if (k >= A.ovf_cap) {
        atomicOr(P.err, (uint32_t)DE_OVERFLOW_LOST);
        return;
    }
    int w = 1 + P.nprobes;
    uint32_t* o = A.ovf + k * (uint64_t)w;
    o[0] = x.r;
    if (w > 1) o[1] = x.b0;
    if (w > 2) o[2] = x.b1;
    if (w > 3) o[3] = x.b2;
    if (w > 4) o[4] = x.b3;
}

// The CTA's direct group index (AggArgs::dslots): entry = group id + 1, 0 until a thread of
// this CTA has looked the slot's key up in the global table.  Every writer of an entry writes
// the same value (a slot stands for one key), so readers need no ordering: a 0 read only sends
// the row to the global table.
__device__ __forceinline__ uint32_t* direct_slots(const AggArgs& A, uint64_t* smem) {
    return (uint32_t*)(smem + (uint64_t)A.smem_groups * A.stride + (uint64_t)A.priv_groups * A.stride * 256);
}

__device__ inline void smem_setup(const AggArgs& A, uint64_t* smem) {
    for (int g = threadIdx.x; g < A.smem_groups; g += blockDim.x) {
        uint64_t* b = smem + (uint64_t)g * A.stride;
        for (int w = 0; w < A.stride; w++) b[w] = 0;
        for (int k = 0; k < A.nagg; k++)
            if (A.aggs[k].func != ML_AGG_COUNT_STAR) b[A.aggs[k].off] = agg_identity(A.aggs[k].kind);
    }
    if (agg_direct_on(A)) {
        uint32_t* d = direct_slots(A, smem);
        for (int i = threadIdx.x; i < kDirectSlots; i += blockDim.x) d[i] = 0;
    }
}

__device__ inline void smem_flush(const AggArgs& A, const uint64_t* smem) {
    for (int g = threadIdx.x; g < A.smem_groups; g += blockDim.x) {
        const uint64_t* b = smem + (uint64_t)g * A.stride;
        if (!b[0]) continue;
        uint64_t* d = A.acc + (uint64_t)g * A.stride;
        atomicAdd((unsigned long long*)d, (unsigned long long)b[0]);
        for (int k = 0; k < A.nagg; k++) {
            const AggDev& a = A.aggs[k];
            if (a.func == ML_AGG_COUNT_STAR) continue;
            acc_merge(a.kind, d + a.off, b + a.off);
        }
    }
}

}  // namespace mlg
