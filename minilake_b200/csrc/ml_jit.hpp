// Runtime specialization of the fused pipeline kernels.
//
// The ahead-of-time kernels interpret each pipeline's programs (a uniform-dispatch stack
// machine).  For the hot sinks the pipeline is also turned into CUDA C++ source in which
// every instruction, key field and accumulator is a straight-line statement over the
// same device helpers (ml_device.cuh, ml_agg.cuh), compiled once per pipeline shape with
// NVRTC for sm_100a and cached for the process.  Literal values, arena offsets and all
// pointers stay kernel arguments, so pipelines that differ only in constants share one
// kernel.  Both forms compute the same results; ML_CTX_INTERPRET selects the interpreter.
#pragma once

#include "ml_pipeline.hpp"

namespace mlg {

// Specialized fused filter/probe/aggregate kernel (signature of k_agg) for this launch,
// or nullptr when runtime compilation is unavailable or disabled for the context.
void* jit_agg_kernel(Ctx* ctx, const Pipeline& pipe, const PipeArgs& P, const AggArgs& A);

// Specialized overflow-resume kernel (signature of k_agg_resume), or nullptr.
void* jit_agg_resume_kernel(Ctx* ctx, const Pipeline& pipe, const PipeArgs& P, const AggArgs& A);

// Specialized join-build insert kernel (signature of k_join_insert), or nullptr.
void* jit_join_insert_kernel(Ctx* ctx, const Pipeline& pipe, const PipeArgs& P, const KeyLayout& L);
// Filter pass bits and per-CTA counts (the layout of launch_select_flags), or nullptr when the
// pipeline has duplicate-key probes or specialization is off.  Arguments: P, bits, block_counts.
void* jit_select_kernel(Ctx* ctx, const Pipeline& pipe, const PipeArgs& P);
// Cardinality features scan of the key layout L (64 KB of dynamic shared memory per CTA).
// Arguments: P, L, cta_regs (gridDim x 4096 words), nulls, minmax.
void* jit_hll_kernel(Ctx* ctx, const Pipeline& pipe, const PipeArgs& P, const KeyLayout& L);
// Sources of the kernels above.
// `contig`: consecutive rows per thread with vector loads (needs no selection vector and 16-byte
// aligned source columns).
std::string jit_select_source(const Pipeline& pipe, const PipeArgs& P, bool contig);
std::string jit_hll_source(const Pipeline& pipe, const PipeArgs& P, const KeyLayout& L, bool contig);

// Rows one thread of the specialized aggregate kernel handles per iteration (its grid
// needs n / rows-per-thread threads).
int jit_rows_per_thread(const PipeArgs& P);

// Launch a specialized kernel with `args` (pointers to the kernel's parameters).
void jit_launch(void* fn, unsigned grid, unsigned block, size_t smem, cudaStream_t s, void** args);
// CTAs of `block` threads with `smem` bytes of dynamic shared memory resident on one SM.
int jit_resident_blocks(void* fn, unsigned block, size_t smem);

// The generated source of the aggregate kernel (exposed for tests of the generator).
std::string jit_agg_source(const Pipeline& pipe, const PipeArgs& P, const AggArgs& A, bool contig = false);

}  // namespace mlg
