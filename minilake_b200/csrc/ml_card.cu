// sm_100a kernels of the learned cardinality estimator.
//
// The HLL scan is one streaming pass over the key columns (HBM-bound) with the 2^14
// registers privatized in shared memory per CTA.  The MLP is 13,057 FP32 parameters:
// far too small for tensor cores to matter, so its layers are plain FP32 CUDA-core
// kernels, one thread per output element.
#include "ml_card.hpp"
#include "ml_device.cuh"

namespace mlg {

namespace {

// MurmurHash3's 64-bit finalizer (fmix64): spreads the engine's key hash over all 64
// bits before the register index and rank are taken from it.
__device__ __forceinline__ uint64_t fmix64(uint64_t k) {
    k ^= k >> 33;
    k *= 0xff51afd7ed558ccdull;
    k ^= k >> 33;
    k *= 0xc4ceb9fe1a85ec53ull;
    k ^= k >> 33;
    return k;
}

__global__ void __launch_bounds__(256) k_hll(const __grid_constant__ PipeArgs P, const __grid_constant__ KeyLayout L,
                                             HllOut o) {
    extern __shared__ uint32_t regs[];
    for (int i = threadIdx.x; i < kHllRegisters; i += blockDim.x) regs[i] = 0;
    __syncthreads();
    const EvalEnv env{P.cols, P.prog, P.arena, P.luts};
    unsigned long long nulls = 0, lo = ~0ull, hi = 0;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < P.n; i += stride) {
        RowCtx x;
        bool ok = true;
        x.r = sel_row(P, i, ok);
        if (!ok) continue;
        x.b0 = x.b1 = x.b2 = x.b3 = 0;
        x.head = 0;
        uint64_t w[2];
        uint32_t nm;
        make_key(env, L, x, w, &nm, false);
        if (nm) {
            nulls++;
        } else {
            lo = w[0] < lo ? w[0] : lo;
            hi = w[0] > hi ? w[0] : hi;
        }
        const uint64_t h = fmix64(key_hash(w, L.nwords, nm));
        const uint32_t idx = (uint32_t)(h >> (64 - kHllP));
        const uint64_t rest = (h << kHllP) | (1ull << (kHllP - 1));  // guard bit: rank <= 64 - kHllP + 1
        atomicMax(&regs[idx], (uint32_t)__clzll((long long)rest) + 1u);
    }
    for (int off = 16; off; off >>= 1) {
        nulls += __shfl_xor_sync(0xFFFFFFFFu, nulls, off);
        unsigned long long l2 = __shfl_xor_sync(0xFFFFFFFFu, lo, off), h2 = __shfl_xor_sync(0xFFFFFFFFu, hi, off);
        lo = l2 < lo ? l2 : lo;
        hi = h2 > hi ? h2 : hi;
    }
    if ((threadIdx.x & 31) == 0) {
        if (nulls) atomicAdd(o.nulls, nulls);
        if (lo != ~0ull) atomicMin(o.minmax, lo);
        if (hi) atomicMax(o.minmax + 1, hi);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < kHllRegisters; i += blockDim.x)
        if (regs[i]) atomicMax(o.regs + i, regs[i]);
}

// Register-wise max over the CTAs' byte registers (4 per word) -> the u32 registers.
__global__ void k_hll_merge(const uint32_t* __restrict__ cta_regs, int ctas, uint32_t* regs) {
    const int w = blockIdx.x * blockDim.x + threadIdx.x;
    if (w >= kHllRegisters / 4) return;
    uint32_t m = 0;
    for (int c = 0; c < ctas; c++) m = __vmaxu4(m, __ldg(cta_regs + (size_t)c * (kHllRegisters / 4) + w));
    for (int b = 0; b < 4; b++) regs[4 * w + b] = (m >> (8 * b)) & 0xFFu;
}

__global__ void k_dense_fwd(const float* __restrict__ X, int in, const float* __restrict__ W, const float* __restrict__ b,
                            float* __restrict__ Y, int out, int B, int relu) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= B * out) return;
    int r = t / out, o = t % out;
    const float* x = X + (size_t)r * in;
    const float* w = W + (size_t)o * in;
    float acc = b[o];
    for (int i = 0; i < in; i++) acc = fmaf(w[i], x[i], acc);
    Y[t] = relu ? fmaxf(acc, 0.0f) : acc;
}

__device__ __forceinline__ float grad_through(const float* Y, const float* dY, size_t k, int relu) {
    return relu && !(Y[k] > 0.0f) ? 0.0f : dY[k];
}

__global__ void k_dense_bwd_params(const float* __restrict__ X, int in, const float* __restrict__ Y, int out,
                                   const float* __restrict__ dY, float* __restrict__ dW, float* __restrict__ db, int B,
                                   int relu) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < out * in) {
        int o = t / in, i = t % in;
        float acc = 0.0f;
        for (int r = 0; r < B; r++) acc = fmaf(grad_through(Y, dY, (size_t)r * out + o, relu), X[(size_t)r * in + i], acc);
        dW[t] = acc;
    } else if (t < out * in + out) {
        int o = t - out * in;
        float acc = 0.0f;
        for (int r = 0; r < B; r++) acc += grad_through(Y, dY, (size_t)r * out + o, relu);
        db[o] = acc;
    }
}

__global__ void k_dense_bwd_data(const float* __restrict__ W, int in, const float* __restrict__ Y, int out,
                                 const float* __restrict__ dY, float* __restrict__ dX, int B, int relu) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= B * in) return;
    int r = t / in, i = t % in;
    float acc = 0.0f;
    for (int o = 0; o < out; o++) acc = fmaf(grad_through(Y, dY, (size_t)r * out + o, relu), W[(size_t)o * in + i], acc);
    dX[t] = acc;
}

__global__ void k_mse_grad(const float* pred, const float* target, float* dpred, float* loss, int B) {
    __shared__ float part[256];
    float l = 0.0f;
    for (int r = threadIdx.x; r < B; r += blockDim.x) {
        float e = pred[r] - target[r];
        dpred[r] = 2.0f * e / (float)B;
        l += e * e;
    }
    part[threadIdx.x] = l;
    __syncthreads();
    for (int k = blockDim.x / 2; k; k >>= 1) {
        if (threadIdx.x < k) part[threadIdx.x] += part[threadIdx.x + k];
        __syncthreads();
    }
    if (threadIdx.x == 0) *loss = part[0] / (float)B;
}

__global__ void k_adam(float* p, const float* g, float* m, float* v, int n, float lr, float b1, float b2, float eps,
                       float bc1, float bc2_sqrt) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float gi = g[i];
    float mi = b1 * m[i] + (1.0f - b1) * gi;
    float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    float denom = sqrtf(vi) / bc2_sqrt + eps;
    p[i] -= (lr / bc1) * mi / denom;
}

__global__ void k_add_column(float* out, const float* X, int B, int cols, int col, float scale) {
    int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r < B) out[r] += scale * X[(size_t)r * cols + col];
}

__global__ void k_gather_rows(const float* X, const uint32_t* idx, int B, int cols, float* out) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= B * cols) return;
    int r = t / cols, c = t % cols;
    out[t] = X[(size_t)idx[r] * cols + c];
}

int blocks_for(long long n, int threads = 256) { return (int)((n + threads - 1) / threads); }

}  // namespace

void launch_hll(const PipeArgs& P, const KeyLayout& L, HllOut o, cudaStream_t s) {
    const int smem = kHllRegisters * 4;  // 64 KB of registers per CTA: above the default 48 KB limit
    cudaFuncSetAttribute(k_hll, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    int sms = 148, dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    long long want = (P.n + 255) / 256;
    int grid = (int)(want < 2LL * sms ? (want > 0 ? want : 1) : 2LL * sms);
    k_hll<<<grid, 256, smem, s>>>(P, L, o);
}

void launch_hll_merge(const uint32_t* cta_regs, int ctas, uint32_t* regs, cudaStream_t s) {
    k_hll_merge<<<(kHllRegisters / 4 + 255) / 256, 256, 0, s>>>(cta_regs, ctas, regs);
}

void launch_dense_fwd(const float* X, int in, const float* W, const float* bias, float* Y, int out, int B, bool relu,
                      cudaStream_t s) {
    if (B > 0) k_dense_fwd<<<blocks_for((long long)B * out), 256, 0, s>>>(X, in, W, bias, Y, out, B, relu);
}
void launch_dense_bwd_params(const float* X, int in, const float* Y, int out, const float* dY, float* dW, float* db,
                             int B, bool relu, cudaStream_t s) {
    k_dense_bwd_params<<<blocks_for((long long)out * in + out), 256, 0, s>>>(X, in, Y, out, dY, dW, db, B, relu);
}
void launch_dense_bwd_data(const float* W, int in, const float* Y, int out, const float* dY, float* dX, int B, bool relu,
                           cudaStream_t s) {
    if (B > 0) k_dense_bwd_data<<<blocks_for((long long)B * in), 256, 0, s>>>(W, in, Y, out, dY, dX, B, relu);
}
void launch_mse_grad(const float* pred, const float* target, float* dpred, float* loss, int B, cudaStream_t s) {
    k_mse_grad<<<1, 256, 0, s>>>(pred, target, dpred, loss, B);
}
void launch_adam(float* p, const float* g, float* m, float* v, int n, float lr, float beta1, float beta2, float eps,
                 int t, cudaStream_t s) {
    float bc1 = 1.0f - powf(beta1, (float)t);
    float bc2_sqrt = sqrtf(1.0f - powf(beta2, (float)t));
    k_adam<<<blocks_for(n), 256, 0, s>>>(p, g, m, v, n, lr, beta1, beta2, eps, bc1, bc2_sqrt);
}
void launch_add_column(float* out, const float* X, int B, int cols, int col, float scale, cudaStream_t s) {
    if (B > 0) k_add_column<<<blocks_for(B), 256, 0, s>>>(out, X, B, cols, col, scale);
}
void launch_gather_rows(const float* X, const uint32_t* idx, int B, int cols, float* out, cudaStream_t s) {
    if (B > 0) k_gather_rows<<<blocks_for((long long)B * cols), 256, 0, s>>>(X, idx, B, cols, out);
}

}  // namespace mlg
