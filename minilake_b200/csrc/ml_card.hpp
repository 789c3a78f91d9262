// Learned cardinality estimator: the HyperLogLog scan kernel and the FP32 MLP kernels
// (forward, backward, Adam) that predict log2 of a GROUP BY / join-build key's distinct
// count from scan statistics.  Used to presize hash tables; results never depend on it.
#pragma once

#include <cuda_runtime.h>

#include "ml_args.hpp"

namespace mlg {

constexpr int kHllP = 14;                      // 2^14 registers, 64-bit hashes
constexpr int kHllRegisters = 1 << kHllP;
constexpr int kCardFeatures = ML_CARD_FEATURES;  // 64-bin register histogram + 8 scan statistics
constexpr int kCardHidden = 64;
constexpr int kCardParams = ML_CARD_PARAMS;      // 72-64-64-64-1
// Offsets of the layers' weights (row-major [out][in]) and biases in the parameter vector.
constexpr int kW1 = 0, kB1 = kW1 + kCardHidden * kCardFeatures;
constexpr int kW2 = kB1 + kCardHidden, kB2 = kW2 + kCardHidden * kCardHidden;
constexpr int kW3 = kB2 + kCardHidden, kB3 = kW3 + kCardHidden * kCardHidden;
constexpr int kW4 = kB3 + kCardHidden, kB4 = kW4 + kCardHidden;
static_assert(kB4 + 1 == kCardParams, "parameter layout");

// Scan statistics of one key: HLL registers (max rank per register), rows with a NULL key,
// min and max of the first normalized key word over the non-NULL rows.
struct HllOut {
    uint32_t* regs;                // kHllRegisters, zeroed by the caller
    unsigned long long* nulls;     // 1, zeroed
    unsigned long long* minmax;    // 2: ~0 and 0 on entry
};
void launch_hll(const PipeArgs& P, const KeyLayout& L, HllOut o, cudaStream_t s);
// Registers of the runtime-specialized scan: max over `ctas` CTAs' byte registers
// (kHllRegisters / 4 words each) into the u32 registers.
void launch_hll_merge(const uint32_t* cta_regs, int ctas, uint32_t* regs, cudaStream_t s);

// Y[b][o] = act(bias[o] + sum_i W[o][i] X[b][i]) for b < B.
void launch_dense_fwd(const float* X, int in, const float* W, const float* bias, float* Y, int out, int B, bool relu,
                      cudaStream_t s);
// Given dY = dLoss/dY of a layer with input X and output Y: dW[o][i] = sum_b G[b][o] X[b][i],
// db[o] = sum_b G[b][o], with G = dY * (relu ? Y > 0 : 1).
void launch_dense_bwd_params(const float* X, int in, const float* Y, int out, const float* dY, float* dW, float* db,
                             int B, bool relu, cudaStream_t s);
// dX[b][i] = sum_o G[b][o] W[o][i].
void launch_dense_bwd_data(const float* W, int in, const float* Y, int out, const float* dY, float* dX, int B, bool relu,
                           cudaStream_t s);
// Mean squared error of pred[0..B) against target: dpred = 2 (pred - target) / B, *loss = mean.
void launch_mse_grad(const float* pred, const float* target, float* dpred, float* loss, int B, cudaStream_t s);
// One Adam step (bias-corrected, as torch.optim.Adam without weight decay) at step t >= 1.
void launch_adam(float* p, const float* g, float* m, float* v, int n, float lr, float beta1, float beta2, float eps,
                 int t, cudaStream_t s);
// out[r] += scale * X[r][col]: the skip connection from the sketch's log-estimate feature.
void launch_add_column(float* out, const float* X, int B, int cols, int col, float scale, cudaStream_t s);
// The prediction is log2(HLL estimate + 1) + MLP(features): feature 67 holds that log2 / 32,
// so the network learns the correction to the sketch.
constexpr int kCardSkipFeature = 67;
constexpr float kCardSkipScale = 32.0f;
// out[r][:] = X[idx[r]][:] for r < B rows of `cols` floats.
void launch_gather_rows(const float* X, const uint32_t* idx, int B, int cols, float* out, cudaStream_t s);

}  // namespace mlg
