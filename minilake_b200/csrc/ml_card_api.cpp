// C ABI of the learned cardinality estimator (include/minilake_gpu.h): scan features from
// the HyperLogLog kernel, and the FP32 MLP's training and inference driven from the host.
#include <algorithm>
#include <cmath>
#include <cstring>

#include "ml_api_common.hpp"
#include "ml_jit.hpp"
#include "ml_kernels.cuh"
#include "ml_card.hpp"
#include "ml_pipeline.hpp"

using namespace mlg;

namespace {

// splitmix64: the model's deterministic host random stream (initialization, shuffles).
struct SplitMix {
    uint64_t s;
    uint64_t next() {
        uint64_t z = (s += 0x9E3779B97F4A7C15ull);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        return z ^ (z >> 31);
    }
    float uniform() { return (float)((next() >> 40) * (1.0 / 16777216.0)); }  // [0, 1)
};

}  // namespace

struct ml_card_model {
    ml_ctx* ctx = nullptr;
    std::unique_ptr<Reservation> res;  // declared first: released last
    DevBuf params, grads, adam_m, adam_v;
    DevBuf work;  // one batch: X, H1, H2, H3, out, y, and the gradients of H1..out; + loss
    int cap = 0;  // batch rows `work` holds
    int t = 0;    // Adam steps taken
    cudaStream_t s = nullptr;
    std::mutex mu;

    // Work layout for `cap` rows (floats).
    size_t off_x() const { return 0; }
    size_t off_h1() const { return off_x() + (size_t)cap * kCardFeatures; }
    size_t off_h2() const { return off_h1() + (size_t)cap * kCardHidden; }
    size_t off_h3() const { return off_h2() + (size_t)cap * kCardHidden; }
    size_t off_out() const { return off_h3() + (size_t)cap * kCardHidden; }
    size_t off_y() const { return off_out() + cap; }
    size_t off_dh1() const { return off_y() + cap; }
    size_t off_dh2() const { return off_dh1() + (size_t)cap * kCardHidden; }
    size_t off_dh3() const { return off_dh2() + (size_t)cap * kCardHidden; }
    size_t off_dout() const { return off_dh3() + (size_t)cap * kCardHidden; }
    size_t off_loss() const { return off_dout() + cap; }
    size_t work_floats() const { return off_loss() + 1; }
    float* w(size_t off) const { return work.get<float>() + off; }
    float* p(int off) const { return params.get<float>() + off; }
    float* g(int off) const { return grads.get<float>() + off; }

    void ensure(int rows) {
        if (rows <= cap) return;
        cap = std::max(rows, 256);
        work = DevBuf(ctx, work_floats() * 4, res.get());
    }
    void forward(int B) {
        launch_dense_fwd(w(off_x()), kCardFeatures, p(kW1), p(kB1), w(off_h1()), kCardHidden, B, true, s);
        launch_dense_fwd(w(off_h1()), kCardHidden, p(kW2), p(kB2), w(off_h2()), kCardHidden, B, true, s);
        launch_dense_fwd(w(off_h2()), kCardHidden, p(kW3), p(kB3), w(off_h3()), kCardHidden, B, true, s);
        launch_dense_fwd(w(off_h3()), kCardHidden, p(kW4), p(kB4), w(off_out()), 1, B, false, s);
        launch_add_column(w(off_out()), w(off_x()), B, kCardFeatures, kCardSkipFeature, kCardSkipScale, s);
        ctx->count_launch(5);
    }
    // Gradients of the mean squared error for the batch in work (forward already run).
    void backward(int B) {
        launch_mse_grad(w(off_out()), w(off_y()), w(off_dout()), w(off_loss()), B, s);
        launch_dense_bwd_params(w(off_h3()), kCardHidden, w(off_out()), 1, w(off_dout()), g(kW4), g(kB4), B, false, s);
        launch_dense_bwd_data(p(kW4), kCardHidden, w(off_out()), 1, w(off_dout()), w(off_dh3()), B, false, s);
        launch_dense_bwd_params(w(off_h2()), kCardHidden, w(off_h3()), kCardHidden, w(off_dh3()), g(kW3), g(kB3), B, true, s);
        launch_dense_bwd_data(p(kW3), kCardHidden, w(off_h3()), kCardHidden, w(off_dh3()), w(off_dh2()), B, true, s);
        launch_dense_bwd_params(w(off_h1()), kCardHidden, w(off_h2()), kCardHidden, w(off_dh2()), g(kW2), g(kB2), B, true, s);
        launch_dense_bwd_data(p(kW2), kCardHidden, w(off_h2()), kCardHidden, w(off_dh2()), w(off_dh1()), B, true, s);
        launch_dense_bwd_params(w(off_x()), kCardFeatures, w(off_h1()), kCardHidden, w(off_dh1()), g(kW1), g(kB1), B, true,
                                s);
        ctx->count_launch(8);
    }
    void adam(float lr) {
        t++;
        launch_adam(params.get<float>(), grads.get<float>(), adam_m.get<float>(), adam_v.get<float>(), kCardParams, lr,
                    0.9f, 0.999f, 1e-8f, t, s);
        ctx->count_launch();
    }
    void reset_adam() {
        CK(cudaMemsetAsync(adam_m.get(), 0, kCardParams * 4, s));
        CK(cudaMemsetAsync(adam_v.get(), 0, kCardParams * 4, s));
        t = 0;
    }
};

extern "C" {

int ml_gpu_card_features(ml_ctx* ctx, const ml_column* cols, int32_t ncols, int64_t nrows, const uint32_t* sel,
                         int64_t nsel, int32_t location, const ml_expr* keys, int32_t nkeys, float* features,
                         double* hll_estimate) {
    API_BEGIN
    REQUIRE(ctx && keys && features && nkeys > 0 && (cols || ncols == 0), "bad arguments");
    ctx->set_current();
    OpStream op_stream(ctx);
    cudaStream_t s = op_stream.s;
    std::vector<int32_t> types;
    for (int c = 0; c < ncols; c++) types.push_back(cols[c].dtype);
    Pipeline p(ctx);
    p.build(nullptr, 0, types.data(), ncols);
    KeyLayout L = p.key_layout(keys, nkeys, p.out, true, nullptr);
    p.upload();
    Staging st(ctx);
    DevBuf sel_hold;
    const uint32_t* dsel = sel;
    if (sel && location == ML_LOC_HOST) {
        for (int64_t i = 0; i < nsel; i++)
            if (sel[i] >= (uint64_t)nrows) raise(ML_ERR_INVALID, "selection index out of range");
        sel_hold = DevBuf(ctx, std::max<size_t>((size_t)nsel * 4, 4), nullptr);
        CK(cudaMemcpyAsync(sel_hold.get(), sel, (size_t)nsel * 4, cudaMemcpyHostToDevice, s));
        dsel = sel_hold.get<uint32_t>();
    }
    Pipeline::Launch La;
    p.prepare(La, cols, ncols, nrows, dsel, nsel, s, st, nullptr);
    for (size_t i = 0; i < p.C.slots.size(); i++)
        if (La.P.cols[i].kind == CK_UTF8 && La.P.cols[i].src == 0)
            raise(ML_ERR_UNSUPPORTED, "cardinality features of a plain (not dictionary-encoded) string key");
    const size_t bytes = kHllRegisters * 4 + 3 * 8;
    DevBuf buf(ctx, bytes, nullptr);
    CK(cudaMemsetAsync(buf.get(), 0, bytes, s));
    HllOut o;
    o.regs = buf.get<uint32_t>();
    o.nulls = (unsigned long long*)(buf.get<uint8_t>() + kHllRegisters * 4);
    o.minmax = o.nulls + 1;
    CK(cudaMemsetAsync(o.minmax, 0xFF, 8, s));  // min starts at ~0, max at 0
    void* jit = jit_hll_kernel(ctx, p, La.P, L);
    DevBuf cta_regs;
    {
        KernelTimer kt(ctx, s, "card_hll");
        if (jit && La.P.n) {
            const int smem = kHllRegisters * 4;
            const int64_t tiles = (La.P.n + 8 * kPipelineThreads - 1) / (8 * kPipelineThreads);
            const int grid = (int)std::min<int64_t>(tiles, (int64_t)jit_resident_blocks(jit, kPipelineThreads, smem) * num_sms());
            cta_regs = DevBuf(ctx, (size_t)grid * kHllRegisters, nullptr);
            uint32_t* cr = cta_regs.get<uint32_t>();
            void* args[] = {&La.P, &L, &cr, &o.nulls, &o.minmax};
            jit_launch(jit, grid, kPipelineThreads, smem, s, args);
            launch_hll_merge(cr, grid, o.regs, s);
            ctx->add_profile("jit_launch", 0);
            ctx->count_launch();
        } else {
            launch_hll(La.P, L, o, s);
        }
        kt.stop();
    }
    ctx->count_launch();
    std::vector<uint32_t> regs(kHllRegisters);
    uint64_t tail[3];
    CK(cudaMemcpyAsync(regs.data(), o.regs, kHllRegisters * 4, cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(tail, o.nulls, 24, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    const int64_t rows = La.P.n;
    const uint64_t nulls = tail[0], lo = tail[1], hi = tail[2];
    // features (the layout is documented with ml_gpu_card_features)
    std::fill(features, features + kCardFeatures, 0.0f);
    double harm = 0.0;
    uint32_t zeros = 0;
    for (uint32_t r : regs) {
        features[std::min<uint32_t>(r, 63)] += 1.0f / kHllRegisters;
        harm += std::ldexp(1.0, -(int)r);
        zeros += r == 0;
    }
    const double m = kHllRegisters;
    double est = 0.7213 / (1.0 + 1.079 / m) * m * m / harm;  // raw HyperLogLog estimate
    if (est <= 2.5 * m && zeros > 0) est = m * std::log(m / zeros);  // linear counting for small sets
    if (rows == 0) est = 0.0;
    const bool any_valid = rows > (int64_t)nulls;
    const double span = any_valid ? (double)(hi - lo) + 1.0 : 0.0;
    int bits = 0;
    for (int k = 0; k < L.nkeys; k++) bits += L.f[k].width;
    features[64] = (float)(std::log2((double)rows + 1.0) / 32.0);
    features[65] = (float)(std::log2(span + 1.0) / 64.0);
    features[66] = rows ? (float)((double)nulls / (double)rows) : 0.0f;
    features[67] = (float)(std::log2(est + 1.0) / 32.0);
    features[68] = (float)L.nkeys / 4.0f;
    features[69] = (float)bits / 128.0f;
    features[70] = (float)(std::log2(std::min((double)rows, span) + 1.0) / 32.0);
    features[71] = nulls ? 1.0f : 0.0f;
    if (hll_estimate) *hll_estimate = est;
    API_END
}

int ml_gpu_card_model_create(ml_ctx* ctx, uint64_t seed, ml_card_model** out) {
    API_BEGIN
    REQUIRE(ctx && out, "null argument");
    ctx->set_current();
    auto m = std::make_unique<ml_card_model>();
    m->ctx = ctx;
    m->res = std::make_unique<Reservation>(ctx, "CardinalityModel");
    m->s = ctx->new_stream();
    m->params = DevBuf(ctx, kCardParams * 4, m->res.get());
    m->grads = DevBuf(ctx, kCardParams * 4, m->res.get());
    m->adam_m = DevBuf(ctx, kCardParams * 4, m->res.get());
    m->adam_v = DevBuf(ctx, kCardParams * 4, m->res.get());
    std::vector<float> init(kCardParams);
    SplitMix rng{seed};
    auto fill = [&](int off, int n, int fan_in) {
        const float bound = 1.0f / std::sqrt((float)fan_in);
        for (int i = 0; i < n; i++) init[off + i] = (2.0f * rng.uniform() - 1.0f) * bound;
    };
    fill(kW1, kCardHidden * kCardFeatures, kCardFeatures);
    fill(kB1, kCardHidden, kCardFeatures);
    fill(kW2, kCardHidden * kCardHidden, kCardHidden);
    fill(kB2, kCardHidden, kCardHidden);
    fill(kW3, kCardHidden * kCardHidden, kCardHidden);
    fill(kB3, kCardHidden, kCardHidden);
    // the output layer starts at zero: an untrained model predicts the sketch's own estimate
    std::fill(init.begin() + kW4, init.end(), 0.0f);
    CK(cudaMemcpyAsync(m->params.get(), init.data(), kCardParams * 4, cudaMemcpyHostToDevice, m->s));
    m->reset_adam();
    CK(cudaStreamSynchronize(m->s));
    *out = m.release();
    API_END
}

int ml_gpu_card_model_params(ml_card_model* m, float* get, const float* set) {
    API_BEGIN
    REQUIRE(m, "null model");
    std::lock_guard<std::mutex> g(m->mu);
    m->ctx->set_current();
    if (get) CK(cudaMemcpyAsync(get, m->params.get(), kCardParams * 4, cudaMemcpyDeviceToHost, m->s));
    if (set) {
        CK(cudaMemcpyAsync(m->params.get(), set, kCardParams * 4, cudaMemcpyHostToDevice, m->s));
        m->reset_adam();
    }
    CK(cudaStreamSynchronize(m->s));
    API_END
}

int ml_gpu_card_model_step(ml_card_model* m, const float* x, const float* y, int32_t batch, float lr, float* loss) {
    API_BEGIN
    REQUIRE(m && x && y && batch > 0, "bad arguments");
    std::lock_guard<std::mutex> g(m->mu);
    m->ctx->set_current();
    m->ensure(batch);
    CK(cudaMemcpyAsync(m->w(m->off_x()), x, (size_t)batch * kCardFeatures * 4, cudaMemcpyHostToDevice, m->s));
    CK(cudaMemcpyAsync(m->w(m->off_y()), y, (size_t)batch * 4, cudaMemcpyHostToDevice, m->s));
    m->forward(batch);
    m->backward(batch);
    m->adam(lr);
    float l = 0;
    CK(cudaMemcpyAsync(&l, m->w(m->off_loss()), 4, cudaMemcpyDeviceToHost, m->s));
    CK(cudaStreamSynchronize(m->s));
    if (loss) *loss = l;
    API_END
}

int ml_gpu_card_model_train(ml_card_model* m, const float* x, const float* y, int64_t n, int32_t epochs, int32_t batch,
                            float lr, uint64_t seed, float* final_loss) {
    API_BEGIN
    REQUIRE(m && x && y && n > 0 && epochs > 0 && batch > 0 && n < 0x7FFFFFFF, "bad arguments");
    std::lock_guard<std::mutex> g(m->mu);
    Ctx* ctx = m->ctx;
    ctx->set_current();
    const int B = (int)std::min<int64_t>(batch, n);
    m->ensure(B);
    DevBuf dx(ctx, (size_t)n * kCardFeatures * 4, m->res.get()), dy(ctx, (size_t)n * 4, m->res.get());
    DevBuf didx(ctx, (size_t)n * 4, nullptr), dloss(ctx, 4 * (size_t)((n + B - 1) / B), nullptr);
    CK(cudaMemcpyAsync(dx.get(), x, (size_t)n * kCardFeatures * 4, cudaMemcpyHostToDevice, m->s));
    CK(cudaMemcpyAsync(dy.get(), y, (size_t)n * 4, cudaMemcpyHostToDevice, m->s));
    std::vector<uint32_t> order(n);
    SplitMix rng{seed};
    const int nb = (int)((n + B - 1) / B);
    std::vector<float> losses(nb);
    for (int e = 0; e < epochs; e++) {
        for (int64_t i = 0; i < n; i++) order[i] = (uint32_t)i;
        for (int64_t i = n - 1; i > 0; i--) std::swap(order[i], order[rng.next() % (uint64_t)(i + 1)]);  // Fisher-Yates
        CK(cudaMemcpyAsync(didx.get(), order.data(), (size_t)n * 4, cudaMemcpyHostToDevice, m->s));
        for (int b = 0; b < nb; b++) {
            const int rows = (int)std::min<int64_t>(B, n - (int64_t)b * B);
            const uint32_t* idx = didx.get<uint32_t>() + (size_t)b * B;
            launch_gather_rows(dx.get<float>(), idx, rows, kCardFeatures, m->w(m->off_x()), m->s);
            launch_gather_rows(dy.get<float>(), idx, rows, 1, m->w(m->off_y()), m->s);
            ctx->count_launch(2);
            m->forward(rows);
            m->backward(rows);
            CK(cudaMemcpyAsync(dloss.get<float>() + b, m->w(m->off_loss()), 4, cudaMemcpyDeviceToDevice, m->s));
            m->adam(lr);
        }
        // the host order buffer is reused by the next epoch: wait for this epoch's copy of it
        CK(cudaStreamSynchronize(m->s));
    }
    CK(cudaMemcpyAsync(losses.data(), dloss.get(), (size_t)nb * 4, cudaMemcpyDeviceToHost, m->s));
    CK(cudaStreamSynchronize(m->s));
    double mean = 0;
    for (float l : losses) mean += l;
    if (final_loss) *final_loss = (float)(mean / nb);
    API_END
}

int ml_gpu_card_model_predict(ml_card_model* m, const float* x, int64_t n, float* out) {
    API_BEGIN
    REQUIRE(m && x && out && n >= 0, "bad arguments");
    std::lock_guard<std::mutex> g(m->mu);
    m->ctx->set_current();
    const int chunk = 4096;
    m->ensure((int)std::min<int64_t>(n, chunk));
    for (int64_t b = 0; b < n; b += chunk) {
        const int rows = (int)std::min<int64_t>(chunk, n - b);
        CK(cudaMemcpyAsync(m->w(m->off_x()), x + b * kCardFeatures, (size_t)rows * kCardFeatures * 4,
                           cudaMemcpyHostToDevice, m->s));
        m->forward(rows);
        CK(cudaMemcpyAsync(out + b, m->w(m->off_out()), (size_t)rows * 4, cudaMemcpyDeviceToHost, m->s));
        CK(cudaStreamSynchronize(m->s));
    }
    API_END
}

int ml_gpu_card_model_destroy(ml_card_model* m) {
    API_BEGIN
    if (m) {
        m->ctx->set_current();
        CK(cudaStreamSynchronize(m->s));
        m->ctx->free_stream(m->s);
        delete m;
    }
    API_END
}

}  // extern "C"
