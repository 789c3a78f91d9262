// Shared by the C-ABI translation units: the context handle and the status wrappers.
#pragma once

#include <chrono>

#include "ml_runtime.hpp"

struct ml_ctx : mlg::Ctx {
    using mlg::Ctx::Ctx;
};

// The stream of one standalone operator call (filter, projection, probe, hashing, upload),
// taken from the context's pool: MiniLake calls Operator::execute on one shared operator from
// every worker thread (pipeline.rs:52-57), so calls from different threads run concurrently on
// the device.  The call's work is finished when it returns.
struct OpStream {
    mlg::Ctx* ctx;
    cudaStream_t s;
    explicit OpStream(mlg::Ctx* c) : ctx(c), s(c->new_stream()) {}
    ~OpStream() {
        cudaStreamSynchronize(s);
        ctx->free_stream(s);
    }
    OpStream(const OpStream&) = delete;
};

// Every entry point returns a status: exceptions become ML_* codes with the message kept
// for ml_gpu_last_error().
#define API_BEGIN try {
#define API_END                                       \
    }                                                 \
    catch (const mlg::MlError& e) {                   \
        mlg::set_last_error(e.what());                \
        return e.code;                                \
    }                                                 \
    catch (const std::bad_alloc&) {                   \
        mlg::set_last_error("host allocation failed"); \
        return ML_ERR_INTERNAL;                       \
    }                                                 \
    catch (const std::exception& e) {                 \
        mlg::set_last_error(e.what());                \
        return ML_ERR_INTERNAL;                       \
    }                                                 \
    return ML_OK;

#define REQUIRE(c, msg) \
    if (!(c)) mlg::raise(ML_ERR_INVALID, msg)

// Host time of one C-ABI call, recorded as "host:<name>" when the context profiles.
struct HostTimer {
    mlg::Ctx* ctx;
    const char* name;
    std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();
    HostTimer(mlg::Ctx* c, const char* n) : ctx(c), name(n) {}
    ~HostTimer() {
        if (ctx && ctx->profiling())
            ctx->add_profile(name, std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count());
    }
};
