// Shared by the C-ABI translation units: the context handle and the status wrappers.
#pragma once

#include <chrono>

#include "ml_runtime.hpp"

struct ml_ctx : mlg::Ctx {
    using mlg::Ctx::Ctx;
    std::mutex op_mu;  // serializes the standalone operators on the context stream
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
