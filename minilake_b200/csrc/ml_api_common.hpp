// Shared by the C-ABI translation units: the context handle and the status wrappers.
#pragma once

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
