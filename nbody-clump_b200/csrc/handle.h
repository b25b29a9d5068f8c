// handle.h -- the C ABI's engine handle and its error plumbing, shared by
// the entry points of capi.cpp and serve.cpp.
#pragma once
#include <memory>
#include <stdexcept>
#include <string>

#include "../../include/nbc.h"
#include "engine.h"
#include "io.h"

namespace nbc {
extern thread_local std::string g_last_error;
}

struct nbc_engine {
    std::unique_ptr<nbc::EngineBase> eng;
    std::unique_ptr<nbc::Workdir> wd;  // set by nbc_open
    nbc_options opt;
};

namespace nbc {

inline nbc_status fail(nbc_status code, const std::string& msg) {
    g_last_error = msg;
    return code;
}

// runs f, turning the engine's exceptions into status codes
template <typename F>
nbc_status guard(F&& f) {
    try {
        f();
        return NBC_OK;
    } catch (const NonFinite& e) {
        return fail(NBC_ERR_NONFINITE, e.what());
    } catch (const StateError& e) {
        return fail(NBC_ERR_STATE, e.what());
    } catch (const std::bad_alloc& e) {
        return fail(NBC_ERR_MEMORY, e.what());
    } catch (const std::invalid_argument& e) {
        return fail(NBC_ERR_ARG, e.what());
    } catch (const std::runtime_error& e) {
        std::string m = e.what();
        if (m.find("no CUDA device") != std::string::npos) return fail(NBC_ERR_NO_DEVICE, m);
        if (m.find("cudaMalloc") != std::string::npos) return fail(NBC_ERR_MEMORY, m);
        if (m.find("scene ") == 0 || m.find("buffer too small") != std::string::npos ||
            m.find("longer than") != std::string::npos || m.find("too many") != std::string::npos)
            return fail(NBC_ERR_ARG, m);
        return fail(NBC_ERR_CUDA, m);
    } catch (...) {
        return fail(NBC_ERR_CUDA, "unknown error");
    }
}

}  // namespace nbc
