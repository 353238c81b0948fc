// Library-wide host runtime: error reporting and identification.
#include "common.cuh"

#include <string>

namespace r2s {

namespace {
thread_local std::string t_last_error;
}

void set_error(const std::string& message) { t_last_error = message; }

int fail(int code, const std::string& message) {
    t_last_error = message;
    return code;
}

// Converts a pending launch error into an R2S_ERR_CUDA status.
int check_launch(const char* what) {
    cudaError_t err = cudaGetLastError();
    if (err != cudaSuccess) {
        return fail(R2S_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(err));
    }
    return R2S_OK;
}

}  // namespace r2s

extern "C" {

int r2s_abi_version(void) { return 1; }

const char* r2s_last_error(void) { return r2s::t_last_error.c_str(); }

}  // extern "C"
