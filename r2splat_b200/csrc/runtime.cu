// Library-wide host runtime: error reporting and identification.
#include "common.cuh"

#include <atomic>
#include <string>

namespace r2s {

namespace {
thread_local std::string t_last_error;
std::atomic<uint64_t> g_launches{0};
}

void set_error(const std::string& message) { t_last_error = message; }

int fail(int code, const std::string& message) {
    t_last_error = message;
    return code;
}

// Converts a pending launch error into an R2S_ERR_CUDA status. Every kernel
// launch of the library is followed by exactly one call, which also counts it.
int check_launch(const char* what) {
    g_launches.fetch_add(1, std::memory_order_relaxed);
    cudaError_t err = cudaGetLastError();
    if (err != cudaSuccess) {
        return fail(R2S_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(err));
    }
    return R2S_OK;
}

// FP32 issue-rate probe: every thread runs 8 independent FMA chains, so the
// kernel is bound by the FMA pipe; 2 flops per FMA.
__global__ void fp32_peak_kernel(float* out, int iters, float seed) {
    float a0 = seed + threadIdx.x, a1 = a0 + 1.f, a2 = a0 + 2.f, a3 = a0 + 3.f;
    float a4 = a0 + 4.f, a5 = a0 + 5.f, a6 = a0 + 6.f, a7 = a0 + 7.f;
    const float m = 0.9999f, c = 1e-7f;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int u = 0; u < 16; ++u) {
            a0 = fmaf(a0, m, c); a1 = fmaf(a1, m, c); a2 = fmaf(a2, m, c); a3 = fmaf(a3, m, c);
            a4 = fmaf(a4, m, c); a5 = fmaf(a5, m, c); a6 = fmaf(a6, m, c); a7 = fmaf(a7, m, c);
        }
    }
    const float s = a0 + a1 + a2 + a3 + a4 + a5 + a6 + a7;
    if (s == 1234.5f) out[blockIdx.x] = s;  // keeps the chains live
}

// SFU (MUFU) issue probe: 8 independent chains x = 2^(-x) per thread. The
// fast exponential compiles to one ex2 per step; x stays in (0, 1).
__global__ void sfu_peak_kernel(float* out, int iters, float seed) {
    float x[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) x[k] = seed * float(k + 1) / 8.f + 1e-3f * float(threadIdx.x & 7);
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int u = 0; u < 16; ++u) {
#pragma unroll
            for (int k = 0; k < 8; ++k) x[k] = exp2f(-x[k]);
        }
    }
    float s = 0.f;
#pragma unroll
    for (int k = 0; k < 8; ++k) s += x[k];
    if (s == 1234.5f) out[blockIdx.x] = s;  // keeps the chains live
}

}  // namespace r2s

extern "C" {

int r2s_abi_version(void) { return 1; }

uint64_t r2s_launch_count(void) { return r2s::g_launches.load(std::memory_order_relaxed); }

// Launches the FP32 peak probe: blocks x threads x iters x 128 FMAs.
int r2s_fp32_peak_probe(float* out, uint32_t blocks, uint32_t threads, int iters, void* stream) {
    r2s::fp32_peak_kernel<<<blocks, threads, 0, static_cast<cudaStream_t>(stream)>>>(out, iters, 0.5f);
    return r2s::check_launch("fp32_peak_probe");
}

// Launches the SFU peak probe: blocks x threads x iters x 128 ex2.
int r2s_sfu_peak_probe(float* out, uint32_t blocks, uint32_t threads, int iters, void* stream) {
    r2s::sfu_peak_kernel<<<blocks, threads, 0, static_cast<cudaStream_t>(stream)>>>(out, iters, 0.5f);
    return r2s::check_launch("sfu_peak_probe");
}

const char* r2s_last_error(void) { return r2s::t_last_error.c_str(); }

}  // extern "C"
