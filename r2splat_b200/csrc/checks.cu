// Batched input value checks: one launch evaluates every finiteness / range /
// structure check that input validation needs and ORs one flag bit per failed
// check, so the host reads a single word instead of synchronising once per
// check (the reference's _validation.py evaluates each with its own
// torch reduction and host read).
#include "common.cuh"

namespace r2s {

constexpr uint32_t kMaxChecks = 32;

struct CheckList {
    r2s_value_check item[kMaxChecks];
    uint32_t count;
};

template <typename S>
__device__ __forceinline__ bool element_fails(const S* data, uint64_t i, uint32_t kind) {
    switch (kind) {
        case R2S_CHECK_FINITE:
            return !isfinite(data[i]);
        case R2S_CHECK_ZERO_ROW4: {
            const S* row = data + 4 * i;
            return row[0] == S(0) && row[1] == S(0) && row[2] == S(0) && row[3] == S(0);
        }
        case R2S_CHECK_POSITIVE:
            return data[i] <= S(0);
        case R2S_CHECK_NONNEGATIVE:
            return data[i] < S(0);
        case R2S_CHECK_FOCAL: {
            const S* k = data + 9 * i;
            return k[0] <= S(0) || k[4] <= S(0);
        }
        case R2S_CHECK_PINHOLE: {
            const S* k = data + 9 * i;
            return k[1] != S(0) || k[3] != S(0) || k[6] != S(0) || k[7] != S(0) || k[8] != S(1);
        }
        case R2S_CHECK_HOMOGENEOUS_ROW: {
            const S* m = data + 16 * i;
            return !(m[12] == S(0) && m[13] == S(0) && m[14] == S(0) && m[15] == S(1));
        }
        default:
            return true;
    }
}

// 16-byte vectors of S for the finiteness scan.
template <typename S> struct Vec16;
template <> struct Vec16<float> { using type = float4; };
template <> struct Vec16<double> { using type = double2; };

__device__ __forceinline__ bool any_nonfinite(const float4& v) {
    return !(isfinite(v.x) && isfinite(v.y) && isfinite(v.z) && isfinite(v.w));
}
__device__ __forceinline__ bool any_nonfinite(const double2& v) { return !(isfinite(v.x) && isfinite(v.y)); }

// grid.y = check index; grid.x strides over that check's elements. The
// finiteness check of 16-byte-aligned data (the image and volume adjoints,
// hundreds of MB) reads 16-byte vectors, four in flight per thread; the other
// checks read element by element.
template <typename S>
__global__ void check_values_kernel(CheckList list, uint32_t* __restrict__ flags) {
    const uint32_t c = blockIdx.y;
    if (c >= list.count) return;
    const r2s_value_check chk = list.item[c];
    const S* data = static_cast<const S*>(chk.data);
    const uint64_t tid = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
    bool bad = false;
    if (chk.kind == R2S_CHECK_FINITE && (reinterpret_cast<uintptr_t>(data) & 15u) == 0u) {
        using V = typename Vec16<S>::type;
        constexpr uint64_t kPer = sizeof(V) / sizeof(S);
        const V* vec = reinterpret_cast<const V*>(data);
        const uint64_t nv = chk.count / kPer;
        uint64_t i = tid;
        for (; i + 3 * stride < nv; i += 4 * stride) {
            const V a = vec[i], b = vec[i + stride], d = vec[i + 2 * stride], e = vec[i + 3 * stride];
            bad |= any_nonfinite(a) | any_nonfinite(b) | any_nonfinite(d) | any_nonfinite(e);
        }
        for (; i < nv; i += stride) bad |= any_nonfinite(vec[i]);
        for (uint64_t t = nv * kPer + tid; t < chk.count; t += stride) bad |= !isfinite(data[t]);
    } else {
        for (uint64_t i = tid; i < chk.count; i += stride) bad |= element_fails(data, i, chk.kind);
    }
    if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31u) == 0u) atomicOr(flags, 1u << chk.bit);
}

}  // namespace r2s

using namespace r2s;

extern "C" {

int r2s_check_values(int dtype, const r2s_value_check* checks, uint32_t n_checks, uint32_t* flags, void* stream) {
    R2S_REQUIRE(n_checks <= kMaxChecks, R2S_ERR_UNSUPPORTED, "at most 32 checks per call");
    R2S_REQUIRE(flags != nullptr, R2S_ERR_ARGUMENT, "flags must be non-null");
    CheckList list{};
    uint64_t longest = 0;
    for (uint32_t c = 0; c < n_checks; ++c) {
        R2S_REQUIRE(checks[c].bit < 32u, R2S_ERR_ARGUMENT, "check bit must be below 32");
        R2S_REQUIRE(checks[c].kind <= R2S_CHECK_HOMOGENEOUS_ROW, R2S_ERR_ARGUMENT, "unknown check kind");
        R2S_REQUIRE(checks[c].count == 0 || checks[c].data != nullptr, R2S_ERR_ARGUMENT, "check data is null");
        list.item[c] = checks[c];
        if (checks[c].count > longest) longest = checks[c].count;
    }
    list.count = n_checks;
    cudaStream_t st = as_stream(stream);
    if (cudaMemsetAsync(flags, 0, sizeof(uint32_t), st) != cudaSuccess) return fail(R2S_ERR_CUDA, "memset failed");
    if (n_checks == 0 || longest == 0) return R2S_OK;
    const unsigned threads = 256;
    uint64_t blocks = (longest + threads - 1) / threads;
    if (blocks > 1184) blocks = 1184;
    dim3 grid(unsigned(blocks), n_checks);
    R2S_DISPATCH(dtype, check_values_kernel<S><<<grid, threads, 0, st>>>(list, flags));
    return check_launch("check_values");
}

}  // extern "C"
