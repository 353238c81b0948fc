// Shared device/host helpers for the r2splat_b200 sm_100a library.
//
// The library is a plain C-ABI shared object: every entry point takes raw
// device pointers, sizes and a cudaStream_t, never allocates, and reports
// failures through an integer status plus r2s_last_error().
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <stddef.h>

#include <string>

#include "../../include/r2splat_b200.h"

namespace r2s {

// ---------------------------------------------------------------------------
// Error reporting (host)
// ---------------------------------------------------------------------------

void set_error(const std::string& message);
int fail(int code, const std::string& message);
int check_launch(const char* what);

#define R2S_REQUIRE(cond, code, msg)             \
    do {                                         \
        if (!(cond)) return ::r2s::fail((code), (msg)); \
    } while (0)

#define R2S_TRY(expr)                            \
    do {                                         \
        int _r2s_status = (expr);                \
        if (_r2s_status != R2S_OK) return _r2s_status; \
    } while (0)

// Workspace carving: the caller passes one byte buffer; kernels take slices.
struct Arena {
    char* base;
    size_t size;
    size_t used;
    __host__ explicit Arena(void* p, size_t n) : base(static_cast<char*>(p)), size(n), used(0) {}
    template <typename T>
    __host__ T* take(size_t count) {
        if (base == nullptr) return nullptr;
        const uintptr_t start = reinterpret_cast<uintptr_t>(base) + used;
        const size_t offset = used + (((start + 255) & ~uintptr_t(255)) - start);
        const size_t bytes = count * sizeof(T);
        if (offset + bytes > size) return nullptr;
        used = offset + bytes;
        return reinterpret_cast<T*>(base + offset);
    }
};

// Size accounting mirror of Arena::take.
struct ArenaSize {
    size_t used = 0;
    template <typename T>
    __host__ void take(size_t count) {
        used = ((used + 255) & ~size_t(255)) + count * sizeof(T);
    }
    __host__ size_t bytes() const { return used + 256; }
};

// Runs the statement(s) with S bound to the element type of the dtype tag.
#define R2S_DISPATCH(dtype, ...)                                                    \
    do {                                                                            \
        if ((dtype) == R2S_F32) {                                                   \
            using S = float;                                                        \
            __VA_ARGS__;                                                            \
        } else if ((dtype) == R2S_F64) {                                            \
            using S = double;                                                       \
            __VA_ARGS__;                                                            \
        } else {                                                                    \
            return ::r2s::fail(R2S_ERR_ARGUMENT, "dtype must be R2S_F32 or R2S_F64");      \
        }                                                                           \
    } while (0)

inline cudaStream_t as_stream(void* s) { return static_cast<cudaStream_t>(s); }

inline unsigned blocks_for(int64_t n, unsigned threads) {
    int64_t b = (n + threads - 1) / threads;
    if (b < 1) b = 1;
    return static_cast<unsigned>(b);
}

// ---------------------------------------------------------------------------
// Device helpers
// ---------------------------------------------------------------------------

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ uint64_t global_timer_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
    return t;
}

// Asynchronous 16-byte global->shared copy (LDGSTS); used to gather
// per-primitive records into shared memory while the previous batch computes.
__device__ __forceinline__ void cp_async16(void* smem_dst, const void* gmem_src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n"
                 :: "r"(smem_u32(smem_dst)), "l"(gmem_src) : "memory");
}
// 4- and 8-byte forms (L1-allocating .ca, the only one these sizes allow).
__device__ __forceinline__ void cp_async4(void* smem_dst, const void* gmem_src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n"
                 :: "r"(smem_u32(smem_dst)), "l"(gmem_src) : "memory");
}
__device__ __forceinline__ void cp_async8(void* smem_dst, const void* gmem_src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n"
                 :: "r"(smem_u32(smem_dst)), "l"(gmem_src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
    asm volatile("cp.async.commit_group;\n" ::: "memory");
}
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;\n" :: "n"(N) : "memory");
}

// Bulk global->shared copies completed on a shared-memory mbarrier (the
// non-tensor form of TMA, sm_90+): one thread arms the barrier with the byte
// count and issues one copy of a contiguous range; every thread then waits on
// the barrier's phase. Source and destination must be 16-byte aligned and the
// size a multiple of 16. Only this GPU's own memory is read, never with
// cluster multicast.
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" :: "r"(smem_u32(bar)), "r"(count) : "memory");
}
// Makes the initialised barriers visible to the bulk-copy unit.
__device__ __forceinline__ void mbar_init_fence() {
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n"
                 :: "r"(smem_u32(bar)), "r"(bytes) : "memory");
}
// Orders this thread's earlier shared-memory accesses (and, after a block
// barrier, the block's) before later bulk copies into shared memory.
__device__ __forceinline__ void fence_proxy_async_shared() {
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
}
__device__ __forceinline__ void bulk_load_g2s(void* smem_dst, const void* gmem_src, uint32_t bytes, uint64_t* bar) {
    asm volatile("cp.async.bulk.shared::cta.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n"
                 :: "r"(smem_u32(smem_dst)), "l"(gmem_src), "r"(bytes), "r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t done;
    asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
                 " selp.u32 %0, 1, 0, p;\n}\n"
                 : "=r"(done) : "r"(smem_u32(bar)), "r"(parity) : "memory");
    return done != 0u;
}
// A staging copy of a few KB completes in microseconds; a wait that has not
// seen its phase complete after this long gives up.
constexpr uint64_t kBulkWaitLimitNs = 200ull * 1000ull * 1000ull;
// Waits for the barrier's phase with the given parity; false when it did not
// complete within kBulkWaitLimitNs.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity) {
    if (mbar_try_wait(bar, parity)) return true;
    const uint64_t t0 = global_timer_ns();
    while (!mbar_try_wait(bar, parity)) {
        if (global_timer_ns() - t0 > kBulkWaitLimitNs) return false;
    }
    return true;
}

// Vector reductions into global memory (sm_90+ red.global.add.v4.f32).
__device__ __forceinline__ void red_add_v4(float* addr, float a, float b, float c, float d) {
    asm volatile("red.global.add.v4.f32 [%0], {%1, %2, %3, %4};\n"
                 :: "l"(addr), "f"(a), "f"(b), "f"(c), "f"(d) : "memory");
}
__device__ __forceinline__ void red_add_v4(double* addr, double a, double b, double c, double d) {
    atomicAdd(addr + 0, a);
    atomicAdd(addr + 1, b);
    atomicAdd(addr + 2, c);
    atomicAdd(addr + 3, d);
}
__device__ __forceinline__ void red_add_v2(float* addr, float a, float b) {
    asm volatile("red.global.add.v2.f32 [%0], {%1, %2};\n" :: "l"(addr), "f"(a), "f"(b) : "memory");
}
__device__ __forceinline__ void red_add_v2(double* addr, double a, double b) {
    atomicAdd(addr + 0, a);
    atomicAdd(addr + 1, b);
}
__device__ __forceinline__ void red_add(float* addr, float v) { atomicAdd(addr, v); }
__device__ __forceinline__ void red_add(double* addr, double v) { atomicAdd(addr, v); }

template <typename S>
__device__ __forceinline__ S warp_sum(S v) {
#pragma unroll
    for (int offset = 16; offset > 0; offset >>= 1) v += __shfl_xor_sync(0xffffffffu, v, offset);
    return v;
}

// Sum of eight per-lane values over each group of kLanes lanes (32: the warp;
// 16 or 8: each half or quarter of it) by recursive halving: each exchange step sends half of
// the lane's values to its partner and keeps the other half, so a warp-wide
// reduction costs 4 + 2 + 2 * 3 shuffles instead of 8 * 5. On return every
// lane of subgroup G = (lane % kLanes) / (kLanes / 4) holds its group's totals
// of values 2G and 2G + 1 in (out0, out1).
template <uint32_t kLanes = 32u, typename S>
__device__ __forceinline__ void warp_sum8_pairs(const S (&v)[8], S& out0, S& out1) {
    static_assert(kLanes == 32u || kLanes == 16u || kLanes == 8u, "groups of 32, 16 or 8 lanes");
    const uint32_t lane = threadIdx.x & 31u;
    const bool upper = (lane & (kLanes / 2u)) != 0;
    S w[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const S send = upper ? v[i] : v[i + 4];
        const S keep = upper ? v[i + 4] : v[i];
        w[i] = keep + __shfl_xor_sync(0xffffffffu, send, kLanes / 2u);
    }
    const bool upper2 = (lane & (kLanes / 4u)) != 0;
    S u[2];
#pragma unroll
    for (int i = 0; i < 2; ++i) {
        const S send = upper2 ? w[i] : w[i + 2];
        const S keep = upper2 ? w[i + 2] : w[i];
        u[i] = keep + __shfl_xor_sync(0xffffffffu, send, kLanes / 4u);
    }
#pragma unroll
    for (int offset = kLanes / 8u; offset > 0; offset >>= 1) {
        u[0] += __shfl_xor_sync(0xffffffffu, u[0], offset);
        u[1] += __shfl_xor_sync(0xffffffffu, u[1], offset);
    }
    out0 = u[0];
    out1 = u[1];
}

// Packed FP32x2 arithmetic (sm_100 FADD2 / FMUL2 / FFMA2): one instruction
// evaluates two independent samples, each component rounded like the scalar
// operation (round to nearest even).
__device__ __forceinline__ float2 splat2(float a) { return make_float2(a, a); }
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }

// Scalar multiply that the compiler may not contract into a following add:
// the per-sample expressions below spell out which products round on their own.
template <typename S>
__device__ __forceinline__ S mul_rn(S a, S b) {
    if constexpr (sizeof(S) == 4) {
        return __fmul_rn(a, b);
    } else {
        return __dmul_rn(a, b);
    }
}

// 1.0f when a > b, else 0.0f (also 0.0f when either is NaN), as one PTX set.
__device__ __forceinline__ float gt_mask(float a, float b) {
    float m;
    asm("set.gt.f32.f32 %0, %1, %2;" : "=f"(m) : "f"(a), "f"(b));
    return m;
}

// Raises a kernel's dynamic shared-memory limit when a launch needs more than
// the default 48 KB in all (its dynamic bytes plus `static_bytes` of static
// shared memory).
template <typename Kernel>
inline int allow_dynamic_smem(Kernel kernel, size_t bytes, size_t static_bytes = 0) {
    if (bytes + static_bytes <= 48 * 1024) return R2S_OK;
    const cudaError_t err =
        cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(bytes));
    if (err != cudaSuccess)
        return fail(R2S_ERR_CUDA, std::string("cudaFuncSetAttribute(dynamic smem): ") + cudaGetErrorString(err));
    return R2S_OK;
}

// Packed per-(camera, primitive) record consumed by the tile kernels.
// Slot meaning: projected centre (x, y), 2x2 conic (a, b, c), density o,
// path factor mu, and the projected Beta exponent (beta + 1/2) for Beta
// primitives (unused otherwise).
template <typename S>
struct alignas(16) Rec2D {
    S x, y, a, b, c, o, mu, beta;
};

// Packed per-primitive record for voxel tiles: voxel-space centre, density,
// the 3x3 conic (c00, c01, c02, c11, c12, c22), the Beta exponent, and the
// uncertainty (relative variance).
template <typename S>
struct alignas(16) Rec3D {
    S x, y, z, o, c00, c01, c02, c11, c12, c22, beta, q, pad0, pad1, pad2, pad3;
};

// Defined in loss.cu: fixed-order sum of fp64 partials into a mean and lambda * mean.
int launch_finish_mean(int dtype, const double* partials, int n_partials, int64_t count, float lambda, void* loss,
                       void* value, cudaStream_t stream);

}  // namespace r2s
