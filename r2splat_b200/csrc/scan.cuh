// Device-wide prefix sums used by the intersection pipeline and the radix
// sort: reduce per block -> scan block totals (recursively) -> scan + offset.
#pragma once

#include "common.cuh"

namespace r2s {

constexpr int kScanThreads = 512;
constexpr int kScanItems = 8;
constexpr int64_t kScanTile = int64_t(kScanThreads) * kScanItems;

template <typename T>
__device__ __forceinline__ T block_exclusive_scan(T value, T& total) {
    __shared__ T warp_totals[kScanThreads / 32];
    __shared__ T grand_total;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    T inclusive = value;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        T other = __shfl_up_sync(0xffffffffu, inclusive, off);
        if (lane >= off) inclusive += other;
    }
    if (lane == 31) warp_totals[warp] = inclusive;
    __syncthreads();
    if (warp == 0) {
        T w = lane < kScanThreads / 32 ? warp_totals[lane] : T(0);
        T winc = w;
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
            T other = __shfl_up_sync(0xffffffffu, winc, off);
            if (lane >= off) winc += other;
        }
        if (lane < kScanThreads / 32) warp_totals[lane] = winc - w;
        if (lane == kScanThreads / 32 - 1) grand_total = winc;
    }
    __syncthreads();
    total = grand_total;
    T result = warp_totals[warp] + inclusive - value;
    __syncthreads();
    return result;
}

template <typename In, typename Out>
__global__ void __launch_bounds__(kScanThreads) scan_reduce_kernel(const In* __restrict__ in, int64_t n,
                                                                  Out* __restrict__ block_totals) {
    const int64_t base = int64_t(blockIdx.x) * kScanTile + int64_t(threadIdx.x) * kScanItems;
    Out sum = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        const int64_t i = base + k;
        if (i < n) sum += static_cast<Out>(in[i]);
    }
    Out total;
    block_exclusive_scan<Out>(sum, total);
    if (threadIdx.x == 0) block_totals[blockIdx.x] = total;
}

// Scans one tile per block; offsets (exclusive block prefixes) may be null.
template <typename In, typename Out, bool kInclusive>
__global__ void __launch_bounds__(kScanThreads) scan_tile_kernel(const In* in, int64_t n,
                                                                const Out* __restrict__ offsets, Out* out) {
    const int64_t base = int64_t(blockIdx.x) * kScanTile + int64_t(threadIdx.x) * kScanItems;
    Out items[kScanItems];
    Out sum = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        const int64_t i = base + k;
        items[k] = i < n ? static_cast<Out>(in[i]) : Out(0);
        sum += items[k];
    }
    Out total;
    Out running = block_exclusive_scan<Out>(sum, total);
    if (offsets != nullptr) running += offsets[blockIdx.x];
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        const int64_t i = base + k;
        if (kInclusive) running += items[k];
        if (i < n) out[i] = running;
        if (!kInclusive) running += items[k];
    }
}

// Workspace bytes for scanning n elements of type Out.
template <typename Out>
constexpr size_t scan_workspace_bytes(int64_t n) {
    size_t bytes = 0;
    while (n > kScanTile) {
        const int64_t nb = (n + kScanTile - 1) / kScanTile;
        bytes += ((size_t(nb) * sizeof(Out) + 255) & ~size_t(255));
        n = nb;
    }
    return bytes + 256;
}

// out[i] = sum(in[0..i]) (inclusive) or sum(in[0..i)) (exclusive).
template <typename In, typename Out, bool kInclusive>
inline int device_scan(const In* in, Out* out, int64_t n, void* ws, size_t ws_bytes, cudaStream_t stream) {
    if (n <= 0) return R2S_OK;
    if (n <= kScanTile) {
        scan_tile_kernel<In, Out, kInclusive><<<1, kScanThreads, 0, stream>>>(in, n, nullptr, out);
        return check_launch("scan_tile");
    }
    const int64_t nb = (n + kScanTile - 1) / kScanTile;
    R2S_REQUIRE(nb < (int64_t(1) << 31), R2S_ERR_UNSUPPORTED, "scan too large");
    Arena arena(ws, ws_bytes);
    Out* totals = arena.take<Out>(size_t(nb));
    R2S_REQUIRE(totals != nullptr, R2S_ERR_WORKSPACE, "scan workspace too small");
    scan_reduce_kernel<In, Out><<<unsigned(nb), kScanThreads, 0, stream>>>(in, n, totals);
    R2S_TRY(check_launch("scan_reduce"));
    // Exclusive scan of the block totals, in place, using the rest of the workspace.
    R2S_TRY((device_scan<Out, Out, false>(totals, totals, nb, arena.base + arena.used, arena.size - arena.used,
                                          stream)));
    scan_tile_kernel<In, Out, kInclusive><<<unsigned(nb), kScanThreads, 0, stream>>>(in, n, totals, out);
    return check_launch("scan_tile");
}

}  // namespace r2s
