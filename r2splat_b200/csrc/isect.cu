// Tile intersection: per-element tile counts, prefix sum, emission of
// (key, element) pairs, a stable LSD radix sort, and per-key offsets.
//
// Ordering contract (IsectTilesKernel.cu:137-217 + the stable radix sort at
// :398-445): within one key the elements appear in ascending element order.
// Emission writes each element's pairs contiguously at its prefix-sum slot
// in ascending element order, and the sort is stable, so any run of equal
// keys keeps ascending element order -- the same arrays the reference's
// CUB-sorted output holds.
#include "geometry.cuh"
#include "scan.cuh"

namespace r2s {

constexpr unsigned kIsectThreads = 256;

// ----------------------------------------------------------------- counting

template <typename S>
__device__ __forceinline__ bool rect_2d(const S* means2d, const int32_t* radii, bool rect, size_t idx,
                                        uint32_t tile_size, uint32_t tiles_x, uint32_t tiles_y, uint32_t& x0,
                                        uint32_t& x1, uint32_t& y0, uint32_t& y1) {
    const S radius_x = static_cast<S>(rect ? radii[2 * idx] : radii[idx]);
    const S radius_y = static_cast<S>(rect ? radii[2 * idx + 1] : radii[idx]);
    if (radius_x <= 0 || radius_y <= 0) return false;
    const S mean_x = means2d[2 * idx];
    const S mean_y = means2d[2 * idx + 1];
    if (!isfinite(mean_x) || !isfinite(mean_y)) return false;
    tile_span(mean_x, radius_x, tile_size, tiles_x, x0, x1);
    tile_span(mean_y, radius_y, tile_size, tiles_y, y0, y1);
    return x1 > x0 && y1 > y0;
}

template <typename S>
__device__ __forceinline__ bool rect_3d(const S* means3d, const int32_t* radii, size_t idx, uint32_t tile_size,
                                        uint32_t tx, uint32_t ty, uint32_t tz, uint32_t* lo, uint32_t* hi) {
    const S rx = static_cast<S>(radii[3 * idx]);
    const S ry = static_cast<S>(radii[3 * idx + 1]);
    const S rz = static_cast<S>(radii[3 * idx + 2]);
    if (rx <= 0 || ry <= 0 || rz <= 0) return false;
    tile_span(means3d[3 * idx + 0], rx, tile_size, tx, lo[0], hi[0]);
    tile_span(means3d[3 * idx + 1], ry, tile_size, ty, lo[1], hi[1]);
    tile_span(means3d[3 * idx + 2], rz, tile_size, tz, lo[2], hi[2]);
    return hi[0] > lo[0] && hi[1] > lo[1] && hi[2] > lo[2];
}

template <typename S>
__global__ void count_2d_kernel(const S* __restrict__ means2d, const int32_t* __restrict__ radii, bool rect,
                                uint32_t total, uint32_t tile_size, uint32_t tiles_x, uint32_t tiles_y,
                                int32_t* __restrict__ counts) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= total) return;
    uint32_t x0, x1, y0, y1;
    counts[i] = rect_2d(means2d, radii, rect, i, tile_size, tiles_x, tiles_y, x0, x1, y0, y1)
                    ? static_cast<int32_t>((y1 - y0) * (x1 - x0)) : 0;
}

template <typename S>
__global__ void count_3d_kernel(const S* __restrict__ means3d, const int32_t* __restrict__ radii, uint32_t N,
                                uint32_t tile_size, uint32_t tx, uint32_t ty, uint32_t tz,
                                int32_t* __restrict__ counts) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    uint32_t lo[3], hi[3];
    counts[i] = rect_3d(means3d, radii, i, tile_size, tx, ty, tz, lo, hi)
                    ? static_cast<int32_t>((hi[2] - lo[2]) * (hi[1] - lo[1]) * (hi[0] - lo[0])) : 0;
}

// ----------------------------------------------------------------- emission

template <typename S>
__global__ void emit_2d_kernel(const S* __restrict__ means2d, const int32_t* __restrict__ radii, bool rect,
                               uint32_t total, uint32_t N, uint32_t tile_size, uint32_t tiles_x, uint32_t tiles_y,
                               const int64_t* __restrict__ cum, uint32_t* __restrict__ keys,
                               uint32_t* __restrict__ vals) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= total) return;
    uint32_t x0, x1, y0, y1;
    if (!rect_2d(means2d, radii, rect, i, tile_size, tiles_x, tiles_y, x0, x1, y0, y1)) return;
    const uint32_t base_key = (i / N) * (tiles_x * tiles_y);
    int64_t w = i == 0 ? 0 : cum[i - 1];
    for (uint32_t y = y0; y < y1; ++y)
        for (uint32_t x = x0; x < x1; ++x, ++w) {
            keys[w] = base_key + y * tiles_x + x;
            vals[w] = i;
        }
}

// Writes element i's intersections at [cum[i-1], cum[i]); positions at or past
// `capacity` are not written (the caller flags that case as an overflow).
__global__ void emit_rects_kernel(const ushort4* __restrict__ rects, uint32_t total, uint32_t N, uint32_t tiles_x,
                                  uint32_t tiles_y, const int64_t* __restrict__ cum, int64_t capacity,
                                  uint32_t* __restrict__ keys, uint32_t* __restrict__ vals) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= total) return;
    const ushort4 r = rects[i];
    if (r.z <= r.x || r.w <= r.y) return;
    const uint32_t base_key = (i / N) * (tiles_x * tiles_y);
    int64_t w = i == 0 ? 0 : cum[i - 1];
    if (cum[i] > capacity) return;
    for (uint32_t y = r.y; y < r.w; ++y)
        for (uint32_t x = r.x; x < r.z; ++x, ++w) {
            keys[w] = base_key + y * tiles_x + x;
            vals[w] = i;
        }
}

// The same output as emit_rects_kernel, written cooperatively: a warp takes 32
// consecutive elements, whose runs form one contiguous range of the output, and
// its lanes stride over that range, so consecutive lanes write consecutive keys
// and values (one-thread-per-element writes are scattered over 32 runs). Each
// lane finds the element owning its position by a 5-step binary search over the
// warp's 32 run starts, exchanged by shuffles.
__global__ void __launch_bounds__(256) emit_rects_warp_kernel(const ushort4* __restrict__ rects, uint32_t total,
                                                               uint32_t N, uint32_t tiles_x, uint32_t tiles_y,
                                                               const int64_t* __restrict__ cum, int64_t capacity,
                                                               uint32_t* __restrict__ keys,
                                                               uint32_t* __restrict__ vals) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint64_t warp = (uint64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    const uint64_t i0 = warp * 32u;
    if (i0 >= total) return;  // warp-uniform
    const uint32_t i = uint32_t(i0) + lane;
    const bool have = i < total;
    ushort4 r = make_ushort4(0, 0, 0, 0);
    int64_t start = 0, end = 0;
    if (have) {
        r = rects[i];
        start = i == 0 ? 0 : cum[i - 1];
        end = cum[i];
    } else {
        start = end = cum[total - 1];
    }
    const bool nonempty = have && r.z > r.x && r.w > r.y;
    const uint32_t width = nonempty ? uint32_t(r.z - r.x) : 1u;
    const int64_t range_start = __shfl_sync(0xffffffffu, start, 0);
    const int64_t range_end = __shfl_sync(0xffffffffu, end, 31);
    const uint32_t n_tiles = tiles_x * tiles_y;
    // The key of the record's first tile, cam * n_tiles + y0 * tiles_x + x0, once per record.
    const uint32_t key0 = (i / N) * n_tiles + uint32_t(r.y) * tiles_x + uint32_t(r.x);
    // A warp-uniform trip count: every lane takes part in every shuffle.
    const int64_t steps = (range_end - range_start + 31) / 32;
    for (int64_t k = 0; k < steps; ++k) {
        const int64_t p = range_start + k * 32 + lane;
        // Owner: the last lane whose run starts at or before p (empty runs start where the next one does,
        // so the search lands on the non-empty run that holds p).
        uint32_t lo = 0u;
#pragma unroll
        for (uint32_t step = 16u; step > 0u; step >>= 1) {
            const int64_t s_mid = __shfl_sync(0xffffffffu, start, int(lo + step));
            if (s_mid <= p) lo += step;
        }
        const int64_t s_owner = __shfl_sync(0xffffffffu, start, int(lo));
        const uint32_t w_owner = __shfl_sync(0xffffffffu, width, int(lo));
        const uint32_t k_owner = __shfl_sync(0xffffffffu, key0, int(lo));
        if (p >= range_end || p >= capacity) continue;
        const uint32_t local = uint32_t(p - s_owner);
        const uint32_t row = local / w_owner, col = local - row * w_owner;
        keys[p] = k_owner + row * tiles_x + col;
        vals[p] = uint32_t(i0) + lo;
    }
}

template <typename S>
__global__ void emit_3d_kernel(const S* __restrict__ means3d, const int32_t* __restrict__ radii, uint32_t N,
                               uint32_t tile_size, uint32_t tx, uint32_t ty, uint32_t tz,
                               const int64_t* __restrict__ cum, int64_t capacity, uint32_t* __restrict__ keys,
                               uint32_t* __restrict__ vals) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    uint32_t lo[3], hi[3];
    if (!rect_3d(means3d, radii, i, tile_size, tx, ty, tz, lo, hi)) return;
    int64_t w = i == 0 ? 0 : cum[i - 1];
    if (cum[i] > capacity) return;
    for (uint32_t z = lo[2]; z < hi[2]; ++z)
        for (uint32_t y = lo[1]; y < hi[1]; ++y)
            for (uint32_t x = lo[0]; x < hi[0]; ++x, ++w) {
                keys[w] = (z * ty + y) * tx + x;
                vals[w] = i;
            }
}

// 3D counterpart of emit_rects_warp_kernel (the output of emit_3d_kernel, written cooperatively).
template <typename S>
__global__ void __launch_bounds__(256) emit_3d_warp_kernel(const S* __restrict__ means3d,
                                                            const int32_t* __restrict__ radii, uint32_t N,
                                                            uint32_t tile_size, uint32_t tx, uint32_t ty, uint32_t tz,
                                                            const int64_t* __restrict__ cum, int64_t capacity,
                                                            uint32_t* __restrict__ keys,
                                                            uint32_t* __restrict__ vals) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint64_t i0 = ((uint64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5) * 32u;
    if (i0 >= N) return;  // warp-uniform
    const uint32_t i = uint32_t(i0) + lane;
    uint32_t lo[3] = {0u, 0u, 0u}, hi[3] = {1u, 1u, 1u};
    int64_t start, end;
    if (i < N) {
        if (!rect_3d(means3d, radii, i, tile_size, tx, ty, tz, lo, hi)) {
            lo[0] = lo[1] = lo[2] = 0u;
            hi[0] = hi[1] = hi[2] = 1u;
        }
        start = i == 0 ? 0 : cum[i - 1];
        end = cum[i];
    } else {
        start = end = cum[N - 1];
    }
    const uint32_t nx = hi[0] - lo[0], ny = hi[1] - lo[1];
    const int64_t range_start = __shfl_sync(0xffffffffu, start, 0);
    const int64_t range_end = __shfl_sync(0xffffffffu, end, 31);
    const int64_t steps = (range_end - range_start + 31) / 32;
    for (int64_t k = 0; k < steps; ++k) {
        const int64_t p = range_start + k * 32 + lane;
        uint32_t owner = 0u;
#pragma unroll
        for (uint32_t step = 16u; step > 0u; step >>= 1) {
            const int64_t s_mid = __shfl_sync(0xffffffffu, start, int(owner + step));
            if (s_mid <= p) owner += step;
        }
        const int64_t s_owner = __shfl_sync(0xffffffffu, start, int(owner));
        const uint32_t onx = __shfl_sync(0xffffffffu, nx, int(owner));
        const uint32_t ony = __shfl_sync(0xffffffffu, ny, int(owner));
        const uint32_t ox = __shfl_sync(0xffffffffu, lo[0], int(owner));
        const uint32_t oy = __shfl_sync(0xffffffffu, lo[1], int(owner));
        const uint32_t oz = __shfl_sync(0xffffffffu, lo[2], int(owner));
        if (p >= range_end || p >= capacity) continue;
        const uint32_t local = uint32_t(p - s_owner);
        const uint32_t plane = onx * ony;
        const uint32_t dz = local / plane;
        const uint32_t rem = local - dz * plane;
        const uint32_t dy = rem / onx, dx = rem - dy * onx;
        keys[p] = ((oz + dz) * ty + (oy + dy)) * tx + (ox + dx);
        vals[p] = uint32_t(i0) + owner;
    }
}

// --------------------------------------------------------------- radix sort// --------------------------------------------------------------- radix sort

constexpr int kSortThreads = 256;
constexpr int kSortWarps = kSortThreads / 32;
constexpr int kSortItems = 16;  // per lane
constexpr int64_t kSortTile = int64_t(kSortThreads) * kSortItems;
constexpr int kMaxDigitBits = 10;

// Digit histogram of elements [begin, end) into shared memory (zeroed here).
template <typename Digit>
__device__ __forceinline__ void block_histogram(const uint32_t* __restrict__ keys, int64_t begin, int64_t end,
                                                Digit digit, uint32_t bins, uint32_t* s_hist) {
    uint32_t k_key[kSortItems];
#pragma unroll
    for (int k = 0; k < kSortItems; ++k) {
        const int64_t i = begin + int64_t(k) * kSortThreads + threadIdx.x;
        k_key[k] = i < end ? keys[i] : 0u;
    }
    for (uint32_t d = threadIdx.x; d < bins; d += kSortThreads) s_hist[d] = 0;
    __syncthreads();
#pragma unroll
    for (int k = 0; k < kSortItems; ++k) {
        const int64_t i = begin + int64_t(k) * kSortThreads + threadIdx.x;
        if (i < end) atomicAdd(&s_hist[digit(k_key[k])], 1u);
    }
    __syncthreads();
}

// Per-block digit histogram, stored digit-major: hist[d * n_blocks + b].
// With n_dev non-null the element count is *n_dev (at most n, the capacity the
// grid was sized for); blocks past it contribute empty histograms.
__global__ void __launch_bounds__(kSortThreads) radix_upsweep_kernel(const uint32_t* __restrict__ keys, int64_t n,
                                                                    const int64_t* __restrict__ n_dev, int shift,
                                                                    uint32_t mask, uint32_t* __restrict__ hist) {
    extern __shared__ uint32_t s_hist[];
    if (n_dev != nullptr && *n_dev < n) n = *n_dev;
    const uint32_t bins = mask + 1;
    const int64_t base = int64_t(blockIdx.x) * kSortTile;
    block_histogram(keys, base, min(n, base + kSortTile), [=](uint32_t key) { return (key >> shift) & mask; }, bins,
                    s_hist);
    for (uint32_t d = threadIdx.x; d < bins; d += kSortThreads) hist[size_t(d) * gridDim.x + blockIdx.x] = s_hist[d];
}

// Stable scatter of one digit for the block's elements [block_base, end).
// Element order inside a block is (warp, item, lane) = index order; ranks come
// from warp-wide matching of equal digits. The block's elements are first
// placed in shared memory in digit order, then written out in that order, so
// consecutive threads store consecutive positions of one digit's run
// (coalesced) instead of scattering 4-byte stores. global(d) is the output
// position of the block's first element of digit d.
// Shared memory: [kSortWarps][bins] warp offsets, [bins] block-local digit
// starts, [bins] global digit bases, then kSortTile staged keys and values.
template <typename KeyOut, typename ValOut, typename Digit, typename Global>
__device__ __forceinline__ void block_scatter(const uint32_t* __restrict__ keys, const uint32_t* __restrict__ vals,
                                              int64_t block_base, int64_t end, Digit digit, uint32_t bins,
                                              Global global, KeyOut* __restrict__ keys_out,
                                              ValOut* __restrict__ vals_out, uint32_t* s_cnt) {
    uint32_t* s_local = s_cnt + kSortWarps * bins;  // block-local start of each digit
    uint32_t* s_global = s_local + bins;             // global position of each digit's first element
    uint32_t* s_key = s_global + bins;               // [kSortTile]
    uint32_t* s_val = s_key + kSortTile;             // [kSortTile]
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (uint32_t d = threadIdx.x; d < bins * kSortWarps; d += kSortThreads) s_cnt[d] = 0;
    __syncthreads();
    uint32_t* my_cnt = s_cnt + warp * bins;
    const uint32_t lt_mask = (1u << lane) - 1u;
    const int64_t base = block_base + int64_t(warp) * (kSortTile / kSortWarps);
    uint32_t k_key[kSortItems], k_rank[kSortItems];
    // The keys are loaded first: the ranking loop below orders its
    // shared-memory updates with __syncwarp, which would otherwise hold each
    // load back until the previous item was ranked. The values are loaded
    // where they are staged.
#pragma unroll
    for (int k = 0; k < kSortItems; ++k) {
        const int64_t i = base + int64_t(k) * 32 + lane;
        k_key[k] = i < end ? keys[i] : 0u;
    }
#pragma unroll
    for (int k = 0; k < kSortItems; ++k) {
        const int64_t i = base + int64_t(k) * 32 + lane;
        const bool valid = i < end;
        const uint32_t d = valid ? digit(k_key[k]) : bins;
        const uint32_t peers = __match_any_sync(0xffffffffu, d);
        const uint32_t leader = __ffs(peers) - 1;
        uint32_t count = 0;
        if (valid) count = my_cnt[d];
        __syncwarp();
        if (valid && lane == static_cast<int>(leader)) my_cnt[d] = count + __popc(peers);
        __syncwarp();
        k_rank[k] = count + __popc(peers & lt_mask);
    }
    __syncthreads();
    // Per digit: total over warps, and warp counts -> block-local warp offsets.
    for (uint32_t d = threadIdx.x; d < bins; d += kSortThreads) {
        uint32_t running = 0;
#pragma unroll
        for (int w = 0; w < kSortWarps; ++w) {
            const uint32_t c = s_cnt[w * bins + d];
            s_cnt[w * bins + d] = running;
            running += c;
        }
        s_local[d] = running;  // digit total for now
        s_global[d] = global(d);
    }
    __syncthreads();
    // Exclusive scan of the digit totals (one warp; at most 1024 digits).
    if (warp == 0) {
        uint32_t carry = 0;
        for (uint32_t d0 = 0; d0 < bins; d0 += 32) {
            const uint32_t d = d0 + lane;
            const uint32_t v = d < bins ? s_local[d] : 0u;
            uint32_t inc = v;
#pragma unroll
            for (int off = 1; off < 32; off <<= 1) {
                const uint32_t o = __shfl_up_sync(0xffffffffu, inc, off);
                if (lane >= off) inc += o;
            }
            if (d < bins) s_local[d] = carry + inc - v;
            carry += __shfl_sync(0xffffffffu, inc, 31);
        }
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < kSortItems; ++k) {
        const int64_t i = base + int64_t(k) * 32 + lane;
        if (i < end) {
            const uint32_t d = digit(k_key[k]);
            const uint32_t slot = s_local[d] + my_cnt[d] + k_rank[k];
            s_key[slot] = k_key[k];
            s_val[slot] = vals[i];
        }
    }
    __syncthreads();
    const int64_t remaining = end - block_base;
    const uint32_t count = remaining < kSortTile ? uint32_t(remaining) : uint32_t(kSortTile);
    for (uint32_t j = threadIdx.x; j < count; j += kSortThreads) {
        const uint32_t key = s_key[j];
        const uint32_t d = digit(key);
        const uint32_t pos = s_global[d] + (j - s_local[d]);
        keys_out[pos] = static_cast<KeyOut>(key);
        vals_out[pos] = static_cast<ValOut>(s_val[j]);
    }
}

// The generic scatter kernel is bounded to three resident blocks per SM (at
// most 85 registers a thread): left to itself ptxas gives it 128 registers and
// two blocks, and the sort runs latency-bound. The segmented scatter, ranked in
// registers by ballots, fits four blocks (64 registers, no spill): 1.075 ->
// 1.050 ms for the CT sort stage, 3.28 -> 3.18 ms for Beta's.
template <typename KeyOut, typename ValOut>
__global__ void __launch_bounds__(kSortThreads, 3) radix_downsweep_kernel(
    const uint32_t* __restrict__ keys, const uint32_t* __restrict__ vals, int64_t n, const int64_t* __restrict__ n_dev,
    int shift, uint32_t mask, const uint32_t* __restrict__ offsets, KeyOut* __restrict__ keys_out,
    ValOut* __restrict__ vals_out) {
    extern __shared__ uint32_t s_cnt[];
    if (n_dev != nullptr && *n_dev < n) n = *n_dev;
    const int64_t block_base = int64_t(blockIdx.x) * kSortTile;
    if (block_base >= n) return;  // the whole block is past the count
    const uint32_t b = blockIdx.x, nb = gridDim.x;
    block_scatter(keys, vals, block_base, min(n, block_base + kSortTile),
                  [=](uint32_t key) { return (key >> shift) & mask; }, mask + 1,
                  [=](uint32_t d) { return offsets[size_t(d) * nb + b]; }, keys_out, vals_out, s_cnt);
}

// Stable scatter of one digit of at most 6 bits (64 bins) for the block's
// elements [block_base, end): the same contract as block_scatter, with the
// ranking done in registers. Each warp ranks its elements item by item with
// six ballots over the digit bits: a lane's peers (same digit, same item) are
// the AND of the ballots it agrees with, and lane L keeps the warp's running
// count of digits L and L + 32, which the lanes with that digit read by a
// shuffle. No shared-memory counter sits between one item and the next, so
// nothing serialises on shared memory (block_scatter's per-item counter
// round trips are what held the 1024-bin pass back). A histogram counted the
// same way (for the upsweep) was slower than shared-memory atomics: 0.14 vs
// 0.06 ms per pass at the CT scene.
// Shared memory: [kSortWarps][64] warp offsets, [64] block-local digit
// starts, [64] global digit bases, then kSortTile staged keys and values.
constexpr uint32_t kBallotBins = 64;

template <typename KeyOut, typename ValOut, typename Digit, typename Global>
__device__ __forceinline__ void block_scatter_ballot(const uint32_t* __restrict__ keys,
                                                     const uint32_t* __restrict__ vals, int64_t block_base,
                                                     int64_t end, Digit digit, uint32_t bins, Global global,
                                                     KeyOut* __restrict__ keys_out, ValOut* __restrict__ vals_out,
                                                     uint32_t* s_cnt) {
    uint32_t* s_local = s_cnt + kSortWarps * kBallotBins;  // block-local start of each digit
    uint32_t* s_global = s_local + kBallotBins;             // global position of each digit's first element
    uint32_t* s_key = s_global + kBallotBins;               // [kSortTile]
    uint32_t* s_val = s_key + kSortTile;                    // [kSortTile]
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    const uint32_t lt_mask = (1u << lane) - 1u;
    const int64_t base = block_base + int64_t(warp) * (kSortTile / kSortWarps);
    uint32_t k_key[kSortItems], k_rank[kSortItems];
#pragma unroll
    for (int k = 0; k < kSortItems; ++k) {
        const int64_t i = base + int64_t(k) * 32 + lane;
        k_key[k] = i < end ? keys[i] : 0u;
    }
    uint32_t cnt_lo = 0u, cnt_hi = 0u;  // this warp's count so far of digit lane (lo) and lane + 32 (hi)
#pragma unroll
    for (int k = 0; k < kSortItems; ++k) {
        const int64_t i = base + int64_t(k) * 32 + lane;
        const bool valid = i < end;
        const uint32_t d = valid ? digit(k_key[k]) : 0u;
        const uint32_t live = __ballot_sync(0xffffffffu, valid);
        uint32_t peers = live, mine_lo = live;
#pragma unroll
        for (int b = 0; b < 6; ++b) {
            const uint32_t bal = __ballot_sync(0xffffffffu, valid && ((d >> b) & 1u));
            peers &= ((d >> b) & 1u) ? bal : ~bal;
            if (b < 5) {
                mine_lo &= ((lane >> b) & 1u) ? bal : ~bal;
            } else {
                // digits lane (bit 5 clear) and lane + 32 (bit 5 set)
                const uint32_t mine_hi = mine_lo & bal;
                mine_lo &= ~bal;
                const uint32_t before_lo = __shfl_sync(0xffffffffu, cnt_lo, d & 31u);
                const uint32_t before_hi = __shfl_sync(0xffffffffu, cnt_hi, d & 31u);
                k_rank[k] = (d >= 32u ? before_hi : before_lo) + __popc(peers & lt_mask);
                cnt_lo += __popc(mine_lo);
                cnt_hi += __popc(mine_hi);
            }
        }
    }
    uint32_t* my_cnt = s_cnt + warp * kBallotBins;
    my_cnt[lane] = cnt_lo;
    my_cnt[lane + 32u] = cnt_hi;
    __syncthreads();
    // Per digit: warp counts -> block-local warp offsets, and the digit totals.
    if (threadIdx.x < bins) {
        const uint32_t d = threadIdx.x;
        uint32_t running = 0;
#pragma unroll
        for (int w = 0; w < kSortWarps; ++w) {
            const uint32_t c = s_cnt[w * kBallotBins + d];
            s_cnt[w * kBallotBins + d] = running;
            running += c;
        }
        s_local[d] = running;
        s_global[d] = global(d);
    }
    __syncthreads();
    // Exclusive scan of the digit totals (one warp; at most 64 digits).
    if (warp == 0) {
        uint32_t carry = 0;
        for (uint32_t d0 = 0; d0 < bins; d0 += 32) {
            const uint32_t d = d0 + lane;
            const uint32_t v = d < bins ? s_local[d] : 0u;
            uint32_t inc = v;
#pragma unroll
            for (int off = 1; off < 32; off <<= 1) {
                const uint32_t o = __shfl_up_sync(0xffffffffu, inc, off);
                if (lane >= uint32_t(off)) inc += o;
            }
            if (d < bins) s_local[d] = carry + inc - v;
            carry += __shfl_sync(0xffffffffu, inc, 31);
        }
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < kSortItems; ++k) {
        const int64_t i = base + int64_t(k) * 32 + lane;
        if (i < end) {
            const uint32_t d = digit(k_key[k]);
            const uint32_t slot = s_local[d] + my_cnt[d] + k_rank[k];
            s_key[slot] = k_key[k];
            s_val[slot] = vals[i];
        }
    }
    __syncthreads();
    const int64_t remaining = end - block_base;
    const uint32_t count = remaining < kSortTile ? uint32_t(remaining) : uint32_t(kSortTile);
    for (uint32_t j = threadIdx.x; j < count; j += kSortThreads) {
        const uint32_t key = s_key[j];
        const uint32_t d = digit(key);
        const uint32_t pos = s_global[d] + (j - s_local[d]);
        keys_out[pos] = static_cast<KeyOut>(key);
        vals_out[pos] = static_cast<ValOut>(s_val[j]);
    }
}

// ------------------------------------------------ camera-segmented 2D sort
//
// 2D keys are cam * n_tiles + tile and emission is camera-major, so the key
// array is already ordered by camera: stable passes on the tile index inside
// each camera's segment sort it completely, and the camera never needs a
// digit of its own. Each sort block takes kSortTile elements of one camera.
// The histogram of camera c, digit d, block j (of nb_c) sits at
// bins * first_block_c + d * nb_c + j, so one exclusive scan over all of them
// gives every block's output position per digit directly (cameras before c,
// then digits before d, then earlier blocks).

struct CamSegment {
    int64_t begin, end;    // elements of the camera
    uint32_t first_block;  // sort blocks before this camera's
    uint32_t n_blocks;
};

// One thread: segment bounds from the inclusive tile-count prefix (one entry
// per (camera, element) pair, C*N in all) and the block layout; the blocks of
// the grid past the last camera's zero-fill the unused histogram tail.
__global__ void cam_segments_kernel(const int64_t* __restrict__ cum, uint32_t C, uint32_t N, int64_t n,
                                    const int64_t* __restrict__ n_dev, CamSegment* __restrict__ seg,
                                    uint32_t* __restrict__ total_blocks) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    if (n_dev != nullptr && *n_dev < n) n = *n_dev;
    int64_t begin = 0;
    uint32_t blocks = 0;
    for (uint32_t c = 0; c < C; ++c) {
        int64_t end = cum[(int64_t(c) + 1) * N - 1];
        if (end > n) end = n;
        if (end < begin) end = begin;
        const uint32_t nb = uint32_t((end - begin + kSortTile - 1) / kSortTile);
        seg[c] = CamSegment{begin, end, blocks, nb};
        blocks += nb;
        begin = end;
    }
    *total_blocks = blocks;
}

// The camera holding sort block b (binary search over first_block).
__device__ __forceinline__ uint32_t block_camera(const CamSegment* seg, uint32_t C, uint32_t b) {
    uint32_t lo = 0, hi = C;  // first_block[lo] <= b < first_block[hi]
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (seg[mid].first_block <= b) lo = mid; else hi = mid;
    }
    return lo;
}

// The digit of a segmented pass: bits [shift, shift + bits(mask)) of the tile
// index key - key0.
struct SegDigit {
    uint32_t key0, shift, mask;
    __device__ __forceinline__ uint32_t operator()(uint32_t key) const { return ((key - key0) >> shift) & mask; }
};

__global__ void __launch_bounds__(kSortThreads) segmented_upsweep_kernel(
    const uint32_t* __restrict__ keys, const CamSegment* __restrict__ seg, uint32_t C, uint32_t n_tiles,
    uint32_t shift, uint32_t mask, uint32_t bins, const uint32_t* __restrict__ total_blocks,
    uint32_t* __restrict__ hist) {
    extern __shared__ uint32_t s_hist[];
    const uint32_t b = blockIdx.x, used = *total_blocks;
    if (b >= used) {
        // Zero the histogram tail that no camera uses (gridDim.x - used blocks of bins).
        uint32_t* tail = hist + size_t(bins) * used + size_t(b - used) * bins;
        for (uint32_t d = threadIdx.x; d < bins; d += kSortThreads) tail[d] = 0;
        return;
    }
    const uint32_t c = block_camera(seg, C, b);
    const CamSegment sg = seg[c];
    const uint32_t j = b - sg.first_block;
    const int64_t begin = sg.begin + int64_t(j) * kSortTile;
    block_histogram(keys, begin, min(sg.end, begin + kSortTile), SegDigit{c * n_tiles, shift, mask}, bins, s_hist);
    uint32_t* out = hist + size_t(bins) * sg.first_block + j;
    for (uint32_t d = threadIdx.x; d < bins; d += kSortThreads) out[size_t(d) * sg.n_blocks] = s_hist[d];
}

template <typename KeyOut, typename ValOut>
__global__ void __launch_bounds__(kSortThreads, 4) segmented_downsweep_kernel(
    const uint32_t* __restrict__ keys, const uint32_t* __restrict__ vals, const CamSegment* __restrict__ seg,
    uint32_t C, uint32_t n_tiles, uint32_t shift, uint32_t mask, uint32_t bins,
    const uint32_t* __restrict__ total_blocks, const uint32_t* __restrict__ offsets, KeyOut* __restrict__ keys_out,
    ValOut* __restrict__ vals_out) {
    extern __shared__ uint32_t s_cnt[];
    const uint32_t b = blockIdx.x;
    if (b >= *total_blocks) return;
    const uint32_t c = block_camera(seg, C, b);
    const CamSegment sg = seg[c];
    const uint32_t j = b - sg.first_block;
    const int64_t begin = sg.begin + int64_t(j) * kSortTile;
    const uint32_t* base = offsets + size_t(bins) * sg.first_block + j;
    const uint32_t nb = sg.n_blocks;
    block_scatter_ballot(keys, vals, begin, min(sg.end, begin + kSortTile), SegDigit{c * n_tiles, shift, mask},
                         bins, [=](uint32_t d) { return base[size_t(d) * nb]; }, keys_out, vals_out, s_cnt);
}

__global__ void widen_kernel(const uint32_t* __restrict__ keys, const uint32_t* __restrict__ vals, int64_t n,
                             const int64_t* __restrict__ n_dev, int64_t* __restrict__ keys_out,
                             int32_t* __restrict__ vals_out) {
    const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (n_dev != nullptr && *n_dev < n) n = *n_dev;
    if (i >= n) return;
    keys_out[i] = keys[i];
    vals_out[i] = static_cast<int32_t>(vals[i]);
}

// offsets[k] = number of sorted keys smaller than k (lower bound).
__global__ void offsets_kernel(const int64_t* __restrict__ keys, int64_t n, const int64_t* __restrict__ n_dev,
                               int64_t n_keys, int32_t* __restrict__ offsets) {
    const int64_t k = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (k >= n_keys) return;
    if (n_dev != nullptr && *n_dev < n) n = *n_dev;
    int64_t lo = 0, hi = n;
    while (lo < hi) {
        const int64_t mid = (lo + hi) >> 1;
        if (keys[mid] < k) lo = mid + 1; else hi = mid;
    }
    offsets[k] = static_cast<int32_t>(lo);
}

// Device-side intersection count for capacity-bounded (graph-capturable)
// pipelines: n_used = total when it fits the capacity, else 0 with the
// overflow flag raised (the emission wrote nothing past the capacity).
__global__ void count_finish_kernel(const int64_t* __restrict__ cum, int64_t last, int64_t capacity,
                                    int64_t* __restrict__ n_used, uint32_t* __restrict__ overflow) {
    const int64_t total = last >= 0 ? cum[last] : 0;
    if (total > capacity) {
        *n_used = 0;
        atomicOr(overflow, 1u);
    } else {
        *n_used = total;
    }
}

inline int bits_for(uint64_t max_key) {
    // Number of bits needed for keys in [0, max_key] (IsectTiles.cpp:146-147
    // sorts on ceil(log2(max_key + 1)) bits of the key).
    int bits = 0;
    while (bits < 64 && (uint64_t(1) << bits) <= max_key) ++bits;
    return bits;
}

struct SortPlan {
    int passes = 0;
    int digit_bits = 0;
    int64_t blocks = 0;
};

inline SortPlan plan_sort(int64_t n, uint64_t n_keys) {
    SortPlan p;
    const int bits = bits_for(n_keys > 0 ? n_keys - 1 : 0);
    p.passes = (bits + kMaxDigitBits - 1) / kMaxDigitBits;
    p.digit_bits = p.passes > 0 ? (bits + p.passes - 1) / p.passes : 0;
    p.blocks = (n + kSortTile - 1) / kSortTile;
    return p;
}

// Camera layout of 2D keys (cam * n_tiles + tile, emitted camera-major) for
// the camera-segmented sort; cum is the inclusive tile-count prefix over the
// C * N (camera, element) pairs.
struct CamLayout {
    const int64_t* cum;
    uint32_t C, N, n_tiles;
};

constexpr uint32_t kMaxCameras = 65535;
// The segmented sort takes the tile index in stable passes of at most
// kSegmentedDigitBits bits (least significant first), ranked in registers by
// ballots (block_scatter_ballot): few bins keep the histogram L2-resident and
// each block's output runs long enough to coalesce. 1024 tiles per camera
// take two passes of 5 bits; a single pass of 1024 bins ranked through
// shared-memory counters took 0.64 ms for the CT scene's 4.7e7 keys, twice as
// long as both ballot passes.
constexpr uint32_t kSegmentedOnePass = 1024;  // bound on the bins any segmented plan had (workspace sizing)
constexpr int kSegmentedDigitBits = 6;
constexpr uint32_t kMaxSegmentedTiles = 1u << 24;
static_assert((1u << kSegmentedDigitBits) <= kBallotBins, "ballot ranking covers at most 64 bins");

struct SegPlan {
    int passes, digit_bits;
    uint32_t bins;  // per pass
};

inline SegPlan plan_segmented(uint32_t n_tiles) {
    const int bits = n_tiles > 1 ? bits_for(n_tiles - 1) : 1;
    const int passes = (bits + kSegmentedDigitBits - 1) / kSegmentedDigitBits;
    const int digit_bits = (bits + passes - 1) / passes;
    return SegPlan{passes, digit_bits, 1u << digit_bits};
}

inline size_t emit_workspace(int64_t n, uint64_t n_keys) {
    const SortPlan p = plan_sort(n, n_keys);
    ArenaSize a;
    a.take<uint32_t>(size_t(n));  // keys A
    a.take<uint32_t>(size_t(n));  // vals A
    a.take<uint32_t>(size_t(n));  // keys B
    a.take<uint32_t>(size_t(n));  // vals B
    const size_t blocks = size_t(p.blocks > 0 ? p.blocks : 1);
    const size_t hist_generic = size_t(1u << (p.digit_bits > 0 ? p.digit_bits : 1)) * blocks;
    // Segmented: bins * (blocks + C) with bins <= kSegmentedOnePass, and
    // bins * C <= n_tiles * C = n_keys (bins = n_tiles in one pass, below it
    // otherwise).
    const size_t hist_segmented = size_t(kSegmentedOnePass) * blocks + size_t(n_keys);
    const size_t hist = hist_generic > hist_segmented ? hist_generic : hist_segmented;
    a.take<CamSegment>(size_t(n_keys < kMaxCameras ? n_keys : kMaxCameras));
    a.take<uint32_t>(1);
    a.take<uint32_t>(hist);
    a.take<char>(scan_workspace_bytes<uint32_t>(int64_t(hist)));
    return a.bytes();
}

// Stable passes on the tile index inside each camera's segment (one pass up to
// kSegmentedOnePass tiles), the last writing the widened result to
// isect_ids/flatten_ids. keys and vals are kept intact for a single pass and
// serve as ping-pong buffers otherwise.
inline int segmented_sort(uint32_t* keys, uint32_t* vals, int64_t n, const CamLayout& cams, Arena& arena,
                          int64_t* isect_ids, int32_t* flatten_ids, cudaStream_t stream, const int64_t* n_dev) {
    const SegPlan plan = plan_segmented(cams.n_tiles);
    const int64_t max_blocks = (n + kSortTile - 1) / kSortTile + int64_t(cams.C);
    R2S_REQUIRE(max_blocks < (int64_t(1) << 31), R2S_ERR_UNSUPPORTED, "too many intersections");
    uint32_t* keys_b = plan.passes > 1 ? arena.take<uint32_t>(size_t(n)) : nullptr;
    uint32_t* vals_b = plan.passes > 1 ? arena.take<uint32_t>(size_t(n)) : nullptr;
    CamSegment* seg = arena.take<CamSegment>(cams.C);
    uint32_t* total_blocks = arena.take<uint32_t>(1);
    const int64_t hist_len = int64_t(plan.bins) * max_blocks;
    uint32_t* hist = arena.take<uint32_t>(size_t(hist_len));
    R2S_REQUIRE(seg && total_blocks && hist && (plan.passes == 1 || (keys_b && vals_b)), R2S_ERR_WORKSPACE,
                "intersection workspace too small");
    void* scan_ws = arena.base + arena.used;
    const size_t scan_bytes = arena.size - arena.used;
    cam_segments_kernel<<<1, 32, 0, stream>>>(cams.cum, cams.C, cams.N, n, n_dev, seg, total_blocks);
    R2S_TRY(check_launch("cam_segments"));
    const size_t down_smem = (size_t(kBallotBins) * (kSortWarps + 2) + 2 * size_t(kSortTile)) * sizeof(uint32_t);
    R2S_TRY(allow_dynamic_smem(segmented_downsweep_kernel<int64_t, int32_t>, down_smem));
    if (plan.passes > 1) R2S_TRY(allow_dynamic_smem(segmented_downsweep_kernel<uint32_t, uint32_t>, down_smem));
    uint32_t *src_k = keys, *src_v = vals, *dst_k = keys_b, *dst_v = vals_b;
    for (int pass = 0; pass < plan.passes; ++pass) {
        const uint32_t shift = uint32_t(pass * plan.digit_bits);
        const uint32_t mask = plan.bins - 1u;
        segmented_upsweep_kernel<<<unsigned(max_blocks), kSortThreads, plan.bins * sizeof(uint32_t), stream>>>(
            src_k, seg, cams.C, cams.n_tiles, shift, mask, plan.bins, total_blocks, hist);
        R2S_TRY(check_launch("segmented_upsweep"));
        R2S_TRY((device_scan<uint32_t, uint32_t, false>(hist, hist, hist_len, scan_ws, scan_bytes, stream)));
        if (pass == plan.passes - 1) {
            segmented_downsweep_kernel<int64_t, int32_t><<<unsigned(max_blocks), kSortThreads, down_smem, stream>>>(
                src_k, src_v, seg, cams.C, cams.n_tiles, shift, mask, plan.bins, total_blocks, hist, isect_ids,
                flatten_ids);
        } else {
            segmented_downsweep_kernel<uint32_t, uint32_t><<<unsigned(max_blocks), kSortThreads, down_smem,
                                                             stream>>>(
                src_k, src_v, seg, cams.C, cams.n_tiles, shift, mask, plan.bins, total_blocks, hist, dst_k, dst_v);
        }
        R2S_TRY(check_launch("segmented_downsweep"));
        uint32_t* t = src_k; src_k = dst_k; dst_k = t;
        t = src_v; src_v = dst_v; dst_v = t;
    }
    return R2S_OK;
}

// Sorts (keys, vals) of length n by key bits [0, bits(n_keys-1)), writing
// the widened result to isect_ids/flatten_ids, then fills offsets. With a
// camera layout (at most kMaxSegmentedTiles tiles per camera) the sort is the
// camera-segmented one, which needs no passes over the camera bits.
inline int sort_and_finish(uint32_t* keys, uint32_t* vals, int64_t n, uint64_t n_keys, Arena& arena,
                           int64_t* isect_ids, int32_t* flatten_ids, int32_t* offsets, cudaStream_t stream,
                           const int64_t* n_dev = nullptr, const CamLayout* cams = nullptr) {
    const SortPlan p = plan_sort(n, n_keys);
    const bool segmented = cams != nullptr && cams->C >= 1 && cams->C <= kMaxCameras && cams->n_tiles >= 1 &&
                           cams->n_tiles <= kMaxSegmentedTiles && p.passes > 1;
    if (n > 0) {
        if (p.passes == 0) {
            widen_kernel<<<blocks_for(n, 256), 256, 0, stream>>>(keys, vals, n, n_dev, isect_ids, flatten_ids);
            R2S_TRY(check_launch("widen"));
        } else if (segmented) {
            R2S_TRY(segmented_sort(keys, vals, n, *cams, arena, isect_ids, flatten_ids, stream, n_dev));
        } else {
            uint32_t* keys_b = arena.take<uint32_t>(size_t(n));
            uint32_t* vals_b = arena.take<uint32_t>(size_t(n));
            const uint32_t bins = 1u << p.digit_bits;
            uint32_t* hist = arena.take<uint32_t>(size_t(bins) * size_t(p.blocks));
            R2S_REQUIRE(keys_b && vals_b && hist, R2S_ERR_WORKSPACE, "intersection workspace too small");
            void* scan_ws = arena.base + arena.used;
            const size_t scan_bytes = arena.size - arena.used;
            R2S_REQUIRE(p.blocks < (int64_t(1) << 31), R2S_ERR_UNSUPPORTED, "too many intersections");
            const size_t up_smem = bins * sizeof(uint32_t);
            const size_t down_smem = (bins * (kSortWarps + 2) + 2 * size_t(kSortTile)) * sizeof(uint32_t);
            if (down_smem > 48 * 1024) {
                cudaFuncSetAttribute(radix_downsweep_kernel<uint32_t, uint32_t>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, int(down_smem));
                cudaFuncSetAttribute(radix_downsweep_kernel<int64_t, int32_t>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, int(down_smem));
            }
            uint32_t *src_k = keys, *src_v = vals, *dst_k = keys_b, *dst_v = vals_b;
            for (int pass = 0; pass < p.passes; ++pass) {
                const int shift = pass * p.digit_bits;
                const uint32_t mask = bins - 1;
                radix_upsweep_kernel<<<unsigned(p.blocks), kSortThreads, up_smem, stream>>>(src_k, n, n_dev, shift,
                                                                                           mask, hist);
                R2S_TRY(check_launch("radix_upsweep"));
                R2S_TRY((device_scan<uint32_t, uint32_t, false>(hist, hist, int64_t(bins) * p.blocks, scan_ws,
                                                                scan_bytes, stream)));
                if (pass == p.passes - 1) {
                    radix_downsweep_kernel<int64_t, int32_t><<<unsigned(p.blocks), kSortThreads, down_smem, stream>>>(
                        src_k, src_v, n, n_dev, shift, mask, hist, isect_ids, flatten_ids);
                } else {
                    radix_downsweep_kernel<uint32_t, uint32_t><<<unsigned(p.blocks), kSortThreads, down_smem,
                                                                 stream>>>(src_k, src_v, n, n_dev, shift, mask, hist,
                                                                           dst_k, dst_v);
                }
                R2S_TRY(check_launch("radix_downsweep"));
                uint32_t* t = src_k; src_k = dst_k; dst_k = t;
                t = src_v; src_v = dst_v; dst_v = t;
            }
        }
    }
    if (offsets != nullptr && n_keys > 0) {
        offsets_kernel<<<blocks_for(int64_t(n_keys), 256), 256, 0, stream>>>(isect_ids, n, n_dev, int64_t(n_keys),
                                                                            offsets);
        R2S_TRY(check_launch("isect_offsets"));
    }
    return R2S_OK;
}

}  // namespace r2s

using namespace r2s;

extern "C" {

size_t r2s_isect_count_workspace(uint64_t n_elems) { return scan_workspace_bytes<int64_t>(int64_t(n_elems)); }

int r2s_scan_tile_counts(const int32_t* counts, uint64_t n, int64_t* cum, void* workspace, size_t workspace_bytes,
                         void* stream) {
    return device_scan<int32_t, int64_t, true>(counts, cum, int64_t(n), workspace, workspace_bytes,
                                               as_stream(stream));
}

size_t r2s_isect_emit_workspace(uint64_t n_isects, uint64_t n_keys) {
    return emit_workspace(int64_t(n_isects), n_keys);
}

int r2s_isect_tiles_count(int dtype, const void* means2d, const int32_t* radii, int radii_is_rect, uint32_t C,
                          uint32_t N, uint32_t tile_size, uint32_t tiles_x, uint32_t tiles_y,
                          int32_t* tiles_per_gauss, int64_t* cum_tiles, void* workspace, size_t workspace_bytes,
                          void* stream) {
    const uint64_t total = uint64_t(C) * N;
    if (total == 0) return R2S_OK;
    R2S_REQUIRE(total < (uint64_t(1) << 31), R2S_ERR_UNSUPPORTED, "C*N exceeds the int32 element range");
    R2S_REQUIRE(tile_size > 0, R2S_ERR_ARGUMENT, "tile_size must be positive");
    R2S_DISPATCH(dtype, count_2d_kernel<S><<<blocks_for(total, kIsectThreads), kIsectThreads, 0, as_stream(stream)>>>(
        static_cast<const S*>(means2d), radii, radii_is_rect != 0, uint32_t(total), tile_size, tiles_x, tiles_y,
        tiles_per_gauss));
    R2S_TRY(check_launch("isect_count"));
    return device_scan<int32_t, int64_t, true>(tiles_per_gauss, cum_tiles, int64_t(total), workspace,
                                               workspace_bytes, as_stream(stream));
}

int r2s_isect_tiles_emit(int dtype, const void* means2d, const int32_t* radii, int radii_is_rect, uint32_t C,
                         uint32_t N, uint32_t tile_size, uint32_t tiles_x, uint32_t tiles_y,
                         const int64_t* cum_tiles, int64_t n_isects, int64_t* isect_ids, int32_t* flatten_ids,
                         int32_t* offsets, void* workspace, size_t workspace_bytes, void* stream) {
    const uint64_t total = uint64_t(C) * N;
    const uint64_t n_keys = uint64_t(C) * tiles_x * tiles_y;
    R2S_REQUIRE(n_keys < (uint64_t(1) << 32), R2S_ERR_UNSUPPORTED, "C*tiles exceeds the 32-bit key range");
    R2S_REQUIRE(n_isects >= 0 && n_isects < (int64_t(1) << 31), R2S_ERR_UNSUPPORTED,
                "intersection count exceeds the int32 range");
    Arena arena(workspace, workspace_bytes);
    if (n_isects > 0 && total > 0) {
        uint32_t* keys = arena.take<uint32_t>(size_t(n_isects));
        uint32_t* vals = arena.take<uint32_t>(size_t(n_isects));
        R2S_REQUIRE(keys && vals, R2S_ERR_WORKSPACE, "intersection workspace too small");
        R2S_DISPATCH(dtype, emit_2d_kernel<S><<<blocks_for(total, kIsectThreads), kIsectThreads, 0, as_stream(stream)>>>(
            static_cast<const S*>(means2d), radii, radii_is_rect != 0, uint32_t(total), N, tile_size, tiles_x, tiles_y,
            cum_tiles, keys, vals));
        R2S_TRY(check_launch("isect_emit"));
        const CamLayout cams{cum_tiles, C, N, tiles_x * tiles_y};
        return sort_and_finish(keys, vals, n_isects, n_keys, arena, isect_ids, flatten_ids, offsets,
                               as_stream(stream), nullptr, &cams);
    }
    return sort_and_finish(nullptr, nullptr, 0, n_keys, arena, isect_ids, flatten_ids, offsets, as_stream(stream));
}

int r2s_raster_emit(const uint16_t* rects, uint32_t C, uint32_t N, uint32_t tiles_x, uint32_t tiles_y,
                    const int64_t* cum_tiles, int64_t n_isects, int64_t* isect_ids, int32_t* flatten_ids,
                    int32_t* offsets, void* workspace, size_t workspace_bytes, void* stream) {
    const uint64_t total = uint64_t(C) * N;
    const uint64_t n_keys = uint64_t(C) * tiles_x * tiles_y;
    R2S_REQUIRE(n_keys < (uint64_t(1) << 32), R2S_ERR_UNSUPPORTED, "C*tiles exceeds the 32-bit key range");
    R2S_REQUIRE(n_isects >= 0 && n_isects < (int64_t(1) << 31), R2S_ERR_UNSUPPORTED,
                "intersection count exceeds the int32 range");
    Arena arena(workspace, workspace_bytes);
    if (n_isects > 0 && total > 0) {
        uint32_t* keys = arena.take<uint32_t>(size_t(n_isects));
        uint32_t* vals = arena.take<uint32_t>(size_t(n_isects));
        R2S_REQUIRE(keys && vals, R2S_ERR_WORKSPACE, "intersection workspace too small");
        emit_rects_warp_kernel<<<blocks_for(total, 256), 256, 0, as_stream(stream)>>>(
            reinterpret_cast<const ushort4*>(rects), uint32_t(total), N, tiles_x, tiles_y, cum_tiles, INT64_MAX, keys,
            vals);
        R2S_TRY(check_launch("raster_emit"));
        const CamLayout cams{cum_tiles, C, N, tiles_x * tiles_y};
        return sort_and_finish(keys, vals, n_isects, n_keys, arena, isect_ids, flatten_ids, offsets,
                               as_stream(stream), nullptr, &cams);
    }
    return sort_and_finish(nullptr, nullptr, 0, n_keys, arena, isect_ids, flatten_ids, offsets, as_stream(stream));
}

int r2s_isect_offset_encode(const int64_t* isect_ids, int64_t n_isects, uint32_t C, uint32_t tiles_x,
                            uint32_t tiles_y, int32_t* offsets, void* stream) {
    const int64_t n_keys = int64_t(C) * tiles_x * tiles_y;
    if (n_keys == 0) return R2S_OK;
    offsets_kernel<<<blocks_for(n_keys, 256), 256, 0, as_stream(stream)>>>(isect_ids, n_isects, nullptr, n_keys,
                                                                            offsets);
    return check_launch("isect_offset_encode");
}

int r2s_isect_tiles_3d_count(int dtype, const void* means3d, const int32_t* radii, uint32_t N, uint32_t tile_size,
                             uint32_t tiles_x, uint32_t tiles_y, uint32_t tiles_z, int32_t* tiles_per_gauss,
                             int64_t* cum_tiles, void* workspace, size_t workspace_bytes, void* stream) {
    if (N == 0) return R2S_OK;
    R2S_REQUIRE(tile_size > 0, R2S_ERR_ARGUMENT, "tile_size must be positive");
    R2S_DISPATCH(dtype, count_3d_kernel<S><<<blocks_for(N, kIsectThreads), kIsectThreads, 0, as_stream(stream)>>>(
        static_cast<const S*>(means3d), radii, N, tile_size, tiles_x, tiles_y, tiles_z, tiles_per_gauss));
    R2S_TRY(check_launch("isect_count_3d"));
    return device_scan<int32_t, int64_t, true>(tiles_per_gauss, cum_tiles, int64_t(N), workspace, workspace_bytes,
                                               as_stream(stream));
}

int r2s_isect_tiles_3d_emit(int dtype, const void* means3d, const int32_t* radii, uint32_t N, uint32_t tile_size,
                            uint32_t tiles_x, uint32_t tiles_y, uint32_t tiles_z, const int64_t* cum_tiles,
                            int64_t n_isects, int64_t* isect_ids, int32_t* flatten_ids, int32_t* offsets,
                            void* workspace, size_t workspace_bytes, void* stream) {
    const uint64_t n_keys = uint64_t(tiles_x) * tiles_y * tiles_z;
    R2S_REQUIRE(n_keys < (uint64_t(1) << 32), R2S_ERR_UNSUPPORTED, "tile count exceeds the 32-bit key range");
    R2S_REQUIRE(n_isects >= 0 && n_isects < (int64_t(1) << 31), R2S_ERR_UNSUPPORTED,
                "intersection count exceeds the int32 range");
    Arena arena(workspace, workspace_bytes);
    if (n_isects > 0 && N > 0) {
        uint32_t* keys = arena.take<uint32_t>(size_t(n_isects));
        uint32_t* vals = arena.take<uint32_t>(size_t(n_isects));
        R2S_REQUIRE(keys && vals, R2S_ERR_WORKSPACE, "intersection workspace too small");
        R2S_DISPATCH(dtype, emit_3d_warp_kernel<S><<<blocks_for(N, 256), 256, 0, as_stream(stream)>>>(
            static_cast<const S*>(means3d), radii, N, tile_size, tiles_x, tiles_y, tiles_z, cum_tiles, INT64_MAX, keys,
            vals));
        R2S_TRY(check_launch("isect_emit_3d"));
        return sort_and_finish(keys, vals, n_isects, n_keys, arena, isect_ids, flatten_ids, offsets,
                               as_stream(stream));
    }
    return sort_and_finish(nullptr, nullptr, 0, n_keys, arena, isect_ids, flatten_ids, offsets, as_stream(stream));
}

int r2s_isect_offset_encode_3d(const int64_t* isect_ids, int64_t n_isects, uint32_t tiles_x, uint32_t tiles_y,
                               uint32_t tiles_z, int32_t* offsets, void* stream) {
    const int64_t n_keys = int64_t(tiles_x) * tiles_y * tiles_z;
    if (n_keys == 0) return R2S_OK;
    offsets_kernel<<<blocks_for(n_keys, 256), 256, 0, as_stream(stream)>>>(isect_ids, n_isects, nullptr, n_keys,
                                                                            offsets);
    return check_launch("isect_offset_encode_3d");
}

int r2s_raster_emit_capacity(const uint16_t* rects, uint32_t C, uint32_t N, uint32_t tiles_x, uint32_t tiles_y,
                             const int64_t* cum_tiles, int64_t capacity, int64_t* n_used, uint32_t* overflow,
                             int64_t* isect_ids, int32_t* flatten_ids, int32_t* offsets, void* workspace,
                             size_t workspace_bytes, void* stream) {
    const uint64_t total = uint64_t(C) * N;
    const uint64_t n_keys = uint64_t(C) * tiles_x * tiles_y;
    R2S_REQUIRE(n_keys < (uint64_t(1) << 32), R2S_ERR_UNSUPPORTED, "C*tiles exceeds the 32-bit key range");
    R2S_REQUIRE(capacity >= 1 && capacity < (int64_t(1) << 31), R2S_ERR_UNSUPPORTED,
                "capacity must be in [1, 2^31)");
    R2S_REQUIRE(n_used != nullptr && overflow != nullptr, R2S_ERR_ARGUMENT, "n_used and overflow must be non-null");
    cudaStream_t st = as_stream(stream);
    count_finish_kernel<<<1, 1, 0, st>>>(cum_tiles, int64_t(total) - 1, capacity, n_used, overflow);
    R2S_TRY(check_launch("count_finish"));
    Arena arena(workspace, workspace_bytes);
    uint32_t* keys = arena.take<uint32_t>(size_t(capacity));
    uint32_t* vals = arena.take<uint32_t>(size_t(capacity));
    R2S_REQUIRE(keys && vals, R2S_ERR_WORKSPACE, "intersection workspace too small");
    if (total > 0) {
        emit_rects_warp_kernel<<<blocks_for(total, 256), 256, 0, st>>>(
            reinterpret_cast<const ushort4*>(rects), uint32_t(total), N, tiles_x, tiles_y, cum_tiles, capacity, keys,
            vals);
        R2S_TRY(check_launch("raster_emit"));
    }
    const CamLayout cams{cum_tiles, C, N, tiles_x * tiles_y};
    return sort_and_finish(keys, vals, capacity, n_keys, arena, isect_ids, flatten_ids, offsets, st, n_used,
                           total > 0 ? &cams : nullptr);
}

int r2s_voxel_emit_capacity(int dtype, const void* means3d, const int32_t* radii, uint32_t N, uint32_t tile_size,
                            uint32_t tiles_x, uint32_t tiles_y, uint32_t tiles_z, const int64_t* cum_tiles,
                            int64_t capacity, int64_t* n_used, uint32_t* overflow, int64_t* isect_ids,
                            int32_t* flatten_ids, int32_t* offsets, void* workspace, size_t workspace_bytes,
                            void* stream) {
    const uint64_t n_keys = uint64_t(tiles_x) * tiles_y * tiles_z;
    R2S_REQUIRE(n_keys < (uint64_t(1) << 32), R2S_ERR_UNSUPPORTED, "tile count exceeds the 32-bit key range");
    R2S_REQUIRE(capacity >= 1 && capacity < (int64_t(1) << 31), R2S_ERR_UNSUPPORTED,
                "capacity must be in [1, 2^31)");
    R2S_REQUIRE(n_used != nullptr && overflow != nullptr, R2S_ERR_ARGUMENT, "n_used and overflow must be non-null");
    cudaStream_t st = as_stream(stream);
    count_finish_kernel<<<1, 1, 0, st>>>(cum_tiles, int64_t(N) - 1, capacity, n_used, overflow);
    R2S_TRY(check_launch("count_finish"));
    Arena arena(workspace, workspace_bytes);
    uint32_t* keys = arena.take<uint32_t>(size_t(capacity));
    uint32_t* vals = arena.take<uint32_t>(size_t(capacity));
    R2S_REQUIRE(keys && vals, R2S_ERR_WORKSPACE, "intersection workspace too small");
    if (N > 0) {
        R2S_DISPATCH(dtype, emit_3d_warp_kernel<S><<<blocks_for(N, 256), 256, 0, st>>>(
            static_cast<const S*>(means3d), radii, N, tile_size, tiles_x, tiles_y, tiles_z, cum_tiles, capacity, keys,
            vals));
        R2S_TRY(check_launch("isect_emit_3d"));
    }
    return sort_and_finish(keys, vals, capacity, n_keys, arena, isect_ids, flatten_ids, offsets, st, n_used);
}

}  // extern "C"
