// Losses: anisotropic total variation over [B,D,H,W] volumes and mean L1 over
// [B,H,W] images, forward (value + optional per-element map) and VJP.
//
// TV forward is one pass over HBM: each voxel reads itself and its +1
// neighbours (neighbour reads hit L1/L2), writes its map entry if requested,
// and blocks reduce in double precision into per-block partials that a single
// block sums in a fixed order -- deterministic, unlike the reference's float
// atomics (VolumeLossFwd.cu:88-119). TV backward folds 1/edges and lambda into
// the same pass (the reference applies lambda in a second torch pass,
// Loss.cpp:187), keeping the reference's rounding order: the sign sum times
// g/edges, then times lambda.
//
// When the upstream gradient is known before the forward (a fit step: the TV
// term enters the loss with weight one), tv_fused_kernel does forward and
// backward in one pass: each thread owns one (y, x) column of a 32 x 8 tile
// and marches down a chunk of depth slices, keeping the previous, current and
// next slice's values in registers, taking its x neighbours from the adjacent
// lanes by shuffle and its y neighbours from the adjacent warps' rows (L1/L2).
// Each voxel is read from DRAM once; the gradient (and the map, if requested)
// is written once. The map and gradient values are the two kernels' above bit
// for bit (same operation order); the loss sums the same fp32 terms in fp64 in
// another fixed order.
#include "common.cuh"

namespace r2s {

constexpr int kLossThreads = 256;
constexpr int kLossMaxBlocks = 148 * 8;

template <typename S>
__device__ __forceinline__ S abs_diff(S x) { return x >= S(0) ? x : -x; }

template <typename S>
__device__ __forceinline__ S sign_of(S x) { return x > S(0) ? S(1) : (x < S(0) ? S(-1) : S(0)); }

__device__ __forceinline__ double block_sum(double v) {
    __shared__ double warp_part[kLossThreads / 32];
    v = warp_sum(v);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) warp_part[warp] = v;
    __syncthreads();
    double total = 0;
    if (threadIdx.x == 0) {
        for (int w = 0; w < kLossThreads / 32; ++w) total += warp_part[w];
    }
    return total;
}

// Each block takes a contiguous range of rows (a row is one (b, d, h) line of W
// voxels) and its threads stride along x. The first row's (d, h) is derived
// once per block and then advanced by one per row, so no voxel pays an index
// division; blocks walk fixed row ranges in a fixed order, so the double
// partial sums (and the loss) are deterministic.
__device__ __forceinline__ void first_row(uint64_t rows, uint32_t D, uint32_t H, uint64_t& r0, uint64_t& r1,
                                          uint32_t& d, uint32_t& h) {
    const uint64_t per = (rows + gridDim.x - 1) / gridDim.x;
    r0 = uint64_t(blockIdx.x) * per;
    r1 = r0 + per < rows ? r0 + per : rows;
    h = uint32_t(r0 % H);
    d = uint32_t((r0 / H) % D);
}

__device__ __forceinline__ void next_row(uint32_t D, uint32_t H, uint32_t& d, uint32_t& h) {
    if (++h == H) {
        h = 0;
        if (++d == D) d = 0;
    }
}

template <typename S>
__global__ void __launch_bounds__(kLossThreads) tv_fwd_kernel(const S* __restrict__ vol, uint32_t D, uint32_t H,
                                                              uint32_t W, uint64_t rows, S* __restrict__ tv_map,
                                                              double* __restrict__ partials) {
    double sum = 0;
    const uint64_t HW = uint64_t(H) * W;
    uint64_t r0, r1;
    uint32_t d, h;
    first_row(rows, D, H, r0, r1, d, h);
    for (uint64_t row = r0; row < r1; ++row, next_row(D, H, d, h)) {
        const uint64_t base = row * W;
        for (uint32_t x = threadIdx.x; x < W; x += kLossThreads) {
            const uint64_t idx = base + x;
            const S val = vol[idx];
            S tv = 0;
            if (d + 1 < D) tv += abs_diff(vol[idx + HW] - val);
            if (h + 1 < H) tv += abs_diff(vol[idx + W] - val);
            if (x + 1 < W) tv += abs_diff(vol[idx + 1] - val);
            if (tv_map != nullptr) tv_map[idx] = tv;
            sum += static_cast<double>(tv);
        }
    }
    const double total_sum = block_sum(sum);
    if (threadIdx.x == 0) partials[blockIdx.x] = total_sum;
}

constexpr uint32_t kTvTileX = 32, kTvTileY = kLossThreads / 32, kTvChunk = 32;

template <typename S, bool kMap>
__global__ void __launch_bounds__(kLossThreads) tv_fused_kernel(
    const S* __restrict__ vol, uint32_t D, uint32_t H, uint32_t W, uint32_t tiles_x, uint32_t tiles_y,
    uint32_t chunks, uint64_t n_tiles, const S* __restrict__ grad_output, int64_t edges, float lambda,
    S* __restrict__ tv_map, S* __restrict__ grad, double* __restrict__ partials) {
    const S grad_out = grad_output[0] / static_cast<S>(edges);
    const S lam = static_cast<S>(lambda);
    const uint64_t HW = uint64_t(H) * W;
    const uint32_t lx = threadIdx.x & 31u, ly = threadIdx.x >> 5;
    double sum = 0;
    for (uint64_t tile = blockIdx.x; tile < n_tiles; tile += gridDim.x) {
        uint64_t t = tile;
        const uint32_t tx = uint32_t(t % tiles_x);
        t /= tiles_x;
        const uint32_t ty = uint32_t(t % tiles_y);
        t /= tiles_y;
        const uint32_t chunk = uint32_t(t % chunks);
        const uint64_t b = t / chunks;
        const uint32_t x = tx * kTvTileX + lx, y = ty * kTvTileY + ly;
        const uint32_t d0 = chunk * kTvChunk, d1 = min(D, d0 + kTvChunk);
        const bool active = x < W && y < H;
        const uint64_t column = b * D * HW + uint64_t(y) * W + x;
        S prev = S(0), cur = S(0), next = S(0);
        if (active) {
            cur = vol[column + uint64_t(d0) * HW];
            if (d0 > 0) prev = vol[column + uint64_t(d0 - 1) * HW];
        }
        for (uint32_t d = d0; d < d1; ++d) {
            const uint64_t idx = column + uint64_t(d) * HW;
            if (active && d + 1 < D) next = vol[idx + HW];
            // Inactive lanes hold 0; a lane reads a neighbour's value only when that neighbour is inside.
            S xp = __shfl_down_sync(0xffffffffu, cur, 1);
            S xm = __shfl_up_sync(0xffffffffu, cur, 1);
            if (active) {
                if (lx == 31u && x + 1 < W) xp = vol[idx + 1];
                if (lx == 0u && x > 0) xm = vol[idx - 1];
                const S yp = y + 1 < H ? vol[idx + W] : S(0);
                const S ym = y > 0 ? vol[idx - W] : S(0);
                S tv = 0;
                if (d + 1 < D) tv += abs_diff(next - cur);
                if (y + 1 < H) tv += abs_diff(yp - cur);
                if (x + 1 < W) tv += abs_diff(xp - cur);
                S g = 0;
                if (d + 1 < D) g -= sign_of(next - cur);
                if (d > 0) g += sign_of(cur - prev);
                if (y + 1 < H) g -= sign_of(yp - cur);
                if (y > 0) g += sign_of(cur - ym);
                if (x + 1 < W) g -= sign_of(xp - cur);
                if (x > 0) g += sign_of(cur - xm);
                if (kMap) tv_map[idx] = tv;
                grad[idx] = (g * grad_out) * lam;
                sum += static_cast<double>(tv);
            }
            prev = cur;
            cur = next;
        }
    }
    const double total_sum = block_sum(sum);
    if (threadIdx.x == 0) partials[blockIdx.x] = total_sum;
}

// The fused pass on fp32 volumes whose rows are whole float4s (W % 4 == 0, 16-byte aligned): each
// lane owns four consecutive voxels of a row (one 16-byte load per slice), a warp 128 voxels of
// one row, the block 8 rows, over kTv4Chunk slices; the centre row two slices ahead and the two
// neighbouring rows one slice ahead are loaded while the current slice is computed. Short chunks
// keep enough warps in flight to cover the loads (a 256^3 volume makes 1024 block tiles). At 256^3:
// chunks of 4, 8 and 16 slices took 0.069, 0.065 and 0.063 ms; 32 slices without the row
// prefetch, 0.075 ms.
// Per voxel the operations and their order are tv_fused_kernel's.
constexpr uint32_t kTv4TileX = 128;
constexpr uint32_t kTv4Chunk = 16;

__device__ __forceinline__ float tv_at(float cur, float next, float yp, float xp, bool dz, bool dy, bool dx) {
    float tv = 0.f;
    if (dz) tv += abs_diff(next - cur);
    if (dy) tv += abs_diff(yp - cur);
    if (dx) tv += abs_diff(xp - cur);
    return tv;
}

__device__ __forceinline__ float tv_grad_at(float cur, float prev, float next, float yp, float ym, float xp,
                                            float xm, bool zn, bool zp, bool yn, bool yq, bool xn, bool xq) {
    float g = 0.f;
    if (zn) g -= sign_of(next - cur);
    if (zp) g += sign_of(cur - prev);
    if (yn) g -= sign_of(yp - cur);
    if (yq) g += sign_of(cur - ym);
    if (xn) g -= sign_of(xp - cur);
    if (xq) g += sign_of(cur - xm);
    return g;
}

template <bool kMap>
__global__ void __launch_bounds__(kLossThreads) tv_fused4_kernel(
    const float* __restrict__ vol, uint32_t D, uint32_t H, uint32_t W, uint32_t tiles_x, uint32_t tiles_y,
    uint32_t chunks, uint64_t n_tiles, const float* __restrict__ grad_output, int64_t edges, float lambda,
    float* __restrict__ tv_map, float* __restrict__ grad, double* __restrict__ partials) {
    const float grad_out = grad_output[0] / static_cast<float>(edges);
    const float lam = lambda;
    const uint64_t HW = uint64_t(H) * W;
    const uint32_t lane = threadIdx.x & 31u, ly = threadIdx.x >> 5;
    double sum = 0;
    for (uint64_t tile = blockIdx.x; tile < n_tiles; tile += gridDim.x) {
        uint64_t t = tile;
        const uint32_t tx = uint32_t(t % tiles_x);
        t /= tiles_x;
        const uint32_t ty = uint32_t(t % tiles_y);
        t /= tiles_y;
        const uint32_t chunk = uint32_t(t % chunks);
        const uint64_t b = t / chunks;
        const uint32_t x = tx * kTv4TileX + 4u * lane, y = ty * kTvTileY + ly;
        const uint32_t d0 = chunk * kTv4Chunk, d1 = min(D, d0 + kTv4Chunk);
        const bool active = x < W && y < H;  // W % 4 == 0: a lane's four voxels are all in or all out
        const uint64_t column = b * D * HW + uint64_t(y) * W + x;
        const float4 zero4 = make_float4(0.f, 0.f, 0.f, 0.f);
        const bool has_yp = active && y + 1 < H, has_ym = active && y > 0;
        auto load4 = [&](bool ok, uint32_t d, int64_t dy) {
            return (ok && d < D)
                       ? __ldg(reinterpret_cast<const float4*>(vol + column + uint64_t(d) * HW + dy * int64_t(W)))
                       : zero4;
        };
        float4 prev = d0 > 0 ? load4(active, d0 - 1, 0) : zero4;
        float4 cur = load4(active, d0, 0);
        float4 next = load4(active, d0 + 1, 0);
        float4 yp_next = load4(has_yp, d0, 1), ym_next = load4(has_ym, d0, -1);
        for (uint32_t d = d0; d < d1; ++d) {
            // In flight while this slice is computed: the centre row two slices ahead, the
            // neighbouring rows one ahead.
            const float4 ahead = load4(active, d + 2, 0);
            const float4 yp = yp_next, ym = ym_next;
            yp_next = load4(has_yp, d + 1, 1);
            ym_next = load4(has_ym, d + 1, -1);
            const uint64_t idx = column + uint64_t(d) * HW;
            // x neighbours: the adjacent lanes' edge voxels; the warp's first and last lanes load them.
            float xp = __shfl_down_sync(0xffffffffu, cur.x, 1);
            float xm = __shfl_up_sync(0xffffffffu, cur.w, 1);
            if (active) {
                if (lane == 31u && x + 4 < W) xp = vol[idx + 4];
                if (lane == 0u && x > 0) xm = vol[idx - 1];
                const bool zn = d + 1 < D, zp = d > 0, yn = y + 1 < H, yq = y > 0;
                const bool xn3 = x + 4 < W, xq0 = x > 0;
                float4 m, g;
                m.x = tv_at(cur.x, next.x, yp.x, cur.y, zn, yn, true);
                m.y = tv_at(cur.y, next.y, yp.y, cur.z, zn, yn, true);
                m.z = tv_at(cur.z, next.z, yp.z, cur.w, zn, yn, true);
                m.w = tv_at(cur.w, next.w, yp.w, xp, zn, yn, xn3);
                g.x = tv_grad_at(cur.x, prev.x, next.x, yp.x, ym.x, cur.y, xm, zn, zp, yn, yq, true, xq0);
                g.y = tv_grad_at(cur.y, prev.y, next.y, yp.y, ym.y, cur.z, cur.x, zn, zp, yn, yq, true, true);
                g.z = tv_grad_at(cur.z, prev.z, next.z, yp.z, ym.z, cur.w, cur.y, zn, zp, yn, yq, true, true);
                g.w = tv_grad_at(cur.w, prev.w, next.w, yp.w, ym.w, xp, cur.z, zn, zp, yn, yq, xn3, true);
                if (kMap) *reinterpret_cast<float4*>(tv_map + idx) = m;
                *reinterpret_cast<float4*>(grad + idx) =
                    make_float4((g.x * grad_out) * lam, (g.y * grad_out) * lam, (g.z * grad_out) * lam,
                                (g.w * grad_out) * lam);
                sum += static_cast<double>(m.x) + static_cast<double>(m.y) + static_cast<double>(m.z) +
                       static_cast<double>(m.w);
            }
            prev = cur;
            cur = next;
            next = ahead;
        }
    }
    const double total_sum = block_sum(sum);
    if (threadIdx.x == 0) partials[blockIdx.x] = total_sum;
}

template <typename S>
__global__ void __launch_bounds__(kLossThreads) l1_fwd_kernel(const S* __restrict__ pred, const S* __restrict__ tgt,
                                                              int64_t total, S* __restrict__ l1_map,
                                                              double* __restrict__ partials) {
    double sum = 0;
    for (int64_t idx = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; idx < total;
         idx += int64_t(gridDim.x) * blockDim.x) {
        const S v = abs_diff(pred[idx] - tgt[idx]);
        if (l1_map != nullptr) l1_map[idx] = v;
        sum += static_cast<double>(v);
    }
    const double total_sum = block_sum(sum);
    if (threadIdx.x == 0) partials[blockIdx.x] = total_sum;
}

// Sums the per-block partials in order; value = sum / count, loss = lambda * value.
template <typename S>
__global__ void finish_mean_kernel(const double* __restrict__ partials, int n_partials, int64_t count,
                                   float lambda, S* __restrict__ loss, S* __restrict__ value) {
    __shared__ double s[kLossThreads];
    double v = 0;
    for (int i = threadIdx.x; i < n_partials; i += kLossThreads) v += partials[i];
    s[threadIdx.x] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        double total = 0;
        for (int i = 0; i < kLossThreads; ++i) total += s[i];
        const S mean = static_cast<S>(total / static_cast<double>(count > 0 ? count : 1));
        *value = mean;
        *loss = static_cast<S>(lambda) * mean;
    }
}

template <typename S>
__global__ void tv_bwd_kernel(const S* __restrict__ vol, const S* __restrict__ grad_output, uint32_t D, uint32_t H,
                              uint32_t W, uint64_t rows, int64_t edges, float lambda, S* __restrict__ grad) {
    const S grad_out = grad_output[0] / static_cast<S>(edges);
    const S lam = static_cast<S>(lambda);
    const uint64_t HW = uint64_t(H) * W;
    uint64_t r0, r1;
    uint32_t d, h;
    first_row(rows, D, H, r0, r1, d, h);
    for (uint64_t row = r0; row < r1; ++row, next_row(D, H, d, h)) {
        const uint64_t base = row * W;
        for (uint32_t x = threadIdx.x; x < W; x += blockDim.x) {
            const uint64_t idx = base + x;
            const S val = vol[idx];
            S g = 0;
            if (d + 1 < D) g -= sign_of(vol[idx + HW] - val);
            if (d > 0) g += sign_of(val - vol[idx - HW]);
            if (h + 1 < H) g -= sign_of(vol[idx + W] - val);
            if (h > 0) g += sign_of(val - vol[idx - W]);
            if (x + 1 < W) g -= sign_of(vol[idx + 1] - val);
            if (x > 0) g += sign_of(val - vol[idx - 1]);
            grad[idx] = (g * grad_out) * lam;
        }
    }
}

template <typename S>
__global__ void l1_bwd_kernel(const S* __restrict__ pred, const S* __restrict__ tgt, const S* __restrict__ grad_output,
                              int64_t total, float lambda, S* __restrict__ grad) {
    const S lam = static_cast<S>(lambda);
    for (int64_t idx = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; idx < total;
         idx += int64_t(gridDim.x) * blockDim.x) {
        const S s = sign_of(pred[idx] - tgt[idx]);
        grad[idx] = grad_output[0] * lam * s / static_cast<S>(total);
    }
}

inline unsigned loss_blocks(int64_t total) {
    int64_t b = (total + kLossThreads - 1) / kLossThreads;
    if (b > kLossMaxBlocks) b = kLossMaxBlocks;
    if (b < 1) b = 1;
    return unsigned(b);
}

// Sums `n_partials` fp64 partials in a fixed order into value = sum / count and
// loss = lambda * value; shared with the forward's fused image-loss epilogue.
int launch_finish_mean(int dtype, const double* partials, int n_partials, int64_t count, float lambda, void* loss,
                       void* value, cudaStream_t stream) {
    R2S_DISPATCH(dtype, {
        finish_mean_kernel<S><<<1, kLossThreads, 0, stream>>>(partials, n_partials, count, lambda,
                                                             static_cast<S*>(loss), static_cast<S*>(value));
        return check_launch("loss_finish");
    });
}

}  // namespace r2s

using namespace r2s;

extern "C" {

size_t r2s_volume_loss_workspace(uint64_t numel) {
    (void)numel;
    return size_t(kLossMaxBlocks) * sizeof(double) + 256;
}

int r2s_volume_loss_fwd(int dtype, const void* volume, uint32_t B, uint32_t D, uint32_t H, uint32_t W,
                        float lambda_tv, void* loss, void* tv, void* tv_map, void* workspace, size_t workspace_bytes,
                        void* stream) {
    const int64_t total = int64_t(B) * D * H * W;
    const int64_t edges_raw = int64_t(B) * ((int64_t(D) - 1) * H * W + int64_t(D) * (H - 1) * W +
                                            int64_t(D) * H * (int64_t(W) - 1));
    const int64_t edges = edges_raw > 1 ? edges_raw : 1;
    Arena arena(workspace, workspace_bytes);
    const unsigned blocks = loss_blocks(total);
    double* partials = arena.take<double>(blocks);
    R2S_REQUIRE(partials, R2S_ERR_WORKSPACE, "loss workspace too small");
    cudaStream_t st = as_stream(stream);
    R2S_DISPATCH(dtype, {
        if (total > 0) {
            const uint64_t rows = uint64_t(B) * D * H;
            tv_fwd_kernel<S><<<blocks, kLossThreads, 0, st>>>(static_cast<const S*>(volume), D, H, W, rows,
                                                             static_cast<S*>(tv_map), partials);
            R2S_TRY(check_launch("volume_loss_fwd"));
        }
        finish_mean_kernel<S><<<1, kLossThreads, 0, st>>>(partials, total > 0 ? int(blocks) : 0, edges, lambda_tv,
                                                         static_cast<S*>(loss), static_cast<S*>(tv));
        return check_launch("volume_loss_finish");
    });
}

int r2s_volume_loss_bwd(int dtype, const void* volume, const void* grad_output, uint32_t B, uint32_t D, uint32_t H,
                        uint32_t W, float lambda_tv, void* grad_volume, void* stream) {
    const int64_t total = int64_t(B) * D * H * W;
    if (total == 0) return R2S_OK;
    const int64_t edges_raw = int64_t(B) * ((int64_t(D) - 1) * H * W + int64_t(D) * (H - 1) * W +
                                            int64_t(D) * H * (int64_t(W) - 1));
    const int64_t edges = edges_raw > 1 ? edges_raw : 1;
    const uint64_t rows = uint64_t(B) * D * H;
    R2S_DISPATCH(dtype, {
        tv_bwd_kernel<S><<<loss_blocks(total), kLossThreads, 0, as_stream(stream)>>>(
            static_cast<const S*>(volume), static_cast<const S*>(grad_output), D, H, W, rows, edges, lambda_tv,
            static_cast<S*>(grad_volume));
        return check_launch("volume_loss_bwd");
    });
}

int r2s_volume_loss_fwd_bwd(int dtype, const void* volume, const void* grad_output, uint32_t B, uint32_t D,
                            uint32_t H, uint32_t W, float lambda_tv, void* loss, void* tv, void* tv_map,
                            void* grad_volume, void* workspace, size_t workspace_bytes, void* stream) {
    const int64_t total = int64_t(B) * D * H * W;
    const int64_t edges_raw = int64_t(B) * ((int64_t(D) - 1) * H * W + int64_t(D) * (H - 1) * W +
                                            int64_t(D) * H * (int64_t(W) - 1));
    const int64_t edges = edges_raw > 1 ? edges_raw : 1;
    R2S_REQUIRE(grad_output != nullptr && grad_volume != nullptr, R2S_ERR_ARGUMENT,
                "grad_output and grad_volume must be non-null");
    const uint32_t tiles_x = (W + kTvTileX - 1) / kTvTileX, tiles_y = (H + kTvTileY - 1) / kTvTileY;
    const uint32_t chunks = (D + kTvChunk - 1) / kTvChunk;
    const uint64_t n_tiles = uint64_t(B) * chunks * tiles_y * tiles_x;
    const unsigned blocks = unsigned(n_tiles < uint64_t(kLossMaxBlocks) ? (n_tiles > 0 ? n_tiles : 1)
                                                                        : uint64_t(kLossMaxBlocks));
    Arena arena(workspace, workspace_bytes);
    double* partials = arena.take<double>(blocks);
    R2S_REQUIRE(partials, R2S_ERR_WORKSPACE, "loss workspace too small");
    cudaStream_t st = as_stream(stream);
    const bool vec4 = dtype == R2S_F32 && W % 4 == 0 && reinterpret_cast<uintptr_t>(volume) % 16 == 0 &&
                      reinterpret_cast<uintptr_t>(grad_volume) % 16 == 0 &&
                      (tv_map == nullptr || reinterpret_cast<uintptr_t>(tv_map) % 16 == 0);
    if (vec4 && total > 0) {
        const uint32_t tiles4_x = (W + kTv4TileX - 1) / kTv4TileX;
        const uint32_t chunks4 = (D + kTv4Chunk - 1) / kTv4Chunk;
        const uint64_t n4 = uint64_t(B) * chunks4 * tiles_y * tiles4_x;
        const unsigned blocks4 = unsigned(n4 < uint64_t(kLossMaxBlocks) ? n4 : uint64_t(kLossMaxBlocks));
        // blocks4 <= kLossMaxBlocks, the partials the workspace was sized for.
        Arena arena4(workspace, workspace_bytes);
        double* partials4 = arena4.take<double>(blocks4);
        R2S_REQUIRE(partials4, R2S_ERR_WORKSPACE, "loss workspace too small");
        if (tv_map != nullptr) {
            tv_fused4_kernel<true><<<blocks4, kLossThreads, 0, st>>>(
                static_cast<const float*>(volume), D, H, W, tiles4_x, tiles_y, chunks4, n4,
                static_cast<const float*>(grad_output), edges, lambda_tv, static_cast<float*>(tv_map),
                static_cast<float*>(grad_volume), partials4);
        } else {
            tv_fused4_kernel<false><<<blocks4, kLossThreads, 0, st>>>(
                static_cast<const float*>(volume), D, H, W, tiles4_x, tiles_y, chunks4, n4,
                static_cast<const float*>(grad_output), edges, lambda_tv, nullptr, static_cast<float*>(grad_volume),
                partials4);
        }
        R2S_TRY(check_launch("volume_loss_fwd_bwd"));
        finish_mean_kernel<float><<<1, kLossThreads, 0, st>>>(partials4, int(blocks4), edges, lambda_tv,
                                                              static_cast<float*>(loss), static_cast<float*>(tv));
        return check_launch("volume_loss_finish");
    }
    R2S_DISPATCH(dtype, {
        if (total > 0) {
            if (tv_map != nullptr) {
                tv_fused_kernel<S, true><<<blocks, kLossThreads, 0, st>>>(
                    static_cast<const S*>(volume), D, H, W, tiles_x, tiles_y, chunks, n_tiles,
                    static_cast<const S*>(grad_output), edges, lambda_tv, static_cast<S*>(tv_map),
                    static_cast<S*>(grad_volume), partials);
            } else {
                tv_fused_kernel<S, false><<<blocks, kLossThreads, 0, st>>>(
                    static_cast<const S*>(volume), D, H, W, tiles_x, tiles_y, chunks, n_tiles,
                    static_cast<const S*>(grad_output), edges, lambda_tv, nullptr, static_cast<S*>(grad_volume),
                    partials);
            }
            R2S_TRY(check_launch("volume_loss_fwd_bwd"));
        }
        finish_mean_kernel<S><<<1, kLossThreads, 0, st>>>(partials, total > 0 ? int(blocks) : 0, edges, lambda_tv,
                                                         static_cast<S*>(loss), static_cast<S*>(tv));
        return check_launch("volume_loss_finish");
    });
}

int r2s_image_loss_l1_fwd(int dtype, const void* prediction, const void* target, uint32_t B, uint32_t H, uint32_t W,
                          float lambda_l1, void* loss, void* l1, void* l1_map, void* workspace,
                          size_t workspace_bytes, void* stream) {
    const int64_t total = int64_t(B) * H * W;
    Arena arena(workspace, workspace_bytes);
    const unsigned blocks = loss_blocks(total);
    double* partials = arena.take<double>(blocks);
    R2S_REQUIRE(partials, R2S_ERR_WORKSPACE, "loss workspace too small");
    cudaStream_t st = as_stream(stream);
    R2S_DISPATCH(dtype, {
        if (total > 0) {
            l1_fwd_kernel<S><<<blocks, kLossThreads, 0, st>>>(static_cast<const S*>(prediction),
                                                             static_cast<const S*>(target), total,
                                                             static_cast<S*>(l1_map), partials);
            R2S_TRY(check_launch("image_loss_fwd"));
        }
        finish_mean_kernel<S><<<1, kLossThreads, 0, st>>>(partials, total > 0 ? int(blocks) : 0, total, lambda_l1,
                                                         static_cast<S*>(loss), static_cast<S*>(l1));
        return check_launch("image_loss_finish");
    });
}

int r2s_image_loss_l1_bwd(int dtype, const void* prediction, const void* target, const void* grad_output, uint32_t B,
                          uint32_t H, uint32_t W, float lambda_l1, void* grad_prediction, void* stream) {
    const int64_t total = int64_t(B) * H * W;
    if (total == 0) return R2S_OK;
    R2S_DISPATCH(dtype, {
        l1_bwd_kernel<S><<<loss_blocks(total), kLossThreads, 0, as_stream(stream)>>>(
            static_cast<const S*>(prediction), static_cast<const S*>(target), static_cast<const S*>(grad_output), total,
            lambda_l1, static_cast<S*>(grad_prediction));
        return check_launch("image_loss_bwd");
    });
}

}  // extern "C"
