// Projection rasterization: per-tile additive line-integral accumulation
// (no alpha compositing) and its VJP, on packed per-(camera, primitive)
// records.
//
// Layout and schedule (B200):
//  * one CTA per (tile, camera); blockIdx.x = tile, blockIdx.y = camera, so
//    CTAs run camera-major and one camera's records ([N] x 32 B) stay resident
//    in L2 while its tiles are processed;
//  * the tile's intersection list (contiguous in the sorted flatten_ids) is
//    staged in shared memory in batches, each thread gathering one 32-byte
//    record with two 16-byte cp.async copies, double-buffered so the next
//    batch's gather overlaps the current batch's arithmetic;
//  * forward: each thread owns up to 4 pixels; backward: each warp owns one
//    record at a time and evaluates it on every pixel of its sub-tile (8 per
//    lane), then warp-reduces and issues two vector atomics per record.
//
// Per-sample arithmetic keeps the reference's expression forms
// (RasterizeToPixelsFwd.cu:160-177, :664-680; RasterizeToPixelsBwd.cu:417-468,
// :910-945): the contribution thresholds (|alpha| < 1e-5, sigma < 0, d2 >= 1)
// decide which samples count, so alpha must round exactly as the reference's
// does. A thread's pixels are placed so that no two share an x or a y
// coordinate, which keeps every product single-use, as in the reference's
// one-pixel-per-thread loops, and so the compiler contracts the same
// multiply-adds.
#include "common.cuh"

namespace r2s {

// Pixel placement: the p-th pixel of a tile sits at row p / T and column
// (p % T + 7 * row) % T -- a per-row rotation, so rows stay bijective while
// pixels p and p + 32k (one lane) or p and p + nthreads (one thread) get
// different columns.
__device__ __forceinline__ void tile_pixel(uint32_t p, uint32_t T, uint32_t& ly, uint32_t& lx) {
    ly = p / T;
    lx = (p - ly * T + 7u * ly) % T;
}

template <typename S>
__device__ __forceinline__ void gather_record(Rec2D<S>* dst, const Rec2D<S>* src) {
    const char* s = reinterpret_cast<const char*>(src);
    char* d = reinterpret_cast<char*>(dst);
#pragma unroll
    for (int k = 0; k < int(sizeof(Rec2D<S>) / 16); ++k) cp_async16(d + 16 * k, s + 16 * k);
}

// --------------------------------------------------------------------------
// Forward
// --------------------------------------------------------------------------

template <typename S, bool kBeta, bool kVar, int PPT>
__global__ void __launch_bounds__(256) raster_fwd_kernel(
    const Rec2D<S>* __restrict__ records, const S* __restrict__ uncertainties, uint32_t N,
    const int32_t* __restrict__ offsets, const int32_t* __restrict__ flatten_ids, int32_t n_isects,
    uint32_t C, uint32_t width, uint32_t height, uint32_t T, uint32_t tiles_x, uint32_t n_tiles,
    S* __restrict__ render, S* __restrict__ render_var) {
    extern __shared__ __align__(16) unsigned char smem[];
    const uint32_t nthreads = blockDim.x;
    Rec2D<S>* s_rec = reinterpret_cast<Rec2D<S>*>(smem);                 // [2][nthreads]
    S* s_q = reinterpret_cast<S*>(s_rec + 2 * nthreads);                   // [2][nthreads]

    const uint32_t tile = blockIdx.x, cam = blockIdx.y;
    const uint32_t key = cam * n_tiles + tile;
    const int32_t start = offsets[key];
    const int32_t end = (key + 1 == C * n_tiles) ? n_isects : offsets[key + 1];
    const uint32_t ty = tile / tiles_x, tx = tile - ty * tiles_x;
    const uint32_t t = threadIdx.x;

    S px[PPT], py[PPT], acc[PPT], accv[PPT];
    uint32_t pix[PPT];
    bool inside[PPT];
#pragma unroll
    for (int k = 0; k < PPT; ++k) {
        const uint32_t p = t + uint32_t(k) * nthreads;
        uint32_t ly, lx;
        tile_pixel(p, T, ly, lx);
        const uint32_t i = ty * T + ly, j = tx * T + lx;
        inside[k] = p < T * T && i < height && j < width;
        px[k] = static_cast<S>(j) + static_cast<S>(0.5);
        py[k] = static_cast<S>(i) + static_cast<S>(0.5);
        pix[k] = i * width + j;
        acc[k] = S(0);
        accv[k] = S(0);
    }

    const int32_t count = end - start;
    const int32_t n_batches = count > 0 ? (count + int32_t(nthreads) - 1) / int32_t(nthreads) : 0;
    auto load = [&](int32_t b, int stage) {
        const int32_t idx = start + b * int32_t(nthreads) + int32_t(t);
        if (idx < end) {
            const int32_t g = flatten_ids[idx];
            gather_record(s_rec + stage * nthreads + t, records + g);
            if (kVar) s_q[stage * nthreads + t] = uncertainties[uint32_t(g) % N];
        }
        cp_async_commit();
    };
    if (n_batches > 0) load(0, 0);
    for (int32_t b = 0; b < n_batches; ++b) {
        if (b + 1 < n_batches) {
            load(b + 1, (b + 1) & 1);
            cp_async_wait<1>();
        } else {
            cp_async_wait<0>();
        }
        __syncthreads();
        const Rec2D<S>* buf = s_rec + (b & 1) * nthreads;
        const S* qbuf = s_q + (b & 1) * nthreads;
        const int32_t batch = min(int32_t(nthreads), count - b * int32_t(nthreads));
#pragma unroll 2
        for (int32_t s = 0; s < batch; ++s) {
            const Rec2D<S> r = buf[s];
            const S om = r.o * r.mu;
            S q = S(0);
            if (kVar) q = qbuf[s];
#pragma unroll
            for (int k = 0; k < PPT; ++k) {
                if (!kBeta) {
                    const S dx = px[k] - r.x;
                    const S dy = py[k] - r.y;
                    const S sigma = static_cast<S>(0.5) * (r.a * dx * dx + r.c * dy * dy) + r.b * dx * dy;
                    const S alpha = om * exp(-sigma);
                    if (!(sigma < static_cast<S>(0) || fabs(alpha) < static_cast<S>(1e-5))) {
                        acc[k] += alpha;
                        if (kVar) accv[k] += q * alpha * alpha;
                    }
                } else {
                    const S dx = r.x - px[k];
                    const S dy = r.y - py[k];
                    const S d2 = r.a * dx * dx + static_cast<S>(2) * r.b * dx * dy + r.c * dy * dy;
                    if (!(d2 < static_cast<S>(0) || d2 >= static_cast<S>(1))) {
                        const S h = static_cast<S>(1) - d2;
                        const S alpha = om * pow(h, r.beta);
                        if (!(fabs(alpha) < static_cast<S>(1e-5))) {
                            acc[k] += alpha;
                            if (kVar) accv[k] += q * alpha * alpha;
                        }
                    }
                }
            }
        }
        __syncthreads();
    }
    const size_t cam_base = size_t(cam) * height * width;
#pragma unroll
    for (int k = 0; k < PPT; ++k) {
        if (inside[k]) {
            render[cam_base + pix[k]] = acc[k];
            if (kVar) render_var[cam_base + pix[k]] = accv[k];
        }
    }
}

// --------------------------------------------------------------------------
// Backward
// --------------------------------------------------------------------------

constexpr int kBwdWarps = 8;
constexpr int kBwdThreads = kBwdWarps * 32;

// Optional outputs are selected at run time by null pointers:
//   v_render null      -> zero image adjoint (uncertainty-only VJP)
//   v_render_var null  -> no variance branch
//   var_q null         -> detached variance branch (no 2 q alpha v_var term)
//   grads null         -> skip the record-slot adjoints
//   v_abs / v_unc null -> skip absgrad / uncertainty adjoints
//
// The per-sample body is branch-free: a skipped sample keeps its arithmetic
// but has its alpha and visibility selected to zero, so every contribution
// it would add is an exact zero and the compiler can interleave the lane's
// pixels (a `continue` per pixel serialises their exp/pow latencies).
template <typename S, bool kBeta, bool kVar, bool kAbs, int PPL>
__global__ void __launch_bounds__(kBwdThreads) raster_bwd_kernel(
    const Rec2D<S>* __restrict__ records, const S* __restrict__ var_q, uint32_t N,
    const int32_t* __restrict__ offsets, const int32_t* __restrict__ flatten_ids, int32_t n_isects,
    uint32_t C, uint32_t width, uint32_t height, uint32_t T, uint32_t tiles_x, uint32_t n_tiles,
    const S* __restrict__ v_render, const S* __restrict__ v_render_var, Rec2D<S>* __restrict__ grads,
    S* __restrict__ v_abs, S* __restrict__ v_unc) {
    extern __shared__ __align__(16) unsigned char smem[];
    Rec2D<S>* s_rec = reinterpret_cast<Rec2D<S>*>(smem);            // [2][kBwdThreads]
    S* s_q = reinterpret_cast<S*>(s_rec + 2 * kBwdThreads);           // [2][kBwdThreads]
    int32_t* s_id = reinterpret_cast<int32_t*>(s_q + 2 * kBwdThreads);  // [2][kBwdThreads]

    const uint32_t tile = blockIdx.x, cam = blockIdx.y;
    const uint32_t key = cam * n_tiles + tile;
    const int32_t start = offsets[key];
    const int32_t end = (key + 1 == C * n_tiles) ? n_isects : offsets[key + 1];
    const int32_t count = end - start;
    if (count <= 0) return;
    const uint32_t ty = tile / tiles_x, tx = tile - ty * tiles_x;
    const uint32_t t = threadIdx.x, lane = t & 31, warp = t >> 5;

    // Sub-tiles of 32 * PPL pixels; warps split over sub-tiles, then records.
    const uint32_t sub_pixels = 32u * PPL;
    uint32_t n_sub = 1;  // a power of two, so it divides kBwdWarps (tiles are at most 32x32)
    while (n_sub * sub_pixels < T * T) n_sub <<= 1;
    const uint32_t my_sub = warp % n_sub;
    const uint32_t warps_per_sub = kBwdWarps / n_sub;
    const uint32_t my_lane_group = warp / n_sub;

    const bool chain_var = kVar && var_q != nullptr;
    S px[PPL], py[PPL], vr[PPL], vv[PPL];
    bool valid[PPL];
    const size_t cam_base = size_t(cam) * height * width;
#pragma unroll
    for (int k = 0; k < PPL; ++k) {
        const uint32_t p = my_sub * sub_pixels + lane + 32u * k;
        uint32_t ly, lx;
        tile_pixel(p, T, ly, lx);
        const uint32_t i = ty * T + ly, j = tx * T + lx;
        valid[k] = p < T * T && i < height && j < width;
        px[k] = static_cast<S>(j) + static_cast<S>(0.5);
        py[k] = static_cast<S>(i) + static_cast<S>(0.5);
        const size_t pid = cam_base + size_t(i) * width + j;
        vr[k] = (valid[k] && v_render != nullptr) ? v_render[pid] : S(0);
        vv[k] = (kVar && valid[k]) ? v_render_var[pid] : S(0);
    }

    const int32_t n_batches = (count + kBwdThreads - 1) / kBwdThreads;
    auto load = [&](int32_t b, int stage) {
        const int32_t idx = start + b * kBwdThreads + int32_t(t);
        if (idx < end) {
            const int32_t g = flatten_ids[idx];
            gather_record(s_rec + stage * kBwdThreads + t, records + g);
            s_id[stage * kBwdThreads + t] = g;
            if (chain_var) s_q[stage * kBwdThreads + t] = var_q[uint32_t(g) % N];
        }
        cp_async_commit();
    };
    load(0, 0);
    for (int32_t b = 0; b < n_batches; ++b) {
        if (b + 1 < n_batches) {
            load(b + 1, (b + 1) & 1);
            cp_async_wait<1>();
        } else {
            cp_async_wait<0>();
        }
        __syncthreads();
        const int stage = b & 1;
        const int32_t batch = min(int32_t(kBwdThreads), count - b * kBwdThreads);
        for (int32_t s = int32_t(my_lane_group); s < batch; s += int32_t(warps_per_sub)) {
            const Rec2D<S> r = s_rec[stage * kBwdThreads + s];
            const int32_t g = s_id[stage * kBwdThreads + s];
            const S q = chain_var ? s_q[stage * kBwdThreads + s] : S(0);
            const S om = r.o * r.mu;
            S g_x = 0, g_y = 0, g_a = 0, g_b = 0, g_c = 0, g_o = 0, g_mu = 0, g_beta = 0, g_q = 0, g_ax = 0,
              g_ay = 0;
#pragma unroll
            for (int k = 0; k < PPL; ++k) {
                if (!kBeta) {
                    const S dx = px[k] - r.x;
                    const S dy = py[k] - r.y;
                    const S sigma = static_cast<S>(0.5) * (r.a * dx * dx + r.c * dy * dy) + r.b * dx * dy;
                    const S vis_raw = exp(-sigma);
                    const S alpha_raw = om * vis_raw;
                    const bool keep = valid[k] && !(sigma < static_cast<S>(0) || fabs(alpha_raw) < static_cast<S>(1e-5));
                    const S vis = keep ? vis_raw : S(0);
                    const S alpha = keep ? alpha_raw : S(0);
                    S v = vr[k];
                    if (kVar) {
                        g_q += vv[k] * alpha * alpha;
                        v += static_cast<S>(2) * q * alpha * vv[k];
                    }
                    const S v_sigma = -v * alpha;
                    const S gx = -v_sigma * (r.a * dx + r.b * dy);
                    const S gy = -v_sigma * (r.c * dy + r.b * dx);
                    g_x += gx;
                    g_y += gy;
                    if (kAbs) {
                        g_ax += fabs(gx);
                        g_ay += fabs(gy);
                    }
                    g_a += v_sigma * static_cast<S>(0.5) * dx * dx;
                    g_b += v_sigma * dx * dy;
                    g_c += v_sigma * static_cast<S>(0.5) * dy * dy;
                    g_o += v * r.mu * vis;
                    g_mu += v * r.o * vis;
                } else {
                    const S dx = r.x - px[k];
                    const S dy = r.y - py[k];
                    const S d2 = r.a * dx * dx + static_cast<S>(2) * r.b * dx * dy + r.c * dy * dy;
                    const S h_raw = static_cast<S>(1) - d2;
                    const bool inside = valid[k] && !(d2 < static_cast<S>(0) || h_raw <= static_cast<S>(0));
                    const S h = inside ? h_raw : S(1);  // keeps pow/log finite on skipped samples
                    const S vis_raw = pow(h, r.beta);
                    const S alpha_raw = om * vis_raw;
                    const bool keep = inside && !(fabs(alpha_raw) < static_cast<S>(1e-5));
                    const S vis = keep ? vis_raw : S(0);
                    const S alpha = keep ? alpha_raw : S(0);
                    S v = keep ? vr[k] : S(0);
                    if (kVar) {
                        g_q += vv[k] * alpha * alpha;
                        v += static_cast<S>(2) * q * alpha * vv[k];
                    }
                    const S v_d2 = -om * r.beta * pow(h, r.beta - static_cast<S>(1)) * v;
                    const S gx = static_cast<S>(2) * v_d2 * (r.a * dx + r.b * dy);
                    const S gy = static_cast<S>(2) * v_d2 * (r.b * dx + r.c * dy);
                    g_x += gx;
                    g_y += gy;
                    if (kAbs) {
                        g_ax += fabs(gx);
                        g_ay += fabs(gy);
                    }
                    g_a += v_d2 * dx * dx;
                    g_b += static_cast<S>(2) * v_d2 * dx * dy;
                    g_c += v_d2 * dy * dy;
                    g_o += v * r.mu * vis;
                    g_mu += v * r.o * vis;
                    g_beta += v * alpha * log(h);
                }
            }
            g_x = warp_sum(g_x);
            g_y = warp_sum(g_y);
            g_a = warp_sum(g_a);
            g_b = warp_sum(g_b);
            g_c = warp_sum(g_c);
            g_o = warp_sum(g_o);
            g_mu = warp_sum(g_mu);
            if (kBeta) g_beta = warp_sum(g_beta);
            if (kVar) g_q = warp_sum(g_q);
            if (kAbs) {
                g_ax = warp_sum(g_ax);
                g_ay = warp_sum(g_ay);
            }
            if (grads != nullptr) {
                S* dst = reinterpret_cast<S*>(grads + g);
                if (lane == 0) red_add_v4(dst, g_x, g_y, g_a, g_b);
                if (lane == 1) red_add_v4(dst + 4, g_c, g_o, g_mu, g_beta);
            }
            if (kVar && lane == 2 && v_unc != nullptr) red_add(v_unc + (uint32_t(g) % N), g_q);
            if (kAbs && lane == 3) {
                red_add(v_abs + 2 * size_t(g), g_ax);
                red_add(v_abs + 2 * size_t(g) + 1, g_ay);
            }
        }
        __syncthreads();
    }
}

// --------------------------------------------------------------------------
// Packing for the low-level (separate-tensor) entry points
// --------------------------------------------------------------------------

template <typename S>
__global__ void pack_records_kernel(const S* __restrict__ means2d, const S* __restrict__ conics,
                                    const S* __restrict__ opacities, const S* __restrict__ mus,
                                    const S* __restrict__ betas, size_t total, Rec2D<S>* __restrict__ out) {
    const size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= total) return;
    Rec2D<S> r;
    r.x = means2d[2 * i];
    r.y = means2d[2 * i + 1];
    r.a = conics[3 * i];
    r.b = conics[3 * i + 1];
    r.c = conics[3 * i + 2];
    r.o = opacities[i];
    r.mu = mus[i];
    r.beta = betas != nullptr ? betas[i] : S(0);
    out[i] = r;
}

template <typename S>
__global__ void unpack_grads_kernel(const Rec2D<S>* __restrict__ grads, size_t total, S* __restrict__ v_means2d,
                                    S* __restrict__ v_conics, S* __restrict__ v_opacities, S* __restrict__ v_mus,
                                    S* __restrict__ v_betas) {
    const size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= total) return;
    const Rec2D<S> g = grads[i];
    v_means2d[2 * i] = g.x;
    v_means2d[2 * i + 1] = g.y;
    v_conics[3 * i] = g.a;
    v_conics[3 * i + 1] = g.b;
    v_conics[3 * i + 2] = g.c;
    v_opacities[i] = g.o;
    v_mus[i] = g.mu;
    if (v_betas != nullptr) v_betas[i] = g.beta;
}

// --------------------------------------------------------------------------
// Launchers
// --------------------------------------------------------------------------

struct RasterGeom {
    uint32_t C, N, n_isects, width, height, T, tiles_x, tiles_y;
};

inline int check_geom(const RasterGeom& g) {
    R2S_REQUIRE(g.T >= 1 && g.T <= 32, R2S_ERR_UNSUPPORTED, "tile_size must be in [1, 32]");
    R2S_REQUIRE(g.C <= 65535, R2S_ERR_UNSUPPORTED, "camera count exceeds 65535");
    R2S_REQUIRE(uint64_t(g.C) * g.N < (uint64_t(1) << 31), R2S_ERR_UNSUPPORTED, "C*N exceeds the int32 range");
    R2S_REQUIRE(uint64_t(g.tiles_x) * g.tiles_y < (uint64_t(1) << 31), R2S_ERR_UNSUPPORTED, "too many tiles");
    R2S_REQUIRE(g.N > 0, R2S_ERR_ARGUMENT, "N must be positive");
    return R2S_OK;
}

template <typename S, bool kBeta, bool kVar, int PPT>
int launch_fwd_t(const RasterGeom& g, const Rec2D<S>* rec, const S* unc, const int32_t* offsets,
                 const int32_t* ids, S* out, S* out_var, unsigned nthreads, cudaStream_t stream) {
    const size_t smem = 2 * nthreads * (sizeof(Rec2D<S>) + sizeof(S));
    dim3 grid(g.tiles_x * g.tiles_y, g.C);
    raster_fwd_kernel<S, kBeta, kVar, PPT><<<grid, nthreads, smem, stream>>>(
        rec, unc, g.N, offsets, ids, int32_t(g.n_isects), g.C, g.width, g.height, g.T, g.tiles_x,
        g.tiles_x * g.tiles_y, out, out_var);
    return check_launch("rasterize_to_pixels_fwd");
}

template <typename S, bool kBeta, bool kVar>
int launch_fwd_p(const RasterGeom& g, const Rec2D<S>* rec, const S* unc, const int32_t* offsets,
                 const int32_t* ids, S* out, S* out_var, cudaStream_t stream) {
    const uint32_t pixels = g.T * g.T;
    if (pixels <= 64) {
        const unsigned nt = (pixels + 31) / 32 * 32;
        return launch_fwd_t<S, kBeta, kVar, 1>(g, rec, unc, offsets, ids, out, out_var, nt, stream);
    }
    if (pixels <= 512) {
        const unsigned nt = ((pixels + 1) / 2 + 31) / 32 * 32;
        return launch_fwd_t<S, kBeta, kVar, 2>(g, rec, unc, offsets, ids, out, out_var, nt, stream);
    }
    const unsigned nt = ((pixels + 3) / 4 + 31) / 32 * 32;
    return launch_fwd_t<S, kBeta, kVar, 4>(g, rec, unc, offsets, ids, out, out_var, nt, stream);
}

template <typename S>
int launch_fwd(const RasterGeom& g, const Rec2D<S>* rec, const S* unc, bool beta, const int32_t* offsets,
               const int32_t* ids, S* out, S* out_var, cudaStream_t stream) {
    R2S_TRY(check_geom(g));
    if (g.tiles_x == 0 || g.tiles_y == 0 || g.C == 0) return R2S_OK;
    const bool var = out_var != nullptr;
    if (beta) {
        return var ? launch_fwd_p<S, true, true>(g, rec, unc, offsets, ids, out, out_var, stream)
                   : launch_fwd_p<S, true, false>(g, rec, unc, offsets, ids, out, out_var, stream);
    }
    return var ? launch_fwd_p<S, false, true>(g, rec, unc, offsets, ids, out, out_var, stream)
               : launch_fwd_p<S, false, false>(g, rec, unc, offsets, ids, out, out_var, stream);
}

template <typename S, bool kBeta, bool kVar, bool kAbs, int PPL>
int launch_bwd_t(const RasterGeom& g, const Rec2D<S>* rec, const S* var_q, const int32_t* offsets,
                 const int32_t* ids, const S* v_render, const S* v_render_var, Rec2D<S>* grads, S* v_abs,
                 S* v_unc, cudaStream_t stream) {
    const size_t smem = 2 * kBwdThreads * (sizeof(Rec2D<S>) + sizeof(S) + sizeof(int32_t));
    dim3 grid(g.tiles_x * g.tiles_y, g.C);
    raster_bwd_kernel<S, kBeta, kVar, kAbs, PPL><<<grid, kBwdThreads, smem, stream>>>(
        rec, var_q, g.N, offsets, ids, int32_t(g.n_isects), g.C, g.width, g.height, g.T, g.tiles_x,
        g.tiles_x * g.tiles_y, v_render, v_render_var, grads, v_abs, v_unc);
    return check_launch("rasterize_to_pixels_bwd");
}

template <typename S, bool kBeta, bool kVar, bool kAbs>
int launch_bwd_p(const RasterGeom& g, const Rec2D<S>* rec, const S* var_q, const int32_t* offsets,
                 const int32_t* ids, const S* v_render, const S* v_render_var, Rec2D<S>* grads, S* v_abs,
                 S* v_unc, cudaStream_t stream) {
    // Pixels per lane: 2 for tiles up to 8x8, else 8 (sub-tiles of 256 pixels).
    if (g.T * g.T <= 64)
        return launch_bwd_t<S, kBeta, kVar, kAbs, 2>(g, rec, var_q, offsets, ids, v_render, v_render_var, grads,
                                                     v_abs, v_unc, stream);
    return launch_bwd_t<S, kBeta, kVar, kAbs, 8>(g, rec, var_q, offsets, ids, v_render, v_render_var, grads,
                                                 v_abs, v_unc, stream);
}

template <typename S, bool kBeta>
int launch_bwd_b(const RasterGeom& g, const Rec2D<S>* rec, const S* var_q, const int32_t* offsets,
                 const int32_t* ids, const S* v_render, const S* v_render_var, Rec2D<S>* grads, S* v_abs,
                 S* v_unc, cudaStream_t stream) {
    const bool var = v_render_var != nullptr, abs = v_abs != nullptr;
    if (var && abs)
        return launch_bwd_p<S, kBeta, true, true>(g, rec, var_q, offsets, ids, v_render, v_render_var, grads, v_abs,
                                                  v_unc, stream);
    if (var)
        return launch_bwd_p<S, kBeta, true, false>(g, rec, var_q, offsets, ids, v_render, v_render_var, grads, v_abs,
                                                   v_unc, stream);
    if (abs)
        return launch_bwd_p<S, kBeta, false, true>(g, rec, var_q, offsets, ids, v_render, v_render_var, grads, v_abs,
                                                   v_unc, stream);
    return launch_bwd_p<S, kBeta, false, false>(g, rec, var_q, offsets, ids, v_render, v_render_var, grads, v_abs,
                                                v_unc, stream);
}

template <typename S>
int launch_bwd(const RasterGeom& g, const Rec2D<S>* rec, bool beta, const S* var_q, const int32_t* offsets,
               const int32_t* ids, const S* v_render, const S* v_render_var, Rec2D<S>* grads, S* v_abs, S* v_unc,
               cudaStream_t stream) {
    R2S_TRY(check_geom(g));
    if (g.n_isects == 0 || g.tiles_x == 0 || g.tiles_y == 0 || g.C == 0) return R2S_OK;
    return beta ? launch_bwd_b<S, true>(g, rec, var_q, offsets, ids, v_render, v_render_var, grads, v_abs, v_unc,
                                        stream)
                : launch_bwd_b<S, false>(g, rec, var_q, offsets, ids, v_render, v_render_var, grads, v_abs, v_unc,
                                         stream);
}

template <typename S>
size_t raster_ws(uint32_t C, uint32_t N, bool with_grads) {
    ArenaSize a;
    a.take<Rec2D<S>>(size_t(C) * N);
    if (with_grads) a.take<Rec2D<S>>(size_t(C) * N);
    return a.bytes();
}

}  // namespace r2s

using namespace r2s;

namespace {

template <typename S>
int pack(const void* means2d, const void* conics, const void* opacities, const void* mus, const void* betas,
         size_t total, Rec2D<S>* out, cudaStream_t stream) {
    if (total == 0) return R2S_OK;
    pack_records_kernel<S><<<blocks_for(int64_t(total), 256), 256, 0, stream>>>(
        static_cast<const S*>(means2d), static_cast<const S*>(conics), static_cast<const S*>(opacities),
        static_cast<const S*>(mus), static_cast<const S*>(betas), total, out);
    return check_launch("pack_records");
}

template <typename S>
int raster_fwd_lowlevel(const void* means2d, const void* conics, const void* opacities, const void* mus,
                        const void* betas, const void* unc, const int32_t* offsets, const int32_t* ids,
                        const RasterGeom& g, void* render, void* render_var, void* ws, size_t ws_bytes,
                        cudaStream_t stream) {
    const size_t pixels_total = size_t(g.C) * g.height * g.width;
    if (g.C == 0 || g.N == 0 || g.n_isects == 0) {
        if (pixels_total) {
            if (cudaMemsetAsync(render, 0, pixels_total * sizeof(S), stream) != cudaSuccess ||
                (render_var && cudaMemsetAsync(render_var, 0, pixels_total * sizeof(S), stream) != cudaSuccess))
                return fail(R2S_ERR_CUDA, "memset failed");
        }
        return R2S_OK;
    }
    Arena arena(ws, ws_bytes);
    Rec2D<S>* rec = arena.take<Rec2D<S>>(size_t(g.C) * g.N);
    R2S_REQUIRE(rec != nullptr, R2S_ERR_WORKSPACE, "raster workspace too small");
    R2S_TRY(pack<S>(means2d, conics, opacities, mus, betas, size_t(g.C) * g.N, rec, stream));
    return launch_fwd<S>(g, rec, static_cast<const S*>(unc), betas != nullptr, offsets, ids, static_cast<S*>(render),
                         static_cast<S*>(render_var), stream);
}

}  // namespace

extern "C" {

size_t r2s_raster_workspace(uint32_t dtype, uint32_t C, uint32_t N, int with_gradients) {
    return dtype == R2S_F64 ? raster_ws<double>(C, N, with_gradients != 0) : raster_ws<float>(C, N, with_gradients != 0);
}

int r2s_rasterize_to_pixels_fwd(int dtype, const void* means2d, const void* conics, const void* opacities,
                                const void* mus, const void* betas, const int32_t* tile_offsets,
                                const int32_t* flatten_ids, uint32_t C, uint32_t N, uint32_t n_isects,
                                uint32_t width, uint32_t height, uint32_t tile_size, uint32_t tiles_x,
                                uint32_t tiles_y, void* render, void* workspace, size_t workspace_bytes,
                                void* stream) {
    const RasterGeom g{C, N, n_isects, width, height, tile_size, tiles_x, tiles_y};
    R2S_DISPATCH(dtype, return raster_fwd_lowlevel<S>(means2d, conics, opacities, mus, betas, nullptr, tile_offsets,
                                                     flatten_ids, g, render, nullptr, workspace, workspace_bytes,
                                                     as_stream(stream)));
}

int r2s_rasterize_to_pixels_mean_var_fwd(int dtype, const void* means2d, const void* conics, const void* opacities,
                                         const void* mus, const void* betas, const void* uncertainties,
                                         const int32_t* tile_offsets, const int32_t* flatten_ids, uint32_t C,
                                         uint32_t N, uint32_t n_isects, uint32_t width, uint32_t height,
                                         uint32_t tile_size, uint32_t tiles_x, uint32_t tiles_y, void* render,
                                         void* render_var, void* workspace, size_t workspace_bytes, void* stream) {
    const RasterGeom g{C, N, n_isects, width, height, tile_size, tiles_x, tiles_y};
    R2S_REQUIRE(uncertainties != nullptr && render_var != nullptr, R2S_ERR_ARGUMENT,
                "mean/variance rasterization needs uncertainties and render_var");
    R2S_DISPATCH(dtype, return raster_fwd_lowlevel<S>(means2d, conics, opacities, mus, betas, uncertainties,
                                                     tile_offsets, flatten_ids, g, render, render_var, workspace,
                                                     workspace_bytes, as_stream(stream)));
}

int r2s_rasterize_to_pixels_bwd(int dtype, const void* means2d, const void* conics, const void* opacities,
                                const void* mus, const void* betas, const int32_t* tile_offsets,
                                const int64_t* isect_ids, const int32_t* flatten_ids, const void* v_render,
                                const void* v_render_var, const void* uncertainties, uint32_t C, uint32_t N,
                                uint32_t n_isects, uint32_t width, uint32_t height, uint32_t tile_size,
                                uint32_t tiles_x, uint32_t tiles_y, void* v_means2d_abs, void* v_means2d,
                                void* v_conics, void* v_opacities, void* v_mus, void* v_betas,
                                void* v_uncertainties, void* workspace, size_t workspace_bytes, void* stream) {
    (void)isect_ids;
    const RasterGeom g{C, N, n_isects, width, height, tile_size, tiles_x, tiles_y};
    R2S_REQUIRE((betas == nullptr) == (v_betas == nullptr), R2S_ERR_ARGUMENT, "v_betas goes with betas");
    R2S_REQUIRE(v_render_var == nullptr || v_uncertainties != nullptr, R2S_ERR_ARGUMENT,
                "variance adjoint needs v_uncertainties");
    R2S_DISPATCH(dtype, {
        const size_t total = size_t(C) * N;
        cudaStream_t st = as_stream(stream);
        if (v_means2d_abs && total && cudaMemsetAsync(v_means2d_abs, 0, total * 2 * sizeof(S), st) != cudaSuccess)
            return fail(R2S_ERR_CUDA, "memset failed");
        if (v_uncertainties && N && cudaMemsetAsync(v_uncertainties, 0, size_t(N) * sizeof(S), st) != cudaSuccess)
            return fail(R2S_ERR_CUDA, "memset failed");
        if (total == 0) return R2S_OK;
        Arena arena(workspace, workspace_bytes);
        Rec2D<S>* rec = arena.take<Rec2D<S>>(total);
        Rec2D<S>* grads = arena.take<Rec2D<S>>(total);
        R2S_REQUIRE(rec && grads, R2S_ERR_WORKSPACE, "raster workspace too small");
        if (cudaMemsetAsync(grads, 0, total * sizeof(Rec2D<S>), st) != cudaSuccess)
            return fail(R2S_ERR_CUDA, "memset failed");
        if (n_isects > 0) {
            R2S_TRY(pack<S>(means2d, conics, opacities, mus, betas, total, rec, st));
            R2S_TRY(launch_bwd<S>(g, rec, betas != nullptr, static_cast<const S*>(uncertainties), tile_offsets,
                                  flatten_ids, static_cast<const S*>(v_render), static_cast<const S*>(v_render_var),
                                  grads, static_cast<S*>(v_means2d_abs), static_cast<S*>(v_uncertainties), st));
        }
        unpack_grads_kernel<S><<<blocks_for(int64_t(total), 256), 256, 0, st>>>(
            grads, total, static_cast<S*>(v_means2d), static_cast<S*>(v_conics), static_cast<S*>(v_opacities),
            static_cast<S*>(v_mus), static_cast<S*>(v_betas));
        return check_launch("unpack_grads");
    });
}

int r2s_rasterize_to_pixels_uncertainty_bwd(int dtype, const void* means2d, const void* conics,
                                            const void* opacities, const void* mus, const void* betas,
                                            const int32_t* tile_offsets, const int32_t* flatten_ids,
                                            const void* v_render_var, uint32_t C, uint32_t N, uint32_t n_isects,
                                            uint32_t width, uint32_t height, uint32_t tile_size, uint32_t tiles_x,
                                            uint32_t tiles_y, void* v_uncertainties, void* workspace,
                                            size_t workspace_bytes, void* stream) {
    const RasterGeom g{C, N, n_isects, width, height, tile_size, tiles_x, tiles_y};
    R2S_DISPATCH(dtype, {
        cudaStream_t st = as_stream(stream);
        if (N && cudaMemsetAsync(v_uncertainties, 0, size_t(N) * sizeof(S), st) != cudaSuccess)
            return fail(R2S_ERR_CUDA, "memset failed");
        const size_t total = size_t(C) * N;
        if (total == 0 || n_isects == 0) return R2S_OK;
        Arena arena(workspace, workspace_bytes);
        Rec2D<S>* rec = arena.take<Rec2D<S>>(total);
        R2S_REQUIRE(rec, R2S_ERR_WORKSPACE, "raster workspace too small");
        R2S_TRY(pack<S>(means2d, conics, opacities, mus, betas, total, rec, st));
        return launch_bwd<S>(g, rec, betas != nullptr, nullptr, tile_offsets, flatten_ids, nullptr,
                             static_cast<const S*>(v_render_var), nullptr, nullptr, static_cast<S*>(v_uncertainties),
                             st);
    });
}

int r2s_raster_render(int dtype, const void* records, const void* uncertainties, int beta,
                      const int32_t* tile_offsets, const int32_t* flatten_ids, uint32_t C, uint32_t N,
                      uint32_t n_isects, uint32_t width, uint32_t height, uint32_t tile_size, uint32_t tiles_x,
                      uint32_t tiles_y, void* render, void* render_var, void* stream) {
    const RasterGeom g{C, N, n_isects, width, height, tile_size, tiles_x, tiles_y};
    R2S_DISPATCH(dtype, return launch_fwd<S>(g, static_cast<const Rec2D<S>*>(records),
                                             static_cast<const S*>(uncertainties), beta != 0, tile_offsets,
                                             flatten_ids, static_cast<S*>(render), static_cast<S*>(render_var),
                                             as_stream(stream)));
}

int r2s_raster_render_bwd(int dtype, const void* records, const void* uncertainties, int beta, int detach_variance,
                          const int32_t* tile_offsets, const int32_t* flatten_ids, const void* v_render,
                          const void* v_render_var, uint32_t C, uint32_t N, uint32_t n_isects, uint32_t width,
                          uint32_t height, uint32_t tile_size, uint32_t tiles_x, uint32_t tiles_y, void* grads,
                          void* v_means2d_abs, void* v_uncertainties, void* stream) {
    const RasterGeom g{C, N, n_isects, width, height, tile_size, tiles_x, tiles_y};
    R2S_DISPATCH(dtype, return launch_bwd<S>(g, static_cast<const Rec2D<S>*>(records), beta != 0,
                                             detach_variance ? nullptr : static_cast<const S*>(uncertainties),
                                             tile_offsets, flatten_ids, static_cast<const S*>(v_render),
                                             static_cast<const S*>(v_render_var), static_cast<Rec2D<S>*>(grads),
                                             static_cast<S*>(v_means2d_abs), static_cast<S*>(v_uncertainties),
                                             as_stream(stream)));
}

}  // extern "C"
