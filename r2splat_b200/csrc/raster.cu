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
//  * each staged record gets a conservative pixel box on this tile (the
//    pixels where its sample can pass the contribution test), computed once
//    per CTA by the thread that staged it;
//  * forward: one pixel per thread, each warp owning an 8x4 block of the
//    tile; a warp ballots which staged records' boxes meet its block and
//    evaluates only those, in list order, so every pixel still sums its
//    contributions in the reference's order;
//  * backward: one warp per record, evaluating only the pixels of its box
//    (about a third of the tile for CT-sized Gaussians), accumulating six to
//    eight partial sums per lane, reducing them with a recursive-halving warp
//    sum and adding them to the packed adjoints with vector atomics.
//
// Per-sample arithmetic keeps the reference's expression forms
// (RasterizeToPixelsFwd.cu:160-177, :664-680; RasterizeToPixelsBwd.cu:417-468,
// :910-945): the contribution thresholds (|alpha| < 1e-5, sigma < 0, d2 >= 1)
// decide which samples count, so alpha must round exactly as the reference's
// does. Each thread evaluates one pixel per record, as in the reference's
// one-pixel-per-thread loops, so the compiler contracts the same multiply-adds.
#include <type_traits>

#include "common.cuh"

namespace r2s {

template <typename S>
__device__ __forceinline__ void gather_record(Rec2D<S>* dst, const Rec2D<S>* src) {
    const char* s = reinterpret_cast<const char*>(src);
    char* d = reinterpret_cast<char*>(dst);
#pragma unroll
    for (int k = 0; k < int(sizeof(Rec2D<S>) / 16); ++k) cp_async16(d + 16 * k, s + 16 * k);
}

// --------------------------------------------------------------------------
// Pixel boxes
// --------------------------------------------------------------------------

// A record's box on one tile, in tile-local pixel indices: column and row bit
// masks, the packed origin and extent (x0 | y0 << 8 | width << 16 |
// height << 24) and ceil(65536 / width), with which (k * magic) >> 16 equals
// k / width for every k < 1024 and width <= 32. An empty box has zero masks
// and extent.
struct alignas(16) TileBox {
    uint32_t cols, rows, packed, magic;
};

__device__ __forceinline__ uint32_t low_bits(uint32_t n) { return n >= 32u ? 0xffffffffu : ((1u << n) - 1u); }

// Clips the inclusive pixel range [x0, x1] x [y0, y1] (indices relative to
// (ox, oy)) to a conservative box of the pixels whose sample can pass the
// contribution test; returns false when no pixel of the range can pass.
//
// Gaussian: a sample counts only if |o mu| exp(-sigma) >= 1e-5, i.e. sigma <=
// s = ln(|o mu| 1e5), with sigma = d^T Q d / 2 and Q = [[a, b], [b, c]]. When Q
// is positive definite with condition number <= (a + c)^2 / det <= 1000, the
// rounded sigma the sample computes is within 8 * 2^-24 * 1000 < 5e-4 of sigma
// relative (each rounding error is relative to |terms| <= cond * sigma), and
// the fast exponential and logarithm add < 1e-5 absolute; so every passing
// pixel lies in the ellipse sigma <= s' = s + 1e-3 |s| + 1e-3, whose bounding
// box has half-widths sqrt(2 s' c / det) and sqrt(2 s' a / det). Those are
// widened by 0.1 % plus 0.01 pixel, and by 1e-6 of the coordinates' magnitude
// for the rounding of the box arithmetic itself.
// Beta: a sample needs d2 = d^T Q d < 1; by the same argument every passing
// pixel has d2 < 1.001.
// Anything outside those conditions (a conic that is not positive definite or
// badly conditioned, non-finite values) falls back to the whole tile, so the
// box never drops a sample the reference would count.
template <typename S, bool kBeta>
__device__ __forceinline__ bool clip_to_record(const Rec2D<S>& r, uint32_t ox, uint32_t oy, uint32_t& x0,
                                               uint32_t& x1, uint32_t& y0, uint32_t& y1) {
    const S a = r.a, b = r.b, c = r.c;
    const S det = a * c - b * b;
    const S tr = a + c;
    bool bounded = a > S(0) && c > S(0) && det > S(0) && tr * tr <= S(1000) * det;
    S reach = S(1.001);
    if (!kBeta) {
        S s = log(fabs(r.o * r.mu)) + S(11.512925464970229);  // ln(1e5)
        s = s + S(1e-3) * fabs(s) + S(1e-3);
        if (bounded && isfinite(s) && s < S(0)) return false;
        bounded = bounded && isfinite(s);
        reach = S(2) * s;
    }
    if (!bounded) return true;
    const S hx = sqrt(reach * c / det) * S(1.001) + S(0.01);
    const S hy = sqrt(reach * a / det) * S(1.001) + S(0.01);
    // Pixel j (centre j + 0.5) can pass only if |j + 0.5 - x| <= hx.
    const S cx = r.x - S(0.5) - static_cast<S>(ox);
    const S cy = r.y - S(0.5) - static_cast<S>(oy);
    const S mx = S(1e-6) * (fabs(r.x) + hx + static_cast<S>(ox));
    const S my = S(1e-6) * (fabs(r.y) + hy + static_cast<S>(oy));
    const S lo_x = ceil(cx - hx - mx), hi_x = floor(cx + hx + mx);
    const S lo_y = ceil(cy - hy - my), hi_y = floor(cy + hy + my);
    if (!(isfinite(lo_x) && isfinite(hi_x) && isfinite(lo_y) && isfinite(hi_y))) return true;
    if (hi_x < static_cast<S>(x0) || lo_x > static_cast<S>(x1) || hi_y < static_cast<S>(y0) ||
        lo_y > static_cast<S>(y1))
        return false;
    if (lo_x > static_cast<S>(x0)) x0 = static_cast<uint32_t>(lo_x);
    if (hi_x < static_cast<S>(x1)) x1 = static_cast<uint32_t>(hi_x);
    if (lo_y > static_cast<S>(y0)) y0 = static_cast<uint32_t>(lo_y);
    if (hi_y < static_cast<S>(y1)) y1 = static_cast<uint32_t>(hi_y);
    return x0 <= x1 && y0 <= y1;
}

// The record's box on the tile with origin (ox, oy) and valid extent vx x vy.
template <typename S, bool kBeta>
__device__ __forceinline__ TileBox record_box(const Rec2D<S>& r, uint32_t ox, uint32_t oy, uint32_t vx, uint32_t vy) {
    uint32_t x0 = 0, x1 = vx - 1, y0 = 0, y1 = vy - 1;
    if (!clip_to_record<S, kBeta>(r, ox, oy, x0, x1, y0, y1)) return TileBox{0u, 0u, 0u, 1u};
    const uint32_t bw = x1 - x0 + 1, bh = y1 - y0 + 1;
    TileBox box;
    box.cols = low_bits(bw) << x0;
    box.rows = low_bits(bh) << y0;
    box.packed = x0 | (y0 << 8) | (bw << 16) | (bh << 24);
    box.magic = (65536u + bw - 1u) / bw;
    return box;
}

// --------------------------------------------------------------------------
// Forward
// --------------------------------------------------------------------------

constexpr uint32_t kBlockW = 8;      // one warp's pixel block in the forward: 8 x 4
constexpr uint32_t kBlockH = 4;
constexpr uint32_t kFwdBatch = 256;  // records staged per batch (at most)

// Image-loss epilogue of the forward. With a target image, every pixel also
// writes the gradient of the mean image loss with respect to the rendered value
// and adds its loss term to its CTA's partial sum (fp64, fixed order):
//   mse: v = (img - tgt) * scale with scale = 2 / numel (as torch computes
//        `(img - tgt).mul_(2 / numel)`), term (img - tgt)^2;
//   l1:  v = lambda * sign(img - tgt) / numel, the reference's L1 gradient with
//        an upstream gradient of one (ImageLossBwd.cu:14-30), term |img - tgt|
//        (ImageLossFwd.cu:19-31).
template <typename S>
struct ImageLossEpilogue {
    const S* target = nullptr;   // [C, H, W]; null: no epilogue
    S* v_render = nullptr;       // [C, H, W]
    double* partials = nullptr;  // [C * n_tiles] per-tile loss sums
    S scale = S(0);              // mse: 2 / numel; l1: lambda
    S numel = S(1);              // l1: numel as S
    uint32_t l1 = 0u;
};

template <typename S, bool kBeta, bool kVar, int kMaxThreads>
__global__ void __launch_bounds__(kMaxThreads) raster_fwd_kernel(
    const Rec2D<S>* __restrict__ records, const S* __restrict__ uncertainties, uint32_t N,
    const int32_t* __restrict__ offsets, const int32_t* __restrict__ flatten_ids, int32_t n_isects,
    const int64_t* __restrict__ n_dev,
    uint32_t C, uint32_t width, uint32_t height, uint32_t T, uint32_t tiles_x, uint32_t n_tiles,
    S* __restrict__ render, S* __restrict__ render_var, uint32_t B, ImageLossEpilogue<S> loss) {
    extern __shared__ __align__(16) unsigned char smem[];  // B = records staged per batch (<= blockDim.x)
    Rec2D<S>* s_rec = reinterpret_cast<Rec2D<S>*>(smem);          // [3][B]
    S* s_q = reinterpret_cast<S*>(s_rec + 3 * B);                   // [3][B]
    uint2* s_mask = reinterpret_cast<uint2*>(s_q + 3 * B);          // [2][B] (column, row) masks
    uint16_t* s_hits = reinterpret_cast<uint16_t*>(s_mask + 2 * B); // [warps][32] hit lists

    const uint32_t tile = blockIdx.x, cam = blockIdx.y;
    const uint32_t key = cam * n_tiles + tile;
    const uint32_t ty = tile / tiles_x, tx = tile - ty * tiles_x;
    const uint32_t ox = tx * T, oy = ty * T;
    if (ox >= width || oy >= height) {
        if (loss.target != nullptr && threadIdx.x == 0) loss.partials[key] = 0.0;
        return;
    }
    const uint32_t vx = min(T, width - ox), vy = min(T, height - oy);
    const int32_t start = offsets[key];
    // n_dev: the intersection count kept on the device (capacity-bounded pipelines).
    const int32_t n_total = n_dev != nullptr ? int32_t(*n_dev) : n_isects;
    const int32_t end = (key + 1 == C * n_tiles) ? n_total : offsets[key + 1];
    const uint32_t t = threadIdx.x, lane = t & 31u, warp = t >> 5;

    const uint32_t blocks_x = (T + kBlockW - 1) / kBlockW;
    const uint32_t bx0 = (warp % blocks_x) * kBlockW, by0 = (warp / blocks_x) * kBlockH;
    const uint32_t lx = bx0 + (lane & 7u), ly = by0 + (lane >> 3);
    const bool inside = lx < vx && ly < vy;
    const uint32_t warp_cols = bx0 < 32u ? ((0xffu << bx0) & low_bits(vx)) : 0u;
    const uint32_t warp_rows = by0 < 32u ? ((0xfu << by0) & low_bits(vy)) : 0u;
    const bool warp_active = warp_cols != 0u && warp_rows != 0u;
    const S px = static_cast<S>(ox + lx) + static_cast<S>(0.5);
    const S py = static_cast<S>(oy + ly) + static_cast<S>(0.5);
    S acc = S(0), accv = S(0);

    const int32_t count = end - start;
    const int32_t n_batches = count > 0 ? (count + int32_t(B) - 1) / int32_t(B) : 0;
    auto load = [&](int32_t bi, uint32_t stage) {
        const int32_t idx = start + bi * int32_t(B) + int32_t(t);
        if (t < B && idx < end) {
            const int32_t g = flatten_ids[idx];
            gather_record(s_rec + stage * B + t, records + g);
            if (kVar) s_q[stage * B + t] = uncertainties[uint32_t(g) % N];
        }
        cp_async_commit();
    };
    if (n_batches > 0) load(0, 0);
    for (int32_t bi = 0; bi < n_batches; ++bi) {
        if (bi + 1 < n_batches) {
            load(bi + 1, uint32_t(bi + 1) % 3u);
            cp_async_wait<1>();
        } else {
            cp_async_wait<0>();
        }
        __syncthreads();
        const uint32_t stage = uint32_t(bi) % 3u;
        const Rec2D<S>* buf = s_rec + stage * B;
        const S* qbuf = s_q + stage * B;
        uint2* masks = s_mask + (uint32_t(bi) & 1u) * B;
        const int32_t batch = min(int32_t(B), count - bi * int32_t(B));
        if (int32_t(t) < batch) {
            Rec2D<S>& rec = s_rec[stage * B + t];
            const TileBox box = record_box<S, kBeta>(rec, ox, oy, vx, vy);
            masks[t] = make_uint2(box.cols, box.rows);
            rec.o = rec.o * rec.mu;  // o mu, once per record (the samples use only the product)
        }
        __syncthreads();
        if (warp_active) {
            for (int32_t base = 0; base < batch; base += 32) {
                bool hit = false;
                if (base + int32_t(lane) < batch) {
                    const uint2 m = masks[base + int32_t(lane)];
                    hit = (m.x & warp_cols) != 0u && (m.y & warp_rows) != 0u;
                }
                // The warp's hits, compacted in lane (= list) order.
                const uint32_t hits = __ballot_sync(0xffffffffu, hit);
                uint16_t* my_hits = s_hits + warp * 32u;
                if (hit) my_hits[__popc(hits & ((1u << lane) - 1u))] = uint16_t(base + int32_t(lane));
                __syncwarp();
                const int32_t n_hits = __popc(hits);
                for (int32_t e = 0; e < n_hits; ++e) {
                    const int32_t s = my_hits[e];
                    const Rec2D<S>& r = buf[s];
                    const S om = r.o;  // o mu
                    S q = S(0);
                    if (kVar) q = qbuf[s];
                    if (!kBeta) {
                        const S dx = px - r.x;
                        const S dy = py - r.y;
                        const S sigma = static_cast<S>(0.5) * (r.a * dx * dx + r.c * dy * dy) + r.b * dx * dy;
                        const S alpha = om * exp(-sigma);
                        if (!(sigma < static_cast<S>(0) || fabs(alpha) < static_cast<S>(1e-5))) {
                            acc += alpha;
                            if (kVar) accv += q * alpha * alpha;
                        }
                    } else {
                        const S dx = r.x - px;
                        const S dy = r.y - py;
                        const S d2 = r.a * dx * dx + static_cast<S>(2) * r.b * dx * dy + r.c * dy * dy;
                        if (!(d2 < static_cast<S>(0) || d2 >= static_cast<S>(1))) {
                            const S h = static_cast<S>(1) - d2;
                            const S alpha = om * pow(h, r.beta);
                            if (!(fabs(alpha) < static_cast<S>(1e-5))) {
                                acc += alpha;
                                if (kVar) accv += q * alpha * alpha;
                            }
                        }
                    }
                }
                __syncwarp();  // the list is rewritten for the next 32 records
            }
        }
        // No barrier here. The next iteration's load goes to the third record
        // buffer, which no warp can still be reading: its batch was evaluated
        // before the previous iteration's first barrier. The masks alternate
        // between two buffers.
    }
    const size_t pid = size_t(cam) * height * width + size_t(oy + ly) * width + (ox + lx);
    if (inside) {
        render[pid] = acc;
        if (kVar) render_var[pid] = accv;
    }
    if (loss.target != nullptr) {
        double term = 0.0;
        if (inside) {
            const S diff = acc - loss.target[pid];
            S v;
            if (loss.l1) {
                const S sgn = diff > S(0) ? S(1) : (diff < S(0) ? S(-1) : S(0));
                v = loss.scale * sgn / loss.numel;
                term = fabs(static_cast<double>(diff));
            } else {
                v = diff * loss.scale;
                term = static_cast<double>(diff) * static_cast<double>(diff);
            }
            loss.v_render[pid] = v;
        }
        // Fixed-order CTA sum: warp butterfly, then warp 0 over the warp sums.
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) term += __shfl_xor_sync(0xffffffffu, term, o);
        double* s_sum = reinterpret_cast<double*>(s_hits);  // hit lists are no longer read
        const uint32_t n_warps = blockDim.x >> 5;
        __syncthreads();
        if (lane == 0) s_sum[warp] = term;
        __syncthreads();
        if (warp == 0) {
            double w = lane < n_warps ? s_sum[lane] : 0.0;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) w += __shfl_xor_sync(0xffffffffu, w, o);
            if (lane == 0) loss.partials[key] = w;
        }
    }
}

// Forward in fp32 with two pixels per lane: lane (x, y) of a warp's 8x8 pixel
// block owns pixels (x, y) and (x, y + 4), which share dx, so the record's
// dx terms are computed once and the two samples go through packed FP32x2
// operations. The reference's expressions are written with the contraction
// nvcc applies to its source in this kernel, so each packed component rounds
// as that scalar operation does and the images stay bit-exact:
//   Gaussian: sigma = fma(b dx, dy, 1/2 fma(a dx, dx, (c dy) dy));
//   Beta:     d^2 = fma(c dy, dy, fma(a dx, dx, ((2 b) dx) dy)), with dx and dy
//             taken mean - pixel as the reference does;
//   variance: accv = fma(q alpha, alpha, accv).
// Staging, culling, list order and the image-loss epilogue are those of
// raster_fwd_kernel.
template <bool kBeta, bool kVar, int kMaxThreads>
__global__ void __launch_bounds__(kMaxThreads) raster_fwd_pair_kernel(
    const Rec2D<float>* __restrict__ records, const float* __restrict__ uncertainties, uint32_t N,
    const int32_t* __restrict__ offsets, const int32_t* __restrict__ flatten_ids, int32_t n_isects,
    const int64_t* __restrict__ n_dev, uint32_t C, uint32_t width, uint32_t height, uint32_t T, uint32_t tiles_x,
    uint32_t n_tiles, float* __restrict__ render, float* __restrict__ render_var, uint32_t B,
    ImageLossEpilogue<float> loss) {
    extern __shared__ __align__(16) unsigned char smem[];
    Rec2D<float>* s_rec = reinterpret_cast<Rec2D<float>*>(smem);   // [3][B]
    float* s_q = reinterpret_cast<float*>(s_rec + 3 * B);           // [3][B] uncertainties (variance only)
    uint2* s_mask = reinterpret_cast<uint2*>(s_q + (kVar ? 3 * B : 0u));  // [2][B] (column, row) masks
    uint16_t* s_hits = reinterpret_cast<uint16_t*>(s_mask + 2 * B); // [warps][32] hit lists

    const uint32_t tile = blockIdx.x, cam = blockIdx.y;
    const uint32_t key = cam * n_tiles + tile;
    const uint32_t ty = tile / tiles_x, tx = tile - ty * tiles_x;
    const uint32_t ox = tx * T, oy = ty * T;
    if (ox >= width || oy >= height) {
        if (loss.target != nullptr && threadIdx.x == 0) loss.partials[key] = 0.0;
        return;
    }
    const uint32_t vx = min(T, width - ox), vy = min(T, height - oy);
    const int32_t start = offsets[key];
    const int32_t n_total = n_dev != nullptr ? int32_t(*n_dev) : n_isects;
    const int32_t end = (key + 1 == C * n_tiles) ? n_total : offsets[key + 1];
    const uint32_t t = threadIdx.x, lane = t & 31u, warp = t >> 5, nthreads = blockDim.x;

    const uint32_t blocks_x = (T + 7u) / 8u;
    const uint32_t bx0 = (warp % blocks_x) * 8u, by0 = (warp / blocks_x) * 8u;
    const uint32_t lx = bx0 + (lane & 7u), ly = by0 + (lane >> 3);
    const bool inside0 = lx < vx && ly < vy, inside1 = lx < vx && ly + 4u < vy;
    const uint32_t warp_cols = bx0 < 32u ? ((0xffu << bx0) & low_bits(vx)) : 0u;
    const uint32_t warp_rows = by0 < 32u ? ((0xffu << by0) & low_bits(vy)) : 0u;
    const bool warp_active = warp_cols != 0u && warp_rows != 0u;
    const float px = static_cast<float>(ox + lx) + 0.5f;
    const float2 py = make_float2(static_cast<float>(oy + ly) + 0.5f, static_cast<float>(oy + ly + 4u) + 0.5f);
    float acc0 = 0.f, acc1 = 0.f, accv0 = 0.f, accv1 = 0.f;

    const int32_t count = end - start;
    const int32_t n_batches = count > 0 ? (count + int32_t(B) - 1) / int32_t(B) : 0;
    auto load = [&](int32_t bi, uint32_t stage) {
        for (uint32_t i = t; i < B; i += nthreads) {
            const int32_t idx = start + bi * int32_t(B) + int32_t(i);
            if (idx < end) {
                const int32_t g = flatten_ids[idx];
                gather_record(s_rec + stage * B + i, records + g);
                if (kVar) s_q[stage * B + i] = uncertainties[uint32_t(g) % N];
            }
        }
        cp_async_commit();
    };
    if (n_batches > 0) load(0, 0);
    for (int32_t bi = 0; bi < n_batches; ++bi) {
        if (bi + 1 < n_batches) {
            load(bi + 1, uint32_t(bi + 1) % 3u);
            cp_async_wait<1>();
        } else {
            cp_async_wait<0>();
        }
        __syncthreads();
        const uint32_t stage = uint32_t(bi) % 3u;
        const Rec2D<float>* buf = s_rec + stage * B;
        const float* qbuf = s_q + stage * B;
        uint2* masks = s_mask + (uint32_t(bi) & 1u) * B;
        const int32_t batch = min(int32_t(B), count - bi * int32_t(B));
        for (int32_t i = int32_t(t); i < batch; i += int32_t(nthreads)) {
            Rec2D<float>& rec = s_rec[stage * B + uint32_t(i)];
            const TileBox box = record_box<float, kBeta>(rec, ox, oy, vx, vy);
            masks[i] = make_uint2(box.cols, box.rows);
            rec.o = rec.o * rec.mu;  // o mu, once per record
        }
        __syncthreads();
        if (warp_active) {
            for (int32_t base = 0; base < batch; base += 32) {
                bool hit = false;
                if (base + int32_t(lane) < batch) {
                    const uint2 m = masks[base + int32_t(lane)];
                    hit = (m.x & warp_cols) != 0u && (m.y & warp_rows) != 0u;
                }
                const uint32_t hits = __ballot_sync(0xffffffffu, hit);
                uint16_t* my_hits = s_hits + warp * 32u;
                if (hit) my_hits[__popc(hits & ((1u << lane) - 1u))] = uint16_t(base + int32_t(lane));
                __syncwarp();
                const int32_t n_hits = __popc(hits);
                // Four records per loop trip: their sample math overlaps, while each pixel
                // still adds them in list order (4.80 -> 4.33 ms at the CT workload).
#pragma unroll 4
                for (int32_t e = 0; e < n_hits; ++e) {
                    const int32_t s = my_hits[e];
                    const Rec2D<float>& r = buf[s];
                    float alpha0, alpha1;
                    bool k0, k1;
                    if (!kBeta) {
                        const float dx = px - r.x;
                        const float adx = __fmul_rn(r.a, dx), bdx = __fmul_rn(r.b, dx);
                        const float2 dy = add2(py, splat2(-r.y));
                        const float2 in = fma2(splat2(adx), splat2(dx), mul2(mul2(splat2(r.c), dy), dy));
                        const float2 sigma = fma2(splat2(bdx), dy, mul2(splat2(0.5f), in));
                        alpha0 = r.o * exp(-sigma.x);
                        alpha1 = r.o * exp(-sigma.y);
                        k0 = !(sigma.x < 0.f || fabs(alpha0) < 1e-5f);
                        k1 = !(sigma.y < 0.f || fabs(alpha1) < 1e-5f);
                    } else {
                        const float dx = r.x - px;
                        const float adx = __fmul_rn(r.a, dx), b2dx = __fmul_rn(__fmul_rn(2.f, r.b), dx);
                        const float2 dy = add2(splat2(r.y), make_float2(-py.x, -py.y));
                        const float2 d2 = fma2(mul2(splat2(r.c), dy), dy,
                                               fma2(splat2(adx), splat2(dx), mul2(splat2(b2dx), dy)));
                        const bool s0 = !(d2.x < 0.f || d2.x >= 1.f), s1 = !(d2.y < 0.f || d2.y >= 1.f);
                        const float2 h = add2(splat2(1.f), make_float2(-d2.x, -d2.y));
                        alpha0 = s0 ? r.o * pow(h.x, r.beta) : 0.f;
                        alpha1 = s1 ? r.o * pow(h.y, r.beta) : 0.f;
                        k0 = s0 && !(fabs(alpha0) < 1e-5f);
                        k1 = s1 && !(fabs(alpha1) < 1e-5f);
                    }
                    if (k0) {
                        acc0 += alpha0;
                        if (kVar) accv0 = __fmaf_rn(__fmul_rn(qbuf[s], alpha0), alpha0, accv0);
                    }
                    if (k1) {
                        acc1 += alpha1;
                        if (kVar) accv1 = __fmaf_rn(__fmul_rn(qbuf[s], alpha1), alpha1, accv1);
                    }
                }
                __syncwarp();  // the list is rewritten for the next 32 records
            }
        }
        // No barrier here (see raster_fwd_kernel): three record buffers, two mask buffers.
    }
    const size_t pid0 = size_t(cam) * height * width + size_t(oy + ly) * width + (ox + lx);
    const size_t pid1 = pid0 + 4u * size_t(width);
    if (inside0) {
        render[pid0] = acc0;
        if (kVar) render_var[pid0] = accv0;
    }
    if (inside1) {
        render[pid1] = acc1;
        if (kVar) render_var[pid1] = accv1;
    }
    if (loss.target != nullptr) {
        double term = 0.0;
        const float accs[2] = {acc0, acc1};
        const size_t pids[2] = {pid0, pid1};
        const bool ins[2] = {inside0, inside1};
#pragma unroll
        for (int k = 0; k < 2; ++k) {
            if (!ins[k]) continue;
            const float diff = accs[k] - loss.target[pids[k]];
            float v;
            if (loss.l1) {
                const float sgn = diff > 0.f ? 1.f : (diff < 0.f ? -1.f : 0.f);
                v = loss.scale * sgn / loss.numel;
                term += fabs(static_cast<double>(diff));
            } else {
                v = diff * loss.scale;
                term += static_cast<double>(diff) * static_cast<double>(diff);
            }
            loss.v_render[pids[k]] = v;
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) term += __shfl_xor_sync(0xffffffffu, term, o);
        double* s_sum = reinterpret_cast<double*>(s_hits);  // hit lists are no longer read
        const uint32_t n_warps = blockDim.x >> 5;
        __syncthreads();
        if (lane == 0) s_sum[warp] = term;
        __syncthreads();
        if (warp == 0) {
            double w = lane < n_warps ? s_sum[lane] : 0.0;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) w += __shfl_xor_sync(0xffffffffu, w, o);
            if (lane == 0) loss.partials[key] = w;
        }
    }
}

// --------------------------------------------------------------------------
// Backward
// --------------------------------------------------------------------------

// One VJP sample: the record's contribution at pixel centre (px, py) with image
// adjoint v and variance adjoint vv, accumulated into the lane's partial sums
// (see raster_bwd_kernel for their meaning). Branch-free: a skipped sample has
// its alpha and visibility selected to zero.
template <typename S, bool kBeta, bool kVar, bool kAbs>
__device__ __forceinline__ void vjp_sample(const Rec2D<S>& r, S om, S q, S px, S py, S v, S vv, bool valid,
                                           S (&part)[8], S& g_ax, S& g_ay) {
    if (!kBeta) {
        const S dx = px - r.x;
        const S dy = py - r.y;
        const S sigma = static_cast<S>(0.5) * (r.a * dx * dx + r.c * dy * dy) + r.b * dx * dy;
        const S vis_raw = exp(-sigma);
        const S alpha_raw = om * vis_raw;
        const bool keep = valid && !(sigma < static_cast<S>(0) || fabs(alpha_raw) < static_cast<S>(1e-5));
        const S vis = keep ? vis_raw : S(0);
        const S alpha = keep ? alpha_raw : S(0);
        if (kVar) {
            part[7] += vv * alpha * alpha;
            v += static_cast<S>(2) * q * alpha * vv;
        }
        const S w = -v * alpha;
        const S wx = w * dx, wy = w * dy;
        part[0] += wx;
        part[1] += wy;
        part[2] += wx * dx;
        part[3] += wx * dy;
        part[4] += wy * dy;
        part[5] += v * vis;
        if (kAbs) {
            g_ax += fabs(r.a * wx + r.b * wy);
            g_ay += fabs(r.c * wy + r.b * wx);
        }
    } else {
        const S dx = r.x - px;
        const S dy = r.y - py;
        const S d2 = r.a * dx * dx + static_cast<S>(2) * r.b * dx * dy + r.c * dy * dy;
        const S h_raw = static_cast<S>(1) - d2;
        const bool in_support = valid && !(d2 < static_cast<S>(0) || h_raw <= static_cast<S>(0));
        const S h = in_support ? h_raw : S(1);  // keeps the logarithm finite on skipped samples
        // h^beta = 2^(beta log2 h) for h in (0, 1]; log2 h also gives ln h and, with one
        // division, h^(beta - 1) = h^beta / h: three special-function operations a sample
        // instead of the five of pow(h, beta), pow(h, beta - 1) and log(h).
        const S lg = log2(h);
        const S vis_raw = exp2(r.beta * lg);
        const S alpha_raw = om * vis_raw;
        const bool keep = in_support && !(fabs(alpha_raw) < static_cast<S>(1e-5));
        const S vis = keep ? vis_raw : S(0);
        const S alpha = keep ? alpha_raw : S(0);
        v = keep ? v : S(0);
        if (kVar) {
            part[7] += vv * alpha * alpha;
            v += static_cast<S>(2) * q * alpha * vv;
        }
        const S w = -om * r.beta * (vis_raw / h) * v;
        const S wx = w * dx, wy = w * dy;
        part[0] += wx;
        part[1] += wy;
        part[2] += wx * dx;
        part[3] += wx * dy;
        part[4] += wy * dy;
        part[5] += v * vis;
        part[6] += v * alpha * (lg * static_cast<S>(0.6931471805599453));  // ln h = ln 2 log2 h
        if (kAbs) {
            g_ax += fabs(static_cast<S>(2) * (r.a * wx + r.b * wy));
            g_ay += fabs(static_cast<S>(2) * (r.b * wx + r.c * wy));
        }
    }
}

// The record-slot adjoints held by lane subgroup grp (lane / 8 in a whole warp,
// (lane / 4) % 4 in a half warp) after warp_sum8_pairs reduced the partial sums to (lo, hi): group 0 gives
// (x, y), group 1 (a, b), group 2 (c, o) and mu (in e2), group 3 beta (in e0).
template <typename S, bool kBeta>
__device__ __forceinline__ void record_adjoints(const Rec2D<S>& r, uint32_t grp, S lo, S hi, S& e0, S& e1, S& e2) {
    e2 = S(0);
    if (grp == 0u) {
        e0 = kBeta ? static_cast<S>(2) * (r.a * lo + r.b * hi) : -(r.a * lo + r.b * hi);
        e1 = kBeta ? static_cast<S>(2) * (r.b * lo + r.c * hi) : -(r.c * hi + r.b * lo);
    } else if (grp == 1u) {
        e0 = kBeta ? lo : static_cast<S>(0.5) * lo;
        e1 = kBeta ? static_cast<S>(2) * hi : hi;
    } else if (grp == 2u) {
        e0 = kBeta ? lo : static_cast<S>(0.5) * lo;
        e1 = r.mu * hi;
        e2 = r.o * hi;
    } else {
        e0 = kBeta ? lo : S(0);
        e1 = S(0);
    }
}

constexpr int kBwdWarps = 8;
constexpr int kBwdThreads = kBwdWarps * 32;

// Optional outputs are selected at run time by null pointers:
//   v_render null      -> zero image adjoint (uncertainty-only VJP)
//   v_render_var null  -> no variance branch
//   var_q null         -> detached variance branch (no 2 q alpha v_var term)
//   grads null         -> skip the record-slot adjoints
//   v_abs / v_unc null -> skip absgrad / uncertainty adjoints
//
// Per sample the lane accumulates, with g the image adjoint (plus the
// variance chain term) and w = -g alpha (Gaussian) or the d2 adjoint (Beta):
//   S0 = sum w dx, S1 = sum w dy, S2 = sum w dx^2, S3 = sum w dx dy,
//   S4 = sum w dy^2, S5 = sum g vis, S6 = sum g alpha log h (Beta),
//   S7 = sum v_var alpha^2 (variance),
// from which the record's adjoints follow once per record: for a Gaussian
// x = -(a S0 + b S1), y = -(c S1 + b S0), a = S2 / 2, b = S3, c = S4 / 2,
// o = mu S5, mu = o S5; for a Beta x = 2 (a S0 + b S1), y = 2 (b S0 + c S1),
// a = S2, b = 2 S3, c = S4, o = mu S5, mu = o S5, beta = S6. These are the
// reference's per-sample terms with the record's constants factored out.
// The body is branch-free: a skipped sample keeps its arithmetic but has its
// alpha and visibility selected to zero.
template <typename S, bool kBeta, bool kVar, bool kAbs>
__global__ void __launch_bounds__(kBwdThreads) raster_bwd_kernel(
    const Rec2D<S>* __restrict__ records, const S* __restrict__ var_q, uint32_t N,
    const int32_t* __restrict__ offsets, const int32_t* __restrict__ flatten_ids, int32_t n_isects,
    const int64_t* __restrict__ n_dev,
    uint32_t C, uint32_t width, uint32_t height, uint32_t T, uint32_t tiles_x, uint32_t n_tiles,
    const S* __restrict__ v_render, const S* __restrict__ v_render_var, Rec2D<S>* __restrict__ grads,
    S* __restrict__ v_abs, S* __restrict__ v_unc) {
    extern __shared__ __align__(16) unsigned char smem[];
    Rec2D<S>* s_rec = reinterpret_cast<Rec2D<S>*>(smem);             // [2][kBwdThreads]
    TileBox* s_box = reinterpret_cast<TileBox*>(s_rec + 2 * kBwdThreads);  // [kBwdThreads]
    S* s_q = reinterpret_cast<S*>(s_box + kBwdThreads);                // [2][kBwdThreads]
    S* s_v = s_q + 2 * kBwdThreads;                                    // [T*T] image adjoint
    S* s_vv = s_v + T * T;                                             // [T*T] variance adjoint
    int32_t* s_id = reinterpret_cast<int32_t*>(s_vv + T * T);          // [2][kBwdThreads]

    const uint32_t tile = blockIdx.x, cam = blockIdx.y;
    const uint32_t key = cam * n_tiles + tile;
    const uint32_t ty = tile / tiles_x, tx = tile - ty * tiles_x;
    const uint32_t ox = tx * T, oy = ty * T;
    if (ox >= width || oy >= height) return;
    const uint32_t vx = min(T, width - ox), vy = min(T, height - oy);
    const int32_t start = offsets[key];
    // n_dev: the intersection count kept on the device (capacity-bounded pipelines).
    const int32_t n_total = n_dev != nullptr ? int32_t(*n_dev) : n_isects;
    const int32_t end = (key + 1 == C * n_tiles) ? n_total : offsets[key + 1];
    const int32_t count = end - start;
    if (count <= 0) return;
    const uint32_t t = threadIdx.x, lane = t & 31u, warp = t >> 5;
    const bool chain_var = kVar && var_q != nullptr;

    const size_t cam_base = size_t(cam) * height * width;
    for (uint32_t p = t; p < T * T; p += kBwdThreads) {
        const uint32_t py_ = p / T, px_ = p - py_ * T;
        const bool ok = px_ < vx && py_ < vy;
        const size_t pid = cam_base + size_t(oy + py_) * width + (ox + px_);
        s_v[p] = (ok && v_render != nullptr) ? v_render[pid] : S(0);
        if (kVar) s_vv[p] = ok ? v_render_var[pid] : S(0);
    }

    const int32_t n_batches = (count + kBwdThreads - 1) / kBwdThreads;
    auto load = [&](int32_t bi, uint32_t stage) {
        const int32_t idx = start + bi * kBwdThreads + int32_t(t);
        if (idx < end) {
            const int32_t g = flatten_ids[idx];
            gather_record(s_rec + stage * kBwdThreads + t, records + g);
            s_id[stage * kBwdThreads + t] = g;
            if (chain_var) s_q[stage * kBwdThreads + t] = var_q[uint32_t(g) % N];
        }
        cp_async_commit();
    };
    load(0, 0);
    for (int32_t bi = 0; bi < n_batches; ++bi) {
        // Double-buffered: batch bi + 1 loads into the stage that batch bi - 1 used, which every warp
        // finished before the barrier that ended the previous iteration.
        if (bi + 1 < n_batches) {
            load(bi + 1, uint32_t(bi + 1) & 1u);
            cp_async_wait<1>();
        } else {
            cp_async_wait<0>();
        }
        __syncthreads();
        const uint32_t stage = uint32_t(bi) & 1u;
        const int32_t batch = min(int32_t(kBwdThreads), count - bi * kBwdThreads);
        if (int32_t(t) < batch) s_box[t] = record_box<S, kBeta>(s_rec[stage * kBwdThreads + t], ox, oy, vx, vy);
        __syncthreads();
        for (int32_t s = int32_t(warp); s < batch; s += kBwdWarps) {
            const TileBox box = s_box[s];
            const uint32_t bw = (box.packed >> 16) & 0xffu, bh = box.packed >> 24;
            const uint32_t area = bw * bh;
            if (area == 0u) continue;
            const uint32_t x0 = box.packed & 0xffu, y0 = (box.packed >> 8) & 0xffu;
            const Rec2D<S> r = s_rec[stage * kBwdThreads + s];
            const int32_t g = s_id[stage * kBwdThreads + s];
            const S q = chain_var ? s_q[stage * kBwdThreads + s] : S(0);
            const S om = r.o * r.mu;
            S part[8];
#pragma unroll
            for (int i = 0; i < 8; ++i) part[i] = S(0);
            S g_ax = S(0), g_ay = S(0);
            for (uint32_t k = lane; k < area; k += 32u) {
                const uint32_t row = (k * box.magic) >> 16;
                const uint32_t col = k - row * bw;
                const uint32_t lx = x0 + col, ly = y0 + row;
                const uint32_t p = ly * T + lx;
                const S px = static_cast<S>(ox + lx) + static_cast<S>(0.5);
                const S py = static_cast<S>(oy + ly) + static_cast<S>(0.5);
                const S vv = kVar ? s_vv[p] : S(0);
                vjp_sample<S, kBeta, kVar, kAbs>(r, om, q, px, py, s_v[p], vv, true, part, g_ax, g_ay);
            }
            S lo, hi;
            warp_sum8_pairs(part, lo, hi);
            const uint32_t grp = lane >> 3;
            if ((lane & 7u) == 0u) {
                if (grads != nullptr) {
                    S* dst = reinterpret_cast<S*>(grads + g);
                    S e0, e1, e2;
                    record_adjoints<S, kBeta>(r, grp, lo, hi, e0, e1, e2);
                    if (grp < 3u) red_add_v2(dst + 2 * grp, e0, e1);
                    if (grp == 2u) red_add(dst + 6, e2);
                    if (kBeta && grp == 3u) red_add(dst + 7, e0);
                }
                if (kVar && grp == 3u && v_unc != nullptr) red_add(v_unc + (uint32_t(g) % N), hi);
            }
            if (kAbs) {
                g_ax = warp_sum(g_ax);
                g_ay = warp_sum(g_ay);
                if (lane == 0u) {
                    red_add(v_abs + 2 * size_t(g), g_ax);
                    red_add(v_abs + 2 * size_t(g) + 1, g_ay);
                }
            }
        }
        __syncthreads();
    }
}

// --------------------------------------------------------------------------
// Record-parallel backward (explicit pipeline)
// --------------------------------------------------------------------------

constexpr int kRecBwdThreads = 256;

// The VJP needs no tile order: a record's adjoints are sums over the pixels it
// covers, which the reference evaluates exactly on the tiles of the record's
// tile rectangle. So one warp takes one (camera, primitive) record, walks the
// pixels of its tile rectangle that its conservative box keeps (row-major,
// 32 lanes per step, the lane position advanced incrementally), reads the
// pixel adjoints from the camera's adjoint image (L2-resident), and writes the
// record's adjoints once: no per-tile overhead, no atomics, every slot of
// grads written (zeros for records without pixels). rects [C,N] hold the
// tile rectangle (x0, y0, x1, y1), upper bounds exclusive, as the projection
// writes it.
// ceil(65536 / w) for w = 1..32: (k * magic) >> 16 == k / w for k < 1024.
__constant__ uint32_t c_div_magic[33] = {
    0u,     65536u, 32768u, 21846u, 16384u, 13108u, 10923u, 9363u, 8192u, 7282u, 6554u,
    5958u,  5462u,  5042u,  4682u,  4370u,  4096u,  3856u,  3641u, 3450u, 3277u, 3121u,
    2979u,  2850u,  2731u,  2622u,  2521u,  2428u,  2341u,  2260u, 2185u, 2115u, 2048u};

// -(log2 e): exp(-s) = 2^(-s log2 e).
constexpr float kNegLog2e = -1.4426950408889634f;

// The walk of one Gaussian record (no variance branch, no absgrad) by kLanes
// lanes (the warp, or a half or quarter of it) in packed FP32x2 form: lane
// l = lane % kLanes evaluates two samples per step, k and k + kLanes of the
// row-major box order (k = l + 2 kLanes it), so one FADD2/FMUL2/FFMA2 serves
// both. iters is uniform over the warp.
// Pixel centres are stepped exactly in float (integers + 0.5); the pixel's
// element offset py * width + px - (width + 1) / 2 is formed exactly in float
// as well and read out through the 2^23 bias (valid while width * height <
// 2^22). The exponent e = -sigma log2(e) is evaluated from prescaled conic
// coefficients as dx (a' dx + b' dy) + c' dy^2, so vis = 2^e. A sample counts
// when e <= 0 (sigma >= 0) and e >= e_min, e_min = log2(1e-5 / |o mu|)
// (|alpha| >= 1e-5): the reference's two decisions, taken on the exponent.
// With w = -g alpha = -(o mu) g vis, the walk sums g vis and its moments and
// scales them by -(o mu) once: part[0..4] are S0..S4 and part[5] = S5 of
// vjp_sample.
template <uint32_t kLanes = 32u>
__device__ __forceinline__ void record_walk_packed(const Rec2D<float>& r, float om, float e_min, const float* vimg,
                                                   uint32_t bx0, uint32_t by0, uint32_t bw, uint32_t barea,
                                                   uint32_t magic, uint32_t width, uint32_t iters, float (&part)[8]) {
    const uint32_t lane = threadIdx.x & (kLanes - 1u);
    // (k * magic) >> 16 == k / bw for k <= 64 (magic = ceil(2^16 / bw)).
    const uint32_t dq = (2u * kLanes * magic) >> 16, dr = 2u * kLanes - dq * bw;
    const uint32_t ra = (lane * magic) >> 16, rb = ((lane + kLanes) * magic) >> 16;
    const uint32_t ca = lane - ra * bw, cb = lane + kLanes - rb * bw;
    float2 px = make_float2(static_cast<float>(bx0 + ca) + 0.5f, static_cast<float>(bx0 + cb) + 0.5f);
    float2 py = make_float2(static_cast<float>(by0 + ra) + 0.5f, static_cast<float>(by0 + rb) + 0.5f);
    const float x_end = static_cast<float>(bx0 + bw);
    const float2 step_x = splat2(static_cast<float>(dr)), step_y = splat2(static_cast<float>(dq));
    const float2 neg_bw = splat2(-static_cast<float>(bw));
    const float2 fw = splat2(static_cast<float>(width));
    // 2^23 - (width + 1) / 2: exact in float for width < 2^22.
    const float2 bias = splat2(8388608.0f - 0.5f * static_cast<float>(width) - 0.5f);
    const uint64_t vbase = reinterpret_cast<uint64_t>(vimg) - uint64_t(0x4B000000u) * sizeof(float);
    const float2 nx = splat2(-r.x), ny = splat2(-r.y);
    const float2 qa = splat2(0.5f * r.a * kNegLog2e), qb = splat2(r.b * kNegLog2e);
    const float2 qc = splat2(0.5f * r.c * kNegLog2e);
    float2 acc0 = splat2(0.f), acc1 = acc0, acc2 = acc0, acc3 = acc0, acc4 = acc0, acc5 = acc0;
    uint32_t k = lane;
    // Two steps per loop trip: the second step's adjoint loads are issued with
    // the first's (1.8 % off the CT VJP; four steps gained nothing more).
#pragma unroll 2
    for (uint32_t it = 0; it < iters; ++it, k += 2u * kLanes) {
        const float2 offb = add2(fma2(py, fw, px), bias);
        const float* pa = reinterpret_cast<const float*>(vbase + uint64_t(__float_as_uint(offb.x)) * sizeof(float));
        const float* pb = reinterpret_cast<const float*>(vbase + uint64_t(__float_as_uint(offb.y)) * sizeof(float));
        const float ga = k < barea ? __ldg(pa) : 0.f;
        const float gb = k + kLanes < barea ? __ldg(pb) : 0.f;
        const float2 dx = add2(px, nx), dy = add2(py, ny);
        const float2 t = fma2(qa, dx, mul2(qb, dy));
        const float2 e = fma2(dx, t, mul2(mul2(qc, dy), dy));
        const float2 vis = make_float2(exp2f(e.x), exp2f(e.y));
        const bool ka = !(e.x > 0.f || e.x < e_min);
        const bool kb = !(e.y > 0.f || e.y < e_min);
        // Select after the product: a skipped sample may have vis = inf (e > 0).
        const float2 gvr = mul2(make_float2(ga, gb), vis);
        const float2 gv = make_float2(ka ? gvr.x : 0.f, kb ? gvr.y : 0.f);
        const float2 wx = mul2(gv, dx), wy = mul2(gv, dy);
        acc0 = add2(acc0, wx);
        acc1 = add2(acc1, wy);
        acc2 = fma2(wx, dx, acc2);
        acc3 = fma2(wx, dy, acc3);
        acc4 = fma2(wy, dy, acc4);
        acc5 = add2(acc5, gv);
        // Advance both samples by 64 box positions: dq rows and dr columns,
        // plus one wrap where the column passes the box's width.
        px = add2(px, step_x);
        py = add2(py, step_y);
        const float2 wrap = make_float2(gt_mask(px.x, x_end), gt_mask(px.y, x_end));
        px = fma2(wrap, neg_bw, px);
        py = add2(py, wrap);
    }
    const float nom = -om;
    part[0] = nom * (acc0.x + acc0.y);
    part[1] = nom * (acc1.x + acc1.y);
    part[2] = nom * (acc2.x + acc2.y);
    part[3] = nom * (acc3.x + acc3.y);
    part[4] = nom * (acc4.x + acc4.y);
    part[5] = acc5.x + acc5.y;
    part[6] = 0.f;
    part[7] = 0.f;
}

// The scalar walk of one record by kLanes lanes (a full warp, or one half of
// it): lane l = lane % kLanes starts at box position k = l (row-major, width
// bw) and steps by kLanes positions, i.e. dq rows and dr columns plus one wrap
// when the column overflows. iters is uniform over the warp; lanes past the
// box end evaluate nothing (valid = false) and load nothing. part and the
// absgrad sums are vjp_sample's.
template <typename S, bool kBeta, bool kVar, bool kAbs, uint32_t kLanes>
__device__ __forceinline__ void record_walk_scalar(const Rec2D<S>& r, S om, S q, const S* vimg, const S* vvar,
                                                   uint32_t bx0, uint32_t by0, uint32_t bw, uint32_t barea,
                                                   uint32_t iters, uint32_t width, S (&part)[8], S& g_ax, S& g_ay) {
    const uint32_t l = threadIdx.x & (kLanes - 1u);
    uint32_t dq = 0u, dr = kLanes, row = 0u, col = l;
    if (bw < kLanes) {
        const uint32_t m = c_div_magic[bw];
        dq = (kLanes * m) >> 16;
        dr = kLanes - dq * bw;
        row = (l * m) >> 16;
        col = l - row * bw;
    }
    uint32_t off = (by0 + row) * width + bx0 + col;
    const uint32_t step = dq * width + dr, wrap_step = width - bw;
    S px = static_cast<S>(bx0 + col) + static_cast<S>(0.5);
    S py = static_cast<S>(by0 + row) + static_cast<S>(0.5);
    const S x_end = static_cast<S>(bx0 + bw);  // a centre past the row is >= x0 + w + 0.5
    const S step_x = static_cast<S>(dr), step_y = static_cast<S>(dq), wrap_x = static_cast<S>(bw);
#pragma unroll
    for (int i = 0; i < 8; ++i) part[i] = S(0);
    uint32_t k = l;
    for (uint32_t it = 0; it < iters; ++it, k += kLanes) {
        const bool valid = k < barea;
        const S v = (valid && vimg != nullptr) ? vimg[off] : S(0);
        const S vv = (kVar && valid) ? vvar[off] : S(0);
        vjp_sample<S, kBeta, kVar, kAbs>(r, om, q, px, py, v, vv, valid, part, g_ax, g_ay);
        px += step_x;
        py += step_y;
        off += step;
        const bool wrap = px > x_end;
        px = wrap ? px - wrap_x : px;
        py = wrap ? py + static_cast<S>(1) : py;
        off = wrap ? off + wrap_step : off;
    }
}

// Boxes of at most kHalfWarpArea pixels are walked by half warps, two records
// at a time, and boxes of at most kQuarterWarpArea by quarter warps, four at a
// time (kPacked*: the same for the packed walk): a small box fills a narrow
// step about as well as a 32-lane one, and the group shares one pass of the
// per-record set-up and reduction. The warp's records are sorted by box size
// first, so a group's boxes take about the same number of steps.
constexpr uint32_t kHalfWarpArea = 1024u;
constexpr uint32_t kQuarterWarpArea = 256u;
constexpr uint32_t kPackedHalfWarpArea = 1024u;
constexpr uint32_t kPackedQuarterWarpArea = 256u;

// Writes the slot adjoints of record subgroup grp (0..3) from its pair of
// reduced sums (see record_adjoints) and the record's uncertainty adjoint
// (v_unc [C,N], one entry per record; summed over cameras in a fixed order by
// r2s_sum_over_cameras).
template <typename S, bool kBeta, bool kVar>
__device__ __forceinline__ void store_record_adjoints(const Rec2D<S>& r, uint32_t grp, S lo, S hi, Rec2D<S>* slot,
                                                      S* v_unc, size_t rid) {
    S* dst = reinterpret_cast<S*>(slot);
    S e0, e1, e2;
    record_adjoints<S, kBeta>(r, grp, lo, hi, e0, e1, e2);
    if (grp < 3u) {
        dst[2 * grp] = e0;
        dst[2 * grp + 1] = e1;
    }
    if (grp == 2u) dst[6] = e2;
    if (grp == 3u) dst[7] = e0;
    if (kVar && grp == 3u && v_unc != nullptr) v_unc[rid] = hi;
}

// A record's walk constants, set up by the lane that loaded the record and
// read by the whole warp from shared memory (broadcast loads).
template <typename S>
struct alignas(16) RecordStage {
    Rec2D<S> r;
    uint32_t x0, y0, w, area;
    uint32_t magic, cam;
    S q;
    float e_min;
};

// Ascending sort of one 32-bit key per lane across the warp (bitonic network,
// 15 compare-exchange stages through shuffles); keys must be distinct.
__device__ __forceinline__ uint32_t warp_sort_ascending(uint32_t key) {
    const uint32_t lane = threadIdx.x & 31u;
#pragma unroll
    for (uint32_t k = 2u; k <= 32u; k <<= 1) {
#pragma unroll
        for (uint32_t j = k >> 1; j > 0u; j >>= 1) {
            const uint32_t other = __shfl_xor_sync(0xffffffffu, key, j);
            const bool ascending = (lane & k) == 0u;
            const bool lower = (lane & j) == 0u;
            key = lower == ascending ? min(key, other) : max(key, other);
        }
    }
    return key;
}

// Walks the staged records at sorted positions [p, p_end) in groups of
// 32 / kLanes, one record per kLanes-lane group of the warp (a group without
// a record walks nothing and stores nothing), with the packed walk
// (kPackedWalk) or the scalar one, a group-wide reduction and the record's
// stores. Lane L of `sorted` holds the L-th smallest (area << 5 | record lane)
// of the warp's records, so a step's records have boxes of about one size.
// base is the warp's first record; var_q is null without the variance chain
// term.
template <typename S, bool kBeta, bool kVar, bool kAbs, uint32_t kLanes, bool kPackedWalk>
__device__ __forceinline__ void walk_record_groups(uint32_t sorted, uint32_t p, uint32_t p_end,
                                                   const RecordStage<S>* stage, size_t base, uint32_t N,
                                                   uint32_t width, uint32_t height, const S* v_render,
                                                   const S* v_render_var, const S* var_q, Rec2D<S>* grads,
                                                   S* v_abs, S* v_unc) {
    constexpr uint32_t kGroups = 32u / kLanes;
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t group = lane / kLanes;
    for (; p < p_end; p += kGroups) {
        const uint32_t j0 = __shfl_sync(0xffffffffu, sorted, p) & 31u;
        const uint32_t mine = __shfl_sync(0xffffffffu, sorted, min(p + group, 31u)) & 31u;
        const uint32_t jg = p + group < p_end ? mine : 32u;
        const bool active = jg < 32u;
        const uint32_t j = active ? jg : j0;
        const RecordStage<S> st = stage[j];
        const Rec2D<S>& r = st.r;
        const uint32_t barea = active ? st.area : 0u;
        constexpr uint32_t kPerStep = kPackedWalk ? 2u * kLanes : kLanes;
        uint32_t iters = (barea + kPerStep - 1u) / kPerStep;
#pragma unroll
        for (uint32_t offset = kLanes; offset < 32u; offset <<= 1)
            iters = max(iters, __shfl_xor_sync(0xffffffffu, iters, offset));
        const size_t rid = base + j;
        const uint32_t cam = st.cam;
        const uint32_t n = uint32_t(rid) - cam * N;
        const size_t cam_base = size_t(cam) * height * width;
        const S* vimg = v_render != nullptr ? v_render + cam_base : nullptr;
        const S* vvar = kVar ? v_render_var + cam_base : nullptr;
        const S q = var_q != nullptr ? st.q : S(0);
        const S om = r.o * r.mu;
        S part[8];
        S g_ax = S(0), g_ay = S(0);
        if constexpr (kPackedWalk)
            record_walk_packed<kLanes>(r, om, st.e_min, vimg, st.x0, st.y0, st.w, barea, st.magic, width, iters,
                                       part);
        else
            record_walk_scalar<S, kBeta, kVar, kAbs, kLanes>(r, om, q, vimg, vvar, st.x0, st.y0, st.w, barea,
                                                             iters, width, part, g_ax, g_ay);
        S lo, hi;
        warp_sum8_pairs<kLanes>(part, lo, hi);
        constexpr uint32_t kSub = kLanes / 4u;  // lanes per reduced pair
        if (active && (lane & (kSub - 1u)) == 0u)
            store_record_adjoints<S, kBeta, kVar>(r, (lane % kLanes) / kSub, lo, hi, grads + rid, v_unc, rid);
        if (kAbs) {
#pragma unroll
            for (uint32_t offset = kLanes / 2u; offset > 0u; offset >>= 1) {
                g_ax += __shfl_xor_sync(0xffffffffu, g_ax, offset);
                g_ay += __shfl_xor_sync(0xffffffffu, g_ay, offset);
            }
            if (active && (lane % kLanes) == 0u) {
                v_abs[2 * rid] = g_ax;
                v_abs[2 * rid + 1] = g_ay;
            }
        }
    }
}

template <typename S, bool kBeta, bool kVar, bool kAbs>
__global__ void __launch_bounds__(kRecBwdThreads) raster_record_bwd_kernel(
    const Rec2D<S>* __restrict__ records, const ushort4* __restrict__ rects, const S* __restrict__ var_q,
    uint32_t C, uint32_t N, uint32_t width, uint32_t height, uint32_t T, const S* __restrict__ v_render,
    const S* __restrict__ v_render_var, Rec2D<S>* __restrict__ grads, S* __restrict__ v_abs,
    S* __restrict__ v_unc) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t warps_per_block = blockDim.x >> 5;
    const size_t total = size_t(C) * N;
    const size_t group_stride = size_t(gridDim.x) * warps_per_block * 32u;
    const bool chain_var = kVar && var_q != nullptr;
    // The packed two-samples-per-lane walk serves the plain Gaussian VJP.
    constexpr bool kPacked = std::is_same<S, float>::value && !kBeta && !kVar && !kAbs;
    const bool packed = kPacked && v_render != nullptr && uint64_t(width) * height < (uint64_t(1) << 22);
    // Each warp takes 32 consecutive records at a time. Lane-parallel set-up:
    // lane L loads record base + L (coalesced) and computes its pixel box and
    // stepping constants into the warp's shared-memory stage; the warp then
    // walks the 32 records one by one, reading each record's constants with
    // broadcast loads.
    __shared__ RecordStage<S> s_stage[kRecBwdThreads];
    RecordStage<S>* stage = s_stage + (threadIdx.x & ~31u);
    for (size_t base = (size_t(blockIdx.x) * warps_per_block + (threadIdx.x >> 5)) * 32u; base < total;
         base += group_stride) {
        const size_t my_rid = base + lane;
        Rec2D<S> mine;
        uint32_t x0 = 0u, y0 = 0u, w = 0u, area = 0u, magic = 0u;
        const uint32_t my_cam = uint32_t(my_rid) / N;  // C * N < 2^31
        S my_q = S(0);
        if (my_rid < total) {
            if (chain_var) my_q = var_q[uint32_t(my_rid) - my_cam * N];
            const ushort4 rect = rects[my_rid];
            x0 = uint32_t(rect.x) * T;
            y0 = uint32_t(rect.y) * T;
            uint32_t x1 = min(uint32_t(rect.z) * T, width), y1 = min(uint32_t(rect.w) * T, height);
            bool any = rect.z > rect.x && rect.w > rect.y && x0 < x1 && y0 < y1;
            mine = records[my_rid];
            if (any) {
                x1 -= 1u;
                y1 -= 1u;
                any = clip_to_record<S, kBeta>(mine, 0u, 0u, x0, x1, y0, y1);
            }
            if (any) {
                w = x1 - x0 + 1u;
                area = w * (y1 - y0 + 1u);
                if (kPacked) magic = (65536u + w - 1u) / w;
            } else {
                // No pixel can contribute: the record's adjoints are zero.
                S* dst = reinterpret_cast<S*>(grads + my_rid);
#pragma unroll
                for (int i = 0; i < 8; ++i) dst[i] = S(0);
                if (kVar && v_unc != nullptr) v_unc[my_rid] = S(0);
                if (kAbs) {
                    v_abs[2 * my_rid] = S(0);
                    v_abs[2 * my_rid + 1] = S(0);
                }
            }
        }
        // Boxes with at most the quarter-warp area go to quarter-warp groups,
        // up to the half-warp area to half-warp pairs; the rest are walked one
        // by one by the whole warp. (A plain Gaussian record that cannot take
        // the packed walk is not grouped.)
        const bool grouped =
            area != 0u && (kPacked ? packed && area <= kPackedHalfWarpArea : area <= kHalfWarpArea);
        const uint32_t quarter_area = kPacked ? kPackedQuarterWarpArea : kQuarterWarpArea;
        uint32_t pending = __ballot_sync(0xffffffffu, area != 0u && !grouped);
        __syncwarp();  // the previous group's constants have been read
        if (area != 0u) {
            RecordStage<S> st;
            st.r = mine;
            st.x0 = x0;
            st.y0 = y0;
            st.w = w;
            st.area = area;
            st.magic = magic;
            st.cam = my_cam;
            st.q = my_q;
            st.e_min = kPacked ? log2f(1e-5f / fabsf(float(mine.o * mine.mu))) : 0.f;
            stage[lane] = st;
        }
        __syncwarp();
        while (pending != 0u) {
            const uint32_t j = __ffs(pending) - 1u;
            pending &= pending - 1u;
            const RecordStage<S> st = stage[j];
            const Rec2D<S>& r = st.r;
            const uint32_t bx0 = st.x0, by0 = st.y0, bw = st.w, barea = st.area;
            const size_t rid = base + j;
            const uint32_t cam = st.cam;
            const uint32_t n = uint32_t(rid) - cam * N;
            const size_t cam_base = size_t(cam) * height * width;
            const S* vimg = v_render != nullptr ? v_render + cam_base : nullptr;
            const S* vvar = kVar ? v_render_var + cam_base : nullptr;
            const S q = chain_var ? st.q : S(0);
            const S om = r.o * r.mu;
            S part[8];
            S g_ax = S(0), g_ay = S(0);
            bool walked = false;
            if constexpr (kPacked) {
                if (packed) {
                    record_walk_packed(r, om, st.e_min, vimg, bx0, by0, bw, barea, st.magic, width,
                                       (barea + 63u) >> 6, part);
                    walked = true;
                }
            }
            if (!walked)
                record_walk_scalar<S, kBeta, kVar, kAbs, 32u>(r, om, q, vimg, vvar, bx0, by0, bw, barea,
                                                              (barea + 31u) >> 5, width, part, g_ax, g_ay);
            S lo, hi;
            warp_sum8_pairs(part, lo, hi);
            const uint32_t grp = lane >> 3;
            if ((lane & 7u) == 0u) {
                S* dst = reinterpret_cast<S*>(grads + rid);
                S e0, e1, e2;
                record_adjoints<S, kBeta>(r, grp, lo, hi, e0, e1, e2);
                if (grp < 3u) {
                    dst[2 * grp] = e0;
                    dst[2 * grp + 1] = e1;
                }
                if (grp == 2u) dst[6] = e2;
                if (grp == 3u) dst[7] = e0;
                if (kVar && grp == 3u && v_unc != nullptr) v_unc[rid] = hi;
            }
            if (kAbs) {
                g_ax = warp_sum(g_ax);
                g_ay = warp_sum(g_ay);
                if (lane == 0u) {
                    v_abs[2 * rid] = g_ax;
                    v_abs[2 * rid + 1] = g_ay;
                }
            }
        }
        // The small boxes, four or two records per warp step, taken in order of
        // box size: sorted positions [0, n_quad) hold the quarter-warp records,
        // [n_quad, n_group) the half-warp ones, and the other lanes sort last.
        {
            const uint32_t n_group = __popc(__ballot_sync(0xffffffffu, grouped));
            const uint32_t n_quad = __popc(__ballot_sync(0xffffffffu, grouped && area <= quarter_area));
            if (n_group != 0u) {
                const uint32_t sorted = warp_sort_ascending(grouped ? (area << 5) | lane : 0xffffffe0u | lane);
                walk_record_groups<S, kBeta, kVar, kAbs, 8u, kPacked>(sorted, 0u, n_quad, stage, base, N, width, height,
                                                             v_render, v_render_var, chain_var ? var_q : nullptr,
                                                             grads, v_abs, v_unc);
                walk_record_groups<S, kBeta, kVar, kAbs, 16u, kPacked>(sorted, n_quad, n_group, stage, base, N, width,
                                                              height, v_render, v_render_var,
                                                              chain_var ? var_q : nullptr, grads, v_abs, v_unc);
            }
        }
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
    const int64_t* n_dev = nullptr;  // device-side intersection count, overrides n_isects
    uint32_t stage_batch = kFwdBatch;  // forward: records staged in shared memory per batch
};

inline int check_geom(const RasterGeom& g) {
    R2S_REQUIRE(g.T >= 1 && g.T <= 32, R2S_ERR_UNSUPPORTED, "tile_size must be in [1, 32]");
    R2S_REQUIRE(g.C <= 65535, R2S_ERR_UNSUPPORTED, "camera count exceeds 65535");
    R2S_REQUIRE(uint64_t(g.C) * g.N < (uint64_t(1) << 31), R2S_ERR_UNSUPPORTED, "C*N exceeds the int32 range");
    R2S_REQUIRE(uint64_t(g.tiles_x) * g.tiles_y < (uint64_t(1) << 31), R2S_ERR_UNSUPPORTED, "too many tiles");
    R2S_REQUIRE(g.N > 0, R2S_ERR_ARGUMENT, "N must be positive");
    return R2S_OK;
}

template <typename S, bool kBeta, bool kVar>
int launch_fwd_p(const RasterGeom& g, const Rec2D<S>* rec, const S* unc, const int32_t* offsets,
                 const int32_t* ids, S* out, S* out_var, const ImageLossEpilogue<S>& loss, cudaStream_t stream) {
    if constexpr (std::is_same<S, float>::value) {
        // Two pixels per lane: warps of 8x8 pixels.
        const uint32_t blocks = ((g.T + 7) / 8) * ((g.T + 7) / 8);
        const unsigned nthreads = 32u * blocks;
        unsigned batch = g.stage_batch < kFwdBatch ? g.stage_batch : kFwdBatch;
        if (batch < 1) batch = 1;
        const size_t smem = 3 * size_t(batch) * (sizeof(Rec2D<S>) + (kVar ? sizeof(S) : 0)) +
                            2 * size_t(batch) * sizeof(uint2) + size_t(nthreads) * sizeof(uint16_t) + 64;
        dim3 grid(g.tiles_x * g.tiles_y, g.C);
        if (nthreads <= 128) {
            R2S_TRY(allow_dynamic_smem(raster_fwd_pair_kernel<kBeta, kVar, 128>, smem));
            raster_fwd_pair_kernel<kBeta, kVar, 128><<<grid, nthreads, smem, stream>>>(
                rec, unc, g.N, offsets, ids, int32_t(g.n_isects), g.n_dev, g.C, g.width, g.height, g.T, g.tiles_x,
                g.tiles_x * g.tiles_y, out, out_var, batch, loss);
        } else {
            R2S_TRY(allow_dynamic_smem(raster_fwd_pair_kernel<kBeta, kVar, 512>, smem));
            raster_fwd_pair_kernel<kBeta, kVar, 512><<<grid, nthreads, smem, stream>>>(
                rec, unc, g.N, offsets, ids, int32_t(g.n_isects), g.n_dev, g.C, g.width, g.height, g.T, g.tiles_x,
                g.tiles_x * g.tiles_y, out, out_var, batch, loss);
        }
        return check_launch("rasterize_to_pixels_fwd");
    } else {
        // fp64: one warp per 8x4 block of the tile, at most 4 x 8 warps for 32x32 tiles.
        const uint32_t blocks = ((g.T + kBlockW - 1) / kBlockW) * ((g.T + kBlockH - 1) / kBlockH);
        const unsigned nthreads = 32u * blocks;
        unsigned batch = g.stage_batch < kFwdBatch ? g.stage_batch : kFwdBatch;
        if (batch > nthreads) batch = nthreads;
        if (batch < 1) batch = 1;
        const size_t smem = 3 * size_t(batch) * (sizeof(Rec2D<S>) + sizeof(S)) + 2 * size_t(batch) * sizeof(uint2) +
                            size_t(nthreads) * sizeof(uint16_t);
        dim3 grid(g.tiles_x * g.tiles_y, g.C);
        if (nthreads <= 256) {
            // Tiles up to 16x16: a register budget sized for 256-thread CTAs.
            R2S_TRY(allow_dynamic_smem(raster_fwd_kernel<S, kBeta, kVar, 256>, smem));
            raster_fwd_kernel<S, kBeta, kVar, 256><<<grid, nthreads, smem, stream>>>(
                rec, unc, g.N, offsets, ids, int32_t(g.n_isects), g.n_dev, g.C, g.width, g.height, g.T, g.tiles_x,
                g.tiles_x * g.tiles_y, out, out_var, batch, loss);
        } else {
            R2S_TRY(allow_dynamic_smem(raster_fwd_kernel<S, kBeta, kVar, 1024>, smem));
            raster_fwd_kernel<S, kBeta, kVar, 1024><<<grid, nthreads, smem, stream>>>(
                rec, unc, g.N, offsets, ids, int32_t(g.n_isects), g.n_dev, g.C, g.width, g.height, g.T, g.tiles_x,
                g.tiles_x * g.tiles_y, out, out_var, batch, loss);
        }
        return check_launch("rasterize_to_pixels_fwd");
    }
}

template <typename S>
int launch_fwd(const RasterGeom& g, const Rec2D<S>* rec, const S* unc, bool beta, const int32_t* offsets,
               const int32_t* ids, S* out, S* out_var, cudaStream_t stream,
               const ImageLossEpilogue<S>& loss = ImageLossEpilogue<S>{}) {
    R2S_TRY(check_geom(g));
    if (g.tiles_x == 0 || g.tiles_y == 0 || g.C == 0) return R2S_OK;
    const bool var = out_var != nullptr;
    if (beta) {
        return var ? launch_fwd_p<S, true, true>(g, rec, unc, offsets, ids, out, out_var, loss, stream)
                   : launch_fwd_p<S, true, false>(g, rec, unc, offsets, ids, out, out_var, loss, stream);
    }
    return var ? launch_fwd_p<S, false, true>(g, rec, unc, offsets, ids, out, out_var, loss, stream)
               : launch_fwd_p<S, false, false>(g, rec, unc, offsets, ids, out, out_var, loss, stream);
}

template <typename S, bool kBeta, bool kVar, bool kAbs>
int launch_bwd_p(const RasterGeom& g, const Rec2D<S>* rec, const S* var_q, const int32_t* offsets,
                 const int32_t* ids, const S* v_render, const S* v_render_var, Rec2D<S>* grads, S* v_abs,
                 S* v_unc, cudaStream_t stream) {
    const size_t smem = 2 * size_t(kBwdThreads) * (sizeof(Rec2D<S>) + sizeof(S) + sizeof(int32_t)) +
                        size_t(kBwdThreads) * sizeof(TileBox) + 2 * size_t(g.T) * g.T * sizeof(S);
    R2S_TRY(allow_dynamic_smem(raster_bwd_kernel<S, kBeta, kVar, kAbs>, smem));
    dim3 grid(g.tiles_x * g.tiles_y, g.C);
    raster_bwd_kernel<S, kBeta, kVar, kAbs><<<grid, kBwdThreads, smem, stream>>>(
        rec, var_q, g.N, offsets, ids, int32_t(g.n_isects), g.n_dev, g.C, g.width, g.height, g.T, g.tiles_x,
        g.tiles_x * g.tiles_y, v_render, v_render_var, grads, v_abs, v_unc);
    return check_launch("rasterize_to_pixels_bwd");
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

template <typename S, bool kBeta, bool kVar, bool kAbs>
int launch_record_bwd_t(const RasterGeom& g, const Rec2D<S>* rec, const ushort4* rects, const S* var_q,
                        const S* v_render, const S* v_render_var, Rec2D<S>* grads, S* v_abs, S* v_unc,
                        cudaStream_t stream) {
    const size_t total = size_t(g.C) * g.N;
    const size_t warps_per_block = kRecBwdThreads / 32;
    int device = 0, sms = 148, per_sm = 4;
    if (cudaGetDevice(&device) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, raster_record_bwd_kernel<S, kBeta, kVar, kAbs>,
                                                  kRecBwdThreads, 0);
    // Persistent grid: exactly the resident blocks, each warp striding over
    // records, so every warp takes the same number of records and none waits
    // for a late wave.
    size_t blocks = (total + warps_per_block - 1) / warps_per_block;
    const size_t cap = size_t(sms > 0 ? sms : 148) * size_t(per_sm > 0 ? per_sm : 1);
    if (blocks > cap) blocks = cap;
    raster_record_bwd_kernel<S, kBeta, kVar, kAbs><<<unsigned(blocks), kRecBwdThreads, 0, stream>>>(
        rec, rects, var_q, g.C, g.N, g.width, g.height, g.T, v_render, v_render_var, grads, v_abs, v_unc);
    return check_launch("raster_record_bwd");
}

template <typename S, bool kBeta>
int launch_record_bwd_b(const RasterGeom& g, const Rec2D<S>* rec, const ushort4* rects, const S* var_q,
                        const S* v_render, const S* v_render_var, Rec2D<S>* grads, S* v_abs, S* v_unc,
                        cudaStream_t stream) {
    const bool var = v_render_var != nullptr, abs = v_abs != nullptr;
    if (var && abs)
        return launch_record_bwd_t<S, kBeta, true, true>(g, rec, rects, var_q, v_render, v_render_var, grads, v_abs,
                                                         v_unc, stream);
    if (var)
        return launch_record_bwd_t<S, kBeta, true, false>(g, rec, rects, var_q, v_render, v_render_var, grads, v_abs,
                                                          v_unc, stream);
    if (abs)
        return launch_record_bwd_t<S, kBeta, false, true>(g, rec, rects, var_q, v_render, v_render_var, grads, v_abs,
                                                          v_unc, stream);
    return launch_record_bwd_t<S, kBeta, false, false>(g, rec, rects, var_q, v_render, v_render_var, grads, v_abs,
                                                       v_unc, stream);
}

template <typename S>
size_t raster_ws(uint32_t C, uint32_t N, bool with_grads) {
    ArenaSize a;
    a.take<Rec2D<S>>(size_t(C) * N);
    if (with_grads) a.take<Rec2D<S>>(size_t(C) * N);
    return a.bytes();
}

// out[n] = sum over c of per_record[c, n], in camera order (deterministic).
template <typename S>
__global__ void sum_over_cameras_kernel(const S* __restrict__ per_record, uint32_t C, uint32_t N,
                                        S* __restrict__ out) {
    const uint32_t n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= N) return;
    S acc = S(0);
    for (uint32_t c = 0; c < C; ++c) acc += per_record[size_t(c) * N + n];
    out[n] = acc;
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

int r2s_sum_over_cameras(int dtype, const void* per_record, uint32_t C, uint32_t N, void* out, void* stream) {
    if (N == 0) return R2S_OK;
    R2S_REQUIRE(per_record != nullptr && out != nullptr, R2S_ERR_ARGUMENT, "per_record and out must be non-null");
    R2S_DISPATCH(dtype, sum_over_cameras_kernel<S><<<blocks_for(N, 256), 256, 0, as_stream(stream)>>>(
        static_cast<const S*>(per_record), C, N, static_cast<S*>(out)));
    return check_launch("sum_over_cameras");
}

int r2s_raster_record_bwd(int dtype, const void* records, const uint16_t* rects, const void* uncertainties, int beta,
                          int detach_variance, const void* v_render, const void* v_render_var, uint32_t C,
                          uint32_t N, uint32_t width, uint32_t height, uint32_t tile_size, void* grads,
                          void* v_means2d_abs, void* v_uncertainties, void* stream) {
    const RasterGeom g{C, N, 0u, width, height, tile_size, 1u, 1u};
    R2S_TRY(check_geom(g));
    R2S_REQUIRE(uint64_t(width) * height < (uint64_t(1) << 32), R2S_ERR_UNSUPPORTED, "image too large");
    R2S_REQUIRE(v_render_var == nullptr || v_uncertainties != nullptr, R2S_ERR_ARGUMENT,
                "variance adjoint needs v_uncertainties");
    if (uint64_t(C) * N == 0) return R2S_OK;
    R2S_DISPATCH(dtype, {
        const S* var_q = detach_variance ? nullptr : static_cast<const S*>(uncertainties);
        const auto* rec = static_cast<const Rec2D<S>*>(records);
        const auto* rc = reinterpret_cast<const ushort4*>(rects);
        return beta ? launch_record_bwd_b<S, true>(g, rec, rc, var_q, static_cast<const S*>(v_render),
                                                   static_cast<const S*>(v_render_var), static_cast<Rec2D<S>*>(grads),
                                                   static_cast<S*>(v_means2d_abs), static_cast<S*>(v_uncertainties),
                                                   as_stream(stream))
                    : launch_record_bwd_b<S, false>(g, rec, rc, var_q, static_cast<const S*>(v_render),
                                                    static_cast<const S*>(v_render_var), static_cast<Rec2D<S>*>(grads),
                                                    static_cast<S*>(v_means2d_abs), static_cast<S*>(v_uncertainties),
                                                    as_stream(stream));
    });
}

int r2s_raster_render_capacity(int dtype, const void* records, const void* uncertainties, int beta,
                               const int32_t* tile_offsets, const int32_t* flatten_ids, const int64_t* n_used,
                               uint32_t C, uint32_t N, uint32_t width, uint32_t height, uint32_t tile_size,
                               uint32_t tiles_x, uint32_t tiles_y, uint32_t stage_batch, void* render,
                               void* render_var, void* stream) {
    R2S_REQUIRE(n_used != nullptr, R2S_ERR_ARGUMENT, "n_used must be non-null");
    RasterGeom g{C, N, 1u, width, height, tile_size, tiles_x, tiles_y};
    g.n_dev = n_used;
    if (stage_batch != 0) g.stage_batch = stage_batch;
    R2S_DISPATCH(dtype, return launch_fwd<S>(g, static_cast<const Rec2D<S>*>(records),
                                             static_cast<const S*>(uncertainties), beta != 0, tile_offsets,
                                             flatten_ids, static_cast<S*>(render), static_cast<S*>(render_var),
                                             as_stream(stream)));
}

size_t r2s_raster_image_loss_workspace(uint32_t C, uint32_t tiles_x, uint32_t tiles_y) {
    ArenaSize a;
    a.take<double>(size_t(C) * tiles_x * tiles_y);
    return a.bytes();
}

int r2s_raster_render_image_loss(int dtype, const void* records, const void* uncertainties, int beta,
                                 const int32_t* tile_offsets, const int32_t* flatten_ids, uint32_t n_isects,
                                 const int64_t* n_used, uint32_t C, uint32_t N, uint32_t width, uint32_t height,
                                 uint32_t tile_size, uint32_t tiles_x, uint32_t tiles_y, uint32_t stage_batch,
                                 const void* target, int loss_kind, float lambda, void* render, void* render_var,
                                 void* v_render, void* loss, void* loss_value, void* workspace,
                                 size_t workspace_bytes, void* stream) {
    R2S_REQUIRE(loss_kind == R2S_IMAGE_LOSS_MSE || loss_kind == R2S_IMAGE_LOSS_L1, R2S_ERR_ARGUMENT,
                "loss_kind must be R2S_IMAGE_LOSS_MSE or R2S_IMAGE_LOSS_L1");
    R2S_REQUIRE(target != nullptr && v_render != nullptr && loss != nullptr && loss_value != nullptr,
                R2S_ERR_ARGUMENT, "target, v_render, loss and loss_value must be non-null");
    RasterGeom g{C, N, n_isects, width, height, tile_size, tiles_x, tiles_y};
    g.n_dev = n_used;
    if (stage_batch != 0) g.stage_batch = stage_batch;
    const uint64_t n_keys = uint64_t(C) * tiles_x * tiles_y;
    R2S_REQUIRE(n_keys < (uint64_t(1) << 31), R2S_ERR_UNSUPPORTED, "too many tiles");
    Arena arena(workspace, workspace_bytes);
    double* partials = arena.take<double>(n_keys);
    R2S_REQUIRE(partials || n_keys == 0, R2S_ERR_WORKSPACE, "image-loss workspace too small");
    const int64_t numel = int64_t(C) * height * width;
    cudaStream_t st = as_stream(stream);
    R2S_DISPATCH(dtype, {
        ImageLossEpilogue<S> ep;
        ep.target = static_cast<const S*>(target);
        ep.v_render = static_cast<S*>(v_render);
        ep.partials = partials;
        ep.l1 = loss_kind == R2S_IMAGE_LOSS_L1 ? 1u : 0u;
        // mse: the factor torch applies in `(img - tgt).mul_(2 / numel)`, rounded to S once.
        ep.scale = ep.l1 ? static_cast<S>(lambda)
                         : static_cast<S>(2.0 * double(lambda) / double(numel > 0 ? numel : 1));
        ep.numel = static_cast<S>(numel > 0 ? numel : 1);
        R2S_TRY(launch_fwd<S>(g, static_cast<const Rec2D<S>*>(records), static_cast<const S*>(uncertainties),
                              beta != 0, tile_offsets, flatten_ids, static_cast<S*>(render),
                              static_cast<S*>(render_var), st, ep));
        const bool launched = g.tiles_x != 0 && g.tiles_y != 0 && g.C != 0;
        return launch_finish_mean(dtype, partials, launched ? int(n_keys) : 0, numel, lambda, loss, loss_value, st);
    });
}

}  // extern "C"
