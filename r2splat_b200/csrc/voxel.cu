// Voxelization: per-tile (T^3 voxels) accumulation of Gaussian / Beta
// densities at voxel centres, and its VJP, on packed per-primitive records.
//
// Same schedule as the rasterizer: one CTA per 3D tile, the tile's
// intersection list gathered into shared memory with cp.async in buffered
// batches (records are [N] x 64 B and stay in L2). Forward threads own a row
// of 8 voxels (Gaussian fp32 at T = 8), 4 voxels of a row, or single voxels;
// backward warps own one record at a time over the record's box in the tile,
// warp-reduce, and either write the record's partial adjoints to its own slot
// (reduced per primitive in a fixed order afterwards) or add them with vector
// atomics.
//
// Per-sample arithmetic keeps the reference's expression forms
// (VoxelizeToVoxelsFwd.cu:180-215, :555-580; VoxelizeToVoxelsBwd.cu:397-433,
// :853-895) so the |alpha| thresholds (1e-6 Gaussian, 1e-5 Beta) select the
// same samples. The tile size is a run-time value, so the compiler cannot
// merge arithmetic across a thread's voxels.
#include <type_traits>

#include "common.cuh"
#include "geometry.cuh"

namespace r2s {

// Voxel placement inside a tile: z-plane p / T^2, then a per-plane rotation of
// (y, x) so a thread's voxels in different planes get different y and x.
__device__ __forceinline__ void tile_voxel(uint32_t p, uint32_t T, uint32_t& lz, uint32_t& ly, uint32_t& lx) {
    const uint32_t plane = T * T;
    lz = p / plane;
    const uint32_t rem = p - lz * plane;
    const uint32_t y = rem / T;
    const uint32_t x = rem - y * T;
    ly = (y + 5u * lz) % T;
    lx = (x + 3u * lz) % T;
}

template <typename S>
__device__ __forceinline__ void gather_record3(Rec3D<S>* dst, const Rec3D<S>* src) {
    const char* s = reinterpret_cast<const char*>(src);
    char* d = reinterpret_cast<char*>(dst);
#pragma unroll
    for (int k = 0; k < int(sizeof(Rec3D<S>) / 16); ++k) cp_async16(d + 16 * k, s + 16 * k);
}

struct VoxelGeom {
    uint32_t N, n_isects, dim2, dim1, dim0, T, tiles_x, tiles_y, tiles_z;
    const int64_t* n_dev = nullptr;  // device-side intersection count, overrides n_isects
};

// Bulk-staging waits that ran out (a tile batch's copy did not complete
// within kBulkWaitLimitNs): counted per device, read and cleared by
// r2s_bulk_wait_faults(). A kernel that gives up on a wait waits (bounded)
// for its copies in flight and leaves the rest of its tile unwritten.
static __device__ unsigned int g_bulk_wait_faults;

// kBulk: `records` is the per-tile packed copy (packed[i] is the record of
// sorted intersection i, flatten_ids unused), and each batch is staged by one
// bulk copy; otherwise records are gathered through flatten_ids by cp.async.
// The two-row form (PPT = 16) runs only at T = 8 (3D tiles are at most 10
// wide), one warp per tile; bounding it to 80 registers keeps its accumulators
// out of local memory.
template <typename S, bool kBeta, bool kVar, int PPT, bool kBulk>
__global__ void __launch_bounds__(PPT == 16 ? 32 : 256, PPT == 16 ? 24 : 1) voxel_fwd_kernel(const Rec3D<S>* __restrict__ records,
                                                        const int32_t* __restrict__ offsets,
                                                        const int32_t* __restrict__ flatten_ids, VoxelGeom g,
                                                        S* __restrict__ volume, S* __restrict__ volume_var) {
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ uint64_t s_bar[3];
    const uint32_t nthreads = blockDim.x;
    Rec3D<S>* s_rec = reinterpret_cast<Rec3D<S>*>(smem);  // [3][nthreads]
    const uint32_t T = g.T;
    const uint32_t n_tiles = g.tiles_x * g.tiles_y * g.tiles_z;
    const uint32_t key = blockIdx.x;
    const int32_t start = offsets[key];
    const int32_t n_total = g.n_dev != nullptr ? int32_t(*g.n_dev) : int32_t(g.n_isects);
    const int32_t end = (key + 1 == n_tiles) ? n_total : offsets[key + 1];
    const uint32_t tz = key / (g.tiles_x * g.tiles_y);
    const uint32_t rem = key - tz * g.tiles_x * g.tiles_y;
    const uint32_t ty = rem / g.tiles_x, tx = rem - ty * g.tiles_x;
    const uint32_t t = threadIdx.x;
    // PPT = 4 or 8: a thread owns PPT consecutive voxels of one row (same y,
    // z), so the Gaussian terms in d2 and d3 alone are computed once per
    // record and the record's shared-memory reads are spread over PPT samples.
    // PPT = 16: eight consecutive voxels of each of two adjacent rows (y and
    // y + 1 of one z-plane; T even), which also share the terms in d1 alone.
    // PPT = 1: voxels placed by tile_voxel.
    constexpr bool kRows = PPT >= 4;
    constexpr bool kRowShared = kRows && !kBeta && std::is_same<S, float>::value;
    constexpr int kRowsPer = PPT == 16 ? 2 : 1;   // rows per thread
    constexpr int kRowLen = PPT / kRowsPer;      // voxels per row segment

    S px[PPT], py[PPT], pz[PPT], acc[PPT], accv[PPT];
    bool inside[PPT];
    const uint32_t segs = (T + uint32_t(kRowLen) - 1u) / uint32_t(kRowLen);
    const uint32_t row = kRows ? (t / segs) * uint32_t(kRowsPer) : 0u;  // the thread's first row
    const uint32_t seg = kRows ? t - (t / segs) * segs : 0u;
    // Global voxel coordinates (i = z, j = y, kk = x) of the thread's k-th voxel.
    auto voxel_of = [&](int k, uint32_t& i, uint32_t& j, uint32_t& kk) {
        uint32_t lz, ly, lx;
        bool in_tile;
        if (kRows) {
            const uint32_t r = row + uint32_t(k / kRowLen);
            lz = r / T;
            ly = r - lz * T;
            lx = uint32_t(kRowLen) * seg + uint32_t(k % kRowLen);
            in_tile = r < T * T && lx < T;
        } else {
            const uint32_t p = t + uint32_t(k) * nthreads;
            tile_voxel(p, T, lz, ly, lx);
            in_tile = p < T * T * T;
        }
        i = tz * T + lz;
        j = ty * T + ly;
        kk = tx * T + lx;
        return in_tile && i < g.dim0 && j < g.dim1 && kk < g.dim2;
    };
#pragma unroll
    for (int k = 0; k < PPT; ++k) {
        uint32_t i, j, kk;
        inside[k] = voxel_of(k, i, j, kk);
        px[k] = static_cast<S>(kk) + static_cast<S>(0.5);
        py[k] = static_cast<S>(j) + static_cast<S>(0.5);
        pz[k] = static_cast<S>(i) + static_cast<S>(0.5);
        acc[k] = S(0);
        accv[k] = S(0);
    }

    const int32_t count = end - start;
    const int32_t n_batches = count > 0 ? (count + int32_t(nthreads) - 1) / int32_t(nthreads) : 0;
    if (kBulk && n_batches > 0) {
        if (t == 0) {
#pragma unroll
            for (int k = 0; k < 3; ++k) mbar_init(&s_bar[k], 1u);
            mbar_init_fence();
        }
        __syncthreads();
    }
    auto load = [&](int32_t b, int stage) {
        if (kBulk) {
            if (t == 0) {
                const int32_t first = start + b * int32_t(nthreads);
                const uint32_t bytes = uint32_t(min(int32_t(nthreads), end - first)) * uint32_t(sizeof(Rec3D<S>));
                fence_proxy_async_shared();
                mbar_arrive_expect_tx(&s_bar[stage], bytes);
                bulk_load_g2s(s_rec + stage * nthreads, records + first, bytes, &s_bar[stage]);
            }
        } else {
            const int32_t idx = start + b * int32_t(nthreads) + int32_t(t);
            if (idx < end) gather_record3(s_rec + stage * nthreads + t, records + flatten_ids[idx]);
            cp_async_commit();
        }
    };
    if (n_batches > 0) load(0, 0);
    for (int32_t b = 0; b < n_batches; ++b) {
        if (b + 1 < n_batches) {
            load(b + 1, (b + 1) % 3);
            if (!kBulk) cp_async_wait<1>();
        } else if (!kBulk) {
            cp_async_wait<0>();
        }
        if (kBulk) {
            // Batch b is the (b / 3)-th use of its stage's barrier.
            const bool ok = mbar_wait_bounded(&s_bar[b % 3], uint32_t(b / 3) & 1u);
            if (__syncthreads_or(!ok)) {
                if (t == 0) {
                    atomicAdd(&g_bulk_wait_faults, 1u);
                    mbar_wait_bounded(&s_bar[b % 3], uint32_t(b / 3) & 1u);
                    if (b + 1 < n_batches) mbar_wait_bounded(&s_bar[(b + 1) % 3], uint32_t((b + 1) / 3) & 1u);
                }
                __syncthreads();
                return;
            }
        } else {
            __syncthreads();
        }
        const Rec3D<S>* buf = s_rec + (b % 3) * nthreads;
        const int32_t batch = min(int32_t(nthreads), count - b * int32_t(nthreads));
        for (int32_t s = 0; s < batch; ++s) {
            const Rec3D<S> r = buf[s];
            if constexpr (kRowShared && PPT == 16) {
                // As below, for two rows (d2 = da, db) of one z-plane: the
                // factors in d1 alone (d1, c00 d1, c01 d1, c02 d1) are shared
                // by the rows; each sample's expression and rounding are the
                // single-row form's.
                const float da = py[0] - r.y, db = py[kRowLen] - r.y, d3 = pz[0] - r.z;
                const float b2a = __fmul_rn(__fmul_rn(r.c11, da), da);
                const float b2b = __fmul_rn(__fmul_rn(r.c11, db), db);
                const float c22d3 = __fmul_rn(r.c22, d3);
                const float c12da = __fmul_rn(r.c12, da), c12db = __fmul_rn(r.c12, db);
                const float2 nx = splat2(-r.x), c00 = splat2(r.c00), c01 = splat2(r.c01), c02 = splat2(r.c02);
                const float2 b22a = splat2(b2a), b22b = splat2(b2b), c22d32 = splat2(c22d3);
                const float2 c12a2 = splat2(c12da), c12b2 = splat2(c12db);
                const float2 da2 = splat2(da), db2 = splat2(db), d32 = splat2(d3), half = splat2(0.5f);
                auto add_sample = [&](int k, float sigma) {
                    const float alpha = r.o * exp(-sigma);
                    if (!(sigma < 0.f || fabs(alpha) < 1e-6f)) {
                        acc[k] += alpha;
                        if (kVar) accv[k] = fmaf(__fmul_rn(r.q, alpha), alpha, accv[k]);
                    }
                };
#pragma unroll
                for (int k = 0; k < kRowLen; k += 2) {
                    const float2 d1 = add2(make_float2(px[k], px[k + 1]), nx);
                    const float2 c00d1 = mul2(c00, d1), c01d1 = mul2(c01, d1), c02d1 = mul2(c02, d1);
                    const float2 s3a = fma2(c22d32, d32, fma2(c00d1, d1, b22a));
                    const float2 s3b = fma2(c22d32, d32, fma2(c00d1, d1, b22b));
                    const float2 laa = fma2(c01d1, da2, mul2(half, s3a));
                    const float2 lab = fma2(c01d1, db2, mul2(half, s3b));
                    const float2 sa = fma2(c12a2, d32, fma2(c02d1, d32, laa));
                    const float2 sb = fma2(c12b2, d32, fma2(c02d1, d32, lab));
                    add_sample(k, sa.x);
                    add_sample(k + 1, sa.y);
                    add_sample(kRowLen + k, sb.x);
                    add_sample(kRowLen + k + 1, sb.y);
                }
            } else if constexpr (kRowShared) {
                // The reference's sigma with its contraction made explicit, as
                // nvcc -O3 --use_fast_math compiles the reference's kernel
                // (VoxelizeToVoxelsFwd.cu:200-205): S3 = fma(c22 d3, d3,
                // fma(c00 d1, d1, (c11 d2) d2)), then sigma = fma(c12 d2, d3,
                // fma(c02 d1, d3, fma(c01 d1, d2, S3 / 2))). The d2/d3 factors are
                // shared by the row, and the four voxels go two at a time through
                // packed FP32x2 operations, each component rounding as the scalar
                // operation does.
                const float d2 = py[0] - r.y, d3 = pz[0] - r.z;
                const float b2 = __fmul_rn(__fmul_rn(r.c11, d2), d2);
                const float c22d3 = __fmul_rn(r.c22, d3), c12d2 = __fmul_rn(r.c12, d2);
                const float2 nx = splat2(-r.x), c00 = splat2(r.c00), c01 = splat2(r.c01), c02 = splat2(r.c02);
                const float2 b22 = splat2(b2), c22d32 = splat2(c22d3), c12d22 = splat2(c12d2);
                const float2 d22 = splat2(d2), d32 = splat2(d3), half = splat2(0.5f);
#pragma unroll
                for (int k = 0; k < PPT; k += 2) {
                    const float2 d1 = add2(make_float2(px[k], px[k + 1]), nx);
                    const float2 s3 = fma2(c22d32, d32, fma2(mul2(c00, d1), d1, b22));
                    const float2 la = fma2(mul2(c01, d1), d22, mul2(half, s3));
                    const float2 sigma = fma2(c12d22, d32, fma2(mul2(c02, d1), d32, la));
                    const float alpha0 = r.o * exp(-sigma.x);
                    const float alpha1 = r.o * exp(-sigma.y);
                    if (!(sigma.x < 0.f || fabs(alpha0) < 1e-6f)) {
                        acc[k] += alpha0;
                        if (kVar) accv[k] = fmaf(__fmul_rn(r.q, alpha0), alpha0, accv[k]);
                    }
                    if (!(sigma.y < 0.f || fabs(alpha1) < 1e-6f)) {
                        acc[k + 1] += alpha1;
                        if (kVar) accv[k + 1] = fmaf(__fmul_rn(r.q, alpha1), alpha1, accv[k + 1]);
                    }
                }
            } else {
#pragma unroll
                for (int k = 0; k < PPT; ++k) {
                    if (!kBeta) {
                        // Same contraction as above (VoxelizeToVoxelsFwd.cu:200-205, :390-396).
                        const S d1 = px[k] - r.x, d2 = py[k] - r.y, d3 = pz[k] - r.z;
                        const S s3 = fma(mul_rn(r.c22, d3), d3, fma(mul_rn(r.c00, d1), d1, mul_rn(mul_rn(r.c11, d2), d2)));
                        const S sigma = fma(mul_rn(r.c12, d2), d3,
                                            fma(mul_rn(r.c02, d1), d3,
                                                fma(mul_rn(r.c01, d1), d2, mul_rn(static_cast<S>(0.5), s3))));
                        const S alpha = r.o * exp(-sigma);
                        if (!(sigma < static_cast<S>(0) || fabs(alpha) < static_cast<S>(1e-6))) {
                            acc[k] += alpha;
                            if (kVar) accv[k] = fma(mul_rn(r.q, alpha), alpha, accv[k]);
                        }
                    } else {
                        // The reference's d^T Q d (VoxelizeToVoxelsFwd.cu:563-567) with its contraction
                        // explicit: s = fma(c d3, d3, fma(a d1, d1, (bb d2) d2)), then
                        // q = fma((2 r) d2, d3, fma((2 q) d1, d3, fma((2 p) d1, d2, s))).
                        const S d1 = r.x - px[k], d2 = r.y - py[k], d3 = r.z - pz[k];
                        const S two = static_cast<S>(2);
                        const S sq = fma(mul_rn(r.c22, d3), d3, fma(mul_rn(r.c00, d1), d1, mul_rn(mul_rn(r.c11, d2), d2)));
                        const S qf = fma(mul_rn(mul_rn(two, r.c12), d2), d3,
                                         fma(mul_rn(mul_rn(two, r.c02), d1), d3, fma(mul_rn(mul_rn(two, r.c01), d1), d2, sq)));
                        if (!(qf < static_cast<S>(0) || qf >= static_cast<S>(1))) {
                            const S h = static_cast<S>(1) - qf;
                            const S alpha = r.o * pow(h, r.beta);
                            if (!(fabs(alpha) < static_cast<S>(1e-5))) {
                                acc[k] += alpha;
                                if (kVar) accv[k] = fma(mul_rn(r.q, alpha), alpha, accv[k]);
                            }
                        }
                    }
                }
            }
        }
        // No barrier here: the next load goes to the third buffer, whose batch
        // every thread finished before this iteration's barrier.
    }
#pragma unroll
    for (int k = 0; k < PPT; ++k) {
        if (inside[k]) {
            uint32_t i, j, kk;
            voxel_of(k, i, j, kk);
            const size_t vid = (size_t(i) * g.dim1 + j) * g.dim2 + kk;
            volume[vid] = acc[k];
            if (kVar) volume_var[vid] = accv[k];
        }
    }
}

constexpr int kVoxBwdWarps = 8;
constexpr int kVoxBwdThreads = kVoxBwdWarps * 32;

// A record's box on one 3D tile, tile-local: origin x0 | y0 << 8 | z0 << 16,
// extent w | h << 8 | d << 16, and ceil(65536 / h), with which
// (k * magic_h) >> 16 == k / h for every k < 1024 and h <= 32. An empty box has
// a zero extent.
struct alignas(16) VoxelBox {
    uint32_t origin, extent, magic_h, unused;
};

// Conservative box of the voxels whose sample can pass the contribution test
// (the 3D form of the rasterizer's pixel box). Gaussian: |o| exp(-sigma) >=
// 1e-6 needs sigma <= s = ln(|o| 1e6), sigma = d^T Q d / 2. For Q positive
// definite with tr(Q)^3 / det(Q) <= 700 (which bounds the ratio of the
// magnitude of sigma's terms to sigma, tr / lambda_min), the rounded sigma is
// within 10 * 2^-24 * 700 < 5e-4 of sigma relative, so every passing voxel
// lies in sigma <= s' = s + 1e-3 |s| + 1e-3, whose bounding box has
// half-widths sqrt(2 s' adj(Q)_ii / det(Q)). Beta: d^T Q d < 1, so d^T Q d <
// 1.001. Half-widths are widened by 0.1 % + 0.01 voxel and by 1e-6 of the
// coordinates' magnitude; any other case takes the whole tile.
template <typename S, bool kBeta>
__device__ __forceinline__ bool voxel_box_bounds(const Rec3D<S>& r, uint32_t ox, uint32_t oy, uint32_t oz,
                                                 uint32_t vx, uint32_t vy, uint32_t vz, uint32_t* lo,
                                                 uint32_t* hi) {
    lo[0] = lo[1] = lo[2] = 0u;
    hi[0] = vx - 1;
    hi[1] = vy - 1;
    hi[2] = vz - 1;
    const S a = r.c00, p = r.c01, q = r.c02, bb = r.c11, rr = r.c12, c = r.c22;
    const S adj0 = bb * c - rr * rr;
    const S adj1 = a * c - q * q;
    const S adj2 = a * bb - p * p;
    const S det = a * adj0 - p * (p * c - rr * q) + q * (p * rr - bb * q);
    const S tr = a + bb + c;
    bool bounded = a > S(0) && bb > S(0) && c > S(0) && adj0 > S(0) && adj1 > S(0) && adj2 > S(0) &&
                   det > S(0) && tr * tr * tr <= S(700) * det;
    S reach = S(1.001);
    if (!kBeta) {
        S s = log(fabs(r.o)) + S(13.815510557964274);  // ln(1e6)
        s = s + S(1e-3) * fabs(s) + S(1e-3);
        if (bounded && isfinite(s) && s < S(0)) return false;
        bounded = bounded && isfinite(s);
        reach = S(2) * s;
    }
    if (bounded) {
        const S adj[3] = {adj0, adj1, adj2};
        const S centre[3] = {r.x, r.y, r.z};
        const uint32_t origin[3] = {ox, oy, oz};
#pragma unroll
        for (int axis = 0; axis < 3; ++axis) {
            const S h = sqrt(reach * adj[axis] / det) * S(1.001) + S(0.01);
            const S cc = centre[axis] - S(0.5) - static_cast<S>(origin[axis]);
            const S m = S(1e-6) * (fabs(centre[axis]) + h + static_cast<S>(origin[axis]));
            const S l = ceil(cc - h - m), u = floor(cc + h + m);
            if (!(isfinite(l) && isfinite(u))) continue;
            if (u < S(0) || l > static_cast<S>(hi[axis])) return false;
            if (l > S(0)) lo[axis] = static_cast<uint32_t>(l);
            if (u < static_cast<S>(hi[axis])) hi[axis] = static_cast<uint32_t>(u);
            if (lo[axis] > hi[axis]) return false;
        }
    }
    return true;
}

template <typename S, bool kBeta>
__device__ __forceinline__ VoxelBox voxel_box(const Rec3D<S>& r, uint32_t ox, uint32_t oy, uint32_t oz, uint32_t vx,
                                              uint32_t vy, uint32_t vz) {
    uint32_t lo[3], hi[3];
    if (!voxel_box_bounds<S, kBeta>(r, ox, oy, oz, vx, vy, vz, lo, hi)) return VoxelBox{0u, 0u, 1u, 0u};
    const uint32_t w = hi[0] - lo[0] + 1, h = hi[1] - lo[1] + 1, d = hi[2] - lo[2] + 1;
    VoxelBox box;
    box.origin = lo[0] | (lo[1] << 8) | (lo[2] << 16);
    box.extent = w | (h << 8) | (d << 16);
    box.magic_h = (65536u + h - 1u) / h;
    box.unused = 0u;
    return box;
}

// A primitive's 3D tile box as the intersection lists enumerate it (the tile
// span of IsectTiles3DKernel.cu:38-112 on the voxel-space mean and radii):
// [lo, hi) per axis; false when it has no tiles.
template <typename S>
__device__ __forceinline__ bool tile_box_3d(const S* mean_v, const int32_t* radius, uint32_t T, uint32_t tiles_x,
                                            uint32_t tiles_y, uint32_t tiles_z, uint32_t* lo, uint32_t* hi) {
    const int32_t rx = radius[0], ry = radius[1], rz = radius[2];
    if (rx <= 0 || ry <= 0 || rz <= 0) return false;
    tile_span(mean_v[0], static_cast<S>(rx), T, tiles_x, lo[0], hi[0]);
    tile_span(mean_v[1], static_cast<S>(ry), T, tiles_y, lo[1], hi[1]);
    tile_span(mean_v[2], static_cast<S>(rz), T, tiles_z, lo[2], hi[2]);
    return hi[0] > lo[0] && hi[1] > lo[1] && hi[2] > lo[2];
}

template <typename S>
__device__ __forceinline__ bool tile_box_3d(const S* means_v, const int32_t* radii, uint32_t n, uint32_t T,
                                            uint32_t tiles_x, uint32_t tiles_y, uint32_t tiles_z, uint32_t* lo,
                                            uint32_t* hi) {
    return tile_box_3d(means_v + 3 * size_t(n), radii + 3 * size_t(n), T, tiles_x, tiles_y, tiles_z, lo, hi);
}

// What the tile VJP needs to find a record's slot, staged into the record's
// padding in shared memory by cp.async alongside the record (so the slot
// costs no dependent global round trip): the primitive's voxel radii (its
// tile box, with the record's voxel-space centre x, y, z) and its first slot
// cum[n - 1]. fp32 records have 16 bytes of padding, which hold the radii and
// the low 32 bits of cum[n - 1] (slots fit 31 bits, and a step whose count
// outgrew that is discarded); fp64 records have 32, and hold all 64 bits.
struct SlotPad {
    int32_t radius[3];
    uint32_t first32;  // fp32 records
    uint64_t first64;  // fp64 records
};
static_assert(sizeof(Rec3D<float>) - 12 * sizeof(float) >= offsetof(SlotPad, first64), "fp32 record padding");
static_assert(sizeof(Rec3D<double>) - 12 * sizeof(double) >= sizeof(SlotPad), "fp64 record padding");
template <typename S>
__device__ __forceinline__ SlotPad* slot_pad(Rec3D<S>* rec) {
    return reinterpret_cast<SlotPad*>(&rec->pad0);
}
template <typename S>
__device__ __forceinline__ const SlotPad* slot_pad(const Rec3D<S>* rec) {
    return reinterpret_cast<const SlotPad*>(&rec->pad0);
}

// Deterministic output of the tile VJP: instead of adding a (tile, primitive)
// pair's 12 sums into the primitive's adjoints with atomics, the pair writes
// them to a slot of its own, slot = cum[n - 1] + the tile's index in the
// primitive's tile box (z, then y, then x), and voxel_slot_reduce_kernel adds
// each primitive's slots in a fixed order. cum is the inclusive scan of the
// per-primitive tile counts, so the slots of the primitives are consecutive;
// slots past `capacity` (an overflowing capacity-bounded step, which is
// discarded) are not written.
template <typename S>
struct VoxelSlots {
    const S* means_v = nullptr;
    const int32_t* radii = nullptr;
    const int64_t* cum = nullptr;
    S* slots = nullptr;  // [capacity][12]; null: accumulate into grads with atomics
    uint64_t capacity = 0;
};

// Null-pointer conventions as in the rasterizer VJP: v_volume null = zero
// adjoint; v_volume_var null = no variance branch; chain_var false =
// detached variance branch.
//
// One warp per record over the record's box, one lane per box row (the box's
// voxels at one (y, z)), walking x with a warp-uniform trip count. Along a row
// d2 and d3 are fixed, so the quadratic form is a per-row constant plus a
// linear and a quadratic term in d1, and each lane keeps four row sums
// (sum w, sum w d1, sum w d1^2, sum g vis; plus the variance and Beta sums)
// that it folds into the record sums once per row. With g the volume adjoint
// (plus the variance chain term) and w = -g alpha (Gaussian) or the d^T Q d
// adjoint (Beta), the record sums are
//   S1..S3 = sum w d_i, Svis = sum g vis, S_ij = sum w d_i d_j (i <= j),
//   Sb = sum g alpha log h (Beta), Sq = sum v_var alpha^2 (variance),
// and the record's adjoints follow once per record: for a Gaussian
// x_i = -(Q d-sums)_i, i.e. x = -(c00 S1 + c01 S2 + c02 S3) and so on,
// c_ii = S_ii / 2, c_ij = S_ij, o = Svis; for a Beta x = 2 (Q d-sums)_i,
// c_ii = S_ii, c_ij = 2 S_ij, o = Svis, beta = Sb -- the reference's
// per-sample terms with the record's constants factored out. The factored
// quadratic form rounds differently from the reference's per-sample
// expression (by about an ulp); the VJP is held to a tolerance, and a
// contribution-threshold decision that flips moves a gradient by one
// threshold-sized sample at most.
// -(log2 e): exp(-s) = 2^(-s log2 e).
constexpr float kVoxNegLog2e = -1.4426950408889634f;

// Resident blocks the VJP is compiled for: the plain Gaussian walk is left to
// ptxas (60 registers, so four blocks of 46 KB shared memory fit an SM; a cap
// of 64 registers made it spill), the Beta and variance forms are held to
// three blocks, for which ptxas would otherwise use 80-120 registers and two.
template <bool kBeta, bool kVar>
constexpr int kVoxBwdMinBlocks = (kBeta || kVar) ? 3 : 0;

// kBulk: `records` is the per-tile packed copy whose padding holds each
// pair's slot (slot output only; flatten_ids unused), staged one bulk copy
// per batch.
template <typename S, bool kBeta, bool kVar, bool kBulk>
__global__ void __launch_bounds__(kVoxBwdThreads, kVoxBwdMinBlocks<kBeta, kVar>) voxel_bwd_kernel(
    const Rec3D<S>* __restrict__ records, bool chain_var, const int32_t* __restrict__ offsets,
    const int32_t* __restrict__ flatten_ids, VoxelGeom g, const S* __restrict__ v_volume,
    const S* __restrict__ v_volume_var, Rec3D<S>* __restrict__ grads, VoxelSlots<S> sl) {
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ uint64_t s_bar[2];
    const uint32_t T = g.T;
    const uint32_t tile_voxels = T * T * T;
    // The tile's adjoints are stored by rows of T voxels at a stride of T + 1,
    // so the lanes of a warp (one box row each) read distinct banks.
    const uint32_t RS = T + 1u;
    const uint32_t tile_slots = T * T * RS + RS;  // + one zero row read by idle lanes
    Rec3D<S>* s_rec = reinterpret_cast<Rec3D<S>*>(smem);                          // [2][threads]
    VoxelBox* s_box = reinterpret_cast<VoxelBox*>(s_rec + 2 * kVoxBwdThreads);     // [threads]
    S* s_v = reinterpret_cast<S*>(s_box + kVoxBwdThreads);                         // [T^2][T+1] adjoint
    S* s_vv = s_v + tile_slots;                                                    // [T^2][T+1] variance adjoint
    int32_t* s_id = reinterpret_cast<int32_t*>(s_vv + tile_slots);                 // [2][threads]
    uint32_t* s_slot = reinterpret_cast<uint32_t*>(s_id + 2 * kVoxBwdThreads);    // [2][threads] (slot output)

    const uint32_t n_tiles = g.tiles_x * g.tiles_y * g.tiles_z;
    const uint32_t key = blockIdx.x;
    const uint32_t tz = key / (g.tiles_x * g.tiles_y);
    const uint32_t rem = key - tz * g.tiles_x * g.tiles_y;
    const uint32_t ty = rem / g.tiles_x, tx = rem - ty * g.tiles_x;
    const uint32_t ox = tx * T, oy = ty * T, oz = tz * T;
    if (ox >= g.dim2 || oy >= g.dim1 || oz >= g.dim0) return;
    const uint32_t vx = min(T, g.dim2 - ox), vy = min(T, g.dim1 - oy), vz = min(T, g.dim0 - oz);
    const int32_t start = offsets[key];
    const int32_t n_total = g.n_dev != nullptr ? int32_t(*g.n_dev) : int32_t(g.n_isects);
    const int32_t end = (key + 1 == n_tiles) ? n_total : offsets[key + 1];
    const int32_t count = end - start;
    if (count <= 0) return;
    const uint32_t t = threadIdx.x, lane = t & 31u, warp = t >> 5;
    // The plain Gaussian VJP walks its rows two voxels per packed step.
    constexpr bool kPackedRow = std::is_same<S, float>::value && !kBeta && !kVar;

    for (uint32_t p = t; p < tile_voxels; p += kVoxBwdThreads) {
        const uint32_t lz = p / (T * T);
        const uint32_t r2 = p - lz * T * T;
        const uint32_t ly = r2 / T, lx = r2 - ly * T;
        const bool ok = lx < vx && ly < vy && lz < vz;
        const size_t vid = (size_t(oz + lz) * g.dim1 + (oy + ly)) * g.dim2 + (ox + lx);
        const uint32_t slot = (lz * T + ly) * RS + lx;
        s_v[slot] = (ok && v_volume != nullptr) ? v_volume[vid] : S(0);
        if (kVar) s_vv[slot] = ok ? v_volume_var[vid] : S(0);
    }
    // Row pads (x = T) and one zero row after the tile: the packed row walk
    // reads them without a bounds test.
    for (uint32_t p = t; p < T * T + RS; p += kVoxBwdThreads)
        s_v[p < T * T ? p * RS + T : T * T * RS + (p - T * T)] = S(0);

    const int32_t n_batches = (count + kVoxBwdThreads - 1) / kVoxBwdThreads;
    if (kBulk) {
        if (t == 0) {
            mbar_init(&s_bar[0], 1u);
            mbar_init(&s_bar[1], 1u);
            mbar_init_fence();
        }
        __syncthreads();
    }
    auto load = [&](int32_t b, uint32_t stage) {
        if constexpr (kBulk) {
            if (t == 0) {
                const int32_t first = start + b * kVoxBwdThreads;
                const uint32_t bytes = uint32_t(min(kVoxBwdThreads, end - first)) * uint32_t(sizeof(Rec3D<S>));
                fence_proxy_async_shared();
                mbar_arrive_expect_tx(&s_bar[stage], bytes);
                bulk_load_g2s(s_rec + stage * kVoxBwdThreads, records + first, bytes, &s_bar[stage]);
            }
            return;
        }
        const int32_t idx = start + b * kVoxBwdThreads + int32_t(t);
        if (idx < end) {
            const int32_t gid = flatten_ids[idx];
            Rec3D<S>* dst = s_rec + stage * kVoxBwdThreads + t;
            if (sl.slots == nullptr) {
                gather_record3(dst, records + gid);
            } else {
                // The record's 12 values, then the slot inputs into its padding.
                const char* src = reinterpret_cast<const char*>(records + gid);
#pragma unroll
                for (int k = 0; k < int(12 * sizeof(S) / 16); ++k)
                    cp_async16(reinterpret_cast<char*>(dst) + 16 * k, src + 16 * k);
                SlotPad* pad = slot_pad(dst);
#pragma unroll
                for (int k = 0; k < 3; ++k) cp_async4(pad->radius + k, sl.radii + 3 * size_t(gid) + k);
                if constexpr (sizeof(S) == 4) {
                    if (gid > 0) cp_async4(&pad->first32, sl.cum + (gid - 1));  // the low word
                    else pad->first32 = 0u;
                } else {
                    if (gid > 0) cp_async8(&pad->first64, sl.cum + (gid - 1));
                    else pad->first64 = 0u;
                }
            }
            s_id[stage * kVoxBwdThreads + t] = gid;
        }
        cp_async_commit();
    };
    load(0, 0);
    for (int32_t b = 0; b < n_batches; ++b) {
        if (b + 1 < n_batches) {
            load(b + 1, uint32_t(b + 1) & 1u);
            if (!kBulk) cp_async_wait<1>();
        } else if (!kBulk) {
            cp_async_wait<0>();
        }
        if (kBulk) {
            // Batch b is the (b / 2)-th use of its stage's barrier.
            const bool ok = mbar_wait_bounded(&s_bar[b & 1], uint32_t(b >> 1) & 1u);
            if (__syncthreads_or(!ok)) {
                if (t == 0) {
                    atomicAdd(&g_bulk_wait_faults, 1u);
                    mbar_wait_bounded(&s_bar[b & 1], uint32_t(b >> 1) & 1u);
                    if (b + 1 < n_batches) mbar_wait_bounded(&s_bar[(b + 1) & 1], uint32_t((b + 1) >> 1) & 1u);
                }
                __syncthreads();
                return;
            }
        } else {
            __syncthreads();
        }
        const uint32_t stage = uint32_t(b) & 1u;
        const int32_t batch = min(int32_t(kVoxBwdThreads), count - b * kVoxBwdThreads);
        if (int32_t(t) < batch) {
            s_box[t] = voxel_box<S, kBeta>(s_rec[stage * kVoxBwdThreads + t], ox, oy, oz, vx, vy, vz);
            if (kBulk) {
                // The pack kernel put the pair's slot (or 0xffffffff) in the padding.
                s_slot[stage * kVoxBwdThreads + t] =
                    *reinterpret_cast<const uint32_t*>(&s_rec[stage * kVoxBwdThreads + t].pad0);
            } else if (sl.slots != nullptr) {
                // The pair's slot: the primitive's first slot plus this tile's index in its tile box
                // (slots fit 31 bits).
                const Rec3D<S>& rec = s_rec[stage * kVoxBwdThreads + t];
                const SlotPad* pad = slot_pad(&rec);
                uint64_t first;
                if constexpr (sizeof(S) == 4) first = pad->first32;
                else first = pad->first64;
                uint32_t slot = 0xffffffffu;
                uint32_t blo[3], bhi[3];
                if (tile_box_3d(&rec.x, pad->radius, T, g.tiles_x, g.tiles_y, g.tiles_z, blo, bhi)) {
                    const uint64_t local = (uint64_t(tz - blo[2]) * (bhi[1] - blo[1]) + (ty - blo[1])) *
                                               (bhi[0] - blo[0]) + (tx - blo[0]);
                    const uint64_t j = first + local;
                    if (j < sl.capacity) slot = uint32_t(j);
                }
                s_slot[stage * kVoxBwdThreads + t] = slot;
            }
        }
        __syncthreads();
        for (int32_t s = int32_t(warp); s < batch; s += kVoxBwdWarps) {
            const VoxelBox box = s_box[s];
            const uint32_t w = box.extent & 0xffu, h = (box.extent >> 8) & 0xffu, d = (box.extent >> 16) & 0xffu;
            const uint32_t rows = h * d;
            const int32_t gid = kBulk ? 0 : s_id[stage * kVoxBwdThreads + s];
            // This pair's slot (deterministic output), written by the leaders of lane groups 0..2.
            const uint32_t slot = sl.slots != nullptr ? s_slot[stage * kVoxBwdThreads + s] : 0xffffffffu;
            if (rows * w == 0u) {
                if (slot != 0xffffffffu && (lane & 7u) == 0u && (lane >> 3) < 3u) {
                    S* out = sl.slots + size_t(slot) * 12u + 4u * (lane >> 3);
                    out[0] = out[1] = out[2] = out[3] = S(0);
                }
                continue;
            }
            const uint32_t x0 = box.origin & 0xffu, y0 = (box.origin >> 8) & 0xffu, z0 = (box.origin >> 16) & 0xffu;
            const Rec3D<S> r = s_rec[stage * kVoxBwdThreads + s];
            const S a = r.c00, p = r.c01, q = r.c02, bb = r.c11, rr = r.c12, c = r.c22;
            const S opac = r.o;
            const S uq = chain_var ? r.q : S(0);
            const S half_a = static_cast<S>(0.5) * a;
            // Packed rows: |alpha| < 1e-6 <=> 2^e < 1e-6 / |opac| <=> e < e_min.
            float e_min = 0.f;
            if constexpr (kPackedRow) e_min = log2f(1e-6f / fabsf(opac));
            const S px0 = static_cast<S>(ox + x0) + static_cast<S>(0.5);
            // part: S1, S2, S3, Svis | S11, S12, S13, S22 | S23, S33, Sb, Sq | unused
            S part[16];
#pragma unroll
            for (int i = 0; i < 16; ++i) part[i] = S(0);
            for (uint32_t r0 = 0; r0 < rows; r0 += 32u) {
                const uint32_t row = r0 + lane;
                const bool valid = row < rows;
                const uint32_t zz = valid ? (row * box.magic_h) >> 16 : 0u;
                const uint32_t yy = valid ? row - zz * h : 0u;
                const uint32_t p0 = ((z0 + zz) * T + (y0 + yy)) * RS + x0;
                const S py = static_cast<S>(oy + y0 + yy) + static_cast<S>(0.5);
                const S pz = static_cast<S>(oz + z0 + zz) + static_cast<S>(0.5);
                S d2, d3, K, L;
                if (!kBeta) {
                    d2 = py - r.y;
                    d3 = pz - r.z;
                    K = static_cast<S>(0.5) * (bb * d2 * d2 + c * d3 * d3) + rr * d2 * d3;
                    L = p * d2 + q * d3;
                } else {
                    d2 = r.y - py;
                    d3 = r.z - pz;
                    K = bb * d2 * d2 + c * d3 * d3 + static_cast<S>(2) * rr * d2 * d3;
                    L = static_cast<S>(2) * (p * d2 + q * d3);
                }
                S A0 = S(0), A1 = S(0), A2 = S(0), A3 = S(0), A4 = S(0), A5 = S(0);
                bool walked = false;
                if constexpr (kPackedRow) {
                    // Two voxels of the row per step (x and x + 1) in packed
                    // FP32x2 form. The exponent e = -sigma log2(e) comes from
                    // prescaled coefficients by Horner in d1, so vis = 2^e; a
                    // sample counts when e <= 0 (sigma >= 0) and e >= e_min
                    // (|alpha| >= 1e-6). With w = -g alpha = -opac g vis, the
                    // row sums carry g vis and are scaled by -opac once per row.
                    const float2 qa = splat2(half_a * kVoxNegLog2e), ql = splat2(L * kVoxNegLog2e);
                    const float2 qk = splat2(K * kVoxNegLog2e), two = splat2(2.f);
                    float2 d1 = make_float2(px0 - r.x, px0 + 1.f - r.x);
                    float2 a1 = splat2(0.f), a2 = a1, a3 = a1;
                    // Idle lanes read the zero row. With an odd width the second
                    // sample of the last step is the next voxel of the row (or
                    // the zero pad at x = T): it lies outside the record's box,
                    // so its contribution test fails like the reference's.
                    const uint32_t pz = valid ? p0 : T * T * RS;
                    for (uint32_t i = 0; i < w; i += 2u) {
                        const float ga = s_v[pz + i];
                        const float gb = s_v[pz + i + 1u];
                        const float2 e = fma2(fma2(qa, d1, ql), d1, qk);
                        const float2 vis = make_float2(exp2f(e.x), exp2f(e.y));
                        const bool ka = !(e.x > 0.f || e.x < e_min);
                        const bool kb = !(e.y > 0.f || e.y < e_min);
                        // Select after the product: a skipped sample may have vis = inf (e > 0).
                        const float2 gvr = mul2(make_float2(ga, gb), vis);
                        const float2 gv = make_float2(ka ? gvr.x : 0.f, kb ? gvr.y : 0.f);
                        a3 = add2(a3, gv);
                        const float2 gvd = mul2(gv, d1);
                        a1 = add2(a1, gvd);
                        a2 = fma2(gvd, d1, a2);
                        d1 = add2(d1, two);
                    }
                    A3 = a3.x + a3.y;
                    A0 = -opac * A3;
                    A1 = -opac * (a1.x + a1.y);
                    A2 = -opac * (a2.x + a2.y);
                    walked = true;
                }
                S px = px0;
                for (uint32_t i = 0; !walked && i < w; ++i, px += S(1)) {
                    S v = valid ? s_v[p0 + i] : S(0);
                    const S vv = (kVar && valid) ? s_vv[p0 + i] : S(0);
                    S wgt, d1;
                    if (!kBeta) {
                        d1 = px - r.x;
                        const S sigma = half_a * d1 * d1 + L * d1 + K;
                        const S vis_raw = exp(-sigma);
                        const S alpha_raw = opac * vis_raw;
                        const bool keep =
                            valid && !(sigma < static_cast<S>(0) || fabs(alpha_raw) < static_cast<S>(1e-6));
                        const S vis = keep ? vis_raw : S(0);
                        const S alpha = keep ? alpha_raw : S(0);
                        if (kVar) {
                            A4 += vv * alpha * alpha;
                            v += static_cast<S>(2) * uq * alpha * vv;
                        }
                        wgt = -v * alpha;
                        A3 += v * vis;
                    } else {
                        d1 = r.x - px;
                        const S qf = a * d1 * d1 + L * d1 + K;
                        const S h_raw = static_cast<S>(1) - qf;
                        const bool in_support = valid && !(qf < static_cast<S>(0) || h_raw <= static_cast<S>(0));
                        const S hh = in_support ? h_raw : S(1);  // keeps the logarithm finite on skipped samples
                        // hh^beta = 2^(beta log2 hh); log2 hh also gives ln hh and, with one
                        // division, hh^(beta - 1) = hh^beta / hh.
                        const S lg = log2(hh);
                        const S vis_raw = exp2(r.beta * lg);
                        const S alpha_raw = opac * vis_raw;
                        const bool keep = in_support && !(fabs(alpha_raw) < static_cast<S>(1e-5));
                        const S vis = keep ? vis_raw : S(0);
                        const S alpha = keep ? alpha_raw : S(0);
                        v = keep ? v : S(0);
                        if (kVar) {
                            A4 += vv * alpha * alpha;
                            v += static_cast<S>(2) * uq * alpha * vv;
                        }
                        wgt = -opac * r.beta * (vis_raw / hh) * v;
                        A3 += v * vis;
                        A5 += v * alpha * (lg * static_cast<S>(0.6931471805599453));  // ln hh = ln 2 log2 hh
                    }
                    const S wd = wgt * d1;
                    A0 += wgt;
                    A1 += wd;
                    A2 += wd * d1;
                }
                part[0] += A1;
                part[1] += d2 * A0;
                part[2] += d3 * A0;
                part[3] += A3;
                part[4] += A2;
                part[5] += d2 * A1;
                part[6] += d3 * A1;
                part[7] += d2 * d2 * A0;
                part[8] += d2 * d3 * A0;
                part[9] += d3 * d3 * A0;
                part[10] += A5;
                part[11] += A4;
            }
            // Recursive halving: 16 -> 8 (lane bit 4) -> 4 (bit 3) values, then
            // a butterfly over lane bits 2..0; lane group G = lane / 8 ends with
            // the warp totals of part[4G .. 4G+3].
            const bool hi16 = (lane & 16u) != 0, hi8 = (lane & 8u) != 0;
            S w8[8];
#pragma unroll
            for (int i = 0; i < 8; ++i) {
                const S send = hi16 ? part[i] : part[i + 8];
                const S keep = hi16 ? part[i + 8] : part[i];
                w8[i] = keep + __shfl_xor_sync(0xffffffffu, send, 16);
            }
            S w4[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                const S send = hi8 ? w8[i] : w8[i + 4];
                const S keep = hi8 ? w8[i + 4] : w8[i];
                w4[i] = keep + __shfl_xor_sync(0xffffffffu, send, 8);
            }
#pragma unroll
            for (int offset = 4; offset > 0; offset >>= 1) {
#pragma unroll
                for (int i = 0; i < 4; ++i) w4[i] += __shfl_xor_sync(0xffffffffu, w4[i], offset);
            }
            const uint32_t grp = lane >> 3;
            if ((lane & 7u) == 0u && grp < 3u) {
                const S two = static_cast<S>(2), half = static_cast<S>(0.5);
                S e0, e1, e2, e3;
                if (grp == 0u) {
                    const S sx = a * w4[0] + p * w4[1] + q * w4[2];
                    const S sy = bb * w4[1] + p * w4[0] + rr * w4[2];
                    const S sz = c * w4[2] + q * w4[0] + rr * w4[1];
                    e0 = kBeta ? two * sx : -sx;
                    e1 = kBeta ? two * sy : -sy;
                    e2 = kBeta ? two * sz : -sz;
                    e3 = w4[3];
                } else if (grp == 1u) {
                    e0 = kBeta ? w4[0] : half * w4[0];
                    e1 = kBeta ? two * w4[1] : w4[1];
                    e2 = kBeta ? two * w4[2] : w4[2];
                    e3 = kBeta ? w4[3] : half * w4[3];
                } else {
                    e0 = kBeta ? two * w4[0] : w4[0];
                    e1 = kBeta ? w4[1] : half * w4[1];
                    e2 = w4[2];
                    e3 = w4[3];
                }
                if (!kBulk && sl.slots == nullptr) {
                    red_add_v4(reinterpret_cast<S*>(grads + gid) + 4 * grp, e0, e1, e2, e3);
                } else if (slot != 0xffffffffu && grp < 3u) {
                    S* out = sl.slots + size_t(slot) * 12u + 4u * grp;
                    out[0] = e0;
                    out[1] = e1;
                    out[2] = e2;
                    out[3] = e3;
                }
            }
        }
        __syncthreads();
    }
}

// grads[n] = the sum of primitive n's slots (12 sums), zero pads. Four lanes
// share a primitive: lane q sums slots q, q + 4, ... in order, and the four
// partial sums are combined by a fixed butterfly ((s0 + s1) + (s2 + s3)), so
// the result does not depend on scheduling. Lane q then writes quarter q of
// the primitive's 16-value entry.
constexpr uint32_t kSlotLanes = 4u;
template <typename S>
__global__ void voxel_slot_reduce_kernel(const S* __restrict__ slots, const int64_t* __restrict__ cum, uint32_t N,
                                         int64_t capacity, Rec3D<S>* __restrict__ grads) {
    const uint64_t t = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    const uint32_t q = uint32_t(t) & (kSlotLanes - 1u);
    const uint64_t n = t / kSlotLanes;
    if ((t & ~uint64_t(31)) / kSlotLanes >= N) return;  // warp-uniform: the warp holds no primitive
    const bool active = n < N;
    int64_t first = 0, last = 0;
    if (active) {
        first = n == 0u ? 0 : min(cum[n - 1], capacity);
        last = min(cum[n], capacity);
    }
    S acc[12];
#pragma unroll
    for (int i = 0; i < 12; ++i) acc[i] = S(0);
    for (int64_t j = first + q; j < last; j += kSlotLanes) {
        if constexpr (sizeof(S) == 4) {
            // A slot is 48 bytes, 16-byte aligned: three vector loads.
            const float4* p = reinterpret_cast<const float4*>(slots + size_t(j) * 12u);
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                const float4 v = __ldg(p + k);
                acc[4 * k] += v.x;
                acc[4 * k + 1] += v.y;
                acc[4 * k + 2] += v.z;
                acc[4 * k + 3] += v.w;
            }
        } else {
            const S* p = slots + size_t(j) * 12u;
#pragma unroll
            for (int i = 0; i < 12; ++i) acc[i] += p[i];
        }
    }
#pragma unroll
    for (uint32_t offset = 1u; offset < kSlotLanes; offset <<= 1) {
#pragma unroll
        for (int i = 0; i < 12; ++i) acc[i] += __shfl_xor_sync(0xffffffffu, acc[i], offset);
    }
    if (!active) return;
    S* out = reinterpret_cast<S*>(grads + n) + 4u * q;
#pragma unroll
    for (int i = 0; i < 4; ++i) out[i] = q == 0u ? acc[i] : q == 1u ? acc[4 + i] : q == 2u ? acc[8 + i] : S(0);
}

// Tile VJP of fp32 Gaussian records on 8^3 tiles without the variance branch
// (the CT fit step's form), one lane per (tile, primitive) pair. The warp
// walks the tile's 512 voxels in lockstep, z, then pairs of rows, then x; the
// voxel is the same for every lane, so its adjoint is one broadcast shared-
// memory read for 32 records, and each lane sums its own record's moments
// serially: no per-pair reduction across lanes, no box set-up. The whole tile
// is walked: a voxel outside the record's conservative box fails the
// contribution test (zero adjoint outside the volume), as every sample the
// reference skips does. The two samples of a packed step are two adjacent rows
// at the same x, so d1 and the record's x terms are shared and the row terms
// come as pairs. With the exponent e = -sigma log2(e) = qa d1^2 + ql d1 + qk
// (conic prescaled by -log2(e); ql and qk per row from d2 and d3), a sample
// counts when e <= 0 and e >= log2(1e-6 / |o|), as in voxel_bwd_kernel, and
// adds g vis, g vis d1 and g vis d1^2 to the row sums. A pair of rows folds
// them with its d2 values, a z slab with its d3; the record's sums are then
// the ones voxel_bwd_kernel forms (w = -o g vis), and the 12 values written
// per pair are the same quantities in the same layout.
constexpr int kVoxLaneWarps = 4;
constexpr int kVoxLaneThreads = kVoxLaneWarps * 32;

template <bool kBulk>
__global__ void __launch_bounds__(kVoxLaneThreads, 6) voxel_bwd_lanes_kernel(
    const Rec3D<float>* __restrict__ records, const int32_t* __restrict__ offsets,
    const int32_t* __restrict__ flatten_ids, VoxelGeom g, const float* __restrict__ v_volume,
    Rec3D<float>* __restrict__ grads, VoxelSlots<float> sl) {
    constexpr uint32_t T = 8u;
    // The tile's adjoint as row pairs: s_g[(z * 4 + yp) * 8 + x] = (g(z, 2 yp, x), g(z, 2 yp + 1, x)).
    __shared__ float2 s_g[T * T * T / 2];
    const uint32_t n_tiles = g.tiles_x * g.tiles_y * g.tiles_z;
    const uint32_t key = blockIdx.x;
    const uint32_t tz = key / (g.tiles_x * g.tiles_y);
    const uint32_t rem = key - tz * g.tiles_x * g.tiles_y;
    const uint32_t ty = rem / g.tiles_x, tx = rem - ty * g.tiles_x;
    const uint32_t ox = tx * T, oy = ty * T, oz = tz * T;
    if (ox >= g.dim2 || oy >= g.dim1 || oz >= g.dim0) return;
    const uint32_t vx = min(T, g.dim2 - ox), vy = min(T, g.dim1 - oy), vz = min(T, g.dim0 - oz);
    const int32_t start = offsets[key];
    const int32_t n_total = g.n_dev != nullptr ? int32_t(*g.n_dev) : int32_t(g.n_isects);
    const int32_t end = (key + 1 == n_tiles) ? n_total : offsets[key + 1];
    const int32_t count = end - start;
    if (count <= 0) return;
    const uint32_t t = threadIdx.x, lane = t & 31u, warp = t >> 5;
    for (uint32_t p = t; p < T * T * T / 2; p += kVoxLaneThreads) {
        const uint32_t x = p & 7u, yp = (p >> 3) & 3u, z = p >> 5;
        float ga = 0.f, gb = 0.f;
        if (v_volume != nullptr && x < vx && z < vz) {
            const size_t vid = (size_t(oz + z) * g.dim1 + (oy + 2u * yp)) * g.dim2 + (ox + x);
            if (2u * yp < vy) ga = v_volume[vid];
            if (2u * yp + 1u < vy) gb = v_volume[vid + g.dim2];
        }
        s_g[p] = make_float2(ga, gb);
    }
    __syncthreads();

    const float fx = static_cast<float>(ox) + 0.5f, fy = static_cast<float>(oy) + 0.5f;
    const float fz = static_cast<float>(oz) + 0.5f;
    const int32_t n_chunks = (count + 31) / 32;
    for (int32_t chunk = int32_t(warp); chunk < n_chunks; chunk += kVoxLaneWarps) {
        const int32_t idx = start + chunk * 32 + int32_t(lane);
        const bool active = idx < end;
        // Idle lanes walk a record with o = 0, whose threshold rejects every sample.
        const Rec3D<float>* rp = nullptr;
        int32_t gid = 0;
        uint32_t slot = 0xffffffffu;
        if (active) {
            if constexpr (kBulk) {
                rp = records + idx;
                slot = __float_as_uint(__ldg(&rp->pad0));  // the pack kernel's slot (or 0xffffffff)
            } else {
                gid = flatten_ids[idx];
                rp = records + gid;
                if (sl.slots != nullptr) {
                    const uint64_t first = gid > 0 ? uint64_t(sl.cum[gid - 1]) : 0u;
                    const float mv[3] = {__ldg(&rp->x), __ldg(&rp->y), __ldg(&rp->z)};
                    uint32_t blo[3], bhi[3];
                    if (tile_box_3d(mv, sl.radii + 3 * size_t(gid), T, g.tiles_x, g.tiles_y, g.tiles_z, blo, bhi)) {
                        const uint64_t local = (uint64_t(tz - blo[2]) * (bhi[1] - blo[1]) + (ty - blo[1])) *
                                                   (bhi[0] - blo[0]) + (tx - blo[0]);
                        if (first + local < sl.capacity) slot = uint32_t(first + local);
                    }
                }
            }
        }
        float4 q0 = make_float4(0.f, 0.f, 0.f, 0.f), q1 = q0, q2 = q0;  // (x, y, z, o), (c00, c01, c02, c11), (c12, c22, ..)
        if (active) {
            const float4* r4 = reinterpret_cast<const float4*>(rp);
            q0 = __ldg(r4);
            q1 = __ldg(r4 + 1);
            q2 = __ldg(r4 + 2);
        }
        const float ry = q0.y, rz = q0.z, opac = q0.w;
        const float e_min = log2f(1e-6f / fabsf(opac));
        const float2 qa = splat2(0.5f * q1.x * kVoxNegLog2e);
        const float pl = q1.y * kVoxNegLog2e, ql3 = q1.z * kVoxNegLog2e;
        const float hb = 0.5f * q1.w * kVoxNegLog2e, rl = q2.x * kVoxNegLog2e, hc = 0.5f * q2.y * kVoxNegLog2e;
        const float2 d1_0 = splat2(fx - q0.x), one = splat2(1.f);
        // Record sums: g vis d1^2, g vis d2^2, g vis d1 d2 (packed over the row pair),
        // then g vis, g vis d1, g vis d2 and the d3 moments.
        float2 r11 = splat2(0.f), r22 = r11, r12 = r11;
        float s0 = 0.f, s1 = 0.f, s2 = 0.f, s3 = 0.f, s13 = 0.f, s23 = 0.f, s33 = 0.f;
        for (uint32_t z = 0; z < T; ++z) {
            const float d3 = (fz + static_cast<float>(z)) - rz;
            const float qd3 = ql3 * d3, rd3 = rl * d3, cd3 = hc * d3 * d3;
            float2 z0 = splat2(0.f), z1 = z0, z2 = z0;
            const float2* gz = s_g + z * (T * T / 2);
#pragma unroll 1
            for (uint32_t yp = 0; yp < T / 2; ++yp) {
                const float fyp = fy + static_cast<float>(2u * yp);
                const float2 d2 = make_float2(fyp - ry, (fyp + 1.f) - ry);
                const float2 ql = make_float2(fmaf(pl, d2.x, qd3), fmaf(pl, d2.y, qd3));
                const float2 qk = make_float2(fmaf(hb * d2.x, d2.x, fmaf(rd3, d2.x, cd3)),
                                              fmaf(hb * d2.y, d2.y, fmaf(rd3, d2.y, cd3)));
                float2 a1 = splat2(0.f), a2 = a1, a3 = a1;
                float2 d1 = d1_0;
#pragma unroll
                for (uint32_t x = 0; x < T; ++x) {
                    const float2 gg = gz[yp * T + x];
                    const float2 e = fma2(fma2(qa, d1, ql), d1, qk);
                    const float2 vis = make_float2(exp2f(e.x), exp2f(e.y));
                    const bool ka = !(e.x > 0.f || e.x < e_min);
                    const bool kb = !(e.y > 0.f || e.y < e_min);
                    // Select after the product: a skipped sample may have vis = inf (e > 0).
                    const float2 gvr = mul2(gg, vis);
                    const float2 gv = make_float2(ka ? gvr.x : 0.f, kb ? gvr.y : 0.f);
                    a3 = add2(a3, gv);
                    const float2 gvd = mul2(gv, d1);
                    a1 = add2(a1, gvd);
                    a2 = fma2(gvd, d1, a2);
                    d1 = add2(d1, one);
                }
                z0 = add2(z0, a3);
                z1 = add2(z1, a1);
                r11 = add2(r11, a2);
                const float2 gd2 = mul2(d2, a3);
                z2 = add2(z2, gd2);
                r22 = fma2(d2, gd2, r22);
                r12 = fma2(d2, a1, r12);
            }
            const float g0 = z0.x + z0.y, g1 = z1.x + z1.y, g2 = z2.x + z2.y;
            s0 += g0;
            s1 += g1;
            s2 += g2;
            s3 = fmaf(d3, g0, s3);
            s13 = fmaf(d3, g1, s13);
            s23 = fmaf(d3, g2, s23);
            s33 = fmaf(d3 * d3, g0, s33);
        }
        if (!active) continue;
        const float nom = -opac;
        const float S1 = nom * s1, S2 = nom * s2, S3 = nom * s3;
        const float S11 = nom * (r11.x + r11.y), S12 = nom * (r12.x + r12.y), S13 = nom * s13;
        const float S22 = nom * (r22.x + r22.y), S23 = nom * s23, S33 = nom * s33;
        // The conic again (read once more rather than held through the walk).
        const float4 c4 = __ldg(reinterpret_cast<const float4*>(rp) + 1);
        const float a = c4.x, p = c4.y, q = c4.z, bb = c4.w, rr = __ldg(&rp->c12), c = __ldg(&rp->c22);
        const float4 o0 = make_float4(-(a * S1 + p * S2 + q * S3), -(bb * S2 + p * S1 + rr * S3),
                                      -(c * S3 + q * S1 + rr * S2), s0);
        const float4 o1 = make_float4(0.5f * S11, S12, S13, 0.5f * S22);
        const float4 o2 = make_float4(S23, 0.5f * S33, 0.f, 0.f);
        if (!kBulk && sl.slots == nullptr) {
            float* out = reinterpret_cast<float*>(grads + gid);
            red_add_v4(out, o0.x, o0.y, o0.z, o0.w);
            red_add_v4(out + 4, o1.x, o1.y, o1.z, o1.w);
            red_add_v4(out + 8, o2.x, o2.y, o2.z, o2.w);
        } else if (slot != 0xffffffffu) {
            float4* out = reinterpret_cast<float4*>(sl.slots + size_t(slot) * 12u);
            out[0] = o0;
            out[1] = o1;
            out[2] = o2;
        }
    }
}

// ---------------------------------------------------------------------------
// Record-parallel voxel VJP (the explicit path).
//
// The reference's VJP is tile-parallel with atomics (VoxelizeToVoxelsBwd.cu:
// 322-514): every (tile, primitive) pair of the sorted lists adds its sums into
// the primitive's adjoints. Here the work is split by primitive instead: a
// work item is one primitive and one z-layer of its tile box (the box of
// tiles its list entries cover: the tile span of IsectTiles3DKernel.cu:38-112,
// one layer = tile_size voxel slices), and one warp walks the item's voxels of
// the primitive's conservative box, reading the volume adjoint from global
// memory (L2). Items of a primitive are numbered consecutively (an inclusive
// scan of the per-primitive layer counts), each writes its 12 sums to its own
// slot, and voxel_record_reduce_kernel adds a primitive's slots in layer
// order. No atomics, no sorted lists, and the result is the same bit for bit
// on every run and in every batch. The evaluated samples are the reference's:
// the union of a primitive's tiles is its tile box, and every sample outside
// the conservative box fails the contribution test.
// ---------------------------------------------------------------------------

struct VoxelRecordGeom {
    uint32_t N, dim2, dim1, dim0, T, tiles_x, tiles_y, tiles_z;
    uint64_t n_items;                 // item count, or the capacity when n_items_dev is set
    const int64_t* n_items_dev;       // device-side item count (capacity-bounded launches), or null
};

// Layers of a primitive's 3D tile box (0 when it has no tiles).
template <typename S>
__device__ __forceinline__ uint32_t record_tile_box(const S* means_v, const int32_t* radii, uint32_t n,
                                                    const VoxelRecordGeom& g, uint32_t* lo, uint32_t* hi) {
    const int32_t rx = radii[3 * size_t(n)], ry = radii[3 * size_t(n) + 1], rz = radii[3 * size_t(n) + 2];
    if (rx <= 0 || ry <= 0 || rz <= 0) return 0u;
    tile_span(means_v[3 * size_t(n)], static_cast<S>(rx), g.T, g.tiles_x, lo[0], hi[0]);
    tile_span(means_v[3 * size_t(n) + 1], static_cast<S>(ry), g.T, g.tiles_y, lo[1], hi[1]);
    tile_span(means_v[3 * size_t(n) + 2], static_cast<S>(rz), g.T, g.tiles_z, lo[2], hi[2]);
    if (!(hi[0] > lo[0] && hi[1] > lo[1] && hi[2] > lo[2])) return 0u;
    return hi[2] - lo[2];
}

template <typename S>
__global__ void voxel_layer_count_kernel(const S* __restrict__ means_v, const int32_t* __restrict__ radii,
                                         VoxelRecordGeom g, int32_t* __restrict__ layers) {
    const uint32_t n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= g.N) return;
    uint32_t lo[3], hi[3];
    layers[n] = static_cast<int32_t>(record_tile_box(means_v, radii, n, g, lo, hi));
}

// Rows of an item are walked 32 at a time (one per lane) in chunks of up to 32
// voxels along x. Each chunk's adjoints are first copied by the warp from
// global memory into a per-warp shared tile [32 rows][33] with coalesced loads
// (one row's chunk per load instruction), then each lane walks its row from
// shared memory as the tile kernel does. Unloaded slots (past the chunk, idle
// rows) hold zero adjoints.
constexpr uint32_t kRecChunk = 32u, kRecStride = kRecChunk + 1u;

template <typename S, bool kBeta, bool kVar>
__global__ void __launch_bounds__(kVoxBwdThreads) voxel_record_bwd_kernel(
    const Rec3D<S>* __restrict__ records, const S* __restrict__ means_v, const int32_t* __restrict__ radii,
    const int64_t* __restrict__ item_cum, bool chain_var, VoxelRecordGeom g, const S* __restrict__ v_volume,
    const S* __restrict__ v_volume_var, Rec3D<S>* __restrict__ partials) {
    extern __shared__ __align__(16) unsigned char smem[];
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    S* s_v = reinterpret_cast<S*>(smem) + size_t(warp) * 32u * kRecStride * (kVar ? 2u : 1u);
    S* s_vv = s_v + 32u * kRecStride;  // used with the variance branch only
    uint64_t n_items = g.n_items;
    if (g.n_items_dev != nullptr) {
        const uint64_t used = uint64_t(*g.n_items_dev);
        n_items = used < n_items ? used : n_items;  // past the capacity the step is flagged and skipped
    }
    // Each warp takes a contiguous run of items, so it finds its first primitive once by binary search
    // and then steps through the primitives in order.
    const uint64_t warps = uint64_t(gridDim.x) * kVoxBwdWarps;
    const uint64_t gw = uint64_t(blockIdx.x) * kVoxBwdWarps + warp;
    const uint64_t per = (n_items + warps - 1) / warps;
    const uint64_t i0 = gw * per, i1 = min(n_items, i0 + per);
    if (i0 >= i1) return;
    uint32_t n;
    {
        uint32_t lo_n = 0u, hi_n = g.N;
        while (lo_n < hi_n) {
            const uint32_t mid = (lo_n + hi_n) >> 1;
            if (uint64_t(item_cum[mid]) > i0) hi_n = mid; else lo_n = mid + 1u;
        }
        n = lo_n;
    }
    constexpr bool kPackedRow = std::is_same<S, float>::value && !kBeta && !kVar;
    const uint32_t T = g.T;
    const bool has_v = v_volume != nullptr;
    for (uint64_t item = i0; item < i1; ++item) {
        while (n < g.N && uint64_t(item_cum[n]) <= item) ++n;  // warp-uniform
        if (n >= g.N) break;                                    // cannot happen while n_items <= item_cum[N - 1]
        S part[16];
#pragma unroll
        for (int i = 0; i < 16; ++i) part[i] = S(0);
        const Rec3D<S> r = records[n];
        uint32_t tlo[3], thi[3];
        const uint32_t layers = record_tile_box(means_v, radii, n, g, tlo, thi);
        const uint64_t first = n == 0u ? 0u : uint64_t(item_cum[n - 1]);
        uint32_t blo[3], bhi[3];
        bool any = layers > 0u && item - first < layers;
        uint32_t ox = 0u, oy = 0u, oz = 0u;
        if (any) {
            const uint32_t layer = tlo[2] + uint32_t(item - first);
            ox = tlo[0] * T;
            oy = tlo[1] * T;
            oz = layer * T;
            const uint32_t vx = min(thi[0] * T, g.dim2) - ox;
            const uint32_t vy = min(thi[1] * T, g.dim1) - oy;
            const uint32_t vz = min(oz + T, g.dim0) - oz;
            any = voxel_box_bounds<S, kBeta>(r, ox, oy, oz, vx, vy, vz, blo, bhi);
        }
        if (any) {
            const uint32_t x0 = blo[0], y0 = blo[1], z0 = blo[2];
            const uint32_t w = bhi[0] - x0 + 1u, h = bhi[1] - y0 + 1u, d = bhi[2] - z0 + 1u;
            const uint32_t rows = h * d;
            const S a = r.c00, p = r.c01, q = r.c02, bb = r.c11, rr = r.c12, c = r.c22;
            const S opac = r.o;
            const S uq = chain_var ? r.q : S(0);
            const S half_a = static_cast<S>(0.5) * a;
            float e_min = 0.f;
            if constexpr (kPackedRow) e_min = log2f(1e-6f / fabsf(opac));
            const size_t item_base = (size_t(oz + z0) * g.dim1 + (oy + y0)) * g.dim2 + (ox + x0);
            const uint32_t plane = g.dim1 * g.dim2;
            for (uint32_t r0 = 0; r0 < rows; r0 += 32u) {
                const uint32_t row = r0 + lane;
                const bool valid = row < rows;
                const uint32_t zz = valid ? row / h : 0u;
                const uint32_t yy = valid ? row - zz * h : 0u;
                // Offset of this lane's row from the item's first voxel (fits 32 bits: z < tile_size).
                const uint32_t row_off = valid ? zz * plane + yy * g.dim2 : 0xffffffffu;
                const uint32_t n_rows = min(32u, rows - r0);
                const S py = static_cast<S>(oy + y0 + yy) + static_cast<S>(0.5);
                const S pz = static_cast<S>(oz + z0 + zz) + static_cast<S>(0.5);
                S d2, d3, K, L;
                if (!kBeta) {
                    d2 = py - r.y;
                    d3 = pz - r.z;
                    K = static_cast<S>(0.5) * (bb * d2 * d2 + c * d3 * d3) + rr * d2 * d3;
                    L = p * d2 + q * d3;
                } else {
                    d2 = r.y - py;
                    d3 = r.z - pz;
                    K = bb * d2 * d2 + c * d3 * d3 + static_cast<S>(2) * rr * d2 * d3;
                    L = static_cast<S>(2) * (p * d2 + q * d3);
                }
                S A0 = S(0), A1 = S(0), A2 = S(0), A3 = S(0), A4 = S(0), A5 = S(0);
                float2 a1 = splat2(0.f), a2 = a1, a3 = a1;
                for (uint32_t xs = 0; xs < w; xs += kRecChunk) {
                    const uint32_t cols = min(kRecChunk, w - xs);
                    // Stage: lane = column; one row of the chunk per iteration.
                    __syncwarp();
                    for (uint32_t k = 0; k < 32u; ++k) {
                        const uint32_t off = __shfl_sync(0xffffffffu, row_off, int(k));
                        const bool load = k < n_rows && lane < cols;
                        const size_t gi = item_base + off + xs + lane;
                        s_v[k * kRecStride + lane] = (load && has_v) ? v_volume[gi] : S(0);
                        if (kVar) s_vv[k * kRecStride + lane] = load ? v_volume_var[gi] : S(0);
                    }
                    if (lane == 0u) {
                        for (uint32_t k = 0; k < 32u; ++k) {
                            s_v[k * kRecStride + kRecChunk] = S(0);
                            if (kVar) s_vv[k * kRecStride + kRecChunk] = S(0);
                        }
                    }
                    __syncwarp();
                    const S* vrow = s_v + lane * kRecStride;
                    const S px0 = static_cast<S>(ox + x0 + xs) + static_cast<S>(0.5);
                    if constexpr (kPackedRow) {
                        // Two voxels of the row per step in packed FP32x2 form, as in the tile kernel:
                        // e = -sigma log2(e) by Horner in d1 from prescaled coefficients, vis = 2^e.
                        const float2 qa = splat2(half_a * kVoxNegLog2e), ql = splat2(L * kVoxNegLog2e);
                        const float2 qk = splat2(K * kVoxNegLog2e), two = splat2(2.f);
                        float2 d1 = make_float2(px0 - r.x, px0 + 1.f - r.x);
                        for (uint32_t i = 0; i < cols; i += 2u) {
                            // Slots past the chunk are zero: the odd tail's second sample adds nothing.
                            const float ga = vrow[i];
                            const float gb = vrow[i + 1u];
                            const float2 e = fma2(fma2(qa, d1, ql), d1, qk);
                            const float2 vis = make_float2(exp2f(e.x), exp2f(e.y));
                            const bool ka = !(e.x > 0.f || e.x < e_min);
                            const bool kb = !(e.y > 0.f || e.y < e_min);
                            const float2 gvr = mul2(make_float2(ga, gb), vis);
                            const float2 gv = make_float2(ka ? gvr.x : 0.f, kb ? gvr.y : 0.f);
                            a3 = add2(a3, gv);
                            const float2 gvd = mul2(gv, d1);
                            a1 = add2(a1, gvd);
                            a2 = fma2(gvd, d1, a2);
                            d1 = add2(d1, two);
                        }
                    } else {
                        S px = px0;
                        for (uint32_t i = 0; i < cols; ++i, px += S(1)) {
                            S v = vrow[i];
                            const S vv = kVar ? s_vv[lane * kRecStride + i] : S(0);
                            S wgt, d1;
                            if (!kBeta) {
                                d1 = px - r.x;
                                const S sigma = half_a * d1 * d1 + L * d1 + K;
                                const S vis_raw = exp(-sigma);
                                const S alpha_raw = opac * vis_raw;
                                const bool keep = valid &&
                                                  !(sigma < static_cast<S>(0) || fabs(alpha_raw) < static_cast<S>(1e-6));
                                const S vis = keep ? vis_raw : S(0);
                                const S alpha = keep ? alpha_raw : S(0);
                                if (kVar) {
                                    A4 += vv * alpha * alpha;
                                    v += static_cast<S>(2) * uq * alpha * vv;
                                }
                                wgt = -v * alpha;
                                A3 += v * vis;
                            } else {
                                d1 = r.x - px;
                                const S qf = a * d1 * d1 + L * d1 + K;
                                const S h_raw = static_cast<S>(1) - qf;
                                const bool in_support =
                                    valid && !(qf < static_cast<S>(0) || h_raw <= static_cast<S>(0));
                                const S hh = in_support ? h_raw : S(1);
                                const S lg = log2(hh);
                                const S vis_raw = exp2(r.beta * lg);
                                const S alpha_raw = opac * vis_raw;
                                const bool keep = in_support && !(fabs(alpha_raw) < static_cast<S>(1e-5));
                                const S vis = keep ? vis_raw : S(0);
                                const S alpha = keep ? alpha_raw : S(0);
                                v = keep ? v : S(0);
                                if (kVar) {
                                    A4 += vv * alpha * alpha;
                                    v += static_cast<S>(2) * uq * alpha * vv;
                                }
                                wgt = -opac * r.beta * (vis_raw / hh) * v;
                                A3 += v * vis;
                                A5 += v * alpha * (lg * static_cast<S>(0.6931471805599453));
                            }
                            const S wd = wgt * d1;
                            A0 += wgt;
                            A1 += wd;
                            A2 += wd * d1;
                        }
                    }
                }
                if constexpr (kPackedRow) {
                    A3 = a3.x + a3.y;
                    A0 = -opac * A3;
                    A1 = -opac * (a1.x + a1.y);
                    A2 = -opac * (a2.x + a2.y);
                }
                part[0] += A1;
                part[1] += d2 * A0;
                part[2] += d3 * A0;
                part[3] += A3;
                part[4] += A2;
                part[5] += d2 * A1;
                part[6] += d3 * A1;
                part[7] += d2 * d2 * A0;
                part[8] += d2 * d3 * A0;
                part[9] += d3 * d3 * A0;
                part[10] += A5;
                part[11] += A4;
            }
        }
        // Recursive halving as in the tile kernel; lane group G = lane / 8 ends with the warp totals of
        // part[4G .. 4G+3].
        const bool hi16 = (lane & 16u) != 0, hi8 = (lane & 8u) != 0;
        S w8[8];
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            const S send = hi16 ? part[i] : part[i + 8];
            const S keep = hi16 ? part[i + 8] : part[i];
            w8[i] = keep + __shfl_xor_sync(0xffffffffu, send, 16);
        }
        S w4[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const S send = hi8 ? w8[i] : w8[i + 4];
            const S keep = hi8 ? w8[i + 4] : w8[i];
            w4[i] = keep + __shfl_xor_sync(0xffffffffu, send, 8);
        }
#pragma unroll
        for (int offset = 4; offset > 0; offset >>= 1) {
#pragma unroll
            for (int i = 0; i < 4; ++i) w4[i] += __shfl_xor_sync(0xffffffffu, w4[i], offset);
        }
        const uint32_t grp = lane >> 3;
        if ((lane & 7u) == 0u) {
            const S a = r.c00, p = r.c01, q = r.c02, bb = r.c11, rr = r.c12, c = r.c22;
            const S two = static_cast<S>(2), half = static_cast<S>(0.5);
            S e0 = S(0), e1 = S(0), e2 = S(0), e3 = S(0);
            if (grp == 0u) {
                const S sx = a * w4[0] + p * w4[1] + q * w4[2];
                const S sy = bb * w4[1] + p * w4[0] + rr * w4[2];
                const S sz = c * w4[2] + q * w4[0] + rr * w4[1];
                e0 = kBeta ? two * sx : -sx;
                e1 = kBeta ? two * sy : -sy;
                e2 = kBeta ? two * sz : -sz;
                e3 = w4[3];
            } else if (grp == 1u) {
                e0 = kBeta ? w4[0] : half * w4[0];
                e1 = kBeta ? two * w4[1] : w4[1];
                e2 = kBeta ? two * w4[2] : w4[2];
                e3 = kBeta ? w4[3] : half * w4[3];
            } else if (grp == 2u) {
                e0 = kBeta ? two * w4[0] : w4[0];
                e1 = kBeta ? w4[1] : half * w4[1];
                e2 = w4[2];
                e3 = w4[3];
            }
            S* out = reinterpret_cast<S*>(partials + item) + 4 * grp;
            out[0] = e0;
            out[1] = e1;
            out[2] = e2;
            out[3] = e3;
        }
    }
}

// grads[n] = sum of the primitive's item slots, in layer order.
template <typename S>
__global__ void voxel_record_reduce_kernel(const Rec3D<S>* __restrict__ partials,
                                           const int64_t* __restrict__ item_cum, uint32_t N, int64_t capacity,
                                           Rec3D<S>* __restrict__ grads) {
    const uint32_t n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= N) return;
    // Slots past the capacity were not computed (that step is flagged); they are never read.
    const int64_t first = n == 0u ? 0 : min(item_cum[n - 1], capacity), last = min(item_cum[n], capacity);
    S acc[12];
#pragma unroll
    for (int i = 0; i < 12; ++i) acc[i] = S(0);
    for (int64_t item = first; item < last; ++item) {
        const S* p = reinterpret_cast<const S*>(partials + item);
#pragma unroll
        for (int i = 0; i < 12; ++i) acc[i] += p[i];
    }
    S* out = reinterpret_cast<S*>(grads + n);
#pragma unroll
    for (int i = 0; i < 12; ++i) out[i] = acc[i];
#pragma unroll
    for (int i = 12; i < 16; ++i) out[i] = S(0);
}

// Per-tile packed copy of the 3D records for the explicit and batched
// pipelines: packed[i] = records[flatten_ids[i]] for each sorted intersection
// i, so the records of a tile's list are one contiguous range, staged by one
// bulk copy per batch in the tile forward and VJP. The padding carries the
// pair's VJP slot (the primitive's first slot cum[n - 1] plus the tile's index
// in the primitive's tile box, z then y then x), or 0xffffffff past
// slot_capacity.
//
// The slot is an affine function of the tile coordinates per primitive:
// slot = base + tz * nxny + ty * nx + tx with base = cum[n - 1] - (lo_z * nxny +
// lo_y * nx + lo_x) for the box [lo, hi), nx and ny its extents. A first pass
// tabulates (base, nx, nxny) per primitive into caller workspace.
struct alignas(16) SlotAffine {
    int64_t base;
    uint32_t nx, nxny;
};

template <typename S>
__global__ void voxel_slot_affine_kernel(const Rec3D<S>* __restrict__ records, const int32_t* __restrict__ radii,
                                         const int64_t* __restrict__ cum, uint32_t N, uint32_t T, uint32_t tiles_x,
                                         uint32_t tiles_y, uint32_t tiles_z, SlotAffine* __restrict__ table) {
    const uint32_t n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= N) return;
    const S centre[3] = {records[n].x, records[n].y, records[n].z};
    SlotAffine e{0, 0u, 0u};
    uint32_t lo[3], hi[3];
    if (tile_box_3d(centre, radii + 3 * size_t(n), T, tiles_x, tiles_y, tiles_z, lo, hi)) {
        e.nx = hi[0] - lo[0];
        e.nxny = e.nx * (hi[1] - lo[1]);
        e.base = (n > 0u ? cum[n - 1] : int64_t(0)) -
                 (int64_t(lo[2]) * e.nxny + int64_t(lo[1]) * e.nx + int64_t(lo[0]));
    }
    table[n] = e;
}

// One warp per tile; four lanes move one record, each a quarter of it (16 B
// fp32, 32 B fp64), so a warp reads and writes eight whole records per
// instruction. With n_used set (capacity-bounded steps) the lists hold
// min(*n_used, n_isects) entries.
template <typename S>
__global__ void __launch_bounds__(256) pack_tile_records3_kernel(
    const Rec3D<S>* __restrict__ records, const int32_t* __restrict__ offsets,
    const int32_t* __restrict__ flatten_ids, const SlotAffine* __restrict__ table, uint32_t tiles_x,
    uint32_t tiles_y, uint32_t tiles_z, uint64_t n_isects, const int64_t* __restrict__ n_used,
    uint64_t slot_capacity, Rec3D<S>* __restrict__ packed) {
    using Quarter = typename std::conditional<sizeof(S) == 4, float4, double4>::type;
    static_assert(sizeof(Rec3D<S>) == 4 * sizeof(Quarter), "a record is four quarters");
    const uint64_t n_tiles = uint64_t(tiles_x) * tiles_y * tiles_z;
    const uint64_t key = (uint64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    if (key >= n_tiles) return;  // warp-uniform
    const int64_t n = n_used != nullptr ? min(max(*n_used, int64_t(0)), int64_t(n_isects)) : int64_t(n_isects);
    const int64_t start = offsets[key];
    const int64_t end = key + 1 == n_tiles ? n : int64_t(offsets[key + 1]);
    const uint32_t plane = tiles_x * tiles_y;
    const uint32_t tz = uint32_t(key) / plane;
    const uint32_t rem = uint32_t(key) - tz * plane;
    const uint32_t ty = rem / tiles_x, tx = rem - ty * tiles_x;
    const uint32_t lane = threadIdx.x & 31u, part = lane & 3u;
    for (int64_t i = start + (lane >> 2); i < end; i += 8) {
        const int32_t gid = flatten_ids[i];
        Quarter v = reinterpret_cast<const Quarter*>(records + gid)[part];
        if (part == 3u) {
            const SlotAffine e = table[gid];
            const int64_t j = e.base + int64_t(tz) * e.nxny + int64_t(ty) * e.nx + int64_t(tx);
            const uint32_t slot = (j >= 0 && uint64_t(j) < slot_capacity) ? uint32_t(j) : 0xffffffffu;
            // pad0 is the first value of the last quarter.
            if constexpr (sizeof(S) == 4) {
                v.x = __uint_as_float(slot);
            } else {
                v.x = __longlong_as_double(static_cast<long long>(slot));
            }
        }
        reinterpret_cast<Quarter*>(packed + i)[part] = v;
    }
}

template <typename S>
__global__ void pack_records3_kernel(const S* __restrict__ means3d, const S* __restrict__ conics,
                                     const S* __restrict__ opacities, const S* __restrict__ betas,
                                     const S* __restrict__ uncertainties, uint32_t N, Rec3D<S>* __restrict__ out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    Rec3D<S> r;
    r.x = means3d[3 * size_t(i)];
    r.y = means3d[3 * size_t(i) + 1];
    r.z = means3d[3 * size_t(i) + 2];
    r.o = opacities[i];
    r.c00 = conics[6 * size_t(i)];
    r.c01 = conics[6 * size_t(i) + 1];
    r.c02 = conics[6 * size_t(i) + 2];
    r.c11 = conics[6 * size_t(i) + 3];
    r.c12 = conics[6 * size_t(i) + 4];
    r.c22 = conics[6 * size_t(i) + 5];
    r.beta = betas != nullptr ? betas[i] : S(0);
    r.q = uncertainties != nullptr ? uncertainties[i] : S(0);
    r.pad0 = r.pad1 = r.pad2 = r.pad3 = S(0);
    out[i] = r;
}

template <typename S>
__global__ void unpack_grads3_kernel(const Rec3D<S>* __restrict__ grads, uint32_t N, S* __restrict__ v_means3d,
                                     S* __restrict__ v_conics, S* __restrict__ v_opacities, S* __restrict__ v_betas,
                                     S* __restrict__ v_uncertainties) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    const Rec3D<S> g = grads[i];
    v_means3d[3 * size_t(i)] = g.x;
    v_means3d[3 * size_t(i) + 1] = g.y;
    v_means3d[3 * size_t(i) + 2] = g.z;
    v_conics[6 * size_t(i)] = g.c00;
    v_conics[6 * size_t(i) + 1] = g.c01;
    v_conics[6 * size_t(i) + 2] = g.c02;
    v_conics[6 * size_t(i) + 3] = g.c11;
    v_conics[6 * size_t(i) + 4] = g.c12;
    v_conics[6 * size_t(i) + 5] = g.c22;
    v_opacities[i] = g.o;
    if (v_betas != nullptr) v_betas[i] = g.beta;
    if (v_uncertainties != nullptr) v_uncertainties[i] = g.q;
}

inline int check_vgeom(const VoxelGeom& g) {
    R2S_REQUIRE(g.T >= 1 && g.T <= 10, R2S_ERR_UNSUPPORTED, "3D tile_size must be in [1, 10]");
    R2S_REQUIRE(uint64_t(g.tiles_x) * g.tiles_y * g.tiles_z < (uint64_t(1) << 31), R2S_ERR_UNSUPPORTED,
                "too many 3D tiles");
    return R2S_OK;
}

template <typename S, bool kBeta, bool kVar, int PPT, bool kBulk>
int launch_vfwd_t(const VoxelGeom& g, const Rec3D<S>* rec, const int32_t* offsets, const int32_t* ids, S* vol,
                  S* vol_var, unsigned nthreads, cudaStream_t stream) {
    const size_t smem = 3 * nthreads * sizeof(Rec3D<S>);
    R2S_TRY(allow_dynamic_smem(voxel_fwd_kernel<S, kBeta, kVar, PPT, kBulk>, smem, 3 * sizeof(uint64_t)));
    const unsigned grid = g.tiles_x * g.tiles_y * g.tiles_z;
    voxel_fwd_kernel<S, kBeta, kVar, PPT, kBulk><<<grid, nthreads, smem, stream>>>(rec, offsets, ids, g, vol,
                                                                                    vol_var);
    return check_launch("voxelize_to_voxels_fwd");
}

template <typename S, bool kBeta, bool kVar, bool kBulk>
int launch_vfwd_p(const VoxelGeom& g, const Rec3D<S>* rec, const int32_t* offsets, const int32_t* ids, S* vol,
                  S* vol_var, cudaStream_t stream) {
    const uint32_t voxels = g.T * g.T * g.T;
    if (voxels <= 128) {
        const unsigned nt = (voxels + 31) / 32 * 32;
        return launch_vfwd_t<S, kBeta, kVar, 1, kBulk>(g, rec, offsets, ids, vol, vol_var, nt, stream);
    }
    if (!kBeta && std::is_same<S, float>::value && g.T == 8) {
        // Eight voxels of each of two adjacent rows per thread: 32 row pairs, one warp.
        const unsigned nt = 32;
        return launch_vfwd_t<S, kBeta, kVar, 16, kBulk>(g, rec, offsets, ids, vol, vol_var, nt, stream);
    }
    // Four consecutive voxels of a row per thread: T^2 rows of ceil(T / 4) segments.
    const unsigned nt = (g.T * g.T * ((g.T + 3) / 4) + 31) / 32 * 32;
    return launch_vfwd_t<S, kBeta, kVar, 4, kBulk>(g, rec, offsets, ids, vol, vol_var, nt, stream);
}

// bulk: `rec` is the per-tile packed copy and `ids` is unused.
template <typename S>
int launch_vfwd(const VoxelGeom& g, const Rec3D<S>* rec, bool beta, const int32_t* offsets, const int32_t* ids,
                S* vol, S* vol_var, cudaStream_t stream, bool bulk = false) {
    R2S_TRY(check_vgeom(g));
    if (uint64_t(g.tiles_x) * g.tiles_y * g.tiles_z == 0) return R2S_OK;
    const bool var = vol_var != nullptr;
    if (bulk) {
        if (beta) return var ? launch_vfwd_p<S, true, true, true>(g, rec, offsets, ids, vol, vol_var, stream)
                             : launch_vfwd_p<S, true, false, true>(g, rec, offsets, ids, vol, vol_var, stream);
        return var ? launch_vfwd_p<S, false, true, true>(g, rec, offsets, ids, vol, vol_var, stream)
                   : launch_vfwd_p<S, false, false, true>(g, rec, offsets, ids, vol, vol_var, stream);
    }
    if (beta) return var ? launch_vfwd_p<S, true, true, false>(g, rec, offsets, ids, vol, vol_var, stream)
                         : launch_vfwd_p<S, true, false, false>(g, rec, offsets, ids, vol, vol_var, stream);
    return var ? launch_vfwd_p<S, false, true, false>(g, rec, offsets, ids, vol, vol_var, stream)
               : launch_vfwd_p<S, false, false, false>(g, rec, offsets, ids, vol, vol_var, stream);
}

template <typename S, bool kBeta, bool kVar, bool kBulk>
int launch_vbwd_p(const VoxelGeom& g, const Rec3D<S>* rec, bool chain_var, const int32_t* offsets,
                  const int32_t* ids, const S* v_vol, const S* v_vol_var, Rec3D<S>* grads, cudaStream_t stream,
                  const VoxelSlots<S>& sl) {
    if constexpr (std::is_same<S, float>::value && !kBeta && !kVar) {
        if (g.T == 8) {
            const unsigned grid = g.tiles_x * g.tiles_y * g.tiles_z;
            voxel_bwd_lanes_kernel<kBulk><<<grid, kVoxLaneThreads, 0, stream>>>(rec, offsets, ids, g, v_vol, grads,
                                                                                  sl);
            return check_launch("voxelize_to_voxels_bwd");
        }
    }
    const size_t tile_slots = size_t(g.T) * g.T * (g.T + 1) + (g.T + 1);
    const size_t smem = 2 * size_t(kVoxBwdThreads) * (sizeof(Rec3D<S>) + 2 * sizeof(int32_t)) +
                        size_t(kVoxBwdThreads) * sizeof(VoxelBox) + 2 * tile_slots * sizeof(S);
    R2S_TRY(allow_dynamic_smem(voxel_bwd_kernel<S, kBeta, kVar, kBulk>, smem, 2 * sizeof(uint64_t)));
    const unsigned grid = g.tiles_x * g.tiles_y * g.tiles_z;
    voxel_bwd_kernel<S, kBeta, kVar, kBulk><<<grid, kVoxBwdThreads, smem, stream>>>(
        rec, chain_var, offsets, ids, g, v_vol, v_vol_var, grads, sl);
    return check_launch("voxelize_to_voxels_bwd");
}

template <typename S, bool kBulk>
int launch_vbwd_b(const VoxelGeom& g, const Rec3D<S>* rec, bool beta, bool chain_var, const int32_t* offsets,
                  const int32_t* ids, const S* v_vol, const S* v_vol_var, Rec3D<S>* grads, cudaStream_t stream,
                  const VoxelSlots<S>& sl) {
    const bool var = v_vol_var != nullptr;
    if (beta)
        return var ? launch_vbwd_p<S, true, true, kBulk>(g, rec, chain_var, offsets, ids, v_vol, v_vol_var, grads,
                                                         stream, sl)
                   : launch_vbwd_p<S, true, false, kBulk>(g, rec, chain_var, offsets, ids, v_vol, v_vol_var, grads,
                                                          stream, sl);
    return var ? launch_vbwd_p<S, false, true, kBulk>(g, rec, chain_var, offsets, ids, v_vol, v_vol_var, grads,
                                                      stream, sl)
               : launch_vbwd_p<S, false, false, kBulk>(g, rec, chain_var, offsets, ids, v_vol, v_vol_var, grads,
                                                       stream, sl);
}

// bulk: `rec` is the per-tile packed copy with the slots in its padding (slot output only).
template <typename S>
int launch_vbwd(const VoxelGeom& g, const Rec3D<S>* rec, bool beta, bool chain_var, const int32_t* offsets,
                const int32_t* ids, const S* v_vol, const S* v_vol_var, Rec3D<S>* grads, cudaStream_t stream,
                const VoxelSlots<S>& sl = VoxelSlots<S>{}, bool bulk = false) {
    R2S_TRY(check_vgeom(g));
    if (g.n_isects == 0 || uint64_t(g.tiles_x) * g.tiles_y * g.tiles_z == 0) return R2S_OK;
    if (bulk) return launch_vbwd_b<S, true>(g, rec, beta, chain_var, offsets, ids, v_vol, v_vol_var, grads, stream, sl);
    return launch_vbwd_b<S, false>(g, rec, beta, chain_var, offsets, ids, v_vol, v_vol_var, grads, stream, sl);
}

// Tile VJP into slots, then the in-order per-primitive sum into grads (written, not accumulated).
template <typename S>
int launch_vbwd_slots(const VoxelGeom& g, const Rec3D<S>* rec, bool beta, bool chain_var, const int32_t* offsets,
                      const int32_t* ids, const S* v_vol, const S* v_vol_var, const VoxelSlots<S>& sl,
                      Rec3D<S>* grads, cudaStream_t stream, bool bulk = false) {
    if (g.N == 0) return R2S_OK;
    R2S_TRY(launch_vbwd<S>(g, rec, beta, chain_var, offsets, ids, v_vol, v_vol_var, grads, stream, sl, bulk));
    voxel_slot_reduce_kernel<S><<<blocks_for(int64_t(g.N) * kSlotLanes, 256), 256, 0, stream>>>(
        sl.slots, sl.cum, g.N, int64_t(sl.capacity), grads);
    return check_launch("voxel_slot_reduce");
}

template <typename S, bool kBeta, bool kVar>
int launch_vrec_p(const VoxelRecordGeom& g, const Rec3D<S>* rec, const S* means_v, const int32_t* radii,
                  const int64_t* item_cum, bool chain_var, const S* v_vol, const S* v_vol_var, Rec3D<S>* partials,
                  cudaStream_t stream) {
    // Persistent over the items: at most four resident 8-warp blocks per SM's worth of blocks.
    const uint64_t needed = (g.n_items + kVoxBwdWarps - 1) / kVoxBwdWarps;
    const unsigned grid = unsigned(needed < uint64_t(148 * 8) ? (needed > 0 ? needed : 1) : uint64_t(148 * 8));
    const size_t smem = size_t(kVoxBwdWarps) * 32u * kRecStride * sizeof(S) * (kVar ? 2u : 1u);
    R2S_TRY(allow_dynamic_smem(voxel_record_bwd_kernel<S, kBeta, kVar>, smem));
    voxel_record_bwd_kernel<S, kBeta, kVar><<<grid, kVoxBwdThreads, smem, stream>>>(
        rec, means_v, radii, item_cum, chain_var, g, v_vol, v_vol_var, partials);
    return check_launch("voxel_record_bwd");
}

template <typename S>
int launch_vrec(const VoxelRecordGeom& g, const Rec3D<S>* rec, const S* means_v, const int32_t* radii,
                const int64_t* item_cum, bool beta, bool chain_var, const S* v_vol, const S* v_vol_var,
                Rec3D<S>* partials, Rec3D<S>* grads, cudaStream_t stream) {
    if (g.N == 0) return R2S_OK;
    if (g.n_items > 0) {
        const bool var = v_vol_var != nullptr;
        int status;
        if (beta)
            status = var ? launch_vrec_p<S, true, true>(g, rec, means_v, radii, item_cum, chain_var, v_vol,
                                                        v_vol_var, partials, stream)
                         : launch_vrec_p<S, true, false>(g, rec, means_v, radii, item_cum, chain_var, v_vol,
                                                         v_vol_var, partials, stream);
        else
            status = var ? launch_vrec_p<S, false, true>(g, rec, means_v, radii, item_cum, chain_var, v_vol,
                                                         v_vol_var, partials, stream)
                         : launch_vrec_p<S, false, false>(g, rec, means_v, radii, item_cum, chain_var, v_vol,
                                                          v_vol_var, partials, stream);
        R2S_TRY(status);
    }
    voxel_record_reduce_kernel<S><<<blocks_for(g.N, 256), 256, 0, stream>>>(partials, item_cum, g.N,
                                                                           int64_t(g.n_items), grads);
    return check_launch("voxel_record_reduce");
}

__global__ void item_capacity_check_kernel(const int64_t* __restrict__ used, uint64_t capacity,
                                           uint32_t* __restrict__ overflow) {
    if (uint64_t(*used) > capacity) *overflow = 1u;
}

template <typename S>
size_t voxel_ws(uint32_t N, bool with_grads) {
    ArenaSize a;
    a.take<Rec3D<S>>(N);
    if (with_grads) a.take<Rec3D<S>>(N);
    return a.bytes();
}

}  // namespace r2s

using namespace r2s;

namespace {

template <typename S>
int voxel_fwd_lowlevel(const void* means3d, const void* conics, const void* opacities, const void* betas,
                       const void* unc, const int32_t* offsets, const int32_t* ids, const VoxelGeom& g, void* vol,
                       void* vol_var, void* ws, size_t ws_bytes, cudaStream_t stream) {
    const size_t voxels = size_t(g.dim0) * g.dim1 * g.dim2;
    if (g.N == 0 || g.n_isects == 0) {
        if (voxels) {
            if (cudaMemsetAsync(vol, 0, voxels * sizeof(S), stream) != cudaSuccess ||
                (vol_var && cudaMemsetAsync(vol_var, 0, voxels * sizeof(S), stream) != cudaSuccess))
                return fail(R2S_ERR_CUDA, "memset failed");
        }
        return R2S_OK;
    }
    Arena arena(ws, ws_bytes);
    Rec3D<S>* rec = arena.take<Rec3D<S>>(g.N);
    R2S_REQUIRE(rec, R2S_ERR_WORKSPACE, "voxel workspace too small");
    pack_records3_kernel<S><<<blocks_for(g.N, 256), 256, 0, stream>>>(
        static_cast<const S*>(means3d), static_cast<const S*>(conics), static_cast<const S*>(opacities),
        static_cast<const S*>(betas), static_cast<const S*>(unc), g.N, rec);
    R2S_TRY(check_launch("pack_records3"));
    return launch_vfwd<S>(g, rec, betas != nullptr, offsets, ids, static_cast<S*>(vol), static_cast<S*>(vol_var),
                          stream);
}

}  // namespace

extern "C" {

size_t r2s_voxel_workspace(uint32_t dtype, uint32_t N, int with_gradients) {
    return dtype == R2S_F64 ? voxel_ws<double>(N, with_gradients != 0) : voxel_ws<float>(N, with_gradients != 0);
}

int r2s_voxelize_to_voxels_fwd(int dtype, const void* means3d, const void* conics, const void* opacities,
                               const void* betas, const int32_t* tile_offsets, const int32_t* flatten_ids,
                               uint32_t N, uint32_t n_isects, uint32_t dim2, uint32_t dim1, uint32_t dim0,
                               uint32_t tile_size, uint32_t tiles_x, uint32_t tiles_y, uint32_t tiles_z,
                               void* volume, void* workspace, size_t workspace_bytes, void* stream) {
    const VoxelGeom g{N, n_isects, dim2, dim1, dim0, tile_size, tiles_x, tiles_y, tiles_z};
    R2S_DISPATCH(dtype, return voxel_fwd_lowlevel<S>(means3d, conics, opacities, betas, nullptr, tile_offsets,
                                                    flatten_ids, g, volume, nullptr, workspace, workspace_bytes,
                                                    as_stream(stream)));
}

int r2s_voxelize_to_voxels_mean_var_fwd(int dtype, const void* means3d, const void* conics, const void* opacities,
                                        const void* betas, const void* uncertainties, const int32_t* tile_offsets,
                                        const int32_t* flatten_ids, uint32_t N, uint32_t n_isects, uint32_t dim2,
                                        uint32_t dim1, uint32_t dim0, uint32_t tile_size, uint32_t tiles_x,
                                        uint32_t tiles_y, uint32_t tiles_z, void* volume, void* volume_var,
                                        void* workspace, size_t workspace_bytes, void* stream) {
    const VoxelGeom g{N, n_isects, dim2, dim1, dim0, tile_size, tiles_x, tiles_y, tiles_z};
    R2S_REQUIRE(uncertainties && volume_var, R2S_ERR_ARGUMENT, "mean/variance voxelization needs uncertainties");
    R2S_DISPATCH(dtype, return voxel_fwd_lowlevel<S>(means3d, conics, opacities, betas, uncertainties, tile_offsets,
                                                    flatten_ids, g, volume, volume_var, workspace, workspace_bytes,
                                                    as_stream(stream)));
}

int r2s_voxelize_to_voxels_bwd(int dtype, const void* means3d, const void* conics, const void* opacities,
                               const void* betas, const int32_t* tile_offsets, const int64_t* isect_ids,
                               const int32_t* flatten_ids, const void* v_volume, const void* v_volume_var,
                               const void* uncertainties, uint32_t N, uint32_t n_isects, uint32_t dim2, uint32_t dim1,
                               uint32_t dim0, uint32_t tile_size, uint32_t tiles_x, uint32_t tiles_y,
                               uint32_t tiles_z, void* v_means3d, void* v_conics, void* v_opacities, void* v_betas,
                               void* v_uncertainties, void* workspace, size_t workspace_bytes, void* stream) {
    (void)isect_ids;
    const VoxelGeom g{N, n_isects, dim2, dim1, dim0, tile_size, tiles_x, tiles_y, tiles_z};
    R2S_REQUIRE((betas == nullptr) == (v_betas == nullptr), R2S_ERR_ARGUMENT, "v_betas goes with betas");
    R2S_REQUIRE(v_volume_var == nullptr || v_uncertainties != nullptr, R2S_ERR_ARGUMENT,
                "variance adjoint needs v_uncertainties");
    R2S_DISPATCH(dtype, {
        if (N == 0) return R2S_OK;
        cudaStream_t st = as_stream(stream);
        Arena arena(workspace, workspace_bytes);
        Rec3D<S>* rec = arena.take<Rec3D<S>>(N);
        Rec3D<S>* grads = arena.take<Rec3D<S>>(N);
        R2S_REQUIRE(rec && grads, R2S_ERR_WORKSPACE, "voxel workspace too small");
        if (cudaMemsetAsync(grads, 0, size_t(N) * sizeof(Rec3D<S>), st) != cudaSuccess)
            return fail(R2S_ERR_CUDA, "memset failed");
        if (n_isects > 0) {
            pack_records3_kernel<S><<<blocks_for(N, 256), 256, 0, st>>>(
                static_cast<const S*>(means3d), static_cast<const S*>(conics), static_cast<const S*>(opacities),
                static_cast<const S*>(betas), static_cast<const S*>(uncertainties), N, rec);
            R2S_TRY(check_launch("pack_records3"));
            R2S_TRY(launch_vbwd<S>(g, rec, betas != nullptr, uncertainties != nullptr, tile_offsets, flatten_ids,
                                   static_cast<const S*>(v_volume), static_cast<const S*>(v_volume_var), grads, st));
        }
        unpack_grads3_kernel<S><<<blocks_for(N, 256), 256, 0, st>>>(
            grads, N, static_cast<S*>(v_means3d), static_cast<S*>(v_conics), static_cast<S*>(v_opacities),
            static_cast<S*>(v_betas), v_volume_var ? static_cast<S*>(v_uncertainties) : nullptr);
        return check_launch("unpack_grads3");
    });
}

int r2s_voxel_render(int dtype, const void* records, int beta, const int32_t* tile_offsets,
                     const int32_t* flatten_ids, uint32_t N, uint32_t n_isects, uint32_t dim2, uint32_t dim1,
                     uint32_t dim0, uint32_t tile_size, uint32_t tiles_x, uint32_t tiles_y, uint32_t tiles_z,
                     void* volume, void* volume_var, void* stream) {
    const VoxelGeom g{N, n_isects, dim2, dim1, dim0, tile_size, tiles_x, tiles_y, tiles_z};
    R2S_DISPATCH(dtype, return launch_vfwd<S>(g, static_cast<const Rec3D<S>*>(records), beta != 0, tile_offsets,
                                              flatten_ids, static_cast<S*>(volume), static_cast<S*>(volume_var),
                                              as_stream(stream)));
}

int r2s_voxel_render_bwd(int dtype, const void* records, int beta, int detach_variance, const int32_t* tile_offsets,
                         const int32_t* flatten_ids, const void* v_volume, const void* v_volume_var, uint32_t N,
                         uint32_t n_isects, uint32_t dim2, uint32_t dim1, uint32_t dim0, uint32_t tile_size,
                         uint32_t tiles_x, uint32_t tiles_y, uint32_t tiles_z, void* grads, void* stream) {
    const VoxelGeom g{N, n_isects, dim2, dim1, dim0, tile_size, tiles_x, tiles_y, tiles_z};
    R2S_DISPATCH(dtype, return launch_vbwd<S>(g, static_cast<const Rec3D<S>*>(records), beta != 0,
                                              detach_variance == 0, tile_offsets, flatten_ids,
                                              static_cast<const S*>(v_volume), static_cast<const S*>(v_volume_var),
                                              static_cast<Rec3D<S>*>(grads), as_stream(stream)));
}

int r2s_voxel_render_capacity(int dtype, const void* records, int beta, const int32_t* tile_offsets,
                              const int32_t* flatten_ids, const int64_t* n_used, uint32_t N, uint32_t dim2,
                              uint32_t dim1, uint32_t dim0, uint32_t tile_size, uint32_t tiles_x, uint32_t tiles_y,
                              uint32_t tiles_z, void* volume, void* volume_var, void* stream) {
    R2S_REQUIRE(n_used != nullptr, R2S_ERR_ARGUMENT, "n_used must be non-null");
    VoxelGeom g{N, 1u, dim2, dim1, dim0, tile_size, tiles_x, tiles_y, tiles_z};
    g.n_dev = n_used;
    R2S_DISPATCH(dtype, return launch_vfwd<S>(g, static_cast<const Rec3D<S>*>(records), beta != 0, tile_offsets,
                                              flatten_ids, static_cast<S*>(volume), static_cast<S*>(volume_var),
                                              as_stream(stream)));
}

int r2s_voxel_render_bwd_capacity(int dtype, const void* records, int beta, int detach_variance,
                                  const int32_t* tile_offsets, const int32_t* flatten_ids, const int64_t* n_used,
                                  const void* v_volume, const void* v_volume_var, uint32_t N, uint32_t dim2,
                                  uint32_t dim1, uint32_t dim0, uint32_t tile_size, uint32_t tiles_x,
                                  uint32_t tiles_y, uint32_t tiles_z, void* grads, void* stream) {
    R2S_REQUIRE(n_used != nullptr, R2S_ERR_ARGUMENT, "n_used must be non-null");
    VoxelGeom g{N, 1u, dim2, dim1, dim0, tile_size, tiles_x, tiles_y, tiles_z};
    g.n_dev = n_used;
    R2S_DISPATCH(dtype, return launch_vbwd<S>(g, static_cast<const Rec3D<S>*>(records), beta != 0,
                                              detach_variance == 0, tile_offsets, flatten_ids,
                                              static_cast<const S*>(v_volume), static_cast<const S*>(v_volume_var),
                                              static_cast<Rec3D<S>*>(grads), as_stream(stream)));
}

int r2s_voxel_render_bwd_slots(int dtype, const void* records, int beta, int detach_variance,
                               const int32_t* tile_offsets, const int32_t* flatten_ids, uint64_t n_isects,
                               const int64_t* n_used, const void* means_v, const int32_t* radii,
                               const int64_t* tile_cum, const void* v_volume, const void* v_volume_var, uint32_t N,
                               uint32_t dim2, uint32_t dim1, uint32_t dim0, uint32_t tile_size, uint32_t tiles_x,
                               uint32_t tiles_y, uint32_t tiles_z, void* slots, uint64_t slot_capacity, void* grads,
                               void* stream) {
    if (N == 0) return R2S_OK;
    R2S_REQUIRE(records != nullptr && means_v != nullptr && radii != nullptr && tile_cum != nullptr &&
                    slots != nullptr && grads != nullptr,
                R2S_ERR_ARGUMENT, "records, means_v, radii, tile_cum, slots and grads must be non-null");
    R2S_REQUIRE(reinterpret_cast<uintptr_t>(slots) % 16 == 0, R2S_ERR_ARGUMENT, "slots must be 16-byte aligned");
    R2S_REQUIRE(n_used != nullptr || n_isects <= slot_capacity, R2S_ERR_ARGUMENT,
                "slot_capacity must hold n_isects slots");
    R2S_REQUIRE(n_isects < (uint64_t(1) << 31), R2S_ERR_UNSUPPORTED, "too many 3D intersections");
    R2S_REQUIRE(slot_capacity < (uint64_t(1) << 31), R2S_ERR_UNSUPPORTED, "slot_capacity must be below 2^31");
    VoxelGeom g{N, uint32_t(n_used != nullptr ? 1u : n_isects), dim2, dim1, dim0, tile_size, tiles_x, tiles_y,
                tiles_z};
    g.n_dev = n_used;
    R2S_DISPATCH(dtype, {
        VoxelSlots<S> sl;
        sl.means_v = static_cast<const S*>(means_v);
        sl.radii = radii;
        sl.cum = tile_cum;
        sl.slots = static_cast<S*>(slots);
        sl.capacity = slot_capacity;
        return launch_vbwd_slots<S>(g, static_cast<const Rec3D<S>*>(records), beta != 0, detach_variance == 0,
                                    tile_offsets, flatten_ids, static_cast<const S*>(v_volume),
                                    static_cast<const S*>(v_volume_var), sl, static_cast<Rec3D<S>*>(grads),
                                    as_stream(stream));
    });
}

size_t r2s_voxel_pack_workspace(uint32_t N) { return size_t(N) * sizeof(SlotAffine) + 256; }

int r2s_voxel_pack_tile_records(int dtype, const void* records, const int32_t* tile_offsets,
                                const int32_t* flatten_ids, const int32_t* radii, const int64_t* tile_cum, uint32_t N,
                                uint64_t n_isects, const int64_t* n_used, uint32_t tile_size, uint32_t tiles_x,
                                uint32_t tiles_y, uint32_t tiles_z, uint64_t slot_capacity, void* packed,
                                void* workspace, size_t workspace_bytes, void* stream) {
    if (n_isects == 0 || N == 0) return R2S_OK;
    R2S_REQUIRE(records != nullptr && tile_offsets != nullptr && flatten_ids != nullptr && radii != nullptr &&
                    tile_cum != nullptr && packed != nullptr,
                R2S_ERR_ARGUMENT, "records, tile_offsets, flatten_ids, radii, tile_cum and packed must be non-null");
    R2S_REQUIRE(n_isects < (uint64_t(1) << 31), R2S_ERR_UNSUPPORTED, "too many 3D intersections");
    R2S_REQUIRE(slot_capacity < (uint64_t(1) << 31), R2S_ERR_UNSUPPORTED, "slot_capacity must be below 2^31");
    R2S_REQUIRE(tile_size >= 1 && uint64_t(tiles_x) * tiles_y * tiles_z < (uint64_t(1) << 31), R2S_ERR_UNSUPPORTED,
                "3D tile grid out of range");
    Arena arena(workspace, workspace_bytes);
    SlotAffine* table = arena.take<SlotAffine>(N);
    R2S_REQUIRE(table != nullptr, R2S_ERR_WORKSPACE, "pack workspace too small (r2s_voxel_pack_workspace)");
    const uint64_t n_tiles = uint64_t(tiles_x) * tiles_y * tiles_z;
    R2S_DISPATCH(dtype, {
        voxel_slot_affine_kernel<S><<<blocks_for(N, 256), 256, 0, as_stream(stream)>>>(
            static_cast<const Rec3D<S>*>(records), radii, tile_cum, N, tile_size, tiles_x, tiles_y, tiles_z, table);
        R2S_TRY(check_launch("voxel_slot_affine"));
        pack_tile_records3_kernel<S><<<blocks_for(int64_t(n_tiles) * 32, 256), 256, 0, as_stream(stream)>>>(
            static_cast<const Rec3D<S>*>(records), tile_offsets, flatten_ids, table, tiles_x, tiles_y, tiles_z,
            n_isects, n_used, slot_capacity, static_cast<Rec3D<S>*>(packed));
    });
    return check_launch("voxel_pack_tile_records");
}

int r2s_voxel_render_packed(int dtype, const void* packed, int beta, const int32_t* tile_offsets,
                            uint64_t n_isects, const int64_t* n_used, uint32_t dim2, uint32_t dim1, uint32_t dim0,
                            uint32_t tile_size, uint32_t tiles_x, uint32_t tiles_y, uint32_t tiles_z, void* volume,
                            void* volume_var, void* stream) {
    R2S_REQUIRE(n_isects < (uint64_t(1) << 31), R2S_ERR_UNSUPPORTED, "too many 3D intersections");
    R2S_REQUIRE(tile_offsets != nullptr && volume != nullptr && (packed != nullptr || n_isects == 0),
                R2S_ERR_ARGUMENT, "packed, tile_offsets and volume must be non-null");
    VoxelGeom g{0u, uint32_t(n_isects), dim2, dim1, dim0, tile_size, tiles_x, tiles_y, tiles_z};
    g.n_dev = n_used;
    R2S_DISPATCH(dtype, return launch_vfwd<S>(g, static_cast<const Rec3D<S>*>(packed), beta != 0, tile_offsets,
                                              nullptr, static_cast<S*>(volume), static_cast<S*>(volume_var),
                                              as_stream(stream), true));
}

int r2s_voxel_render_bwd_packed(int dtype, const void* packed, int beta, int detach_variance,
                                const int32_t* tile_offsets, uint64_t n_isects, const int64_t* n_used,
                                const int64_t* tile_cum, const void* v_volume, const void* v_volume_var, uint32_t N,
                                uint32_t dim2, uint32_t dim1, uint32_t dim0, uint32_t tile_size, uint32_t tiles_x,
                                uint32_t tiles_y, uint32_t tiles_z, void* slots, uint64_t slot_capacity, void* grads,
                                void* stream) {
    if (N == 0) return R2S_OK;
    R2S_REQUIRE(tile_offsets != nullptr && tile_cum != nullptr && slots != nullptr && grads != nullptr &&
                    (packed != nullptr || n_isects == 0),
                R2S_ERR_ARGUMENT, "packed, tile_offsets, tile_cum, slots and grads must be non-null");
    R2S_REQUIRE(reinterpret_cast<uintptr_t>(slots) % 16 == 0, R2S_ERR_ARGUMENT, "slots must be 16-byte aligned");
    R2S_REQUIRE(n_used != nullptr || n_isects <= slot_capacity, R2S_ERR_ARGUMENT,
                "slot_capacity must hold n_isects slots");
    R2S_REQUIRE(n_isects < (uint64_t(1) << 31), R2S_ERR_UNSUPPORTED, "too many 3D intersections");
    R2S_REQUIRE(slot_capacity < (uint64_t(1) << 31), R2S_ERR_UNSUPPORTED, "slot_capacity must be below 2^31");
    VoxelGeom g{N, uint32_t(n_used != nullptr ? 1u : n_isects), dim2, dim1, dim0, tile_size, tiles_x, tiles_y,
                tiles_z};
    g.n_dev = n_used;
    R2S_DISPATCH(dtype, {
        VoxelSlots<S> sl;
        sl.cum = tile_cum;
        sl.slots = static_cast<S*>(slots);
        sl.capacity = slot_capacity;
        return launch_vbwd_slots<S>(g, static_cast<const Rec3D<S>*>(packed), beta != 0, detach_variance == 0,
                                    tile_offsets, nullptr, static_cast<const S*>(v_volume),
                                    static_cast<const S*>(v_volume_var), sl, static_cast<Rec3D<S>*>(grads),
                                    as_stream(stream), true);
    });
}

int r2s_bulk_wait_faults(int device, int clear, uint32_t* count) {
    R2S_REQUIRE(count != nullptr, R2S_ERR_ARGUMENT, "count must be non-null");
    int previous = 0;
    cudaError_t err = cudaGetDevice(&previous);
    if (err == cudaSuccess && previous != device) err = cudaSetDevice(device);
    unsigned int value = 0u;
    if (err == cudaSuccess) err = cudaMemcpyFromSymbol(&value, g_bulk_wait_faults, sizeof(value));
    if (err == cudaSuccess && clear != 0) {
        const unsigned int zero = 0u;
        err = cudaMemcpyToSymbol(g_bulk_wait_faults, &zero, sizeof(zero));
    }
    if (previous != device) cudaSetDevice(previous);
    if (err != cudaSuccess) return fail(R2S_ERR_CUDA, std::string("bulk wait fault counter: ") + cudaGetErrorString(err));
    *count = value;
    return R2S_OK;
}

int r2s_voxel_layer_counts(int dtype, const void* means_v, const int32_t* radii, uint32_t N, uint32_t dim2,
                           uint32_t dim1, uint32_t dim0, uint32_t tile_size, uint32_t tiles_x, uint32_t tiles_y,
                           uint32_t tiles_z, int32_t* layers, void* stream) {
    if (N == 0) return R2S_OK;
    R2S_REQUIRE(means_v != nullptr && radii != nullptr && layers != nullptr, R2S_ERR_ARGUMENT,
                "means_v, radii and layers must be non-null");
    VoxelRecordGeom g{N, dim2, dim1, dim0, tile_size, tiles_x, tiles_y, tiles_z, 0u, nullptr};
    R2S_DISPATCH(dtype, voxel_layer_count_kernel<S><<<blocks_for(N, 256), 256, 0, as_stream(stream)>>>(
        static_cast<const S*>(means_v), radii, g, layers));
    return check_launch("voxel_layer_counts");
}

int r2s_voxel_record_bwd(int dtype, const void* records, const void* means_v, const int32_t* radii,
                         const int64_t* layer_cum, uint64_t n_items, const int64_t* n_items_dev, int beta,
                         int detach_variance, const void* v_volume, const void* v_volume_var, uint32_t N,
                         uint32_t dim2, uint32_t dim1, uint32_t dim0, uint32_t tile_size, uint32_t tiles_x,
                         uint32_t tiles_y, uint32_t tiles_z, void* partials, void* grads, uint32_t* overflow,
                         void* stream) {
    if (N == 0) return R2S_OK;
    R2S_REQUIRE(records != nullptr && means_v != nullptr && radii != nullptr && layer_cum != nullptr &&
                    grads != nullptr && (partials != nullptr || n_items == 0),
                R2S_ERR_ARGUMENT, "records, means_v, radii, layer_cum, partials and grads must be non-null");
    R2S_REQUIRE(tile_size >= 1 && tile_size <= 10, R2S_ERR_UNSUPPORTED, "3D tile_size must be in [1, 10]");
    VoxelRecordGeom g{N, dim2, dim1, dim0, tile_size, tiles_x, tiles_y, tiles_z, n_items, n_items_dev};
    cudaStream_t st = as_stream(stream);
    if (n_items_dev != nullptr && overflow != nullptr) {
        item_capacity_check_kernel<<<1, 1, 0, st>>>(n_items_dev, n_items, overflow);
        R2S_TRY(check_launch("voxel_record_capacity"));
    }
    R2S_DISPATCH(dtype, return launch_vrec<S>(g, static_cast<const Rec3D<S>*>(records), static_cast<const S*>(means_v),
                                              radii, layer_cum, beta != 0, detach_variance == 0,
                                              static_cast<const S*>(v_volume), static_cast<const S*>(v_volume_var),
                                              static_cast<Rec3D<S>*>(partials), static_cast<Rec3D<S>*>(grads), st));
}

}  // extern "C"
