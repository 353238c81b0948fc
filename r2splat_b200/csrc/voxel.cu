// Voxelization: per-tile (T^3 voxels) accumulation of Gaussian / Beta
// densities at voxel centres, and its VJP, on packed per-primitive records.
//
// Same schedule as the rasterizer: one CTA per 3D tile, the tile's
// intersection list gathered into shared memory with cp.async in
// double-buffered batches (records are [N] x 64 B and stay in L2), forward
// threads own up to 4 voxels, backward warps own one record at a time over a
// 256-voxel sub-tile (8 voxels per lane), warp-reduce, then issue three
// vector atomics per record.
//
// Per-sample arithmetic keeps the reference's expression forms
// (VoxelizeToVoxelsFwd.cu:180-215, :555-580; VoxelizeToVoxelsBwd.cu:397-433,
// :853-895) so the |alpha| thresholds (1e-6 Gaussian, 1e-5 Beta) select the
// same samples. The tile size is a run-time value, so the compiler cannot
// merge arithmetic across a thread's voxels.
#include "common.cuh"

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
};

template <typename S, bool kBeta, bool kVar, int PPT>
__global__ void __launch_bounds__(256) voxel_fwd_kernel(const Rec3D<S>* __restrict__ records,
                                                        const int32_t* __restrict__ offsets,
                                                        const int32_t* __restrict__ flatten_ids, VoxelGeom g,
                                                        S* __restrict__ volume, S* __restrict__ volume_var) {
    extern __shared__ __align__(16) unsigned char smem[];
    const uint32_t nthreads = blockDim.x;
    Rec3D<S>* s_rec = reinterpret_cast<Rec3D<S>*>(smem);  // [2][nthreads]
    const uint32_t T = g.T;
    const uint32_t n_tiles = g.tiles_x * g.tiles_y * g.tiles_z;
    const uint32_t key = blockIdx.x;
    const int32_t start = offsets[key];
    const int32_t end = (key + 1 == n_tiles) ? int32_t(g.n_isects) : offsets[key + 1];
    const uint32_t tz = key / (g.tiles_x * g.tiles_y);
    const uint32_t rem = key - tz * g.tiles_x * g.tiles_y;
    const uint32_t ty = rem / g.tiles_x, tx = rem - ty * g.tiles_x;
    const uint32_t t = threadIdx.x;

    S px[PPT], py[PPT], pz[PPT], acc[PPT], accv[PPT];
    size_t vid[PPT];
    bool inside[PPT];
#pragma unroll
    for (int k = 0; k < PPT; ++k) {
        const uint32_t p = t + uint32_t(k) * nthreads;
        uint32_t lz, ly, lx;
        tile_voxel(p, T, lz, ly, lx);
        const uint32_t i = tz * T + lz, j = ty * T + ly, kk = tx * T + lx;
        inside[k] = p < T * T * T && i < g.dim0 && j < g.dim1 && kk < g.dim2;
        px[k] = static_cast<S>(kk) + static_cast<S>(0.5);
        py[k] = static_cast<S>(j) + static_cast<S>(0.5);
        pz[k] = static_cast<S>(i) + static_cast<S>(0.5);
        vid[k] = (size_t(i) * g.dim1 + j) * g.dim2 + kk;
        acc[k] = S(0);
        accv[k] = S(0);
    }

    const int32_t count = end - start;
    const int32_t n_batches = count > 0 ? (count + int32_t(nthreads) - 1) / int32_t(nthreads) : 0;
    auto load = [&](int32_t b, int stage) {
        const int32_t idx = start + b * int32_t(nthreads) + int32_t(t);
        if (idx < end) gather_record3(s_rec + stage * nthreads + t, records + flatten_ids[idx]);
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
        const Rec3D<S>* buf = s_rec + (b & 1) * nthreads;
        const int32_t batch = min(int32_t(nthreads), count - b * int32_t(nthreads));
        for (int32_t s = 0; s < batch; ++s) {
            const Rec3D<S> r = buf[s];
#pragma unroll
            for (int k = 0; k < PPT; ++k) {
                if (!kBeta) {
                    const S d1 = px[k] - r.x, d2 = py[k] - r.y, d3 = pz[k] - r.z;
                    const S sigma = static_cast<S>(0.5) * (r.c00 * d1 * d1 + r.c11 * d2 * d2 + r.c22 * d3 * d3) +
                                    r.c01 * d1 * d2 + r.c02 * d1 * d3 + r.c12 * d2 * d3;
                    const S alpha = r.o * exp(-sigma);
                    if (!(sigma < static_cast<S>(0) || fabs(alpha) < static_cast<S>(1e-6))) {
                        acc[k] += alpha;
                        if (kVar) accv[k] += r.q * alpha * alpha;
                    }
                } else {
                    const S d1 = r.x - px[k], d2 = r.y - py[k], d3 = r.z - pz[k];
                    const S qf = r.c00 * d1 * d1 + r.c11 * d2 * d2 + r.c22 * d3 * d3 +
                                 static_cast<S>(2) * r.c01 * d1 * d2 + static_cast<S>(2) * r.c02 * d1 * d3 +
                                 static_cast<S>(2) * r.c12 * d2 * d3;
                    if (!(qf < static_cast<S>(0) || qf >= static_cast<S>(1))) {
                        const S h = static_cast<S>(1) - qf;
                        const S alpha = r.o * pow(h, r.beta);
                        if (!(fabs(alpha) < static_cast<S>(1e-5))) {
                            acc[k] += alpha;
                            if (kVar) accv[k] += r.q * alpha * alpha;
                        }
                    }
                }
            }
        }
        __syncthreads();
    }
#pragma unroll
    for (int k = 0; k < PPT; ++k) {
        if (inside[k]) {
            volume[vid[k]] = acc[k];
            if (kVar) volume_var[vid[k]] = accv[k];
        }
    }
}

constexpr int kVoxBwdWarps = 8;
constexpr int kVoxBwdThreads = kVoxBwdWarps * 32;

// Null-pointer conventions as in the rasterizer VJP: v_volume null = zero
// adjoint; v_volume_var null = no variance branch; chain_var false =
// detached variance branch.
template <typename S, bool kBeta, bool kVar, int PPL>
__global__ void __launch_bounds__(kVoxBwdThreads) voxel_bwd_kernel(
    const Rec3D<S>* __restrict__ records, bool chain_var, const int32_t* __restrict__ offsets,
    const int32_t* __restrict__ flatten_ids, VoxelGeom g, const S* __restrict__ v_volume,
    const S* __restrict__ v_volume_var, Rec3D<S>* __restrict__ grads) {
    extern __shared__ __align__(16) unsigned char smem[];
    Rec3D<S>* s_rec = reinterpret_cast<Rec3D<S>*>(smem);                    // [2][threads]
    int32_t* s_id = reinterpret_cast<int32_t*>(s_rec + 2 * kVoxBwdThreads);  // [2][threads]
    const uint32_t T = g.T;
    const uint32_t n_tiles = g.tiles_x * g.tiles_y * g.tiles_z;
    const uint32_t key = blockIdx.x;
    const int32_t start = offsets[key];
    const int32_t end = (key + 1 == n_tiles) ? int32_t(g.n_isects) : offsets[key + 1];
    const int32_t count = end - start;
    if (count <= 0) return;
    const uint32_t tz = key / (g.tiles_x * g.tiles_y);
    const uint32_t rem = key - tz * g.tiles_x * g.tiles_y;
    const uint32_t ty = rem / g.tiles_x, tx = rem - ty * g.tiles_x;
    const uint32_t t = threadIdx.x, lane = t & 31, warp = t >> 5;

    const uint32_t sub_voxels = 32u * PPL;
    uint32_t n_sub = 1;
    while (n_sub * sub_voxels < T * T * T) n_sub <<= 1;
    const uint32_t my_sub = warp % n_sub;
    const uint32_t warps_per_sub = kVoxBwdWarps / n_sub;
    const uint32_t my_group = warp / n_sub;

    S px[PPL], py[PPL], pz[PPL], vr[PPL], vv[PPL];
    bool valid[PPL];
#pragma unroll
    for (int k = 0; k < PPL; ++k) {
        const uint32_t p = my_sub * sub_voxels + lane + 32u * k;
        uint32_t lz, ly, lx;
        tile_voxel(p, T, lz, ly, lx);
        const uint32_t i = tz * T + lz, j = ty * T + ly, kk = tx * T + lx;
        valid[k] = p < T * T * T && i < g.dim0 && j < g.dim1 && kk < g.dim2;
        px[k] = static_cast<S>(kk) + static_cast<S>(0.5);
        py[k] = static_cast<S>(j) + static_cast<S>(0.5);
        pz[k] = static_cast<S>(i) + static_cast<S>(0.5);
        const size_t vid = (size_t(i) * g.dim1 + j) * g.dim2 + kk;
        vr[k] = (valid[k] && v_volume != nullptr) ? v_volume[vid] : S(0);
        vv[k] = (kVar && valid[k]) ? v_volume_var[vid] : S(0);
    }

    const int32_t n_batches = (count + kVoxBwdThreads - 1) / kVoxBwdThreads;
    auto load = [&](int32_t b, int stage) {
        const int32_t idx = start + b * kVoxBwdThreads + int32_t(t);
        if (idx < end) {
            const int32_t gid = flatten_ids[idx];
            gather_record3(s_rec + stage * kVoxBwdThreads + t, records + gid);
            s_id[stage * kVoxBwdThreads + t] = gid;
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
        const int32_t batch = min(int32_t(kVoxBwdThreads), count - b * kVoxBwdThreads);
        for (int32_t s = int32_t(my_group); s < batch; s += int32_t(warps_per_sub)) {
            const Rec3D<S> r = s_rec[stage * kVoxBwdThreads + s];
            const int32_t gid = s_id[stage * kVoxBwdThreads + s];
            const S a = r.c00, p = r.c01, q = r.c02, bb = r.c11, rr = r.c12, c = r.c22;
            const S opac = r.o;
            const S uq = chain_var ? r.q : S(0);
            S gx = 0, gy = 0, gz = 0, go = 0, g0 = 0, g1 = 0, g2 = 0, g3 = 0, g4 = 0, g5 = 0, gb = 0, gq = 0;
#pragma unroll
            for (int k = 0; k < PPL; ++k) {
                if (!kBeta) {
                    const S d1 = px[k] - r.x, d2 = py[k] - r.y, d3 = pz[k] - r.z;
                    const S sigma = static_cast<S>(0.5) * (a * d1 * d1 + bb * d2 * d2 + c * d3 * d3) +
                                    p * d1 * d2 + q * d1 * d3 + rr * d2 * d3;
                    const S vis_raw = exp(-sigma);
                    const S alpha_raw = opac * vis_raw;
                    const bool keep = valid[k] && !(sigma < static_cast<S>(0) || fabs(alpha_raw) < static_cast<S>(1e-6));
                    const S vis = keep ? vis_raw : S(0);
                    const S alpha = keep ? alpha_raw : S(0);
                    S v_O = vr[k];
                    if (kVar) {
                        gq += vv[k] * alpha * alpha;
                        v_O += static_cast<S>(2) * uq * alpha * vv[k];
                    }
                    const S v_sigma = -v_O * opac * vis;
                    const S oI = opac * vis;
                    go += v_O * vis;
                    g0 += v_sigma * static_cast<S>(0.5) * d1 * d1;
                    g1 += v_sigma * d1 * d2;
                    g2 += v_sigma * d1 * d3;
                    g3 += v_sigma * static_cast<S>(0.5) * d2 * d2;
                    g4 += v_sigma * d2 * d3;
                    g5 += v_sigma * static_cast<S>(0.5) * d3 * d3;
                    gx += v_O * oI * (a * d1 + p * d2 + q * d3);
                    gy += v_O * oI * (bb * d2 + p * d1 + rr * d3);
                    gz += v_O * oI * (c * d3 + q * d1 + rr * d2);
                } else {
                    const S d1 = r.x - px[k], d2 = r.y - py[k], d3 = r.z - pz[k];
                    const S qf = a * d1 * d1 + bb * d2 * d2 + c * d3 * d3 + static_cast<S>(2) * p * d1 * d2 +
                                 static_cast<S>(2) * q * d1 * d3 + static_cast<S>(2) * rr * d2 * d3;
                    const S h_raw = static_cast<S>(1) - qf;
                    const bool inside = valid[k] && !(qf < static_cast<S>(0) || h_raw <= static_cast<S>(0));
                    const S h = inside ? h_raw : S(1);  // keeps pow/log finite on skipped samples
                    const S vis_raw = pow(h, r.beta);
                    const S alpha_raw = opac * vis_raw;
                    const bool keep = inside && !(fabs(alpha_raw) < static_cast<S>(1e-5));
                    const S vis = keep ? vis_raw : S(0);
                    const S alpha = keep ? alpha_raw : S(0);
                    S v_O = keep ? vr[k] : S(0);
                    if (kVar) {
                        gq += vv[k] * alpha * alpha;
                        v_O += static_cast<S>(2) * uq * alpha * vv[k];
                    }
                    const S v_q = -opac * r.beta * pow(h, r.beta - static_cast<S>(1)) * v_O;
                    const S wx = a * d1 + p * d2 + q * d3;
                    const S wy = bb * d2 + p * d1 + rr * d3;
                    const S wz = c * d3 + q * d1 + rr * d2;
                    gx += static_cast<S>(2) * v_q * wx;
                    gy += static_cast<S>(2) * v_q * wy;
                    gz += static_cast<S>(2) * v_q * wz;
                    g0 += v_q * d1 * d1;
                    g1 += static_cast<S>(2) * v_q * d1 * d2;
                    g2 += static_cast<S>(2) * v_q * d1 * d3;
                    g3 += v_q * d2 * d2;
                    g4 += static_cast<S>(2) * v_q * d2 * d3;
                    g5 += v_q * d3 * d3;
                    go += v_O * vis;
                    gb += v_O * alpha * log(h);
                }
            }
            gx = warp_sum(gx); gy = warp_sum(gy); gz = warp_sum(gz); go = warp_sum(go);
            g0 = warp_sum(g0); g1 = warp_sum(g1); g2 = warp_sum(g2); g3 = warp_sum(g3);
            g4 = warp_sum(g4); g5 = warp_sum(g5);
            if (kBeta) gb = warp_sum(gb);
            if (kVar) gq = warp_sum(gq);
            S* dst = reinterpret_cast<S*>(grads + gid);
            if (lane == 0) red_add_v4(dst, gx, gy, gz, go);
            if (lane == 1) red_add_v4(dst + 4, g0, g1, g2, g3);
            if (lane == 2) red_add_v4(dst + 8, g4, g5, gb, gq);
        }
        __syncthreads();
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

template <typename S, bool kBeta, bool kVar, int PPT>
int launch_vfwd_t(const VoxelGeom& g, const Rec3D<S>* rec, const int32_t* offsets, const int32_t* ids, S* vol,
                  S* vol_var, unsigned nthreads, cudaStream_t stream) {
    const size_t smem = 2 * nthreads * sizeof(Rec3D<S>);
    if (smem > 48 * 1024)
        cudaFuncSetAttribute(voxel_fwd_kernel<S, kBeta, kVar, PPT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             int(smem));
    const unsigned grid = g.tiles_x * g.tiles_y * g.tiles_z;
    voxel_fwd_kernel<S, kBeta, kVar, PPT><<<grid, nthreads, smem, stream>>>(rec, offsets, ids, g, vol, vol_var);
    return check_launch("voxelize_to_voxels_fwd");
}

template <typename S, bool kBeta, bool kVar>
int launch_vfwd_p(const VoxelGeom& g, const Rec3D<S>* rec, const int32_t* offsets, const int32_t* ids, S* vol,
                  S* vol_var, cudaStream_t stream) {
    const uint32_t voxels = g.T * g.T * g.T;
    if (voxels <= 128) {
        const unsigned nt = (voxels + 31) / 32 * 32;
        return launch_vfwd_t<S, kBeta, kVar, 1>(g, rec, offsets, ids, vol, vol_var, nt, stream);
    }
    const unsigned nt = ((voxels + 3) / 4 + 31) / 32 * 32;
    return launch_vfwd_t<S, kBeta, kVar, 4>(g, rec, offsets, ids, vol, vol_var, nt, stream);
}

template <typename S>
int launch_vfwd(const VoxelGeom& g, const Rec3D<S>* rec, bool beta, const int32_t* offsets, const int32_t* ids,
                S* vol, S* vol_var, cudaStream_t stream) {
    R2S_TRY(check_vgeom(g));
    if (uint64_t(g.tiles_x) * g.tiles_y * g.tiles_z == 0) return R2S_OK;
    const bool var = vol_var != nullptr;
    if (beta) return var ? launch_vfwd_p<S, true, true>(g, rec, offsets, ids, vol, vol_var, stream)
                         : launch_vfwd_p<S, true, false>(g, rec, offsets, ids, vol, vol_var, stream);
    return var ? launch_vfwd_p<S, false, true>(g, rec, offsets, ids, vol, vol_var, stream)
               : launch_vfwd_p<S, false, false>(g, rec, offsets, ids, vol, vol_var, stream);
}

template <typename S, bool kBeta, bool kVar, int PPL>
int launch_vbwd_t(const VoxelGeom& g, const Rec3D<S>* rec, bool chain_var, const int32_t* offsets,
                  const int32_t* ids, const S* v_vol, const S* v_vol_var, Rec3D<S>* grads, cudaStream_t stream) {
    const size_t smem = 2 * kVoxBwdThreads * (sizeof(Rec3D<S>) + sizeof(int32_t));
    if (smem > 48 * 1024)
        cudaFuncSetAttribute(voxel_bwd_kernel<S, kBeta, kVar, PPL>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             int(smem));
    const unsigned grid = g.tiles_x * g.tiles_y * g.tiles_z;
    voxel_bwd_kernel<S, kBeta, kVar, PPL><<<grid, kVoxBwdThreads, smem, stream>>>(rec, chain_var, offsets, ids, g,
                                                                                   v_vol, v_vol_var, grads);
    return check_launch("voxelize_to_voxels_bwd");
}

template <typename S, bool kBeta, bool kVar>
int launch_vbwd_p(const VoxelGeom& g, const Rec3D<S>* rec, bool chain_var, const int32_t* offsets,
                  const int32_t* ids, const S* v_vol, const S* v_vol_var, Rec3D<S>* grads, cudaStream_t stream) {
    if (g.T * g.T * g.T <= 64)
        return launch_vbwd_t<S, kBeta, kVar, 2>(g, rec, chain_var, offsets, ids, v_vol, v_vol_var, grads, stream);
    return launch_vbwd_t<S, kBeta, kVar, 8>(g, rec, chain_var, offsets, ids, v_vol, v_vol_var, grads, stream);
}

template <typename S>
int launch_vbwd(const VoxelGeom& g, const Rec3D<S>* rec, bool beta, bool chain_var, const int32_t* offsets,
                const int32_t* ids, const S* v_vol, const S* v_vol_var, Rec3D<S>* grads, cudaStream_t stream) {
    R2S_TRY(check_vgeom(g));
    if (g.n_isects == 0 || uint64_t(g.tiles_x) * g.tiles_y * g.tiles_z == 0) return R2S_OK;
    const bool var = v_vol_var != nullptr;
    if (beta)
        return var ? launch_vbwd_p<S, true, true>(g, rec, chain_var, offsets, ids, v_vol, v_vol_var, grads, stream)
                   : launch_vbwd_p<S, true, false>(g, rec, chain_var, offsets, ids, v_vol, v_vol_var, grads, stream);
    return var ? launch_vbwd_p<S, false, true>(g, rec, chain_var, offsets, ids, v_vol, v_vol_var, grads, stream)
               : launch_vbwd_p<S, false, false>(g, rec, chain_var, offsets, ids, v_vol, v_vol_var, grads, stream);
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

}  // extern "C"
