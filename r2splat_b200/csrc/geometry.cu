// Geometry kernels: parameter transform, world->image projection, conic/mu,
// world->volume mapping (forward and VJP), plus the fused per-primitive
// kernels of the explicit operators (projection+packing, chain-rule VJPs).
#include "geometry.cuh"

namespace r2s {

constexpr unsigned kThreads = 256;

// --------------------------------------------------------------------------
// Low-level operators
// --------------------------------------------------------------------------

template <typename S>
__global__ void parameter_transform_fwd_kernel(const S* __restrict__ quats, const S* __restrict__ scales,
                                               S* __restrict__ covars, S* __restrict__ max_scales, uint32_t n) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    S q[4], s[3], cov[6], ms;
#pragma unroll
    for (int k = 0; k < 4; ++k) q[k] = quats[size_t(i) * 4 + k];
#pragma unroll
    for (int k = 0; k < 3; ++k) s[k] = scales[size_t(i) * 3 + k];
    covariance_from_parameters(q, s, cov, ms);
#pragma unroll
    for (int k = 0; k < 6; ++k) covars[size_t(i) * 6 + k] = cov[k];
    max_scales[i] = ms;
}

template <typename S>
__global__ void parameter_transform_bwd_kernel(const S* __restrict__ quats, const S* __restrict__ scales,
                                               const S* __restrict__ v_covars, S* __restrict__ v_quats,
                                               S* __restrict__ v_scales, uint32_t n) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    S q[4], s[3], vc[6], vq[4], vs[3];
#pragma unroll
    for (int k = 0; k < 4; ++k) q[k] = quats[size_t(i) * 4 + k];
#pragma unroll
    for (int k = 0; k < 3; ++k) s[k] = scales[size_t(i) * 3 + k];
#pragma unroll
    for (int k = 0; k < 6; ++k) vc[k] = v_covars[size_t(i) * 6 + k];
    covariance_vjp(q, s, vc, vq, vs);
#pragma unroll
    for (int k = 0; k < 4; ++k) v_quats[size_t(i) * 4 + k] = vq[k];
#pragma unroll
    for (int k = 0; k < 3; ++k) v_scales[size_t(i) * 3 + k] = vs[k];
}

// One thread per (camera, primitive); camera-major element order c*N+n.
template <typename S>
__global__ void projection_fwd_kernel(const S* __restrict__ means, const S* __restrict__ covars,
                                      const S* __restrict__ viewmats, const S* __restrict__ Ks,
                                      uint32_t C, uint32_t N, uint32_t width, uint32_t height,
                                      S eps_blur, S radius_clip, S* __restrict__ means2d,
                                      S* __restrict__ cov2d, int32_t* __restrict__ radii) {
    const uint32_t n = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t c = blockIdx.y;
    if (n >= N) return;
    const size_t idx = size_t(c) * N + n;
    const Camera<S> cam = load_camera(viewmats, Ks, c);
    S sig[6];
#pragma unroll
    for (int k = 0; k < 6; ++k) sig[k] = covars[size_t(n) * 6 + k];
    Projected<S> p;
    project(cam, means[size_t(n) * 3 + 0], means[size_t(n) * 3 + 1], means[size_t(n) * 3 + 2], sig,
            width, height, eps_blur, radius_clip, p);
    means2d[idx * 2 + 0] = p.mx;
    means2d[idx * 2 + 1] = p.my;
    S* out = cov2d + idx * 6;
    out[0] = p.c00; out[1] = p.c01; out[2] = p.c02; out[3] = p.c11; out[4] = p.c12; out[5] = p.c22;
    radii[idx * 2 + 0] = p.rx;
    radii[idx * 2 + 1] = p.ry;
}

// One thread per primitive summing its cameras in order (replaces the
// reference's per-camera atomics, WorldToImageProjectionBwd.cu:548-553).
template <typename S>
__global__ void projection_bwd_kernel(const S* __restrict__ means, const S* __restrict__ covars,
                                      const S* __restrict__ viewmats, const S* __restrict__ Ks,
                                      uint32_t C, uint32_t N, uint32_t width, uint32_t height,
                                      const S* __restrict__ v_means2d, const S* __restrict__ v_cov2d,
                                      S* __restrict__ v_means, S* __restrict__ v_covars) {
    const uint32_t n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= N) return;
    S sig[6];
#pragma unroll
    for (int k = 0; k < 6; ++k) sig[k] = covars[size_t(n) * 6 + k];
    const S px = means[size_t(n) * 3 + 0], py = means[size_t(n) * 3 + 1], pz = means[size_t(n) * 3 + 2];
    S acc_p[3] = {0, 0, 0}, acc_s[6] = {0, 0, 0, 0, 0, 0};
    for (uint32_t c = 0; c < C; ++c) {
        const size_t idx = size_t(c) * N + n;
        const Camera<S> cam = load_camera(viewmats, Ks, c);
        S vcov[6], vp[3], vs[6];
#pragma unroll
        for (int k = 0; k < 6; ++k) vcov[k] = v_cov2d[idx * 6 + k];
        if (!project_vjp(cam, px, py, pz, sig, width, height, v_means2d[idx * 2], v_means2d[idx * 2 + 1],
                         vcov, vp, vs)) continue;
#pragma unroll
        for (int k = 0; k < 3; ++k) acc_p[k] += vp[k];
#pragma unroll
        for (int k = 0; k < 6; ++k) acc_s[k] += vs[k];
    }
#pragma unroll
    for (int k = 0; k < 3; ++k) v_means[size_t(n) * 3 + k] = acc_p[k];
#pragma unroll
    for (int k = 0; k < 6; ++k) v_covars[size_t(n) * 6 + k] = acc_s[k];
}

template <typename S>
__global__ void conics_mu_fwd_kernel(const S* __restrict__ cov2d, S eps, S* __restrict__ conics,
                                     S* __restrict__ mus, uint32_t total) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= total) return;
    S cov[6];
#pragma unroll
    for (int k = 0; k < 6; ++k) cov[k] = cov2d[size_t(i) * 6 + k];
    S u11, u12, u22, mu;
    conic_and_mu(cov, eps, u11, u12, u22, mu);
    conics[size_t(i) * 3 + 0] = u11;
    conics[size_t(i) * 3 + 1] = u12;
    conics[size_t(i) * 3 + 2] = u22;
    mus[i] = mu;
}

template <typename S>
__global__ void conics_mu_bwd_kernel(const S* __restrict__ cov2d, const S* __restrict__ conics,
                                     const S* __restrict__ mus, const S* __restrict__ v_conics,
                                     const S* __restrict__ v_mus, S* __restrict__ v_cov2d, uint32_t total) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= total) return;
    S cov[6], vcov[6];
#pragma unroll
    for (int k = 0; k < 6; ++k) cov[k] = cov2d[size_t(i) * 6 + k];
    conic_and_mu_vjp(cov, conics[size_t(i) * 3], conics[size_t(i) * 3 + 1], conics[size_t(i) * 3 + 2], mus[i],
                     v_conics[size_t(i) * 3], v_conics[size_t(i) * 3 + 1], v_conics[size_t(i) * 3 + 2],
                     v_mus[i], vcov);
#pragma unroll
    for (int k = 0; k < 6; ++k) v_cov2d[size_t(i) * 6 + k] = vcov[k];
}

template <typename S>
__global__ void volume_mapping_fwd_kernel(const S* __restrict__ means, const S* __restrict__ covars,
                                          const S* __restrict__ ranges, const S* __restrict__ centers,
                                          uint32_t N, uint32_t dim2, uint32_t dim1, uint32_t dim0, S eps3d,
                                          S radius_clip, S* __restrict__ means_v, S* __restrict__ conics,
                                          int32_t* __restrict__ radii) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    const VolumeFrame<S> f = load_frame(ranges, centers, dim2, dim1, dim0);
    S s[6], m[3], con[6];
    int32_t r[3];
#pragma unroll
    for (int k = 0; k < 6; ++k) s[k] = covars[size_t(i) * 6 + k];
    map_to_volume(f, means[size_t(i) * 3], means[size_t(i) * 3 + 1], means[size_t(i) * 3 + 2], s, eps3d,
                  radius_clip, m, con, r);
#pragma unroll
    for (int k = 0; k < 3; ++k) means_v[size_t(i) * 3 + k] = m[k];
#pragma unroll
    for (int k = 0; k < 6; ++k) conics[size_t(i) * 6 + k] = con[k];
#pragma unroll
    for (int k = 0; k < 3; ++k) radii[size_t(i) * 3 + k] = r[k];
}

template <typename S>
__global__ void volume_mapping_bwd_kernel(const S* __restrict__ covars, const S* __restrict__ ranges,
                                          const S* __restrict__ centers, uint32_t N, uint32_t dim2,
                                          uint32_t dim1, uint32_t dim0, S eps3d,
                                          const S* __restrict__ v_means_v, const S* __restrict__ v_conics,
                                          S* __restrict__ v_means, S* __restrict__ v_covars) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    const VolumeFrame<S> f = load_frame(ranges, centers, dim2, dim1, dim0);
    S s[6], vm[3], vc[6], om[3], oc[6];
#pragma unroll
    for (int k = 0; k < 6; ++k) s[k] = covars[size_t(i) * 6 + k];
#pragma unroll
    for (int k = 0; k < 3; ++k) vm[k] = v_means_v[size_t(i) * 3 + k];
#pragma unroll
    for (int k = 0; k < 6; ++k) vc[k] = v_conics[size_t(i) * 6 + k];
    map_to_volume_vjp(f, s, eps3d, vm, vc, om, oc);
#pragma unroll
    for (int k = 0; k < 3; ++k) v_means[size_t(i) * 3 + k] = om[k];
#pragma unroll
    for (int k = 0; k < 6; ++k) v_covars[size_t(i) * 6 + k] = oc[k];
}

// --------------------------------------------------------------------------
// Fused explicit-path kernels
// --------------------------------------------------------------------------

// Projection, conic/mu and record packing for one (camera, primitive), plus
// its tile rectangle and tile count for the intersection pass.
template <typename S>
__global__ void raster_project_kernel(const S* __restrict__ means, const S* __restrict__ covars,
                                      const S* __restrict__ densities, const S* __restrict__ betas,
                                      const S* __restrict__ ratio, const S* __restrict__ viewmats,
                                      const S* __restrict__ Ks, uint32_t C, uint32_t N, uint32_t width,
                                      uint32_t height, S eps_blur, S eps, S radius_clip, uint32_t tile_size,
                                      uint32_t tiles_x, uint32_t tiles_y, Rec2D<S>* __restrict__ records,
                                      ushort4* __restrict__ rects, int32_t* __restrict__ tiles_per_gauss) {
    const uint32_t n = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t c = blockIdx.y;
    if (n >= N) return;
    const size_t idx = size_t(c) * N + n;
    const Camera<S> cam = load_camera(viewmats, Ks, c);
    S sig[6];
#pragma unroll
    for (int k = 0; k < 6; ++k) sig[k] = covars[size_t(n) * 6 + k];
    Projected<S> p;
    project(cam, means[size_t(n) * 3 + 0], means[size_t(n) * 3 + 1], means[size_t(n) * 3 + 2], sig, width,
            height, eps_blur, radius_clip, p);
    const S cov[6] = {p.c00, p.c01, p.c02, p.c11, p.c12, p.c22};
    Rec2D<S> r;
    S mu;
    conic_and_mu(cov, eps, r.a, r.b, r.c, mu);
    r.x = p.mx;
    r.y = p.my;
    r.o = densities[n];
    if (betas != nullptr) {
        r.mu = mu * ratio[n];
        r.beta = betas[n] + S(0.5);
    } else {
        r.mu = mu;
        r.beta = S(0);
    }
    records[idx] = r;

    // Tile rectangle from the projected centre and radii, exactly as the
    // intersection pass computes it from the stored tensors.
    uint32_t x0 = 0, x1 = 0, y0 = 0, y1 = 0;
    int32_t count = 0;
    if (p.rx > 0 && p.ry > 0 && isfinite(p.mx) && isfinite(p.my)) {
        tile_span(p.mx, static_cast<S>(p.rx), tile_size, tiles_x, x0, x1);
        tile_span(p.my, static_cast<S>(p.ry), tile_size, tiles_y, y0, y1);
        if (x1 > x0 && y1 > y0) {
            count = static_cast<int32_t>((y1 - y0) * (x1 - x0));
        } else {
            x0 = x1 = y0 = y1 = 0;
        }
    }
    rects[idx] = make_ushort4(static_cast<unsigned short>(x0), static_cast<unsigned short>(y0),
                              static_cast<unsigned short>(x1), static_cast<unsigned short>(y1));
    tiles_per_gauss[idx] = count;
}

// Chain rule for the rasterizer: four lanes per primitive, each looping over
// every fourth camera, partial sums combined by shuffles (no atomics). grads
// [C,N,8] holds the adjoints of the packed record slots.
constexpr uint32_t kChainGroup = 4;  // lanes per primitive in the chain-rule pass
constexpr uint32_t kChainThreads = 128;
// Up to this many cameras the block first writes the camera table (extrinsics,
// intrinsics and clamp limits) to shared memory; beyond it each pair loads its
// camera and derives the limits itself.
constexpr uint32_t kChainTableCameras = 256;

template <typename S>
struct CameraEntry {
    Camera<S> cam;
    CameraLimits<S> lim;
};

// Per (camera, primitive) pair: the projection's frame once, the projected
// covariance from it, the conic/mu VJP, then the projection VJP from the same
// frame (the forward projection and its VJP share the camera-space centre,
// Jacobian and camera-space covariance).
template <typename S, bool kTable>
__global__ void __launch_bounds__(kChainThreads) raster_chain_bwd_kernel(
    const S* __restrict__ means, const S* __restrict__ quats, const S* __restrict__ scales,
    const S* __restrict__ covars, const S* __restrict__ ratio, const S* __restrict__ log_grad,
    const S* __restrict__ viewmats, const S* __restrict__ Ks, uint32_t C, uint32_t N, uint32_t width,
    uint32_t height, S eps, const Rec2D<S>* __restrict__ grads, S* __restrict__ v_means, S* __restrict__ v_quats,
    S* __restrict__ v_scales, S* __restrict__ v_densities, S* __restrict__ v_betas) {
    extern __shared__ __align__(16) unsigned char chain_smem[];
    CameraEntry<S>* s_cams = reinterpret_cast<CameraEntry<S>*>(chain_smem);
    if (kTable) {
        for (uint32_t c = threadIdx.x; c < C; c += blockDim.x) {
            CameraEntry<S> e;
            e.cam = load_camera(viewmats, Ks, c);
            e.lim = camera_limits(e.cam, width, height);
            s_cams[c] = e;
        }
        __syncthreads();
    }
    // kChainGroup consecutive lanes share a primitive, each taking every
    // kChainGroup-th camera; their partial sums are combined by shuffles in a
    // fixed order (deterministic).
    const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t part = tid % kChainGroup;
    const bool active = tid / kChainGroup < N;
    const uint32_t n = active ? tid / kChainGroup : N - 1;
    S sig[6];
#pragma unroll
    for (int k = 0; k < 6; ++k) sig[k] = covars[size_t(n) * 6 + k];
    const S px = means[size_t(n) * 3 + 0], py = means[size_t(n) * 3 + 1], pz = means[size_t(n) * 3 + 2];
    const bool is_beta = ratio != nullptr;
    const S beta_ratio = is_beta ? ratio[n] : S(1);
    S acc[12] = {};  // means 0-2, covariance 3-8, density 9, beta 10, mu * mu 11
    S* acc_p = acc;
    S* acc_s = acc + 3;
    S& acc_o = acc[9];
    S& acc_beta = acc[10];
    S& acc_mu_mu = acc[11];
    // The next camera's adjoint record is loaded before this one's arithmetic.
    uint32_t c = active ? part : C;
    Rec2D<S> g_next{};
    if (c < C) g_next = grads[size_t(c) * N + n];
    for (; c < C; c += kChainGroup) {
        const Rec2D<S> g = g_next;
        if (c + kChainGroup < C) g_next = grads[size_t(c + kChainGroup) * N + n];
        acc_o += g.o;
        if (g.x == S(0) && g.y == S(0) && g.a == S(0) && g.b == S(0) && g.c == S(0) && g.mu == S(0) &&
            g.beta == S(0)) continue;
        Camera<S> cam;
        CameraLimits<S> lim;
        if (kTable) {
            cam = s_cams[c].cam;
            lim = s_cams[c].lim;
        } else {
            cam = load_camera(viewmats, Ks, c);
            lim = camera_limits(cam, width, height);
        }
        ProjectionFrame<S> f;
        if (!projection_frame(cam, lim, px, py, pz, sig, f)) {
            // Behind the camera: no covariance, mu = 0; only the Beta slot's
            // own adjoint passes through.
            if (is_beta) acc_beta += g.beta;
            continue;
        }
        S cov[6];
        projection_cov(f, cov);
        S u11, u12, u22, base_mu;
        conic_and_mu(cov, eps, u11, u12, u22, base_mu);
        S v_mu = g.mu;
        if (is_beta) {
            const S mu = base_mu * beta_ratio;
            acc_beta += g.beta;
            acc_mu_mu += g.mu * mu;
            v_mu = g.mu * beta_ratio;
        }
        S vcov[6], vp[3], vs[6];
        conic_and_mu_vjp(cov, u11, u12, u22, base_mu, g.a, g.b, g.c, v_mu, vcov);
        projection_vjp(cam, f, g.x, g.y, vcov, vp, vs);
#pragma unroll
        for (int k = 0; k < 3; ++k) acc_p[k] += vp[k];
#pragma unroll
        for (int k = 0; k < 6; ++k) acc_s[k] += vs[k];
    }
#pragma unroll
    for (int offset = 1; offset < kChainGroup; offset <<= 1) {
#pragma unroll
        for (int k = 0; k < 12; ++k) acc[k] += __shfl_xor_sync(0xffffffffu, acc[k], offset);
    }
    if (!active || part != 0) return;
    S q[4], s[3], vq[4], vsc[3];
#pragma unroll
    for (int k = 0; k < 4; ++k) q[k] = quats[size_t(n) * 4 + k];
#pragma unroll
    for (int k = 0; k < 3; ++k) s[k] = scales[size_t(n) * 3 + k];
    covariance_vjp(q, s, acc_s, vq, vsc);
#pragma unroll
    for (int k = 0; k < 3; ++k) v_means[size_t(n) * 3 + k] = acc_p[k];
#pragma unroll
    for (int k = 0; k < 4; ++k) v_quats[size_t(n) * 4 + k] = vq[k];
#pragma unroll
    for (int k = 0; k < 3; ++k) v_scales[size_t(n) * 3 + k] = vsc[k];
    v_densities[n] = acc_o;
    if (is_beta) v_betas[n] = acc_beta + acc_mu_mu * log_grad[n];
}

// Volume mapping + record packing for one primitive, plus its 3D tile count.
template <typename S>
__global__ void voxel_project_kernel(const S* __restrict__ means, const S* __restrict__ covars,
                                     const S* __restrict__ densities, const S* __restrict__ betas,
                                     const S* __restrict__ uncertainties, const S* __restrict__ ranges,
                                     const S* __restrict__ centers, uint32_t N, uint32_t dim2, uint32_t dim1,
                                     uint32_t dim0, S eps3d, S radius_clip, uint32_t tile_size,
                                     uint32_t tiles_x, uint32_t tiles_y, uint32_t tiles_z,
                                     Rec3D<S>* __restrict__ records, S* __restrict__ means_v,
                                     int32_t* __restrict__ radii, int32_t* __restrict__ tiles_per_gauss) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    const VolumeFrame<S> f = load_frame(ranges, centers, dim2, dim1, dim0);
    S s[6], m[3], con[6];
    int32_t r[3];
#pragma unroll
    for (int k = 0; k < 6; ++k) s[k] = covars[size_t(i) * 6 + k];
    map_to_volume(f, means[size_t(i) * 3], means[size_t(i) * 3 + 1], means[size_t(i) * 3 + 2], s, eps3d,
                  radius_clip, m, con, r);
    Rec3D<S> rec;
    rec.x = m[0]; rec.y = m[1]; rec.z = m[2];
    rec.o = densities[i];
    rec.c00 = con[0]; rec.c01 = con[1]; rec.c02 = con[2]; rec.c11 = con[3]; rec.c12 = con[4]; rec.c22 = con[5];
    rec.beta = betas != nullptr ? betas[i] : S(0);
    rec.q = uncertainties != nullptr ? uncertainties[i] : S(0);
    rec.pad0 = rec.pad1 = rec.pad2 = rec.pad3 = S(0);
    records[i] = rec;
#pragma unroll
    for (int k = 0; k < 3; ++k) means_v[size_t(i) * 3 + k] = m[k];
#pragma unroll
    for (int k = 0; k < 3; ++k) radii[size_t(i) * 3 + k] = r[k];
    int32_t count = 0;
    if (r[0] > 0 && r[1] > 0 && r[2] > 0) {
        uint32_t x0, x1, y0, y1, z0, z1;
        tile_span(m[0], static_cast<S>(r[0]), tile_size, tiles_x, x0, x1);
        tile_span(m[1], static_cast<S>(r[1]), tile_size, tiles_y, y0, y1);
        tile_span(m[2], static_cast<S>(r[2]), tile_size, tiles_z, z0, z1);
        if (x1 > x0 && y1 > y0 && z1 > z0) count = static_cast<int32_t>((z1 - z0) * (y1 - y0) * (x1 - x0));
    }
    tiles_per_gauss[i] = count;
}

// Chain rule for voxelization, one thread per primitive. grads [N] holds the
// tile-accumulated adjoints of the packed record slots.
template <typename S>
__global__ void voxel_chain_bwd_kernel(const S* __restrict__ quats, const S* __restrict__ scales,
                                       const S* __restrict__ covars, const S* __restrict__ ranges,
                                       const S* __restrict__ centers, uint32_t N, uint32_t dim2, uint32_t dim1,
                                       uint32_t dim0, S eps3d, const Rec3D<S>* __restrict__ grads,
                                       S* __restrict__ v_means, S* __restrict__ v_quats,
                                       S* __restrict__ v_scales, S* __restrict__ v_densities,
                                       S* __restrict__ v_betas, S* __restrict__ v_uncertainties) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    const VolumeFrame<S> f = load_frame(ranges, centers, dim2, dim1, dim0);
    const Rec3D<S> g = grads[i];
    S s[6], q[4], sc[3];
#pragma unroll
    for (int k = 0; k < 6; ++k) s[k] = covars[size_t(i) * 6 + k];
    const S vm[3] = {g.x, g.y, g.z};
    const S vc[6] = {g.c00, g.c01, g.c02, g.c11, g.c12, g.c22};
    S om[3], oc[6], vq[4], vs[3];
    map_to_volume_vjp(f, s, eps3d, vm, vc, om, oc);
#pragma unroll
    for (int k = 0; k < 4; ++k) q[k] = quats[size_t(i) * 4 + k];
#pragma unroll
    for (int k = 0; k < 3; ++k) sc[k] = scales[size_t(i) * 3 + k];
    covariance_vjp(q, sc, oc, vq, vs);
#pragma unroll
    for (int k = 0; k < 3; ++k) v_means[size_t(i) * 3 + k] = om[k];
#pragma unroll
    for (int k = 0; k < 4; ++k) v_quats[size_t(i) * 4 + k] = vq[k];
#pragma unroll
    for (int k = 0; k < 3; ++k) v_scales[size_t(i) * 3 + k] = vs[k];
    v_densities[i] = g.o;
    if (v_betas != nullptr) v_betas[i] = g.beta;
    if (v_uncertainties != nullptr) v_uncertainties[i] = g.q;
}

}  // namespace r2s

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------

using namespace r2s;

extern "C" {

int r2s_parameter_transform_fwd(int dtype, const void* quats, const void* scales, void* covars,
                                void* max_scales, uint32_t n, void* stream) {
    if (n == 0) return R2S_OK;
    R2S_DISPATCH(dtype, parameter_transform_fwd_kernel<S><<<blocks_for(n, kThreads), kThreads, 0, as_stream(stream)>>>(
        static_cast<const S*>(quats), static_cast<const S*>(scales), static_cast<S*>(covars),
        static_cast<S*>(max_scales), n));
    return check_launch("parameter_transform_fwd");
}

int r2s_parameter_transform_bwd(int dtype, const void* quats, const void* scales, const void* v_covars,
                                void* v_quats, void* v_scales, uint32_t n, void* stream) {
    if (n == 0) return R2S_OK;
    R2S_DISPATCH(dtype, parameter_transform_bwd_kernel<S><<<blocks_for(n, kThreads), kThreads, 0, as_stream(stream)>>>(
        static_cast<const S*>(quats), static_cast<const S*>(scales), static_cast<const S*>(v_covars),
        static_cast<S*>(v_quats), static_cast<S*>(v_scales), n));
    return check_launch("parameter_transform_bwd");
}

int r2s_world_to_image_projection_fwd(int dtype, const void* means, const void* covars, const void* viewmats,
                                      const void* Ks, uint32_t C, uint32_t N, uint32_t width, uint32_t height,
                                      float eps_blur, float radius_clip, void* means2d, void* cov2d,
                                      int32_t* radii, void* stream) {
    if (C == 0 || N == 0) return R2S_OK;
    R2S_REQUIRE(C <= 65535, R2S_ERR_UNSUPPORTED, "camera count exceeds 65535");
    dim3 grid(blocks_for(N, kThreads), C);
    R2S_DISPATCH(dtype, projection_fwd_kernel<S><<<grid, kThreads, 0, as_stream(stream)>>>(
        static_cast<const S*>(means), static_cast<const S*>(covars), static_cast<const S*>(viewmats),
        static_cast<const S*>(Ks), C, N, width, height, static_cast<S>(eps_blur), static_cast<S>(radius_clip),
        static_cast<S*>(means2d), static_cast<S*>(cov2d), radii));
    return check_launch("world_to_image_projection_fwd");
}

int r2s_world_to_image_projection_bwd(int dtype, const void* means, const void* covars, const void* viewmats,
                                      const void* Ks, uint32_t C, uint32_t N, uint32_t width, uint32_t height,
                                      const void* v_means2d, const void* v_cov2d, void* v_means,
                                      void* v_covars, void* stream) {
    if (N == 0) return R2S_OK;
    R2S_DISPATCH(dtype, projection_bwd_kernel<S><<<blocks_for(N, 128), 128, 0, as_stream(stream)>>>(
        static_cast<const S*>(means), static_cast<const S*>(covars), static_cast<const S*>(viewmats),
        static_cast<const S*>(Ks), C, N, width, height, static_cast<const S*>(v_means2d),
        static_cast<const S*>(v_cov2d), static_cast<S*>(v_means), static_cast<S*>(v_covars)));
    return check_launch("world_to_image_projection_bwd");
}

int r2s_conics_mu_fwd(int dtype, const void* cov2d, uint32_t total, double eps, void* conics, void* mus,
                      void* stream) {
    if (total == 0) return R2S_OK;
    R2S_DISPATCH(dtype, conics_mu_fwd_kernel<S><<<blocks_for(total, kThreads), kThreads, 0, as_stream(stream)>>>(
        static_cast<const S*>(cov2d), static_cast<S>(eps), static_cast<S*>(conics), static_cast<S*>(mus), total));
    return check_launch("conics_mu_fwd");
}

int r2s_conics_mu_bwd(int dtype, const void* cov2d, uint32_t total, double eps, const void* conics,
                      const void* mus, const void* v_conics, const void* v_mus, void* v_cov2d, void* stream) {
    (void)eps;
    if (total == 0) return R2S_OK;
    R2S_DISPATCH(dtype, conics_mu_bwd_kernel<S><<<blocks_for(total, kThreads), kThreads, 0, as_stream(stream)>>>(
        static_cast<const S*>(cov2d), static_cast<const S*>(conics), static_cast<const S*>(mus),
        static_cast<const S*>(v_conics), static_cast<const S*>(v_mus), static_cast<S*>(v_cov2d), total));
    return check_launch("conics_mu_bwd");
}

int r2s_world_to_volume_mapping_fwd(int dtype, const void* means, const void* covars, const void* ranges,
                                    const void* centers, uint32_t N, uint32_t dim2, uint32_t dim1, uint32_t dim0,
                                    double eps3d, double radius_clip, void* means3d_v, void* conics,
                                    int32_t* radii, void* stream) {
    if (N == 0) return R2S_OK;
    R2S_DISPATCH(dtype, volume_mapping_fwd_kernel<S><<<blocks_for(N, kThreads), kThreads, 0, as_stream(stream)>>>(
        static_cast<const S*>(means), static_cast<const S*>(covars), static_cast<const S*>(ranges),
        static_cast<const S*>(centers), N, dim2, dim1, dim0, static_cast<S>(eps3d), static_cast<S>(radius_clip),
        static_cast<S*>(means3d_v), static_cast<S*>(conics), radii));
    return check_launch("world_to_volume_mapping_fwd");
}

int r2s_world_to_volume_mapping_bwd(int dtype, const void* means, const void* covars, const void* ranges,
                                    const void* centers, uint32_t N, uint32_t dim2, uint32_t dim1, uint32_t dim0,
                                    double eps3d, const void* v_means3d_v, const void* v_conics, void* v_means,
                                    void* v_covars, void* stream) {
    (void)means;
    if (N == 0) return R2S_OK;
    R2S_DISPATCH(dtype, volume_mapping_bwd_kernel<S><<<blocks_for(N, kThreads), kThreads, 0, as_stream(stream)>>>(
        static_cast<const S*>(covars), static_cast<const S*>(ranges), static_cast<const S*>(centers), N, dim2,
        dim1, dim0, static_cast<S>(eps3d), static_cast<const S*>(v_means3d_v), static_cast<const S*>(v_conics),
        static_cast<S*>(v_means), static_cast<S*>(v_covars)));
    return check_launch("world_to_volume_mapping_bwd");
}

int r2s_raster_project(int dtype, const void* means, const void* covars, const void* densities, const void* betas,
                       const void* ratio, const void* viewmats, const void* Ks, uint32_t C, uint32_t N,
                       uint32_t width, uint32_t height, float eps_blur, double eps, float radius_clip,
                       uint32_t tile_size, uint32_t tiles_x, uint32_t tiles_y, void* records, uint16_t* rects,
                       int32_t* tiles_per_gauss, void* stream) {
    if (C == 0 || N == 0) return R2S_OK;
    R2S_REQUIRE(C <= 65535, R2S_ERR_UNSUPPORTED, "camera count exceeds 65535");
    R2S_REQUIRE(tiles_x <= 65535 && tiles_y <= 65535, R2S_ERR_UNSUPPORTED, "more than 65535 tiles along an axis");
    R2S_REQUIRE((betas == nullptr) == (ratio == nullptr), R2S_ERR_ARGUMENT, "betas and ratio go together");
    dim3 grid(blocks_for(N, kThreads), C);
    R2S_DISPATCH(dtype, raster_project_kernel<S><<<grid, kThreads, 0, as_stream(stream)>>>(
        static_cast<const S*>(means), static_cast<const S*>(covars), static_cast<const S*>(densities),
        static_cast<const S*>(betas), static_cast<const S*>(ratio), static_cast<const S*>(viewmats),
        static_cast<const S*>(Ks), C, N, width, height, static_cast<S>(eps_blur), static_cast<S>(eps),
        static_cast<S>(radius_clip), tile_size, tiles_x, tiles_y, static_cast<Rec2D<S>*>(records),
        reinterpret_cast<ushort4*>(rects), tiles_per_gauss));
    return check_launch("raster_project");
}

int r2s_raster_chain_bwd(int dtype, const void* means, const void* quats, const void* scales, const void* covars,
                         const void* betas, const void* ratio, const void* log_grad, const void* viewmats,
                         const void* Ks, uint32_t C, uint32_t N, uint32_t width, uint32_t height, float eps_blur,
                         double eps, const void* grads, void* v_means, void* v_quats, void* v_scales,
                         void* v_densities, void* v_betas, void* stream) {
    if (N == 0) return R2S_OK;
    const bool beta = betas != nullptr;
    R2S_REQUIRE(!beta || (ratio != nullptr && log_grad != nullptr && v_betas != nullptr), R2S_ERR_ARGUMENT,
                "Beta chain rule needs ratio, log_grad and v_betas");
    (void)eps_blur;  // only the pixel radii depend on it, and the chain rule does not use them
    R2S_DISPATCH(dtype, {
        const unsigned blocks = blocks_for(uint64_t(N) * kChainGroup, kChainThreads);
        const auto* mp = static_cast<const S*>(means);
        const auto* qp = static_cast<const S*>(quats);
        const auto* sp = static_cast<const S*>(scales);
        const auto* cp = static_cast<const S*>(covars);
        const auto* rp = beta ? static_cast<const S*>(ratio) : nullptr;
        const auto* lp = beta ? static_cast<const S*>(log_grad) : nullptr;
        const auto* vm = static_cast<const S*>(viewmats);
        const auto* kp = static_cast<const S*>(Ks);
        const auto* gp = static_cast<const Rec2D<S>*>(grads);
        if (C <= kChainTableCameras) {
            const size_t smem = size_t(C) * sizeof(CameraEntry<S>);
            R2S_TRY(allow_dynamic_smem(raster_chain_bwd_kernel<S, true>, smem));
            raster_chain_bwd_kernel<S, true><<<blocks, kChainThreads, smem, as_stream(stream)>>>(
                mp, qp, sp, cp, rp, lp, vm, kp, C, N, width, height, static_cast<S>(eps), gp, static_cast<S*>(v_means),
                static_cast<S*>(v_quats), static_cast<S*>(v_scales), static_cast<S*>(v_densities),
                static_cast<S*>(v_betas));
        } else {
            raster_chain_bwd_kernel<S, false><<<blocks, kChainThreads, 0, as_stream(stream)>>>(
                mp, qp, sp, cp, rp, lp, vm, kp, C, N, width, height, static_cast<S>(eps), gp, static_cast<S*>(v_means),
                static_cast<S*>(v_quats), static_cast<S*>(v_scales), static_cast<S*>(v_densities),
                static_cast<S*>(v_betas));
        }
    });
    return check_launch("raster_chain_bwd");
}

int r2s_voxel_project(int dtype, const void* means, const void* covars, const void* densities, const void* betas,
                      const void* uncertainties, const void* ranges, const void* centers, uint32_t N,
                      uint32_t dim2, uint32_t dim1, uint32_t dim0, double eps3d, double radius_clip,
                      uint32_t tile_size, uint32_t tiles_x, uint32_t tiles_y, uint32_t tiles_z, void* records,
                      void* means_v, int32_t* radii, int32_t* tiles_per_gauss, void* stream) {
    if (N == 0) return R2S_OK;
    R2S_DISPATCH(dtype, voxel_project_kernel<S><<<blocks_for(N, kThreads), kThreads, 0, as_stream(stream)>>>(
        static_cast<const S*>(means), static_cast<const S*>(covars), static_cast<const S*>(densities),
        static_cast<const S*>(betas), static_cast<const S*>(uncertainties), static_cast<const S*>(ranges),
        static_cast<const S*>(centers), N, dim2, dim1, dim0, static_cast<S>(eps3d), static_cast<S>(radius_clip),
        tile_size, tiles_x, tiles_y, tiles_z, static_cast<Rec3D<S>*>(records), static_cast<S*>(means_v), radii,
        tiles_per_gauss));
    return check_launch("voxel_project");
}

int r2s_voxel_chain_bwd(int dtype, const void* means, const void* quats, const void* scales, const void* covars,
                        const void* ranges, const void* centers, uint32_t N, uint32_t dim2, uint32_t dim1,
                        uint32_t dim0, double eps3d, const void* grads, void* v_means, void* v_quats,
                        void* v_scales, void* v_densities, void* v_betas, void* v_uncertainties, void* stream) {
    (void)means;
    if (N == 0) return R2S_OK;
    R2S_DISPATCH(dtype, voxel_chain_bwd_kernel<S><<<blocks_for(N, kThreads), kThreads, 0, as_stream(stream)>>>(
        static_cast<const S*>(quats), static_cast<const S*>(scales), static_cast<const S*>(covars),
        static_cast<const S*>(ranges), static_cast<const S*>(centers), N, dim2, dim1, dim0, static_cast<S>(eps3d),
        static_cast<const Rec3D<S>*>(grads), static_cast<S*>(v_means), static_cast<S*>(v_quats),
        static_cast<S*>(v_scales), static_cast<S*>(v_densities), static_cast<S*>(v_betas),
        static_cast<S*>(v_uncertainties)));
    return check_launch("voxel_chain_bwd");
}

}  // extern "C"
