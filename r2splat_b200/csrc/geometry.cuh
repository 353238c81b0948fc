// Per-primitive geometry math shared by the geometry kernels.
//
// Numerics note: the tile lists (tile counts, sorted keys and ids) must be
// bit-identical to the reference build, and those depend on the projected
// centre and the diagonal of the projected covariance. The expressions below
// therefore keep the reference's operation order and association
// (WorldToImageProjectionFwd.cu:124-282, ConicsMuFwd.cu:55-103,
// WorldToVolumeMappingFwd.cu:79-156, ParameterTransform.cuh:10-73) and the
// library is compiled with the same fast-math flags, so the compiler emits the
// same rounding for every step. Do not refactor these expressions for style.
#pragma once

#include "common.cuh"

namespace r2s {

// --------------------------------------------------------------------------
// Parameter transform: raw quaternion (wxyz) and physical scales -> packed
// covariance (00, 01, 02, 11, 12, 22).
// --------------------------------------------------------------------------

__device__ __forceinline__ float exact_div(float a, float b) {
    float r;
    asm("div.rn.f32 %0, %1, %2;" : "=f"(r) : "f"(a), "f"(b));
    return r;
}
__device__ __forceinline__ double exact_div(double a, double b) { return __ddiv_rn(a, b); }
__device__ __forceinline__ float exact_sqrt(float v) { return __fsqrt_rn(v); }
__device__ __forceinline__ double exact_sqrt(double v) { return __dsqrt_rn(v); }

__device__ __forceinline__ float largest_magnitude(const float* v) {
    // Non-negative IEEE-754 bit patterns order like their values, including
    // subnormals that a flush-to-zero float compare would lose.
    unsigned bits = 0;
#pragma unroll
    for (int i = 0; i < 4; ++i) bits = max(bits, __float_as_uint(v[i]) & 0x7fffffffu);
    return __uint_as_float(bits);
}
__device__ __forceinline__ double largest_magnitude(const double* v) {
    return fmax(fmax(fabs(v[0]), fabs(v[1])), fmax(fabs(v[2]), fabs(v[3])));
}

// Unit quaternion from raw input; also returns the two normalisation factors
// (largest magnitude, then the norm of the pre-scaled vector).
template <typename S>
__device__ __forceinline__ void unit_quaternion(const S* raw, S* q, S& magnitude, S& scaled_norm) {
    magnitude = largest_magnitude(raw);
    S norm_sq = 0;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        q[i] = exact_div(raw[i], magnitude);
        norm_sq += q[i] * q[i];
    }
    scaled_norm = exact_sqrt(norm_sq);
#pragma unroll
    for (int i = 0; i < 4; ++i) q[i] = exact_div(q[i], scaled_norm);
}

template <typename S>
__device__ __forceinline__ void rotation_from_unit(const S* q, S R[3][3]) {
    const S w = q[0], x = q[1], y = q[2], z = q[3];
    R[0][0] = S(1) - S(2) * (y * y + z * z);
    R[0][1] = S(2) * (x * y - w * z);
    R[0][2] = S(2) * (x * z + w * y);
    R[1][0] = S(2) * (x * y + w * z);
    R[1][1] = S(1) - S(2) * (x * x + z * z);
    R[1][2] = S(2) * (y * z - w * x);
    R[2][0] = S(2) * (x * z - w * y);
    R[2][1] = S(2) * (y * z + w * x);
    R[2][2] = S(1) - S(2) * (x * x + y * y);
}

template <typename S>
__device__ __forceinline__ void covariance_from_parameters(const S* raw_q, const S* s, S* cov, S& max_scale) {
    S q[4], magnitude, scaled_norm;
    unit_quaternion(raw_q, q, magnitude, scaled_norm);
    S R[3][3];
    rotation_from_unit(q, R);
    max_scale = max(s[0], max(s[1], s[2]));
    int packed = 0;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
#pragma unroll
        for (int j = i; j < 3; ++j) {
            S value = 0;
#pragma unroll
            for (int k = 0; k < 3; ++k) value += R[i][k] * R[j][k] * s[k] * s[k];
            cov[packed++] = value;
        }
    }
}

// VJP of covariance_from_parameters back to the raw quaternion and scales
// (ParameterTransformBwd.cu:17-70): the packed off-diagonals appear once, so
// their adjoint is split evenly over the two symmetric entries.
template <typename S>
__device__ __forceinline__ void covariance_vjp(const S* raw_q, const S* s, const S* vc, S* vq, S* vs) {
    S q[4], magnitude, scaled_norm;
    unit_quaternion(raw_q, q, magnitude, scaled_norm);
    const S w = q[0], x = q[1], y = q[2], z = q[3];
    S R[3][3];
    rotation_from_unit(q, R);
    const S G[3][3] = {
        {vc[0], S(0.5) * vc[1], S(0.5) * vc[2]},
        {S(0.5) * vc[1], vc[3], S(0.5) * vc[4]},
        {S(0.5) * vc[2], S(0.5) * vc[4], vc[5]}};
    S vR[3][3];
#pragma unroll
    for (int j = 0; j < 3; ++j) {
        S scale_gradient = 0;
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            S vM = 0;
#pragma unroll
            for (int k = 0; k < 3; ++k) vM += G[i][k] * R[k][j];
            vM *= S(2) * s[j];
            vR[i][j] = vM * s[j];
            scale_gradient += R[i][j] * vM;
        }
        vs[j] = scale_gradient;
    }
    const S g[4] = {
        S(2) * (x * (vR[2][1] - vR[1][2]) + y * (vR[0][2] - vR[2][0]) + z * (vR[1][0] - vR[0][1])),
        S(2) * (-S(2) * x * (vR[1][1] + vR[2][2]) + y * (vR[0][1] + vR[1][0]) +
                z * (vR[0][2] + vR[2][0]) + w * (vR[2][1] - vR[1][2])),
        S(2) * (x * (vR[0][1] + vR[1][0]) - S(2) * y * (vR[0][0] + vR[2][2]) +
                z * (vR[1][2] + vR[2][1]) + w * (vR[0][2] - vR[2][0])),
        S(2) * (x * (vR[0][2] + vR[2][0]) + y * (vR[1][2] + vR[2][1]) -
                S(2) * z * (vR[0][0] + vR[1][1]) + w * (vR[1][0] - vR[0][1]))};
    S q_dot_g = 0;
#pragma unroll
    for (int i = 0; i < 4; ++i) q_dot_g += q[i] * g[i];
#pragma unroll
    for (int i = 0; i < 4; ++i) vq[i] = exact_div(exact_div(g[i] - q[i] * q_dot_g, scaled_norm), magnitude);
}

// --------------------------------------------------------------------------
// World -> image projection of one (camera, primitive) pair.
// --------------------------------------------------------------------------

template <typename S>
struct Projected {
    S mx, my;                         // projected centre
    S c00, c01, c02, c11, c12, c22;   // projected 3x3 covariance (two pixel axes + ray axis)
    int32_t rx, ry;                   // rectangular pixel radii (0 = culled)
    bool front;                       // z > 0.01
};

template <typename S>
struct Camera {
    S R00, R01, R02, R10, R11, R12, R20, R21, R22, t0, t1, t2, fx, fy, cx, cy;
};

template <typename S>
__device__ __forceinline__ Camera<S> load_camera(const S* viewmats, const S* Ks, uint32_t c) {
    const S* vm = viewmats + size_t(c) * 16;
    const S* K = Ks + size_t(c) * 9;
    Camera<S> cam;
    cam.R00 = vm[0]; cam.R01 = vm[1]; cam.R02 = vm[2];
    cam.R10 = vm[4]; cam.R11 = vm[5]; cam.R12 = vm[6];
    cam.R20 = vm[8]; cam.R21 = vm[9]; cam.R22 = vm[10];
    cam.t0 = vm[3]; cam.t1 = vm[7]; cam.t2 = vm[11];
    cam.fx = K[0]; cam.fy = K[4]; cam.cx = K[2]; cam.cy = K[5];
    return cam;
}

template <typename S>
__device__ __forceinline__ void project(
    const Camera<S>& cam, S px, S py, S pz, const S* sig, uint32_t width, uint32_t height,
    S eps_blur, S radius_clip, Projected<S>& out
) {
    const S R00 = cam.R00, R01 = cam.R01, R02 = cam.R02;
    const S R10 = cam.R10, R11 = cam.R11, R12 = cam.R12;
    const S R20 = cam.R20, R21 = cam.R21, R22 = cam.R22;
    const S fx = cam.fx, fy = cam.fy, cx = cam.cx, cy = cam.cy;

    const S x = R00 * px + R01 * py + R02 * pz + cam.t0;
    const S y = R10 * px + R11 * py + R12 * pz + cam.t1;
    const S z = R20 * px + R21 * py + R22 * pz + cam.t2;
    if (z <= static_cast<S>(0.01)) {
        out.mx = out.my = S(0);
        out.c00 = out.c01 = out.c02 = out.c11 = out.c12 = out.c22 = S(0);
        out.rx = out.ry = 0;
        out.front = false;
        return;
    }
    out.front = true;
    const S rz = static_cast<S>(1) / z;
    const S rz2 = rz * rz;
    out.mx = fx * x * rz + cx;
    out.my = fy * y * rz + cy;

    const S Wd = static_cast<S>(width);
    const S Hd = static_cast<S>(height);
    const S tan_fovx = static_cast<S>(0.5) * Wd / fx;
    const S tan_fovy = static_cast<S>(0.5) * Hd / fy;
    const S lim_x_pos = (Wd - cx) / fx + static_cast<S>(0.3) * tan_fovx;
    const S lim_x_neg = cx / fx + static_cast<S>(0.3) * tan_fovx;
    const S lim_y_pos = (Hd - cy) / fy + static_cast<S>(0.3) * tan_fovy;
    const S lim_y_neg = cy / fy + static_cast<S>(0.3) * tan_fovy;
    const S tx = z * min(lim_x_pos, max(-lim_x_neg, x * rz));
    const S ty = z * min(lim_y_pos, max(-lim_y_neg, y * rz));

    const S l = sqrt(tx * tx + ty * ty + z * z);
    const S rl = static_cast<S>(1) / l;
    const S J00 = fx * rz;
    const S J02 = -fx * tx * rz2;
    const S J11 = fy * rz;
    const S J12 = -fy * ty * rz2;
    const S J20 = tx * rl;
    const S J21 = ty * rl;
    const S J22 = z * rl;

    const S s00 = sig[0], s01 = sig[1], s02 = sig[2], s11 = sig[3], s12 = sig[4], s22 = sig[5];
    // M = Sigma R^T, then Sigma_c = R M.
    const S M00 = s00*R00 + s01*R01 + s02*R02;
    const S M01 = s00*R10 + s01*R11 + s02*R12;
    const S M02 = s00*R20 + s01*R21 + s02*R22;
    const S M10 = s01*R00 + s11*R01 + s12*R02;
    const S M11 = s01*R10 + s11*R11 + s12*R12;
    const S M12 = s01*R20 + s11*R21 + s12*R22;
    const S M20 = s02*R00 + s12*R01 + s22*R02;
    const S M21 = s02*R10 + s12*R11 + s22*R12;
    const S M22 = s02*R20 + s12*R21 + s22*R22;
    const S Sc00 = R00*M00 + R01*M10 + R02*M20;
    const S Sc01 = R00*M01 + R01*M11 + R02*M21;
    const S Sc02 = R00*M02 + R01*M12 + R02*M22;
    const S Sc11 = R10*M01 + R11*M11 + R12*M21;
    const S Sc12 = R10*M02 + R11*M12 + R12*M22;
    const S Sc22 = R20*M02 + R21*M12 + R22*M22;
    // N = Sigma_c J^T (J01 = J10 = 0), then J N.
    const S N00 = Sc00*J00 +              Sc02*J02;
    const S N01 = Sc00*static_cast<S>(0) + Sc01*J11 + Sc02*J12;
    const S N02 = Sc00*J20 + Sc01*J21 + Sc02*J22;
    const S N10 = Sc01*J00 +              Sc12*J02;
    const S N11 = Sc01*static_cast<S>(0) + Sc11*J11 + Sc12*J12;
    const S N12 = Sc01*J20 + Sc11*J21 + Sc12*J22;
    const S N20 = Sc02*J00 +              Sc22*J02;
    const S N21 = Sc02*static_cast<S>(0) + Sc12*J11 + Sc22*J12;
    const S N22 = Sc02*J20 + Sc12*J21 + Sc22*J22;
    const S C00 = J00*N00 +              J02*N20;
    const S C01 = J00*N01 +              J02*N21;
    const S C02 = J00*N02 +              J02*N22;
    const S C11 =              J11*N11 + J12*N21;
    const S C12 =              J11*N12 + J12*N22;
    const S C22 = J20*N02 + J21*N12 + J22*N22;
    (void)N10;
    out.c00 = C00; out.c01 = C01; out.c02 = C02; out.c11 = C11; out.c12 = C12; out.c22 = C22;

    // Rectangular radii from the blurred 2x2 block (non-differentiable).
    out.rx = out.ry = 0;
    const S a_blur = C00 + eps_blur;
    const S d_blur = C11 + eps_blur;
    const S b_off = C01;
    const S det_blur = a_blur * d_blur - b_off * b_off;
    if (det_blur <= static_cast<S>(0)) return;
    const S radius_x = ceil(radius_clip * sqrt(max(static_cast<S>(0), a_blur)));
    const S radius_y = ceil(radius_clip * sqrt(max(static_cast<S>(0), d_blur)));
    if (!isfinite(radius_x) || !isfinite(radius_y) ||
        radius_x <= static_cast<S>(0) || radius_y <= static_cast<S>(0)) return;
    const S mean_x = out.mx;
    const S mean_y = out.my;
    if (mean_x + radius_x <= static_cast<S>(0) || mean_x - radius_x >= static_cast<S>(width) ||
        mean_y + radius_y <= static_cast<S>(0) || mean_y - radius_y >= static_cast<S>(height)) return;
    out.rx = static_cast<int32_t>(radius_x);
    out.ry = static_cast<int32_t>(radius_y);
}

// Conic (inverse of the blurred 2x2 footprint, scale-normalised) and the
// Gaussian path factor mu = sqrt(2 pi (f + eps - [c e] P [c e]^T))
// (ConicsMuFwd.cu:47-103). Returns false (all zeros) for degenerate input.
template <typename S>
__device__ __forceinline__ bool conic_and_mu(const S* cov, S eps, S& u11, S& u12, S& u22, S& mu) {
    const S a = cov[0], b = cov[1], c = cov[2], d = cov[3], e = cov[4], f = cov[5];
    const S ab = a + eps;
    const S db = d + eps;
    const S fb = f + eps;
    const S scale = fmax(fmax(fabs(ab), fabs(db)), fabs(b));
    const S an = ab / scale;
    const S bn = b / scale;
    const S dn = db / scale;
    const S determinant = an * dn - bn * bn;
    const S p11 = (dn / determinant) / scale;
    const S p12 = (-bn / determinant) / scale;
    const S p22 = (an / determinant) / scale;
    if (!(ab > static_cast<S>(0) && db > static_cast<S>(0) && determinant > static_cast<S>(0)) ||
        !isfinite(p11) || !isfinite(p12) || !isfinite(p22)) {
        u11 = u12 = u22 = mu = S(0);
        return false;
    }
    u11 = p11; u12 = p12; u22 = p22;
    const S w0 = p11 * c + p12 * e;
    const S w1 = p12 * c + p22 * e;
    const S ratio = fb - c * w0 - e * w1;
    if (ratio > static_cast<S>(0) && isfinite(ratio)) {
        mu = sqrt(static_cast<S>(6.283185307179586476925286766559) * ratio);
    } else {
        mu = S(0);
    }
    return true;
}

// VJP of conic_and_mu using the saved conic and mu (ConicsMuBwd.cu:71-120).
template <typename S>
__device__ __forceinline__ void conic_and_mu_vjp(
    const S* cov, S u11, S u12, S u22, S mu, S v_u11, S v_u12, S v_u22, S v_mu, S* v_cov
) {
    if (u11 == S(0) && u12 == S(0) && u22 == S(0)) {
#pragma unroll
        for (int i = 0; i < 6; ++i) v_cov[i] = S(0);
        return;
    }
    S grad_a = -(v_u11 * u11 * u11 + v_u12 * u11 * u12 + v_u22 * u12 * u12);
    S grad_b = -(v_u11 * static_cast<S>(2) * u11 * u12
              + v_u12 * u11 * u22 + v_u12 * u12 * u12
              + v_u22 * static_cast<S>(2) * u12 * u22);
    S grad_c = S(0);
    S grad_d = -(v_u11 * u12 * u12 + v_u12 * u12 * u22 + v_u22 * u22 * u22);
    S grad_e = S(0);
    S grad_f = S(0);
    if (mu > S(0)) {
        const S w0 = u11 * cov[2] + u12 * cov[4];
        const S w1 = u12 * cov[2] + u22 * cov[4];
        const S v_s = (static_cast<S>(3.141592653589793238462643383279) / mu) * v_mu;
        grad_a += v_s * w0 * w0;
        grad_b += v_s * static_cast<S>(2) * w0 * w1;
        grad_c -= v_s * static_cast<S>(2) * w0;
        grad_d += v_s * w1 * w1;
        grad_e -= v_s * static_cast<S>(2) * w1;
        grad_f += v_s;
    }
    v_cov[0] = grad_a; v_cov[1] = grad_b; v_cov[2] = grad_c;
    v_cov[3] = grad_d; v_cov[4] = grad_e; v_cov[5] = grad_f;
}

// Clamp limits of the normalised image coordinates x/z, y/z used for the
// Jacobian (the same expressions as in project()): they depend only on the
// intrinsics and the image size, so per-camera tables can hold them.
template <typename S>
struct CameraLimits {
    S x_pos, x_neg, y_pos, y_neg;
};

template <typename S>
__device__ __forceinline__ CameraLimits<S> camera_limits(const Camera<S>& cam, uint32_t width, uint32_t height) {
    const S Wd = static_cast<S>(width);
    const S Hd = static_cast<S>(height);
    const S tan_fovx = static_cast<S>(0.5) * Wd / cam.fx;
    const S tan_fovy = static_cast<S>(0.5) * Hd / cam.fy;
    CameraLimits<S> lim;
    lim.x_pos = (Wd - cam.cx) / cam.fx + static_cast<S>(0.3) * tan_fovx;
    lim.x_neg = cam.cx / cam.fx + static_cast<S>(0.3) * tan_fovx;
    lim.y_pos = (Hd - cam.cy) / cam.fy + static_cast<S>(0.3) * tan_fovy;
    lim.y_neg = cam.cy / cam.fy + static_cast<S>(0.3) * tan_fovy;
    return lim;
}

// The intermediates of the projection of one (camera, primitive) pair that
// both its covariance and its VJP use: camera-space centre, clamped centre,
// Jacobian and camera-space covariance.
template <typename S>
struct ProjectionFrame {
    S x, y, z, rz, rz2, tx, ty, rl;
    S J00, J02, J11, J12, J20, J21, J22;
    S Sc00, Sc01, Sc02, Sc11, Sc12, Sc22;
    bool x_clipped, y_clipped;
};

// Fills f; false when the pair is behind the camera (z <= 0.01).
template <typename S>
__device__ __forceinline__ bool projection_frame(const Camera<S>& cam, const CameraLimits<S>& lim, S px, S py, S pz,
                                                 const S* sig, ProjectionFrame<S>& f) {
    const S R00 = cam.R00, R01 = cam.R01, R02 = cam.R02;
    const S R10 = cam.R10, R11 = cam.R11, R12 = cam.R12;
    const S R20 = cam.R20, R21 = cam.R21, R22 = cam.R22;
    const S s00 = sig[0], s01 = sig[1], s02 = sig[2], s11 = sig[3], s12 = sig[4], s22 = sig[5];

    const S x = R00 * px + R01 * py + R02 * pz + cam.t0;
    const S y = R10 * px + R11 * py + R12 * pz + cam.t1;
    const S z = R20 * px + R21 * py + R22 * pz + cam.t2;
    if (z <= static_cast<S>(0.01)) return false;
    const S rz = static_cast<S>(1) / z;
    const S rz2 = rz * rz;
    const S xrz = x * rz;
    const S yrz = y * rz;
    const S tx = z * min(lim.x_pos, max(-lim.x_neg, xrz));
    const S ty = z * min(lim.y_pos, max(-lim.y_neg, yrz));
    f.x_clipped = (xrz > lim.x_pos) || (xrz < -lim.x_neg);
    f.y_clipped = (yrz > lim.y_pos) || (yrz < -lim.y_neg);
    const S l = sqrt(tx * tx + ty * ty + z * z);
    const S rl = static_cast<S>(1) / l;
    f.x = x; f.y = y; f.z = z; f.rz = rz; f.rz2 = rz2; f.tx = tx; f.ty = ty; f.rl = rl;
    f.J00 = cam.fx * rz;
    f.J02 = -cam.fx * tx * rz2;
    f.J11 = cam.fy * rz;
    f.J12 = -cam.fy * ty * rz2;
    f.J20 = tx * rl;
    f.J21 = ty * rl;
    f.J22 = z * rl;

    const S M00 = s00*R00 + s01*R01 + s02*R02;
    const S M01 = s00*R10 + s01*R11 + s02*R12;
    const S M02 = s00*R20 + s01*R21 + s02*R22;
    const S M10 = s01*R00 + s11*R01 + s12*R02;
    const S M11 = s01*R10 + s11*R11 + s12*R12;
    const S M12 = s01*R20 + s11*R21 + s12*R22;
    const S M20 = s02*R00 + s12*R01 + s22*R02;
    const S M21 = s02*R10 + s12*R11 + s22*R12;
    const S M22 = s02*R20 + s12*R21 + s22*R22;
    f.Sc00 = R00*M00 + R01*M10 + R02*M20;
    f.Sc01 = R00*M01 + R01*M11 + R02*M21;
    f.Sc02 = R00*M02 + R01*M12 + R02*M22;
    f.Sc11 = R10*M01 + R11*M11 + R12*M21;
    f.Sc12 = R10*M02 + R11*M12 + R12*M22;
    f.Sc22 = R20*M02 + R21*M12 + R22*M22;
    return true;
}

// Projected covariance J Sigma_c J^T of a frame (project()'s c00..c22).
template <typename S>
__device__ __forceinline__ void projection_cov(const ProjectionFrame<S>& f, S* cov) {
    const S N00 = f.Sc00*f.J00 +                f.Sc02*f.J02;
    const S N01 = f.Sc01*f.J11 + f.Sc02*f.J12;
    const S N02 = f.Sc00*f.J20 + f.Sc01*f.J21 + f.Sc02*f.J22;
    const S N11 = f.Sc11*f.J11 + f.Sc12*f.J12;
    const S N12 = f.Sc01*f.J20 + f.Sc11*f.J21 + f.Sc12*f.J22;
    const S N20 = f.Sc02*f.J00 +                f.Sc22*f.J02;
    const S N21 = f.Sc12*f.J11 + f.Sc22*f.J12;
    const S N22 = f.Sc02*f.J20 + f.Sc12*f.J21 + f.Sc22*f.J22;
    cov[0] = f.J00*N00 + f.J02*N20;
    cov[1] = f.J00*N01 + f.J02*N21;
    cov[2] = f.J00*N02 + f.J02*N22;
    cov[3] = f.J11*N11 + f.J12*N21;
    cov[4] = f.J11*N12 + f.J12*N22;
    cov[5] = f.J20*N02 + f.J21*N12 + f.J22*N22;
}

// VJP of the projection of one pair from its frame, with respect to the world
// mean and the packed world covariance (WorldToImageProjectionBwd.cu:97-545):
// vm2 is the adjoint of the projected centre, vcov that of the packed
// projected covariance.
template <typename S>
__device__ __forceinline__ void projection_vjp(const Camera<S>& cam, const ProjectionFrame<S>& f, S vm2_x, S vm2_y,
                                               const S* vcov, S* v_p, S* v_s) {
    const S R00 = cam.R00, R01 = cam.R01, R02 = cam.R02;
    const S R10 = cam.R10, R11 = cam.R11, R12 = cam.R12;
    const S R20 = cam.R20, R21 = cam.R21, R22 = cam.R22;
    const S fx = cam.fx, fy = cam.fy;
    const S x = f.x, y = f.y, z = f.z, rz = f.rz, rz2 = f.rz2, tx = f.tx, ty = f.ty, rl = f.rl;
    const S rz3 = rz2 * rz;
    const S rl2 = rl * rl;
    const S J00 = f.J00, J02 = f.J02, J11 = f.J11, J12 = f.J12, J20 = f.J20, J21 = f.J21, J22 = f.J22;
    const S Sc00 = f.Sc00, Sc01 = f.Sc01, Sc02 = f.Sc02, Sc11 = f.Sc11, Sc12 = f.Sc12, Sc22 = f.Sc22;
    const bool x_clipped = f.x_clipped, y_clipped = f.y_clipped;

    const S va = vcov[0], vb = vcov[1], vc_ = vcov[2], vd = vcov[3], ve = vcov[4], vf = vcov[5];

    // Means: through the perspective division.
    S v_pc_x = fx * rz * vm2_x;
    S v_pc_y = fy * rz * vm2_y;
    S v_pc_z = -(fx * x * rz2 * vm2_x + fy * y * rz2 * vm2_y);
    // Covariance: v_Sigma_c = J^T G_upper J with the packed (upper-triangular)
    // adjoint, then v_Sigma = R^T v_Sigma_c R; off-diagonal packed entries
    // collect both symmetric positions.
    const S T00 = va*J00 + vc_*J20;
    const S T01 = vb*J11 + vc_*J21;
    const S T02 = va*J02 + vb*J12 + vc_*J22;
    const S T10 = ve*J20;
    const S T11 = vd*J11 + ve*J21;
    const S T12 = vd*J12 + ve*J22;
    const S T20 = vf*J20;
    const S T21 = vf*J21;
    const S T22 = vf*J22;
    const S vSc00 = J00*T00 + J20*T20;
    const S vSc01 = J00*T01 + J20*T21;
    const S vSc02 = J00*T02 + J20*T22;
    const S vSc10 = J11*T10 + J21*T20;
    const S vSc11 = J11*T11 + J21*T21;
    const S vSc12 = J11*T12 + J21*T22;
    const S vSc20 = J02*T00 + J12*T10 + J22*T20;
    const S vSc21 = J02*T01 + J12*T11 + J22*T21;
    const S vSc22 = J02*T02 + J12*T12 + J22*T22;
    const S Q00 = vSc00*R00 + vSc01*R10 + vSc02*R20;
    const S Q01 = vSc00*R01 + vSc01*R11 + vSc02*R21;
    const S Q02 = vSc00*R02 + vSc01*R12 + vSc02*R22;
    const S Q10 = vSc10*R00 + vSc11*R10 + vSc12*R20;
    const S Q11 = vSc10*R01 + vSc11*R11 + vSc12*R21;
    const S Q12 = vSc10*R02 + vSc11*R12 + vSc12*R22;
    const S Q20 = vSc20*R00 + vSc21*R10 + vSc22*R20;
    const S Q21 = vSc20*R01 + vSc21*R11 + vSc22*R21;
    const S Q22 = vSc20*R02 + vSc21*R12 + vSc22*R22;
    const S vS00 = R00*Q00 + R10*Q10 + R20*Q20;
    const S vS01 = R00*Q01 + R10*Q11 + R20*Q21;
    const S vS02 = R00*Q02 + R10*Q12 + R20*Q22;
    const S vS10 = R01*Q00 + R11*Q10 + R21*Q20;
    const S vS11 = R01*Q01 + R11*Q11 + R21*Q21;
    const S vS12 = R01*Q02 + R11*Q12 + R21*Q22;
    const S vS20 = R02*Q00 + R12*Q10 + R22*Q20;
    const S vS21 = R02*Q01 + R12*Q11 + R22*Q21;
    const S vS22 = R02*Q02 + R12*Q12 + R22*Q22;
    v_s[0] = vS00;
    v_s[1] = vS01 + vS10;
    v_s[2] = vS02 + vS20;
    v_s[3] = vS11;
    v_s[4] = vS12 + vS21;
    v_s[5] = vS22;

    // Jacobian path: v_J = (G + G^T) (J Sigma_c).
    const S GG00 = static_cast<S>(2) * va, GG01 = vb, GG02 = vc_;
    const S GG10 = vb, GG11 = static_cast<S>(2) * vd, GG12 = ve;
    const S GG20 = vc_, GG21 = ve, GG22 = static_cast<S>(2) * vf;
    const S U00 = J00*Sc00 + J02*Sc02;
    const S U01 = J00*Sc01 + J02*Sc12;
    const S U02 = J00*Sc02 + J02*Sc22;
    const S U10 = J11*Sc01 + J12*Sc02;
    const S U11 = J11*Sc11 + J12*Sc12;
    const S U12 = J11*Sc12 + J12*Sc22;
    const S U20 = J20*Sc00 + J21*Sc01 + J22*Sc02;
    const S U21 = J20*Sc01 + J21*Sc11 + J22*Sc12;
    const S U22 = J20*Sc02 + J21*Sc12 + J22*Sc22;
    const S vJ00 = GG00*U00 + GG01*U10 + GG02*U20;
    const S vJ02 = GG00*U02 + GG01*U12 + GG02*U22;
    const S vJ11 = GG10*U01 + GG11*U11 + GG12*U21;
    const S vJ12 = GG10*U02 + GG11*U12 + GG12*U22;
    const S vJ20 = GG20*U00 + GG21*U10 + GG22*U20;
    const S vJ21 = GG20*U01 + GG21*U11 + GG22*U21;
    const S vJ22 = GG20*U02 + GG21*U12 + GG22*U22;

    v_pc_z += -fx * rz2 * vJ00;
    v_pc_z += -fy * rz2 * vJ11;
    v_pc_z += rl * vJ22;
    if (!x_clipped) v_pc_x += -fx * rz2 * vJ02;
    v_pc_z += static_cast<S>(2) * fx * tx * rz3 * vJ02;
    if (!y_clipped) v_pc_y += -fy * rz2 * vJ12;
    v_pc_z += static_cast<S>(2) * fy * ty * rz3 * vJ12;
    if (!x_clipped) v_pc_x += rl * vJ20;
    if (!y_clipped) v_pc_y += rl * vJ21;
    const S v_l = -tx * rl2 * vJ20 - ty * rl2 * vJ21 - z * rl2 * vJ22;
    if (!x_clipped) v_pc_x += v_l * tx * rl;
    if (!y_clipped) v_pc_y += v_l * ty * rl;
    v_pc_z += v_l * z * rl;
    if (x_clipped) {
        v_pc_z += v_l * tx * rl * (tx / z);
        v_pc_z += (tx / z) * rl * vJ20;
    }
    if (y_clipped) {
        v_pc_z += v_l * ty * rl * (ty / z);
        v_pc_z += (ty / z) * rl * vJ21;
    }
    if (x_clipped) v_pc_z += -fx * (tx / z) * rz2 * vJ02;
    if (y_clipped) v_pc_z += -fy * (ty / z) * rz2 * vJ12;

    v_p[0] = R00 * v_pc_x + R10 * v_pc_y + R20 * v_pc_z;
    v_p[1] = R01 * v_pc_x + R11 * v_pc_y + R21 * v_pc_z;
    v_p[2] = R02 * v_pc_x + R12 * v_pc_y + R22 * v_pc_z;
}

// VJP of project() for one (camera, primitive) pair with respect to the
// world mean and packed world covariance (WorldToImageProjectionBwd.cu:97-545).
// Returns false when the pair is behind the camera (no contribution).
template <typename S>
__device__ __forceinline__ bool project_vjp(
    const Camera<S>& cam, S px, S py, S pz, const S* sig, uint32_t width, uint32_t height,
    S vm2_x, S vm2_y, const S* vcov, S* v_p, S* v_s
) {
    ProjectionFrame<S> f;
    if (!projection_frame(cam, camera_limits(cam, width, height), px, py, pz, sig, f)) return false;
    projection_vjp(cam, f, vm2_x, vm2_y, vcov, v_p, v_s);
    return true;
}

// --------------------------------------------------------------------------
// World -> volume mapping.
// --------------------------------------------------------------------------

// Scale-normalised Cholesky inverse of an SPD 3x3 matrix
// (CovarianceMath.cuh:10-66); false (zeros) for singular/indefinite input.
template <typename S>
__device__ __forceinline__ bool spd3_inverse(
    S a00, S a01, S a02, S a11, S a12, S a22, S* inv
) {
#pragma unroll
    for (int i = 0; i < 6; ++i) inv[i] = S(0);
    if (!isfinite(a00) || !isfinite(a01) || !isfinite(a02) ||
        !isfinite(a11) || !isfinite(a12) || !isfinite(a22) ||
        a00 <= S(0) || a11 <= S(0) || a22 <= S(0)) return false;
    const S scale = max(a00, max(a11, a22));
    a00 /= scale; a01 /= scale; a02 /= scale;
    a11 /= scale; a12 /= scale; a22 /= scale;
    const S l00 = sqrt(a00);
    const S l10 = a01 / l00;
    const S l20 = a02 / l00;
    const S pivot11 = a11 - l10 * l10;
    if (!(pivot11 > S(0))) return false;
    const S l11 = sqrt(pivot11);
    const S l21 = (a12 - l20 * l10) / l11;
    const S pivot22 = a22 - l20 * l20 - l21 * l21;
    if (!(pivot22 > S(0))) return false;
    const S l22 = sqrt(pivot22);
    const S k00 = S(1) / l00;
    const S k11 = S(1) / l11;
    const S k22 = S(1) / l22;
    const S k10 = -l10 * k00 * k11;
    const S k21 = -l21 * k11 * k22;
    const S k20 = -(l20 * k00 + l21 * k10) * k22;
    const S p00 = (k00 * k00 + k10 * k10 + k20 * k20) / scale;
    const S p01 = (k10 * k11 + k20 * k21) / scale;
    const S p02 = k20 * k22 / scale;
    const S p11 = (k11 * k11 + k21 * k21) / scale;
    const S p12 = k21 * k22 / scale;
    const S p22 = k22 * k22 / scale;
    if (!isfinite(p00) || !isfinite(p01) || !isfinite(p02) ||
        !isfinite(p11) || !isfinite(p12) || !isfinite(p22)) return false;
    inv[0] = p00; inv[1] = p01; inv[2] = p02; inv[3] = p11; inv[4] = p12; inv[5] = p22;
    return true;
}

template <typename S>
struct VolumeFrame {
    S r0, r1, r2, cx, cy, cz, D2, D1, D0;
};

template <typename S>
__device__ __forceinline__ VolumeFrame<S> load_frame(const S* ranges, const S* centers,
                                                     uint32_t dim2, uint32_t dim1, uint32_t dim0) {
    VolumeFrame<S> f;
    f.D2 = static_cast<S>(dim2);
    f.D1 = static_cast<S>(dim1);
    f.D0 = static_cast<S>(dim0);
    f.r0 = f.D2 / ranges[0];
    f.r1 = f.D1 / ranges[1];
    f.r2 = f.D0 / ranges[2];
    f.cx = centers[0]; f.cy = centers[1]; f.cz = centers[2];
    return f;
}

// Voxel-space centre, conic and radii for one primitive
// (WorldToVolumeMappingFwd.cu:86-156). Returns false when culled.
template <typename S>
__device__ __forceinline__ bool map_to_volume(
    const VolumeFrame<S>& f, S px, S py, S pz, const S* s, S eps3d, S radius_clip,
    S* mean_v, S* conic, int32_t* radii
) {
    const S r0 = f.r0, r1 = f.r1, r2 = f.r2;
    mean_v[0] = (px - f.cx) * r0 + f.D2 * static_cast<S>(0.5);
    mean_v[1] = (py - f.cy) * r1 + f.D1 * static_cast<S>(0.5);
    mean_v[2] = (pz - f.cz) * r2 + f.D0 * static_cast<S>(0.5);
    S Sv00 = r0 * r0 * s[0];
    S Sv01 = r0 * r1 * s[1];
    S Sv02 = r0 * r2 * s[2];
    S Sv11 = r1 * r1 * s[3];
    S Sv12 = r1 * r2 * s[4];
    S Sv22 = r2 * r2 * s[5];
    Sv00 += eps3d;
    Sv11 += eps3d;
    Sv22 += eps3d;
    radii[0] = radii[1] = radii[2] = 0;
    if (!spd3_inverse(Sv00, Sv01, Sv02, Sv11, Sv12, Sv22, conic)) return false;
    const S radius_x = ceil(radius_clip * sqrt(max(S(0), Sv00)));
    const S radius_y = ceil(radius_clip * sqrt(max(S(0), Sv11)));
    const S radius_z = ceil(radius_clip * sqrt(max(S(0), Sv22)));
    if (!isfinite(radius_x) || !isfinite(radius_y) || !isfinite(radius_z) ||
        radius_x <= S(0) || radius_y <= S(0) || radius_z <= S(0)) return false;
    radii[0] = static_cast<int32_t>(radius_x);
    radii[1] = static_cast<int32_t>(radius_y);
    radii[2] = static_cast<int32_t>(radius_z);
    return true;
}

// VJP of map_to_volume (WorldToVolumeMappingBwd.cu:76-166): the packed
// conic adjoint is upper-triangular; v_Sv = -P V_upper P.
template <typename S>
__device__ __forceinline__ void map_to_volume_vjp(
    const VolumeFrame<S>& f, const S* s, S eps3d, const S* v_mean_v, const S* vc, S* v_mean, S* v_cov
) {
    const S r0 = f.r0, r1 = f.r1, r2 = f.r2;
    v_mean[0] = v_mean_v[0] * r0;
    v_mean[1] = v_mean_v[1] * r1;
    v_mean[2] = v_mean_v[2] * r2;
    S Sv00 = r0 * r0 * s[0] + eps3d;
    S Sv01 = r0 * r1 * s[1];
    S Sv02 = r0 * r2 * s[2];
    S Sv11 = r1 * r1 * s[3] + eps3d;
    S Sv12 = r1 * r2 * s[4];
    S Sv22 = r2 * r2 * s[5] + eps3d;
    S P[6];
    if (!spd3_inverse(Sv00, Sv01, Sv02, Sv11, Sv12, Sv22, P)) {
#pragma unroll
        for (int i = 0; i < 6; ++i) v_cov[i] = S(0);
        return;
    }
    const S P00 = P[0], P01 = P[1], P02 = P[2], P11 = P[3], P12 = P[4], P22 = P[5];
    const S vc00 = vc[0], vc01 = vc[1], vc02 = vc[2], vc11 = vc[3], vc12 = vc[4], vc22 = vc[5];
    const S T00 = vc00*P00 + vc01*P01 + vc02*P02;
    const S T01 = vc00*P01 + vc01*P11 + vc02*P12;
    const S T02 = vc00*P02 + vc01*P12 + vc02*P22;
    const S T10 = vc11*P01 + vc12*P02;
    const S T11 = vc11*P11 + vc12*P12;
    const S T12 = vc11*P12 + vc12*P22;
    const S T20 = vc22*P02;
    const S T21 = vc22*P12;
    const S T22 = vc22*P22;
    const S vSv00 = -(P00*T00 + P01*T10 + P02*T20);
    const S vSv01 = -(P00*T01 + P01*T11 + P02*T21);
    const S vSv02 = -(P00*T02 + P01*T12 + P02*T22);
    const S vSv10 = -(P01*T00 + P11*T10 + P12*T20);
    const S vSv11 = -(P01*T01 + P11*T11 + P12*T21);
    const S vSv12 = -(P01*T02 + P11*T12 + P12*T22);
    const S vSv20 = -(P02*T00 + P12*T10 + P22*T20);
    const S vSv21 = -(P02*T01 + P12*T11 + P22*T21);
    const S vSv22 = -(P02*T02 + P12*T12 + P22*T22);
    v_cov[0] = vSv00 * r0 * r0;
    v_cov[1] = (vSv01 + vSv10) * r0 * r1;
    v_cov[2] = (vSv02 + vSv20) * r0 * r2;
    v_cov[3] = vSv11 * r1 * r1;
    v_cov[4] = (vSv12 + vSv21) * r1 * r2;
    v_cov[5] = vSv22 * r2 * r2;
}

// --------------------------------------------------------------------------
// Tile rectangles (IsectTilesKernel.cu:30-40, 79-103; IsectTiles3DKernel.cu:38-112)
// --------------------------------------------------------------------------

template <typename F>
__device__ __forceinline__ uint32_t clamp_tile(F value, uint32_t upper) {
    if (!isfinite(value) || value <= static_cast<F>(0)) return 0u;
    if (value >= static_cast<F>(upper)) return upper;
    return static_cast<uint32_t>(value);
}

// Half-open tile range [lo, hi) along one axis covered by a centre and an
// integer radius at a given tile size, computed in the input precision.
template <typename F>
__device__ __forceinline__ void tile_span(F mean, F radius, uint32_t tile_size, uint32_t n_tiles,
                                          uint32_t& lo, uint32_t& hi) {
    const F tile_size_f = static_cast<F>(tile_size);
    const F tile_radius = radius / tile_size_f;
    const F tile_centre = mean / tile_size_f;
    lo = clamp_tile(floor(tile_centre - tile_radius), n_tiles);
    hi = clamp_tile(ceil(tile_centre + tile_radius), n_tiles);
}

}  // namespace r2s
