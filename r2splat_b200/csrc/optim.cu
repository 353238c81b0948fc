// Fused parameter update for fit loops: activation chain + Adam in one pass.
//
// The reference leaves this to the caller (its example fit loop,
// examples/optimize.py: raw parameters means, quats, log-scales, pre-softplus
// densities and log-beta; physical VJPs of the image and volume passes summed,
// multiplied by the activation derivatives, then torch.optim.Adam). Here one
// thread per primitive does all of it: sums the two VJPs, applies the
// activation derivatives (exp for scales and beta, sigmoid for densities), runs
// the Adam update (no weight decay, no amsgrad), and writes the activated
// physical parameters for the next step.
//
// The update follows the operations torch.optim.Adam issues per element:
// m.lerp_(g, 1 - beta1), i.e. m + (1 - beta1) (g - m) for a weight below 1/2;
// v.mul_(beta2).addcmul_(g, g, 1 - beta2); the bias corrections, step size and
// sqrt of the second correction in double precision on the host side of torch
// (here in double in the kernel), then rounded to the parameter type;
// denom = sqrt(v) / sqrt(bias2) + eps; p.addcdiv_(m, denom, -step_size).
// Division and square root are the correctly rounded ones, as in torch's
// kernels, although this library otherwise builds with fast math. The
// activation derivatives (exp, sigmoid) use the fast-math functions, so the
// result agrees with torch to rounding, not bit for bit.
// The step counter lives on the device so the update can be captured in a
// CUDA graph; a nonzero skip flag (an intersection-capacity overflow of this
// step) turns the whole update, counter included, into a no-op.
#include "common.cuh"

namespace r2s {

template <typename S>
struct AdamParams {
    S* means;          // [N,3] raw = physical
    S* quats;          // [N,4] raw = physical (normalised inside the projection)
    S* raw_scales;     // [N,3] log of scales
    S* raw_densities;  // [N]   softplus^-1 of densities
    S* raw_beta;       // [N]   log of beta, or null
    S* scales;         // [N,3] exp(raw_scales), written
    S* densities;      // [N]   softplus(raw_densities), written
    S* beta;           // [N]   exp(raw_beta), written (null without beta)
    S* m;              // [N,12] first moments
    S* v;              // [N,12] second moments
    const S* g1[5];    // first VJP: means, quats, scales, densities, beta (beta may be null)
    const S* g2[5];    // second VJP, or all null
};

template <typename S>
__device__ __forceinline__ S softplus(S x) {
    // torch.nn.functional.softplus with beta = 1, threshold = 20.
    return x > S(20) ? x : log1p(exp(x));
}

template <typename S>
__device__ __forceinline__ S sigmoid(S x) {
    return S(1) / (S(1) + exp(-x));
}

template <typename S>
__device__ __forceinline__ S div_rn(S a, S b) {
    if constexpr (sizeof(S) == 4) {
        return __fdiv_rn(a, b);
    } else {
        return __ddiv_rn(a, b);
    }
}

template <typename S>
__device__ __forceinline__ S sqrt_rn(S a) {
    if constexpr (sizeof(S) == 4) {
        return __fsqrt_rn(a);
    } else {
        return __dsqrt_rn(a);
    }
}

template <typename S>
__global__ void adam_kernel(AdamParams<S> p, uint32_t N, double lr, double beta1, double beta2, double eps,
                            const int32_t* __restrict__ step, const uint32_t* __restrict__ skip) {
    const uint32_t n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= N) return;
    if (skip != nullptr && *skip != 0u) return;
    const double t = static_cast<double>(*step + 1);
    const S step_size = static_cast<S>(lr / (1.0 - pow(beta1, t)));
    const S bias2_sqrt = static_cast<S>(sqrt(1.0 - pow(beta2, t)));
    const S w1 = static_cast<S>(1.0 - beta1);
    const S w2 = static_cast<S>(1.0 - beta2);
    const S b2 = static_cast<S>(beta2);
    const S e = static_cast<S>(eps);
    const bool has_beta = p.raw_beta != nullptr;

    S* raw[12];
    S grad[12];
    int k = 0;
    auto g_sum = [&](int slot, size_t idx) {
        S g = p.g1[slot] != nullptr ? p.g1[slot][idx] : S(0);
        if (p.g2[slot] != nullptr) g += p.g2[slot][idx];
        return g;
    };
    for (int c = 0; c < 3; ++c, ++k) {
        raw[k] = p.means + 3 * size_t(n) + c;
        grad[k] = g_sum(0, 3 * size_t(n) + c);
    }
    for (int c = 0; c < 4; ++c, ++k) {
        raw[k] = p.quats + 4 * size_t(n) + c;
        grad[k] = g_sum(1, 4 * size_t(n) + c);
    }
    for (int c = 0; c < 3; ++c, ++k) {
        raw[k] = p.raw_scales + 3 * size_t(n) + c;
        grad[k] = g_sum(2, 3 * size_t(n) + c) * p.scales[3 * size_t(n) + c];
    }
    raw[k] = p.raw_densities + n;
    grad[k] = g_sum(3, n) * sigmoid(p.raw_densities[n]);
    ++k;
    if (has_beta) {
        raw[k] = p.raw_beta + n;
        grad[k] = g_sum(4, n) * p.beta[n];
        ++k;
    }
    for (int i = 0; i < k; ++i) {
        const size_t mi = 12 * size_t(n) + i;
        const S g = grad[i];
        const S m_old = p.m[mi];
        const S m = fma(w1, g - m_old, m_old);
        const S v = fma(w2 * g, g, p.v[mi] * b2);
        p.m[mi] = m;
        p.v[mi] = v;
        const S denom = div_rn(sqrt_rn(v), bias2_sqrt) + e;
        *raw[i] = fma(-step_size, div_rn(m, denom), *raw[i]);
    }
    for (int c = 0; c < 3; ++c) p.scales[3 * size_t(n) + c] = exp(p.raw_scales[3 * size_t(n) + c]);
    p.densities[n] = softplus(p.raw_densities[n]);
    if (has_beta) p.beta[n] = exp(p.raw_beta[n]);
}

__global__ void step_increment_kernel(int32_t* __restrict__ step, const uint32_t* __restrict__ skip) {
    if (skip == nullptr || *skip == 0u) *step += 1;
}

}  // namespace r2s

using namespace r2s;

extern "C" {

int r2s_adam_activation_step(int dtype, uint32_t N, void* means, void* quats, void* raw_scales, void* raw_densities,
                             void* raw_beta, void* scales, void* densities, void* beta, void* adam_m, void* adam_v,
                             const void* const* grads_a, const void* const* grads_b, double lr, double beta1,
                             double beta2, double eps, int32_t* step, const uint32_t* skip, void* stream) {
    R2S_REQUIRE(step != nullptr && grads_a != nullptr, R2S_ERR_ARGUMENT, "step and grads_a must be non-null");
    R2S_REQUIRE((raw_beta == nullptr) == (beta == nullptr), R2S_ERR_ARGUMENT, "raw_beta goes with beta");
    cudaStream_t st = as_stream(stream);
    if (N > 0) {
        R2S_DISPATCH(dtype, {
            AdamParams<S> p{};
            p.means = static_cast<S*>(means);
            p.quats = static_cast<S*>(quats);
            p.raw_scales = static_cast<S*>(raw_scales);
            p.raw_densities = static_cast<S*>(raw_densities);
            p.raw_beta = static_cast<S*>(raw_beta);
            p.scales = static_cast<S*>(scales);
            p.densities = static_cast<S*>(densities);
            p.beta = static_cast<S*>(beta);
            p.m = static_cast<S*>(adam_m);
            p.v = static_cast<S*>(adam_v);
            for (int i = 0; i < 5; ++i) {
                p.g1[i] = static_cast<const S*>(grads_a[i]);
                p.g2[i] = grads_b != nullptr ? static_cast<const S*>(grads_b[i]) : nullptr;
            }
            adam_kernel<S><<<blocks_for(N, 256), 256, 0, st>>>(p, N, lr, beta1, beta2, eps, step, skip);
        });
        R2S_TRY(check_launch("adam_activation_step"));
    }
    step_increment_kernel<<<1, 1, 0, st>>>(step, skip);
    return check_launch("adam_step_increment");
}

}  // extern "C"
