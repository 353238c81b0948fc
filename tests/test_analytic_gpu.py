"""Closed-form cases of the explicit operators on the GPU.

Primitives on a camera's optical axis, or at a voxel centre, have outputs and gradients with exact
expressions, which pin the CUDA path (and the float64 oracle behind the other tests) independently
of any implementation:

* An axis-aligned primitive on the optical axis at depth z projects to an axis-aligned profile with
  standard deviations (fx s_x / z, fy s_y / z) around the principal point. Its path factor, the
  line integral along the ray, is sqrt(2 pi) s_z for a Gaussian and s_z Gamma(1/2) Gamma(beta + 1) /
  Gamma(beta + 3/2) for a Beta primitive, whose image profile is (1 - d^2)^(beta + 1/2).
* At the principal point the profile is 1, so a one-pixel image holds o times the path factor:
  sqrt(2 pi (s^2 + eps)) for an isotropic Gaussian of scale s whose covariance gets eps.
* At a voxel centre a primitive contributes its density.

Expected gradients are those of the same expressions, by autograd in float64 on the host. These
are the analytic cases the reference's own tests hold for this path (tests/test_functional.py,
tests/test_beta_api.py, tests/test_conics_numeric.py), restated.
"""

import math

import pytest
import torch

import r2splat_b200 as r2s
from r2splat_b200.cuda import _wrapper as low

pytestmark = pytest.mark.gpu


def _log_beta_path(beta):
    """log of Gamma(1/2) Gamma(beta + 1) / Gamma(beta + 3/2)."""
    return math.lgamma(0.5) + torch.lgamma(beta + 1) - torch.lgamma(beta + 1.5)


@pytest.mark.parametrize("use_beta", [False, True])
def test_on_axis_projection_matches_its_closed_form(device, use_beta):
    dtype = torch.float64
    scales = torch.tensor([[0.4, 0.3, 0.25]], dtype=dtype)
    density = torch.tensor([0.8], dtype=dtype)
    beta = torch.tensor([3.5], dtype=dtype) if use_beta else None
    q = torch.tensor([0.2], dtype=dtype)
    means = torch.tensor([[0.0, 0.0, 2.0]], dtype=dtype, device=device)
    quats = torch.tensor([[1.0, 0.0, 0.0, 0.0]], dtype=dtype, device=device)
    viewmats = torch.eye(4, dtype=dtype, device=device)[None]
    # fx / z = 6 and fy / z = 5 at z = 2; principal point at the centre of a 9 x 7 image.
    Ks = torch.tensor([[[12.0, 0.0, 4.5], [0.0, 10.0, 3.5], [0.0, 0.0, 1.0]]], dtype=dtype, device=device)
    (image, variance), ctx = r2s.rasterize_fwd(
        means, quats, scales.to(device), density.to(device), viewmats, Ks, (7, 9),
        beta=None if beta is None else beta.to(device), uncertainty=q.to(device), eps=0.0, radius_clip=8.0)

    leaves = [scales.clone().requires_grad_(True), density.clone().requires_grad_(True)]
    if use_beta:
        leaves.append(beta.clone().requires_grad_(True))
    leaves.append(q.clone().requires_grad_(True))
    s, o = leaves[0][0], leaves[1][0]
    yy, xx = torch.meshgrid(torch.arange(7, dtype=dtype) + 0.5, torch.arange(9, dtype=dtype) + 0.5, indexing="ij")
    d2 = ((xx - 4.5) / (6 * s[0])) ** 2 + ((yy - 3.5) / (5 * s[1])) ** 2
    if use_beta:
        b = leaves[2][0]
        expected = o * s[2] * torch.exp(_log_beta_path(b)) * (1 - d2).clamp_min(0) ** (b + 0.5)
    else:
        expected = o * math.sqrt(2 * math.pi) * s[2] * torch.exp(-d2 / 2)
    # The rasterizer's contribution threshold.
    expected = torch.where(expected.abs() >= 1e-5, expected, torch.zeros_like(expected))[None]
    expected_var = leaves[-1][0] * expected ** 2
    assert image.shape == (1, 7, 9)
    torch.testing.assert_close(image.cpu(), expected.detach(), atol=1e-12, rtol=1e-10)
    torch.testing.assert_close(variance.cpu(), expected_var.detach(), atol=1e-12, rtol=1e-10)

    grads = r2s.rasterize_bwd(ctx, torch.ones_like(image), torch.ones_like(variance))
    want = torch.autograd.grad((expected + expected_var).sum(), leaves)
    names = ["scales", "densities"] + (["beta"] if use_beta else []) + ["uncertainty"]
    for name, w in zip(names, want):
        torch.testing.assert_close(getattr(grads, name).cpu(), w, atol=1e-10, rtol=1e-9, msg=name)


@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
@pytest.mark.parametrize("scale", [0.01, 1e-3, 1e-12])
@pytest.mark.parametrize("eps", [0.0, 1e-4])
def test_path_factor_and_its_scale_gradient_at_the_principal_point(device, dtype, scale, eps):
    means = torch.tensor([[0.0, 0.0, 2.0]], dtype=dtype, device=device)
    quats = means.new_tensor([[1.0, 0.0, 0.0, 0.0]])
    scales = means.new_full((1, 3), scale)
    density = means.new_ones(1)
    viewmats = torch.eye(4, dtype=dtype, device=device)[None]
    Ks = means.new_tensor([[[2.0, 0.0, 0.5], [0.0, 2.0, 0.5], [0.0, 0.0, 1.0]]])
    expected = math.sqrt(2 * math.pi * (scale ** 2 + eps))
    expected_grad = math.sqrt(2 * math.pi) * scale / math.sqrt(scale ** 2 + eps)
    if expected >= 1e-5:
        image, ctx = r2s.rasterize_fwd(means, quats, scales, density, viewmats, Ks, (1, 1), eps=eps)
        value = image.squeeze()
        grad = r2s.rasterize_bwd(ctx, torch.ones_like(image)).scales[0, 2]
    else:
        # Below the rasterizer's contribution threshold: the path factor through the low-level
        # conic / path-factor operator and its VJP, d mu / d s_z = 2 s_z d mu / d cov_zz.
        cov = means.new_tensor([[[scale ** 2, 0.0, 0.0, scale ** 2, 0.0, scale ** 2]]])
        conics, mu = low.conics_mu_fwd(cov, eps)
        v_cov = low.conics_mu_bwd(cov, eps, conics, mu, torch.zeros_like(conics), torch.ones_like(mu))
        value = mu.squeeze()
        grad = 2 * scale * v_cov[..., 5].squeeze()
    tol = 3e-5 if dtype == torch.float32 else 1e-10
    torch.testing.assert_close(value.cpu(), torch.tensor(expected, dtype=dtype), atol=0, rtol=tol)
    torch.testing.assert_close(grad.cpu(), torch.tensor(expected_grad, dtype=dtype), atol=0, rtol=tol)


def _two_on_axis_primitives(device, dtype):
    means = torch.tensor([[0.0, 0.0, 2.0], [0.0, 0.0, 2.0]], dtype=dtype, device=device)
    quats = means.new_tensor([[2.0, 0.0, 0.0, 0.0], [3.0, 0.0, 0.0, 0.0]])  # unnormalised identities
    scales = means.new_tensor([[0.2, 0.3, 0.4], [0.3, 0.4, 0.5]])
    densities = means.new_tensor([1.2, 0.8])
    return means, quats, scales, densities


@pytest.mark.parametrize("operation", ["rasterize", "voxelize"])
@pytest.mark.parametrize("with_uncertainty", [False, True])
@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
def test_beta_and_uncertainty_values_and_vjps_in_closed_form(device, operation, with_uncertainty, dtype):
    prims = _two_on_axis_primitives(device, dtype)
    beta = prims[0].new_tensor([3.5, 99.0, 1.25, 99.0])[::2]  # a strided view
    assert not beta.is_contiguous()
    q = prims[0].new_tensor([0.2, 0.3]) if with_uncertainty else None
    if operation == "rasterize":
        # Two identical cameras at the origin, a one-pixel image at the principal point.
        cameras = 2
        viewmats = torch.eye(4, dtype=dtype, device=device).repeat(2, 1, 1)
        Ks = prims[0].new_tensor([[[1.0, 0.0, 0.5], [0.0, 1.0, 0.5], [0.0, 0.0, 1.0]]]).repeat(2, 1, 1)
        out, ctx = r2s.rasterize_fwd(*prims, viewmats, Ks, (1, 1), beta=beta, uncertainty=q, eps=0.0)
        b64 = beta.double().cpu()
        path = (prims[2][:, 2].double().cpu() * torch.exp(_log_beta_path(b64))).to(dtype)
        dlog_path = (torch.special.digamma(b64 + 1) - torch.special.digamma(b64 + 1.5)).to(dtype)
        backward = r2s.rasterize_bwd
    else:
        # One voxel whose centre is the primitives' centre: each contributes its density.
        cameras = 1
        out, ctx = r2s.voxelize_fwd(*prims, (1, 1, 1), volume_extent=(1, 1, 1), volume_center=(0, 0, 2),
                                    beta=beta, uncertainty=q, eps=0.0)
        path = torch.ones(2, dtype=dtype)
        dlog_path = torch.zeros(2, dtype=dtype)
        backward = r2s.voxelize_bwd
    mean, variance = out if with_uncertainty else (out, None)
    contribution = prims[3].cpu() * path
    torch.testing.assert_close(mean.cpu(), contribution.sum().expand_as(mean.cpu()))
    factor = torch.ones(2, dtype=dtype)
    if with_uncertainty:
        q_cpu = q.cpu()
        torch.testing.assert_close(variance.cpu(), (q_cpu * contribution ** 2).sum().expand_as(variance.cpu()))
        factor = factor + 0.8 * q_cpu * contribution  # d/dc of c + 0.4 q c^2
    grads = backward(ctx, torch.ones_like(mean), torch.full_like(variance, 0.4) if with_uncertainty else None)
    torch.testing.assert_close(grads.densities.cpu(), cameras * factor * path)
    torch.testing.assert_close(grads.beta.cpu(), cameras * factor * contribution * dlog_path)
    if with_uncertainty:
        torch.testing.assert_close(grads.uncertainty.cpu(), cameras * 0.4 * contribution ** 2)
    else:
        assert grads.uncertainty is None
