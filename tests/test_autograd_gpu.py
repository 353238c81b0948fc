"""torch.autograd interface: finite differences, recompute, retain_graph, explicit parity.

The finite-difference checks use central differences (h = 1e-6) in float64 on
a 64-primitive, 2-view, 32x32 scene (and a 16^3 volume). Primitives are large
enough that every pixel (voxel) of the scene passes the contribution threshold
and every tile rectangle covers the whole image, so the loss is smooth in the
parameters and the differences are exact to rounding.
"""

import math

import pytest
import torch

import r2splat_b200 as r2s
from r2splat_b200 import autograd as ag
from r2splat_b200 import scenes

pytestmark = pytest.mark.gpu


def _large_scene(device, n=64, seed=3, beta=False, scale=0.3, radius=2.0, focal=120.0):
    g = torch.Generator(device="cpu").manual_seed(seed)
    means = (torch.rand(n, 3, generator=g, dtype=torch.float64) - 0.5) * 0.6
    quats = torch.randn(n, 4, generator=g, dtype=torch.float64)
    scales = scale * torch.exp(0.05 * torch.randn(n, 3, generator=g, dtype=torch.float64))
    densities = 1.0 + 0.5 * torch.rand(n, generator=g, dtype=torch.float64)
    viewmats, Ks = scenes.orbit_cameras(2, radius, focal, 32, 32, dtype=torch.float64)
    out = [t.to(device) for t in (means, quats, scales, densities, viewmats, Ks)]
    if beta:
        out.append((2.0 + torch.rand(n, generator=g, dtype=torch.float64)).to(device))
    return out


def _fd_check(loss_fn, params, picks, h=1e-6):
    grads = torch.autograd.grad(loss_fn(*params), params)
    worst = 0.0
    for p_index, rows in picks:
        p, g = params[p_index], grads[p_index]
        for row in rows:
            for col in range(p.shape[1] if p.dim() > 1 else 1):
                idx = (row, col) if p.dim() > 1 else (row,)
                with torch.no_grad():
                    base = p[idx].item()
                    p[idx] = base + h
                    up = loss_fn(*params).item()
                    p[idx] = base - h
                    down = loss_fn(*params).item()
                    p[idx] = base
                fd = (up - down) / (2 * h)
                scale = max(1.0, g.abs().max().item())
                worst = max(worst, abs(fd - g[idx].item()) / scale)
    return worst


def test_rasterize_matches_float64_finite_differences(device):
    means, quats, scales, densities, viewmats, Ks = _large_scene(device)
    weights = torch.randn(2, 32, 32, dtype=torch.float64, device=device,
                          generator=torch.Generator(device=device).manual_seed(5))
    params = [t.clone().requires_grad_() for t in (means, quats, scales, densities)]

    def loss(m, q, s, d):
        return (ag.rasterize(m, q, s, d, viewmats, Ks, (32, 32)) * weights).sum()

    worst = _fd_check(loss, params, [(0, [0, 17]), (1, [3, 40]), (2, [9, 63]), (3, [0, 5, 31])])
    assert worst < 1e-6, worst


def test_rasterize_beta_matches_float64_finite_differences(device):
    # Beta support is d2 < 1 (one projected sigma): primitives large enough to cover the image.
    means, quats, scales, densities, viewmats, Ks, beta = _large_scene(device, beta=True, scale=1.0, radius=4.0,
                                                                       focal=240.0)
    weights = torch.randn(2, 32, 32, dtype=torch.float64, device=device,
                          generator=torch.Generator(device=device).manual_seed(6))
    params = [t.clone().requires_grad_() for t in (means, quats, scales, densities, beta)]

    def loss(m, q, s, d, b):
        return (ag.rasterize(m, q, s, d, viewmats, Ks, (32, 32), beta=b) * weights).sum()

    worst = _fd_check(loss, params, [(0, [2]), (2, [11]), (3, [7]), (4, [1, 30])])
    assert worst < 1e-6, worst


def test_voxelize_matches_float64_finite_differences(device):
    means, quats, scales, densities, _, _ = _large_scene(device)
    scales = scales * 1.5
    weights = torch.randn(16, 16, 16, dtype=torch.float64, device=device,
                          generator=torch.Generator(device=device).manual_seed(7))
    params = [t.clone().requires_grad_() for t in (means, quats, scales, densities)]

    def loss(m, q, s, d):
        return (ag.voxelize(m, q, s, d, (16, 16, 16), volume_extent=(1.0, 1.0, 1.0)) * weights).sum()

    worst = _fd_check(loss, params, [(0, [1, 50]), (1, [8]), (2, [22]), (3, [4, 44])])
    assert worst < 1e-6, worst


def _ct_like(device):
    sc = scenes.small_scene(dtype=torch.float32).to(device)
    return sc


@pytest.mark.parametrize("operation", ["rasterize", "voxelize"])
def test_autograd_equals_explicit_and_recompute(device, operation):
    sc = _ct_like(device)
    means, quats, scales, densities = sc.primitives

    def run(recompute):
        params = [t.clone().requires_grad_() for t in (means, quats, scales, densities)]
        if operation == "rasterize":
            out = ag.rasterize(*params, sc.viewmats, sc.Ks, sc.image_size, recompute=recompute)
        else:
            out = ag.voxelize(*params, sc.volume_shape, volume_extent=sc.volume_extent, recompute=recompute)
        w = torch.randn(out.shape, device=device, generator=torch.Generator(device=device).manual_seed(11))
        (out * w).sum().backward()
        return [p.grad for p in params], w

    kept, w = run(False)
    recomputed, _ = run(True)
    if operation == "rasterize":
        _, ctx = r2s.rasterize_fwd(means, quats, scales, densities, sc.viewmats, sc.Ks, sc.image_size)
        ref = r2s.rasterize_bwd(ctx, w)
    else:
        _, ctx = r2s.voxelize_fwd(means, quats, scales, densities, sc.volume_shape, volume_extent=sc.volume_extent)
        ref = r2s.voxelize_bwd(ctx, w)
    for a, b, c in zip(kept, recomputed, (ref.means, ref.quats, ref.scales, ref.densities)):
        scale = c.abs().max().item() + 1e-12
        assert (a - c).abs().max().item() <= 1e-5 * scale
        assert (b - c).abs().max().item() <= 1e-5 * scale


def test_retain_graph_second_backward_recomputes(device):
    sc = _ct_like(device)
    params = [t.clone().requires_grad_() for t in sc.primitives]
    image = ag.rasterize(*params, sc.viewmats, sc.Ks, sc.image_size)
    loss = image.square().sum()
    first = torch.autograd.grad(loss, params, retain_graph=True)
    second = torch.autograd.grad(loss, params)
    for a, b in zip(first, second):
        assert torch.allclose(a, b, rtol=1e-6, atol=1e-9)


def test_variance_outputs_are_differentiable(device):
    sc = scenes.small_scene(dtype=torch.float64).to(device)
    n = sc.means.shape[0]
    unc = torch.full((n,), 0.05, dtype=torch.float64, device=device)
    params = [t.clone().requires_grad_() for t in (*sc.primitives, unc)]
    image, variance = ag.rasterize(*params[:4], sc.viewmats, sc.Ks, sc.image_size, uncertainty=params[4])
    (image.sum() + 3.0 * variance.sum()).backward()
    _, ctx = r2s.rasterize_fwd(*sc.primitives, sc.viewmats, sc.Ks, sc.image_size, uncertainty=unc)
    ref = r2s.rasterize_bwd(ctx, torch.ones_like(image), torch.full_like(variance, 3.0))
    assert torch.allclose(params[4].grad, ref.uncertainty, rtol=1e-9, atol=1e-12)
    assert torch.allclose(params[0].grad, ref.means, rtol=1e-9, atol=1e-12)
    assert math.isfinite(params[3].grad.sum().item())
