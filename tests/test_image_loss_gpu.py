"""Forward with the image loss fused into the tile kernel's epilogue.

``explicit.rasterize_fwd_with_loss`` must give:
* the image of ``rasterize_fwd``, bit for bit;
* the MSE gradient bit-identical to torch's ``(image - target).mul_(2 w / numel)``;
* the L1 gradient bit-identical to the low-level ``image_loss_l1_bwd`` (the
  reference's formula, ImageLossBwd.cu:14-30) with an upstream gradient of one;
* the loss within 1e-12 (MSE, fp64 sum of exact squares) or 1e-6 (L1, two fp64
  sums in different orders, each rounded once to fp32) of a float64 reduction;
* a context that ``rasterize_bwd`` consumes like the plain forward's.
"""

import pytest
import torch

import r2splat_b200 as r2s
from r2splat_b200 import explicit, scenes
from r2splat_b200.cuda import _wrapper as low

pytestmark = pytest.mark.gpu


def _scene(device, n=2000, cams=4, h=64, w=64, beta=False, unc=False, dtype=torch.float32, seed=0):
    means, quats, scales, densities, b, q = scenes.random_primitives(
        n, seed, 0.03, 0.3, beta_range=(0.5, 4.0) if beta else None, uncertainty_max=0.1 if unc else None,
        dtype=dtype)
    viewmats, Ks = scenes.orbit_cameras(cams, 2.0, 100.0 * w / 64, w, h, dtype=dtype)
    prim = [t.to(device) for t in (means, quats, scales, densities)]
    extra = {"beta": None if b is None else b.to(device), "uncertainty": None if q is None else q.to(device)}
    gen = torch.Generator(device="cpu").manual_seed(seed + 7)
    target = (0.05 * torch.rand((cams, h, w), generator=gen, dtype=dtype)).to(device)
    return prim, viewmats.to(device), Ks.to(device), (h, w), extra, target


def _image(out):
    return out[0] if isinstance(out, tuple) else out


@pytest.mark.parametrize("beta,unc", [(False, False), (True, False), (False, True), (True, True)])
@pytest.mark.parametrize("size", [(64, 64), (37, 50)])
def test_mse_epilogue_matches_separate_passes(device, beta, unc, size):
    prim, vm, Ks, hw, extra, target = _scene(device, h=size[0], w=size[1], beta=beta, unc=unc)
    plain, ctx_plain = r2s.rasterize_fwd(*prim, vm, Ks, hw, **extra)
    out, ctx, v, loss, value = explicit.rasterize_fwd_with_loss(*prim, vm, Ks, hw, target, **extra)
    assert torch.equal(_image(out), _image(plain))
    if unc:
        assert torch.equal(out[1], plain[1])
    image = _image(plain)
    expected_v = (image - target).mul_(2.0 / image.numel())
    assert torch.equal(v, expected_v)
    ref = ((image.double() - target.double()) ** 2).mean().item()
    assert abs(value.item() - ref) <= 1e-6 * ref  # fp32 rounding of an fp64 mean
    assert loss.item() == value.item()
    g_plain = r2s.rasterize_bwd(ctx_plain, expected_v)
    g = r2s.rasterize_bwd(ctx, v)
    for name in ("means", "quats", "scales", "densities", "beta", "uncertainty"):
        a, b = getattr(g, name), getattr(g_plain, name)
        assert (a is None) == (b is None)
        if a is not None:
            assert torch.equal(a, b), name


def test_mse_loss_in_float64(device):
    prim, vm, Ks, hw, extra, target = _scene(device, dtype=torch.float64, n=500)
    out, _, v, loss, value = explicit.rasterize_fwd_with_loss(*prim, vm, Ks, hw, target, loss_weight=0.25)
    plain, _ = r2s.rasterize_fwd(*prim, vm, Ks, hw)
    assert torch.equal(out, plain)
    assert torch.equal(v, (plain - target).mul_(2.0 * 0.25 / plain.numel()))
    ref = ((plain - target) ** 2).mean().item()
    assert abs(value.item() - ref) <= 1e-12 * ref
    assert abs(loss.item() - 0.25 * ref) <= 1e-12 * ref


@pytest.mark.parametrize("weight", [1.0, 0.7])
def test_l1_epilogue_matches_low_level_l1(device, weight):
    prim, vm, Ks, hw, extra, target = _scene(device, beta=True)
    out, _, v, loss, value = explicit.rasterize_fwd_with_loss(*prim, vm, Ks, hw, target, loss="l1",
                                                              loss_weight=weight, **extra)
    plain, _ = r2s.rasterize_fwd(*prim, vm, Ks, hw, **extra)
    assert torch.equal(out, plain)
    ones = torch.ones(1, device=device)
    assert torch.equal(v, low.image_loss_l1_bwd(plain, target, ones, weight))
    ref_loss, ref_value, _ = low.image_loss_l1_fwd(plain, target, weight)
    assert abs(value.item() - ref_value.item()) <= 1e-6 * ref_value.item()
    assert abs(loss.item() - ref_loss.item()) <= 1e-6 * abs(ref_loss.item())
    exact = (plain.double() - target.double()).abs().mean().item()
    assert abs(value.item() - exact) <= 1e-6 * exact


def test_no_primitives_gives_loss_of_a_zero_image(device):
    prim, vm, Ks, hw, extra, target = _scene(device)
    empty = [t[:0] for t in prim]
    out, ctx, v, loss, value = explicit.rasterize_fwd_with_loss(*empty, vm, Ks, hw, target)
    assert not out.any()
    assert torch.equal(v, (out - target).mul_(2.0 / out.numel()))
    ref = (target.double() ** 2).mean().item()
    assert abs(value.item() - ref) <= 1e-6 * ref
    g = r2s.rasterize_bwd(ctx, v)
    assert g.means.shape == (0, 3)


def test_rejects_bad_loss_arguments(device):
    prim, vm, Ks, hw, extra, target = _scene(device, n=100)
    with pytest.raises(ValueError, match="loss must be"):
        explicit.rasterize_fwd_with_loss(*prim, vm, Ks, hw, target, loss="l2")
    with pytest.raises(ValueError, match="target must have shape"):
        explicit.rasterize_fwd_with_loss(*prim, vm, Ks, hw, target[:, :-1])
    with pytest.raises(ValueError, match="same device and dtype"):
        explicit.rasterize_fwd_with_loss(*prim, vm, Ks, hw, target.double())
    bad = target.clone()
    bad[0, 0, 0] = float("nan")
    with pytest.raises(ValueError, match="finite"):
        explicit.rasterize_fwd_with_loss(*prim, vm, Ks, hw, bad)
    with pytest.raises(ValueError, match="loss_weight"):
        explicit.rasterize_fwd_with_loss(*prim, vm, Ks, hw, target, loss_weight=float("inf"))
